"""The Rust shim crate (rust-wl_b200/rust/vxl-phys-gpu-b200) against the C header, on CPU.

There is no Rust toolchain here, so the crate is checked as text against include/vxl_sph.h:
every function the header declares is declared in src/ffi.rs with the same number of
parameters (and nothing else is), and every #[repr(C)] struct lists the header struct's
fields in the same order with types of the same size. The library itself is loaded and
every declared symbol resolved, so the shim links against what the build produces.
"""
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
HEADER = (ROOT / "include" / "vxl_sph.h").read_text()
CRATE = ROOT / "rust-wl_b200" / "rust" / "vxl-phys-gpu-b200"
FFI = (CRATE / "src" / "ffi.rs").read_text()

C_SIZE = {"uint32_t": 4, "int32_t": 4, "float": 4, "uint64_t": 8, "double": 8, "int": 4}
R_SIZE = {"u32": 4, "i32": 4, "f32": 4, "u64": 8, "f64": 8}
STRUCTS = {"vxl_block_header": "BlockHeader", "vxl_sph_params": "Params", "vxl_sph_desc": "Desc",
           "vxl_sph_span": "Span", "vxl_sph_reaction": "Reaction", "vxl_sph_grid_info": "GridInfo",
           "vxl_sph_stats": "Stats", "vxl_sph_tuning": "Tuning", "vxl_sph_body_pose": "BodyPose",
           "vxl_sph_rigid_body": "RigidBody", "vxl_sph_wall_plane": "WallPlane", "vxl_sph_provider": "Provider",
           "vxl_sph_request_status": "RequestStatus", "vxl_sph_serve_report": "ServeReport"}


def _strip_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def header_functions():
    body = _strip_comments(HEADER)
    out = {}
    for m in re.finditer(r"\b(vxl_sph_\w+)\s*\(([^;{]*?)\)\s*;", body):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def rust_functions():
    block = FFI[FFI.index('extern "C"'):]
    out = {}
    for m in re.finditer(r"pub fn (vxl_sph_\w+)\(([^)]*)\)", block, flags=re.S):
        args = [a for a in m.group(2).split(",") if a.strip()]
        out[m.group(1)] = len(args)
    return out


def header_struct(name):
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), _strip_comments(HEADER), flags=re.S)
    fields = []
    for line in m.group(1).split(";"):
        line = line.strip()
        if not line:
            continue
        mm = re.match(r"(?:const\s+)?([\w]+)\s*(\*?)\s*(\w+)(?:\[(\d+)\])?", line)
        typ, ptr, fname, n = mm.groups()
        size = 8 if ptr else C_SIZE.get(typ)
        fields.append((fname, typ if not ptr else "ptr", size, int(n or 1)))
    return fields


def rust_struct(name):
    m = re.search(r"pub struct %s \{(.*?)\n\}" % name, FFI, flags=re.S)
    fields = []
    for mm in re.finditer(r"pub (\w+): ([^,\n]+),", m.group(1)):
        fname, typ = mm.group(1), mm.group(2).strip()
        arr = re.match(r"\[(\w+); (\d+)\]", typ)
        if arr:
            fields.append((fname, arr.group(1), R_SIZE[arr.group(1)], int(arr.group(2))))
        elif typ.startswith("*"):
            fields.append((fname, "ptr", 8, 1))
        else:
            fields.append((fname, typ, R_SIZE.get(typ), 1))
    return fields


def test_every_header_function_is_declared_with_its_arity():
    h, r = header_functions(), rust_functions()
    assert set(h) == set(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    bad = {k: (h[k], r[k]) for k in h if h[k] != r[k]}
    assert not bad, bad


def test_repr_c_structs_match_the_header():
    for cname, rname in STRUCTS.items():
        hf, rf = header_struct(cname), rust_struct(rname)
        assert [f[0] for f in hf] == [f[0] for f in rf], (cname, hf, rf)
        for (fn, ht, hs, hn), (_, rt, rs, rn) in zip(hf, rf):
            if ht in STRUCTS:  # nested struct: by name
                assert rt == STRUCTS[ht], (cname, fn, ht, rt)
            else:
                assert hn == rn and hs == rs, (cname, fn, ht, rt)


def test_crate_files_and_trait_impls_present():
    lib = (CRATE / "src" / "lib.rs").read_text()
    assert "impl FluidStepper for B200FluidStepper" in lib and "impl PhysGpuBackend for B200Backend" in lib
    for fn in ("fn step(", "fn reactions(", "fn bounds(", "fn gather_walls("):
        assert fn in lib, fn
    assert "vxl-phys-core" in (CRATE / "Cargo.toml").read_text()
    assert "rustc-link-lib=dylib=vxl_sph" in (CRATE / "build.rs").read_text()
    # every status returned by the library is checked (no call whose result is dropped)
    calls = re.findall(r"ffi::(vxl_sph_\w+)\(", lib)
    unchecked = [c for c in calls if c not in ("vxl_sph_last_error", "vxl_sph_destroy", "vxl_sph_abi_version",
                                               "vxl_sph_backend_available", "vxl_sph_bounds")]
    for c in unchecked:
        assert re.search(r"(must|check)\(unsafe \{\s*ffi::%s" % c, lib), c


def test_library_exports_every_declared_symbol():
    import ctypes
    import sys
    sys.path.insert(0, str(ROOT / "rust-wl_b200"))
    from vxl_sph import build
    lib = ctypes.CDLL(str(build.build()))
    for name in rust_functions():
        getattr(lib, name)
