"""The allocation-free neighbour-table build, vxl_sph_build_grid_static, on a B200.

Some callers of this library cannot allocate device memory while they run: an engine
that reserves one fixed arena for all GPU work at start-up and forbids any further
cudaMalloc, or a per-frame plugin that must not call cudaMalloc/cudaFree because both can
synchronise the device and stall its frame loop. vxl_sph_build_grid_static serves them:
the caller passes device buffers for positions, items and start, and the sort's working
memory is a fixed array inside the library.

The check: through the C ABI, the table it builds equals the table the handle-based
path builds for the same positions (vxl_sph_create + vxl_sph_substep +
vxl_sph_export_grid, which builds its table from the positions at the start of the
substep) and the oracle's restatement of the reference's UniformGrid::rebuild
(crates/vxl-phys-fluid/src/grid.rs:29-76). The tables are integer data, so the
tolerance is zero. Two calls in a row, on different scenes, show that the shared array's
leftover contents do not leak into the next call. Cells crowded with hundreds to
thousands of particles sort in bounded time. After the first (set-up) call on the
device, a call leaves the device's free memory unchanged. Sizes past the fixed limit are
refused.

The file name sorts last so that a run stopping at the first failure has run every
other test first; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 19


def _handle_table(vxl, spec, max_bins):
    """The existing path: scene handle, one substep, exported table of that substep."""
    p = spec.params
    p.max_bins = max_bins
    g = vxl.Scene(p, spec.pos, spec.vel, spec.pmass, spec.n_fluid)
    g.substep(float(np.float32(np.float32(1.0) / np.float32(60.0)) / np.float32(p.substeps)))
    items, start, _, info = g.export_grid()
    g.close()
    return items, start, info


def _static_table(vxl, torch, pos, h, max_bins):
    lib = vxl.load()
    n = pos.shape[0]
    d_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    d_items = torch.empty(n, dtype=torch.int32, device="cuda")
    d_start = torch.empty(max_bins + 1, dtype=torch.int32, device="cuda")
    info = vxl.GridInfo()
    info.hdr = vxl.header(vxl.GridInfo)
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.vxl_sph_build_grid_static(C.c_void_p(d_pos.data_ptr()), n, h, max_bins, C.c_void_p(d_items.data_ptr()),
                                       C.c_void_p(d_start.data_ptr()), max_bins + 1, C.byref(info),
                                       C.c_void_p(stream))
    assert st == vxl.OK, lib.vxl_sph_last_error()
    total = int(info.total)
    items = d_items.cpu().numpy().view(np.uint32)
    start = d_start[: total + 1].cpu().numpy().view(np.uint32)
    return items, start, info


def _same(a_info, b_info):
    return (list(a_info.dims) == list(b_info.dims) and a_info.total == b_info.total
            and np.float32(a_info.inv) == np.float32(b_info.inv) and np.float32(a_info.bin) == np.float32(b_info.bin)
            and list(np.float32(a_info.min[:])) == list(np.float32(b_info.min[:])))


def test_static_grid_matches_handle_path_two_calls(oracle_mod):
    torch = pytest.importorskip("torch")
    import vxl_sph as vxl
    from vxl_sph import build, scenes

    build.build()
    vxl.load()
    specs = [
        scenes.small_dam(n=(10, 12, 9), spacing=0.05, tank=(0.8, 0.7, 0.6)),  # 1,080 fluid + walls
        scenes.dam0(),                                                         # 16,384 fluid + 17,000 walls
    ]
    for call, spec in enumerate(specs):
        h = float(spec.params.smoothing_radius)
        items_h, start_h, info_h = _handle_table(vxl, spec, LIMIT)
        items_s, start_s, info_s = _static_table(vxl, torch, spec.pos, h, LIMIT)
        assert _same(info_s, info_h), f"call {call}: grid box differs"
        assert np.array_equal(start_s, start_h), f"call {call}: start differs"
        assert np.array_equal(items_s, items_h), f"call {call}: items differ"
        start_o, items_o, dims_o = oracle_mod.rebuild_grid(spec.pos, h, LIMIT)
        assert list(dims_o) == list(info_s.dims), f"call {call}: dims differ from the oracle"
        assert np.array_equal(start_s, start_o), f"call {call}: start differs from the oracle"
        assert np.array_equal(items_s, items_o), f"call {call}: items differ from the oracle"


def test_static_grid_crowded_cells_in_bounded_time(oracle_mod):
    """One cell of 300, 2,000 and 5,000 particles (the shared-memory rank and the index
    bitmap), then a cluster of a few crowded cells among sparse ones: each table equals
    the oracle's, and each call takes well under a second."""
    import time

    torch = pytest.importorskip("torch")
    import vxl_sph as vxl
    vxl.load()
    rng = np.random.default_rng(5)
    cases = [rng.uniform(0.0, 0.05, (n, 3)).astype(np.float32) for n in (300, 2000, 5000)]
    mixed = np.concatenate([rng.uniform(0.0, 0.04, (2500, 3)), rng.uniform(0.3, 0.34, (700, 3)),
                            rng.uniform(0.0, 2.0, (4000, 3))]).astype(np.float32)
    cases.append(rng.permutation(mixed))
    for k, pos in enumerate(cases):
        _static_table(vxl, torch, pos, 0.1, LIMIT)  # first call of the shape (kernel loading)
        t0 = time.perf_counter()
        items_s, start_s, info_s = _static_table(vxl, torch, pos, 0.1, LIMIT)
        dt = time.perf_counter() - t0
        start_o, items_o, dims_o = oracle_mod.rebuild_grid(pos, 0.1, LIMIT)
        assert list(dims_o) == list(info_s.dims), k
        assert np.array_equal(start_s, start_o), f"case {k}: start differs from the oracle"
        assert np.array_equal(items_s, items_o), f"case {k}: items differ from the oracle"
        assert dt < 0.5, f"case {k}: {dt:.3f} s"


def test_static_grid_takes_no_device_memory_after_set_up():
    """After a warm-up call (the set-up on this device), a further call leaves the
    device's free memory as it was: all its working memory is the fixed array."""
    torch = pytest.importorskip("torch")
    import vxl_sph as vxl
    from vxl_sph import scenes
    lib = vxl.load()
    spec = scenes.dam0()
    n = spec.n_total
    d_pos = torch.from_numpy(np.ascontiguousarray(spec.pos, np.float32)).cuda()
    d_items = torch.empty(n, dtype=torch.int32, device="cuda")
    d_start = torch.empty(LIMIT + 1, dtype=torch.int32, device="cuda")
    info = vxl.GridInfo()
    info.hdr = vxl.header(vxl.GridInfo)
    stream = torch.cuda.current_stream().cuda_stream
    args = (C.c_void_p(d_pos.data_ptr()), n, float(spec.params.smoothing_radius), LIMIT,
            C.c_void_p(d_items.data_ptr()), C.c_void_p(d_start.data_ptr()), LIMIT + 1, C.byref(info),
            C.c_void_p(stream))
    assert lib.vxl_sph_build_grid_static(*args) == vxl.OK, lib.vxl_sph_last_error()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert lib.vxl_sph_build_grid_static(*args) == vxl.OK, lib.vxl_sph_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_static_grid_rejects_sizes_past_its_limit():
    torch = pytest.importorskip("torch")
    import vxl_sph as vxl

    lib = vxl.load()
    info = vxl.GridInfo()
    info.hdr = vxl.header(vxl.GridInfo)
    d = torch.zeros(16, dtype=torch.float32, device="cuda")
    ptr = C.c_void_p(d.data_ptr())
    st = lib.vxl_sph_build_grid_static(ptr, LIMIT + 1, 0.1, LIMIT, ptr, ptr, LIMIT + 1, C.byref(info), None)
    assert st == vxl.INVALID_ARGUMENT and b"524288" in lib.vxl_sph_last_error()
    st = lib.vxl_sph_build_grid_static(ptr, 4, 0.1, LIMIT + 1, ptr, ptr, LIMIT + 2, C.byref(info), None)
    assert st == vxl.INVALID_ARGUMENT
