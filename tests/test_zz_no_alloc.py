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
substep). The tables are integer data, so the tolerance is zero. Two calls in a row,
on different scenes, show that the shared array's leftover contents do not leak into
the next call. Sizes past the fixed limit are refused.

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


def test_static_grid_matches_handle_path_two_calls():
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
