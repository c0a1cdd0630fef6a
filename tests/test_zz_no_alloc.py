"""dcb_mark_active_cells_noalloc — active-cell marking without any device allocation, for
callers that manage all device memory themselves (a fixed memory budget or pool) or cannot
afford an allocation's implicit synchronisation. Checked through the C ABI against the
active-cell list of the regular extraction entry point, call after call, since every call
reuses the same file-scope scratch array and must not see the previous call's data.
This file is collected last so that a run stopping at the first failure has run the rest."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(values, dims, spacing, origin, capacity, check_alloc=False):
    import torch
    from contouring_b200 import _lib
    L = _lib.lib()
    grid = _lib.DcbGrid(int(dims[0]), int(dims[1]), int(dims[2]), float(spacing[0]), float(spacing[1]),
                        float(spacing[2]), float(origin[0]), float(origin[1]), float(origin[2]), values.data_ptr())
    out = torch.full((max(capacity, 1),), -1, dtype=torch.int64, device=values.device)
    count = ctypes.c_int64(-1)
    free_before = _device_free_bytes()
    status = L.dcb_mark_active_cells_noalloc(ctypes.byref(grid), ctypes.c_void_p(out.data_ptr()), int(capacity),
                                             ctypes.byref(count),
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if check_alloc:
        # the device's free memory is unchanged across the call: nothing was allocated
        assert _device_free_bytes() == free_before, "device memory was allocated inside the call"
    torch.cuda.synchronize()
    n = max(count.value, 0)
    # nothing is written past the active cells
    assert bool((out[n:] == -1).all()), "entry point wrote past its count"
    return status, out[:n].cpu().numpy(), count.value


def _device_free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_noalloc_matches_extraction_call_after_call():
    from contouring_b200 import B200DualContouringBackend, DenseSdfGridDevice, synth
    be = B200DualContouringBackend(0)
    a = synth.csg(96, seed=2, device="cuda")
    b = synth.sphere(128, 0.35, device="cuda")
    c = synth.noise((37, 21, 30), seed=5)
    c = (c[0].cuda(), c[1], c[2], c[3])
    try:
        refs = []
        for vals, dims, sp, org in (a, b, a, c):
            be.extract_tensor_ptr(DenseSdfGridDevice(*dims, *sp, *org, d_values=vals))
            refs.append(be.active_cells())
        # the first call may load the library's device code (and with it the scratch array);
        # every later call allocates nothing
        _noalloc(*a, len(refs[0]) + 5)
        for (vals, dims, sp, org), ref in zip((a, b, a, c), refs):
            status, got, n = _noalloc(vals, dims, sp, org, len(ref) + 5, check_alloc=True)
            assert status == 0
            assert n == len(ref)
            assert np.array_equal(got, ref)
    finally:
        be.close()


def test_noalloc_reports_small_capacity_and_large_grids():
    import torch
    from contouring_b200 import _lib, synth
    vals, dims, sp, org = synth.sphere(64, 0.3, device="cuda")
    status, _, n = _noalloc(vals, dims, sp, org, 10)
    assert status == _lib.DCB_ERR_TOO_LARGE and n > 10       # count tells the size needed
    status, got, n2 = _noalloc(vals, dims, sp, org, n)
    assert status == 0 and n2 == n and np.all(np.diff(got) > 0)
    big = torch.ones(1024 * 1024 * 130, dtype=torch.float32, device="cuda")  # scratch > 16 MiB
    status, _, _ = _noalloc(big, (1024, 1024, 130), (0.01,) * 3, (0.0,) * 3, 1)
    assert status == _lib.DCB_ERR_TOO_LARGE
    del big
    # the largest cube the fixed scratch is documented to hold: a 450^3 sphere (r = 0.35)
    vals, dims, sp, org = synth.sphere(450, 0.35, device="cuda")
    status, got, n = _noalloc(vals, dims, sp, org, 4_000_000)
    assert status == 0 and n > 0 and np.all(np.diff(got) > 0)
    # every listed cell has corners of both strict signs, and the list has every such cell
    v = vals.view(450, 450, 450)      # [k][j][i]
    corners = torch.stack([v[dk:449 + dk, dj:449 + dj, di:449 + di]
                           for dk in (0, 1) for dj in (0, 1) for di in (0, 1)])
    active = ((corners < 0).any(0) & (corners > 0).any(0)).flatten()
    expect = torch.nonzero(active).flatten().cpu().numpy()
    assert np.array_equal(got, expect)
