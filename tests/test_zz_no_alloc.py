"""pac_union_measure_noalloc: the union volume/area measure for callers that
cannot allocate device memory (a framework whose allocator has reserved the
GPU, a loop that cannot afford cudaMalloc's implicit synchronisation).  It
must give what pac_union_measure_device gives, call after call, while using
only the library's fixed scratch array.

Collected last on purpose (file name), so a failure here leaves every other
test already run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOL, ALPHA = 1.4, 1.0


def test_noalloc_matches_allocating_entry_point_twice(pac):
    import torch
    balls = pac.globule(3000, seed=pac.SEED_BASE + 41)
    with pac.Engine(tet_mode="as-written") as eng:
        d = torch.from_numpy(balls).cuda()
        cx, _ = eng.alpha_complex_device(d.data_ptr(), len(balls), SOL, ALPHA)
        x = torch.from_numpy(pac.grown_radii(balls, SOL, ALPHA)).cuda()
        dv0 = torch.empty_like(x)
        da0 = torch.empty_like(x)
        torch.cuda.synchronize()  # torch's stream is not the engine's
        v0, a0 = eng.union_measure_device(x.data_ptr(), len(balls), cx, dv0.data_ptr(),
                                          da0.data_ptr())
        for _ in range(2):  # two calls in a row share the scratch array
            dv = torch.full_like(x, 7.0)  # stale contents must not leak in
            da = torch.full_like(x, -3.0)
            torch.cuda.synchronize()
            v, a = eng.union_measure_noalloc(x.data_ptr(), len(balls), cx, dv.data_ptr(),
                                             da.data_ptr())
            assert abs(v - v0) <= 1e-10 * abs(v0)
            assert abs(a - a0) <= 1e-10 * abs(a0)
            assert (dv - dv0).abs().max().item() <= 1e-10 * dv0.abs().max().item()
            assert (da - da0).abs().max().item() <= 1e-10 * da0.abs().max().item()
        # totals only, no gradient buffers
        v, a = eng.union_measure_noalloc(x.data_ptr(), len(balls), cx)
        assert abs(v - v0) <= 1e-10 * abs(v0) and abs(a - a0) <= 1e-10 * abs(a0)


def test_noalloc_rejects_oversized_complex(pac):
    """Beyond the fixed scratch (65,536 blocks of 128 simplices) the call
    fails before running anything.  The complex is backed by real zeroed
    device buffers, so that even a launch would read valid memory."""
    import torch
    n = 16
    x = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    tets = torch.zeros(4 * 9_000_000, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with pac.Engine() as eng:
        cx = pac.Complex(n, 1, 0, 0, 9_000_000, None, None,
                         ctypes.cast(ctypes.c_void_p(tets.data_ptr()),
                                     ctypes.POINTER(ctypes.c_uint32)))
        with pytest.raises(pac.PacError) as ei:
            eng.union_measure_noalloc(x.data_ptr(), n, cx)
        assert ei.value.status == -3
        assert "65536" in str(ei.value)


def test_noalloc_rejects_host_lists_and_size_mismatch(pac):
    """The kernels read the lists in place, so a complex with host lists
    (on_device 0 or 3) or one built for another number of balls is refused
    with an invalid-argument status before anything is launched: the host
    pointers below are never handed to a kernel."""
    import torch
    n = 8
    x = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    host_tets = np.zeros((3, 4), np.uint32)
    ptr = host_tets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    with pac.Engine() as eng:
        for kind in (0, 3):
            cx = pac.Complex(n, kind, 0, 0, 3, None, None, ptr)
            with pytest.raises(pac.PacError) as ei:
                eng.union_measure_noalloc(x.data_ptr(), n, cx)
            assert ei.value.status == -1 and "device lists" in str(ei.value)
        dev_tets = torch.zeros(12, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        cx = pac.Complex(n + 5, 1, 0, 0, 3, None, None,
                         ctypes.cast(ctypes.c_void_p(dev_tets.data_ptr()),
                                     ctypes.POINTER(ctypes.c_uint32)))
        with pytest.raises(pac.PacError) as ei:
            eng.union_measure_noalloc(x.data_ptr(), n, cx)
        assert ei.value.status == -1 and "differ in size" in str(ei.value)
        # a non-empty list without a pointer
        cx = pac.Complex(n, 1, 0, 0, 3, None, None, None)
        with pytest.raises(pac.PacError) as ei:
            eng.union_measure_noalloc(x.data_ptr(), n, cx)
        assert ei.value.status == -1
