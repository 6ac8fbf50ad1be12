"""The allocation-free A^-1 entry point (dphd_ainv_noalloc) against the allocating one (dphd_debug_ainv).

dphd_ainv_noalloc serves callers that cannot call cudaMalloc while stepping (a fixed memory budget, a host
framework that owns the device allocator, or code that must not trigger the implicit device synchronisation
an allocation can cause).  It keeps its temporaries in a static device array, so this test calls it twice in
a row through the C ABI: the second call must not be disturbed by what the first left in that array.  Both
entry points run the same kernels in the same summation order (the input is rounded to FP32 the same way on
the host and on the device), so the results must be bit-identical in FP64 and in FP32.  The test also checks
the contract itself: free device memory does not change across the calls.
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fp32", [0, 1])
def test_noalloc_ainv_matches_allocating_entry_point_twice(fp32):
    import torch
    sc = scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=1)
    d = core.from_scene(sc)
    rng = np.random.default_rng(11)
    b1 = rng.standard_normal(sc.dofs)
    b2 = 3.0 * rng.standard_normal(sc.dofs)
    x1_ref = d.debug_ainv(b1, sc.dt, fp32=bool(fp32))   # allocating entry point; also builds the factor
    x2_ref = d.debug_ainv(b2, sc.dt, fp32=bool(fp32))
    L = core.load_library()
    dev = torch.device("cuda")
    stream = torch.cuda.Stream()
    assert d.device() == torch.cuda.current_device()
    bufs = [(torch.as_tensor(b, device=dev).contiguous(),
             torch.full((sc.dofs,), float("nan"), dtype=torch.float64, device=dev)) for b in (b1, b2)]
    outs = []
    free0 = None
    for db, dx in bufs:
        torch.cuda.synchronize()
        rc = L.dphd_ainv_noalloc(d._h, C.c_double(sc.dt), C.c_void_p(db.data_ptr()), C.c_void_p(dx.data_ptr()),
                                 int(fp32), C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.dphd_last_error().decode()
        stream.synchronize()
        if free0 is None:  # after the first call (which looks the scratch address up), nothing may allocate
            free0 = torch.cuda.mem_get_info()[0]
        outs.append(dx.cpu().numpy())
    assert torch.cuda.mem_get_info()[0] == free0
    for x, ref in zip(outs, (x1_ref, x2_ref)):
        assert np.all(np.isfinite(x))
        assert np.array_equal(x, ref), np.abs(x - ref).max() / np.abs(ref).max()


def test_noalloc_requires_a_built_factor():
    import torch
    sc = scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=1)
    d = core.from_scene(sc)
    L = core.load_library()
    db = torch.zeros(sc.dofs, dtype=torch.float64, device="cuda")
    dx = torch.zeros(sc.dofs, dtype=torch.float64, device="cuda")
    rc = L.dphd_ainv_noalloc(d._h, C.c_double(sc.dt), C.c_void_p(db.data_ptr()), C.c_void_p(dx.data_ptr()), 0,
                             C.c_void_p(0))
    assert rc != 0
    assert b"not on the device yet" in L.dphd_last_error()
