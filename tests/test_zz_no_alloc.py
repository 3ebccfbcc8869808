"""GPU test of the allocation-free entry point kapsel_gpu_solenoidal_u_noalloc.

Callers that cannot allocate device memory (their device memory belongs to
another allocator, or they must not allocate in the middle of a step) use
this entry point; it keeps its work space in a static device array instead
of calling cudaMalloc.  The test calls it through the C ABI on device buffers
that the test itself allocates, twice in a row with different inputs, and
compares each result with the existing allocating entry point
kapsel_gpu_solenoidal_u on the same fields and with the oracle's
Solenoidal_u (relative error <= 1e-12, the FP64 tolerance of the other
spectral tests).  The grids include the largest ones the static array
holds (64^3 and 128x16x128).  The file name sorts last so a
stop-at-first-failure run has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from oracle import spm

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("np_xyz", [(5, 5, 5), (6, 5, 4), (6, 6, 6), (7, 4, 7)])
def test_noalloc_solenoidal_matches_existing_entry_point(np_xyz):
    import torch

    import kapsel_old_b200 as kg

    L = kg.load_library()
    fn = L.kapsel_gpu_solenoidal_u_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_double] + [ctypes.c_void_p] * 7
    cfg = {"np_xyz": np_xyz, "particles": []}
    sim = kg.Simulation(cfg, precision=kg.FP64)
    oracle = spm.Spectral(spm.Params(cfg))
    N = (sim.NX, sim.NY, sim.NZ)
    npx = (ctypes.c_int * 3)(*np_xyz)
    rng = np.random.default_rng(11)
    for call in range(2):
        u = rng.standard_normal((3,) + N) * (1.0 + call)
        expected = sim.solenoidal_u(u)
        dev_in = [torch.tensor(u[d], dtype=torch.float64, device="cuda").contiguous() for d in range(3)]
        dev_out = [torch.full(N, float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()
        rc = fn(npx, 1.0, *[t.data_ptr() for t in dev_in], *[t.data_ptr() for t in dev_out], None)
        assert rc == 0, L.kapsel_gpu_strerror(rc)
        torch.cuda.synchronize()
        got = np.stack([t.cpu().numpy() for t in dev_out])
        assert np.isfinite(got).all()
        assert _rel(got, expected) < 1e-12, (call, _rel(got, expected))
        assert _rel(got, oracle.solenoidal_u(u)) < 1e-12
    sim.close()


def test_noalloc_rejects_oversized_grid():
    import kapsel_old_b200 as kg

    L = kg.load_library()
    fn = L.kapsel_gpu_solenoidal_u_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_double] + [ctypes.c_void_p] * 7
    big = (ctypes.c_int * 3)(7, 7, 7)  # 128^3 exceeds the static work space
    dummy = ctypes.c_void_p(1)
    assert fn(big, 1.0, dummy, dummy, dummy, dummy, dummy, dummy, None) == -6
