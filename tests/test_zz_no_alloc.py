"""The allocation-free contour step, lfts_step_fwd_noalloc (collected last).

Callers that cannot allocate device memory -- their device memory comes from a
pool or framework that owns every allocation, or they run where allocation is
not allowed -- call this entry point with their own device inputs and
outputs; its scratch is a fixed static device array.  Here it is called
through the C ABI on two calls in a row and each result is checked against
the context-based lfts_step_fwd on the same inputs, at the FP64 tolerance the
other GPU tests use (1e-10 relative).  Runs alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _params(N, NA, m, L):
    from lfts_cpu_b200.capi import Params
    p = Params()
    p.N, p.NA, p.XbN, p.C, p.dt = N, NA, 15.0, 50.0, 0.5
    for d in range(3):
        p.m[d] = m[d]
        p.L[d] = L[d]
    return p


def _calls(lib, m, N, NA, steps):
    """Calls of the allocation-free step at monomer indices `steps`, each
    checked against the context step on the same inputs."""
    import torch

    import lfts_cpu_b200 as lfts
    M = int(np.prod(m))
    L = (m[0] / 16.0, m[1] / 15.0, m[2] / 17.0)
    rng = np.random.default_rng(M + N)
    ref = lfts.System(N, NA, 15.0, 50.0, 0.5, m, L)
    p = _params(N, NA, m, L)
    dev = torch.device("cuda:0")
    q_out = torch.empty(2 * M, dtype=torch.float64, device=dev)
    for call, i in enumerate(steps):
        q_in = rng.uniform(0.2, 1.5, 2 * M)
        h = rng.uniform(0.5, 1.2, 2 * M)
        expect = ref.step_fwd(q_in, h, i)
        q_in_d = torch.from_numpy(q_in).to(dev)
        h_d = torch.from_numpy(h).to(dev)
        q_out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.lfts_step_fwd_noalloc(C.byref(p), C.c_void_p(q_in_d.data_ptr()), C.c_void_p(q_out.data_ptr()),
                                       C.c_void_p(h_d.data_ptr()), i, None)
        assert rc == 0, lib.lfts_last_error_string().decode()
        torch.cuda.synchronize()
        got = q_out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        assert rel_err(got, expect) < FP64_TOL, f"call {call}"
    ref.close()


# 128 x 32 x 64 fills the scratch exactly: 2 * 128 * 32 * 33 = LFTS_NOALLOC_MAX_SPECTRUM,
# with the 128-point x twiddles and 128 per-plane partial sums at their limits
@pytest.mark.parametrize("m,N,NA", [((64, 64, 64), 16, 6), ((12, 24, 16), 9, 4), ((128, 32, 64), 8, 3)])
def test_noalloc_step_matches_context_step(native_lib, m, N, NA):
    _calls(native_lib, m, N, NA, (1, N - 1))  # two calls in a row, chain-1 h switches between them


def test_noalloc_step_after_a_larger_mesh(native_lib):
    """The scratch keeps the last call's contents; a smaller mesh after the
    largest one reads none of the larger call's tables or spectrum."""
    _calls(native_lib, (128, 32, 64), 8, 3, (2,))
    _calls(native_lib, (8, 12, 20), 7, 3, (1, 5))


def test_noalloc_step_rejects_meshes_above_its_limit(native_lib):
    import torch
    lib = native_lib
    p = _params(8, 4, (128, 128, 128), (8.0, 8.0, 8.0))
    x = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    ptr = C.c_void_p(x.data_ptr())
    rc = lib.lfts_step_fwd_noalloc(C.byref(p), ptr, ptr, ptr, 1, None)
    assert rc == 1  # LFTS_ERR_ARG, before any launch
    assert "limit" in lib.lfts_last_error_string().decode()
    for bad in (0.0, -1.0, float("nan")):
        q = _params(8, 4, (16, 16, 16), (2.0, bad, 2.0))
        assert lib.lfts_step_fwd_noalloc(C.byref(q), ptr, ptr, ptr, 1, None) == 1
        assert "box" in lib.lfts_last_error_string().decode()
    torch.cuda.synchronize()
