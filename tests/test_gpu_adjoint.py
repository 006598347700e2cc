"""Adjoint of H (lfts_backward) against central finite differences (step
1e-5) of the reference's H (src/lfts_simulation.cc:122-135) at fixed mesh
fields, on the GPU and on the CPU oracle; checkpointed recomputation against
the all-stored pass; and a torch.autograd.Function wrapper (test harness only)
whose gradient matches the same differences."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

EPS = 1e-5


def fields(M, seed, sd_m=1.0, sd_p=0.3):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.normal(0, sd_m, M), rng.normal(0, sd_p, M)])


def H_of(lfts, N, NA, XbN, m, L, w2):
    s = lfts.System(N, NA, XbN, 50.0, 0.5, m, L)
    s.set_fields(w2)
    h = s.get_H()
    s.close()
    return h


def fd_grad(lfts, N, NA, XbN, m, L, w2):
    g = np.zeros(3)
    for d in range(3):
        Lp, Lm = list(L), list(L)
        Lp[d] += EPS
        Lm[d] -= EPS
        g[d] = (H_of(lfts, N, NA, XbN, m, Lp, w2) - H_of(lfts, N, NA, XbN, m, Lm, w2)) / (2 * EPS)
    gx = (H_of(lfts, N, NA, XbN + EPS, m, L, w2) - H_of(lfts, N, NA, XbN - EPS, m, L, w2)) / (2 * EPS)
    return g, gx


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


@pytest.mark.parametrize("m,N,NA,L", [((16, 16, 16), 12, 5, (3.0, 3.3, 2.8)), ((12, 24, 16), 9, 4, (2.5, 4.0, 3.1)),
                                      ((32, 32, 32), 16, 8, (4.0, 4.2, 3.8))])
def test_adjoint_matches_finite_differences(lfts, m, N, NA, L):
    M = int(np.prod(m))
    w2 = fields(M, M + N)
    XbN = 13.0
    s = lfts.System(N, NA, XbN, 50.0, 0.5, m, L)
    s.set_fields(w2)
    dL, dX, H = s.backward()
    g, gx = fd_grad(lfts, N, NA, XbN, m, L, w2)
    assert abs(H - H_of(lfts, N, NA, XbN, m, L, w2)) < 1e-12
    assert rel_err(dL, g) < 1e-6, (dL, g)
    assert abs(dX - gx) < 1e-7 * max(1.0, abs(gx))


@pytest.mark.parametrize("K", [3, 8])
def test_checkpointed_adjoint_equals_stored(lfts, K):
    m, N, NA, L = (16, 16, 16), 20, 9, (3.0, 3.1, 3.2)
    M = int(np.prod(m))
    s = lfts.System(N, NA, 14.0, 50.0, 0.5, m, L)
    s.set_fields(fields(M, 5))
    full = s.backward(0)
    ck = s.backward(K)
    assert rel_err(ck[0], full[0]) < 1e-10
    assert abs(ck[2] - full[2]) < 1e-12 and ck[1] == full[1]


def test_adjoint_headline_configuration(lfts):
    """N=64, NA=32, XN=15, C=50, 64^3, L=6, (300) lamellar start after the
    initial Anderson mix; checkpoints every 8 contour steps; FD step 1e-5."""
    m, N, NA, XbN, L = (64, 64, 64), 64, 32, 15.0, (6.0, 6.0, 6.0)
    s = lfts.System(N, NA, XbN, 50.0, 0.5, m, L)
    s.set_fields(lfts.lamellar_field(XbN, m))
    s.mix()
    w2 = s.get_fields()[: 2 * int(np.prod(m))]
    dL, dX, H = s.backward(8)
    g, gx = fd_grad(lfts, N, NA, XbN, m, L, w2)
    assert rel_err(dL, g) < 1e-6, (dL, g)
    assert abs(dX - gx) < 1e-6 * max(1.0, abs(gx))
    # lamellae along x: the box is strained only along x
    assert abs(dL[0]) > 10 * max(abs(dL[1]), abs(dL[2]))


def test_adjoint_matches_reference_finite_differences(lfts, oracle_built):
    """The same gradient from central differences of the CPU oracle's getH."""
    from pyoracle import Oracle
    m, N, NA, XbN, L = (16, 16, 16), 12, 5, 13.0, (3.0, 3.3, 2.8)
    M = int(np.prod(m))
    w2 = fields(M, 77)

    def H_ref(Lv):
        w = np.zeros(4 * M)
        w[: 2 * M] = w2
        return Oracle(NA, N - NA, m, Lv).getH(w, XbN)

    g = np.zeros(3)
    for d in range(3):
        Lp, Lm = list(L), list(L)
        Lp[d] += EPS
        Lm[d] -= EPS
        g[d] = (H_ref(Lp) - H_ref(Lm)) / (2 * EPS)
    s = lfts.System(N, NA, XbN, 50.0, 0.5, m, L)
    s.set_fields(w2)
    dL, _, H = s.backward()
    assert rel_err(dL, g) < 1e-6
    assert abs(H - H_ref(list(L))) < 1e-10


def test_torch_autograd_wrapper(lfts):
    """torch.autograd.Function over the C ABI: forward = H(L, XbN) via
    lfts_get_H-equivalent lfts_backward, backward = the adjoint."""
    import torch

    m, N, NA = (16, 16, 16), 12, 5
    M = int(np.prod(m))
    w2 = fields(M, 9)

    class LftsH(torch.autograd.Function):
        @staticmethod
        def forward(ctx, Lt, Xt):
            s = lfts.System(N, NA, float(Xt), 50.0, 0.5, m, [float(v) for v in Lt])
            s.set_fields(w2)
            dL, dX, H = s.backward()
            s.close()
            ctx.save_for_backward(torch.tensor(dL, dtype=torch.float64), torch.tensor(dX, dtype=torch.float64))
            return torch.tensor(H, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            dL, dX = ctx.saved_tensors
            return gout * dL, gout * dX

    Lt = torch.tensor([3.0, 3.3, 2.8], dtype=torch.float64, requires_grad=True)
    Xt = torch.tensor(13.0, dtype=torch.float64, requires_grad=True)
    H = LftsH.apply(Lt, Xt)
    (2.0 * H).backward()
    g, gx = fd_grad(lfts, N, NA, 13.0, m, [3.0, 3.3, 2.8], w2)
    assert rel_err(Lt.grad.numpy(), 2.0 * g) < 1e-6
    assert abs(float(Xt.grad) - 2.0 * gx) < 1e-6
