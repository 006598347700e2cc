"""Long-run statistics against the reference's own whole run of the plain-FP64
CPU configuration (32^3, N=64, NA=32, XN=14, C=50, dt=0.5, L=4, seeded
Gaussian sd 0.01 start; 1000 equilibration and 1000 statistics steps, S(k)
sampled every 10th statistics step; tests/golden/long_cfg1.npz, made by
tests/golden/make_golden.py from the reference's unmodified sources).

Both precisions are run with the reference's noise stream.  A long run is
compared by its statistics: the mean of H = -ln Q + (sum W-^2 / XbN -
sum w+)/M and of the Anderson count K over the statistics steps, and the
binned S(k), each against the reference's within 4 standard errors (from 10
blocks of 100 steps; S(k): mean squared z over the bins below 2, none above
6).  At this configuration the trajectories do not separate: the FP64 path
also reproduces the reference's run step by step, all 2000 Anderson counts
and H to 1e-9 at every step, and the numbers printed for FP32-mixed show how
closely it follows."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


def block_stats(x, blocks):
    """mean and standard error of the mean from `blocks` equal blocks (axis 0)"""
    b = np.asarray(x).reshape(blocks, -1, *np.shape(x)[1:]).mean(axis=1)
    return b.mean(axis=0), b.std(axis=0, ddof=1) / np.sqrt(blocks)


def run(lfts, g, precision):
    from pyoracle import Oracle
    m = tuple(int(v) for v in g["m"])
    L = tuple(float(v) for v in g["L"])
    M = int(np.prod(m))
    N, NA, XbN = int(g["N"]), int(g["NA"]), float(g["XbN"])
    neq, nst, nsm, blocks = int(g["n_eq"]), int(g["n_st"]), int(g["n_smpl"]), int(g["blocks"])
    s = lfts.System(N, NA, XbN, float(g["C"]), float(g["dt"]), m, L, precision=precision)
    rng = lfts.Rng(123456789, float(g["sigma"]))
    s.langevin_init(rng.normal(M))
    s.set_fields(np.random.default_rng(int(g["field_seed"])).normal(0.0, 0.01, 2 * M))
    s.mix()
    Ks, lnQs, Hs, Sb_blocks = [], [], [], []
    S_prev, ns_prev = None, 0
    per_block = nst // blocks
    for it in range(1, neq + nst + 1):
        s.langevin_step(rng.normal(M))
        Ks.append(s.mix())
        lq = s.calc_concs()
        w = s.get_fields()
        lnQs.append(lq)
        Hs.append(-lq + (np.sum(w[:M] ** 2) / XbN - np.sum(w[M:2 * M])) / M)
        st = it > neq
        if st and (it - neq) % nsm == 0:
            s.sk_sample()
        if st and (it - neq) % per_block == 0:
            S, ns = s.sk_get()
            dS = S if S_prev is None else S - S_prev
            _, Sb = Oracle.sk_bin(m, L, dS, ns - ns_prev, float(g["CV"]), XbN)
            Sb_blocks.append(Sb)
            S_prev, ns_prev = S.copy(), ns
    s.close()
    return np.array(Ks), np.array(lnQs), np.array(Hs), np.array(Sb_blocks)


@pytest.mark.parametrize("precision", [0, 1])
def test_long_run_statistics_match_the_reference(lfts, precision):
    g = golden("long_cfg1")
    neq, blocks = int(g["n_eq"]), int(g["blocks"])
    K, lnQ, H, Sb = run(lfts, g, precision)
    dH = float(np.max(np.abs(H - g["H"])))
    k_diff = int(np.sum(K != g["K"]))
    report = {"steps with another K": k_diff, "max |H - H_ref| over the steps": dH}
    if precision == 0:
        assert k_diff == 0
        assert dH < 1e-9
        assert np.max(np.abs(lnQ - g["lnQ"])) < 1e-9
    for name, a, b in (("H", H[neq:], g["H"][neq:]), ("K", K[neq:].astype(float), g["K"][neq:].astype(float))):
        ma, sa = block_stats(a, blocks)
        mb, sb = block_stats(b, blocks)
        z = (ma - mb) / np.sqrt(sa ** 2 + sb ** 2)
        report[name] = (ma, mb, sa, sb, z)
        assert abs(z) < 4.0, (name, ma, mb, sa, sb)
    assert Sb.shape == g["Sb_blocks"].shape
    ma, sa = block_stats(Sb, blocks)
    mb, sb = block_stats(g["Sb_blocks"], blocks)
    z = (ma - mb) / np.sqrt(sa ** 2 + sb ** 2 + 1e-300)
    report["S(k) bins"] = (len(z), float(np.mean(z ** 2)), float(np.max(np.abs(z))))
    print(f"precision {precision}: {report}")
    assert np.mean(z ** 2) < 2.0
    assert np.max(np.abs(z)) < 6.0
