"""Parity at the benchmark configurations' own sizes (N = 64), against
fixtures made by the reference itself (tests/golden/make_golden.py, cases
cfg1_32, cfg2_64, cfg3_128, cfg4_64; 4M field arrays kept as every stride-th
value plus per-quarter sums):

* the plain-FP64 CPU configuration: 32^3, N=64, NA=32, XN=14, C=50, dt=0.5,
  L=4, seeded Gaussian (sd 0.01) start fed as loadType 1; initial mix and 10
  Langevin steps with S(k) sampled every step;
* the plain-FP64 B200 configuration: 64^3, N=64, NA=32, XN=16, C=100,
  L=6.4, (300) lamellar start; initial mix and 3 steps;
* the mixed-precision B200 configuration at its own size: 128^3, N=64, NA=25,
  XN=20, C=100, dt=0.5, L=8, the bench's seeded Gaussian (sd 0.01) start;
  initial mix and one Langevin step with S(k) sampled;
* the adjoint configuration: 64^3, N=64, NA=32, XN=15, C=50, L=6.0,
  lamellar; one step, then H, phi and the backward pass.

Per call (calc_concs of the start fields) the FP64 path is held to 1e-10 and
FP32-mixed to 1e-5 on phi.  Over trajectories the FP64 path is held to 1e-10
on ln Q with the Anderson counts equal, or, where the reference itself is not
that reproducible, to 20 times how far the reference's own run moves when its
start is perturbed by 1e-15 (the fixture records that run: at 32^3 its mixed
w+ moves by 2e-7 relative with the same counts; the 64^3 lamellar starts
change their Anderson counts)."""
import numpy as np
import pytest

from conftest import golden, rel_err
from helpers import parse_header

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


SPREAD_FACTOR = 20.0  # times the reference's own change under a 1e-15 perturbation of the start


def check_compact(w, g, prefix, tol, quarters=(0, 1, 2, 3), spread=None):
    """w (4M) against the fixture's strided values and per-quarter sums.
    Errors are relative to the quarter's largest value (to the larger of
    phi- and phi+ for the two phi quarters).  With `spread` (per-quarter
    absolute change of the reference's own run under a 1e-15 perturbation of
    its start) the tolerance is at least SPREAD_FACTOR times that."""
    M = len(w) // 4
    stride = int(g["stride"])
    s_ref = g[prefix + "_s"]
    idx = np.arange(0, 4 * M, stride)
    sel = [(idx >= q * M) & (idx < (q + 1) * M) for q in range(4)]
    for qtr in quarters:
        a, b = w[::stride][sel[qtr]], s_ref[sel[qtr]]
        scale = np.max(np.abs(b))
        if qtr >= 2:
            scale = max(np.max(np.abs(s_ref[sel[2]])), np.max(np.abs(s_ref[sel[3]])))
        scale = max(scale, 1e-300)
        t = tol if spread is None else max(tol, SPREAD_FACTOR * float(spread[qtr]) / scale)
        err = float(np.max(np.abs(a - b))) / scale
        assert err < t, (prefix, qtr, err, t)
        q = w[qtr * M:(qtr + 1) * M]
        assert abs(q.sum() - g[prefix + "_sum"][qtr]) <= t * scale * M, (prefix, qtr)
        assert abs((q * q).sum() - g[prefix + "_sq"][qtr]) <= 2 * t * scale * scale * M, (prefix, qtr)


def start_fields(lfts, g, hdr, M):
    if int(g["loadType"]) == 1:
        w2 = np.random.default_rng(int(g["field_seed"])).normal(0.0, 0.01, 2 * M)
        assert np.allclose(w2.reshape(2, M).sum(axis=1), g["fields_sum"], rtol=0, atol=1e-12)
        return w2
    return lfts.lamellar_field(float(g["XbN"]), hdr["m"])


def setup(lfts, name, precision=0):
    g = golden(name)
    hdr = parse_header([str(s) for s in g["header"]])
    M = int(np.prod(hdr["m"]))
    s = lfts.System(hdr["N"], hdr["NA"], float(g["XbN"]), hdr["C"], hdr["dt"], hdr["m"], hdr["L"],
                    precision=precision)
    return g, hdr, M, s


def sensitive(g):
    """The reference's own Anderson counts change under a 1e-15 perturbation
    of the start (initial mix or any step)."""
    return (int(g["mix_K_unperturbed"]) != int(g["mix_K_perturbed"])
            or list(g["K_perturbed"]) != list(g["K"]))


@pytest.mark.parametrize("name", ["cfg1_32", "cfg2_64", "cfg3_128", "cfg4_64"])
@pytest.mark.parametrize("precision", [0, 1])
def test_config_calc_concs_of_the_start(lfts, name, precision):
    g, hdr, M, s = setup(lfts, name, precision)
    w2 = start_fields(lfts, g, hdr, M)
    s.set_fields(w2)
    lnQ = s.calc_concs()
    w = s.get_fields()
    tol = FP64_TOL if precision == 0 else 1e-5
    assert abs(lnQ - float(g["cc_lnQ"])) < tol * max(1.0, abs(float(g["cc_lnQ"])))
    check_compact(w, g, "cc_w", tol, quarters=(2, 3))  # phi relative to its largest value
    s.close()


def run_trajectory(lfts, g, hdr, M, s):
    rng = lfts.Rng(123456789, float(g["sigma"]))
    s.langevin_init(rng.normal(M))
    s.set_fields(start_fields(lfts, g, hdr, M))
    s.mix()
    w0 = s.get_fields()
    Ks, lnQs = [], []
    every = int(g["sample_every"])
    for it in range(int(g["n_steps"])):
        s.langevin_step(rng.normal(M))
        Ks.append(s.mix())
        lnQs.append(s.calc_concs())
        if (it + 1) % every == 0:
            s.sk_sample()
    return w0, Ks, np.array(lnQs)


@pytest.mark.parametrize("name", ["cfg1_32", "cfg2_64", "cfg3_128", "cfg4_64"])
def test_config_trajectory_fp64(lfts, name):
    """Initial mix and Langevin steps with the reference's noise stream: the
    mixed start, K per step, ln Q per step, fields, S(k) and its binned text,
    H.  Each is held to the FP64 bar (1e-10 on ln Q, 1e-9 .. 1e-8 on fields)
    or to SPREAD_FACTOR times how far the reference's own run moves when its
    start is perturbed by 1e-15, whichever is looser; the Anderson counts
    must be equal wherever the reference's own counts are reproducible."""
    g, hdr, M, s = setup(lfts, name)
    w0, Ks, lnQs = run_trajectory(lfts, g, hdr, M, s)
    check_compact(w0, g, "w0", 1e-9, spread=g["spread_w0"])
    if not sensitive(g):
        assert Ks == list(g["K"])
    lnq_tol = np.maximum(FP64_TOL * max(1.0, np.max(np.abs(g["lnQ"]))), SPREAD_FACTOR * g["spread_lnQ"])
    assert np.all(np.abs(lnQs - g["lnQ"]) < lnq_tol), (lnQs - g["lnQ"], lnq_tol)
    w = s.get_fields()
    check_compact(w, g, "w_end", 1e-8, spread=g["spread_w_end"])
    stride = int(g["stride"])
    S, ns = s.sk_get()
    assert ns == int(g["nsamples"])
    # S(k) = |FFT(W-)|^2 summed over the samples: its error follows W-'s
    sw = float(np.max(np.abs(g["w_end_s"][: (M + stride - 1) // stride])))
    s_tol = max(1e-8, 2 * SPREAD_FACTOR * float(g["spread_w_end"][0]) / sw)
    assert rel_err(S[::stride], g["S_s"]) < s_tol
    assert abs(S.sum() - float(g["S_sum"])) < s_tol * abs(float(g["S_sum"]))
    K, Sb = s.sk_bin(1e-5)
    ref = np.array([[float(v) for v in ln.split("\t")] for ln in str(g["struct_text"]).strip().split("\n")])
    assert len(K) == len(ref)
    assert np.max(np.abs(K - ref[:, 0])) < 1e-8
    assert np.max(np.abs(Sb - ref[:, 1])) < max(1e-6, s_tol * np.max(np.abs(ref[:, 1])))
    h_tol = max(FP64_TOL * 10 * max(1.0, abs(float(g["H"]))), SPREAD_FACTOR * float(g["spread_H"]))
    assert abs(s.get_H() - float(g["H"])) < h_tol
    check_compact(s.get_fields(), g, "w_H", 1e-8, spread=g["spread_w_end"])
    s.close()


def test_adjoint_configuration_against_reference(lfts):
    """The adjoint configuration (64^3, N=64, NA=32, XN=15, C=50, L=6.0,
    lamellar start): on the start fields the backward pass's H equals the
    reference's H = -ln Q + (sum W-^2/XbN - sum w+)/M (src/lfts_simulation.cc:
    122-135, ln Q of the reference's calc_concs) and, without checkpoints, it
    leaves the reference's phi; with propagators checkpointed every 8
    contour steps it gives the same H and gradients.  (The start's Anderson
    mix is roundoff-sensitive in the reference itself -- the fixture records
    its iteration count changing under a 1e-15 perturbation -- so the pinned
    state is the start, not the mixed field.)"""
    g, hdr, M, s = setup(lfts, "cfg4_64")
    w2 = start_fields(lfts, g, hdr, M)
    s.set_fields(w2)
    H_ref = -float(g["cc_lnQ"]) + (np.sum(w2[:M] ** 2) / float(g["XbN"]) - np.sum(w2[M:])) / M
    dL0, dX0, H0 = s.backward(0)
    assert abs(H0 - H_ref) < FP64_TOL * 10 * max(1.0, abs(H_ref))
    check_compact(s.get_fields(), g, "cc_w", FP64_TOL, quarters=(2, 3))
    assert np.all(np.isfinite(dL0)) and np.isfinite(dX0)
    dL8, dX8, H8 = s.backward(8)
    assert abs(H8 - H0) < 1e-12 * max(1.0, abs(H0))
    assert np.max(np.abs(np.array(dL8) - np.array(dL0))) < 1e-10 * max(1e-12, np.max(np.abs(dL0)))
    assert abs(dX8 - dX0) < 1e-12 * max(1e-12, abs(dX0))
    s.close()
