"""The CPU oracle pinned against the reference (golden fixtures made by
tests/golden/make_golden.py from the reference's own classes) and numpy."""
import numpy as np
import pytest

from conftest import golden, rel_err
from helpers import parse_header, ref_input40_fields


@pytest.fixture(scope="module")
def Oracle(oracle_built):
    from pyoracle import Oracle as O
    return O


@pytest.mark.parametrize("m", [(16, 16, 16), (12, 10, 20), (8, 6, 15), (40, 40, 40), (5, 7, 9), (3, 3, 1)])
def test_fft_core_matches_numpy(Oracle, m):
    x = np.random.default_rng(sum(m)).standard_normal(m)
    X = Oracle.r2c3d(x)
    Xn = np.fft.rfftn(x)
    assert rel_err(X, Xn) < 1e-14
    assert rel_err(Oracle.c2r3d(X, m) / np.prod(m), x) < 1e-14


@pytest.mark.parametrize("name", ["comp_16", "comp_12x24x16", "comp_8x12x20"])
def test_oracle_components_match_reference(Oracle, name):
    g = golden(name)
    m, L = tuple(int(v) for v in g["m"]), tuple(float(v) for v in g["L"])
    NA, NB = int(g["NA"]), int(g["NB"])
    M = int(np.prod(m))
    o = Oracle(NA, NB, m, L)
    assert rel_err(o.g(), g["g"]) == 0.0
    w = np.zeros(4 * M)
    w[: 2 * M] = g["w_in"]
    lnQ = o.calc_concs(w)
    assert abs(lnQ - float(g["lnQ"])) <= 1e-14 * max(1.0, abs(float(g["lnQ"])))
    assert rel_err(w[2 * M:], g["phi"]) < 1e-14
    for j, i in enumerate(g["steps"]):
        assert rel_err(o.step_fwd(g["q_in"], g["h"], int(i)), g["q_out"][j]) < 1e-14
    w[2 * M:] = 0.0
    K = o.mix(w)
    assert K == int(g["mix_K"])
    assert rel_err(w, g["mix_w"]) < 1e-12


def replay(Oracle, g, rng_cls, lamellar):
    """Re-run a reference trajectory with the oracle and the host RNG."""
    hdr = parse_header([str(s) for s in g["header"]])
    N, NA, m, L = hdr["N"], hdr["NA"], tuple(hdr["m"]), tuple(hdr["L"])
    M = int(np.prod(m))
    XbN, sigma, dt = float(g["XbN"]), float(g["sigma"]), float(g["dt"])
    rng = rng_cls(123456789, sigma)
    prev = rng.normal(M)
    assert np.array_equal(prev, g["noise_prev0"])
    if hdr["loadType"] == 2:
        w2 = lamellar(XbN, m)
    else:
        w2 = rng.random_field(XbN, M)
    o = Oracle(NA, N - NA, m, L)
    w = np.zeros(4 * M)
    w[: 2 * M] = w2
    o.mix(w)
    out = dict(w0=w.copy(), K=[], lnQ=[])
    S = np.zeros(o.Mk)
    ns = 0
    n_eq, n_st, every = int(g["n_eq"]), int(g["n_st"]), int(g["sample_every"])
    for it in range(n_eq + n_st):
        eta = rng.normal(M)
        Oracle.langevin_update(w, prev, eta, XbN, dt)
        prev = eta
        out["K"].append(o.mix(w))
        out["lnQ"].append(o.calc_concs(w))
        if it >= n_eq and (it - n_eq + 1) % every == 0:
            o.sk_sample(w, S)
            ns += 1
    out.update(w_end=w.copy(), S=S, ns=ns, H=o.getH(w, XbN), o=o, m=m, L=L)
    return out


@pytest.mark.parametrize("name", ["traj_valgrind16", "traj_16", "traj_lam24"])
def test_oracle_trajectory_matches_reference(Oracle, native_lib, name):
    from lfts_cpu_b200 import Rng, lamellar_field
    g = golden(name)
    r = replay(Oracle, g, Rng, lamellar_field)
    assert rel_err(r["w0"], g["w0"]) < 1e-12
    assert r["K"] == list(g["K"])
    assert np.max(np.abs(np.array(r["lnQ"]) - g["lnQ"])) < 1e-12
    assert rel_err(r["w_end"], g["w_end"]) < 1e-10
    assert abs(r["H"] - float(g["H"])) < 1e-11
    assert r["ns"] == int(g["nsamples"])
    if r["ns"]:
        assert rel_err(r["S"], g["S"]) < 1e-10
        K, Sb = Oracle.sk_bin(r["m"], r["L"], r["S"], r["ns"], float(g["CV"]), float(g["XbN"]))
        lines = [ln.split("\t") for ln in str(g["struct_text"]).strip().split("\n")]
        assert len(lines) == len(K)
        text = "".join(f"{k:.8f}\t{s:.8f}\n" for k, s in zip(K, Sb))
        assert text == str(g["struct_text"])


def test_oracle_reference_input40(Oracle):
    g = golden("ref_input40")
    hdr, fields = ref_input40_fields()
    p = parse_header(hdr)
    M = int(np.prod(p["m"]))
    o = Oracle(p["NA"], p["N"] - p["NA"], p["m"], p["L"])
    w = np.zeros(4 * M)
    w[: 2 * M] = fields
    lnQ = o.calc_concs(w)
    assert abs(lnQ - float(g["lnQ"])) < 1e-13
    phi = w[2 * M:]
    assert rel_err(phi[g["phi_idx"]], g["phi_at"]) < 1e-13
    assert rel_err(phi.reshape(2, M).sum(axis=1), g["phi_sum"]) < 1e-12


def test_oracle_discrete_chain_identities(Oracle):
    """mean(phi+) = 1 and mean(phi-) = (NA-NB)/N hold exactly for the discrete chain."""
    m, N, NA = (12, 24, 16), 11, 4
    M = int(np.prod(m))
    o = Oracle(NA, N - NA, m, (2.0, 3.0, 2.5))
    w = np.zeros(4 * M)
    w[: 2 * M] = np.random.default_rng(5).normal(0, 1.5, 2 * M)
    o.calc_concs(w)
    assert abs(w[3 * M:].mean() - 1.0) < 1e-12
    assert abs(w[2 * M:3 * M].mean() - (2 * NA - N) / N) < 1e-12


def test_z_inf_matches_reference_conversion(Oracle):
    g = golden("traj_valgrind16")
    hdr = parse_header([str(s) for s in g["header"]])
    z = Oracle.z_inf(hdr["L"], hdr["m"], hdr["N"], hdr["C"] ** 2)
    assert float(g["XbN"]) == hdr["XN"] / z
    assert abs(float(g["XeN"]) - hdr["XN"]) == 0.0


def test_oracle_matches_reference_harness_live(Oracle):
    """Random systems, oracle vs the reference's classes, where oracle/_ref exists."""
    from pyoracle import RefHarness, RefSys
    if not RefHarness.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    rng = np.random.default_rng(7)
    for m, NA, NB in [((8, 8, 8), 2, 5), ((10, 6, 12), 5, 5)]:
        M = int(np.prod(m))
        L = tuple(rng.uniform(2, 4, 3))
        w = np.zeros(4 * M)
        w[: 2 * M] = rng.normal(0, 1, 2 * M)
        w2 = w.copy()
        a = Oracle(NA, NB, m, L).calc_concs(w)
        b = RefSys(NA, NB, m, L).calc_concs(w2)
        assert a == b and np.array_equal(w, w2)


def test_lamellar_mix_is_roundoff_sensitive(Oracle, native_lib):
    """The reference's Anderson mix from the (300) lamellar start is chaotic at
    roundoff level: a 1e-15 relative change of the input fields changes the
    iteration count and moves w+ by ~1e-5.  (This is why that trajectory is
    compared at the mixing tolerance on the GPU, not at 1e-10.)"""
    from lfts_cpu_b200 import lamellar_field
    g = golden("traj_lam24")
    m = (24, 24, 24)
    M = int(np.prod(m))
    w2 = lamellar_field(float(g["XbN"]), m)
    out = []
    for pert in (0.0, 1e-15):
        o = Oracle(12, 12, m, (3.6, 3.6, 3.6))
        w = np.zeros(4 * M)
        w[: 2 * M] = w2 * (1.0 + pert)
        out.append((o.mix(w), w))
    assert rel_err(out[0][1], g["w0"]) < 1e-12
    assert out[0][0] != out[1][0]
    assert rel_err(out[1][1], out[0][1]) > 1e-7


EDGE_CHAINS = [(0, 8), (8, 0), (1, 1), (3, 4), (4, 3)]  # NA, NB: homopolymer ends, N = 2, odd N


@pytest.mark.parametrize("NA,NB", EDGE_CHAINS)
def test_oracle_matches_reference_chain_edges(oracle_built, NA, NB):
    """Pure-A / pure-B chains, the shortest chain and odd N: the restatement
    equals the reference's own classes (shim build) bitwise, calc_concs and mix."""
    from pyoracle import Oracle, RefHarness, RefSys
    if not RefHarness.available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    m, L = (8, 12, 20), (2.0, 2.5, 3.0)
    M = int(np.prod(m))
    rng = np.random.default_rng(NA * 10 + NB)
    w = np.zeros(4 * M)
    w[:2 * M] = rng.normal(0.0, 0.8, 2 * M)
    a, b = w.copy(), w.copy()
    o, r = Oracle(NA, NB, m, L), RefSys(NA, NB, m, L)
    assert o.calc_concs(a) == r.calc_concs(b)
    assert np.array_equal(a, b)
    a[2 * M:] = 0.0
    b[2 * M:] = 0.0
    assert o.mix(a) == r.mix(b)
    assert np.array_equal(a, b, equal_nan=True)  # NB = 0: the reference's mix diverges to NaN
    o.close()
    r.close()


@pytest.mark.parametrize("m,NA,NB", [((16, 12, 20), 5, 7), ((8, 8, 8), 0, 4), ((12, 16, 8), 3, 0)])
def test_scipy_bound_restatement_matches_oracle(Oracle, m, NA, NB):
    """The scipy.fft calc_concs that bench.py times as the best-CPU-FFT bound
    computes what the oracle computes."""
    from scipy_path import ScipyConcs
    L = (3.0, 2.5, 3.4)
    M = int(np.prod(m))
    w = np.zeros(4 * M)
    w[:2 * M] = np.random.default_rng(M).normal(0.0, 1.0, 2 * M)
    w2 = w.copy()
    a = Oracle(NA, NB, m, L).calc_concs(w)
    b = ScipyConcs(NA, NB, m, L, workers=2).calc_concs(w2)
    assert abs(a - b) < 1e-13 * max(1.0, abs(a))
    assert rel_err(w2[2 * M:], w[2 * M:]) < 1e-13


def test_reference_full_step_matches_oracle(Oracle):
    """The reference's own loop body as bench.py's reference arm times it
    (langevin object on mt19937_64, step_wm, mix, the extra calc_concs) equals
    the oracle fed the same noise, bitwise."""
    import pyoracle
    if not pyoracle.RefHarness.available():
        pytest.skip("oracle/_ref not built (no reference tree on this machine)")
    m, NA, NB, L, XbN, dt = (12, 16, 8), 5, 7, (3.0, 3.2, 2.4), 14.0, 0.5
    M = int(np.prod(m))
    sigma = 0.8
    w = np.zeros(4 * M)
    w[:2 * M] = np.random.default_rng(2).normal(0.0, 0.3, 2 * M)
    wo = w.copy()
    ref = pyoracle.RefSys(NA, NB, m, L)
    lg = pyoracle.RefLangevin(99, sigma, M)
    ref.mix(w)
    o = Oracle(NA, NB, m, L)
    o.mix(wo)
    noise = np.empty(3 * M)
    pyoracle.RefHarness.lib().ref_normal_stream(99, sigma, 3 * M, noise)
    for st in range(2):
        K, lnQ = lg.full_step(ref, w, XbN, dt)
        Oracle.langevin_update(wo, noise[st * M:(st + 1) * M], noise[(st + 1) * M:(st + 2) * M], XbN, dt)
        assert o.mix(wo) == K
        assert o.calc_concs(wo) == lnQ
        assert np.array_equal(w, wo)
    lam = pyoracle.ref_lamellar(16.0, m)
    expect = 16.0 * np.cos(2.0 * np.pi * (3.0 * np.arange(m[0]) / m[0]))
    assert np.max(np.abs(lam[:M].reshape(m)[:, 0, 0] - expect)) < 1e-13
    assert np.all(lam[M:] == 0.0)


def test_oracle_matches_reference_at_config1_size(Oracle):
    """The oracle against the reference at the plain-FP64 configuration's own
    size (32^3, N=64, NA=32, seeded Gaussian start): calc_concs of the start
    and the initial Anderson mix (fixture cfg1_32, compact)."""
    g = golden("cfg1_32")
    hdr = parse_header([str(s) for s in g["header"]])
    m, L = tuple(hdr["m"]), tuple(hdr["L"])
    M = int(np.prod(m))
    stride = int(g["stride"])
    w = np.zeros(4 * M)
    w[:2 * M] = np.random.default_rng(int(g["field_seed"])).normal(0.0, 0.01, 2 * M)
    o = Oracle(hdr["NA"], hdr["N"] - hdr["NA"], m, L, threads=4)
    assert abs(o.calc_concs(w) - float(g["cc_lnQ"])) < 1e-14
    assert rel_err(w[::stride][2 * M // stride + 1:], g["cc_w_s"][2 * M // stride + 1:]) < 1e-13
    w[2 * M:] = 0.0
    assert o.mix(w) == int(g["mix_K_unperturbed"])
    o.close()
