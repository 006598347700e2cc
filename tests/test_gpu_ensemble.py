"""Replica ensemble (lfts_ensemble_*): on-device Philox noise against its
restatement; every replica of a mixed-mesh ensemble equals a single
FP32-mixed context fed the same noise (Anderson counts per step, fields,
ln Q); a run shaped like the batched configuration (32 replicas, meshes
32/48/64/96, L = mesh/16, N = 64, NA in [16, 48], XN in [12, 20], C = 50)."""
import numpy as np
import pytest

import philox_ref

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


@pytest.mark.parametrize("seed,step,n", [(1, 0, 1001), (0xDEADBEEF12345, 7, 65536), (2**63 + 5, 2**33 + 1, 4096)])
def test_device_noise_matches_restatement(lfts, seed, step, n):
    dev = lfts.noise_philox(seed, step, n, 0.37)
    ref = philox_ref.noise(seed, step, n, 0.37)
    assert np.max(np.abs(dev - ref)) < 1e-12


def replicas_small():
    return [
        dict(N=12, NA=5, XbN=13.0, C=50.0, dt=0.5, m=(16, 16, 16), L=(3.0, 3.0, 3.0), seed=11),
        dict(N=12, NA=7, XbN=15.5, C=80.0, dt=0.4, m=(24, 24, 24), L=(3.6, 3.6, 3.6), seed=12),
        dict(N=12, NA=4, XbN=12.0, C=50.0, dt=0.5, m=(32, 32, 32), L=(4.0, 4.0, 4.0), seed=13),
        dict(N=12, NA=6, XbN=17.0, C=50.0, dt=0.5, m=(16, 16, 16), L=(2.5, 2.5, 2.5), seed=14),
    ]


def single_run(lfts, d, w2, nsteps, tiles):
    # a single FP32-mixed context with the replica's tiles (the ensemble picks
    # its tiles by timing its batched chain; they can differ from the tiles a
    # lone context of the same mesh picks)
    s = lfts.System(d["N"], d["NA"], d["XbN"], d["C"], d["dt"], d["m"], d["L"], precision=lfts.LFTS_FP32_MIXED)
    s.set_tiles(**tiles)
    assert s.tiles() == tiles
    M = int(np.prod(d["m"]))
    sigma = float(np.sqrt(2.0 * M * d["dt"] / (d["C"] * np.prod(d["L"]))))
    s.set_fields(w2)
    k0 = s.mix()
    lnq0 = s.calc_concs()
    w0 = s.get_fields()
    s.langevin_init(lfts.noise_philox(d["seed"], 0, M, sigma))
    ks = []
    for st in range(1, nsteps + 1):
        s.langevin_step(lfts.noise_philox(d["seed"], st, M, sigma))
        ks.append(s.mix())
        lnq = s.calc_concs()
    w = s.get_fields()
    s.close()
    return k0, lnq0, w0, ks, lnq, w


def test_replicas_equal_single_contexts(lfts):
    reps = replicas_small()
    rng = np.random.default_rng(5)
    fields = [rng.normal(0.0, 1.0, 2 * int(np.prod(d["m"]))) for d in reps]
    e = lfts.Ensemble(reps)
    for r, w2 in enumerate(fields):
        e.set_fields(r, w2)
    k0, lnq0 = e.mix()
    w0 = [e.get_fields(r) for r in range(len(reps))]
    nsteps = 3
    ks, lnq = e.run(nsteps)
    w = [e.get_fields(r) for r in range(len(reps))]
    tiles = [e.tiles(r) for r in range(len(reps))]
    e.close()
    for r, d in enumerate(reps):
        sk0, slnq0, sw0, sks, slnq, sw = single_run(lfts, d, fields[r], nsteps, tiles[r])
        assert k0[r] == sk0
        assert lnq0[r] == slnq0
        assert np.array_equal(w0[r], sw0)
        assert list(ks[:, r]) == sks
        assert lnq[r] == slnq
        assert np.array_equal(w[r], sw)


def test_batched_configuration_shape(lfts):
    """32 replicas drawn from seed like the batched configuration; two steps;
    discrete-chain identities per replica and one replica of each mesh
    against its single context."""
    rng = np.random.default_rng(2024)
    meshes = rng.choice([32, 48, 64, 96], size=32)
    reps = []
    for r, mm in enumerate(meshes):
        reps.append(dict(N=64, NA=int(rng.integers(16, 49)), XbN=float(rng.uniform(12.0, 20.0)), C=50.0, dt=0.5,
                         m=(int(mm),) * 3, L=(mm / 16.0,) * 3, seed=1000 + r))
    fields = [rng.normal(0.0, 0.01, 2 * int(mm) ** 3) for mm in meshes]
    e = lfts.Ensemble(reps)
    for r, w2 in enumerate(fields):
        e.set_fields(r, w2)
    k0, _ = e.mix()
    ks, lnq = e.run(2)
    assert all(e.tuning(r) in (8, 16, 32) for r in range(32))
    for r, mm in enumerate(meshes):
        t = e.tiles(r)
        assert t["two_streams"] == 0
        assert t["plane_stages"] in ((3, 2) if mm in (64, 96) else (2,))
        assert t["h_in_pencil"] in ((0, 1) if mm == 96 else (0,))
        assert t["phi_in_chain"] <= t["h_in_pencil"]
    for r, d in enumerate(reps):
        w = e.get_fields(r)
        M = int(np.prod(d["m"]))
        assert np.all(np.isfinite(w))
        assert abs(w[3 * M:].mean() - 1.0) < 1e-5
        assert abs(w[2 * M:3 * M].mean() - (2 * d["NA"] - d["N"]) / d["N"]) < 1e-5
    checked = set()
    for r, mm in enumerate(meshes):
        if mm in checked:
            continue
        checked.add(mm)
        sk0, _, _, sks, slnq, sw = single_run(lfts, reps[r], fields[r], 2, e.tiles(r))
        assert k0[r] == sk0 and list(ks[:, r]) == sks
        assert lnq[r] == slnq
        assert np.array_equal(e.get_fields(r), sw)
    e.close()


def test_ensemble_rejects_bad_input(lfts):
    from lfts_cpu_b200.capi import LftsError
    base = dict(N=12, NA=5, XbN=13.0, C=50.0, dt=0.5, m=(16, 16, 16), L=(3.0, 3.0, 3.0), seed=1)
    with pytest.raises(LftsError) as e:
        lfts.Ensemble([base, dict(base, m=(128, 128, 128), L=(8.0, 8.0, 8.0))])
    assert e.value.status == 2  # unsupported mesh
    with pytest.raises(LftsError) as e:
        lfts.Ensemble([base, dict(base, N=14)])
    assert e.value.status == 1  # replicas must share N
    ens = lfts.Ensemble([base])
    from lfts_cpu_b200.capi import lib
    assert lib().lfts_ensemble_get_fields(ens._h, 1, np.empty(8)) == 1  # replica index out of range
    with pytest.raises(LftsError):
        ens.mix(max_iter=1)
    ens.close()


@pytest.mark.parametrize("N,NA,phi", [(10, 4, 0), (11, 4, 1), (12, 11, 1)])
def test_h_in_pencil_replicas_equal_single_contexts(lfts, N, NA, phi):
    """96^3 replicas on the h-in-pencil chain (forced for this group, with and
    without the concentration sums formed in the chain; odd N pairs the middle
    slot with itself; NA = 11 of 12 switches h at the last step) against single contexts with the
    same tiles: bitwise, over a mix and two Langevin steps."""
    import os
    reps = [dict(N=N, NA=NA, XbN=14.0 + r, C=50.0, dt=0.5, m=(96, 96, 96), L=(6.0, 6.0, 6.0), seed=300 + r)
            for r in range(2)]
    rng = np.random.default_rng(N)
    fields = [rng.normal(0.0, 0.3, 2 * 96 ** 3) for _ in reps]
    saved = {k: os.environ.get(k) for k in ("LFTS_XH_CHAIN", "LFTS_PHI_IN_CHAIN")}
    os.environ["LFTS_XH_CHAIN"] = "1"
    os.environ["LFTS_PHI_IN_CHAIN"] = str(phi)
    try:
        e = lfts.Ensemble(reps)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    for r, w2 in enumerate(fields):
        e.set_fields(r, w2)
    k0, lnq0 = e.mix()
    ks, lnq = e.run(2)
    tiles = [e.tiles(r) for r in range(len(reps))]
    w = [e.get_fields(r) for r in range(len(reps))]
    e.close()
    for r, d in enumerate(reps):
        assert tiles[r]["h_in_pencil"] == 1 and tiles[r]["phi_in_chain"] == phi and tiles[r]["plane_stages"] == 3
        sk0, slnq0, _, sks, slnq, sw = single_run(lfts, d, fields[r], 2, tiles[r])
        assert k0[r] == sk0 and lnq0[r] == slnq0
        assert list(ks[:, r]) == sks
        assert lnq[r] == slnq
        assert np.array_equal(w[r], sw)
