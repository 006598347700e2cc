"""Failure statuses of the Anderson loop, made on the host (no GPU fault):

* a NaN written into W- with set_fields: LFTS_ERR_NONFINITE, w+ not updated
  with the NaN residual;
* an iteration cap below what the field needs: LFTS_ERR_NOTCONV with the
  reference's k and the reference's fields (the oracle with the same cap);
* an exactly singular least-squares system (zero fields, so phi+ = 1
  exactly and every residual is zero; a negative tolerance keeps the loop
  going into the Anderson step): LFTS_ERR_SINGULAR, where the reference's
  GSL solve would abort the program;

each for single contexts in both precisions and for a 2-replica ensemble,
whose device-side loop ends at its cap and reports per replica while the
healthy replica runs on unchanged."""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

M3, N, NA, L = (16, 16, 16), 16, 6, (3.0, 3.0, 3.0)
M = int(np.prod(M3))


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


@pytest.fixture(params=["device", "host"])
def system(lfts, request):
    """A 16^3 context with its Anderson loop on the device or
    on the host (the default; LFTS_DEVICE_MIX=1 selects the device loop)."""
    def make(precision):
        old = os.environ.get("LFTS_DEVICE_MIX")
        os.environ["LFTS_DEVICE_MIX"] = "1" if request.param == "device" else "0"
        try:
            return lfts.System(N, NA, 12.0, 50.0, 0.5, M3, L, precision=precision)
        finally:
            if old is None:
                del os.environ["LFTS_DEVICE_MIX"]
            else:
                os.environ["LFTS_DEVICE_MIX"] = old
    return make


def rough(seed=3):
    return np.random.default_rng(seed).normal(0.0, 1.0, 2 * M)


@pytest.mark.parametrize("precision", [0, 1])
def test_nan_field_reports_nonfinite(lfts, system, precision):
    s = system(precision)
    w2 = rough()
    w2[123] = np.nan
    s.set_fields(w2)
    with pytest.raises(lfts.LftsError) as e:
        s.mix()
    assert e.value.status == lfts.LFTS_ERR_NONFINITE
    assert np.array_equal(s.get_fields()[M:2 * M], w2[M:2 * M])  # w+ untouched
    s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_iteration_cap_reports_notconv(lfts, system, oracle_built, precision):
    from pyoracle import Oracle
    s = system(precision)
    w2 = rough()
    s.set_fields(w2)
    k = s.mix(max_iter=3)
    assert k == 3 and s.last_status == lfts.LFTS_ERR_NOTCONV
    with pytest.raises(lfts.LftsError) as e:
        s.mix(max_iter=3, strict=True)
    assert e.value.status == lfts.LFTS_ERR_NOTCONV
    # the fields after the first capped mix are the reference's (oracle, same cap)
    s2 = system(precision)
    s2.set_fields(w2)
    s2.mix(max_iter=3)
    o = Oracle(NA, N - NA, M3, L)
    w = np.zeros(4 * M)
    w[:2 * M] = w2
    assert o.mix(w, max_iter=3) == 3
    tol = 1e-9 if precision == 0 else 1e-5
    assert rel_err(s2.get_fields()[M:2 * M], w[M:2 * M]) < tol
    # a full step past the cap completes (the extra calc_concs runs) and reports it
    import torch
    s2.langevin_init(np.zeros(M))
    noise = torch.from_numpy(np.random.default_rng(9).normal(0.0, 1.0, M)).to("cuda:0")
    k2, lnq = s2.full_step_device(noise.data_ptr(), max_iter=2)
    assert k2 == 2 and s2.last_status == lfts.LFTS_ERR_NOTCONV and np.isfinite(lnq)
    for x in (s, s2, o):
        x.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_singular_system_reports_singular(lfts, system, precision):
    s = system(precision)
    s.set_fields(np.zeros(2 * M))
    with pytest.raises(lfts.LftsError) as e:
        s.mix(max_iter=10, tol=-1.0)
    assert e.value.status == lfts.LFTS_ERR_SINGULAR
    s.close()


def ensemble_pair(lfts):
    reps = [dict(N=N, NA=NA, XbN=12.0, C=50.0, dt=0.5, m=M3, L=L, seed=1 + r) for r in range(2)]
    return reps, lfts.Ensemble(reps)


def test_ensemble_statuses_per_replica(lfts):
    reps, e = ensemble_pair(lfts)
    good = rough(4)
    bad = rough(5)
    bad[77] = np.nan
    # NaN in replica 1: the call reports it, replica 0 mixes as a single context does
    e.set_fields(0, good)
    e.set_fields(1, bad)
    with pytest.raises(lfts.LftsError) as ex:
        e.mix()
    assert ex.value.status == lfts.LFTS_ERR_NONFINITE
    assert e.replica_status(1) == lfts.LFTS_ERR_NONFINITE
    assert e.replica_status(0) == lfts.LFTS_OK
    s = lfts.System(N, NA, 12.0, 50.0, 0.5, M3, L, precision=lfts.LFTS_FP32_MIXED)
    s.set_fields(good)
    s.mix()
    s.calc_concs()
    assert np.array_equal(e.get_fields(0), s.get_fields())
    assert np.array_equal(e.get_fields(1)[M:2 * M], bad[M:2 * M])  # w+ untouched
    # the cap: both replicas stop at it and the call carries on (non-strict)
    e.set_fields(0, good)
    e.set_fields(1, rough(6))
    k, lnq = e.mix(max_iter=3)
    assert list(k) == [3, 3] and e.last_status == lfts.LFTS_ERR_NOTCONV
    assert all(e.replica_status(r) == lfts.LFTS_ERR_NOTCONV for r in range(2)) and np.all(np.isfinite(lnq))
    # a singular system in replica 1 only
    e.set_fields(0, good)
    e.set_fields(1, np.zeros(2 * M))
    with pytest.raises(lfts.LftsError) as ex:
        e.mix(max_iter=10, tol=-1.0)
    assert ex.value.status == lfts.LFTS_ERR_SINGULAR
    assert e.replica_status(1) == lfts.LFTS_ERR_SINGULAR
    assert e.replica_status(0) == lfts.LFTS_ERR_NOTCONV  # tol < 0: replica 0 runs to the cap
    # a run whose steps stop at the cap completes every step
    e.set_fields(0, good)
    e.set_fields(1, rough(6))
    e.mix()
    ks, lnq = e.run(2, max_iter=2)
    assert ks.shape == (2, 2) and np.all(ks == 2) and e.last_status == lfts.LFTS_ERR_NOTCONV
    assert np.all(np.isfinite(lnq))
    s.close()
    e.close()
