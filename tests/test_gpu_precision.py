"""Error of the FP32-mixed path against the FP64 path (which matches the
reference to 1e-10) for each output -- phi, H and the binned S(k) -- at the
headline size: 128^3, N=64, NA=25, XN=20, C=100, the bench workload's start
and noise.  The same measurement is in bench.py's line (fp32_err_vs_fp64).

Bounds: per call (same fields) phi below 1e-5 relative (the target of the
FP32-mixed form), ln Q below 1e-5 absolute, H below 1e-6 relative; over three
Langevin steps in which each precision runs its own Anderson iterations, phi
and the binned S(k) below 1e-4 (relative to their largest value) and H below
1e-5 relative."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp32_mixed_error_per_output_128(native_lib):
    import bench
    import lfts_cpu_b200 as lfts
    e = bench.fp32_mixed_errors(lfts, 0, nsteps=3)
    pc, tr = e["per_call"], e["trajectory"]
    print(e)
    assert pc["phi_rel"] < 1e-5
    assert pc["lnQ_abs"] < 1e-5
    assert pc["H_rel"] < 1e-6
    assert tr["phi_rel"] < 1e-4
    assert tr["Sk_binned_rel"] < 1e-4
    assert tr["H_rel"] < 1e-5
    assert len(tr["K_fp64"]) == len(tr["K_fp32_mixed"]) == 3
