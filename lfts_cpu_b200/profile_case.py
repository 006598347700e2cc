"""Run a few calc_concs of one system -- a small, self-contained case for
profilers (ncu) and quick timing.

    python -m lfts_cpu_b200.profile_case --mesh 128 --N 8 --precision fp32 --reps 3

--all also runs, after the chain timing, every other kernel of the path once:
an Anderson mix, a Langevin step, an S(k) sample and its binning, H, the
adjoint (FP64) and one Langevin step of a small replica ensemble.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

import lfts_cpu_b200 as lfts


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--mesh", type=int, default=128)
    ap.add_argument("--N", type=int, default=8)
    ap.add_argument("--NA", type=int, default=0, help="default N*25/64")
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--mix", action="store_true", help="also run one Anderson mix")
    ap.add_argument("--all", action="store_true", help="also run every other kernel of the path once")
    a = ap.parse_args(argv)
    m = (a.mesh,) * 3
    M = a.mesh ** 3
    NA = a.NA or max(1, a.N * 25 // 64)
    prec = lfts.LFTS_FP32_MIXED if a.precision == "fp32" else lfts.LFTS_FP64
    s = lfts.System(a.N, NA, 20.0, 100.0, 0.5, m, (a.mesh / 16.0,) * 3, precision=prec)
    s.set_fields(np.random.default_rng(1).normal(0.0, 0.5, 2 * M))
    t0 = time.perf_counter()
    for _ in range(a.reps):
        lnq = s.calc_concs()
    t1 = time.perf_counter()
    k = s.mix() if a.mix else None
    pl, pe, ch = s.profile_chain()
    print(f"mesh {a.mesh}^3 N={a.N} {a.precision}: lnQ {lnq:.12g} calc_concs {1e3 * (t1 - t0) / a.reps:.3f} ms "
          f"plane {1e3 * pl:.1f} us pencil {1e3 * pe:.1f} us chain {ch:.3f} ms mixK {k}")
    if a.all:
        run_all_kernels(s, a, M, prec)


def run_all_kernels(s, a, M, prec):
    """Each remaining kernel of the path once, in the order of a Langevin step."""
    s.calc_concs()
    k = s.mix(20, 1e-4)
    rng = lfts.Rng(5, 0.01)
    s.langevin_init(rng.normal(M))
    s.langevin_step(rng.normal(M))
    s.mix(20, 1e-4)
    s.calc_concs()
    s.sk_sample()
    s.sk_bin()
    H = s.get_H()
    line = f"all kernels: mixK {k} H {H:.12g}"
    if prec == lfts.LFTS_FP64:
        dL, dX, _ = s.backward(max(1, a.N // 4))
        line += f" dH/dL {dL[0]:.6g} dH/dXbN {dX:.6g}"
    reps = [dict(N=a.N, NA=max(1, a.N // 3), XbN=15.0, C=50.0, dt=0.5, m=(mm,) * 3, L=(mm / 16.0,) * 3, seed=7 + r)
            for r, mm in enumerate((32, 48, 64, 32))]
    e = lfts.Ensemble(reps)
    for r, d in enumerate(reps):
        e.set_fields(r, np.random.default_rng(r).normal(0.0, 0.05, 2 * int(np.prod(d["m"]))))
    k0, _ = e.mix(20, 1e-4)
    ks, _ = e.run(1, 20, 1e-4)
    e.close()
    print(line + f"; ensemble mix K {list(k0)} step K {list(ks[0])}")


if __name__ == "__main__":
    main()
