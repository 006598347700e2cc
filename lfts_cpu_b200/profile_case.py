"""Run a few calc_concs of one system -- a small, self-contained case for
profilers (ncu) and quick timing.

    python -m lfts_cpu_b200.profile_case --mesh 128 --N 8 --precision fp32 --reps 3
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


if __name__ == "__main__":
    main()
