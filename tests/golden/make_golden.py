"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own classes (oracle/_ref/libref_harness.so: the
reference's unmodified src/*.cc compiled against the FFTW/GSL API shims) and
stores inputs and outputs at full precision.  Needs the reference tree (build
with ``make -C oracle all``); the fixtures it writes are committed, so the
tests never need the reference at run time.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from pyoracle import RefHarness, RefSim, RefSys, build_oracle  # noqa: E402

REF_TREE = os.environ.get("LFTS_REFERENCE", "/root/reference")


def write_input(path, hdr, fields=None):
    """A reference-format input file: 3 header lines, then W- and w+."""
    (N, NA, XN, C, dt, isXeN), (m, L), (neq, nst, nsm, sf, lt) = hdr
    with open(path, "w") as f:
        f.write(f"{N} {NA} {XN!r} {C!r} {dt!r} {isXeN}\n")
        f.write(f"{m[0]} {m[1]} {m[2]} {L[0]!r} {L[1]!r} {L[2]!r}\n")
        f.write(f"{neq} {nst} {nsm} {sf} {lt}\n")
        if fields is not None:
            for v in fields:
                f.write(repr(float(v)) + "\n")


def case_components(name, NA, NB, m, L, seed, wm_sd, wp_sd, steps=(1, 3)):
    """calc_concs, step::fwd and anderson::mix of the reference's classes."""
    rng = np.random.default_rng(seed)
    M = int(np.prod(m))
    w = np.zeros(4 * M)
    w[:M] = rng.normal(0.0, wm_sd, M)
    w[M:2 * M] = rng.normal(0.0, wp_sd, M)
    w_in = w[:2 * M].copy()
    sys_ = RefSys(NA, NB, m, L)
    lnQ = sys_.calc_concs(w)
    phi = w[2 * M:].copy()
    q_in = rng.uniform(0.2, 1.5, 2 * M)
    h = rng.uniform(0.5, 1.2, 2 * M)
    q_out = np.stack([sys_.step_fwd(q_in, h, i) for i in steps])
    g = sys_.g()
    wm = w.copy()
    wm[2 * M:] = 0.0
    K = sys_.mix(wm)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), NA=NA, NB=NB, m=np.array(m), L=np.array(L),
                        w_in=w_in, lnQ=lnQ, phi=phi, q_in=q_in, h=h, steps=np.array(steps), q_out=q_out,
                        g=g, mix_K=K, mix_w=wm)
    sys_.close()
    print(name, "lnQ", lnQ, "mix K", K)


def case_trajectory(name, hdr, n_eq, n_st, sample_every=1, fields=None):
    """A whole reference lfts_simulation: constructor (initial mix), n_eq + n_st
    Langevin steps with full-precision ln Q and K per step, S(k), H."""
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    try:
        os.chdir(work)
        write_input("input", hdr, fields)
        sim = RefSim("input")
        M = sim.M
        w0 = sim.w()
        noise_prev0, _ = sim.noise()
        Ks, lnQs = [], []
        for it in range(1, n_eq + 1):
            k, l = sim.step(sample=False)
            Ks.append(k)
            lnQs.append(l)
        for it in range(1, n_st + 1):
            k, l = sim.step(sample=(it % sample_every == 0))
            Ks.append(k)
            lnQs.append(l)
        w_end = sim.w()
        S, ns = sim.sk_raw()
        sim.sk_save("struct_out")
        with open("struct_out") as f:
            struct_text = f.read()
        H = sim.getH()
        w_H = sim.w()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), header=np.array(
            [open("input").read().split("\n")[i] for i in range(3)]), N=sim.N, NA=sim.NA, m=np.array(sim.m),
            XbN=sim.XbN, XeN=sim.XeN, sigma=sim.sigma, CV=sim.CV, dt=sim.dt, loadType=sim.loadType,
            w0=w0, noise_prev0=noise_prev0, K=np.array(Ks), lnQ=np.array(lnQs), w_end=w_end, S=S,
            nsamples=ns, struct_text=struct_text, H=H, w_H=w_H, n_eq=n_eq, n_st=n_st,
            sample_every=sample_every)
        sim.close()
        print(name, "K", Ks, "H", H, "M", M)
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)


def case_ref_input40(name):
    """calc_concs and one mix on the reference's own 40^3 fixture field
    (input_files/input, loadType 1)."""
    src = os.path.join(REF_TREE, "input_files", "input")
    lines = open(src).read().split("\n")
    hdr = lines[:3]
    N, NA = int(hdr[0].split()[0]), int(hdr[0].split()[1])
    m = [int(x) for x in hdr[1].split()[:3]]
    L = [float(x) for x in hdr[1].split()[3:6]]
    M = int(np.prod(m))
    body = lines[3:3 + 2 * M]
    with gzip.open(os.path.join(HERE, name + "_fields.txt.gz"), "wt") as f:
        f.write("\n".join(hdr) + "\n" + "\n".join(body) + "\n")
    wfield = np.array([float(x) for x in body])
    w = np.zeros(4 * M)
    w[:2 * M] = wfield
    sys_ = RefSys(NA, N - NA, m, L)
    lnQ = sys_.calc_concs(w)
    phi = w[2 * M:].copy()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), N=N, NA=NA, m=np.array(m), L=np.array(L),
                        lnQ=lnQ, phi_sum=phi.reshape(2, M).sum(axis=1), phi_sq=(phi.reshape(2, M) ** 2).sum(axis=1),
                        phi_idx=np.arange(0, 2 * M, 997), phi_at=phi[::997])
    sys_.close()
    print(name, "lnQ", lnQ)


def case_program_run(name, hdr):
    """The reference program itself (oracle/_ref/lfts-ref) on one input: its
    stdout and every output file, packed as tests/golden/<name>.tar.gz."""
    import subprocess
    import tarfile
    from pyoracle import REF_BIN
    work = tempfile.mkdtemp()
    try:
        write_input(os.path.join(work, "input"), hdr)
        out = subprocess.run([REF_BIN, "input"], cwd=work, capture_output=True, text=True,
                             env=dict(os.environ, OMP_NUM_THREADS="4"), check=True).stdout
        with open(os.path.join(work, "stdout.txt"), "w") as f:
            f.write(out)
        with tarfile.open(os.path.join(HERE, name + ".tar.gz"), "w:gz") as tar:
            for fn in sorted(os.listdir(work)):
                tar.add(os.path.join(work, fn), arcname=fn)
        print(name, sorted(os.listdir(work)))
    finally:
        shutil.rmtree(work, ignore_errors=True)


def main():
    build_oracle(ref=True)
    if not RefHarness.available():
        raise SystemExit("oracle/_ref/libref_harness.so missing: the reference tree is needed")
    RefHarness.lib().ref_quiet(1)
    case_components("comp_16", 6, 10, (16, 16, 16), (3.2, 3.0, 3.4), 11, 2.0, 0.5)
    case_components("comp_12x24x16", 7, 9, (12, 24, 16), (2.5, 4.1, 3.3), 12, 1.5, 0.3, steps=(2, 8, 15))
    case_components("comp_8x12x20", 3, 5, (8, 12, 20), (2.0, 2.4, 3.0), 13, 1.0, 0.2, steps=(1, 4, 7))
    # the reference CI's valgrind input (tests/valgrind/input_valgrind): 16^3, N=90, random start
    case_trajectory("traj_valgrind16", ((90, 40, 13.15, 100.0, 1.0, 1), ((16, 16, 16), (4.38, 4.38, 4.38)),
                                        (1, 1, 1, 1000, 3)), 1, 1)
    # a small disordered-start run with S(k) sampling
    case_trajectory("traj_16", ((16, 6, 12.0, 50.0, 0.5, 0), ((16, 16, 16), (3.0, 3.0, 3.0)),
                                (3, 4, 1, 1000, 0)), 3, 4, sample_every=1)
    # lamellar (300) start at 24^3
    case_trajectory("traj_lam24", ((24, 12, 16.0, 100.0, 0.5, 0), ((24, 24, 24), (3.6, 3.6, 3.6)),
                                   (2, 2, 1, 1000, 2)), 2, 2, sample_every=1)
    case_ref_input40("ref_input40")
    # the reference CI's valgrind input, run by the reference program itself
    case_program_run("prog_valgrind16", ((90, 40, 13.15, 100.0, 1.0, 1), ((16, 16, 16), (4.38, 4.38, 4.38)),
                                         (1, 1, 1, 1000, 3)))
    # a disordered-start run that saves and samples every step
    case_program_run("prog_saves16", ((16, 6, 12.0, 50.0, 0.5, 0), ((16, 16, 16), (3.0, 3.0, 3.0)),
                                      (2, 2, 1, 1, 0)))


if __name__ == "__main__":
    main()
