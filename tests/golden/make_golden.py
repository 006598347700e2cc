"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own classes (oracle/_ref/libref_harness.so: the
reference's unmodified src/*.cc compiled against the FFTW/GSL API shims) and
stores inputs and outputs at full precision.  Needs the reference tree (build
with ``make -C oracle all``); the fixtures it writes are committed, so the
tests never need the reference at run time.

    LFTS_REFERENCE=<reference tree> python tests/golden/make_golden.py [case ...]

With case names, only those fixtures are written (see CASES below).
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

REF_TREE = os.environ.get("LFTS_REFERENCE")


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


def _compact(prefix, w, M, stride):
    """A 4M field array as every stride-th value plus per-quarter sums and sums of squares."""
    q = w.reshape(4, M)
    return {prefix + "_s": w[::stride].copy(), prefix + "_sum": q.sum(axis=1), prefix + "_sq": (q * q).sum(axis=1)}


def case_config(name, hdr, n_steps, stride, field_seed=None, sample_every=1, sensitivity=False, threads=None):
    """A run at one of the benchmark configurations' own sizes (N = 64), kept
    compact: 4M field arrays are stored as every stride-th value plus
    per-quarter sums.  Stores
      * calc_concs of the start fields (RefSys): ln Q, phi;
      * with ``sensitivity``: whether the reference's own mix of the start
        fields changes its iteration count under a 1e-15 relative perturbation;
      * the reference constructor's initial mix (RefSim): the mixed fields;
      * n_steps Langevin steps: K and ln Q per step, S(k) samples, fields, H.
    Start fields: a seeded Gaussian (numpy default_rng(field_seed), mean 0,
    sd 0.01, fed as loadType 1) or the reference's own generator (loadType 2)."""
    (N, NA, XN, C, dt, isXeN), (m, L), rest = hdr
    M = int(np.prod(m))
    if threads:
        # FFT threads of the reference's plans (the shim splits a batch of
        # line transforms across threads; each line's arithmetic is unchanged)
        RefHarness.lib().ref_set_threads(int(threads))
    out = {"stride": stride}
    fields = None
    if field_seed is not None:
        fields = np.random.default_rng(field_seed).normal(0.0, 0.01, 2 * M)
        out.update(field_seed=field_seed, fields_sum=fields.reshape(2, M).sum(axis=1))
        start = fields.copy()
    else:
        from pyoracle import ref_lamellar
        start = ref_lamellar(XN, m)  # isXeN = 0: XbN = XN
    sys_ = RefSys(NA, N - NA, m, L)
    w = np.zeros(4 * M)
    w[:2 * M] = start
    out["cc_lnQ"] = sys_.calc_concs(w)
    out.update(_compact("cc_w", w, M, stride))
    sys_.close()
    if sensitivity:
        # the reference's own reproducibility: the same run (initial mix, the
        # same Langevin steps and noise) from the start and from the start
        # times (1 + 1e-15); how far its fields, ln Q and H move is the
        # tolerance a faithful restatement can be held to on this run
        from pyoracle import RefLangevin
        sigma = float(np.sqrt(2.0 * M * dt / (C * np.prod(L))))
        runs = []
        for eps in (0.0, 1e-15):
            s2 = RefSys(NA, N - NA, m, L)
            lg = RefLangevin(123456789, sigma, M)
            wp = np.zeros(4 * M)
            wp[:2 * M] = start * (1.0 + eps)
            k0 = s2.mix(wp)
            w0 = wp.copy()
            ks, lqs = [k0], []
            for _ in range(n_steps):
                k, lq = lg.full_step(s2, wp, XN, dt)
                ks.append(k)
                lqs.append(lq)
            lnq_end = s2.calc_concs(wp)
            H = -lnq_end + (np.sum(wp[:M] ** 2) / XN - np.sum(wp[M:2 * M])) / M
            runs.append((ks, w0, wp.copy(), np.array(lqs), H))
            s2.close()
            lg.close()
        (ka, w0a, wea, lqa, Ha), (kb, w0b, web, lqb, Hb) = runs
        quarter_diff = lambda a, b: np.abs(a - b).reshape(4, M).max(axis=1)  # noqa: E731
        out.update(mix_K_unperturbed=ka[0], mix_K_perturbed=kb[0], K_perturbed=np.array(kb[1:]),
                   spread_w0=quarter_diff(w0a, w0b), spread_w_end=quarter_diff(wea, web),
                   spread_lnQ=np.abs(lqa - lqb), spread_H=abs(Ha - Hb))
        print(name, "K with and without a 1e-15 perturbation", ka, kb, "spread w0", out["spread_w0"],
              "spread H", out["spread_H"])
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    try:
        os.chdir(work)
        write_input("input", hdr, fields)
        sim = RefSim("input")
        out.update(_compact("w0", sim.w(), M, stride))
        Ks, lnQs = [], []
        for it in range(1, n_steps + 1):
            k, l = sim.step(sample=(it % sample_every == 0))
            Ks.append(k)
            lnQs.append(l)
        out.update(_compact("w_end", sim.w(), M, stride))
        S, ns = sim.sk_raw()
        sim.sk_save("struct_out")
        with open("struct_out") as f:
            out["struct_text"] = f.read()
        out["H"] = sim.getH()
        out.update(_compact("w_H", sim.w(), M, stride))  # phi of getH's calc_concs: of the final fields
        out.update(header=np.array([open("input").read().split("\n")[i] for i in range(3)]), N=sim.N, NA=sim.NA,
                   m=np.array(sim.m), L=np.array(L), XbN=sim.XbN, sigma=sim.sigma, CV=sim.CV, dt=sim.dt,
                   loadType=sim.loadType, K=np.array(Ks), lnQ=np.array(lnQs), S_s=S[::stride], S_sum=S.sum(),
                   nsamples=ns, n_steps=n_steps,
                   sample_every=sample_every)
        sim.close()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "K", Ks, "H", out["H"], "M", M)
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


def case_program_compact(name, src_input, every=997):
    """The reference program (oracle/_ref/lfts-ref) on one of the reference's own
    input files, for meshes whose output files are too large to keep: its
    stdout, and per output file the line count and every `every`-th line
    (lines 0, every, 2 every, ...), in tests/golden/<name>.npz."""
    import subprocess
    from pyoracle import REF_BIN
    work = tempfile.mkdtemp()
    try:
        shutil.copy(src_input, os.path.join(work, "input"))
        out = subprocess.run([REF_BIN, "input"], cwd=work, capture_output=True, text=True,
                             env=dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count())), check=True).stdout
        files = sorted(f for f in os.listdir(work) if f != "input")
        rec = {"input": open(os.path.join(work, "input")).read(), "stdout": out, "files": np.array(files),
               "every": every}
        for f in files:
            lines = open(os.path.join(work, f)).read().splitlines()
            rec["n_" + f] = len(lines)
            rec["s_" + f] = np.array(lines[::every])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **rec)
        print(name, files, [rec["n_" + f] for f in files])
    finally:
        shutil.rmtree(work, ignore_errors=True)


def case_long_run(name, hdr, field_seed, blocks=10):
    """A whole run of the reference at one configuration (its n_eq
    equilibration and n_st statistics steps, S(k) sampled every n_smpl
    statistics steps), kept as what a long run is compared by: K, ln Q and
    H = -ln Q + (sum W-^2 / XbN - sum w+)/M per step, and the binned S(k) of
    each of `blocks` equal blocks of the statistics steps (binned with the
    oracle's restatement of strFunc::save, checked here against the
    reference's own struct file for the whole accumulation)."""
    from pyoracle import Oracle
    (N, NA, XN, C, dt, isXeN), (m, L), (neq, nst, nsm, sf, lt) = hdr
    M = int(np.prod(m))
    fields = np.random.default_rng(field_seed).normal(0.0, 0.01, 2 * M)
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    try:
        os.chdir(work)
        write_input("input", hdr, fields)
        RefHarness.lib().ref_set_threads(os.cpu_count())
        sim = RefSim("input")
        XbN, CV = sim.XbN, sim.CV
        Ks, lnQs, Hs = [], [], []
        S_prev, ns_prev = np.zeros(sim.Mk), 0
        per_block = nst // blocks
        Sb_blocks, K_bins = [], None
        for it in range(1, neq + nst + 1):
            st = it > neq
            k, lq = sim.step(sample=st and ((it - neq) % nsm == 0))
            w = sim.w()
            Ks.append(k)
            lnQs.append(lq)
            Hs.append(-lq + (np.sum(w[:M] ** 2) / XbN - np.sum(w[M:2 * M])) / M)
            if st and (it - neq) % per_block == 0:
                S, ns = sim.sk_raw()
                Kb, Sb = Oracle.sk_bin(m, L, S - S_prev, ns - ns_prev, CV, XbN)
                K_bins = Kb
                Sb_blocks.append(Sb)
                S_prev, ns_prev = S.copy(), ns
        S, ns = sim.sk_raw()
        sim.sk_save("struct_out")
        ref = np.array([[float(v) for v in ln.split("\t")] for ln in open("struct_out").read().strip().split("\n")])
        Kb, Sb = Oracle.sk_bin(m, L, S, ns, CV, XbN)
        assert len(Kb) == len(ref) and np.max(np.abs(Kb - ref[:, 0])) < 1e-8
        assert np.max(np.abs(Sb - ref[:, 1])) < 1e-7 * max(1.0, np.max(np.abs(ref[:, 1])))
        sim.close()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), K=np.array(Ks), lnQ=np.array(lnQs), H=np.array(Hs),
                            K_bins=K_bins, Sb_blocks=np.array(Sb_blocks), field_seed=field_seed, n_eq=neq,
                            n_st=nst, n_smpl=nsm, blocks=blocks, XbN=XbN, CV=CV, sigma=sim.sigma, N=N, NA=NA,
                            m=np.array(m), L=np.array(L), C=C, dt=dt)
        print(name, "mean K", np.mean(Ks), "H st mean", np.mean(Hs[neq:]), "bins", len(K_bins))
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)


def case_program_spread(name, src_input, every=997):
    """How reproducible the reference program's w_0 / phi_0 (the fields after
    its initial Anderson mix, src/lfts_simulation.cc:52-56) are on one of its
    own inputs: its random start (the program's generator, after the langevin
    constructor's draws) mixed twice by the reference's objects, as is and
    times (1 + 1e-15); the 6-significant-digit text of the two results is
    compared value by value, over all values and over the lines the compact
    program fixture keeps (every `every`-th line of the file).  The first run
    must equal the program's own w_0 bit for bit."""
    from pyoracle import RefLangevin
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    try:
        os.chdir(work)
        shutil.copy(src_input, "input")
        RefHarness.lib().ref_set_threads(os.cpu_count())
        sim = RefSim("input")
        w_prog = sim.w()
        M, N, NA, XbN, sigma = sim.M, sim.N, sim.NA, sim.XbN, sim.sigma
        m = list(sim.m)
        L = [float(x) for x in open("input").read().split("\n")[1].split()[3:6]]
        sim.close()
    finally:
        os.chdir(cwd)
        shutil.rmtree(work, ignore_errors=True)
    lg = RefLangevin(123456789, sigma, M)
    start = lg.uniform_field(XbN, M)
    lg.close()
    runs = []
    for eps in (0.0, 1e-15):
        s2 = RefSys(NA, N - NA, m, L)
        w = np.zeros(4 * M)
        w[:2 * M] = start * (1.0 + eps)
        s2.mix(w)
        runs.append(w)
        s2.close()
    assert np.array_equal(runs[0], w_prog), "the harness start is not the program's"
    text = lambda a: np.array(["%g" % v for v in a])  # noqa: E731  (the files' default 6 digits)
    out = {"every": every, "spread": np.abs(runs[0] - runs[1]).reshape(4, M).max(axis=1)}
    for f, lo, hi, header in (("w_0", 0, 2 * M, 3), ("phi_0", 2 * M, 4 * M, 0)):
        ta, tb = text(runs[0][lo:hi]), text(runs[1][lo:hi])
        diff = ta != tb
        lines = np.arange(header, header + (hi - lo))  # file line of each value
        out["flips_all_" + f] = int(diff.sum())
        out["flips_sampled_" + f] = int(diff[lines % every == 0].sum())
        out["n_sampled_" + f] = int((lines % every == 0).sum())
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: v for k, v in out.items()})


CASES = {
    "comp_16": lambda: case_components("comp_16", 6, 10, (16, 16, 16), (3.2, 3.0, 3.4), 11, 2.0, 0.5),
    "comp_12x24x16": lambda: case_components("comp_12x24x16", 7, 9, (12, 24, 16), (2.5, 4.1, 3.3), 12, 1.5, 0.3,
                                             steps=(2, 8, 15)),
    "comp_8x12x20": lambda: case_components("comp_8x12x20", 3, 5, (8, 12, 20), (2.0, 2.4, 3.0), 13, 1.0, 0.2,
                                            steps=(1, 4, 7)),
    # the reference CI's valgrind input (tests/valgrind/input_valgrind): 16^3, N=90, random start
    "traj_valgrind16": lambda: case_trajectory(
        "traj_valgrind16", ((90, 40, 13.15, 100.0, 1.0, 1), ((16, 16, 16), (4.38, 4.38, 4.38)), (1, 1, 1, 1000, 3)),
        1, 1),
    # a small disordered-start run with S(k) sampling
    "traj_16": lambda: case_trajectory(
        "traj_16", ((16, 6, 12.0, 50.0, 0.5, 0), ((16, 16, 16), (3.0, 3.0, 3.0)), (3, 4, 1, 1000, 0)), 3, 4,
        sample_every=1),
    # lamellar (300) start at 24^3
    "traj_lam24": lambda: case_trajectory(
        "traj_lam24", ((24, 12, 16.0, 100.0, 0.5, 0), ((24, 24, 24), (3.6, 3.6, 3.6)), (2, 2, 1, 1000, 2)), 2, 2,
        sample_every=1),
    "ref_input40": lambda: case_ref_input40("ref_input40"),
    # the reference CI's valgrind input, run by the reference program itself
    "prog_valgrind16": lambda: case_program_run(
        "prog_valgrind16", ((90, 40, 13.15, 100.0, 1.0, 1), ((16, 16, 16), (4.38, 4.38, 4.38)), (1, 1, 1, 1000, 3))),
    # a disordered-start run that saves and samples every step
    "prog_saves16": lambda: case_program_run(
        "prog_saves16", ((16, 6, 12.0, 50.0, 0.5, 0), ((16, 16, 16), (3.0, 3.0, 3.0)), (2, 2, 1, 1, 0))),
    # the reference's own 128^3 input (input_files/input128: N=90, NA=40,
    # XeN=13.15 with isXeN=1, random start, 2 equilibration steps), run by the
    # reference program; its 2M-line field files kept as every 997th line
    "prog_input128": lambda: case_program_compact(
        "prog_input128", os.path.join(REF_TREE, "input_files", "input128")),
    # the reference's own reproducibility of that run's w_0 / phi_0
    "spread_input128": lambda: case_program_spread(
        "spread_input128", os.path.join(REF_TREE, "input_files", "input128")),
    "spread_input64": lambda: case_program_spread(
        "spread_input64", os.path.join(REF_TREE, "input_files", "input64"), every=97),
    # the same at 64^3 (input_files/input64)
    "prog_input64": lambda: case_program_compact(
        "prog_input64", os.path.join(REF_TREE, "input_files", "input64"), every=97),
    # the plain-FP64 CPU configuration run whole (1000 + 1000 steps, S(k)
    # every 10th statistics step) for the long-run statistics
    "long_cfg1": lambda: case_long_run(
        "long_cfg1", ((64, 32, 14.0, 50.0, 0.5, 0), ((32, 32, 32), (4.0, 4.0, 4.0)), (1000, 1000, 10, 1000000, 1)),
        101),
    # plain-FP64 configuration, CPU-runnable: 32^3, N=64, NA=32, XN=14, C=50,
    # dt=0.5, L=4, seeded Gaussian (sd 0.01) start; initial mix + 10 steps,
    # S(k) sampled every step
    "cfg1_32": lambda: case_config(
        "cfg1_32", ((64, 32, 14.0, 50.0, 0.5, 0), ((32, 32, 32), (4.0, 4.0, 4.0)), (1000, 1000, 10, 1000000, 1)),
        10, 7, field_seed=101, sample_every=1, sensitivity=True),
    # plain-FP64 B200 configuration: 64^3, N=64, NA=32, XN=16, C=100, dt=0.5,
    # L=6.4, (300) lamellar start; initial mix + 3 steps
    "cfg2_64": lambda: case_config(
        "cfg2_64", ((64, 32, 16.0, 100.0, 0.5, 0), ((64, 64, 64), (6.4, 6.4, 6.4)), (5000, 5000, 20, 1000000, 2)),
        3, 61, sample_every=1, sensitivity=True),
    # the mixed-precision B200 configuration at its own size: 128^3, N=64,
    # NA=25, XN=20, C=100, dt=0.5, L=8, seeded Gaussian (sd 0.01) start with
    # the bench's seed; initial mix + 1 step, S(k) sampled
    "cfg3_128": lambda: case_config(
        "cfg3_128", ((64, 25, 20.0, 100.0, 0.5, 0), ((128, 128, 128), (8.0, 8.0, 8.0)), (1, 1, 1, 1000000, 1)),
        1, 997, field_seed=2024, sample_every=1, sensitivity=True, threads=os.cpu_count()),
    # adjoint configuration: 64^3, N=64, NA=32, XN=15, C=50, L=6.0, lamellar;
    # the mixed start (phi) and H after one step
    "cfg4_64": lambda: case_config(
        "cfg4_64", ((64, 32, 15.0, 50.0, 0.5, 0), ((64, 64, 64), (6.0, 6.0, 6.0)), (10, 10, 1, 1000000, 2)),
        1, 61, sample_every=1, sensitivity=True),
}


def main(argv=None):
    names = list(argv if argv is not None else sys.argv[1:]) or list(CASES)
    unknown = [n for n in names if n not in CASES]
    if unknown:
        raise SystemExit(f"unknown cases {unknown}; known: {sorted(CASES)}")
    if not REF_TREE or not os.path.isdir(os.path.join(REF_TREE, "src")):
        raise SystemExit("LFTS_REFERENCE must name the reference project's tree")
    os.environ["REF"] = REF_TREE
    build_oracle(ref=True)
    if not RefHarness.available():
        raise SystemExit("oracle/_ref/libref_harness.so missing: the reference tree is needed")
    RefHarness.lib().ref_quiet(1)
    for n in names:
        CASES[n]()


if __name__ == "__main__":
    main()
