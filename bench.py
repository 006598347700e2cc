"""Benchmark: Langevin steps/s of the L-FTS diblock step at 128^3, N=64.

Workload (the mixed-precision headline configuration): N=64, NA=25, XN=20
(bare), C=100, Ndt=0.5, mesh 128^3, L=8.0 R0, disordered start (W-, w+ i.i.d.
Gaussian, mean 0, sd 0.01, numpy seed 2024), Langevin noise from the
reference's generator (mt19937_64 seed 123456789, normal(0, sigma)).
One step = langevin::step_wm + anderson::mix (tol 1e-4, history 10) + the
extra calc_concs of the reference's loop.  The working set (propagators,
>1 GB) exceeds the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun every rank runs an independent replica (different seed) on its
own GPU ("replicas only": the step has no data-parallel split); value =
total steps of all ranks / max elapsed over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CFG = dict(N=64, NA=25, XN=20.0, C=100.0, dt=0.5, m=(128, 128, 128), L=(8.0, 8.0, 8.0), init_sd=0.01,
           field_seed=2024, noise_seed=123456789, max_iter=200, tol=1e-4)
METRIC = "Langevin steps/sec at 128^3, N=64 (FP32-mixed vs FP64 GPU at stated error); HBM GB/s"
HBM_FALLBACK = 6650.0


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (every 50 ms, time-stamped; samples outside [begin, end] are dropped)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.t_begin = self.t_end = None

    def start(self):
        """Start sampling; returns once the first sample is written (at most 5 s)."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None and os.path.getsize(self.path) == 0:
            time.sleep(0.02)

    def begin(self):
        self.t_begin = time.time()

    def end(self):
        self.t_end = time.time()

    @staticmethod
    def _stamp(text):
        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(text, fmt).timestamp()
            except ValueError:
                pass
        return None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                rows.append((self._stamp(f[0]), float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        os.unlink(self.path)
        if self.t_begin is not None and self.t_end is not None:
            inside = [r for r in rows if r[0] is not None and self.t_begin - 0.05 <= r[0] <= self.t_end + 0.05]
            if inside:
                rows = inside
                out["window"] = "timed region"
            else:
                out["window"] = "whole sampling (no sample inside the timed region)"
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {n for r in rows for n, v in zip(names, r[3]) if v.lower().startswith("active")}
        if rows:
            out.update(sm_mhz=statistics.median(r[1] for r in rows), sm_max_mhz=max(r[2] for r in rows),
                       reasons=sorted(reasons), samples=len(rows))
        return out


def make_initial_fields(M, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, CFG["init_sd"], 2 * M)


def _cpu_objects(threads):
    """The reference's classes at the bench configuration (oracle/_ref: the
    reference's own src/*.cc on the FFTW/GSL API shims, `threads` FFT
    threads), else the C oracle port; (diblock-like object, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    m, N, NA = CFG["m"], CFG["N"], CFG["NA"]
    if pyoracle.RefHarness.available():
        pyoracle.RefHarness.lib().ref_set_threads(threads)
        return pyoracle.RefSys(NA, N - NA, m, CFG["L"]), "reference"
    pyoracle.build_oracle()
    return pyoracle.Oracle(NA, N - NA, m, CFG["L"], threads=threads), "port"


def cpu_baseline_sample(K_mean, k_source):
    """Bounded CPU sample for the main line: one calc_concs of the reference
    at the bench configuration on all host threads (~2 s), projected to
    steps/s with the mean Anderson count K of the reference on this workload
    (K + 1 calc_concs per step).  The measured complete step is the
    reference arm's line (--impl reference)."""
    threads = os.cpu_count() or 1
    M = int(np.prod(CFG["m"]))
    w = np.zeros(4 * M)
    w[: 2 * M] = make_initial_fields(M, CFG["field_seed"])
    obj, kind = _cpu_objects(threads)
    t0 = time.perf_counter()
    obj.calc_concs(w)
    dt = time.perf_counter() - t0
    obj.close()
    return {"value": 1.0 / ((K_mean + 1.0) * dt), "unit": "steps/s", "cores": threads, "kind": kind,
            "sample": f"projection: one calc_concs at 128^3 N=64 ({dt:.2f} s, {threads} threads, the reference's "
                      f"code on a self-written FFT), steps/s = 1/((K+1) t) with {k_source} = {K_mean:.2f}; "
                      f"the measured complete step is the --impl reference line",
            "calc_concs_s": dt}


def reference_steps_measured(budget_s=100.0, max_steps=3):
    """Complete reference Langevin steps at the bench configuration, timed:
    the reference's own diblock / anderson / langevin objects (oracle/_ref)
    from the bench's start fields, with its langevin object on
    mt19937_64(noise seed) as in src/lfts_simulation.cc:23,36; the initial
    anderson::mix (untimed, src/lfts_simulation.cc:52), then the loop body of
    src/lfts_simulation.cc:69-76 -- step_wm, mix with the reference's own
    iteration count, the extra calc_concs -- timed step by step until
    budget_s is spent (at least one step, at most max_steps)."""
    threads = os.cpu_count() or 1
    m, N = CFG["m"], CFG["N"]
    M = int(np.prod(m))
    sigma = float(np.sqrt(2.0 * M * CFG["dt"] / (CFG["C"] * np.prod(CFG["L"]))))
    w = np.zeros(4 * M)
    w[: 2 * M] = make_initial_fields(M, CFG["field_seed"])
    obj, kind = _cpu_objects(threads)
    t0 = time.perf_counter()
    K0 = obj.mix(w)
    init_s = time.perf_counter() - t0
    times, Ks = [], []
    if kind == "reference":
        import pyoracle
        lg = pyoracle.RefLangevin(CFG["noise_seed"], sigma, M)
        step = lambda: lg.full_step(obj, w, CFG["XN"], CFG["dt"])[0]  # noqa: E731
    else:
        # the port (no reference build on this machine): the same loop body,
        # Gaussian noise of the same sigma from numpy
        rng = np.random.default_rng(CFG["noise_seed"])
        prev = [rng.normal(0.0, sigma, M)]

        def step():
            new = rng.normal(0.0, sigma, M)
            obj.langevin_update(w, prev[0], new, CFG["XN"], CFG["dt"])
            prev[0] = new
            k = obj.mix(w)
            obj.calc_concs(w)
            return k
    while len(times) < max_steps and (not times or sum(times) + times[-1] <= budget_s):
        t0 = time.perf_counter()
        Ks.append(int(step()))
        times.append(time.perf_counter() - t0)
    obj.close()
    s = float(np.mean(times))
    return {"kind": kind, "cores": threads, "s_per_step": s, "K": Ks, "steps_timed": len(times),
            "init_mix_K": int(K0), "init_mix_s": init_s,
            "sample": f"{len(times)} complete reference Langevin step(s) at 128^3 N=64 after the initial mix "
                      f"(step_wm, anderson::mix with its own K = {Ks}, the extra calc_concs), {threads} threads, "
                      f"the reference's code on a self-written FFT (FFTW is not in the image): {s:.1f} s per step"}


def scipy_fft_bound(K_mean, threads=None):
    """The best CPU FFT in the image (scipy.fft / pocketfft, all host
    threads) under a restatement of calc_concs (oracle/scipy_path.py): one
    calc_concs timed, projected to steps/s with K + 1 calc_concs per step.
    A bound on how much of the GPU/CPU ratio the reference's FFT accounts
    for -- not the reference."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from scipy_path import ScipyConcs
    threads = threads or os.cpu_count() or 1
    m, N, NA = CFG["m"], CFG["N"], CFG["NA"]
    M = int(np.prod(m))
    w = np.zeros(4 * M)
    w[: 2 * M] = make_initial_fields(M, CFG["field_seed"])
    sc = ScipyConcs(NA, N - NA, m, CFG["L"], workers=threads)
    sc.calc_concs(w.copy())  # warm (plans, pages)
    t0 = time.perf_counter()
    sc.calc_concs(w)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / ((K_mean + 1.0) * dt), "unit": "steps/s", "cores": threads, "calc_concs_s": dt,
            "kind": "best available CPU FFT (scipy.fft, pocketfft), not the reference",
            "sample": f"projection: one calc_concs ({dt:.2f} s) x (K+1) with K = {K_mean:.2f}"}


def run_precision(lfts, precision, steps, warmup, rank, device, torch, clocks=None, do_e2e=True):
    """Device-resident timing and the end-to-end (host-buffer API) timing."""
    m, N, NA = CFG["m"], CFG["N"], CFG["NA"]
    M = int(np.prod(m))
    inp_sigma = np.sqrt(2.0 * M * CFG["dt"] / (CFG["C"] * np.prod(CFG["L"])))
    s = lfts.System(N, NA, CFG["XN"], CFG["C"], CFG["dt"], m, CFG["L"], precision=precision, device=device)
    rng = lfts.Rng(CFG["noise_seed"] + rank, inp_sigma)
    eta0 = rng.normal(M)
    s.langevin_init(eta0)
    s.set_fields(make_initial_fields(M, CFG["field_seed"] + rank))
    s.mix(CFG["max_iter"], CFG["tol"])
    nsteps_dev = warmup + steps
    noise = torch.empty((nsteps_dev, M), dtype=torch.float64, pin_memory=True)
    for i in range(nsteps_dev):
        noise[i].numpy()[:] = rng.normal(M)
    noise_dev = noise.to(f"cuda:{device}")
    torch.cuda.synchronize(device)
    stream = torch.cuda.ExternalStream(s.stream, device=f"cuda:{device}")
    Ks = []
    for i in range(warmup):
        k, _ = s.full_step_device(noise_dev[i].data_ptr(), CFG["max_iter"], CFG["tol"])
    # the state the timed steps start from, replayed by the end-to-end timing
    snap = s.get_fields()[: 2 * M].copy() if do_e2e else None
    barrier(torch)
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = s.kernel_launches
    mix0 = s.anderson_stats()
    if clocks:
        clocks.start()
        clocks.begin()
    ev0.record(stream)
    for i in range(warmup, nsteps_dev):
        k, _ = s.full_step_device(noise_dev[i].data_ptr(), CFG["max_iter"], CFG["tol"])
        Ks.append(k - 1)  # mix returns iterations + 1
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize(device)
    if clocks:
        clocks.end()
    clk = clocks.stop() if clocks else None
    ms = ev0.elapsed_time(ev1) / steps
    launches = s.kernel_launches - launches0
    mix1 = s.anderson_stats()
    iters = mix1[1] - mix0[1]
    res = {"ms_per_step": ms, "launches": launches, "iters": iters, "K": Ks, "clocks": clk,
           "calc_concs_per_step": iters / steps + 1.0}
    del noise_dev
    # End to end through the C ABI with host (pinned) noise buffers: after
    # warm-up steps of its own, the context is put back into the state the
    # device-resident timing started from (fields, previous noise, phi) and the
    # same K steps are replayed from the same noise rows, now read from host
    # memory.  The arithmetic is the same, so the Anderson counts repeat and
    # the two timings differ only by the host-buffer API's transfers and syncs.
    if do_e2e:
        host = torch.empty((warmup, M), dtype=torch.float64, pin_memory=True)
        for i in range(warmup):
            host[i].numpy()[:] = rng.normal(M)
        for i in range(warmup):
            s.langevin_step(host[i].numpy())
            s.mix(CFG["max_iter"], CFG["tol"])
            s.calc_concs()
        s.set_fields(snap)
        s.langevin_init(noise[warmup - 1].numpy() if warmup > 0 else eta0)
        s.calc_concs()
        barrier(torch)
        torch.cuda.synchronize(device)
        mix0 = s.anderson_stats()
        Ks_e2e = []
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(warmup, warmup + steps):
            s.langevin_step(noise[i].numpy())
            Ks_e2e.append(s.mix(CFG["max_iter"], CFG["tol"]) - 1)
            s.calc_concs()
        e1.record(stream)
        e1.synchronize()
        mix1 = s.anderson_stats()
        it_e2e = mix1[1] - mix0[1]
        res["e2e_ms_per_step"] = e0.elapsed_time(e1) / steps
        res["e2e_same_K"] = Ks_e2e == Ks
        res["h2d_bytes_per_step"] = 8 * M
        # per Anderson iteration S1 and <Dh0,Dh_m> (<= 11 doubles), plus Q and ln Q
        res["d2h_bytes_per_step"] = int(round((it_e2e / steps) * 8 * 11 + 16))
    res["profile"] = s.profile_chain()
    res["system"] = s
    return res


def time_calc_concs(s, torch, device, reps=5):
    """Mean ms of one calc_concs (contour chain, Q, concentrations) on the
    context's current fields: CUDA events on the context's stream around the
    C-ABI call, after one warm call."""
    stream = torch.cuda.ExternalStream(s.stream, device=f"cuda:{device}")
    s.calc_concs()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(reps):
        s.calc_concs()
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1) / reps


def ensemble_config(seed=2024, nrep=32):
    """The batched configuration: nrep replicas, meshes drawn from seed among
    32^3, 48^3, 64^3, 96^3, L = mesh/16, N=64, NA in [16,48], XN in [12,20],
    C=50, Ndt=0.5, separate Philox streams, disordered start (sd 0.01)."""
    rng = np.random.default_rng(seed)
    meshes = rng.choice([32, 48, 64, 96], size=nrep)
    reps = [dict(N=64, NA=int(rng.integers(16, 49)), XbN=float(rng.uniform(12.0, 20.0)), C=50.0, dt=0.5,
                 m=(int(mm),) * 3, L=(mm / 16.0,) * 3, seed=1000 + r) for r, mm in enumerate(meshes)]
    fields = [rng.normal(0.0, 0.01, 2 * int(mm) ** 3) for mm in meshes]
    return reps, fields


def ensemble_bench(lfts, torch, device, steps=5, warmup=3):
    """Replica-steps/s of the batched configuration: one graph launch per
    Langevin step of all replicas, CUDA events on the ensemble's stream."""
    reps, fields = ensemble_config()
    e = lfts.Ensemble(reps, device=device)
    for r, w2 in enumerate(fields):
        e.set_fields(r, w2)
    e.mix(CFG["max_iter"], CFG["tol"])
    ks, _ = e.run(warmup, CFG["max_iter"], CFG["tol"], record_k=True)
    stream = torch.cuda.ExternalStream(e.stream(), device=f"cuda:{device}")
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    ks, _ = e.run(steps, CFG["max_iter"], CFG["tol"], record_k=True)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    K = ks.astype(float) - 1.0  # mix returns iterations + 1
    N = reps[0]["N"]
    point_steps = sum(float(np.prod(d["m"])) * (N - 1) * (K[:, r].mean() + 1.0) for r, d in enumerate(reps))
    # algorithmic bytes of the timed steps, replica by replica, with the
    # single-context formula: (K+1) W_cc + K W_am + 7M, FP32-mixed word sizes
    alg = 0.0
    for r, d in enumerate(reps):
        M = float(np.prod(d["m"]))
        Kr = float(K[:, r].mean())
        alg += (Kr + 1.0) * (7 * d["N"] * M * 4 + 6 * M * 8) + Kr * (3 * 10 + 7) * M * 8 + 7 * M * 8
    peak, peak_kind = measured_peak()
    achieved = alg / (ms * 1e-3) / 1e9
    seq_ms = sequential_single_contexts(lfts, torch, device, reps, fields)
    out = {"replicas": len(reps), "meshes": {str(mm): int(sum(1 for d in reps if d["m"][0] == mm))
                                             for mm in (32, 48, 64, 96)},
           "ms_per_step": ms, "replica_steps_per_s": len(reps) * 1e3 / ms,
           "mean_anderson_K": float(K.mean()),
           "mesh_point_contour_steps_per_s": point_steps * 1e3 / ms,
           "tiles": {str(d["m"][0]): e.tiles(r) for r, d in enumerate(reps)},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_kind": peak_kind, "algorithmic_bytes_per_step": alg,
                        "unit_of_work": "one Langevin step of every replica, sum over replicas of (K+1) W_cc + "
                                        "K W_am + 7M with each replica's own M, N and K"},
           "timing": f"{steps} steps after {warmup} warm-up steps, the timed steps as one CUDA graph launch",
           "sequential_single_contexts_ms_per_step": seq_ms,
           "speedup_vs_sequential_single_contexts": seq_ms / ms}
    e.close()
    return out


def sequential_single_contexts(lfts, torch, device, reps, fields):
    """The same replicas one after another as single FP32-mixed contexts: sum
    over replicas of one Langevin step (after the mix and two warm-up
    steps), CUDA events on each context's stream, same Philox noise."""
    total = 0.0
    for d, w2 in zip(reps, fields):
        M = int(np.prod(d["m"]))
        sigma = float(np.sqrt(2.0 * M * d["dt"] / (d["C"] * np.prod(d["L"]))))
        s = lfts.System(d["N"], d["NA"], d["XbN"], d["C"], d["dt"], d["m"], d["L"],
                        precision=lfts.LFTS_FP32_MIXED, device=device)
        s.set_fields(w2)
        s.mix(CFG["max_iter"], CFG["tol"])
        s.calc_concs()
        s.langevin_init(lfts.noise_philox(d["seed"], 0, M, sigma))
        noise = torch.from_numpy(np.stack([lfts.noise_philox(d["seed"], st, M, sigma) for st in (1, 2, 3)]))
        noise = noise.to(f"cuda:{device}")
        stream = torch.cuda.ExternalStream(s.stream, device=f"cuda:{device}")
        for i in range(2):
            s.full_step_device(noise[i].data_ptr(), CFG["max_iter"], CFG["tol"])
        torch.cuda.synchronize(device)
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.full_step_device(noise[2].data_ptr(), CFG["max_iter"], CFG["tol"])
        ev1.record(stream)
        ev1.synchronize()
        total += ev0.elapsed_time(ev1)
        del noise
        s.close()
    return total


def barrier(torch):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(torch, v, device):
    """Max of v over the ranks (device None: a host tensor, for gloo)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        t = torch.tensor([v], dtype=torch.float64, device="cpu" if device is None else f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return v


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def fp32_mixed_errors(lfts, device, nsteps=3):
    """FP32-mixed against FP64 on the bench workload for each output of the
    path (phi, H, S(k)):
      per_call   -- both precisions on the same fields (the FP64 context's
                    state after the run below): phi (max relative), ln Q and H
                    (absolute and relative);
      trajectory -- each precision from the same start with the same noise
                    (the reference's stream) for nsteps Langevin steps, each
                    with its own Anderson iterations, S(k) sampled every step:
                    phi and W- (max relative), H, the binned S(k) (max
                    difference over bins relative to the largest bin), and
                    both K sequences."""
    m, N, NA = CFG["m"], CFG["N"], CFG["NA"]
    M = int(np.prod(m))
    sigma = float(np.sqrt(2.0 * M * CFG["dt"] / (CFG["C"] * np.prod(CFG["L"]))))
    rng = lfts.Rng(CFG["noise_seed"], sigma)
    eta = [rng.normal(M) for _ in range(nsteps + 1)]
    w_start = make_initial_fields(M, CFG["field_seed"])
    run = {}
    for prec in (lfts.LFTS_FP64, lfts.LFTS_FP32_MIXED):
        s = lfts.System(N, NA, CFG["XN"], CFG["C"], CFG["dt"], m, CFG["L"], precision=prec, device=device)
        s.langevin_init(eta[0])
        s.set_fields(w_start)
        s.mix(CFG["max_iter"], CFG["tol"])
        Ks = []
        for st in range(1, nsteps + 1):
            s.langevin_step(eta[st])
            Ks.append(s.mix(CFG["max_iter"], CFG["tol"]) - 1)
            s.calc_concs()
            s.sk_sample()
        H = s.get_H()
        _, Sb = s.sk_bin(1e-5)
        run[prec] = dict(s=s, K=Ks, H=H, w=s.get_fields(), Sb=Sb)
    a, b = run[lfts.LFTS_FP32_MIXED], run[lfts.LFTS_FP64]
    traj = {"steps": nsteps, "K_fp64": b["K"], "K_fp32_mixed": a["K"],
            "phi_rel": _rel(a["w"][2 * M:], b["w"][2 * M:]), "wminus_rel": _rel(a["w"][:M], b["w"][:M]),
            "H_abs": abs(a["H"] - b["H"]), "H_rel": abs(a["H"] - b["H"]) / abs(b["H"]),
            "Sk_binned_rel": _rel(a["Sb"], b["Sb"]), "Sk_bins": int(len(b["Sb"]))}
    s32, s64 = a["s"], b["s"]
    w2 = b["w"][: 2 * M].copy()
    s32.set_fields(w2)
    lnq32 = s32.calc_concs()
    phi32 = s32.get_fields()[2 * M:]
    lnq64 = s64.calc_concs()
    phi64 = s64.get_fields()[2 * M:]
    H32, H64 = s32.get_H(), s64.get_H()
    per_call = {"phi_rel": _rel(phi32, phi64), "lnQ_abs": abs(lnq32 - lnq64), "H_abs": abs(H32 - H64),
                "H_rel": abs(H32 - H64) / abs(H64),
                "fields": "the FP64 trajectory's state after its last step, given to both precisions"}
    s32.close()
    s64.close()
    return {"per_call": per_call, "trajectory": traj,
            "note": "S(k) is sampled in FP64 in both precisions, so its error is the W- trajectory's"}


def reference_arm(args, rank, world):
    """The reference's own CPU implementation of the path on this host's
    cores (oracle/_ref, else the C oracle port): complete Langevin steps at
    the bench configuration, timed one by one after the initial mix (the
    warm-up), as many as fit a ~100 s budget (at least one; --steps caps
    them); plus, labelled, the one-calc_concs projection and its error, and
    the scipy.fft bound."""
    if rank != 0:
        return 0
    meas = reference_steps_measured(max_steps=max(1, args.steps))
    v = 1.0 / meas["s_per_step"]
    iters = float(np.mean(meas["K"])) - 1.0  # anderson::mix returns iterations + 1
    proj = cpu_baseline_sample(iters, "the measured steps' mean Anderson iteration count")
    proj_s = 1.0 / proj["value"]
    extra = {"projection_from_one_calc_concs": {"s_per_step": proj_s, "calc_concs_s": proj["calc_concs_s"],
                                                "measured_over_projected": meas["s_per_step"] / proj_s}}
    try:
        extra["scipy_fft_bound"] = scipy_fft_bound(iters)
    except Exception as e:  # reported, not fatal
        extra["scipy_fft_bound"] = {"failed": str(e)}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": meas["steps_timed"], "steps_requested": args.steps,
            "warmup": f"the initial anderson::mix ({meas['init_mix_K'] - 1} iterations, {meas['init_mix_s']:.1f} s)",
            "ms_per_step": 1e3 * meas["s_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
            "reference_K": meas["K"], "mean_anderson_K": iters,
            "cpu_baseline": {"kind": meas["kind"], "cores": meas["cores"], "sample": meas["sample"], "value": v,
                             "unit": "steps/s"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line.update(extra)
    print(json.dumps(line), flush=True)
    return 0


def workload_config():
    return {"workload": "L-FTS diblock Langevin step, 128^3 mesh, N=64 (NA=25), XN=20, C=100, Ndt=0.5, "
                        "L=8 R0, disordered start (sd 0.01), reference noise stream",
            "mesh": list(CFG["m"]), "N": CFG["N"], "NA": CFG["NA"], "XN": CFG["XN"], "C": CFG["C"],
            "dt": CFG["dt"], "L": list(CFG["L"]), "anderson_tol": CFG["tol"], "anderson_history": 10,
            "parallelism": "replicas", "l2": "working set > L2 (propagators >1 GB), no flush"}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    args = ap.parse_args(argv)
    rank, world, local = dist_env()
    if args.impl == "reference":
        return reference_arm(args, rank, world)

    import torch
    import lfts_cpu_b200 as lfts
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device(f"cuda:{local}"))
    device = local
    torch.cuda.set_device(device)
    lfts.lib()

    clocks = ClockSampler(device) if rank == 0 else None
    fp32 = run_precision(lfts, lfts.LFTS_FP32_MIXED, args.steps, args.warmup, rank, device, torch, clocks)
    fp32_sys = fp32.pop("system")
    ms32 = max_over_ranks(torch, fp32["ms_per_step"], device)
    e2e32 = max_over_ranks(torch, fp32["e2e_ms_per_step"], device)
    # per-step split of the FP32-mixed step: each part of an Anderson
    # iteration timed on its own (CUDA events, full history), times the
    # counts per step; the rest is host round trips, launch gaps and the
    # once-per-step kernels
    part_chain, part_conc, part_upd = fp32_sys.profile_iteration(5)
    tiles32 = fp32_sys.tiles()
    ms_calc = time_calc_concs(fp32_sys, torch, device)
    # the yz-plane kernel split over a thread-block cluster (tile plane_split)
    # against the tuned choice: chain of one calc_concs, CUDA events
    split_alt = None
    alt = dict(tiles32, plane_split=8 if tiles32.get("plane_split", 1) == 1 else 1)
    try:
        fp32_sys.set_tiles(**alt)
        ms_alt = min(fp32_sys.profile_iteration(3)[0] for _ in range(2))
        fp32_sys.set_tiles(**tiles32)
        ms_tuned = min(fp32_sys.profile_iteration(3)[0] for _ in range(2))
        split_alt = {"tuned_plane_split": tiles32["plane_split"],
                     "chain_ms": {str(tiles32["plane_split"]): ms_tuned, str(alt["plane_split"]): ms_alt},
                     "note": "contour chain of one calc_concs with one CTA per 128x128 x-plane (1) or the plane "
                             "spread over an 8-CTA cluster (8); results bitwise equal"}
    except lfts.LftsError:
        fp32_sys.set_tiles(**tiles32)
    # the contour step of a chain that stores every slot (the tuned chain may
    # form the concentration sums in its second half instead)
    ch_storing = None
    if tiles32.get("phi_in_chain"):
        fp32_sys.set_tiles(**dict(tiles32, phi_in_chain=0))
        ch_storing = min(fp32_sys.profile_chain()[2] for _ in range(3))
        fp32_sys.set_tiles(**tiles32)
    fp32_sys.close()
    fp64 = run_precision(lfts, lfts.LFTS_FP64, args.steps, args.warmup, rank, device, torch, None)
    fp64_sys = fp64.pop("system")
    tiles64 = fp64_sys.tiles()
    ms_calc64 = time_calc_concs(fp64_sys, torch, device)
    fp64_sys.close()
    ms64 = max_over_ranks(torch, fp64["ms_per_step"], device)
    e2e64 = max_over_ranks(torch, fp64["e2e_ms_per_step"], device)

    if rank == 0:
        m = CFG["m"]
        M = int(np.prod(m))
        N = CFG["N"]
        peak, peak_kind = measured_peak()
        pl, pe, ch = fp32["profile"]
        # algorithmic bytes of one contour step, both chains: read q, read h,
        # write q (3M words per chain), propagator words FP32; time = the
        # production chain's duration / (N-1) steps (CUDA events on its stream)
        step_bytes = 6 * M * 4
        step_ms = ch / (N - 1)
        achieved = step_bytes / (step_ms * 1e-3) / 1e9
        # whole Langevin step, algorithmic words: (K+1) W_cc + K W_am + 7M
        K_mean = float(np.mean(fp32["K"]))
        W_cc_bytes = 7 * N * M * 4 + 6 * M * 8  # propagator words FP32, field words FP64
        W_am_bytes = (3 * 10 + 7) * M * 8
        step_alg = (K_mean + 1) * W_cc_bytes + K_mean * W_am_bytes + 7 * M * 8
        value = world * 1e3 / ms32
        errs = fp32_mixed_errors(lfts, device)
        cc_per_step = fp32["calc_concs_per_step"]
        split = {"chain": cc_per_step * part_chain, "concentrations_and_dots": cc_per_step * part_conc,
                 "anderson_update": (cc_per_step - 1.0) * part_upd}
        split["other"] = ms32 - sum(split.values())
        split_info = {"ms_per_step": split, "ms_per_part": {"chain": part_chain, "concentrations_and_dots": part_conc,
                                                           "anderson_update": part_upd},
                      "calc_concs_per_step": cc_per_step,
                      "other": "host round trips of the Anderson loop, launch gaps, Langevin update"}
        K64 = float(np.mean(fp64["K"]))
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                cpu = cpu_baseline_sample(K64, "the FP64 path's mean Anderson iteration count on these steps, "
                                               "which is the reference's (same start and noise)")
                cpu.pop("calc_concs_s", None)
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
                       "sample": f"failed: {e}"}
        ens = None
        if not args.no_ensemble and world == 1:
            try:
                ens = ensemble_bench(lfts, torch, device)
            except Exception as e:  # reported, not fatal
                ens = {"failed": str(e)}
        traffic = None
        traffic_cc = None
        traffic64 = None
        tp = os.path.join(ROOT, "profiles", "contour_step_traffic.json")
        if os.path.exists(tp):
            tj = json.load(open(tp))
            traffic = tj.get("bytes_per_step_fp32_128")
            traffic_cc = tj.get("bytes_per_calc_concs_fp32_128", {}).get("phi_in_chain" if tiles32.get(
                "phi_in_chain") else "separate_pass")
            traffic64 = tj.get("bytes_per_calc_concs_fp64_128")
        # the roofline unit: one calc_concs (the contour chain, Q
        # and the concentrations), algorithmic bytes W_cc = 7 N M propagator
        # words (FP32) + 6 M field words (FP64): read q, read h, write q per
        # chain step, the N stored propagators read back for phi, w in, h and
        # phi out -- wherever the work happens (with phi_in_chain the stored
        # propagators are read inside the chain instead of by a later pass)
        achieved_cc = W_cc_bytes / (ms_calc * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32-mixed (f32 FFT/propagators, f64 Q/log/Anderson/H/fields)",
            "data": "synthetic", "config": workload_config(),
            "e2e": {"value": world * 1e3 / e2e32, "unit": "steps/s",
                    "h2d_bytes_per_step": fp32["h2d_bytes_per_step"],
                    "d2h_bytes_per_step": fp32["d2h_bytes_per_step"],
                    "steps": "the timed steps replayed from the same state and noise, noise read from pinned host memory",
                    "same_anderson_K": fp32["e2e_same_K"]},
            "roofline": {"bound": "hbm", "kernel": "calc_concs: contour chain (yz-plane + x-pencil kernels, both "
                                                   "chains, FP32) + Q + concentrations, one graph replay",
                         "achieved": achieved_cc, "peak": peak, "unit": "GB/s", "frac": achieved_cc / peak,
                         "peak_kind": peak_kind, "traffic": traffic_cc,
                         "algorithmic_bytes_per_launch": W_cc_bytes, "ms_per_launch": ms_calc,
                         "unit_of_work": "one calc_concs, W_cc = 7 N M propagator words (4 B) + 6 M field words (8 B)"},
            "roofline_contour_step": {"bound": "hbm", "kernel": "one contour step (yz-plane + x-pencil kernels)",
                                      "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                                      "peak_kind": peak_kind, "traffic": traffic,
                                      "algorithmic_bytes_per_launch": step_bytes, "ms_per_step": step_ms,
                                      "ms_plane_alone": pl, "ms_pencil_alone": pe,
                                      "storing_chain": None if ch_storing is None else {
                                          "ms_per_step": ch_storing / (N - 1),
                                          "achieved": step_bytes / (ch_storing / (N - 1) * 1e-3) / 1e9,
                                          "frac": step_bytes / (ch_storing / (N - 1) * 1e-3) / 1e9 / peak},
                                      "note": "with phi_in_chain the second half of the steps also reads the "
                                              "partner slots and adds the concentration sums (not in these bytes); "
                                              "storing_chain: the same step in a chain that stores every slot"},
            "cpu_baseline": cpu,
            "clocks": fp32["clocks"],
            "gpu_launches": fp32["launches"],
            "mean_anderson_K": K_mean,
            "calc_concs_per_s": fp32["calc_concs_per_step"] * 1e3 / ms32,
            "mesh_point_contour_steps_per_s": fp32["calc_concs_per_step"] * M * (N - 1) * 1e3 / ms32,
            "hbm_gbs_algorithmic_step": step_alg / (ms32 * 1e-3) / 1e9,
            "step_split": split_info,
            "tiles": tiles32,
            "plane_split_alternative": split_alt,
            "fp64": {"value": world * 1e3 / ms64, "ms_per_step": ms64, "mean_anderson_K": K64,
                     "e2e": {"value": world * 1e3 / e2e64, "unit": "steps/s",
                             "h2d_bytes_per_step": fp64["h2d_bytes_per_step"],
                             "d2h_bytes_per_step": fp64["d2h_bytes_per_step"],
                             "same_anderson_K": fp64["e2e_same_K"]},
                     "ms_plane": fp64["profile"][0], "ms_pencil": fp64["profile"][1], "tiles": tiles64,
                     "roofline": {"bound": "hbm", "kernel": "calc_concs, FP64", "unit": "GB/s", "peak": peak,
                                  "peak_kind": peak_kind, "ms_per_launch": ms_calc64, "traffic": traffic64,
                                  "algorithmic_bytes_per_launch": 7 * N * M * 8 + 6 * M * 8,
                                  "achieved": (7 * N * M * 8 + 6 * M * 8) / (ms_calc64 * 1e-3) / 1e9,
                                  "frac": (7 * N * M * 8 + 6 * M * 8) / (ms_calc64 * 1e-3) / 1e9 / peak,
                                  "unit_of_work": "one calc_concs, W_cc = 7 N M + 6 M words, all FP64"},
                     "calc_concs_per_s": fp64["calc_concs_per_step"] * 1e3 / ms64},
            "speedup_fp32_mixed_vs_fp64": ms64 / ms32,
            "fp32_err_vs_fp64": errs,
            "fp32_phi_rel_err_vs_fp64": errs["per_call"]["phi_rel"],
            "fp32_lnQ_abs_err_vs_fp64": errs["per_call"]["lnQ_abs"],
            "ensemble": ens,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
