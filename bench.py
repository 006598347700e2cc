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


# mean Anderson count of this workload (its FP64 path reproduces the
# reference's iteration counts): the reference arm's steps/s projection
REFERENCE_K = 31.0


def cpu_baseline_sample(K_mean, k_source="the GPU run's mean Anderson K"):
    """The reference's own calc_concs (oracle/_ref: the reference sources on
    the FFTW/GSL API shims; else the C oracle port) at the bench configuration,
    all host threads, projected to steps/s with the GPU run's mean K."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    threads = os.cpu_count() or 1
    m, N, NA = CFG["m"], CFG["N"], CFG["NA"]
    M = int(np.prod(m))
    w = np.zeros(4 * M)
    w[: 2 * M] = make_initial_fields(M, CFG["field_seed"])
    if pyoracle.RefHarness.available():
        pyoracle.RefHarness.lib().ref_set_threads(threads)
        obj, kind = pyoracle.RefSys(NA, N - NA, m, CFG["L"]), "reference"
    else:
        pyoracle.build_oracle()
        obj, kind = pyoracle.Oracle(NA, N - NA, m, CFG["L"], threads=threads), "port"
    t0 = time.perf_counter()
    obj.calc_concs(w)
    dt = time.perf_counter() - t0
    steps_per_s = 1.0 / ((K_mean + 1.0) * dt)
    return {"value": steps_per_s, "unit": "steps/s", "cores": threads, "kind": kind,
            "sample": f"one calc_concs at 128^3 N=64 ({dt:.2f} s, {threads} threads, shim FFT); "
                      f"steps/s = 1/((K+1) t) with {k_source} = {K_mean:.2f}",
            "calc_concs_s": dt}


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
    e.run(steps, CFG["max_iter"], CFG["tol"], record_k=False)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    K = ks.astype(float) - 1.0  # mix returns iterations + 1
    N = reps[0]["N"]
    point_steps = sum(float(np.prod(d["m"])) * (N - 1) * (K[:, r].mean() + 1.0) for r, d in enumerate(reps))
    seq_ms = sequential_single_contexts(lfts, torch, device, reps, fields)
    out = {"replicas": len(reps), "meshes": {str(mm): int(sum(1 for d in reps if d["m"][0] == mm))
                                             for mm in (32, 48, 64, 96)},
           "ms_per_step": ms, "replica_steps_per_s": len(reps) * 1e3 / ms,
           "mean_anderson_K": float(K.mean()),
           "mesh_point_contour_steps_per_s": point_steps * 1e3 / ms,
           "pencil_cw": {str(d["m"][0]): e.tuning(r) for r, d in enumerate(reps)},
           "timing": f"{steps} steps after {warmup} warm-up steps, one CUDA graph launch per step",
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


def phi_error_fp32_vs_fp64(lfts, device):
    m, N, NA = CFG["m"], CFG["N"], CFG["NA"]
    M = int(np.prod(m))
    w2 = make_initial_fields(M, 7) * 50.0  # a rougher field than the start
    out = []
    for prec in (0, 1):
        s = lfts.System(N, NA, CFG["XN"], CFG["C"], CFG["dt"], m, CFG["L"], precision=prec, device=device)
        s.set_fields(w2)
        lnq = s.calc_concs()
        out.append((lnq, s.get_fields()[2 * M:]))
        s.close()
    err = float(np.max(np.abs(out[1][1] - out[0][1])) / np.max(np.abs(out[0][1])))
    return err, abs(out[1][0] - out[0][0])


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    K_mean = float(os.environ.get("LFTS_BENCH_K", str(REFERENCE_K)))
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = cpu_baseline_sample(K_mean, "this workload's mean Anderson K (FP64 GPU run, reference counts)")
        if i >= args.warmup:
            vals.append(info["value"])
    v = float(np.mean(vals)) if vals else info["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(), "cpu_baseline": {k: info[k] for k in ("kind", "cores", "sample")} | {
                "value": v, "unit": "steps/s"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    fp32_sys.close()
    fp64 = run_precision(lfts, lfts.LFTS_FP64, args.steps, args.warmup, rank, device, torch, None, do_e2e=False)
    fp64.pop("system").close()
    ms64 = max_over_ranks(torch, fp64["ms_per_step"], device)

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
        err_phi, err_lnq = phi_error_fp32_vs_fp64(lfts, device)
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            try:
                cpu = cpu_baseline_sample(K_mean)
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
        tp = os.path.join(ROOT, "profiles", "contour_step_traffic.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get("bytes_per_step_fp32_128")
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
            "roofline": {"bound": "hbm", "kernel": "contour step (yz-plane + x-pencil kernels, both chains, FP32)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": step_bytes, "ms_per_step": step_ms,
                         "ms_plane_alone": pl, "ms_pencil_alone": pe},
            "cpu_baseline": cpu,
            "clocks": fp32["clocks"],
            "gpu_launches": fp32["launches"],
            "mean_anderson_K": K_mean,
            "calc_concs_per_s": fp32["calc_concs_per_step"] * 1e3 / ms32,
            "mesh_point_contour_steps_per_s": fp32["calc_concs_per_step"] * M * (N - 1) * 1e3 / ms32,
            "hbm_gbs_algorithmic_step": step_alg / (ms32 * 1e-3) / 1e9,
            "fp64": {"value": world * 1e3 / ms64, "ms_per_step": ms64, "mean_anderson_K": float(np.mean(fp64["K"])),
                     "ms_plane": fp64["profile"][0], "ms_pencil": fp64["profile"][1],
                     "calc_concs_per_s": fp64["calc_concs_per_step"] * 1e3 / ms64},
            "speedup_fp32_mixed_vs_fp64": ms64 / ms32,
            "fp32_phi_rel_err_vs_fp64": err_phi, "fp32_lnQ_abs_err_vs_fp64": err_lnq,
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
