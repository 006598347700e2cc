"""lfts_cpu_b200 -- B200-native Langevin field-theoretic simulation step for AB
diblock copolymers (the hot path of tmbeardsley/lfts_cpu), behind a C ABI.

Python here is a thin host layer over ``liblfts_b200.so``:

* :class:`System` -- one GPU context: the reference's diblock + anderson +
  langevin + strFunc objects (``diblock::calc_concs``, ``anderson::mix``,
  ``langevin::step_wm``, ``strFunc::sample/save``, ``getH``).
* :class:`Rng` -- the reference's ``std::mt19937_64`` / ``normal_distribution``
  stream, for bit-identical noise.
* :func:`read_input` -- the reference's input-file header semantics.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .capi import (LFTS_ERR_NONFINITE, LFTS_ERR_NOTCONV, LFTS_ERR_SINGULAR, LFTS_FP32_MIXED, LFTS_FP64, LFTS_OK,
                   Input, LftsError, Params, Tiles, check, check_mix, lib)

__all__ = ["System", "Rng", "read_input", "LftsError", "LFTS_FP64", "LFTS_FP32_MIXED", "LFTS_OK",
           "LFTS_ERR_SINGULAR", "LFTS_ERR_NOTCONV", "LFTS_ERR_NONFINITE", "lib"]


def read_input(path: str) -> Input:
    """Parse an input file header like the reference's lfts_params."""
    inp = Input()
    check(lib().lfts_read_input(path.encode(), C.byref(inp)), "lfts_read_input")
    return inp


def z_inf_discrete(L, m, N, Nbar, tmax=100) -> float:
    return lib().lfts_z_inf_discrete((C.c_double * 3)(*L), (C.c_int * 3)(*m), int(N), float(Nbar), int(tmax))


def lamellar_field(amplitude, m, kx=3, ky=0, kz=0) -> np.ndarray:
    M = int(m[0]) * int(m[1]) * int(m[2])
    w = np.empty(2 * M)
    check(lib().lfts_lamellar_field(w, float(amplitude), (C.c_int * 3)(*m), kx, ky, kz), "lamellar")
    return w


class Rng:
    """std::mt19937_64(seed) feeding one normal_distribution(0, sigma)."""

    def __init__(self, seed: int = 123456789, sigma: float = 1.0):
        self._h = C.c_void_p()
        check(lib().lfts_rng_create(int(seed), float(sigma), C.byref(self._h)), "lfts_rng_create")

    def normal(self, n: int) -> np.ndarray:
        out = np.empty(int(n))
        check(lib().lfts_rng_normal(self._h, int(n), out), "lfts_rng_normal")
        return out

    def uniform(self, n: int) -> np.ndarray:
        out = np.empty(int(n))
        check(lib().lfts_rng_uniform(self._h, int(n), out), "lfts_rng_uniform")
        return out

    def random_field(self, XbN: float, M: int) -> np.ndarray:
        w = np.empty(2 * int(M))
        check(lib().lfts_random_field(self._h, w, float(XbN), int(M)), "lfts_random_field")
        return w

    def close(self):
        if self._h:
            lib().lfts_rng_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class System:
    """One simulated system on one GPU (an lfts_ctx)."""

    last_status = LFTS_OK  # status of the last mix / full step (LFTS_ERR_NOTCONV is not raised)

    def __init__(self, N: int, NA: int, XbN: float, C_: float, dt: float, m, L,
                 precision: int = LFTS_FP64, device: int = 0):
        p = Params()
        p.N, p.NA, p.XbN, p.C, p.dt = int(N), int(NA), float(XbN), float(C_), float(dt)
        for d in range(3):
            p.m[d] = int(m[d])
            p.L[d] = float(L[d])
        self.params = p
        self.N, self.NA = int(N), int(NA)
        self.m = tuple(int(x) for x in m)
        self.L = tuple(float(x) for x in L)
        self.M = self.m[0] * self.m[1] * self.m[2]
        self.Mk = self.m[0] * self.m[1] * (self.m[2] // 2 + 1)
        self.precision = precision
        self._h = C.c_void_p()
        check(lib().lfts_create(C.byref(p), int(precision), int(device), C.byref(self._h)), "lfts_create")

    @classmethod
    def from_input(cls, inp: Input, precision: int = LFTS_FP64, device: int = 0) -> "System":
        return cls(inp.N, inp.NA, inp.XbN, inp.C, inp.dt, list(inp.m), list(inp.L), precision, device)

    def close(self):
        if getattr(self, "_h", None):
            lib().lfts_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- fields --------------------------------------------------------------
    def set_fields(self, w2: np.ndarray) -> None:
        w2 = np.ascontiguousarray(w2[: 2 * self.M], dtype=np.float64)
        check(lib().lfts_set_fields(self._h, w2), "lfts_set_fields")

    def get_fields(self) -> np.ndarray:
        out = np.empty(4 * self.M)
        check(lib().lfts_get_fields(self._h, out), "lfts_get_fields")
        return out

    def fields_device_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().lfts_fields_device(self._h, C.byref(p)), "lfts_fields_device")
        return p.value

    # -- hot path ------------------------------------------------------------
    def calc_concs(self) -> float:
        v = C.c_double()
        check(lib().lfts_calc_concs(self._h, C.byref(v)), "lfts_calc_concs")
        return v.value

    def mix(self, max_iter: int = 200, tol: float = 1e-4, strict: bool = False) -> int:
        """anderson::mix; returns the reference's k.  A loop that stops at
        max_iter above tol sets ``last_status`` to LFTS_ERR_NOTCONV and raises
        only with ``strict``; a singular system or a non-finite residual raises."""
        k = C.c_int()
        self.last_status = check_mix(lib().lfts_anderson_mix(self._h, int(max_iter), float(tol), C.byref(k)),
                                     "lfts_anderson_mix", strict)
        return k.value

    def langevin_init(self, noise_prev: np.ndarray) -> None:
        check(lib().lfts_langevin_init(self._h, np.ascontiguousarray(noise_prev, np.float64)),
              "lfts_langevin_init")

    def langevin_step(self, noise_new: np.ndarray) -> None:
        check(lib().lfts_langevin_step(self._h, np.ascontiguousarray(noise_new, np.float64)),
              "lfts_langevin_step")

    def langevin_step_device(self, noise_ptr: int) -> None:
        check(lib().lfts_langevin_step_device(self._h, C.c_void_p(noise_ptr)), "lfts_langevin_step_device")

    def full_step_device(self, noise_ptr: int, max_iter: int = 200, tol: float = 1e-4, strict: bool = False):
        k = C.c_int()
        lnq = C.c_double()
        self.last_status = check_mix(lib().lfts_langevin_full_step(self._h, C.c_void_p(noise_ptr), int(max_iter),
                                                                   float(tol), C.byref(k), C.byref(lnq)),
                                     "lfts_langevin_full_step", strict)
        return k.value, lnq.value

    def sk_sample(self) -> None:
        check(lib().lfts_sk_sample(self._h), "lfts_sk_sample")

    def sk_get(self):
        S = np.empty(self.Mk)
        n = C.c_int()
        check(lib().lfts_sk_get(self._h, S, C.byref(n)), "lfts_sk_get")
        return S, n.value

    def sk_reset(self) -> None:
        check(lib().lfts_sk_reset(self._h), "lfts_sk_reset")

    def sk_bin(self, dK: float = 1e-5):
        K = np.empty(self.Mk)
        S = np.empty(self.Mk)
        n = C.c_int()
        check(lib().lfts_sk_bin(self._h, float(dK), K, S, C.byref(n)), "lfts_sk_bin")
        return K[: n.value].copy(), S[: n.value].copy()

    def get_H(self) -> float:
        v = C.c_double()
        check(lib().lfts_get_H(self._h, C.byref(v)), "lfts_get_H")
        return v.value

    def backward(self, ckpt_every: int = 0):
        """(dH/dL[3], dH/dXbN, H) for the current fields (FP64 contexts)."""
        dL = np.empty(3)
        dX = C.c_double()
        H = C.c_double()
        check(lib().lfts_backward(self._h, int(ckpt_every), dL, C.byref(dX), C.byref(H)), "lfts_backward")
        return dL, dX.value, H.value

    def step_fwd(self, q_in: np.ndarray, h: np.ndarray, i: int) -> np.ndarray:
        out = np.empty(2 * self.M)
        check(lib().lfts_step_fwd(self._h, np.ascontiguousarray(q_in, np.float64), out,
                                  np.ascontiguousarray(h, np.float64), int(i)), "lfts_step_fwd")
        return out

    def g_lookup(self) -> np.ndarray:
        out = np.empty(self.Mk)
        check(lib().lfts_g_lookup(self._h, out), "lfts_g_lookup")
        return out

    def propagators(self) -> np.ndarray:
        out = np.empty(2 * (self.N + 1) * self.M)
        check(lib().lfts_get_propagators(self._h, out), "lfts_get_propagators")
        return out.reshape(self.N + 1, 2, self.M)

    # -- bookkeeping -----------------------------------------------------------
    @property
    def stream(self) -> int:
        return lib().lfts_stream(self._h) or 0

    @property
    def kernel_launches(self) -> int:
        return int(lib().lfts_kernel_launches(self._h))

    def tuning(self):
        """(x-pencil columns per CTA, yz-plane transform stages per axis)"""
        a, b = C.c_int(), C.c_int()
        check(lib().lfts_tuning(self._h, C.byref(a), C.byref(b)), "lfts_tuning")
        return a.value, b.value

    def tiles(self) -> dict:
        """the contour chain's tile choice (lfts_tiles) as a dict"""
        t = Tiles()
        check(lib().lfts_get_tiles(self._h, C.byref(t)), "lfts_get_tiles")
        return t.as_dict()

    def set_tiles(self, pencil_cw: int, plane_stages: int, h_in_pencil: int = 0, two_streams: int = 0,
                  phi_in_chain: int = 0, plane_split: int = 1) -> None:
        t = Tiles(int(pencil_cw), int(plane_stages), int(h_in_pencil), int(two_streams), int(phi_in_chain),
                  int(plane_split))
        check(lib().lfts_set_tiles(self._h, C.byref(t)), "lfts_set_tiles")

    def profile_chain(self):
        """(ms per yz-plane step kernel, ms per x-pencil kernel, ms per chain)"""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib().lfts_profile_chain(self._h, C.byref(a), C.byref(b), C.byref(c)), "lfts_profile_chain")
        return a.value, b.value, c.value

    def profile_iteration(self, reps: int = 5):
        """(ms chain, ms concentrations + dot products, ms w+ update) of one
        Anderson iteration with a full history; fields unchanged"""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        check(lib().lfts_profile_iteration(self._h, int(reps), C.byref(a), C.byref(b), C.byref(c)),
              "lfts_profile_iteration")
        return a.value, b.value, c.value

    def anderson_stats(self):
        a, b = C.c_longlong(), C.c_longlong()
        check(lib().lfts_anderson_stats(self._h, C.byref(a), C.byref(b)), "lfts_anderson_stats")
        return a.value, b.value

    def device_bytes(self) -> int:
        v = C.c_size_t()
        check(lib().lfts_device_bytes(self._h, C.byref(v)), "lfts_device_bytes")
        return int(v.value)


def noise_philox(seed: int, step: int, n: int, sigma: float) -> np.ndarray:
    """sigma * N(0,1) deviates of points 0..n-1 of step `step` of Philox
    stream `seed` (the ensemble's noise), computed on the GPU."""
    out = np.empty(int(n))
    check(lib().lfts_noise_philox(int(seed), int(step), int(n), float(sigma), out), "lfts_noise_philox")
    return out


class Ensemble:
    """Independent FP32-mixed replicas advanced together (an lfts_ensemble).

    replicas: list of dicts with keys N, NA, XbN, C, dt, m, L and seed."""

    last_status = LFTS_OK  # most severe replica status of the last mix / run

    def __init__(self, replicas, device: int = 0):
        n = len(replicas)
        params = (Params * n)()
        seeds = (C.c_ulonglong * n)()
        self.M, self.m, self.sigma = [], [], []
        for r, d in enumerate(replicas):
            p = params[r]
            p.N, p.NA, p.XbN, p.C, p.dt = int(d["N"]), int(d["NA"]), float(d["XbN"]), float(d["C"]), float(d["dt"])
            for k in range(3):
                p.m[k] = int(d["m"][k])
                p.L[k] = float(d["L"][k])
            seeds[r] = int(d["seed"])
            M = int(np.prod(d["m"]))
            self.M.append(M)
            self.m.append(tuple(int(x) for x in d["m"]))
            V = float(np.prod(d["L"]))
            self.sigma.append(float(np.sqrt(2.0 * M * float(d["dt"]) / (float(d["C"]) * V))))
        self.nrep = n
        self.seeds = [int(d["seed"]) for d in replicas]
        self._h = C.c_void_p()
        check(lib().lfts_ensemble_create(C.cast(params, C.c_void_p), seeds, n, int(device), C.byref(self._h)),
              "lfts_ensemble_create")

    def close(self):
        if getattr(self, "_h", None):
            lib().lfts_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, r: int, w2: np.ndarray) -> None:
        w2 = np.ascontiguousarray(w2[: 2 * self.M[r]], dtype=np.float64)
        check(lib().lfts_ensemble_set_fields(self._h, int(r), w2), "lfts_ensemble_set_fields")

    def get_fields(self, r: int) -> np.ndarray:
        out = np.empty(4 * self.M[r])
        check(lib().lfts_ensemble_get_fields(self._h, int(r), out), "lfts_ensemble_get_fields")
        return out

    def mix(self, max_iter: int = 200, tol: float = 1e-4, strict: bool = False):
        """(K per replica, ln Q per replica); statuses as System.mix, per
        replica in replica_status()"""
        k = np.zeros(self.nrep, dtype=np.int32)
        lnq = np.zeros(self.nrep)
        self.last_status = check_mix(lib().lfts_ensemble_mix(self._h, int(max_iter), float(tol), k.ctypes.data,
                                                             lnq.ctypes.data), "lfts_ensemble_mix", strict)
        return k, lnq

    def run(self, nsteps: int, max_iter: int = 200, tol: float = 1e-4, record_k: bool = True,
            strict: bool = False):
        """(K[nsteps][nrep] or None, ln Q per replica after the last step)"""
        k = np.zeros((nsteps, self.nrep), dtype=np.int32) if record_k else None
        lnq = np.zeros(self.nrep)
        self.last_status = check_mix(lib().lfts_ensemble_run(self._h, int(nsteps), int(max_iter), float(tol),
                                                             k.ctypes.data if record_k else None, lnq.ctypes.data),
                                     "lfts_ensemble_run", strict)
        return k, lnq

    def replica_status(self, r: int) -> int:
        """lfts_status of replica r's last mix or run"""
        s = C.c_int()
        check(lib().lfts_ensemble_replica_status(self._h, int(r), C.byref(s)), "lfts_ensemble_replica_status")
        return s.value

    def tuning(self, r: int) -> int:
        cw = C.c_int()
        check(lib().lfts_ensemble_tuning(self._h, int(r), C.byref(cw)), "lfts_ensemble_tuning")
        return cw.value

    def tiles(self, r: int) -> dict:
        """replica r's tile choice (batched autotuning), as System.tiles()"""
        t = Tiles()
        check(lib().lfts_ensemble_tiles(self._h, int(r), C.byref(t)), "lfts_ensemble_tiles")
        return t.as_dict()

    def stream(self) -> int:
        return int(lib().lfts_ensemble_stream(self._h) or 0)

    def kernel_launches(self) -> int:
        return int(lib().lfts_ensemble_kernel_launches(self._h))
