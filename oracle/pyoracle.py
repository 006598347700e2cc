"""TEST INFRASTRUCTURE ONLY -- ctypes bindings for the CPU oracle.

Imported only by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py``, as the oracle.  The product package never imports it.

* :class:`Oracle` wraps ``oracle/liblfts_oracle.so`` -- the plain-C restatement
  of the reference's hot path (``lfts_oracle.c``).
* :class:`RefHarness` wraps ``oracle/_ref/libref_harness.so`` -- the reference's
  own sources compiled against the FFTW/GSL API shims (built only where the
  reference tree is present; absent on machines without it).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liblfts_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_harness.so")
REF_BIN = os.path.join(HERE, "_ref", "lfts-ref")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build_oracle(ref: bool = False) -> None:
    """Compile the oracle (and, when ``ref`` and the reference tree exist, oracle/_ref)."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


class Oracle:
    """The C restatement.  One instance per (NA, NB, mesh, box)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build_oracle()
            lib = C.CDLL(ORACLE_SO)
            lib.orc_create.restype = C.c_void_p
            lib.orc_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
            lib.orc_destroy.argtypes = [C.c_void_p]
            lib.orc_set_threads.argtypes = [C.c_int]
            lib.orc_g_lookup.argtypes = [C.c_void_p, _dp]
            lib.orc_step_fwd.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int]
            lib.orc_calc_concs.restype = C.c_double
            lib.orc_calc_concs.argtypes = [C.c_void_p, _dp]
            lib.orc_propagators.restype = C.POINTER(C.c_double)
            lib.orc_propagators.argtypes = [C.c_void_p]
            lib.orc_anderson_create.restype = C.c_void_p
            lib.orc_anderson_create.argtypes = [C.c_int, C.c_int]
            lib.orc_anderson_destroy.argtypes = [C.c_void_p]
            lib.orc_anderson_mix.restype = C.c_int
            lib.orc_anderson_mix.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, _dp]
            lib.orc_langevin_update.argtypes = [_dp, _dp, _dp, C.c_double, C.c_double, C.c_int]
            lib.orc_sk_sample.argtypes = [C.c_void_p, _dp, _dp]
            lib.orc_sk_bin.restype = C.c_int
            lib.orc_sk_bin.argtypes = [C.c_void_p, C.c_void_p, _dp, C.c_int, C.c_double,
                                       C.c_double, C.c_double, _dp, _dp]
            lib.orc_getH.restype = C.c_double
            lib.orc_getH.argtypes = [C.c_void_p, _dp, C.c_double]
            lib.orc_z_inf_discrete.restype = C.c_double
            lib.orc_z_inf_discrete.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int]
            lib.fc_plan3d_init.argtypes = [C.c_void_p, C.c_void_p]
            lib.fc_plan3d_free.argtypes = [C.c_void_p]
            lib.fc_r2c3d.argtypes = [C.c_void_p, _dp, _dp]
            lib.fc_c2r3d.argtypes = [C.c_void_p, _dp, _dp]
            cls._lib = lib
        return cls._lib

    def __init__(self, NA: int, NB: int, m, L, threads: int = 1):
        self.NA, self.NB, self.N = int(NA), int(NB), int(NA) + int(NB)
        self.m = tuple(int(x) for x in m)
        self.L = tuple(float(x) for x in L)
        self.M = self.m[0] * self.m[1] * self.m[2]
        self.Mk = self.m[0] * self.m[1] * (self.m[2] // 2 + 1)
        lib = self.lib()
        lib.orc_set_threads(int(threads))
        self._s = lib.orc_create(self.NA, self.NB, _i3(self.m), _d3(self.L))
        if not self._s:
            raise MemoryError("orc_create failed")
        self._am = None

    def close(self):
        lib = self.lib()
        if self._am:
            lib.orc_anderson_destroy(self._am)
            self._am = None
        if self._s:
            lib.orc_destroy(self._s)
            self._s = None

    __del__ = close

    def g(self):
        out = np.empty(self.Mk)
        self.lib().orc_g_lookup(self._s, out)
        return out

    def step_fwd(self, q_in, h, i):
        out = np.empty(2 * self.M)
        self.lib().orc_step_fwd(self._s, np.ascontiguousarray(q_in, np.float64), out,
                                np.ascontiguousarray(h, np.float64), int(i))
        return out

    def calc_concs(self, w):
        """w: 4M array updated in place (phi-, phi+); returns ln Q."""
        return self.lib().orc_calc_concs(self._s, w)

    def propagators(self):
        p = self.lib().orc_propagators(self._s)
        n = 2 * (self.N + 1) * self.M
        return np.ctypeslib.as_array(p, shape=(n,)).copy().reshape(self.N + 1, 2, self.M)

    def mix(self, w, max_iter=200, tol=1e-4):
        lib = self.lib()
        if self._am is None:
            self._am = lib.orc_anderson_create(self.M, 10)
        return lib.orc_anderson_mix(self._am, self._s, int(max_iter), float(tol), w)

    def sk_sample(self, w, S):
        self.lib().orc_sk_sample(self._s, np.ascontiguousarray(w[: self.M]), S)

    def getH(self, w, XbN):
        return self.lib().orc_getH(self._s, w, float(XbN))

    @classmethod
    def langevin_update(cls, w, noise_prev, noise_new, XbN, dt):
        M = len(noise_prev)
        cls.lib().orc_langevin_update(w, noise_prev, noise_new, float(XbN), float(dt), int(M))

    @classmethod
    def sk_bin(cls, m, L, S, nsamples, CV, chi_b, dK=1e-5):
        Mk = len(S)
        K = np.empty(Mk)
        Sb = np.empty(Mk)
        n = cls.lib().orc_sk_bin(_i3(m), _d3(L), S, int(nsamples), float(CV), float(chi_b),
                                 float(dK), K, Sb)
        return K[:n].copy(), Sb[:n].copy()

    @classmethod
    def z_inf(cls, L, m, N, Nbar, tmax=100):
        return cls.lib().orc_z_inf_discrete(_d3(L), _i3(m), int(N), float(Nbar), int(tmax))

    @classmethod
    def r2c3d(cls, x):
        """3-D r2c of a real (m0, m1, m2) array with the oracle's FFT (tests only)."""
        x = np.ascontiguousarray(x, np.float64)
        m = x.shape
        plan = C.create_string_buffer(4096)
        lib = cls.lib()
        lib.fc_plan3d_init(plan, _i3(m))
        out = np.empty(2 * m[0] * m[1] * (m[2] // 2 + 1))
        lib.fc_r2c3d(plan, x.ravel(), out)
        lib.fc_plan3d_free(plan)
        return out.view(np.complex128).reshape(m[0], m[1], m[2] // 2 + 1)

    @classmethod
    def c2r3d(cls, X, m):
        X = np.ascontiguousarray(X, np.complex128).copy()
        plan = C.create_string_buffer(4096)
        lib = cls.lib()
        lib.fc_plan3d_init(plan, _i3(m))
        out = np.empty(m[0] * m[1] * m[2])
        lib.fc_c2r3d(plan, X.view(np.float64).ravel(), out)
        lib.fc_plan3d_free(plan)
        return out.reshape(m)


class RefHarness:
    """The reference's own classes (oracle/_ref).  Only where the build exists."""

    _lib = None

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    @classmethod
    def lib(cls):
        if cls._lib is None:
            lib = C.CDLL(REF_SO)
            lib.ref_sys_create.restype = C.c_void_p
            lib.ref_sys_create.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
            lib.ref_sys_destroy.argtypes = [C.c_void_p]
            lib.ref_sys_calc_concs.restype = C.c_double
            lib.ref_sys_calc_concs.argtypes = [C.c_void_p, _dp]
            lib.ref_sys_mix.restype = C.c_int
            lib.ref_sys_mix.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp]
            lib.ref_sys_step_fwd.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int]
            lib.ref_sys_g.argtypes = [C.c_void_p, _dp, C.c_int]
            lib.ref_set_threads.argtypes = [C.c_int]
            lib.ref_quiet.argtypes = [C.c_int]
            lib.ref_sim_create.restype = C.c_void_p
            lib.ref_sim_create.argtypes = [C.c_char_p]
            lib.ref_sim_destroy.argtypes = [C.c_void_p]
            lib.ref_sim_M.restype = C.c_int
            lib.ref_sim_M.argtypes = [C.c_void_p]
            lib.ref_sim_params.argtypes = [C.c_void_p, _dp, C.c_void_p]
            lib.ref_sim_get_w.argtypes = [C.c_void_p, _dp]
            lib.ref_sim_get_noise.argtypes = [C.c_void_p, _dp, _dp]
            lib.ref_sim_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                         C.POINTER(C.c_double)]
            lib.ref_sim_getH.restype = C.c_double
            lib.ref_sim_getH.argtypes = [C.c_void_p]
            lib.ref_sim_sk_save.argtypes = [C.c_void_p, C.c_char_p]
            lib.ref_sim_sk_raw.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_int)]
            lib.ref_normal_stream.argtypes = [C.c_ulonglong, C.c_double, C.c_int, _dp]
            lib.ref_lamellar.argtypes = [_dp, C.c_double, C.c_void_p]
            lib.ref_lgv_create.restype = C.c_void_p
            lib.ref_lgv_create.argtypes = [C.c_ulonglong, C.c_double, C.c_int]
            lib.ref_lgv_destroy.argtypes = [C.c_void_p]
            lib.ref_lgv_uniform_field.argtypes = [C.c_void_p, C.c_double, C.c_int, _dp]
            lib.ref_sys_full_step.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, _dp,
                                              C.POINTER(C.c_int), C.POINTER(C.c_double)]
            cls._lib = lib
        return cls._lib


class RefSys:
    """diblock + anderson + step objects of the reference."""

    def __init__(self, NA, NB, m, L):
        self.M = int(m[0]) * int(m[1]) * int(m[2])
        self.Mk = int(m[0]) * int(m[1]) * (int(m[2]) // 2 + 1)
        self._lib = RefHarness.lib()
        self._s = self._lib.ref_sys_create(int(NA), int(NB), _i3(m), _d3(L))

    def close(self):
        if self._s:
            self._lib.ref_sys_destroy(self._s)
            self._s = None

    __del__ = close

    def calc_concs(self, w):
        return self._lib.ref_sys_calc_concs(self._s, w)

    def mix(self, w, max_iter=200, tol=1e-4):
        return self._lib.ref_sys_mix(self._s, int(max_iter), float(tol), w)

    def step_fwd(self, q_in, h, i):
        out = np.empty(2 * self.M)
        self._lib.ref_sys_step_fwd(self._s, np.ascontiguousarray(q_in), out,
                                   np.ascontiguousarray(h), int(i))
        return out

    def g(self):
        out = np.empty(self.Mk)
        self._lib.ref_sys_g(self._s, out, self.Mk)
        return out


def ref_lamellar(amp, m):
    """W-, w+ (2M) of the reference's (300) lamellar start, amplitude amp."""
    M = int(m[0]) * int(m[1]) * int(m[2])
    w = np.zeros(2 * M)
    RefHarness.lib().ref_lamellar(w, float(amp), _i3(m))
    return w


class RefLangevin:
    """The reference's langevin object on its own mt19937_64(seed); its
    constructor draws the initial noise.  ``full_step`` runs the reference's
    loop body (step_wm, mix, the extra calc_concs) on a RefSys."""

    def __init__(self, seed, sigma, M):
        self._lib = RefHarness.lib()
        self.sigma = float(sigma)
        self._l = self._lib.ref_lgv_create(int(seed), self.sigma, int(M))

    def close(self):
        if self._l:
            self._lib.ref_lgv_destroy(self._l)
            self._l = None

    __del__ = close

    def uniform_field(self, XbN, M):
        """W-, w+ (2M) of the reference program's random start (loadType 0 or
        3), drawn from this generator after the constructor's noise"""
        w = np.zeros(2 * int(M))
        self._lib.ref_lgv_uniform_field(self._l, float(XbN), int(M), w)
        return w

    def full_step(self, sys_: RefSys, w, XbN, dt):
        K = C.c_int()
        lnQ = C.c_double()
        self._lib.ref_sys_full_step(sys_._s, self._l, float(XbN), self.sigma, float(dt), w, C.byref(K),
                                    C.byref(lnQ))
        return K.value, lnQ.value


class RefSim:
    """A whole reference lfts_simulation built from an input file.  The
    constructor writes w_0/phi_0 into the current directory."""

    def __init__(self, input_file: str, quiet: bool = True):
        self._lib = RefHarness.lib()
        self._lib.ref_quiet(1 if quiet else 0)
        self._s = self._lib.ref_sim_create(input_file.encode())
        self.M = self._lib.ref_sim_M(self._s)
        d = np.empty(5)
        i = (C.c_int * 10)()
        self._lib.ref_sim_params(self._s, d, i)
        self.XbN, self.XeN, self.sigma, self.CV, self.dt = [float(x) for x in d]
        (self.N, self.NA, m0, m1, m2, self.equil_its, self.sim_its, self.sample_freq,
         self.save_freq, self.loadType) = [int(x) for x in i]
        self.m = (m0, m1, m2)
        self.Mk = m0 * m1 * (m2 // 2 + 1)

    def close(self):
        if self._s:
            self._lib.ref_sim_destroy(self._s)
            self._s = None

    __del__ = close

    def w(self):
        out = np.empty(4 * self.M)
        self._lib.ref_sim_get_w(self._s, out)
        return out

    def noise(self):
        p = np.empty(self.M)
        n = np.empty(self.M)
        self._lib.ref_sim_get_noise(self._s, p, n)
        return p, n

    def step(self, sample=False):
        K = C.c_int()
        lnQ = C.c_double()
        self._lib.ref_sim_step(self._s, 1 if sample else 0, C.byref(K), C.byref(lnQ))
        return K.value, lnQ.value

    def getH(self):
        return self._lib.ref_sim_getH(self._s)

    def sk_save(self, fname):
        self._lib.ref_sim_sk_save(self._s, fname.encode())

    def sk_raw(self):
        S = np.empty(self.Mk)
        ns = C.c_int()
        self._lib.ref_sim_sk_raw(self._s, S, C.byref(ns))
        return S, ns.value
