"""TEST AND CPU-TIMING INFRASTRUCTURE ONLY -- the reference's calc_concs
(src/diblock.cc:30-60 with step::fwd, src/step.cc:35-65, and normalize_phi,
src/diblock.cc:85-95) restated on scipy.fft (pocketfft) with `workers`
threads and in-place numpy arithmetic.

It is the fastest CPU FFT available on this image, and bench.py times it
beside the reference (whose FFT here is the self-written FFTW shim) as a
labelled bound: "best available CPU FFT, not the reference".  Nothing in the
product imports it.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft


class ScipyConcs:
    """calc_concs of one (NA, NB, mesh, box) with the reference's slot layout:
    slot i = [q_i | q^_{N+1-i}], i = 1..N (src/diblock.cc:9-25)."""

    def __init__(self, NA, NB, m, L, workers=1):
        self.NA, self.NB, self.N = int(NA), int(NB), int(NA) + int(NB)
        self.m = tuple(int(x) for x in m)
        self.M = int(np.prod(self.m))
        self.workers = int(workers)
        # g(k) = exp(-(2 pi)^2 (kx^2/Lx^2 + ky^2/Ly^2 + kz^2/Lz^2)/(6N)) / M, half spectrum
        # (src/step.cc:69-89)
        k = [np.fft.fftfreq(n, 1.0 / n) for n in self.m[:2]] + [np.arange(self.m[2] // 2 + 1, dtype=float)]
        ksq = (k[0][:, None, None] / L[0]) ** 2 + (k[1][None, :, None] / L[1]) ** 2 + (k[2][None, None, :] / L[2]) ** 2
        self.g = np.exp(-(2.0 * np.pi) ** 2 * ksq / (6.0 * self.N)) / self.M
        self.q = np.empty((self.N + 1, 2) + self.m)

    def calc_concs(self, w):
        """w: 4M array [W-, w+, phi-, phi+]; phi written in place; returns ln Q."""
        M, N, NA, NB, m = self.M, self.N, self.NA, self.NB, self.m
        wm = w[:M].reshape(m)
        wp = w[M:2 * M].reshape(m)
        hA = np.exp(-(wm + wp) / N)  # src/diblock.cc:64-72
        hB = np.exp(-(-wm + wp) / N)
        q = self.q
        q[1, 0] = hA
        q[1, 1] = hB
        for i in range(1, N):
            # unnormalised transforms both ways, as FFTW's (g carries 1/M)
            X = sfft.rfftn(q[i], axes=(1, 2, 3), workers=self.workers)
            X *= self.g
            q[i + 1] = sfft.irfftn(X, s=m, axes=(1, 2, 3), norm="forward", workers=self.workers, overwrite_x=True)
            q[i + 1, 0] *= hA if i < NA else hB  # src/step.cc:53-57
            q[i + 1, 1] *= hB if i < NB else hA  # src/step.cc:60-64
        Q = q[N, 0].sum() / M
        phiA = np.zeros(m)
        phiB = np.zeros(m)
        for i in range(1, N + 1):
            (phiA if i <= NA else phiB).__iadd__(q[i, 0] * q[N + 1 - i, 1])
        phiA /= N * Q * hA
        phiB /= N * Q * hB
        w[2 * M:3 * M] = (phiA - phiB).ravel()
        w[3 * M:] = (phiA + phiB).ravel()
        return float(np.log(Q))
