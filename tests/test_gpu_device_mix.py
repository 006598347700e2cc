"""The Anderson loop of a single context on the device (one CUDA graph per
mix: a WHILE node around the contour chain, the concentrations with the
residual dot products, the least squares on one warp, the w+ update) against
the host-driven loop (the default; LFTS_DEVICE_MIX=1 selects the device loop): the same Anderson counts and the same
fields bit for bit, over an initial mix and Langevin steps, both precisions,
both FP32 chain orders, the yz-plane kernel of 128 x 128 planes per CTA and
split over a cluster."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


def make(lfts, host_loop, N, NA, m, precision, tiles=None):
    old = os.environ.get("LFTS_DEVICE_MIX")
    os.environ["LFTS_DEVICE_MIX"] = "0" if host_loop else "1"
    try:
        s = lfts.System(N, NA, 15.0, 80.0, 0.5, m, tuple(x / 16.0 for x in m), precision=precision)
    finally:
        if old is None:
            del os.environ["LFTS_DEVICE_MIX"]
        else:
            os.environ["LFTS_DEVICE_MIX"] = old
    if tiles:
        s.set_tiles(**tiles)
    return s


@pytest.mark.parametrize("precision,m,N,NA,tiles", [
    (0, (32, 32, 32), 16, 6, None),
    (1, (32, 32, 32), 16, 6, None),
    (0, (24, 24, 24), 12, 7, None),
    (1, (24, 24, 24), 12, 1, None),
    (1, (128, 128, 128), 8, 3, dict(pencil_cw=16, plane_stages=3, h_in_pencil=1, two_streams=0)),
    (1, (128, 128, 128), 8, 5, dict(pencil_cw=16, plane_stages=3, h_in_pencil=0, two_streams=0)),
    (1, (128, 128, 128), 7, 3, dict(pencil_cw=16, plane_stages=3, h_in_pencil=1, two_streams=0, phi_in_chain=1)),
    (1, (128, 128, 128), 7, 3, dict(pencil_cw=16, plane_stages=3, h_in_pencil=1, two_streams=0, phi_in_chain=1,
                                    plane_split=8)),
])
def test_device_loop_equals_host_loop(lfts, precision, m, N, NA, tiles):
    M = int(np.prod(m))
    w2 = np.random.default_rng(M + N).normal(0.0, 0.6, 2 * M)
    noise = np.random.default_rng(1).normal(0.0, 2.0, (3, M))
    out = []
    for host_loop in (True, False):
        s = make(lfts, host_loop, N, NA, m, precision, tiles)
        s.set_fields(w2)
        ks = [s.mix()]
        s.calc_concs()
        s.langevin_init(noise[0])
        for st in (1, 2):
            s.langevin_step(noise[st])
            ks.append(s.mix())
            s.calc_concs()
        out.append((ks, s.get_fields(), s.anderson_stats()))
        s.close()
    (k_h, w_h, st_h), (k_d, w_d, st_d) = out
    assert k_h == k_d
    assert np.array_equal(w_h, w_d)
    assert st_h == st_d  # calls and iterations counted alike
