"""Autotuned tile shapes of the contour chain: the x-pencil tile width is
bitwise-neutral, and the autotuner's choice is one of the candidates."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


def _phi(lfts, precision, m, N, NA, cw, w2):
    old = os.environ.get("LFTS_PENCIL_CW")
    os.environ["LFTS_PENCIL_CW"] = str(cw)
    try:
        s = lfts.System(N, NA, 16.0, 100.0, 0.5, m, tuple(x / 16.0 for x in m), precision=precision)
    finally:
        if old is None:
            del os.environ["LFTS_PENCIL_CW"]
        else:
            os.environ["LFTS_PENCIL_CW"] = old
    assert s.tuning()[0] == cw
    s.set_fields(w2)
    lnq = s.calc_concs()
    w = s.get_fields()
    s.close()
    return lnq, w


@pytest.mark.parametrize("precision,m,N,NA", [(0, (32, 32, 32), 16, 8), (1, (32, 32, 32), 16, 8),
                                              (0, (64, 64, 64), 12, 5), (1, (128, 128, 128), 10, 4)])
def test_pencil_tile_width_is_bitwise_neutral(lfts, precision, m, N, NA):
    M = int(np.prod(m))
    w2 = np.random.default_rng(M + N).normal(0.0, 0.7, 2 * M)
    ref = _phi(lfts, precision, m, N, NA, 32, w2)
    for cw in (8, 16):
        lnq, w = _phi(lfts, precision, m, N, NA, cw, w2)
        assert lnq == ref[0]
        assert np.array_equal(w, ref[1])


def test_autotuned_choices(lfts):
    os.environ.pop("LFTS_PENCIL_CW", None)
    for precision, m, stages in ((1, (128, 128, 128), 3), (1, (96, 96, 96), 3), (1, (64, 64, 64), 3),
                                 (1, (48, 48, 48), 2), (0, (128, 128, 128), 2)):
        s = lfts.System(8, 3, 16.0, 100.0, 0.5, m, (4.0, 4.0, 4.0), precision=precision)
        cw, st = s.tuning()
        assert cw in (8, 16, 32)
        assert st == stages
        s.close()
