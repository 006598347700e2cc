"""Tile choices of the contour chain and their autotuner: the x-pencil width
and (FP64) the stream split are bitwise-neutral; every FP32-mixed choice
(plane stages, where h is applied, concentration sums formed in the chain)
agrees with the others and with FP64 within the FP32-mixed tolerance; the
autotuner's choice is a valid candidate; invalid choices are refused and
leave the context as it was."""
import itertools

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

FP32_PHI_TOL = 1e-5


@pytest.fixture(scope="module")
def lfts(native_lib):
    import lfts_cpu_b200
    return lfts_cpu_b200


def candidates(precision, m):
    """Every tile combination, valid or not, for the context to accept or refuse."""
    out = []
    for cw, st, xh, two, phi, split in itertools.product((8, 16, 32), (2, 3), (0, 1), (0, 1), (0, 1), (1, 8)):
        if precision == 0 and (st != 2 or xh or phi or split != 1):
            continue
        if precision == 1 and (two or (phi and not xh)):
            continue
        out.append(dict(pencil_cw=cw, plane_stages=st, h_in_pencil=xh, two_streams=two, phi_in_chain=phi,
                        plane_split=split))
    return out


def valid(precision, m, t):
    if precision == 0:
        return True
    if t["plane_stages"] == 3 and m[1] not in (64, 96, 128):
        return False
    if t["h_in_pencil"] and not (t["plane_stages"] == 3 and m[0] in (96, 128) and m[1] in (96, 128)):
        return False
    # the cluster-split plane kernel: PLANE_G of 128 x 128 planes
    if t["plane_split"] != 1 and not (t["h_in_pencil"] and m[1] == 128 and m[2] == 128):
        return False
    return True


def run_all(lfts, precision, m, N, NA):
    M = int(np.prod(m))
    w2 = np.random.default_rng(M + N).normal(0.0, 0.7, 2 * M)
    s = lfts.System(N, NA, 16.0, 100.0, 0.5, m, tuple(x / 16.0 for x in m), precision=precision)
    s.set_fields(w2)
    tuned = s.tiles()
    results = []
    for t in candidates(precision, m):
        if not valid(precision, m, t):
            with pytest.raises(lfts.LftsError):
                s.set_tiles(**t)
            assert s.tiles() == (results[-1][0] if results else tuned)  # unchanged by the refusal
            continue
        s.set_tiles(**t)
        assert s.tiles() == t
        lnq = s.calc_concs()
        results.append((t, lnq, s.get_fields()[2 * M:]))
    s.close()
    return tuned, results


@pytest.mark.parametrize("m,N,NA", [((32, 32, 32), 16, 8), ((64, 64, 64), 12, 5), ((128, 128, 128), 10, 4)])
def test_fp64_tiles_are_bitwise_neutral(lfts, m, N, NA):
    tuned, res = run_all(lfts, 0, m, N, NA)
    assert any(t == tuned for t, _, _ in res)
    for t, lnq, phi in res[1:]:
        assert lnq == res[0][1], t
        assert np.array_equal(phi, res[0][2]), t


@pytest.mark.parametrize("m,N,NA", [((32, 32, 32), 16, 8), ((64, 64, 64), 12, 5), ((96, 96, 96), 8, 3),
                                    ((128, 128, 128), 10, 4)])
def test_fp32_tiles_agree_within_tolerance(lfts, m, N, NA):
    tuned, res = run_all(lfts, 1, m, N, NA)
    assert any(t == tuned for t, _, _ in res)
    M = int(np.prod(m))
    w2 = np.random.default_rng(M + N).normal(0.0, 0.7, 2 * M)
    s64 = lfts.System(N, NA, 16.0, 100.0, 0.5, m, tuple(x / 16.0 for x in m))
    s64.set_fields(w2)
    lnq64 = s64.calc_concs()
    phi64 = s64.get_fields()[2 * M:]
    s64.close()
    for t, lnq, phi in res:
        assert abs(lnq - lnq64) < FP32_PHI_TOL * max(1.0, abs(lnq64)), t
        assert rel_err(phi, phi64) < FP32_PHI_TOL, t
    # the pencil width and the plane split change no value
    by_rest = {}
    for t, lnq, phi in res:
        key = (t["plane_stages"], t["h_in_pencil"], t["phi_in_chain"])
        if key in by_rest:
            assert lnq == by_rest[key][0] and np.array_equal(phi, by_rest[key][1]), t
        else:
            by_rest[key] = (lnq, phi)


def test_autotuned_choices_are_candidates(lfts):
    for precision, m in ((1, (128, 128, 128)), (1, (96, 96, 96)), (1, (64, 64, 64)), (1, (48, 48, 48)),
                         (0, (128, 128, 128)), (0, (32, 32, 32))):
        s = lfts.System(8, 3, 16.0, 100.0, 0.5, m, (4.0, 4.0, 4.0), precision=precision)
        t = s.tiles()
        assert t in candidates(precision, m) and valid(precision, m, t), (m, t)
        assert s.tuning() == (t["pencil_cw"], t["plane_stages"])
        s.close()


@pytest.mark.parametrize("N,NA", [(2, 1), (3, 1), (3, 2), (7, 3), (8, 8), (8, 0), (64, 25)])
def test_phi_in_chain_matches_the_separate_pass(lfts, N, NA):
    """Concentration sums formed in the x-pencil from the middle of the chain
    on (each new slot times its stored partner; odd N: the middle slot with
    itself; the last step pairs slot N with h) against the separate pass over
    all stored slots: ln Q bitwise (both take Q from the stored slot N), phi to
    the FP32-mixed tolerance, and the propagators bitwise (the storing chain
    is rerun for them)."""
    m = (128, 128, 128)
    M = int(np.prod(m))
    w2 = np.random.default_rng(N * 100 + NA).normal(0.0, 0.5, 2 * M)
    s = lfts.System(N, NA, 16.0, 100.0, 0.5, m, (8.0, 8.0, 8.0), precision=1)
    s.set_fields(w2)
    out = []
    for phi in (0, 1):
        s.set_tiles(16, 3, 1, 0, phi)
        lnq = s.calc_concs()
        out.append((lnq, s.get_fields()[2 * M:], s.propagators() if N <= 8 else None))
    (lq0, p0, q0), (lq1, p1, q1) = out
    assert lq1 == lq0
    assert rel_err(p1, p0) < FP32_PHI_TOL
    if q0 is not None:
        assert np.array_equal(q1, q0)
    s.close()


@pytest.mark.parametrize("N,NA,phi", [(2, 1, 0), (7, 3, 1), (8, 3, 0), (64, 25, 1)])
def test_plane_split_is_bitwise_neutral(lfts, N, NA, phi):
    """The yz-plane kernel with each 128 x 128 x-plane spread over a cluster of
    8 CTAs (transposes through distributed shared memory) computes every value
    the one-CTA-per-plane kernel computes: ln Q, phi and the propagators
    bitwise equal."""
    m = (128, 128, 128)
    M = int(np.prod(m))
    w2 = np.random.default_rng(N * 10 + phi).normal(0.0, 0.5, 2 * M)
    s = lfts.System(N, NA, 16.0, 100.0, 0.5, m, (8.0, 8.0, 8.0), precision=1)
    s.set_fields(w2)
    out = []
    for split in (1, 8):
        s.set_tiles(16, 3, 1, 0, phi, split)
        assert s.tiles()["plane_split"] == split
        lnq = s.calc_concs()
        out.append((lnq, s.get_fields()[2 * M:], s.propagators() if N <= 8 else None))
    (lq0, p0, q0), (lq1, p1, q1) = out
    assert lq1 == lq0
    assert np.array_equal(p1, p0)
    if q0 is not None:
        assert np.array_equal(q1, q0)
    # refused where the cluster kernel does not apply
    with pytest.raises(lfts.LftsError):
        s.set_tiles(16, 3, 0, 0, 0, 8)
    with pytest.raises(lfts.LftsError):
        s.set_tiles(16, 3, 1, 0, phi, 4)
    s.close()
