"""The drop-in program lfts-b200 against the reference program's own output
(tests/golden/prog_*.tar.gz: the reference's stdout and w_*, phi_*,
struct_st_* files for the same input).  Files must match line for line: the
header lines exactly, the values to the 6 significant digits the reference
prints (FP64 path), with at most MAX_FLIPS lines per file whose last digit
rounds the other way (the count per file is printed)."""
import os
import subprocess
import tarfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

EXE = os.path.join(ROOT, "lfts_cpu_b200", "lfts-b200")


def _values(lines):
    out = []
    for ln in lines:
        for tok in ln.replace("\t", " ").split():
            try:
                out.append(float(tok))
            except ValueError:
                out.append(np.nan)
    return np.array(out)


MAX_FLIPS = 2  # lines per file whose 6th significant digit may round the other way


def compare_text(got, ref, name):
    """Line for line; returns the number of lines whose text differs (each a
    last-digit rounding flip of a value within 2e-5 of the reference's)."""
    g = got.splitlines()
    r = ref.splitlines()
    assert len(g) == len(r), f"{name}: {len(g)} lines vs {len(r)}"
    flips = sum(a != b for a, b in zip(g, r))
    gv, rv = _values(g), _values(r)
    assert gv.shape == rv.shape, name
    finite = np.isfinite(rv)
    assert np.array_equal(np.isfinite(gv), finite), name
    rel = np.abs(gv[finite] - rv[finite]) / np.maximum(np.abs(rv[finite]), 1e-3)
    assert rel.max() < 2e-5, f"{name}: max rel diff {rel.max()}"
    assert flips <= MAX_FLIPS, f"{name}: {flips} of {len(r)} lines differ in text"
    return flips


def test_driver_usage_without_gpu(native_lib):
    r = subprocess.run([EXE], capture_output=True, text=True)
    assert r.returncode == 1
    assert "Please supply an input file name" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["prog_valgrind16", "prog_saves16"])
def test_driver_reproduces_reference_outputs(native_lib, tmp_path, name):
    ref = tmp_path / "ref"
    run = tmp_path / "run"
    ref.mkdir()
    run.mkdir()
    with tarfile.open(os.path.join(GOLDEN, name + ".tar.gz")) as tar:
        tar.extractall(ref, filter="data")
    (run / "input").write_text((ref / "input").read_text())
    r = subprocess.run([EXE, "input"], cwd=run, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    expected = sorted(f for f in os.listdir(ref) if f not in ("input", "stdout.txt"))
    produced = sorted(f for f in os.listdir(run) if f != "input")
    assert produced == expected
    flips = {f: compare_text((run / f).read_text(), (ref / f).read_text(), f) for f in expected}
    print(f"{name}: text lines differing per file {flips}; total {sum(flips.values())} of "
          f"{sum(len((ref / f).read_text().splitlines()) for f in expected)}")
    # stdout: same lines except the wall-clock timings and the FFTW-threads
    # banner that only an OpenMP build of the reference prints
    keep = lambda s: [ln for ln in s.splitlines() if "time =" not in ln and "threads for FFTs" not in ln]
    compare_text("\n".join(keep(r.stdout)), "\n".join(keep((ref / "stdout.txt").read_text())), "stdout")
