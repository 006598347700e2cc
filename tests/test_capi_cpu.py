"""C ABI checks that need no GPU: the library loads, exports every symbol
include/lfts_b200.h declares, and its host helpers (input parsing, RNG stream,
initial fields) reproduce the reference's driver semantics."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from helpers import parse_header, write_input


def header_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(lfts_\w+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(native_lib):
    names = header_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(native_lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(native_lib):
    from lfts_cpu_b200.capi import SIGNATURES
    assert set(header_functions()) <= set(SIGNATURES)


def test_no_gpu_means_error_not_fallback(native_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from lfts_cpu_b200 import LftsError, System
    with pytest.raises(LftsError):
        System(8, 4, 10.0, 50.0, 0.5, (16, 16, 16), (3, 3, 3))


def test_unsupported_mesh_is_rejected(native_lib):
    from lfts_cpu_b200 import LftsError, System
    assert native_lib.lfts_mesh_supported(128) == 1
    assert native_lib.lfts_mesh_supported(17) == 0
    with pytest.raises(LftsError):
        System(8, 4, 10.0, 50.0, 0.5, (17, 16, 16), (3, 3, 3))


@pytest.mark.parametrize("name", ["traj_valgrind16", "traj_16", "traj_lam24"])
def test_host_rng_and_fields_match_reference(native_lib, name):
    from lfts_cpu_b200 import Rng, lamellar_field
    g = golden(name)
    hdr = parse_header([str(s) for s in g["header"]])
    M = int(np.prod(hdr["m"]))
    rng = Rng(123456789, float(g["sigma"]))
    assert np.array_equal(rng.normal(M), g["noise_prev0"])
    if hdr["loadType"] == 2:
        w2 = lamellar_field(float(g["XbN"]), hdr["m"])
    else:
        w2 = rng.random_field(float(g["XbN"]), M)
    # the initial mix changes only w+, so W- is the generated field
    assert np.array_equal(w2[:M], g["w0"][:M])


@pytest.mark.parametrize("name", ["traj_valgrind16", "traj_16", "traj_lam24"])
def test_read_input_matches_reference_params(native_lib, tmp_path, name):
    from lfts_cpu_b200 import read_input
    g = golden(name)
    p = str(tmp_path / "input")
    write_input(p, [str(s) for s in g["header"]])
    inp = read_input(p)
    assert inp.XbN == float(g["XbN"])
    assert inp.XeN == float(g["XeN"])
    assert inp.sigma == float(g["sigma"])
    assert inp.N == int(g["N"]) and inp.NA == int(g["NA"])


def test_read_input_rounds_step_counts(native_lib, tmp_path):
    from lfts_cpu_b200 import read_input
    p = str(tmp_path / "input")
    write_input(p, ["64 32 14.0 50.0 0.5 0", "32 32 32 4.0 4.0 4.0", "1005 999 10 1000 0"])
    inp = read_input(p)
    assert (inp.equil_its, inp.sim_its) == (1000, 990)


def test_read_input_rejects_zero_sample_freq(native_lib, tmp_path):
    from lfts_cpu_b200 import LftsError, read_input
    p = str(tmp_path / "input")
    write_input(p, ["64 32 14.0 50.0 0.5 0", "32 32 32 4.0 4.0 4.0", "10 10 0 1000 0"])
    with pytest.raises(LftsError):
        read_input(p)


@pytest.mark.parametrize("kw,status", [
    (dict(N=1, NA=1), 1),                    # a chain needs two monomers
    (dict(NA=9), 1),                         # NA > N
    (dict(NA=-1), 1),
    (dict(C_=0.0), 1),
    (dict(XbN=0.0), 1),
    (dict(L=(3.0, 0.0, 3.0)), 1),            # box length not positive
    (dict(L=(3.0, float("nan"), 3.0)), 1),
    (dict(precision=7), 1),                  # neither FP64 nor FP32-mixed
    (dict(m=(17, 16, 16)), 2),               # no FFT plan for 17
    (dict(m=(16, 15, 16)), 2),               # odd my
])
def test_create_rejects_bad_parameters_before_any_device_call(native_lib, kw, status):
    """lfts_create validates its parameters first: bad ones give
    LFTS_ERR_ARG (1) or LFTS_ERR_UNSUPPORTED (2) on any machine, while valid
    ones get as far as the device query (LFTS_ERR_CUDA without a GPU)."""
    from lfts_cpu_b200 import LftsError, System
    args = dict(N=8, NA=4, XbN=10.0, C_=50.0, dt=0.5, m=(16, 16, 16), L=(3.0, 3.0, 3.0), precision=0)
    args.update(kw)
    with pytest.raises(LftsError) as e:
        System(**args)
    assert e.value.status == status


def _replica(**kw):
    d = dict(N=16, NA=8, XbN=12.0, C=50.0, dt=0.5, m=(32, 32, 32), L=(2.0, 2.0, 2.0), seed=1)
    d.update(kw)
    return d


@pytest.mark.parametrize("reps,status", [
    ([], 1),                                               # no replicas
    ([_replica(), _replica(N=12, NA=6)], 1),               # the chain length is shared
    ([_replica(), _replica(m=(128, 128, 128))], 2),        # ensemble meshes 16..96 per side
    ([_replica(m=(32, 32, 48))], 2),                       # square yz planes only
])
def test_ensemble_create_rejects_bad_replicas_before_any_device_call(native_lib, reps, status):
    """lfts_ensemble_create checks the replica list first (LFTS_ERR_ARG,
    LFTS_ERR_UNSUPPORTED) on any machine, before it touches a device."""
    from lfts_cpu_b200 import Ensemble, LftsError
    with pytest.raises(LftsError) as e:
        Ensemble(reps)
    assert e.value.status == status


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the header's structs (lfts_params, lfts_input,
    lfts_tiles) have the C compiler's size and field offsets, field by field."""
    import ctypes
    import shutil
    import subprocess

    from lfts_cpu_b200.capi import Input, Params, Tiles

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"lfts_params": Params, "lfts_input": Input, "lfts_tiles": Tiles}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "lfts_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
