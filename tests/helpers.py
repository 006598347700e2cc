"""Test helpers shared by the CPU and GPU suites."""
import gzip
import os

import numpy as np

from conftest import GOLDEN


def ref_input40_fields():
    """(header lines, 2M field values) of the reference's 40^3 fixture."""
    with gzip.open(os.path.join(GOLDEN, "ref_input40_fields.txt.gz"), "rt") as f:
        lines = f.read().split("\n")
    return lines[:3], np.array([float(x) for x in lines[3:] if x.strip()])


def parse_header(hdr_lines):
    a = hdr_lines[0].split()
    b = hdr_lines[1].split()
    c = hdr_lines[2].split()
    return dict(N=int(a[0]), NA=int(a[1]), XN=float(a[2]), C=float(a[3]), dt=float(a[4]), isXeN=int(a[5]),
                m=[int(x) for x in b[:3]], L=[float(x) for x in b[3:6]], n_eq=int(c[0]), n_st=int(c[1]),
                n_smpl=int(c[2]), save_freq=int(c[3]), loadType=int(c[4]))


def write_input(path, header_lines, fields=None):
    with open(path, "w") as f:
        f.write("\n".join(str(h) for h in header_lines) + "\n")
        if fields is not None:
            f.write("\n".join(repr(float(v)) for v in fields) + "\n")
