"""The ctypes mirrors of the ABI's structs against the C compiler's layout.

Each struct of include/picb200.h that the Python binding passes by pointer is
compiled into a small C program that prints its size and the offset of every
field; the ctypes Structure of pic_b200/_lib.py must agree field by field (a
field added on one side only, as min_cycles was to pic_sim_desc, shifts every
later offset).  CPU only: gcc and the header, no GPU.
"""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from pic_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> ctypes Structure
PAIRS = {
    "pic_mg_options": _lib.MgOptions,
    "pic_mg_info": _lib.MgInfo,
    "pic_mcc_species_desc": _lib.MccSpeciesDesc,
    "pic_mcc_desc": _lib.MccDesc,
    "pic_birth_buffer": _lib.BirthBuffer,
    "pic_species_desc": _lib.SpeciesDesc,
    "pic_sim_desc": _lib.SimDesc,
    "pic_sim_counters": _lib.SimCounters,
    "pic_sim_diag": _lib.SimDiag,
    "pic_sim_profile": _lib.SimProfile,
    "pic_adj_species": _lib.AdjSpecies,
    "pic_adj_desc": _lib.AdjDesc,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "picb200.h"', "int main(void) {"]
    for cname, cls in PAIRS.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'    printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["    return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    layout = {}
    for line in out:
        if line:
            parts = line.split()
            layout[(parts[0], parts[1])] = int(parts[2])
    return layout


@pytest.mark.parametrize("cname", list(PAIRS))
def test_ctypes_struct_matches_c_layout(c_layout, cname):
    cls = PAIRS[cname]
    assert C.sizeof(cls) == c_layout[(cname, "size")], cname
    for fname, _ in cls._fields_:
        assert getattr(cls, fname).offset == c_layout[(cname, fname)], (cname, fname)
