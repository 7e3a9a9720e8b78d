"""The C-ABI library loads and exports every function include/picb200.h declares (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "picb200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(pic_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def libpath():
    from pic_b200 import build

    return build.build()


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["pic_update_R", "pic_update_V", "pic_deposit", "pic_update_E", "pic_absorb", "pic_mg_create",
                 "pic_mg_solve", "pic_sort", "pic_mcc_apply", "pic_sim_create", "pic_sim_step", "pic_last_error"]:
        assert must in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(libpath)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared_functions()) <= exported


def test_python_binding_covers_the_header(libpath):
    from pic_b200 import _lib

    assert set(declared_functions()) == set(_lib.SIGNATURES)
    lib = _lib.load()
    assert lib.pic_abi_version() == 4
    assert lib.pic_last_error() == b""


def test_library_is_built_for_sm100a(libpath):
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", libpath], capture_output=True, text=True)
    assert "sm_100a" in out.stdout
