"""The C ABI library loads and exports every function include/dmpm.h declares
(no GPU calls)."""
import os
import re
import subprocess

import pytest

import dmpm

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(REPO, "include", "dmpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dmpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = dmpm.load_library()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", dmpm.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dmpm_\w+)", out))
    assert set(names) <= exported, sorted(set(names) - exported)


def test_params_struct_matches_header():
    p = dmpm.Params()
    dmpm.load_library().dmpm_default_params(p)
    assert p.adjoint_mode == dmpm.ADJ_REFCOMPAT and p.control_mode == dmpm.CTRL_PER_LAYER
    assert abs(p.dt - 1.0 / 120.0) < 1e-15 and p.drag == 0.5 and abs(p.smoothing - 0.1) < 1e-15


def test_null_arguments_are_rejected_without_gpu():
    lib = dmpm.load_library()
    assert lib.dmpm_create(0, 7, None) == dmpm.ERR_ARG
    assert lib.dmpm_destroy(None) == dmpm.ERR_ARG
    assert lib.dmpm_forward(None, 0) == dmpm.ERR_ARG
