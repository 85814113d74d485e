"""The reference's optimisation input file (OptInput) read and written in
cereal's JSON layout: golden files written by cereal's own JSON archive
(tests/golden/make_opt_input.sh) load with the right values, and what
optinput.save writes loads back unchanged and has cereal's structure.  Where
the reference tree is present, cereal itself also reads the written file."""
import json
import os
import subprocess

import numpy as np
import pytest

import optinput
from oracle.lib import reference_source_dir
from tests.helpers import GOLDEN

REF = reference_source_dir()


def f32(x):
    return float(np.float32(x))


def test_default_file_matches_reference_defaults():
    o = optinput.load(os.path.join(GOLDEN, "opt_input_default.json"))
    d = optinput.OptInput()
    for k, v in vars(d).items():
        got = getattr(o, k)
        if isinstance(v, tuple):
            assert got == tuple(f32(x) for x in v), k
        elif isinstance(v, float):
            assert got == f32(v), k
        else:
            assert got == v, k
    assert optinput.grid_dims(o) == (32, 32, 32)
    assert optinput.point_mass(o) == pytest.approx(0.125 * 40.0)


def test_custom_file_values_and_derived_setup():
    o = optinput.load(os.path.join(GOLDEN, "opt_input_custom.json"))
    assert o.mpm_input_mesh_path == "meshes/sphere.obj" and o.points_per_cell_cuberoot == 3
    assert o.grid_min_point == (-1.0, -2.0, -3.0) and o.grid_max_point == (4.0, 5.0, 6.0)
    assert o.f_ext == (0.0, f32(-9.8), 0.0) and o.dt == f32(1e-3) and o.control_stride == 5
    # the reference sizes every axis from the x extent (MPMPolyscope.cpp:96-99)
    assert optinput.grid_dims(o) == (10, 10, 10)
    assert optinput.point_mass(o) == pytest.approx((0.5 / 3) ** 3 * 2.5)
    p = optinput.params(o)
    assert p["dt"] == f32(1e-3) and p["smoothing"] == f32(0.2) and p["control_stride"] == 5


@pytest.mark.parametrize("name", ["opt_input_default.json", "opt_input_custom.json"])
def test_save_reproduces_cereal_structure(tmp_path, name):
    src = os.path.join(GOLDEN, name)
    o = optinput.load(src)
    out = tmp_path / "o.json"
    optinput.save(o, str(out))
    a, b = json.load(open(src)), json.load(open(out))
    assert list(a["value0"].keys()) == list(b["value0"].keys())
    assert a == b
    assert optinput.load(str(out)) == o


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include", "cereal")), reason="reference tree not present")
def test_cereal_reads_what_save_writes(tmp_path):
    o = optinput.load(os.path.join(GOLDEN, "opt_input_custom.json"))
    o.num_timesteps = 13
    o.f_ext = (1.5, -2.0, 0.25)
    mine = tmp_path / "mine.json"
    back = tmp_path / "back.json"
    optinput.save(o, str(mine))
    subprocess.check_call(["bash", os.path.join(GOLDEN, "make_opt_input.sh"), REF, str(mine), str(back)])
    assert optinput.load(str(back)) == o
