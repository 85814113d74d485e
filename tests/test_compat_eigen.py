"""The compat C++ API with Eigen value types (libdmpm_compat_eigen.so): a
caller doing Eigen arithmetic on MaterialPoint fields, as the reference's own
code does, compiles against the compat headers unchanged and links
(tests/cpp/eigen_compat_check.cpp; host-side parts, no GPU).  Needs an Eigen
tree: $DMPM_EIGEN_INCLUDE, or the one the reference vendors."""
import os
import subprocess

import pytest

from oracle.lib import reference_source_dir

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "a-differentiable-material-point-method-for-shape-morphing_b200")
EIGEN = os.environ.get("DMPM_EIGEN_INCLUDE") or os.path.join(reference_source_dir(), "include")


@pytest.mark.skipif(not os.path.exists(os.path.join(EIGEN, "Eigen", "Dense")), reason="no Eigen tree at hand")
def test_eigen_caller_compiles_links_and_runs(tmp_path):
    import build as pkg_build

    lib = pkg_build.build_compat_eigen(EIGEN)
    exe = tmp_path / "eigen_compat_check"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(PKG, "compat"), "-I", EIGEN,
                           os.path.join(REPO, "tests", "cpp", "eigen_compat_check.cpp"), "-L", PKG,
                           "-l:" + os.path.basename(lib), "-ldmpm", "-Wl,-rpath," + PKG, "-o", str(exe)])
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "eigen compat ok" in res.stdout
