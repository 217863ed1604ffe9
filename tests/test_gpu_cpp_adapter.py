"""A C++ program built on the library's C++ host wrapper (include/zmpm.hpp
over include/zmpm.h; compiled here with g++ and linked with the CUDA library)
drives the implicit substep in phases, as a reference-side MpmSimulationBase
subclass would, and matches whole substeps."""
import os
import subprocess

import pytest

from ziran2019_b200 import build

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cpp_phase_adapter_matches_substep(tmp_path, cuda_lib, precision):
    lib = build.build()
    exe = tmp_path / "phase_adapter"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "phase_adapter.cpp"), "-o", str(exe),
                    "-L", os.path.dirname(lib), "-lzmpm", "-Wl,-rpath," + os.path.dirname(lib)], check=True)
    out = subprocess.run([str(exe), precision[0]], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    fields = out.stdout.split()
    assert fields[0] == "max_rel_dx", out.stdout
    # the two runs differ only in the order of floating-point atomics (FP32
    # sums in the mixed substep's transfers and products)
    assert float(fields[1]) < (1e-9 if precision == "fp64" else 1e-5), out.stdout
