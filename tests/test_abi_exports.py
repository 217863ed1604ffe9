"""The CUDA library builds, loads without a GPU, and exports every entry point
declared in include/zmpm.h (no compute call is made here)."""
import ctypes
import os
import re

from ziran2019_b200 import abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "zmpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(zmpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    path = build.build()
    dll = ctypes.CDLL(path)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(dll, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    names = declared_functions()
    bound = set("zmpm_" + k for k in list(abi._SIGS) + list(abi._PRODUCT_ONLY))
    assert set(names) <= bound, sorted(set(names) - bound)


def test_status_strings_need_no_device():
    lib = abi.Lib(build.build(), "zmpm_")
    assert lib.status_string(0) == b"ok"
    assert b"CFL" in lib.status_string(1)


def test_restart_file_names_follow_the_reference():
    """SimulationBase::outputFileName (SimulationBase.h:192-199)."""
    from ziran2019_b200 import mpm
    assert mpm.MpmSimulation.outputFileName(7) == "restart_7.dat"
    assert mpm.MpmSimulation.outputFileName(7, 0) == "restart_7.dat"
    assert mpm.MpmSimulation.outputFileName(7, 3) == "restart_7_3.dat"
    assert mpm.MpmSimulation.outputFileName(0, 1, name="state", suffix=".bin") == "state_0_1.bin"


def test_cpp_wrapper_compiles_without_a_gpu():
    """include/zmpm.hpp (the GpuMpmSimulation host wrapper) and the C++ adapter
    built on it compile with g++ -Wall -Wextra -Werror against the headers."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "phase_adapter.cpp")], check=True)
