"""TEST INFRASTRUCTURE: ctypes binding of the CPU oracle (oracle/build/libzmpm_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this.  The
oracle exports the zmpm C ABI under the prefix ``zoracle_`` plus a few
single-kernel helpers (SVD, model evaluation, return map, SPGrid masks).
"""
import ctypes as C
import os
import subprocess

from ziran2019_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libzmpm_oracle.so")
# the same source built for the host it runs on (-march=native), for the timed CPU baseline
NATIVE_PATH = os.path.join(HERE, "build", "libzmpm_oracle_native.so")
_libs = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_native_async():
    """Starts the -march=native build (about 20 s) and returns the process, or
    None when it is already built."""
    if os.path.exists(NATIVE_PATH) and os.path.getmtime(NATIVE_PATH) >= os.path.getmtime(os.path.join(HERE, "zmpm_oracle.cpp")):
        return None
    return subprocess.Popen(["make", "-s", "-C", HERE, "native"], stdout=subprocess.DEVNULL, stderr=subprocess.STDOUT)


def lib(native=False):
    """The oracle library; native=True: the -march=native build when it exists
    (the portable build otherwise)."""
    path = NATIVE_PATH if native and os.path.exists(NATIVE_PATH) else LIB_PATH
    if path not in _libs:
        if not os.path.exists(path):
            build()
        L = abi.Lib(path, "zoracle_", product=False)
        d = L.dll
        d.zoracle_model_eval.restype = C.c_int
        d.zoracle_model_eval.argtypes = [C.c_int32, C.c_double, C.c_double, abi.c_double_p, abi.c_double_p,
                                         abi.c_double_p, abi.c_double_p, abi.c_double_p]
        d.zoracle_svd3.restype = C.c_int
        d.zoracle_svd3.argtypes = [abi.c_double_p, abi.c_double_p, abi.c_double_p, abi.c_double_p, C.c_int32]
        d.zoracle_von_mises.restype = C.c_int
        d.zoracle_von_mises.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                        abi.c_double_p, abi.c_double_p]
        d.zoracle_plastic_project.restype = C.c_int
        d.zoracle_plastic_project.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, abi.c_double_p, C.c_int32,
                                              abi.c_double_p, abi.c_double_p]
        d.zoracle_dp_project_sigma.restype = C.c_int
        d.zoracle_dp_project_sigma.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, abi.c_double_p, abi.c_double_p,
                                               abi.c_double_p]
        d.zoracle_linear_offset.restype = C.c_uint64
        d.zoracle_linear_offset.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        d.zoracle_packed_add.restype = C.c_uint64
        d.zoracle_packed_add.argtypes = [C.c_int32, C.c_uint64, C.c_uint64]
        d.zoracle_masks.restype = None
        d.zoracle_masks.argtypes = [C.c_int32, abi.c_uint64_p]
        L.native = path == NATIVE_PATH
        _libs[path] = L
    return _libs[path]
