"""ctypes mirror of include/zmpm.h.

`Lib(path, prefix)` binds one shared library exporting the zmpm C ABI under a
symbol prefix.  The product library is `ziran2019_b200/lib/libzmpm.so` (prefix
``zmpm_``), built from `ziran2019_b200/csrc` by `ziran2019_b200/build.py`.
"""
import ctypes as C
import os

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)
c_int64_p = C.POINTER(C.c_int64)
c_uint64_p = C.POINTER(C.c_uint64)

# status codes (zmpm_status_code)
OK = 0
CFL_VIOLATION = 1
NEWTON_NOT_CONVERGED = 2
NAN_DETECTED = 3
TIMEOUT = 4
BAD_ARG = -1
OUT_OF_GRID = -2
CUDA_ERROR = -3
NO_MEMORY = -4
NOT_READY = -5
UNSUPPORTED = -6

FP64 = 0
MIXED = 1
NOALLOC_MAX_PARTICLES = 262144
LAYOUT_AUTO, LAYOUT_244, LAYOUT_444 = 0, 1, 2
MODEL_NONE, MODEL_NEOHOOKEAN_BORDEN, MODEL_STVK_HENCKY_ISOTROPIC, MODEL_FIXED_COROTATED = 0, 1, 2, 3
PLASTIC_NONE, PLASTIC_VON_MISES, PLASTIC_DRUCKER_PRAGER, PLASTIC_CAM_CLAY = 0, 1, 2, 3
DAMAGE_NONE, DAMAGE_RANKINE, DAMAGE_PHASE_FIELD, DAMAGE_RANKINE_REFERENCE = 0, 1, 2, 3
NEWTON, ADMM, EXPLICIT = 0, 1, 2
BGEO_POSITION, BGEO_VELOCITY, BGEO_PHASE_FIELD = 0, 1, 2
MINRES, CG = 0, 1
HALF_SPACE, SPHERE, BOX = 0, 1, 2
STICKY, SLIP, SEPARATE, GHOST = 1, 2, 3, 4


class Config(C.Structure):
    _fields_ = [
        ("precision", C.c_int32),
        ("layout", C.c_int32),
        ("grid_log2", C.c_int32),
        ("device", C.c_int32),
        ("dx", C.c_double),
        ("gravity", C.c_double * 3),
        ("apic_rpic_ratio", C.c_double),
        ("cfl", C.c_double),
    ]


class Solver(C.Structure):
    _fields_ = [
        ("linear_solver", C.c_int32),
        ("newton_max_iterations", C.c_int32),
        ("newton_tolerance", C.c_double),
        ("krylov_max_iterations", C.c_int32),
        ("pad0", C.c_int32),
        ("krylov_tolerance", C.c_double),
        ("linear_solve_tolerance_scale", C.c_double),
        ("integrator", C.c_int32),
        ("admm_iterations", C.c_int32),
        ("admm_rho_scale", C.c_double),
        ("admm_local_tolerance", C.c_double),
        ("admm_global_tolerance", C.c_double),
        ("admm_global_max_iterations", C.c_int32),
        ("trial_collision", C.c_int32),
        ("mls_mpm", C.c_int32),
        ("pad1", C.c_int32),
    ]


class Collider(C.Structure):
    _fields_ = [
        ("shape", C.c_int32),
        ("type", C.c_int32),
        ("friction", C.c_double),
        ("a", C.c_double * 3),
        ("b", C.c_double * 3),
        ("radius", C.c_double),
        ("rotation", C.c_double * 4),
        ("angular_velocity", C.c_double * 3),
        ("translation", C.c_double * 3),
        ("translation_velocity", C.c_double * 3),
        ("scale", C.c_double),
        ("scale_velocity", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("newton_iterations", C.c_int32),
        ("krylov_iterations", C.c_int32),
        ("hvp_count", C.c_int32),
        ("cfl_violation", C.c_int32),
        ("newton_converged", C.c_int32),
        ("status_flags", C.c_int32),
        ("num_particles", C.c_int64),
        ("num_groups", C.c_int64),
        ("num_blocks", C.c_int64),
        ("num_nodes", C.c_int64),
        ("num_collision_nodes", C.c_int64),
        ("newton_residual_initial", C.c_double),
        ("newton_residual_final", C.c_double),
        ("ms_total", C.c_double),
        ("ms_hvp", C.c_double),
        ("hvp_timed", C.c_int32),
        ("kernel_launches", C.c_int32),
        ("phase_field_iterations", C.c_int32),
        ("fp64_residual", C.c_int32),
        ("phase_field_residual", C.c_double),
        ("rankine_first_not_max", C.c_int64),
        ("svd_fp64_reevaluations", C.c_int64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class BinResult(C.Structure):
    _fields_ = [
        ("particle_sorter", c_uint64_p),
        ("particle_order", c_int32_p),
        ("particle_base_offset", c_uint64_p),
        ("particle_group", c_int32_p),
        ("block_offset", c_uint64_p),
        ("page_offsets", c_uint64_p),
    ]


_SIGS = {
    "create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "destroy": (C.c_int, [C.c_void_p]),
    "last_error": (C.c_char_p, [C.c_void_p]),
    "add_particles": (C.c_int, [C.c_void_p, C.c_int64, c_double_p, c_double_p, c_double_p, c_double_p, c_int64_p]),
    "add_fbased_force": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_double]),
    "set_lame": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, c_double_p, c_double_p]),
    "add_plasticity": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "add_drucker_prager": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_int32]),
    "add_cam_clay": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32]),
    "get_log_jp": (C.c_int, [C.c_void_p, c_double_p]),
    "max_particle_speed": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p]),
    "calculate_dt": (C.c_int, [C.c_void_p, C.c_double, c_double_p]),
    "add_damage": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_double]),
    "get_damage": (C.c_int, [C.c_void_p, c_double_p]),
    "add_phase_field": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int32, C.c_double]),
    "set_phase_field_solver": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.c_double, C.c_int32, C.c_double]),
    "get_phase_field": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, c_double_p]),
    "set_phase_field_sigma_c": (C.c_int, [C.c_void_p, c_double_p]),
    "add_viscoelastic": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double]),
    "get_viscoelastic_strain": (C.c_int, [C.c_void_p, c_double_p]),
    "set_viscoelastic_strain": (C.c_int, [C.c_void_p, c_double_p]),
    "add_collision_object": (C.c_int, [C.c_void_p, C.POINTER(Collider), c_int32_p]),
    "set_collision_object": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Collider)]),
    "get_particles": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, c_double_p]),
    "set_particles": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p, c_double_p]),
    "get_plastic_state": (C.c_int, [C.c_void_p, c_double_p, c_int32_p]),
    "num_particles": (C.c_int64, [C.c_void_p]),
    "time": (C.c_double, [C.c_void_p]),
    "substep": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Solver), C.POINTER(Stats)]),
    "bin": (C.c_int, [C.c_void_p, c_int64_p]),
    "bin_fetch": (C.c_int, [C.c_void_p, C.POINTER(BinResult)]),
    "begin_implicit": (C.c_int, [C.c_void_p, C.c_double, c_int64_p]),
    "get_grid": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_int32_p]),
    "get_initial_dv": (C.c_int, [C.c_void_p, c_double_p, c_int32_p]),
    "residual": (C.c_int, [C.c_void_p, c_double_p, c_double_p, c_double_p]),
    "multiply": (C.c_int, [C.c_void_p, c_double_p, c_double_p, C.c_int32]),
    "adjoint_substep": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Solver), C.c_double, c_double_p, c_double_p, c_double_p,
                                  c_double_p, c_double_p, C.POINTER(Stats)]),
    "checkpoint_save": (C.c_int, [C.c_void_p, C.c_int32]),
    "checkpoint_load": (C.c_int, [C.c_void_p, C.c_int32]),
}

# entry points exported by the product library only
_PRODUCT_ONLY = {
    "get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "status_string": (C.c_char_p, [C.c_int]),
    "sort_keys_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "default_solver": (None, [C.POINTER(Solver), C.c_int32, C.c_int32]),
    "write_state": (C.c_int, [C.c_void_p, C.c_char_p]),
    "read_state": (C.c_int, [C.c_void_p, C.c_char_p]),
    "write_restart": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_int32]),
    "read_restart": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "write_bgeo": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "particles_to_grid": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Solver)]),
    "backward_euler_step": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "grid_to_particles": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(Stats)]),
    "apply_plasticity": (C.c_int, [C.c_void_p]),
    "set_spin_limit": (C.c_int, [C.c_void_p, C.c_int64]),
}


class ZmpmError(RuntimeError):
    def __init__(self, status, where, msg=""):
        super().__init__(f"{where} failed with status {status}: {msg}")
        self.status = status


class Lib:
    """A loaded library exporting the zmpm ABI under `prefix`."""

    def __init__(self, path, prefix="zmpm_", product=True):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.prefix = prefix
        self.dll = C.CDLL(path)
        sigs = dict(_SIGS)
        if product:
            sigs.update(_PRODUCT_ONLY)
        for name, (res, args) in sigs.items():
            fn = getattr(self.dll, prefix + name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)

    def check(self, status, where, ctx=None):
        if status < 0:
            msg = ""
            if ctx is not None:
                try:
                    m = self.last_error(ctx)
                    msg = m.decode() if m else ""
                except Exception:  # noqa: BLE001 - best effort message only
                    msg = ""
            raise ZmpmError(status, where, msg)
        return status


def ptr(a, ctype=C.c_double):
    """Pointer to a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


BINARY_VER = 1  # ZMPM_BINARY_VER: the restart format version in binary_ver.txt

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB_PATH = os.path.join(_PKG_DIR, "lib", "libzmpm.so")
_product = None


def product_lib():
    """The CUDA library.  Raises if it has not been built: there is no fallback."""
    global _product
    if _product is None:
        if not os.path.exists(PRODUCT_LIB_PATH):
            raise RuntimeError(
                f"CUDA library missing at {PRODUCT_LIB_PATH}; build it with "
                "`python -m ziran2019_b200.build` (there is no CPU fallback)")
        _product = Lib(PRODUCT_LIB_PATH, "zmpm_", product=True)
    return _product
