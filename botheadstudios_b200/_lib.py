"""ctypes binding of ``libsph_b200.so`` (the C ABI declared in ``include/sph_b200.h``).

Loading fails loudly if the library is missing: there is no CPU fallback on any path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libsph_b200.so")

# Status codes (sph_status)
SPH_OK = 0
SPH_CLAMPED = 1
SPH_NOT_READY = 2
SPH_ERR_INVALID = -1
SPH_ERR_CUDA = -2
SPH_ERR_OOM = -3
SPH_ERR_TIMEOUT = -4
SPH_ERR_OVERFLOW = -5
SPH_ERR_STATE = -6

# Inspection selectors (SPH_Q_*)
Q = dict(BBOX=0, CODES=1, ORDER=2, LEFT=3, RIGHT=4, PARENT=5, NODE_COM=6, NODE_BMIN=7, NODE_BMAX=8,
         NBR_COUNT=9, NBR_LIST=10, RHO=11, PRESSURE=12, SOUND=13, ACC_SPH=14, ACC_GRAV=15, H=16, N_LEAVES=17,
         IMPACT_DT=18, IMPACT_TIME=19)
MAX_IMPACTS = 256  # SPH_MAX_IMPACTS

KERNEL = dict(cubic=0, wendland=1)
GRAVITY = dict(tree=0, direct=1, none=2)

# 48-byte exchange layout (gpu_sph.rs:25-37) as a numpy structured dtype
PARTICLE_DTYPE = np.dtype([("pos", "<f4", (3,)), ("h", "<f4"), ("vel", "<f4", (3,)), ("u", "<f4"),
                           ("mass", "<f4"), ("mat", "<u4"), ("rho", "<f4"), ("prov", "<u4")])
assert PARTICLE_DTYPE.itemsize == 48


class SphConfig(C.Structure):
    _fields_ = [("G", C.c_double), ("theta", C.c_float), ("leaf_size", C.c_uint32), ("kernel", C.c_uint32),
                ("gravity", C.c_uint32), ("multipole", C.c_uint32), ("precision", C.c_uint32),
                ("h_mode", C.c_uint32), ("h_neighbours", C.c_float), ("h_tol", C.c_float),
                ("h_iters", C.c_uint32), ("max_neighbours", C.c_uint32), ("cfl", C.c_float),
                ("rho_floor", C.c_float), ("du_floor", C.c_float), ("r_min", C.c_float), ("sig_floor", C.c_float),
                ("device", C.c_int32), ("mac", C.c_uint32), ("graph", C.c_uint32),
                ("block_threads", C.c_uint32), ("walk_warps", C.c_uint32), ("h_skin", C.c_float),
                ("walk_stack", C.c_uint32), ("local_theta", C.c_float)]


class SphDiag(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("internal", C.c_double), ("potential", C.c_double),
                ("momentum", C.c_double * 3), ("angular_momentum", C.c_double * 3), ("mass", C.c_double),
                ("dt", C.c_double), ("time", C.c_double), ("steps", C.c_uint32),
                ("max_neighbours_seen", C.c_uint32), ("overflow_flags", C.c_uint32), ("h_iterations", C.c_uint32),
                ("h_residual", C.c_float), ("h_accepted", C.c_uint32), ("walk_nodes", C.c_uint64),
                ("walk_pops", C.c_uint64), ("m2p_interactions", C.c_uint64), ("p2p_interactions", C.c_uint64),
                ("local_expansions", C.c_uint64), ("p2p_slots", C.c_uint64)]


PHASES = ["sort", "tree", "gravity", "neighbours", "hsolve", "density", "forces", "integrate"]


class SphProfile(C.Structure):
    _fields_ = [("ms", C.c_double * 8), ("calls", C.c_uint64 * 8), ("kernel_launches", C.c_uint64)]


# Every symbol declared in include/sph_b200.h (checked by tests/test_abi.py).
EXPORTS = ["sph_config_default", "sph_create", "sph_destroy", "sph_upload", "sph_upload_batch", "sph_set_dt",
           "sph_set_av",
           "sph_set_omega", "sph_step_kdk", "sph_step_relax", "sph_eval_forces", "sph_readback_begin",
           "sph_readback_take", "sph_readback_into", "sph_sync", "sph_count", "sph_particle_buffer", "sph_diag", "sph_stream",
           "sph_last_error", "sph_status_string", "sph_inspect", "sph_profile_enable", "sph_profile_read",
           "sph_gravity", "sph_gravity_direct64", "sph_gravity_tree_noalloc", "sph_dem_create", "sph_dem_destroy",
           "sph_dem_replace", "sph_dem_set_params", "sph_dem_step", "sph_dem_readback", "sph_dem_contacts",
           "sph_dem_count", "sph_mlp_set", "sph_mlp_record", "sph_mlp_features", "sph_set_progress",
           "sph_mlp_forward", "sph_mlp_grad", "sph_mlp_train", "sph_measure_default", "sph_measure_disk",
           "sph_body_bulk", "sph_assemble", "sph_dem_set_ground", "sph_dem_set_terrain"]

H_MODE = dict(fixed=0, solve=1, learned=2)
MLP_PARAMS = 4819     # SPH_MLP_PARAMS
MLP_TRAINABLE = 4801  # SPH_MLP_TRAINABLE


class Placement(C.Structure):
    _fields_ = [("offset", C.c_double * 3), ("vel", C.c_double * 3), ("spin", C.c_double * 3)]


class MeasureCfg(C.Structure):
    _fields_ = [("variant", C.c_int32), ("reserved", C.c_int32), ("G", C.c_double), ("remnant_frac", C.c_double),
                ("link_factor", C.c_double), ("roche", C.c_double), ("rho_fallback", C.c_double),
                ("pe_floor", C.c_double), ("pe_softening", C.c_double)]


class DiskMeasure(C.Structure):
    _fields_ = [("earth_frac", C.c_double), ("disk_mass", C.c_double), ("disk_target", C.c_double),
                ("disk_impactor", C.c_double), ("remnant_target", C.c_double), ("remnant_impactor", C.c_double),
                ("escaped_target", C.c_double), ("escaped_impactor", C.c_double), ("r_remnant", C.c_double),
                ("m_remnant", C.c_double), ("clump_mass", C.c_double), ("clump_target_frac", C.c_double),
                ("clump_n", C.c_uint32), ("n_clumps", C.c_uint32), ("n_bound", C.c_uint32), ("n_disk", C.c_uint32)]


class MlpTrainCfg(C.Structure):
    _fields_ = [("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("weight_decay", C.c_float), ("seed", C.c_uint32)]

# 80-byte grain layout (particle_step.wgsl:127-137)
GRAIN_DTYPE = np.dtype([("offset", "<f4", (3,)), ("u", "<f4"), ("vel", "<f4", (3,)), ("resting", "<f4"),
                        ("color", "<f4", (3,)), ("material", "<f4"), ("emission", "<f4", (3,)), ("rho", "<f4"),
                        ("radius", "<f4"), ("_p", "<f4", (3,))])
assert GRAIN_DTYPE.itemsize == 80


class DemGround(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("air_rho", C.c_float), ("drag_cd", C.c_float),
                ("specific_heat", C.c_float), ("cool_rate", C.c_float), ("reserved", C.c_float)]


class DemParams(C.Structure):
    _fields_ = [("gravity", C.c_float * 3), ("dt", C.c_float), ("c_stiffness", C.c_float),
                ("c_normal_damp", C.c_float), ("c_friction", C.c_float), ("c_tangent_damp", C.c_float),
                ("c_cohesion", C.c_float), ("reserved", C.c_float * 3)]

_lib = None


def load():
    """Load the library (once). Raises RuntimeError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m botheadstudios_b200.build` "
                           "(nvcc, sm_100a). There is no CPU fallback.")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.sph_config_default.argtypes = [C.POINTER(SphConfig)]
    L.sph_create.argtypes = [C.POINTER(SphConfig), C.c_uint32, C.POINTER(vp)]
    L.sph_destroy.argtypes = [vp]
    L.sph_destroy.restype = None
    L.sph_upload.argtypes = [vp, vp, C.c_uint32, vp, C.c_uint32, C.c_float]
    L.sph_upload_batch.argtypes = [vp, vp, vp, C.c_uint32, vp, C.c_uint32, vp]
    L.sph_set_dt.argtypes = [vp, C.c_double, C.c_float]
    L.sph_set_av.argtypes = [vp, C.c_float, C.c_float]
    L.sph_set_omega.argtypes = [vp, C.c_float]
    L.sph_step_kdk.argtypes = [vp, C.c_uint32]
    L.sph_step_relax.argtypes = [vp, C.c_uint32]
    L.sph_eval_forces.argtypes = [vp]
    L.sph_readback_begin.argtypes = [vp]
    L.sph_readback_take.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_int)]
    L.sph_readback_into.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_uint32)]
    L.sph_sync.argtypes = [vp, C.c_uint32]
    L.sph_count.argtypes = [vp]
    L.sph_count.restype = C.c_uint32
    L.sph_particle_buffer.argtypes = [vp, C.POINTER(vp)]
    L.sph_diag.argtypes = [vp, C.POINTER(SphDiag)]
    L.sph_stream.argtypes = [vp]
    L.sph_stream.restype = vp
    L.sph_last_error.argtypes = [vp]
    L.sph_last_error.restype = C.c_char_p
    L.sph_status_string.argtypes = [C.c_int]
    L.sph_status_string.restype = C.c_char_p
    L.sph_inspect.argtypes = [vp, C.c_uint32, vp, C.c_size_t]
    L.sph_profile_enable.argtypes = [vp, C.c_int]
    L.sph_profile_read.argtypes = [vp, C.POINTER(SphProfile)]
    L.sph_gravity.argtypes = [vp, vp, vp, C.c_uint32, C.c_double, C.c_uint32, vp]
    L.sph_gravity_direct64.argtypes = [vp, vp, vp, C.c_uint32, vp, C.c_uint32, C.c_double, vp]
    L.sph_gravity_tree_noalloc.argtypes = [vp, C.c_uint32, C.c_double, C.c_float, C.c_float, C.c_uint32, C.c_uint32,
                                           vp, vp]
    L.sph_dem_create.argtypes = [C.c_uint32, C.c_int32, C.POINTER(vp)]
    L.sph_dem_destroy.argtypes = [vp]
    L.sph_dem_destroy.restype = None
    L.sph_dem_replace.argtypes = [vp, vp, C.c_uint32]
    L.sph_dem_set_params.argtypes = [vp, C.POINTER(DemParams)]
    L.sph_dem_step.argtypes = [vp, C.c_uint32]
    L.sph_dem_readback.argtypes = [vp, vp, C.c_uint32, C.POINTER(C.c_uint32)]
    L.sph_dem_contacts.argtypes = [vp, vp, C.c_size_t]
    L.sph_dem_set_ground.argtypes = [vp, C.POINTER(DemGround)]
    L.sph_dem_set_terrain.argtypes = [vp, vp, C.c_uint32, C.c_uint32]
    L.sph_mlp_set.argtypes = [vp, vp, C.c_uint32]
    L.sph_mlp_record.argtypes = [vp, C.c_int]
    L.sph_mlp_features.argtypes = [vp, vp, vp, C.c_uint32]
    L.sph_set_progress.argtypes = [vp, C.c_float]
    L.sph_mlp_forward.argtypes = [vp, vp, C.c_uint32, vp]
    L.sph_mlp_grad.argtypes = [vp, vp, vp, C.c_uint32, vp, vp]
    L.sph_mlp_train.argtypes = [vp, vp, vp, C.c_uint32, C.POINTER(MlpTrainCfg), vp]
    L.sph_dem_count.argtypes = [vp]
    L.sph_measure_default.argtypes = [C.POINTER(MeasureCfg)]
    L.sph_body_bulk.argtypes = [vp, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.sph_assemble.argtypes = [vp, C.POINTER(Placement), C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    L.sph_measure_disk.argtypes = [vp, C.c_uint32, C.POINTER(MeasureCfg), C.POINTER(DiskMeasure)]
    L.sph_dem_count.restype = C.c_uint32
    no_status = ("sph_destroy", "sph_count", "sph_stream", "sph_last_error", "sph_status_string", "sph_dem_destroy",
                 "sph_dem_count")
    for name in EXPORTS:
        if name not in no_status:
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def default_config(**kw) -> SphConfig:
    cfg = SphConfig()
    load().sph_config_default(C.byref(cfg))
    for k, v in kw.items():
        if isinstance(v, str):
            v = (H_MODE if k == "h_mode" else {**KERNEL, **GRAVITY})[v]
        setattr(cfg, k, v)
    return cfg
