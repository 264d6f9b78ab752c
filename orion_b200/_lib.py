"""ctypes binding of include/orion_gpu.h (liborion_gpu.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ORION_GPU_LIB") or os.path.join(HERE, "liborion_gpu.so")

PREC_FP64 = 0
PREC_MIXED = 1
SWEEP_PLANES, SWEEP_GRID, SWEEP_CLUSTER, SWEEP_TILES = 0, 1, 2, 3
SWEEP_NAMES = {SWEEP_PLANES: "planes", SWEEP_GRID: "grid", SWEEP_CLUSTER: "cluster", SWEEP_TILES: "tiles"}

FIELD_PRIM, FIELD_Q, FIELD_DQ, FIELD_METRICS, FIELD_VOL, FIELD_DT, FIELD_C, FIELD_MU = range(8)
FIELD_NCOMP = {FIELD_PRIM: 6, FIELD_Q: 5, FIELD_DQ: 5, FIELD_METRICS: 9, FIELD_VOL: 1, FIELD_DT: 1,
               FIELD_C: 1, FIELD_MU: 1}
FIELD_NAMES = {"prim": FIELD_PRIM, "q": FIELD_Q, "dq": FIELD_DQ, "metrics": FIELD_METRICS, "vol": FIELD_VOL,
               "dt": FIELD_DT, "c": FIELD_C, "mu": FIELD_MU}


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("gamma", "moo", "reynolds", "prl", "cfl", "twall", "tref", "visc",
                                          "roo", "uoo", "voo", "woo", "poo", "too")] + \
               [(n, C.c_int) for n in ("nvis", "method", "ntmst", "csrv")]


class Region(C.Structure):
    _fields_ = [("s_st", C.c_int * 3), ("s_ed", C.c_int * 3), ("bctype", C.c_int),
                ("t_st", C.c_int * 3), ("t_ed", C.c_int * 3), ("nbt", C.c_int), ("ibcwin", C.c_int)]


class BlockDesc(C.Structure):
    _fields_ = [("idim", C.c_int), ("jdim", C.c_int), ("kdim", C.c_int), ("nregions", C.c_int),
                ("regions", C.POINTER(Region))]


class Schedule(C.Structure):
    _fields_ = [("sweep_form", C.c_int), ("cluster_size", C.c_int), ("lanes", C.c_int), ("ms_per_step", C.c_float)]


class Residual(C.Structure):
    _fields_ = [("rms", C.c_double), ("max", C.c_double), ("max_loc", C.c_int * 5), ("pad", C.c_int),
                ("phydtime", C.c_double)]


XCHG_HALO, XCHG_IFACE = 0, 1


class ShardResidual(C.Structure):
    _fields_ = [("sum", C.c_double), ("max", C.c_double), ("key", C.c_longlong), ("dtmin", C.c_double),
                ("points", C.c_longlong)]


# every symbol the header declares, with its signature
SIGNATURES = {
    "orion_last_error": (C.c_char_p, []),
    "orion_abi_version": (C.c_int, []),
    "orion_gpu_init": (C.c_int, [C.c_int]),
    "orion_case_create": (C.c_int, [C.c_int, C.POINTER(BlockDesc), C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]),
    "orion_case_destroy": (C.c_int, [C.c_void_p]),
    "orion_case_set_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "orion_step_submit": (C.c_int, [C.c_void_p, C.c_int]),
    "orion_case_pack_output": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "orion_case_set_schedule": (C.c_int, [C.c_void_p, C.POINTER(Schedule)]),
    "orion_case_get_schedule": (C.c_int, [C.c_void_p, C.POINTER(Schedule)]),
    "orion_case_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Schedule), C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(Schedule)]),
    "orion_case_grid_metrics": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "orion_case_poll": (C.c_int, [C.c_void_p, C.POINTER(Residual), C.c_int, C.POINTER(C.c_int)]),
    "orion_io_put": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "orion_io_step": (C.c_int, [C.c_void_p, C.c_int]),
    "orion_io_get": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "orion_io_wait": (C.c_int, [C.c_void_p]),
    "orion_group_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "orion_group_submit": (C.c_int, [C.c_void_p, C.c_int]),
    "orion_group_sync": (C.c_int, [C.c_void_p]),
    "orion_group_step_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "orion_group_destroy": (C.c_int, [C.c_void_p]),
    "orion_case_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "orion_case_sync": (C.c_int, [C.c_void_p]),
    "orion_case_footprint": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    "orion_case_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "orion_case_step_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "orion_case_sweep_schedule": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "orion_footprint_estimate": (C.c_size_t, [C.c_int, C.POINTER(BlockDesc), C.c_int]),
    "orion_case_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "orion_case_download": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "orion_case_init_flow": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double]),
    "orion_grid_metrics_host": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_void_p, C.c_void_p]),
    "orion_exchange_bc": (C.c_int, [C.c_void_p]),
    "orion_apply_physical_bc": (C.c_int, [C.c_void_p]),
    "orion_update_flow_states": (C.c_int, [C.c_void_p]),
    "orion_calculate_time_step": (C.c_int, [C.c_void_p]),
    "orion_compute_viscous_rhs": (C.c_int, [C.c_void_p]),
    "orion_average_interface_residuals": (C.c_int, [C.c_void_p]),
    "orion_compute_inviscid_rhs": (C.c_int, [C.c_void_p]),
    "orion_update_solution": (C.c_int, [C.c_void_p]),
    "orion_residual_compute": (C.c_int, [C.c_void_p, C.POINTER(Residual)]),
    "orion_phydtime": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "orion_step": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Residual)]),
    "orion_step_async": (C.c_int, [C.c_void_p, C.c_int]),
    "orion_last_residual": (C.c_int, [C.c_void_p, C.POINTER(Residual)]),
    "orion_residual_block_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                               C.c_void_p, C.POINTER(Residual)]),
    "orion_case_create_shard": (C.c_int, [C.c_int, C.POINTER(BlockDesc), C.POINTER(C.c_int), C.c_int,
                                          C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]),
    "orion_shard_blocks": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "orion_shard_counts": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_longlong),
                                     C.POINTER(C.c_longlong)]),
    "orion_shard_pack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "orion_shard_unpack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "orion_shard_average_begin": (C.c_int, [C.c_void_p]),
    "orion_shard_average_end": (C.c_int, [C.c_void_p]),
    "orion_shard_residual": (C.c_int, [C.c_void_p, C.POINTER(ShardResidual)]),
    "orion_shard_plan_counts": (C.c_int, [C.c_int, C.POINTER(BlockDesc), C.POINTER(C.c_int), C.c_int, C.c_int,
                                          C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
}

_lib = None


class OrionError(RuntimeError):
    pass


def load(path: str = LIB_PATH) -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OrionError(f"native library missing: {path} (run python -m orion_b200.build)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = load().orion_last_error()
        raise OrionError(f"orion error {rc}: {msg.decode() if msg else ''}")
