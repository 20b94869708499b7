"""ctypes binding of ``libpsierra_b200.so`` (the C ABI declared in ``include/psierra_b200.h``).

The library is required: importing the product path without it raises, and there
is no CPU fallback for any kernel.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PSIERRA_B200_LIB") or os.path.join(_HERE, "libpsierra_b200.so")

PSX_OK = 0
PSX_ERR_ARG = 1
PSX_ERR_CUDA = 2
PSX_ERR_LIMIT = 3

PSX_WANT_F = 1
PSX_WANT_K = 2
PSX_LINEAR = 4
PSX_KV = 8
PSX_MASS = 32

PSX_FP64 = 0
PSX_FP32_MIXED = 1

PSX_PRECOND_NONE = 0
PSX_PRECOND_JACOBI = 1
PSX_PRECOND_BJACOBI = 2
PSX_PCG_NODAL = 0x100

_ERRORS = {
    PSX_ERR_ARG: "invalid argument",
    PSX_ERR_CUDA: "CUDA launch or copy failed",
    PSX_ERR_LIMIT: "mesh exceeds a kernel limit",
}

_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_f64 = ctypes.c_double

# name -> (argtypes); every function returns int except psx_status_bytes (size_t)
SIGNATURES: dict[str, list] = {
    "psx_graph_count": [_p, _i64, _i32, _i64, _p, _p],
    "psx_graph_fill": [_p, _i64, _i32, _i64, _p, _p, _p, _p, _p],
    "psx_csr_pattern": [_i64, _p, _p, _p, _p],
    "psx_block_lists": [_p, _i64, _i32, _i64, _p, _p, _p, _p],
    "psx_plan_count": [_p, _i64, _i32, _i64, _p, _p, _p],
    "psx_plan_fill": [_p, _i64, _i32, _i64, _p, _p, _i64, _p, _p, _p, _p, _p, _p, _p, _p, _p],
    "psx_task_count": [_p, _i32, _i32, _i32, _i32, _p],
    "psx_task_fill": [_p, _i32, _i32, _i32, _i32, _p, _p],
    "psx_work_bytes": [_p, _i32, _p, _p],
    "psx_tet4_assemble": [_p, _p, _p, _p, _p, _f64, _f64, _f64, _i32, _i32, _p, _p, _p, _i64, _p, _p],
    "psx_tet4_kv": [_p, _p, _p, _p, _p, _f64, _f64, _i32, _p, _p, _p, _i64, _p, _p],
    "psx_tet4_dr_step": [_p, _p, _p, _p, _p, _f64, _f64, _i32, _p, _p, _f64, _f64, _f64, _p, _p, _p, _p, _i64,
                         _p, _p],
    "psx_tet4_element_dets": [_p, _p, _p, _i64, _p, _p],
    "psx_tet10_assemble": [_p, _p, _p, _p, _p, _f64, _f64, _f64, _i32, _i32, _p, _p, _p, _i64, _p, _p],
    "psx_tet10_element_dets": [_p, _p, _p, _i64, _p, _p],
    "psx_pcg_work_bytes": [_i64, _i32, _p],
    "psx_csr_dirichlet": [_i64, _p, _p, _p, _i32, _p, _p],
    "psx_tet4_adjoint": [_p, _p, _p, _p, _p, _f64, _f64, _p, _p, _p, _p, _p, _i64, _p, _p],
    "psx_pcg": [_i64, _p, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, _p, _i64, _p, _p],
    "psx_pcg_enqueue": [_i64, _p, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, _p, _i64, _p, _p],
    "psx_segment_sumsq": [_i64, _p, _p, _p, _p],
    "psx_fbar_plan_count": [_i64, _p, _p, _p, _p],
    "psx_fbar_plan_fill": [_i64, _p, _p, _i64, _p, _p, _p, _p, _p, _p, _p, _p],
    "psx_fbar_work_doubles": [_i64, _i64, _i64],
    "psx_fbar_element": [_i64, _p, _p, _p, _f64, _f64, _p, _p, _p, _p],
    "psx_ecsw_work_doubles": [_i64, _i32],
    "psx_csr_spmv": [_i64, _p, _p, _p, _i32, _p, _f64, _f64, _p, _p],
    "psx_ecsw_evaluate": [_i64, _i32, _p, _p, _p, _p, _p, _p, _f64, _f64, _p, _p, _p, _i64, _p, _p],
    "psx_fbar_assemble": [_p, _i64, _i64, _p, _p, _f64, _f64, _p, _p, _p, _p, _i64, _p, _p, _i64, _p, _p, _p, _p, _p,
                          _p, _p, _p, _p, _p, _p, _p, _i64, _p, _p, _i64, _p, _p],
    "psx_tet4_assemble_effective": [_p, _p, _p, _p, _p, _f64, _f64, _f64, _f64, _f64, _f64, _f64, _i32, _i32, _p, _p,
                                    _p, _i64, _p, _p],
    "psx_tile_plan_fill": [_p, _i64, _i32, _i32, _p, _p, _i64, _p, _p, _i64, _p, _p, _p, _p, _p, _p],
    "psx_tile_meta_stride": [_i32],
    "psx_tet4_split_ready": [],
    "psx_fma_roof": [_i32, _i64, _i32, _p, _p, _p],
    "psx_fma_roof_sink_bytes": [_i32],
    "psx_coarse_probe": [_p, _p, _i32, _i32, _p, _p],
    "psx_coarse_restrict": [_p, _p, _p, _p],
    "psx_pcg_coarse": [_i64, _p, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, _p, _p, _i64, _p, _p, _i32],
    "psx_pcg_batched_work_bytes": [_i64, _i32, _p],
    "psx_pcg_batched": [_i64, _p, _p, _p, _i32, _p, _p, _f64, _f64, _i32, _i32, _i32, _p, _p, _p, _p, _i64, _p, _p,
                        _p],
}



class PlanStruct(ctypes.Structure):
    """Mirror of ``psx_plan_t`` (include/psierra_b200.h)."""

    _fields_ = [
        ("npe", ctypes.c_int32),
        ("n_granules", ctypes.c_int32),
        ("n_elements", ctypes.c_int64),
        ("n_nodes", ctypes.c_int64),
        ("n_pairs", ctypes.c_int64),
        ("granule", ctypes.c_int64),
        ("max_span", ctypes.c_int64),
        ("conn", ctypes.c_void_p),
        ("pair_info", ctypes.c_void_p),
        ("pair_ptr", ctypes.c_void_p),
        ("pair_src", ctypes.c_void_p),
        ("node_info", ctypes.c_void_p),
        ("node_ptr", ctypes.c_void_p),
        ("node_src", ctypes.c_void_p),
        ("pair_gptr", ctypes.c_void_p),
        ("node_gptr", ctypes.c_void_p),
        ("tile", ctypes.c_int32),
        ("lag", ctypes.c_int32),
        ("tile_items", ctypes.c_int32),
        ("blocks_per_sm", ctypes.c_int32),
        ("n_tasks_k", ctypes.c_int64),
        ("n_tasks_f", ctypes.c_int64),
        ("tasks_k", ctypes.c_void_p),
        ("tasks_f", ctypes.c_void_p),
        ("btiles_k", ctypes.c_void_p),
        ("btiles_f", ctypes.c_void_p),
        ("ring_slack", ctypes.c_int32),
        ("lag_f", ctypes.c_int32),
        ("tile_cap_pairs", ctypes.c_int32),
        ("tile_cap_nodes", ctypes.c_int32),
        ("tile_meta", ctypes.c_void_p),
        ("pair_ptr_t", ctypes.c_void_p),
        ("pair_src_t", ctypes.c_void_p),
        ("node_ptr_t", ctypes.c_void_p),
        ("node_src_t", ctypes.c_void_p),
        ("n_gtasks_k", ctypes.c_int64),
        ("gtasks_k", ctypes.c_void_p),
        ("wait_spins", ctypes.c_int32),
        ("reserved0", ctypes.c_int32),
    ]


class CoarseStruct(ctypes.Structure):
    """Mirror of ``psx_coarse_t`` (include/psierra_b200.h)."""

    _fields_ = [
        ("n_nodes", ctypes.c_int64),
        ("n_agg", ctypes.c_int64),
        ("node_agg", ctypes.c_void_p),
        ("agg_ptr", ctypes.c_void_p),
        ("agg_nodes", ctypes.c_void_p),
        ("d", ctypes.c_void_p),
        ("fixed", ctypes.c_void_p),
        ("n_blocks", ctypes.c_int32),
        ("nc", ctypes.c_int32),
        ("block_agg", ctypes.c_void_p),
        ("ainv", ctypes.c_void_p),
        ("rc", ctypes.c_void_p),
        ("yc", ctypes.c_void_p),
    ]


_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """Load (once) and return the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m psierra_b200.build` "
                "(psierra_b200 has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = argtypes
            fn.restype = ctypes.c_int
        L.psx_status_bytes.argtypes = []
        L.psx_status_bytes.restype = ctypes.c_size_t
        L.psx_tile_meta_stride.restype = ctypes.c_int64
        L.psx_fbar_work_doubles.restype = ctypes.c_int64
        L.psx_ecsw_work_doubles.restype = ctypes.c_int64
        L.psx_fma_roof_sink_bytes.restype = ctypes.c_int64
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != PSX_OK:
        raise RuntimeError(f"{what} failed: {_ERRORS.get(rc, 'error')} (code {rc})")


def ptr(t) -> int | None:
    """Raw address of a torch tensor or numpy array (None stays NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data
