"""ctypes binding of libmagasm.so (the C ABI declared in include/magasm.h).

The library is built in place (``magpackage_b200/libmagasm.so``) by
``magpackage_b200.build.build()``. There is no CPU fallback: if the library is
missing or CUDA is unavailable, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmagasm.so")

MAG_OK = 0
SCHEDULE_TWO_PASS, SCHEDULE_ROW_BLOCKS, SCHEDULE_SHARED_ROW_BLOCKS = 0, 2, 3
SCHEDULE_NZ_ROW_BLOCKS, SCHEDULE_TILE_BLOCKS = 5, 6
_ERRNAMES = {-1: "MAG_E_ARG", -2: "MAG_E_RANGE", -3: "MAG_E_GEOMETRY", -4: "MAG_E_CUDA",
             -5: "MAG_E_TIMEOUT", -6: "MAG_E_NOMEM", -7: "MAG_E_UNSUPPORTED"}


class MagError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class MeshInfo(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("num_elements", C.c_int64), ("num_dofs", C.c_int64),
                ("nnz", C.c_int64), ("num_incidences", C.c_int64), ("max_row_nnz", C.c_int32),
                ("wide_positions", C.c_int32), ("signs_derived", C.c_int32), ("schedule", C.c_int32),
                ("tile_blocks", C.c_int32), ("tile_colors", C.c_int32), ("device_bytes", C.c_int64),
                ("shared_blocks", C.c_int32), ("reserved0", C.c_int32), ("nz_pass", C.c_int32),
                ("tile_evals_per_elem", C.c_double), ("tile_plan_ms", C.c_double)]


_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
_i64 = C.c_int64
_int = C.c_int

_PROTOS = {
    "mag_version": ([], _int),
    "mag_last_error": ([], C.c_char_p),
    "mag_sync": ([_vp], _int),
    "mag_generate_edges": ([_vp, _i64, _i64, _vp, _vp, _vp, C.POINTER(_i64), _vp], _int),
    "mag_mesh_create": ([_vp, _i64, _vp, _i64, _vp, _vp, _vp, _i64, C.POINTER(_vp), _vp], _int),
    "mag_mesh_destroy": ([_vp], _int),
    "mag_mesh_get_info": ([_vp, C.POINTER(MeshInfo)], _int),
    "mag_mesh_pattern": ([_vp, _vp, _vp, _vp], _int),
    "mag_mesh_set_option": ([_vp, _int, _i64], _int),
    "mag_mesh_tune": ([_vp, _vp, _vp, _vp, _int, _vp, C.POINTER(_int), C.POINTER(_int), _vp], _int),
    "mag_mesh_check": ([_vp, _vp], _int),
    "mag_mesh_set_quadrature": ([_vp, _dp, _int, _dp, _dp], _int),
    "mag_mesh_set_materials": ([_vp, _dp, _dp, _dp, _int, _dp, _int, _dp, _int, _dp, _dp, _dp], _int),
    "mag_assemble_jacobian": ([_vp, _vp, _vp, _vp, _int, _vp], _int),
    "mag_assemble_stiffness": ([_vp, _vp, _vp, _vp], _int),
    "mag_assemble_mass": ([_vp, _vp, _vp, _vp], _int),
    "mag_assemble_source": ([_vp, _vp, _vp, _vp], _int),
    "mag_assemble_winding": ([_vp, _int, _vp, _dp, C.c_double, _vp, _vp], _int),
    "mag_element_b": ([_vp, _vp, _vp, _vp, _vp], _int),
    "mag_element_nu": ([_vp, _vp, _vp, _vp, _vp], _int),
    "mag_assemble_hbfem": ([_vp, _vp, _vp, _int, _vp, _vp, _vp, _vp, _int, _vp, _vp, _vp, _vp], _int),
    "mag_assemble_jacobian_seeded": ([_vp, _vp, _vp, _vp, _vp, _vp], _int),
    "mag_seed_midpoint": ([_vp, _vp, _vp, C.c_double, _vp, _vp], _int),
    "mag_csr_spmv": ([_i64, _vp, _vp, _vp, _vp, _vp, _vp], _int),
    "mag_csr_apply_dirichlet": ([_i64, _vp, _vp, _vp, _vp, _vp, _vp], _int),
    "mag_pcg_create": ([_i64, C.POINTER(_vp)], _int),
    "mag_pcg_destroy": ([_vp], _int),
    "mag_pcg_set_aux": ([_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp], _int),
    "mag_pcg_solve": ([_vp, _vp, _vp, _vp, _vp, _vp, C.c_double, _int, C.POINTER(_int), _dp, C.POINTER(_int),
                       _vp], _int),
    "mag_batch_create": ([_vp, _int, _vp, _vp, _dp, _vp, C.POINTER(_vp), _vp], _int),
    "mag_batch_assemble": ([_vp, _vp], _int),
    "mag_batch_variants": ([], _int),
    "mag_batch_tuning": ([_vp, C.POINTER(_int), _dp, C.c_char_p, _int], _int),
    "mag_batch_select": ([_vp, _int], _int),
    "mag_batch_destroy": ([_vp], _int),
    "mag_mlp_num_params": ([], _int),
    "mag_mlp_create": ([C.POINTER(C.c_float), C.POINTER(_vp)], _int),
    "mag_mlp_destroy": ([_vp], _int),
    "mag_mlp_get_params": ([_vp, C.POINTER(C.c_float)], _int),
    "mag_mlp_set_params": ([_vp, C.POINTER(C.c_float)], _int),
    "mag_mlp_forward": ([_vp, _vp, _i64, _vp, _vp, _vp], _int),
    "mag_mlp_predict_nu": ([_vp, _vp, _i64, _vp, C.c_double, C.c_double, C.c_double, C.c_double, _vp, _vp],
                           _int),
    "mag_mlp_gradient": ([_vp, _vp, _vp, _i64, C.c_float, _vp, _vp, _vp, _vp], _int),
    "mag_mlp_train_step": ([_vp, _vp, _vp, _i64, C.c_float, _vp, _vp, _vp], _int),
    "mag_mlp_train_epoch": ([_vp, _vp, _vp, _i64, _vp, _i64, C.c_float, _vp, _vp, _vp, _vp, _vp, _vp], _int),
    "mag_mlp_check": ([_vp, _vp], _int),
    "mag_mlp_set_spin_limit": ([_vp, _i64], _int),
    "mag_csr_drop_zeros": ([_vp, _vp, _vp, _i64, _vp, _vp, _vp, C.POINTER(_i64), _vp], _int),
    "mag_mex_jacobian": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _i64, _dp, _int, _dp, _dp, _dp,
                          _dp, _int, _dp, _int, _dp, _int, _dp, _dp, _dp, _int, _dp, _dp, _dp, _dp,
                          _dp], _int),
    "mag_mex_curl_curl": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _int, _dp, _dp, _dp, _dp], _int),
    "mag_mex_mass": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _i64, _dp, _int, _dp, _dp, _dp, _dp], _int),
    "mag_mex_source": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _int, _dp, _dp, _dp], _int),
    "mag_mex_winding": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, C.c_double, _dp, _dp, C.c_double, _dp, _int,
                         _dp, _dp, _dp], _int),
    "mag_mex_jacobian_sparse": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _i64, _dp, _int, _dp, _dp, _dp,
                                 _dp, _int, _dp, _int, _dp, _int, _dp, _dp, _dp, _int, C.POINTER(_vp), _dp],
                                _int),
    "mag_mex_curl_curl_sparse": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _dp, _int, _dp, _i64, C.POINTER(_vp)],
                                 _int),
    "mag_mex_mass_sparse": ([_dp, _i64, _dp, _i64, _dp, _dp, _dp, _i64, _dp, _int, _dp, _i64, C.POINTER(_vp)],
                            _int),
    "mag_mex_cache_clear": ([], _int),
    "mag_sparse_info": ([_vp, C.POINTER(_i64), C.POINTER(_i64)], _int),
    "mag_sparse_copy": ([_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _dp], _int),
    "mag_sparse_destroy": ([_vp], _int),
    "mag_mex_jacobian_noalloc": ([_vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _dp, _int, _dp, _dp,
                                  _dp, _dp, _int, _dp, _int, _dp, _int, _dp, _dp, _dp, _int, _vp, _vp,
                                  _vp, _vp, _vp, _vp], _int),
}

_LIB = None


def exported_symbols():
    return sorted(_PROTOS)


def load(path: str = LIB_PATH):
    """Load the shared library and declare prototypes (no CUDA call is made)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -c 'import magpackage_b200.build as b; b.build()'`")
    lib = C.CDLL(path)
    for name, (args, res) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def lib():
    """The loaded library, after checking that a CUDA device is present."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("magpackage_b200 needs a CUDA device (sm_100a); there is no CPU path")
    return load()


def check(rc: int) -> None:
    if rc != MAG_OK:
        msg = _LIB.mag_last_error().decode() if _LIB is not None else ""
        raise MagError(rc, msg)


def dptr(a):
    """Pointer to a contiguous float64 numpy array, or None."""
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def sync(stream=None) -> None:
    """mag_sync: wait for the stream's enqueued work; raises MagError if it failed."""
    check(lib().mag_sync(stream_ptr(stream)))


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)
