"""ctypes binding of the CUDA library ``librbb200.so`` (C ABI in
``include/redbird_b200.h``).

The library is required: importing the compute functions of this package on a
machine where it is missing or cannot be loaded raises immediately, there is
no CPU fallback.  Device memory, streams and tensors come from PyTorch; the
library receives raw pointers plus the current CUDA stream.
"""

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librbb200.so")

RB_OK, RB_EARG, RB_ECUDA, RB_ESIZE, RB_ENOCONV, RB_EBREAKDOWN, RB_ENOTSPD = range(7)
RB_F64, RB_C128, RB_F32, RB_C64 = range(4)
RB_PROP_NODE, RB_PROP_ELEM = 0, 1
RB_MIXED, RB_FP64 = 0, 1
RB_JAC_MUA_REF, RB_JAC_MUA_NODAL, RB_JAC_D = 0, 1, 2
RB_JAC_SPLIT_F32, RB_JAC_SPLIT_F64, RB_JAC_SPLIT_BF16, RB_JAC_BF16 = 4, 5, 6, 7
RB_JAC_SPLIT_F32_ACC64, RB_JAC_F32_ACC64 = 8, 9

_i64, _i32, _vp, _dbl, _sz = ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_double, ctypes.c_size_t


class RbMesh(ctypes.Structure):
    _fields_ = [("nn", _i64), ("ne", _i64), ("nf", _i64), ("nnz", _i64),
                ("node", _vp), ("elem", _vp), ("face", _vp), ("area", _vp),
                ("node_eptr", _vp), ("node_elist", _vp), ("node_fptr", _vp), ("node_flist", _vp),
                ("indptr", _vp), ("indices", _vp), ("inc_slot", _vp), ("slot_mask", _vp)]


class RbOptics(ctypes.Structure):
    _fields_ = [("kind", _i32), ("mua", _vp), ("musp", _vp), ("nref", _vp),
                ("nref_scalar", _dbl), ("omega", _dbl), ("reff", _dbl)]


class RbCsr(ctypes.Structure):
    _fields_ = [("n", _i64), ("nnz", _i64), ("indptr", _vp), ("indices", _vp), ("val64", _vp),
                ("val32", _vp), ("dinv64", _vp), ("dinv32", _vp), ("is_complex", _i32)]


class RbCoarse(ctypes.Structure):
    _fields_ = [("nc", _i64), ("agg", _vp), ("agg_ptr", _vp), ("agg_rows", _vp)]


class RbRowGroups(ctypes.Structure):
    _fields_ = [("ng", _i64), ("rows", _vp), ("uptr", _vp), ("ucol", _vp), ("umask", _vp), ("nu", _i64),
                ("coef", _vp)]


class RbInstances(ctypes.Structure):
    _fields_ = [("ninst", _i64), ("row_ptr", _vp), ("row_inst", _vp), ("status", _vp), ("relres", _vp)]


class RbSolveOpts(ctypes.Structure):
    _fields_ = [("precision", _i32), ("max_outer", _i32), ("maxiter", _i32), ("check_every", _i32),
                ("tol", _dbl), ("inner_tol", _dbl), ("profile", _i32), ("use_x0", _i32),
                ("coarse", ctypes.POINTER(RbCoarse)), ("groups", ctypes.POINTER(RbRowGroups)),
                ("instances", ctypes.POINTER(RbInstances)), ("spmm_lanes", _i32)]


class RbSolveInfo(ctypes.Structure):
    _fields_ = [("iters", _i32), ("outer", _i32), ("flag", _i32), ("launches", _i32), ("relres", _dbl),
                ("spmm_ms", _dbl), ("update_ms", _dbl), ("spmm_launches", _i32), ("update_launches", _i32),
                ("coarse_ms", _dbl), ("coarse_launches", _i32), ("sweep_iters_max", _i32)]


_SIGS = {
    "rb_last_error": (ctypes.c_char_p, []),
    "rb_version": (ctypes.c_int, []),
    "rb_incidence_work_bytes": (_sz, [_i64, _i32, _i64]),
    "rb_incidence": (ctypes.c_int, [_vp, _i32, _i64, _i64, _vp, _vp, _vp, _sz, _vp]),
    "rb_csr_pattern_work_bytes": (_sz, [_i64]),
    "rb_csr_pattern_count": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp, _vp, _sz, _vp]),
    "rb_csr_pattern_fill": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "rb_assembly_tables": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "rb_femlhs_work_bytes": (_sz, [_i64, _i64]),
    "rb_instances_work_bytes": (_sz, [_i64, _i64]),
    "rb_femlhs": (ctypes.c_int, [ctypes.POINTER(RbMesh), ctypes.POINTER(RbOptics), _vp, _vp, _vp, _vp, _vp, _vp,
                                 _vp, _sz, _vp]),
    "rb_femlhs_noalloc": (ctypes.c_int, [ctypes.POINTER(RbMesh), ctypes.POINTER(RbOptics), _vp, _vp, _vp, _vp, _vp,
                                         _vp, _vp]),
    "rb_deldotdel": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, _vp]),
    "rb_reorient": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp, _vp]),
    "rb_volface_work_bytes": (_sz, [_i64]),
    "rb_volface": (ctypes.c_int, [_vp, _i64, _i64, _vp, ctypes.POINTER(_i64), _vp, _sz, _vp]),
    "rb_face_area": (ctypes.c_int, [_vp, _vp, _i64, _vp, _vp]),
    "rb_nodevolume": (ctypes.c_int, [_i64, _vp, _vp, _vp, _vp, _vp]),
    "rb_tsearch": (ctypes.c_int, [_vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp]),
    "rb_point_rhs": (ctypes.c_int, [_vp, _vp, _vp, _i64, _i64, _i64, _i64, _vp, _vp]),
    "rb_prop_from_labels": (ctypes.c_int, [_vp, _i64, _vp, _i64, _i32, _vp, _vp, _vp]),
    "rb_adjoint_fields": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _i32, _vp, _vp]),
    "rb_femgetdet": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp, _i64, _i64, _i32, _vp, _vp]),
    "rb_wide_rhs": (ctypes.c_int, [_vp, _i64, _i64, _i64, _i64, _i64, _vp, _vp]),
    "rb_wide_getdet_work_bytes": (_sz, [_i64, _i64, _i32]),
    "rb_wide_getdet": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _i64, _i64, _i32, _vp, _vp, _sz, _vp]),
    "rb_femsolve_work_bytes": (_sz, [_i64, _i64, _i64, _i32, _i32]),
    "rb_coarse_work_bytes": (_sz, [_i64, _i64, _i32, _i32]),
    "rb_coarse_aggregate_work_bytes": (_sz, [_i64, _i64]),
    "rb_coarse_aggregate": (ctypes.c_int, [_vp, _i64, _dbl, _dbl, _dbl, _dbl, _i32, _i32, _i32, _vp, _vp, _vp,
                                           ctypes.POINTER(_i64), _vp, _sz, _vp]),
    "rb_rowgroups_work_bytes": (_sz, [_i64, _i64]),
    "rb_rowgroups_bin": (ctypes.c_int, [_vp, _i64, _dbl, _dbl, _dbl, _dbl, _i32, _i32, _i32, _vp,
                                        ctypes.POINTER(_i64), _vp, _sz, _vp]),
    "rb_rowgroups_union_work_bytes": (_sz, [_i64]),
    "rb_rowgroups_union_count": (ctypes.c_int, [ctypes.POINTER(RbCsr), _vp, _i64, _vp, ctypes.POINTER(_i64), _vp,
                                                _sz, _vp]),
    "rb_rowgroups_union_fill": (ctypes.c_int, [ctypes.POINTER(RbCsr), _vp, _i64, _vp, _vp, _vp, _vp]),
    "rb_femsolve": (ctypes.c_int, [ctypes.POINTER(RbCsr), _vp, _vp, _i64, ctypes.POINTER(RbSolveOpts),
                                   ctypes.POINTER(RbSolveInfo), _vp, _sz, _vp]),
    "rb_csr_prepare": (ctypes.c_int, [ctypes.POINTER(RbCsr), _vp, _vp, _vp, _vp]),
    "rb_spmm": (ctypes.c_int, [ctypes.POINTER(RbCsr), _i32, _vp, _vp, _i64, _vp]),
    "rb_jac": (ctypes.c_int, [ctypes.POINTER(RbMesh), _i32, _vp, _i32, _i64, _vp, _i32, _i32, _i32, _vp, _vp,
                              _i64, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _vp]),
    "rb_jac_tensor_cores": (ctypes.c_int, [_i32]),
    "rb_jac_status": (ctypes.c_int, [_vp]),
    "rb_jac_range": (ctypes.c_int, [ctypes.POINTER(RbMesh), _i32, _vp, _i32, _i64, _vp, _i32, _i32, _i32, _vp,
                                    _vp, _i64, _vp, _i64, _i32, _i32, _i32, _vp, _vp, _i64, _i64, _vp]),
    "rb_jac_remap": (ctypes.c_int, [_vp, _i32, _i64, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _vp]),
    "rb_jac_block": (ctypes.c_int, [_vp, _i32, _i64, _i64, _i64, _dbl, _dbl, _vp, _vp, _i64, _i64, _i64, _i64, _vp]),
    "rb_jac_elem": (ctypes.c_int, [ctypes.POINTER(RbMesh), _vp, _vp, _i32, _i64, _vp, _vp, _i64, _vp, _vp]),
    "rb_gram_work_bytes": (_sz, []),
    "rb_gram": (ctypes.c_int, [_vp, _vp, _i64, _i64, _i64, _dbl, _vp, _i64, _vp, _sz, _vp]),
    "rb_gram_bf16": (ctypes.c_int, [_vp, _i64, _i64, _i64, _dbl, _vp, _i64, _vp, _sz, _vp]),
    "rb_gram_stage_bytes": (_sz, [_i64, _i64, _i64, _i32, _i32]),
    "rb_gram_staged": (ctypes.c_int, [_vp, _vp, _i64, _i64, _i64, _dbl, _vp, _i64, _vp, _sz, _vp, _sz, _vp]),
    "rb_gram_bf16_staged": (ctypes.c_int, [_vp, _i64, _i64, _i64, _dbl, _vp, _i64, _vp, _sz, _vp, _sz, _vp]),
    "rb_split_tf32": (ctypes.c_int, [_vp, _vp, _i64, _i64, _i64, _vp]),
    "rb_reginv_prepare": (ctypes.c_int, [_vp, _i64, _i64, _dbl, _vp, _vp]),
    "rb_cholesky_work_bytes": (_sz, []),
    "rb_cholesky": (ctypes.c_int, [_vp, _i64, _i64, _vp, _sz, _vp]),
    "rb_chol_solve_work_bytes": (_sz, [_i64]),
    "rb_chol_solve": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp, _sz, _vp]),
    "rb_gemv_t_work_bytes": (_sz, [_i64]),
    "rb_gemv_t": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _dbl, _dbl, _vp, _vp, _sz, _vp]),
    "rb_gemv_t_bf16": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _dbl, _dbl, _vp, _vp, _sz, _vp]),
    "rb_sumsq_work_bytes": (_sz, []),
    "rb_sumsq": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _vp, _sz, _vp]),
    "rb_sumsq_bf16": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _vp, _sz, _vp]),
    "rb_vec_mul": (ctypes.c_int, [_vp, _vp, _vp, _i64, _vp]),
    "rb_row_sumsq": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _vp, _vp]),
    "rb_row_sumsq_bf16": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _vp, _vp]),
    "rb_set_diag": (ctypes.c_int, [_vp, _i64, _i64, _vp, _dbl, _vp]),
    "rb_row_sumsq_to_bf16": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _vp, _vp, _i64, _vp]),
    "rb_gemv_n_work_bytes": (_sz, [_i64, _i64]),
    "rb_gemv_n": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _dbl, _dbl, _vp, _vp, _sz, _vp]),
    "rb_gemv_n_bf16": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _dbl, _dbl, _vp, _vp, _sz, _vp]),
    "rb_axpby": (ctypes.c_int, [_i64, _dbl, _vp, _dbl, _vp, _vp]),
    "rb_dot_work_bytes": (_sz, []),
    "rb_dot": (ctypes.c_int, [_i64, _vp, _vp, _vp, _vp, _sz, _vp]),
}

_lib = None


class RedbirdError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


def lib():
    """Load (once) and return the CUDA library; raises if it is unavailable."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"redbirdpy_b200 CUDA library not built ({LIB_PATH} missing); run "
                "`python redbirdpy_b200/csrc/build.py` (or __graft_entry__.build())")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def exported_symbols():
    return list(_SIGS)


def call(name, *args):
    """Call ``name`` from the library and raise RedbirdError on a bad status."""
    code = getattr(lib(), name)(*args)
    if code != RB_OK:
        raise RedbirdError(name, code, lib().rb_last_error().decode())
    return code


def ptr(t):
    """Raw device (or host) address of a tensor, None for None."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream():
    """The current CUDA stream as the void* the C ABI expects."""
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("redbirdpy_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists")
    lib()
    return torch.device("cuda", torch.cuda.current_device())
