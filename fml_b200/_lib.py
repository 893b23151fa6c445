"""ctypes binding of libfmlb.so (the C ABI declared in include/fmlb.h).

The library is the only compute path: if it is missing, or no CUDA device is
visible, every entry point raises. There is no CPU fallback.
"""

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfmlb.so")

_vp = ctypes.c_void_p
_i = ctypes.c_int
_ll = ctypes.c_longlong
_d = ctypes.c_double
_sz = ctypes.c_size_t
_dp = ctypes.POINTER(ctypes.c_double)

#: name -> (restype, argtypes) for every function in include/fmlb.h
SIGNATURES = {
    "fmlb_last_error_string": (ctypes.c_char_p, []),
    "fmlb_version": (_i, []),
    "fmlb_coulomb_matrices": (_i, [_vp, _vp, _vp, _i, _i, _vp, _i, _vp, _i, _vp, _vp, _vp]),
    "fmlb_vector_kernels_packed_f64": (_i, [_i, _vp, _vp, _i, _i, _vp, _vp, _i, _i, _i, _dp,
                                            _i, _vp, _vp, _vp]),
    "fmlb_segment_exp_sum_f64": (_i, [_vp, _ll, _i, _i, _vp, _i, _vp, _i, _d, _vp, _ll, _vp]),
    "fmlb_exp_colsum_scratch_doubles": (_sz, [_i]),
    "fmlb_exp_weighted_colsum_f64": (_i, [_vp, _ll, _i, _i, _d, _vp, _vp, _vp, _vp]),
    "fmlb_xyz_scan": (_i, [_vp, _i, _vp, _vp, _i]),
    "fmlb_xyz_parse": (_i, [_vp, _i, _vp, _vp, _vp, _i, _vp, _vp, _vp, _i]),
    "fmlb_unsorted_coulomb_matrices": (_i, [_vp, _vp, _vp, _i, _i, _vp, _i, _vp, _vp]),
    "fmlb_local_coulomb_matrices": (_i, [_vp, _vp, _vp, _i, _i, _i, _vp, _i, _vp, _vp]),
    "fmlb_vector_kernels_f64": (_i, [_i, _vp, _vp, _i, _i, _vp, _vp, _i, _i, _i, _dp, _i, _vp,
                                     _vp, _vp]),
    "fmlb_arad_descriptors": (_i, [_vp, _vp, _vp, _i, _i, _d, _vp, _vp, _vp]),
    "fmlb_gaussian_kernel_f64": (_i, [_vp, _i, _i, _vp, _i, _i, _i, _dp, _i, _vp, _ll, _ll, _i,
                                      _vp]),
    "fmlb_laplacian_kernel_f64": (_i, [_vp, _i, _i, _vp, _i, _i, _i, _dp, _i, _vp, _ll, _ll, _i,
                                       _vp]),
    "fmlb_arad_workspace_bytes": (_sz, [_i, _i, _i, _i]),
    "fmlb_arad_kernels": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _i, _i, _dp, _i, _d, _d, _d, _d,
                               _i, _i, _vp, _vp, _sz, _vp]),
    "fmlb_arad_atomic_workspace_bytes": (_sz, [_i, _i, _i]),
    "fmlb_arad_alpha_kernel_f64": (_i, [_vp, _vp, _vp, _i, _i, _d, _d, _vp, _vp, _sz, _vp]),
    "fmlb_arad_distances": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _i, _i, _d, _d, _d, _d, _vp,
                                 _vp, _sz, _vp]),
    "fmlb_arad_atomic_distances": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _i, _i, _d, _d, _d, _d,
                                        _vp, _vp, _sz, _vp]),
    "fmlb_arad_atomic_kernels": (_i, [_vp, _vp, _vp, _i, _vp, _vp, _vp, _i, _i, _dp, _i, _d, _d,
                                      _d, _d, _vp, _vp, _sz, _vp]),
    "fmlb_distance_matrix_f64": (_i, [_i, _vp, _i, _i, _vp, _i, _i, _i, _i, _d, _vp, _ll, _vp]),
    "fmlb_potrf_workspace_bytes": (_sz, [_i]),
    "fmlb_potrf_f64": (_i, [_vp, _ll, _i, _vp, _vp, _vp]),
    "fmlb_potri_f64": (_i, [_vp, _ll, _i, _vp, _vp, _ll, _vp, _vp]),
    "fmlb_potrs_f64": (_i, [_vp, _ll, _i, _vp, _vp, _vp]),
    "fmlb_syrk_lower_f64": (_i, [_vp, _ll, _i, _vp, _ll, _i, _i, _vp, _vp]),
    "fmlb_potrf_ozaki_workspace_bytes": (_sz, [_i, _i]),
    "fmlb_potrf_ozaki_f64": (_i, [_vp, _ll, _i, _i, _vp, _sz, _vp, _vp]),
    "fmlb_syrk_ozaki_workspace_bytes": (_sz, [_i, _i, _i]),
    "fmlb_syrk_lower_ozaki": (_i, [_vp, _ll, _i, _vp, _ll, _i, _i, _i, _vp, _sz, _vp, _vp]),
    "fmlb_tc_test_hooks": (_i, [_ll, _i]),
    "fmlb_get_diagonal_f64": (_i, [_vp, _ll, _i, _vp, _vp]),
    "fmlb_krr_refine_dd_scratch_doubles": (_sz, [_i]),
    "fmlb_krr_refine_dd": (_i, [_vp, _ll, _i, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp]),
    "fmlb_krr_refine_scratch_doubles": (_sz, [_i]),
    "fmlb_symmetrize_lower_f64": (_i, [_vp, _ll, _i, _vp]),
    "fmlb_krr_refine_f64": (_i, [_vp, _ll, _i, _d, _vp, _ll, _vp, _vp, _vp, _i, _vp, _vp, _vp]),
    "fmlb_add_diagonal_f64": (_i, [_vp, _ll, _i, _d, _vp]),
    "fmlb_gemv_f64": (_i, [_vp, _ll, _i, _i, _vp, _vp, _vp]),
    "fmlb_kernel_predict_workspace_bytes": (_sz, [_i, _i, _i]),
    "fmlb_kernel_predict_f64": (_i, [_i, _vp, _i, _i, _vp, _i, _i, _i, _dp, _i, _vp, _ll, _vp,
                                     _ll, _vp, _sz, _vp]),
    "fmlb_laplacian_kernel_f32": (_i, [_vp, _i, _i, _vp, _i, _i, _i, _dp, _i, _vp, _ll, _ll, _i,
                                       _vp]),
    "fmlb_tc_operand_bytes": (_sz, [_i, _i]),
    "fmlb_column_mean_f64": (_i, [_vp, _i, _i, _i, _vp, _vp]),
    "fmlb_gaussian_kernel_tc": (_i, [_vp, _i, _i, _vp, _i, _i, _i, _vp, _dp, _i, _vp, _ll, _ll,
                                     _i, _vp, _sz, _vp, _vp]),
    "fmlb_batch_problem_bytes": (_sz, []),
    "fmlb_batch_buffer_doubles": (_sz, [_i]),
    "fmlb_krr_batched_f64": (_i, [_vp, _vp, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _i, _vp]),
    "fmlb_kernel_predict_f64_noalloc": (_i, [_i, _vp, _i, _i, _vp, _i, _i, _i, _dp, _i, _vp, _ll,
                                             _vp, _ll, _vp]),
}

FMLB_EINVAL = -22
FMLB_ENOMEM = -12
FMLB_ECUDA = -5
FMLB_ENOTSUP = -95
FMLB_ETIMEDOUT = -110

_LIB = None


class FmlbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (code %d)" % (msg, code))
        self.code = code


def load(require_cuda=True):
    """Load libfmlb.so; raise if it (or, with require_cuda, a GPU) is missing."""
    global _LIB
    if require_cuda and not torch.cuda.is_available():
        raise RuntimeError("fml_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libfmlb.so is not built: run `python -m fml_b200.build` "
                               "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


# host-only entry points (no device work): callable without a GPU
HOST_ONLY = frozenset(["fmlb_xyz_scan", "fmlb_xyz_parse", "fmlb_tc_test_hooks"])


def call(name, *args):
    """Call an fmlb entry point and raise FmlbError on a negative return."""
    lib = load(require_cuda=name not in HOST_ONLY)
    rc = getattr(lib, name)(*args)
    if isinstance(rc, int) and rc < 0:
        msg = lib.fmlb_last_error_string().decode(errors="replace")
        if rc == FMLB_EINVAL:
            raise ValueError("%s: %s" % (name, msg))
        raise FmlbError(rc, "%s: %s" % (name, msg))
    return rc


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def host_doubles(values):
    arr = (ctypes.c_double * len(values))(*[float(v) for v in values])
    return ctypes.cast(arr, _dp), arr
