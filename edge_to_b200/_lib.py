"""ctypes binding of libedge_b200.so (include/edge_b200.h).

The library must be built (``python -m edge_to_b200.build``); there is no fallback:
loading fails loudly when the shared object is missing.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libedge_b200.so")

EDGE_OK, EDGE_EINVAL, EDGE_ECUDA, EDGE_ENOTPD, EDGE_ESTATE = 0, 1, 2, 3, 4
EDGE_FP64, EDGE_MIXED = 0, 1

_lib = None

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
vp = ctypes.c_void_p

_SIGS = {
    "edge_last_error": (ctypes.c_char_p, []),
    "edge_version": (ctypes.c_int, []),
    "edge_problem_create": (ctypes.c_int, [ctypes.c_int, c_int_p, c_double_p, ctypes.c_int, ctypes.POINTER(vp)]),
    "edge_problem_destroy": (ctypes.c_int, [vp]),
    "edge_set_stream": (ctypes.c_int, [vp, vp]),
    "edge_set_constraints": (ctypes.c_int, [vp, vp]),
    "edge_set_rho": (ctypes.c_int, [vp, vp]),
    "edge_matvec": (ctypes.c_int, [vp, vp, vp]),
    "edge_matvec_dense": (ctypes.c_int, [vp, vp, vp]),
    "edge_matvec_f32": (ctypes.c_int, [vp, vp, vp]),
    "edge_diagonal": (ctypes.c_int, [vp, vp]),
    "edge_process_grad": (ctypes.c_int, [vp, vp, vp]),
    "edge_process_grad_adjoint": (ctypes.c_int, [vp, vp, vp, vp]),
    "edge_set_springs": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), c_double_p]),
    "edge_uses_transform": (ctypes.c_int, [vp]),
    "edge_uses_cube_form": (ctypes.c_int, [vp]),
    "edge_set_tma": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_fine_tile": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    "edge_autotune_fine": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, c_double_p, c_int_p, c_int_p]),
    "edge_set_stencil_quad": (ctypes.c_int, [vp, ctypes.c_longlong]),
    "edge_set_coarse_bf16": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_residual32": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_pdl": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_mm_law": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, vp, c_double_p, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, vp, vp, vp]),
    "edge_set_stencil_pair": (ctypes.c_int, [vp, ctypes.c_longlong]),
    "edge_set_stencil_tiled": (ctypes.c_int, [vp, ctypes.c_longlong]),
    "edge_set_galerkin_axis": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_graph": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_mg_set_sweeps": (ctypes.c_int, [vp, c_int_p, ctypes.c_int]),
    "edge_mg_set_omega_carry": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_fuse": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_fuse_xr": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_set_rho_embedded": (ctypes.c_int, [vp, vp, c_int_p]),
    "edge_fine_kind_tiles": (ctypes.c_int, [vp, c_int_p, c_int_p]),
    "edge_set_kind_tune": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_oc_update_multi": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, vp, vp, vp, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_double, c_double_p, c_double_p, vp, vp]),
    "edge_mg_solve_embedded": (ctypes.c_int, [vp, c_int_p, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                              c_double_p, c_int_p]),
    "edge_set_tail": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_gen_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, c_int_p, c_int_p, c_double_p,
                                       ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(vp)]),
    "edge_gen_destroy": (ctypes.c_int, [vp]),
    "edge_gen_set_stream": (ctypes.c_int, [vp, vp]),
    "edge_gen_set_rho": (ctypes.c_int, [vp, vp]),
    "edge_gen_set_constraints": (ctypes.c_int, [vp, vp]),
    "edge_gen_matvec": (ctypes.c_int, [vp, vp, vp]),
    "edge_gen_diagonal": (ctypes.c_int, [vp, vp]),
    "edge_gen_process_grad": (ctypes.c_int, [vp, vp, vp]),
    "edge_gen_cg_solve": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, c_double_p,
                                         c_int_p]),
    "edge_csr_create": (ctypes.c_int, [ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong), c_int_p, c_double_p,
                                       ctypes.POINTER(vp)]),
    "edge_csr_destroy": (ctypes.c_int, [vp]),
    "edge_csr_apply": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, vp]),
    "edge_fea_integrals": (ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int, vp, vp, vp]),
    "edge_cg_solve": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, c_double_p, c_int_p]),
    "edge_launch_count": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_longlong)]),
    "edge_time_level": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, c_double_p]),
    "edge_time_fine": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      c_double_p]),
    "edge_mg_config": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      c_int_p, ctypes.c_int, ctypes.c_int]),
    "edge_mg_solve": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, c_double_p, c_int_p]),
    "edge_mg_setup": (ctypes.c_int, [vp]),
    "edge_mg_level_dense": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_longlong]),
    "edge_jacobi_sweep": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, ctypes.c_double, ctypes.c_int, vp]),
    "edge_restrict": (ctypes.c_int, [ctypes.c_int, c_int_p, vp, vp, vp]),
    "edge_prolong": (ctypes.c_int, [ctypes.c_int, c_int_p, vp, vp, vp]),
    "edge_filter_create": (ctypes.c_int, [ctypes.c_int, c_int_p, ctypes.c_int, c_int_p, c_double_p, ctypes.POINTER(vp)]),
    "edge_filter_destroy": (ctypes.c_int, [vp]),
    "edge_filter_apply": (ctypes.c_int, [vp, vp, vp, vp]),
    "edge_filter_apply_T": (ctypes.c_int, [vp, vp, vp, vp]),
    "edge_oc_update": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      vp, c_double_p, c_int_p, c_double_p]),
    "edge_oc_update_static": (ctypes.c_int, [ctypes.c_longlong, vp, vp, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_double, vp, c_double_p, c_int_p, c_double_p,
                                             vp]),
    "edge_simp_solve_and_process": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, ctypes.c_double, vp, vp, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_int, c_double_p, vp, vp, c_double_p,
                                                   c_int_p]),
    "edge_simp_iteration": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double, vp, vp, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int, vp, vp, vp, c_double_p, c_double_p, c_int_p,
                                           c_double_p, c_int_p, c_double_p]),
    "edge_batch_create": (ctypes.c_int, [ctypes.c_int, vp, vp, c_int_p, c_int_p, ctypes.POINTER(vp)]),
    "edge_batch_destroy": (ctypes.c_int, [vp]),
    "edge_batch_set_threads": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    "edge_batch_set_split": (ctypes.c_int, [vp, ctypes.c_longlong, ctypes.c_int]),
    "edge_batch_last_problem_times": (ctypes.c_int, [vp, c_double_p, c_double_p]),
    "edge_batch_last_times": (ctypes.c_int, [vp, c_double_p, c_double_p, c_double_p]),
    "edge_batch_oc_update": (ctypes.c_int, [vp, vp, vp, vp, vp, vp, ctypes.c_double, vp, c_double_p, c_int_p, vp]),
    "edge_batch_solve_and_process": (ctypes.c_int, [vp, vp, ctypes.c_double, ctypes.c_double, vp, vp, ctypes.c_int,
                                                    ctypes.c_double, ctypes.c_int, c_double_p, vp, c_double_p,
                                                    c_int_p, vp]),
    "edge_last_solve_stats": (ctypes.c_int, [vp, c_double_p, c_double_p, c_int_p, c_int_p]),
    "edge_profile_begin": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_breakdown_begin": (ctypes.c_int, [vp, ctypes.c_int]),
    "edge_breakdown_end": (ctypes.c_int, [vp, c_double_p, c_int_p, ctypes.c_int]),
    "edge_profile_end": (ctypes.c_int, [vp, c_double_p, c_double_p, c_int_p, ctypes.POINTER(ctypes.c_longlong)]),
}


def lib():
    """The loaded library (loads on first use)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m edge_to_b200.build` "
                               "(the CUDA path has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(code):
    if code == EDGE_OK:
        return
    msg = lib().edge_last_error().decode("utf-8", "replace")
    if code in (EDGE_EINVAL, EDGE_ESTATE):
        raise ValueError(msg)
    if code == EDGE_ENOTPD:
        raise RuntimeError("not positive definite: " + msg)
    raise RuntimeError(msg)


def call(name, *args):
    check(getattr(lib(), name)(*args))


def ptr(t):
    """Device pointer of a contiguous torch tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return vp(t.data_ptr())


def int_array(vals):
    arr = (ctypes.c_int * len(vals))(*[int(v) for v in vals])
    return arr


def double_array(vals):
    return (ctypes.c_double * len(vals))(*[float(v) for v in vals])


def stream_ptr():
    import torch
    return vp(torch.cuda.current_stream().cuda_stream)
