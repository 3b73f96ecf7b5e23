"""ctypes binding of libwspm.so (declarations mirror include/wspm.h).

Importing this module loads the CUDA library built in-tree next to it.  There
is no fallback: if the library is missing or fails to load, the import raises
``RuntimeError`` so a GPU run can never silently compute on the host.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwspm.so")

WSPM_OK, WSPM_MAXITER, WSPM_NAN, WSPM_BREAKDOWN = 0, 1, 2, 3
WSPM_BAD_ARG, WSPM_CUDA_ERROR, WSPM_UNSUPPORTED = 10, 11, 12
SOLVERS = {"cg": 0, "bicgstab": 1, "gmres": 2}
PRECONDS = {"none": 0, None: 0, "jacobi": 1}
SOIL_VG, SOIL_EXP = 0, 1
NOALLOC_MAX_ROWS = 262144     # WSPM_NOALLOC_MAX_ROWS in include/wspm.h

c_int32, c_int64, c_double, c_void_p = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class WspmMesh(ctypes.Structure):
    _fields_ = [("n_nodes", c_int32), ("n_elems", c_int32), ("dim", c_int32), ("nv", c_int32),
                ("conn", c_void_p), ("coords", c_void_p)]


class WspmPattern(ctypes.Structure):
    _fields_ = [("n_rows", c_int32), ("n_slices", c_int32), ("max_width", c_int32), ("max_inc", c_int32),
                ("nnz_padded", c_int64),
                ("slice_ptr", c_void_p), ("slice_width", c_void_p), ("cols", c_void_p), ("diag_pos", c_void_p),
                ("inc_ptr", c_void_p), ("inc_width", c_void_p), ("inc_elem", c_void_p), ("inc_slots", c_void_p),
                ("n_diags", c_int32), ("pad_", c_int32), ("diag_offsets", c_void_p)]


class WspmEdges(ctypes.Structure):
    _fields_ = [("n_bnodes", c_int32), ("pad_", c_int32), ("node", c_void_p), ("e_cnt", c_void_p),
                ("e_local", c_void_p), ("e_other", c_void_p), ("e_kother", c_void_p), ("e_jac", c_void_p)]


class WspmPatternSizes(ctypes.Structure):
    _fields_ = [("n_rows", c_int32), ("n_slices", c_int32), ("max_width", c_int32), ("max_inc", c_int32),
                ("n_diags", c_int32), ("layout", c_int32), ("nnz", c_int64), ("nnz_padded", c_int64),
                ("n_inc", c_int64), ("ld", c_int64), ("diag_offsets", c_int32 * 64)]


class WspmPicardDesc(ctypes.Structure):
    _fields_ = [("mesh", ctypes.POINTER(WspmMesh)), ("pat", ctypes.POINTER(WspmPattern)),
                ("soil_model", c_int32), ("phi", c_double * 6), ("Ks_elem", c_void_p), ("bc_val", c_void_p),
                ("quad_points", c_double * 48), ("weights", c_double * 16), ("nq", c_int32),
                ("solver", c_int32), ("precond", c_int32), ("krylov_tol", c_double), ("krylov_maxiter", c_int32),
                ("restart", c_int32),
                ("mixed", c_int32), ("inner_tol", c_double), ("inner_maxiter", c_int32), ("refine_maxiter", c_int32),
                ("picard_tol", c_double), ("picard_maxiter", c_int32), ("picard_relative", c_int32),
                ("neumann", ctypes.POINTER(WspmEdges)), ("neumann_flux", c_double),
                ("drainage", ctypes.POINTER(WspmEdges)),
                ("h_n", c_void_p), ("theta_n", c_void_p), ("h_m", c_void_p), ("x", c_void_p),
                ("K", c_void_p), ("C", c_void_p), ("theta_m", c_void_p),
                ("vals", c_void_p), ("vals32", c_void_p), ("rhs", c_void_p), ("dinv", c_void_p),
                ("work", c_void_p), ("work_doubles", c_int64), ("dt_dev", c_void_p),
                ("result", c_void_p), ("result_f64", c_void_p), ("Ks_inc", c_void_p), ("shapes", c_void_p)]


class WspmEnsemble(ctypes.Structure):
    _fields_ = [("n_domains", c_int32), ("node_off", c_void_p), ("order", c_void_p), ("phi", c_void_p),
                ("Ks_elem", c_void_p), ("bc_val", c_void_p),
                ("quad_points", c_double * 48), ("weights", c_double * 16), ("nq", c_int32),
                ("krylov_tol", c_double), ("krylov_maxiter", c_int32),
                ("picard_tol", c_double), ("picard_maxiter", c_int32), ("picard_relative", c_int32),
                ("tmax", c_double), ("m_it", c_int32), ("M_it", c_int32), ("lambda_amp", c_double),
                ("lambda_red", c_double),
                ("h_n", c_void_p), ("work", c_void_p), ("work_doubles", c_int64), ("dt", c_void_p), ("t", c_void_p),
                ("its", c_void_p), ("kits", c_void_p), ("status", c_void_p), ("err", c_void_p),
                ("queue", c_void_p), ("cluster_size", c_int32)]


def _ptr(t):
    return ctypes.POINTER(t)


class WspmPatternHost(ctypes.Structure):
    _fields_ = [("n_rows", c_int32), ("n_slices", c_int32), ("max_width", c_int32), ("max_inc", c_int32),
                ("n_diags", c_int32), ("layout", c_int32), ("nnz", c_int64), ("nnz_padded", c_int64),
                ("n_inc", c_int64), ("ld", c_int64),
                ("csr_indptr", _ptr(c_int64)), ("csr_indices", _ptr(c_int32)), ("sell_index", _ptr(c_int64)),
                ("slice_ptr", _ptr(c_int64)), ("slice_width", _ptr(c_int32)), ("cols", _ptr(c_int32)),
                ("diag_pos", _ptr(c_int32)), ("diag_offsets", _ptr(c_int32)), ("inc_ptr", _ptr(c_int64)),
                ("inc_width", _ptr(c_int32)), ("inc_elem", _ptr(c_int32)), ("inc_slots", _ptr(ctypes.c_uint32))]


class WspmLevels(ctypes.Structure):
    _fields_ = [("n_levels", c_int32), ("level_ptr", c_void_p), ("rows", c_void_p)]


PRECOND_KIND = {"ilu": 2, "ssor": 3, "block_jacobi": 4, "ilu0": 5}
P = ctypes.POINTER
_SIGS = {
    "wspm_balance_workspace_doubles": (c_int64, []),
    "wspm_integrate_2d": (c_int32, [P(WspmMesh), c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_peclet_courant": (c_int32, [P(WspmMesh), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                                      c_void_p, c_void_p, c_void_p]),
    "wspm_ilu0_factor": (c_int32, [P(WspmPattern), c_void_p, P(WspmLevels), c_void_p, c_void_p]),
    "wspm_precond_apply": (c_int32, [P(WspmPattern), c_void_p, c_int32, c_double, c_int32, P(WspmLevels),
                                     P(WspmLevels), c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_ensemble_workspace_doubles": (c_int64, [c_int32, c_int64]),
    "wspm_elem_assemble_richards": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_double, c_double,
                                              P(c_double), P(c_double), c_int32, c_double, c_void_p, c_void_p,
                                              c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_elem_assemble_jt": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_double, c_double, P(c_double),
                                        P(c_double), c_int32, c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "wspm_elem_adjoint_rhs": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_double, c_double, P(c_double),
                                        P(c_double), c_int32, c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "wspm_elem_theta_node": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_double, c_double, P(c_double),
                                       P(c_double), c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_elem_param_grad": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_double, c_double, P(c_double),
                                       P(c_double), c_int32, c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_ensemble_step": (c_int32, [P(WspmMesh), P(WspmPattern), P(WspmEnsemble), c_int32, c_void_p]),
    "wspm_ensemble_run": (c_int32, [P(WspmMesh), P(WspmPattern), P(WspmEnsemble), c_int32, c_int32, c_void_p,
                                    c_void_p, c_void_p, c_void_p]),
    "wspm_soil_van_genuchten": (c_int32, [c_void_p, c_int64, P(c_double), c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_soil_exponential": (c_int32, [c_void_p, c_int64, P(c_double), c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_assemble_richards": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p,
                                         c_void_p, c_void_p, P(c_double), P(c_double), c_int32, c_double, c_void_p,
                                         c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_flux_dispersion_2d": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, P(c_double), c_double, c_double,
                                          c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p]),
    "wspm_assemble_adr_2d": (c_int32, [P(WspmMesh), P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_double, c_double,
                                       c_int32, P(c_double), P(c_double), c_int32, c_double, c_void_p, c_void_p,
                                       c_void_p, c_void_p]),
    "wspm_apply_edge_terms": (c_int32, [P(WspmPattern), P(WspmEdges), c_int32, c_double, c_double, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_spmv_f64": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_spmv_f32": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p]),
    "wspm_apply_dirichlet": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "wspm_jacobi_dinv": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_void_p]),
    "wspm_krylov_workspace_doubles": (c_int64, [c_int32, c_int32, c_int32]),
    "wspm_krylov_solve": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double,
                                    c_double, c_int32, c_int32, c_void_p, c_int64, c_void_p, c_void_p]),
    "wspm_krylov_mixed_workspace_doubles": (c_int64, [c_int32, c_int64, c_int32, c_int32]),
    "wspm_krylov_solve_mixed": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
                                          c_int32, c_double, c_double, c_int32, c_int32, c_void_p, c_int64, c_void_p,
                                          c_void_p]),
    "wspm_cg_iterations": (c_int32, [P(WspmPattern), c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_int32,
                                     c_void_p, c_int64, c_void_p, c_void_p]),
    "wspm_read_probe": (c_int32, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_void_p]),
    "wspm_cg_solve_noalloc": (c_int32, [P(WspmPattern), c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_double,
                                        c_int32, c_void_p, c_void_p]),
    "wspm_picard_workspace_doubles": (c_int64, [c_int32, c_int32]),
    "wspm_picard_ks_inc_doubles": (c_int64, [P(WspmPattern)]),
    "wspm_picard_shape_bytes": (c_int64, [P(WspmMesh), P(WspmPattern)]),
    "wspm_picard_create": (c_int32, [P(WspmPicardDesc), P(c_void_p)]),
    "wspm_picard_step": (c_int32, [c_void_p, c_void_p]),
    "wspm_picard_step_host": (c_int32, [c_void_p, c_void_p]),
    "wspm_picard_destroy": (c_int32, [c_void_p]),
    "wspm_picard_dia_live": (c_int64, [c_void_p]),
    "wspm_picard_shapes": (c_int32, [c_void_p]),
    "wspm_picard_assemble": (c_int32, [c_void_p, c_void_p]),
    "wspm_pattern_build": (c_int32, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_int64, c_int32,
                                     P(P(WspmPatternHost))]),
    "wspm_pattern_free": (None, [P(WspmPatternHost)]),
    "wspm_pattern_device_scratch_bytes": (c_int64, [c_int64, c_int32, c_int32]),
    "wspm_pattern_device_count": (c_int32, [c_void_p, c_int64, c_int32, c_int32, c_int32, c_void_p, c_int64,
                                            P(WspmPatternSizes), c_void_p]),
    "wspm_pattern_device_fill": (c_int32, [c_void_p, c_int64, c_int32, c_int32, P(WspmPatternSizes), c_void_p,
                                           c_int64] + [c_void_p] * 12 + [c_void_p]),
    "wspm_pattern_levels": (c_int32, [c_void_p, c_void_p, c_int32, c_int32, c_void_p, P(c_int32)]),
    "wspm_version": (ctypes.c_char_p, []),
    "wspm_status_string": (ctypes.c_char_p, [c_int32]),
}
EXPORTED = tuple(_SIGS)


def _load():
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libwspm.so not built at {LIB_PATH}; run __graft_entry__.build() "
                           "or python jax-wspm_b200/wspm_b200/build.py")
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise RuntimeError(f"failed to load {LIB_PATH}: {e}") from e
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class WspmError(RuntimeError):
    def __init__(self, fn, code):
        msg = lib.wspm_status_string(code).decode()
        super().__init__(f"{fn} failed: {msg} (status {code})")
        self.code = code


def check(fn, code):
    if code != WSPM_OK:
        raise WspmError(fn, code)
    return code


def dptr(t):
    """Device address of a torch tensor (or None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def dbl_array(values):
    arr = (c_double * max(len(values), 1))(*[float(v) for v in values])
    return arr
