"""Python mirror of the B200 GLR library's C ABI (include/lgh_b200.h).

A thin ctypes layer over ``liblgh_b200.so``: the same objects and calls as
the reference's C API (lgh_prior_* / lgh_glr_*, include/lgpsf_hessian/
prior.h and glr.h), with numpy arrays in and out.  Every call goes to the
CUDA library; there is no CPU implementation here, and importing this
module without the built library raises.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "liblgh_b200.so")

P = ctypes.c_void_p
I64 = ctypes.c_int64
c_dbl_p = ctypes.POINTER(ctypes.c_double)

LGH_MEM_HOST, LGH_MEM_DEVICE = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
CHECK_PROJ, CHECK_APPLY = 0, 1
PC_AMG, PC_JACOBI = 0, 1
ERR_NAMES = {0: "SUCCESS", 55: "ERR_MEM", 56: "ERR_SUP", 58: "ERR_ORDER",
             60: "ERR_ARG_SIZ", 62: "ERR_ARG_WRONG",
             63: "ERR_ARG_OUTOFRANGE", 73: "ERR_ARG_WRONGSTATE",
             76: "ERR_LIB", 82: "ERR_CONV_FAILED", 85: "ERR_ARG_NULL",
             91: "ERR_NOT_CONVERGED",
             97: "ERR_GPU"}


class LghError(RuntimeError):
    def __init__(self, code, where, msg):
        super().__init__("%s failed: %s (%d): %s"
                         % (where, ERR_NAMES.get(code, "?"), code, msg))
        self.code = code


class GlrOpts(ctypes.Structure):
    """lgh_glr_opts_t, field for field (include/lgpsf_hessian/glr.h:68-86)."""

    _fields_ = [("ell", ctypes.c_int), ("q_power", ctypes.c_int),
                ("trunc_abs", ctypes.c_double),
                ("trunc_rel", ctypes.c_double), ("treat", ctypes.c_int),
                ("seed", ctypes.c_ulong), ("backend", ctypes.c_int),
                ("nb", ctypes.c_int), ("panel", ctypes.c_int),
                ("grid2d", ctypes.c_int), ("check", ctypes.c_int)]


class GlrReport(ctypes.Structure):
    """lgh_glr_report_t (include/lgpsf_hessian/glr.h:90-102)."""

    _fields_ = [("kept", ctypes.c_int), ("lam_abs_max", ctypes.c_double),
                ("lam_raw_min", ctypes.c_double),
                ("lam_raw_max", ctypes.c_double),
                ("next_abs", ctypes.c_double),
                ("n_negative_raw", ctypes.c_int),
                ("resid_max", ctypes.c_double),
                ("t_operator", ctypes.c_double),
                ("t_dense", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PriorMatOpts(ctypes.Structure):
    """lgh_prior_mat_opts_t (include/lgpsf_hessian/prior.h:76-89)."""

    _fields_ = [("ksp_rtol", ctypes.c_double),
                ("blocked_mode", ctypes.c_int), ("tile", ctypes.c_int),
                ("cheb_rtol", ctypes.c_double),
                ("smax_krylov", ctypes.c_int),
                ("smoother_top", ctypes.c_double),
                ("nu_force", ctypes.c_int), ("verbose", ctypes.c_int)]


class ExecOpts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int),
                ("inner_rtol", ctypes.c_double),
                ("verbose", ctypes.c_int), ("rank_cap", ctypes.c_int),
                ("check_form", ctypes.c_int)]


ALLGATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_size_t, ctypes.c_void_p)


class Comm(ctypes.Structure):
    """lgh_comm_t: the communicator of a column-sharded build."""
    _fields_ = [("rank", ctypes.c_int), ("size", ctypes.c_int),
                ("send", ctypes.c_void_p), ("recv", ctypes.c_void_p),
                ("bytes", ctypes.c_size_t), ("allgather", ALLGATHER_FN),
                ("ctx", ctypes.c_void_p)]


ROWS_ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.c_void_p)
ROWS_ALLTOALLV_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.c_void_p,
                                     ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.c_void_p)


class RowsComm(ctypes.Structure):
    """lgh_rows_comm_t: the communicator of a build over row slabs."""
    _fields_ = [("rank", ctypes.c_int), ("size", ctypes.c_int),
                ("allreduce", ROWS_ALLREDUCE_FN),
                ("alltoallv", ROWS_ALLTOALLV_FN), ("ctx", ctypes.c_void_p)]


class ServerOpts(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("hbm_reserve", ctypes.c_double),
                ("verbose", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_long), ("columns", ctypes.c_long),
                ("ticks", ctypes.c_long), ("pending", ctypes.c_long),
                ("p50_s", ctypes.c_double), ("p99_s", ctypes.c_double),
                ("max_s", ctypes.c_double), ("columns_per_s", ctypes.c_double),
                ("t_admit_s", ctypes.c_double), ("t_tick_s", ctypes.c_double),
                ("t_harvest_s", ctypes.c_double), ("harvests", ctypes.c_long),
                ("t_up_s", ctypes.c_double), ("t_down_s", ctypes.c_double),
                ("occupancy", ctypes.c_double),
                ("wait_stage_s", ctypes.c_double),
                ("wait_admit_s", ctypes.c_double), ("run_s", ctypes.c_double),
                ("copy_out_s", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GlrStats(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("ell", ctypes.c_int),
                ("kept", ctypes.c_int), ("precision", ctypes.c_int),
                ("t_build", ctypes.c_double), ("t_sketch", ctypes.c_double),
                ("t_zsolve", ctypes.c_double), ("t_spmm", ctypes.c_double),
                ("t_orth", ctypes.c_double), ("t_eig", ctypes.c_double),
                ("t_check", ctypes.c_double),
                ("zsolve_calls", ctypes.c_long),
                ("zsolve_iters", ctypes.c_long),
                ("zsolve_mean_col_iters", ctypes.c_double),
                ("device_bytes", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CorrectOpts(ctypes.Structure):
    """lgh_glr_correct_opts_t (include/lgpsf_hessian/glr.h:200-225)."""

    _fields_ = [("c0", ctypes.c_double), ("rank", ctypes.c_int),
                ("applies", ctypes.c_int), ("n_qc", ctypes.c_int),
                ("q_power", ctypes.c_int), ("clamp_eps", ctypes.c_double),
                ("d_keep_min", ctypes.c_double), ("drop_tol", ctypes.c_double),
                ("seed", ctypes.c_ulong), ("verbose", ctypes.c_int)]


class CorrectReport(ctypes.Structure):
    """lgh_glr_correct_report_t (include/lgpsf_hessian/glr.h:229-242)."""

    _fields_ = [("kept", ctypes.c_int), ("basis", ctypes.c_int),
                ("clamped", ctypes.c_int), ("hd_applies", ctypes.c_int),
                ("d_min", ctypes.c_double), ("d_max", ctypes.c_double),
                ("floor", ctypes.c_double), ("qc_before", ctypes.c_double),
                ("qc_after", ctypes.c_double), ("t_operator", ctypes.c_double),
                ("t_dense", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


HESS_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double),
                           ctypes.POINTER(ctypes.c_double), P)

VEC_FN = ctypes.CFUNCTYPE(None, P, P, P)
MAT_FN = ctypes.CFUNCTYPE(None, P, P, P)


class PriorCallbacks(ctypes.Structure):
    _fields_ = [("applyZ", VEC_FN), ("applyZt", VEC_FN), ("solveZ", VEC_FN),
                ("solveZt", VEC_FN), ("solveZ_blocked", MAT_FN),
                ("solveZt_blocked", MAT_FN), ("ctx", P)]


_L = None

# every function the header declares: name -> (restype, argtypes)
SIGNATURES = {
    "lgh_last_error": (ctypes.c_char_p, []),
    "lgh_mat_create_csr": (ctypes.c_int, [I64, P, P, P, ctypes.c_int,
                                          ctypes.POINTER(P)]),
    "lgh_mat_create_dense": (ctypes.c_int, [I64, P, I64, ctypes.c_int,
                                            ctypes.POINTER(P)]),
    "lgh_mat_get_info": (ctypes.c_int, [P, ctypes.POINTER(I64),
                                        ctypes.POINTER(I64)]),
    "lgh_mat_mult": (ctypes.c_int, [P, P, P]),
    "lgh_mat_dense_get_array": (ctypes.c_int, [P, ctypes.POINTER(P),
                                               ctypes.POINTER(I64),
                                               ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(I64)]),
    "lgh_mat_destroy": (ctypes.c_int, [ctypes.POINTER(P)]),
    "lgh_vec_create": (ctypes.c_int, [I64, ctypes.POINTER(P)]),
    "lgh_vec_create_with_array": (ctypes.c_int, [I64, P, ctypes.POINTER(P)]),
    "lgh_vec_get_array": (ctypes.c_int, [P, ctypes.POINTER(P),
                                         ctypes.POINTER(I64)]),
    "lgh_vec_set_host": (ctypes.c_int, [P, P]),
    "lgh_vec_get_host": (ctypes.c_int, [P, P]),
    "lgh_vec_destroy": (ctypes.c_int, [ctypes.POINTER(P)]),
    "lgh_prior_create_callbacks": (ctypes.c_int, [
        P, ctypes.POINTER(PriorCallbacks), ctypes.POINTER(P)]),
    "lgh_prior_mat_opts_default": (PriorMatOpts, []),
    "lgh_prior_create_mat": (ctypes.c_int, [P, P, ctypes.POINTER(PriorMatOpts),
                                            ctypes.POINTER(P)]),
    "lgh_prior_create_mat_pc": (ctypes.c_int, [P, P,
                                               ctypes.POINTER(PriorMatOpts),
                                               ctypes.c_int,
                                               ctypes.POINTER(P)]),
    "lgh_prior_create_ksp": (ctypes.c_int, [P, P,
                                            ctypes.POINTER(PriorMatOpts),
                                            ctypes.POINTER(P)]),
    "lgh_prior_destroy": (None, [P]),
    "lgh_prior_apply": (ctypes.c_int, [P, P, P]),
    "lgh_prior_solve": (ctypes.c_int, [P, P, P]),
    "lgh_prior_solve_block": (ctypes.c_int, [P, ctypes.c_int, P, I64, P,
                                             I64]),
    "lgh_prior_get_info": (ctypes.c_int, [P, c_dbl_p]),
    "lgh_glr_opts_default": (GlrOpts, []),
    "lgh_glr_compute": (ctypes.c_int, [P, P, ctypes.POINTER(GlrOpts),
                                       ctypes.POINTER(P),
                                       ctypes.POINTER(GlrReport)]),
    "lgh_glr_extend": (ctypes.c_int, [P, ctypes.c_int,
                                      ctypes.POINTER(GlrReport)]),
    "lgh_glr_destroy": (None, [P]),
    "lgh_glr_solve": (ctypes.c_int, [P, ctypes.c_double, P, P]),
    "lgh_glr_apply": (ctypes.c_int, [P, ctypes.c_double, P, P]),
    "lgh_glr_sample": (ctypes.c_int, [P, ctypes.c_double, P, P]),
    "lgh_glr_factor": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_int, P,
                                      P]),
    "lgh_glr_logdet": (ctypes.c_double, [P, ctypes.c_double]),
    "lgh_glr_pow": (ctypes.c_int, [P, ctypes.c_double, ctypes.c_double, P,
                                   P]),
    "lgh_glr_filter": (ctypes.c_int, [P, c_dbl_p, ctypes.c_double, P, P]),
    "lgh_glr_eigs": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(c_dbl_p)]),
    "lgh_exec_opts_default": (ExecOpts, []),
    "lgh_cols_range": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P]),
    "lgh_cols_exchange_bytes": (ctypes.c_size_t, [I64, ctypes.c_int,
                                                  ctypes.c_int]),
    "lgh_glr_compute_cols": (ctypes.c_int, [P, P, ctypes.POINTER(GlrOpts),
                                            ctypes.POINTER(ExecOpts),
                                            ctypes.POINTER(Comm),
                                            ctypes.POINTER(P),
                                            ctypes.POINTER(GlrReport)]),
    "lgh_comm_local_create": (ctypes.c_int, [ctypes.c_int, P]),
    "lgh_comm_local_destroy": (None, [P]),
    "lgh_glr_compute_ex": (ctypes.c_int, [P, P, ctypes.POINTER(GlrOpts),
                                          ctypes.POINTER(ExecOpts),
                                          ctypes.POINTER(P),
                                          ctypes.POINTER(GlrReport)]),
    "lgh_glr_get_stats": (ctypes.c_int, [P, ctypes.POINTER(GlrStats)]),
    "lgh_glr_get_U": (ctypes.c_int, [P, P, I64]),
    "lgh_glr_solve_batch": (ctypes.c_int, [P, ctypes.c_int, c_dbl_p,
                                           ctypes.c_int, P, I64, P, I64]),
    "lgh_glr_sample_batch": (ctypes.c_int, [P, ctypes.c_int, c_dbl_p,
                                            ctypes.c_int, P, I64, P, I64]),
    "lgh_glr_logdet_batch": (ctypes.c_int, [P, ctypes.c_int, c_dbl_p,
                                            c_dbl_p]),
    "lgh_server_opts_default": (ServerOpts, []),
    "lgh_server_create": (ctypes.c_int, [P, ctypes.POINTER(ServerOpts),
                                         ctypes.POINTER(P)]),
    "lgh_server_submit": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, P, I64, P, I64,
                                         ctypes.POINTER(I64)]),
    "lgh_server_wait": (ctypes.c_int, [P, I64, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_double)]),
    "lgh_server_get_stats": (ctypes.c_int, [P, ctypes.POINTER(ServerStats)]),
    "lgh_server_destroy": (None, [P]),
    "lgh_glr_correct_opts_default": (CorrectOpts, []),
    "lgh_glr_correct_probes": (ctypes.c_int, [P, ctypes.c_int, P, P, HESS_FN,
                                              P, ctypes.POINTER(CorrectOpts),
                                              ctypes.POINTER(CorrectReport)]),
    "lgh_glr_correct": (ctypes.c_int, [P, HESS_FN, P,
                                       ctypes.POINTER(CorrectOpts),
                                       ctypes.POINTER(CorrectReport)]),
    "lgh_glr_save": (ctypes.c_int, [P, ctypes.c_char_p, ctypes.c_int]),
    "lgh_glr_load": (ctypes.c_int, [P, P, ctypes.c_char_p, ctypes.POINTER(P)]),
    "lgh_shard_range": (None, [I64, ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "lgh_shard_create": (ctypes.c_int, [I64, ctypes.c_int, ctypes.c_int, P, P,
                                        ctypes.POINTER(P)]),
    "lgh_shard_info": (ctypes.c_int, [P, ctypes.POINTER(I64),
                                      ctypes.POINTER(I64),
                                      ctypes.POINTER(I64)]),
    "lgh_shard_ghosts": (ctypes.c_int, [P, ctypes.POINTER(ctypes.POINTER(I64)),
                                        ctypes.POINTER(ctypes.POINTER(I64))]),
    "lgh_shard_local_colidx": (ctypes.c_int, [
        P, ctypes.POINTER(ctypes.POINTER(ctypes.c_int32))]),
    "lgh_shard_set_sends": (ctypes.c_int, [P, ctypes.c_int, I64, P]),
    "lgh_shard_sends": (ctypes.c_int, [P, ctypes.c_int, ctypes.POINTER(I64),
                                       ctypes.POINTER(ctypes.POINTER(I64))]),
    "lgh_shard_pack": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, I64,
                                      P]),
    "lgh_shard_unpack": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_int, P, P,
                                        I64]),
    "lgh_shard_destroy": (None, [P]),
    "lgh_sketch_rows": (ctypes.c_int, [ctypes.c_uint64, I64, I64, I64,
                                       ctypes.c_int, P, I64]),
    "lgh_mat_create_rows": (ctypes.c_int, [I64, P, I64, I64, P, P, P,
                                           ctypes.POINTER(P)]),
    "lgh_mat_rows_info": (ctypes.c_int, [P, P, P, P]),
    "lgh_mat_rows_traffic": (ctypes.c_int, [P, P, P, P]),
    "lgh_rows_local_create": (ctypes.c_int, [ctypes.c_int, P]),
    "lgh_rows_local_destroy": (None, [P]),
    "lgh_launch_count": (ctypes.c_long, []),
    "lgh_runtime_counters": (ctypes.c_int, [c_dbl_p]),
    "lgh_kernel_timing": (ctypes.c_int, [ctypes.c_int]),
    "lgh_kernel_timing_get": (ctypes.c_char_p, [ctypes.c_int, c_dbl_p,
                                                ctypes.POINTER(ctypes.c_long),
                                                c_dbl_p]),
    "lgh_test_sketch": (ctypes.c_int, [ctypes.c_uint64, I64, I64,
                                       ctypes.c_int, P]),
    "lgh_test_rng_state": (ctypes.c_int, [ctypes.c_uint64, I64, I64,
                                          ctypes.c_int, P]),
    "lgh_glr_batch_info": (ctypes.c_int, [P, P, P, P, P]),
    "lgh_probe_peaks": (ctypes.c_int, [P]),
    "lgh_test_spmm": (ctypes.c_int, [P, ctypes.c_int, P, P, ctypes.c_int]),
    "lgh_test_spmm_strip": (ctypes.c_int, [P, ctypes.c_int, P, P, ctypes.c_int,
                                           ctypes.c_int, P]),
    "lgh_test_zsolve": (ctypes.c_int, [P, ctypes.c_int, P, P, ctypes.c_int]),
    "lgh_test_cheb_step": (ctypes.c_int, [P, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, P, P, P, P, P,
                                          ctypes.c_double]),
    "lgh_test_gram": (ctypes.c_int, [I64, ctypes.c_int, P, P]),
    "lgh_gram_noalloc": (ctypes.c_int, [I64, ctypes.c_int, P, I64, P, I64]),
    "lgh_test_gemm_nn": (ctypes.c_int, [I64, ctypes.c_int, ctypes.c_int, P,
                                        P, P]),
    "lgh_test_potrf": (ctypes.c_int, [ctypes.c_int, P, ctypes.c_int, P, P,
                                      P]),
    "lgh_test_syev": (ctypes.c_int, [ctypes.c_int, P, P, P, P]),
    "lgh_test_mg_galerkin": (ctypes.c_int, [I64, P, P, P, ctypes.c_int, P,
                                            P, P, P, I64, P, P, P, P, I64,
                                            P]),
}


def load(path=None):
    """Load the CUDA library (raises if it has not been built)."""
    global _L
    if _L is not None:
        return _L
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError("liblgh_b200.so not built (%s): run "
                           "__graft_entry__.build() or make -C "
                           "lgpsf-hessian_b200" % path)
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _L = L
    return L


def _chk(rc, where):
    if rc != 0:
        msg = load().lgh_last_error().decode(errors="replace")
        raise LghError(rc, where, msg)


def glr_opts(**kw):
    o = load().lgh_glr_opts_default()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def prior_opts(**kw):
    o = load().lgh_prior_mat_opts_default()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def exec_opts(**kw):
    o = load().lgh_exec_opts_default()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Vec:
    """Device vector handle (the reference's Vec)."""

    def __init__(self, n=None, data=None, handle=None):
        L = load()
        self.h = P()
        if handle is not None:
            self.h = handle
            self.owned = False
            nn = I64()
            _chk(L.lgh_vec_get_array(self.h, None, ctypes.byref(nn)),
                 "lgh_vec_get_array")
            self.n = nn.value
            return
        if data is not None:
            data = np.ascontiguousarray(data, dtype=np.float64)
            n = data.shape[0]
        _chk(L.lgh_vec_create(int(n), ctypes.byref(self.h)), "lgh_vec_create")
        self.n = int(n)
        self.owned = True
        if data is not None:
            self.set(data)

    def set(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape[0] == self.n
        _chk(load().lgh_vec_set_host(self.h, a.ctypes.data), "lgh_vec_set_host")

    def get(self):
        out = np.empty(self.n)
        _chk(load().lgh_vec_get_host(self.h, out.ctypes.data),
             "lgh_vec_get_host")
        return out

    def ptr(self):
        p = P()
        _chk(load().lgh_vec_get_array(self.h, ctypes.byref(p), None),
             "lgh_vec_get_array")
        return p.value

    def __del__(self):
        if getattr(self, "owned", False) and _L is not None and self.h:
            _L.lgh_vec_destroy(ctypes.byref(self.h))


class DeviceBlock:
    """A column-major n x m device block backed by one Vec of n*m."""

    def __init__(self, n, m, data=None):
        self.n, self.m = n, m
        self.v = Vec(n * m)
        if data is not None:
            self.set(data)

    def set(self, a):
        a = np.asarray(a, dtype=np.float64).reshape(self.n, self.m)
        self.v.set(np.asfortranarray(a).reshape(-1, order="F"))

    def get(self):
        return self.v.get().reshape(self.m, self.n).T.copy()

    def ptr(self):
        return self.v.ptr()


class Mat:
    """Device CSR operator (the reference's Mat for B and Z).  With rows =
    (N, comm) or (N, comm, row0): this rank's row slab of an N x N operator
    (csr holds the rank's rows, from global row row0, with global column
    indices; row0 defaults to lgh_shard_range's split), sharded over the
    row-slab communicator comm (a RowsComm)."""

    def __init__(self, csr=None, dense=None, rows=None):
        L = load()
        self.h = P()
        if rows is not None:
            N, comm = rows[0], rows[1]
            rp = np.ascontiguousarray(csr["rowptr"], dtype=np.int64)
            ci = np.ascontiguousarray(csr["colidx"], dtype=np.int32)
            va = np.ascontiguousarray(csr["vals"], dtype=np.float64)
            row0 = rows[2] if len(rows) > 2 else \
                shard_range(N, comm.size, comm.rank)[0]
            self._comm = comm
            _chk(L.lgh_mat_create_rows(int(N), ctypes.addressof(comm),
                                       int(row0), len(rp) - 1,
                                       rp.ctypes.data, ci.ctypes.data,
                                       va.ctypes.data, ctypes.byref(self.h)),
                 "lgh_mat_create_rows")
            self.n = len(rp) - 1
            return
        if dense is not None:
            D = np.asfortranarray(dense, dtype=np.float64)
            _chk(L.lgh_mat_create_dense(D.shape[0], D.ctypes.data, D.shape[0],
                                        LGH_MEM_HOST, ctypes.byref(self.h)),
                 "lgh_mat_create_dense")
            self.n = D.shape[0]
        else:
            rp = np.ascontiguousarray(csr["rowptr"], dtype=np.int64)
            ci = np.ascontiguousarray(csr["colidx"], dtype=np.int32)
            va = np.ascontiguousarray(csr["vals"], dtype=np.float64)
            _chk(L.lgh_mat_create_csr(len(rp) - 1, rp.ctypes.data,
                                      ci.ctypes.data, va.ctypes.data,
                                      LGH_MEM_HOST, ctypes.byref(self.h)),
                 "lgh_mat_create_csr")
            self.n = len(rp) - 1

    def info(self):
        n, nnz = I64(), I64()
        _chk(load().lgh_mat_get_info(self.h, ctypes.byref(n),
                                     ctypes.byref(nnz)), "lgh_mat_get_info")
        return n.value, nnz.value

    def rows_info(self):
        """(row0, row1, nghost) of a row-sharded Mat."""
        a, b, g = I64(), I64(), I64()
        _chk(load().lgh_mat_rows_info(self.h, ctypes.addressof(a),
                                      ctypes.addressof(b),
                                      ctypes.addressof(g)),
             "lgh_mat_rows_info")
        return a.value, b.value, g.value

    def rows_traffic(self):
        """(exchanges, bytes sent, seconds) of a row-sharded Mat's halo."""
        e, b, t = ctypes.c_long(), I64(), ctypes.c_double()
        _chk(load().lgh_mat_rows_traffic(self.h, ctypes.addressof(e),
                                         ctypes.addressof(b),
                                         ctypes.addressof(t)),
             "lgh_mat_rows_traffic")
        return e.value, b.value, t.value

    def mult(self, x):
        vx, vy = Vec(data=x), Vec(len(x))
        _chk(load().lgh_mat_mult(self.h, vx.h, vy.h), "lgh_mat_mult")
        return vy.get()

    def __del__(self):
        if _L is not None and getattr(self, "h", None):
            _L.lgh_mat_destroy(ctypes.byref(self.h))


class Prior:
    """lgh_prior_t: Mat path (Z + mass) or callbacks path."""

    def __init__(self, Z=None, mass=None, opts=None, callbacks=None,
                 pc=None):
        L = load()
        self.h = P()
        self.mass = Vec(data=mass)
        self.n = self.mass.n
        self._keep = []
        if callbacks is not None:
            cb = PriorCallbacks()
            for k in ("applyZ", "applyZt", "solveZ", "solveZt"):
                fn = callbacks.get(k)
                setattr(cb, k, VEC_FN(fn) if fn else VEC_FN())
            for k in ("solveZ_blocked", "solveZt_blocked"):
                fn = callbacks.get(k)
                setattr(cb, k, MAT_FN(fn) if fn else MAT_FN())
            cb.ctx = None
            self._keep.append(cb)
            _chk(L.lgh_prior_create_callbacks(self.mass.h, ctypes.byref(cb),
                                              ctypes.byref(self.h)),
                 "lgh_prior_create_callbacks")
        else:
            o = opts if opts is not None else prior_opts()
            self.Z = Z
            if pc is None:
                _chk(L.lgh_prior_create_mat(Z.h, self.mass.h, ctypes.byref(o),
                                            ctypes.byref(self.h)),
                     "lgh_prior_create_mat")
            else:
                code = {"amg": PC_AMG, "jacobi": PC_JACOBI}[pc]
                _chk(L.lgh_prior_create_mat_pc(Z.h, self.mass.h,
                                               ctypes.byref(o), code,
                                               ctypes.byref(self.h)),
                     "lgh_prior_create_mat_pc")

    def info(self):
        out = np.zeros(14)
        _chk(load().lgh_prior_get_info(self.h, out.ctypes.data_as(c_dbl_p)),
             "lgh_prior_get_info")
        return dict(emin=out[0], emax=out[1], lmin=out[2], lmax=out[3],
                    nit=int(out[4]), bound_its=int(out[5]),
                    mean_col_iters=out[6], calls=int(out[7]),
                    mg_levels=int(out[8]), mg_coarse=int(out[9]),
                    mg_setup_s=out[10], pc=int(out[11]),
                    pc32_calls=int(out[12]))

    def apply(self, x):
        vx, vy = Vec(data=x), Vec(self.n)
        _chk(load().lgh_prior_apply(self.h, vx.h, vy.h), "lgh_prior_apply")
        return vy.get()

    def solve(self, x):
        vx, vy = Vec(data=x), Vec(self.n)
        _chk(load().lgh_prior_solve(self.h, vx.h, vy.h), "lgh_prior_solve")
        return vy.get()

    def solve_block(self, X):
        X = np.asarray(X, dtype=np.float64)
        m = X.shape[1]
        bx, by = DeviceBlock(self.n, m, X), DeviceBlock(self.n, m)
        _chk(load().lgh_prior_solve_block(self.h, m, bx.ptr(), self.n,
                                          by.ptr(), self.n),
             "lgh_prior_solve_block")
        return by.get()

    def __del__(self):
        if _L is not None and getattr(self, "h", None):
            _L.lgh_prior_destroy(self.h)
            self.h = P()


class Glr:
    """lgh_glr_t: build, extend and the downstream operations."""

    def __init__(self, B, prior, opts=None, exec=None, comm=None):
        L = load()
        self.h = P()
        self.B, self.prior = B, prior
        o = opts if opts is not None else glr_opts()
        rep = GlrReport()
        if comm is not None:
            e = exec if exec is not None else L.lgh_exec_opts_default()
            self._comm = comm
            _chk(L.lgh_glr_compute_cols(B.h, prior.h, ctypes.byref(o),
                                        ctypes.byref(e), ctypes.byref(comm),
                                        ctypes.byref(self.h),
                                        ctypes.byref(rep)),
                 "lgh_glr_compute_cols")
        elif exec is None:
            _chk(L.lgh_glr_compute(B.h, prior.h, ctypes.byref(o),
                                   ctypes.byref(self.h), ctypes.byref(rep)),
                 "lgh_glr_compute")
        else:
            _chk(L.lgh_glr_compute_ex(B.h, prior.h, ctypes.byref(o),
                                      ctypes.byref(exec), ctypes.byref(self.h),
                                      ctypes.byref(rep)), "lgh_glr_compute_ex")
        self.report = rep.as_dict()
        self.n = prior.n

    @staticmethod
    def _hess(fn, n):
        def cb(xin, xout, ctx):
            x = np.ctypeslib.as_array(xin, shape=(n,))
            y = np.ctypeslib.as_array(xout, shape=(n,))
            y[:] = fn(x.copy())
        return HESS_FN(cb)

    def correct_probes(self, V, HV, hessian, opts=None):
        """Value-pass deflation correction from probe pairs (N x k host
        arrays) and a true-Hessian callable x -> H_d x (host arrays)."""
        L = load()
        o = opts if opts is not None else L.lgh_glr_correct_opts_default()
        Vf = np.asfortranarray(V, dtype=np.float64)
        HVf = np.asfortranarray(HV, dtype=np.float64)
        cb = self._hess(hessian, self.n)
        rep = CorrectReport()
        _chk(L.lgh_glr_correct_probes(self.h, Vf.shape[1], Vf.ctypes.data,
                                      HVf.ctypes.data, cb, None,
                                      ctypes.byref(o), ctypes.byref(rep)),
             "lgh_glr_correct_probes")
        return rep.as_dict()

    def correct(self, hessian, opts=None):
        """Fresh randomized deflation correction."""
        L = load()
        o = opts if opts is not None else L.lgh_glr_correct_opts_default()
        cb = self._hess(hessian, self.n)
        rep = CorrectReport()
        _chk(L.lgh_glr_correct(self.h, cb, None, ctypes.byref(o),
                               ctypes.byref(rep)), "lgh_glr_correct")
        return rep.as_dict()

    def save(self, path, with_extension=False):
        _chk(load().lgh_glr_save(self.h, str(path).encode(),
                                 1 if with_extension else 0), "lgh_glr_save")

    @classmethod
    def load(cls, B, prior, path):
        """Restore a saved object against the same B and prior."""
        g = cls.__new__(cls)
        g.h = P()
        g.B, g.prior = B, prior
        _chk(load().lgh_glr_load(B.h, prior.h, str(path).encode(),
                                 ctypes.byref(g.h)), "lgh_glr_load")
        g.report = {}
        g.n = prior.n
        return g

    def extend(self, k):
        rep = GlrReport()
        _chk(load().lgh_glr_extend(self.h, int(k), ctypes.byref(rep)),
             "lgh_glr_extend")
        self.report = rep.as_dict()
        return self.report

    def eigs(self):
        nk = ctypes.c_int()
        p = c_dbl_p()
        _chk(load().lgh_glr_eigs(self.h, ctypes.byref(nk), ctypes.byref(p)),
             "lgh_glr_eigs")
        if nk.value == 0:
            return np.zeros(0)
        return np.ctypeslib.as_array(p, shape=(nk.value,)).copy()

    def stats(self):
        st = GlrStats()
        _chk(load().lgh_glr_get_stats(self.h, ctypes.byref(st)),
             "lgh_glr_get_stats")
        return st.as_dict()

    def U(self):
        k = len(self.eigs())
        b = DeviceBlock(self.n, max(k, 1))
        _chk(load().lgh_glr_get_U(self.h, b.ptr(), self.n), "lgh_glr_get_U")
        return b.get()[:, :k]

    def _vv(self, fname, c, v, *extra):
        vx, vy = Vec(data=v), Vec(self.n)
        f = getattr(load(), fname)
        _chk(f(self.h, c, *extra, vx.h, vy.h), fname)
        return vy.get()

    def solve(self, c, rhs):
        return self._vv("lgh_glr_solve", c, rhs)

    def sample(self, c, xi):
        return self._vv("lgh_glr_sample", c, xi)

    def apply(self, c, v):
        return self._vv("lgh_glr_apply", c, v)

    def factor(self, c, which, v):
        return self._vv("lgh_glr_factor", c, v, int(which))

    def pow(self, c, p, v):
        return self._vv("lgh_glr_pow", c, v, float(p))

    def filter(self, f_lam, f_c, v):
        f = np.ascontiguousarray(f_lam, dtype=np.float64)
        vx, vy = Vec(data=v), Vec(self.n)
        _chk(load().lgh_glr_filter(self.h, f.ctypes.data_as(c_dbl_p), f_c,
                                   vx.h, vy.h), "lgh_glr_filter")
        return vy.get()

    def logdet(self, c):
        return load().lgh_glr_logdet(self.h, c)

    def logdet_batch(self, cs):
        cs = np.ascontiguousarray(cs, dtype=np.float64)
        out = np.empty_like(cs)
        _chk(load().lgh_glr_logdet_batch(self.h, len(cs),
                                         cs.ctypes.data_as(c_dbl_p),
                                         out.ctypes.data_as(c_dbl_p)),
             "lgh_glr_logdet_batch")
        return out

    def batch_info(self):
        """Graph captures / replays of the batched operations, the tile
        variant of the last combination and the autotuner's table size."""
        c, r = ctypes.c_long(), ctypes.c_long()
        v, t = ctypes.c_int(), ctypes.c_int()
        _chk(load().lgh_glr_batch_info(self.h, ctypes.addressof(c),
                                       ctypes.addressof(r),
                                       ctypes.addressof(v),
                                       ctypes.addressof(t)),
             "lgh_glr_batch_info")
        return dict(captures=c.value, replays=r.value, variant=v.value,
                    tuned_shapes=t.value)

    def _batch(self, fname, cs, R):
        cs = np.ascontiguousarray(cs, dtype=np.float64)
        R = np.asarray(R, dtype=np.float64)
        m = R.shape[1]
        bi = DeviceBlock(self.n, m, R)
        bo = DeviceBlock(self.n, m * len(cs))
        _chk(getattr(load(), fname)(self.h, len(cs),
                                    cs.ctypes.data_as(c_dbl_p), m, bi.ptr(),
                                    self.n, bo.ptr(), self.n), fname)
        out = bo.get()
        return [out[:, s * m:(s + 1) * m] for s in range(len(cs))]

    def solve_batch(self, cs, R):
        return self._batch("lgh_glr_solve_batch", cs, R)

    def sample_batch(self, cs, R):
        return self._batch("lgh_glr_sample_batch", cs, R)

    def __del__(self):
        if _L is not None and getattr(self, "h", None):
            _L.lgh_glr_destroy(self.h)
            self.h = P()


def kernel_timing(on):
    """Switch the library's per-kernel CUDA-event timing on or off."""
    _chk(load().lgh_kernel_timing(1 if on else 0), "lgh_kernel_timing")


def kernel_timing_get():
    """{name: (device ms, launches, algorithmic bytes)} since switched on."""
    out = {}
    i = 0
    while True:
        ms, n, by = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
        name = load().lgh_kernel_timing_get(i, ctypes.byref(ms),
                                            ctypes.byref(n), ctypes.byref(by))
        if name is None:
            return out
        out[name.decode()] = (ms.value, n.value, by.value)
        i += 1


def runtime_counters():
    """Host-side runtime counters (lgh_runtime_counters)."""
    out = np.zeros(5)
    _chk(load().lgh_runtime_counters(out.ctypes.data_as(c_dbl_p)),
         "lgh_runtime_counters")
    return dict(allocs=int(out[0]), alloc_s=out[1], frees=int(out[2]),
                free_s=out[3], launches=int(out[4]))


def correct_opts(**kw):
    o = load().lgh_glr_correct_opts_default()
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def shard_range(N, nranks, rank):
    a, b = I64(), I64()
    load().lgh_shard_range(N, nranks, rank, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


class Shard:
    """One rank's row slab of a symmetric CSR operator (lgh_shard_*): the
    host-side partition and halo plan.  csr: the global CSR dict
    (rowptr, colidx[, vals]); only this rank's rows are handed over."""

    def __init__(self, csr, nranks, rank):
        L = load()
        N = len(csr["rowptr"]) - 1
        self.N, self.nranks, self.rank = N, nranks, rank
        self.row0, self.row1 = shard_range(N, nranks, rank)
        rp = np.ascontiguousarray(csr["rowptr"][self.row0:self.row1 + 1],
                                  dtype=np.int64)
        k0, k1 = int(rp[0]), int(rp[-1])
        self.rowptr = rp - k0
        self.colidx = np.ascontiguousarray(csr["colidx"][k0:k1],
                                           dtype=np.int32)
        self.vals = (np.ascontiguousarray(csr["vals"][k0:k1])
                     if "vals" in csr else None)
        self.h = P()
        _chk(L.lgh_shard_create(N, nranks, rank, self.rowptr.ctypes.data,
                                self.colidx.ctypes.data, ctypes.byref(self.h)),
             "lgh_shard_create")

    @property
    def nloc(self):
        return self.row1 - self.row0

    def ghosts(self):
        """(ghost rows ascending, counts per owner rank)"""
        rows, counts = ctypes.POINTER(I64)(), ctypes.POINTER(I64)()
        nl = I64()
        _chk(load().lgh_shard_info(self.h, None, None, ctypes.byref(nl)),
             "lgh_shard_info")
        _chk(load().lgh_shard_ghosts(self.h, ctypes.byref(rows),
                                     ctypes.byref(counts)), "lgh_shard_ghosts")
        g = (np.ctypeslib.as_array(rows, shape=(nl.value,)).copy()
             if nl.value else np.zeros(0, np.int64))
        c = np.ctypeslib.as_array(counts, shape=(self.nranks,)).copy()
        return g, c

    def local_colidx(self):
        p = ctypes.POINTER(ctypes.c_int32)()
        _chk(load().lgh_shard_local_colidx(self.h, ctypes.byref(p)),
             "lgh_shard_local_colidx")
        n = len(self.colidx)
        return (np.ctypeslib.as_array(p, shape=(n,)).copy() if n
                else np.zeros(0, np.int32))

    def set_sends(self, peer, rows):
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        _chk(load().lgh_shard_set_sends(self.h, peer, len(rows),
                                        rows.ctypes.data if len(rows) else None),
             "lgh_shard_set_sends")

    def sends(self, peer):
        cnt = I64()
        p = ctypes.POINTER(I64)()
        _chk(load().lgh_shard_sends(self.h, peer, ctypes.byref(cnt),
                                    ctypes.byref(p)), "lgh_shard_sends")
        return (np.ctypeslib.as_array(p, shape=(cnt.value,)).copy()
                if cnt.value else np.zeros(0, np.int64))

    def close(self):
        if _L is not None and getattr(self, "h", None):
            _L.lgh_shard_destroy(self.h)
            self.h = P()

    def __del__(self):
        self.close()


class Server:
    """The request loop (lgh_server_*) over a resident Glr object."""

    SOLVE, SAMPLE, LOGDET = 0, 1, 2

    def __init__(self, glr, slots=64, hbm_reserve=0.05):
        L = load()
        o = L.lgh_server_opts_default()
        o.slots = slots
        o.hbm_reserve = hbm_reserve
        self.h = P()
        self.glr = glr
        self.n = glr.n
        self._bufs = {}
        _chk(L.lgh_server_create(glr.h, ctypes.byref(o), ctypes.byref(self.h)),
             "lgh_server_create")

    def submit(self, kind, c, X=None):
        """Queue a request; returns its id.  X: (n, m) host block."""
        L = load()
        rid = I64()
        if kind == self.LOGDET:
            out = np.zeros(1)
            _chk(L.lgh_server_submit(self.h, kind, c, 0, None, 0,
                                     out.ctypes.data, 1, ctypes.byref(rid)),
                 "lgh_server_submit")
            self._bufs[rid.value] = (None, out)
            return rid.value
        Xin = np.asfortranarray(X, dtype=np.float64)
        out = np.empty_like(Xin, order="F")   # every entry is written
        _chk(L.lgh_server_submit(self.h, kind, c, Xin.shape[1],
                                 Xin.ctypes.data, self.n, out.ctypes.data,
                                 self.n, ctypes.byref(rid)),
             "lgh_server_submit")
        self._bufs[rid.value] = (Xin, out)
        return rid.value

    def wait(self, rid, timeout=600.0):
        """(result, latency seconds): the (n, m) column-major block the
        library wrote (no reordering copy), or the logdet value."""
        lat = ctypes.c_double()
        _chk(load().lgh_server_wait(self.h, rid, timeout, ctypes.byref(lat)),
             "lgh_server_wait")
        _, out = self._bufs.pop(rid)
        return (out[0] if out.ndim == 1 else out), lat.value

    def stats(self):
        st = ServerStats()
        _chk(load().lgh_server_get_stats(self.h, ctypes.byref(st)),
             "lgh_server_get_stats")
        return st.as_dict()

    def close(self):
        if _L is not None and getattr(self, "h", None):
            _L.lgh_server_destroy(self.h)
            self.h = P()

    def __del__(self):
        self.close()


# ---- kernel-level test hooks --------------------------------------------


def test_sketch(seed, n, j0, k):
    out = np.empty((n, k))
    _chk(load().lgh_test_sketch(seed, n, j0, k, out.ctypes.data),
         "lgh_test_sketch")
    return out


def test_rng_state(seed, n, j0, k):
    out = np.empty((n, k), dtype=np.uint64)
    _chk(load().lgh_test_rng_state(seed, n, j0, k, out.ctypes.data),
         "lgh_test_rng_state")
    return out


def test_spmm(A, X, fp32=False):
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.empty_like(X)
    _chk(load().lgh_test_spmm(A.h, X.shape[1], X.ctypes.data, Y.ctypes.data,
                              1 if fp32 else 0), "lgh_test_spmm")
    return Y


def probe_peaks():
    """FP64 / FP32 FMA, FP64 mma.sync TFLOP/s and L2 read GB/s."""
    out = np.zeros(4)
    _chk(load().lgh_probe_peaks(out.ctypes.data), "lgh_probe_peaks")
    return dict(fp64_fma_tflops=out[0], fp32_fma_tflops=out[1],
                fp64_mma_tflops=out[2], l2_read_gbs=out[3])


def cols_range(w, rank, size):
    """Columns [c0, c1) of a width-w block owned by rank of size."""
    c0, c1 = ctypes.c_int(), ctypes.c_int()
    load().lgh_cols_range(w, rank, size, ctypes.addressof(c0),
                          ctypes.addressof(c1))
    return c0.value, c1.value


def local_comms(size):
    """size in-process communicators (ranks as threads on one device)."""
    arr = (Comm * size)()
    _chk(load().lgh_comm_local_create(size, ctypes.addressof(arr)),
         "lgh_comm_local_create")
    return arr


def free_local_comms(arr):
    load().lgh_comm_local_destroy(ctypes.addressof(arr))


def local_rows_comms(size):
    """size in-process row-slab communicators (ranks as threads on one
    device)."""
    arr = (RowsComm * size)()
    _chk(load().lgh_rows_local_create(size, ctypes.addressof(arr)),
         "lgh_rows_local_create")
    return arr


def free_local_rows_comms(arr):
    load().lgh_rows_local_destroy(ctypes.addressof(arr))


def rows_slab(csr, row0, row1):
    """Rows [row0, row1) of a host CSR dict (global column indices)."""
    rp = np.asarray(csr["rowptr"], dtype=np.int64)
    a, b = int(rp[row0]), int(rp[row1])
    return dict(n=row1 - row0, rowptr=rp[row0:row1 + 1] - a,
                colidx=np.asarray(csr["colidx"])[a:b],
                vals=np.asarray(csr["vals"])[a:b])


def test_spmm_strip(A, X, fp32=False, R=0):
    """B X through the strip form at height R (0: the cost model's choice);
    returns (Y, R used)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.empty_like(X)
    ru = ctypes.c_int(0)
    _chk(load().lgh_test_spmm_strip(A.h, X.shape[1], X.ctypes.data,
                                    Y.ctypes.data, 1 if fp32 else 0, int(R),
                                    ctypes.addressof(ru)),
         "lgh_test_spmm_strip")
    return Y, ru.value


def test_zsolve(prior, X, fp32=False):
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.empty_like(X)
    _chk(load().lgh_test_zsolve(prior.h, X.shape[1], X.ctypes.data,
                                Y.ctypes.data, 1 if fp32 else 0),
         "lgh_test_zsolve")
    return Y


CHEB_FIRST, CHEB_ZERO_X, CHEB_STORE_D = 1, 2, 4
CHEB_R_ONLY, CHEB_PREV_R = 8, 16


def test_cheb_step(A, X, R, D, a, b, flags, fp32=False, bp=0.0):
    """One Chebyshev-Jacobi smoothing step (lgh_test_cheb_step); returns
    the new (X, R, D)."""
    X = np.array(X, dtype=np.float64, order="C")
    R = np.ascontiguousarray(R, dtype=np.float64)
    D = np.ascontiguousarray(D, dtype=np.float64)
    Rn = np.zeros_like(R)
    Dn = np.zeros_like(R)
    _chk(load().lgh_test_cheb_step(A.h, X.shape[1], a, b, flags,
                                   1 if fp32 else 0, X.ctypes.data,
                                   R.ctypes.data, D.ctypes.data,
                                   Rn.ctypes.data, Dn.ctypes.data, bp),
         "lgh_test_cheb_step")
    return X, Rn, Dn


def test_gram(X):
    X = np.ascontiguousarray(X, dtype=np.float64)
    w = X.shape[1]
    G = np.empty((w, w), order="F")
    _chk(load().lgh_test_gram(X.shape[0], w, X.ctypes.data, G.ctypes.data),
         "lgh_test_gram")
    return G


def test_gemm_nn(X, M):
    X = np.ascontiguousarray(X, dtype=np.float64)
    Mf = np.asfortranarray(M, dtype=np.float64)
    Y = np.empty((X.shape[0], Mf.shape[1]))
    _chk(load().lgh_test_gemm_nn(X.shape[0], X.shape[1], Mf.shape[1],
                                 X.ctypes.data, Mf.ctypes.data, Y.ctypes.data),
         "lgh_test_gemm_nn")
    return Y


def test_potrf(G, jitter_mode=0):
    Gf = np.asfortranarray(G, dtype=np.float64)
    n = Gf.shape[0]
    L = np.empty((n, n), order="F")
    Li = np.empty((n, n), order="F")
    info = np.zeros(2, dtype=np.int32)
    _chk(load().lgh_test_potrf(n, Gf.ctypes.data, jitter_mode, L.ctypes.data,
                               Li.ctypes.data, info.ctypes.data),
         "lgh_test_potrf")
    return L, (Li if info[0] == 0 else None), info


def test_mg_galerkin(csr, threads=0):
    """The multigrid set-up's first coarsening of a square CSR dict (n,
    rowptr, colidx, vals), run on the host alone (lgh_test_mg_galerkin):
    returns (P, Ac) as CSR dicts, P n x nc, Ac = P^T A P (nc x nc)."""
    n = int(csr["n"]) if "n" in csr else len(csr["rowptr"]) - 1
    rp = np.ascontiguousarray(csr["rowptr"], dtype=np.int64)
    ci = np.ascontiguousarray(csr["colidx"], dtype=np.int32)
    v = np.ascontiguousarray(csr["vals"], dtype=np.float64)
    nc, pn, cn = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
    L = load()
    args = (n, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, threads,
            ctypes.byref(nc))
    _chk(L.lgh_test_mg_galerkin(*args, None, None, None, 0, ctypes.byref(pn),
                                None, None, None, 0, ctypes.byref(cn)),
         "lgh_test_mg_galerkin")
    Prp = np.empty(n + 1, dtype=np.int64)
    Pci = np.empty(pn.value, dtype=np.int32)
    Pv = np.empty(pn.value)
    Crp = np.empty(nc.value + 1, dtype=np.int64)
    Cci = np.empty(cn.value, dtype=np.int32)
    Cv = np.empty(cn.value)
    _chk(L.lgh_test_mg_galerkin(*args, Prp.ctypes.data, Pci.ctypes.data,
                                Pv.ctypes.data, pn.value, ctypes.byref(pn),
                                Crp.ctypes.data, Cci.ctypes.data,
                                Cv.ctypes.data, cn.value, ctypes.byref(cn)),
         "lgh_test_mg_galerkin")
    return (dict(n=n, m=nc.value, rowptr=Prp, colidx=Pci, vals=Pv),
            dict(n=nc.value, m=nc.value, rowptr=Crp, colidx=Cci, vals=Cv))


def test_syev(A):
    Af = np.asfortranarray(A, dtype=np.float64)
    n = Af.shape[0]
    w = np.empty(n)
    V = np.empty((n, n), order="F")
    sw = ctypes.c_int(0)
    _chk(load().lgh_test_syev(n, Af.ctypes.data, w.ctypes.data, V.ctypes.data,
                              ctypes.byref(sw)), "lgh_test_syev")
    return w, V, sw.value
