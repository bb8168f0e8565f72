"""ctypes binding of the C ABI in ``include/rcwa_b200.h``.

The library is loaded from ``openrcwa_b200/lib/librcwa_b200.so`` (built by
``openrcwa_b200.build``); a missing library raises immediately: there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librcwa_b200.so")

RCWA_OK = 0
RCWA_ERR_INVALID = 1
RCWA_ERR_CUDA = 2
RCWA_ERR_NOCONV = 3
RCWA_ERR_SINGULAR = 4
RCWA_ERR_NONFINITE = 5
RCWA_ERR_GRAZING = 6
RCWA_ERR_NOMEM = 7
RCWA_ERR_NODEVICE = 8
RCWA_ERR_UNSUPPORTED = 9
RCWA_CONTINUOUS_XY, RCWA_DISCONTINUOUS_X, RCWA_DISCONTINUOUS_Y = 0, 1, 2
RCWA_PREC_FP64 = 0
RCWA_PREC_MIXED = 1
RCWA_TUNE_LU, RCWA_TUNE_SCHUR, RCWA_TUNE_PRODUCT = 0, 1, 2
RCWA_TUNING_OFF, RCWA_TUNING_TABLE, RCWA_TUNING_AUTO = 0, 1, 2
TUNE_OPS = {"lu": RCWA_TUNE_LU, "schur": RCWA_TUNE_SCHUR, "product": RCWA_TUNE_PRODUCT}

# every symbol declared in include/rcwa_b200.h
EXPORTS = [
    "rcwa_status_string", "rcwa_engine_create", "rcwa_engine_destroy", "rcwa_engine_last_error",
    "rcwa_engine_solve_batch", "rcwa_plan_create", "rcwa_plan_execute", "rcwa_plan_results",
    "rcwa_plan_launch_count", "rcwa_plan_rescatter", "rcwa_plan_set_profiling", "rcwa_plan_stage_times", "rcwa_stage_name",
    "rcwa_plan_destroy", "rcwa_fourier1d", "rcwa_fourier2d",
    "rcwa_layer_solve", "rcwa_zgeev_batched", "rcwa_zgeev_batched_noalloc", "rcwa_ofd_solve",
    "rcwa_slab_smatrix_batched", "rcwa_star_product_batched", "rcwa_rcwa_integrate", "rcwa_differential_integrate",
    "rcwa_redheffer_integrate", "rcwa_zgemm_batched",
    "rcwa_mlp_create", "rcwa_mlp_destroy", "rcwa_mlp_param_count", "rcwa_mlp_get_params", "rcwa_mlp_set_params",
    "rcwa_mlp_set_data", "rcwa_mlp_train", "rcwa_mlp_loss_grad", "rcwa_mlp_predict_fp32", "rcwa_mlp_predict",
    "rcwa_plan_schedule", "rcwa_tuner_create", "rcwa_tuner_destroy", "rcwa_tuner_set_sms", "rcwa_tuner_candidates",
    "rcwa_tuner_default", "rcwa_tuner_set", "rcwa_tuner_get", "rcwa_tuner_count", "rcwa_tuner_entry",
    "rcwa_tuner_save", "rcwa_tuner_load", "rcwa_engine_set_tuner", "rcwa_tuner_measure",
    "rcwa_set_qr_sweep_limit", "rcwa_plan_smatrix", "rcwa_mlp_nn_distance", "rcwa_engine_solve_tables",
    "rcwa_plan_create_tables", "rcwa_set_eig_cluster", "rcwa_eig_cluster_size",
    "rcwa_set_lu_cluster", "rcwa_lu_cluster_size", "rcwa_plan_field_rows", "rcwa_plan_field",
]

_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
# rcwa_sampler: int (*)(void* user, double z, rcwa_cplx* P, rcwa_cplx* Q)
RCWA_SAMPLER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p)


class rcwa_cplx(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class rcwa_stack(C.Structure):
    _fields_ = [("nHx", C.c_int), ("nHy", C.c_int), ("ncx", C.c_int), ("ncy", C.c_int),
                ("cx", C.c_void_p), ("cy", C.c_void_p), ("n_layers", C.c_int),
                ("eps", C.c_void_p), ("thickness", C.c_void_p), ("mu", C.c_void_p)]


class rcwa_table_stack(C.Structure):
    _fields_ = [("nHx", C.c_int), ("nHy", C.c_int), ("Lx", C.c_double), ("Ly", C.c_double),
                ("n_layers", C.c_int), ("eps_half", C.c_void_p), ("f2d", C.c_void_p), ("thickness", C.c_void_p)]


class rcwa_point(C.Structure):
    _fields_ = [("stack", C.c_int), ("lambda_", C.c_double), ("kx0", C.c_double), ("ky0", C.c_double)]


class rcwa_layer_spec(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("eps1", "eps2", "eps1i", "eps2i", "fill", "fill_y", "thickness")]


class rcwa_pole_spec(C.Structure):
    _fields_ = [("layer", C.c_int), ("side", C.c_int)] + [(k, C.c_double) for k in ("einf", "ae", "be", "ce")]


class rcwa_ofd_setup(C.Structure):
    _fields_ = [("nHx", C.c_int), ("period_x", C.c_double), ("nHy", C.c_int), ("period_y", C.c_double),
                ("n_layers", C.c_int), ("layers", C.POINTER(rcwa_layer_spec)),
                ("n_poles", C.c_int), ("poles", C.POINTER(rcwa_pole_spec)),
                ("theta_deg", C.c_double), ("phi_deg", C.c_double),
                ("n_freq", C.c_int), ("freq", _DP)]


_lib = None


def load() -> C.CDLL:
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"RCWA engine library missing: {LIB_PATH} (run python -m openrcwa_b200.build)")
    lib = C.CDLL(LIB_PATH)
    lib.rcwa_status_string.restype = C.c_char_p
    lib.rcwa_status_string.argtypes = [C.c_int]
    lib.rcwa_engine_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    lib.rcwa_engine_destroy.argtypes = [C.c_void_p]
    lib.rcwa_engine_destroy.restype = None
    lib.rcwa_engine_last_error.argtypes = [C.c_void_p]
    lib.rcwa_engine_last_error.restype = C.c_char_p
    lib.rcwa_engine_solve_batch.argtypes = [C.c_void_p, C.POINTER(rcwa_stack), C.c_int, C.POINTER(rcwa_point),
                                            C.c_int, C.c_int, C.c_void_p, C.c_int, _DP, _DP, _DP, _DP, _IP]
    lib.rcwa_plan_create.argtypes = [C.c_void_p, C.POINTER(rcwa_stack), C.c_int, C.POINTER(rcwa_point), C.c_int,
                                     C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
    lib.rcwa_engine_solve_tables.argtypes = [C.c_void_p, C.POINTER(rcwa_table_stack), C.c_int,
                                             C.POINTER(rcwa_point), C.c_int, C.c_int, C.c_void_p, C.c_int, _DP, _DP,
                                             _DP, _DP, _IP]
    lib.rcwa_plan_create_tables.argtypes = [C.c_void_p, C.POINTER(rcwa_table_stack), C.c_int,
                                            C.POINTER(rcwa_point), C.c_int, C.c_int, C.c_void_p, C.c_int,
                                            C.POINTER(C.c_void_p)]
    lib.rcwa_plan_execute.argtypes = [C.c_void_p, C.c_void_p]
    lib.rcwa_plan_results.argtypes = [C.c_void_p, _DP, _DP, _DP, _DP, _IP]
    lib.rcwa_plan_launch_count.argtypes = [C.c_void_p]
    lib.rcwa_plan_launch_count.restype = C.c_longlong
    lib.rcwa_plan_rescatter.argtypes = [C.c_void_p, C.c_void_p]
    lib.rcwa_plan_set_profiling.argtypes = [C.c_void_p, C.c_int]
    lib.rcwa_plan_stage_times.argtypes = [C.c_void_p, _DP, C.c_int]
    lib.rcwa_stage_name.argtypes = [C.c_int]
    lib.rcwa_stage_name.restype = C.c_char_p
    lib.rcwa_plan_destroy.argtypes = [C.c_void_p]
    lib.rcwa_plan_destroy.restype = None
    lib.rcwa_fourier1d.argtypes = [C.c_void_p, _DP, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    lib.rcwa_fourier2d.argtypes = [C.c_void_p, _DP, C.c_int, _DP, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                   C.c_void_p]
    lib.rcwa_layer_solve.argtypes = [C.c_void_p, _DP, C.c_int, _DP, C.c_int, C.c_void_p, C.c_int, C.c_int, _DP, _DP,
                                     C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rcwa_zgeev_batched.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, _IP]
    lib.rcwa_zgeev_batched_noalloc.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p]
    lib.rcwa_ofd_solve.argtypes = [C.c_void_p, C.POINTER(rcwa_ofd_setup), _DP, _DP, _DP, _DP, _IP]
    lib.rcwa_slab_smatrix_batched.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 5 + [_DP, _DP] + \
        [C.c_void_p, C.c_void_p, _IP]
    lib.rcwa_star_product_batched.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 8 + [_IP]
    lib.rcwa_rcwa_integrate.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double] + \
        [C.c_void_p] * 12
    lib.rcwa_differential_integrate.argtypes = lib.rcwa_rcwa_integrate.argtypes
    lib.rcwa_redheffer_integrate.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                             C.c_int, RCWA_SAMPLER, C.c_void_p] + [C.c_void_p] * 10 + [_IP, _IP]
    lib.rcwa_zgemm_batched.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p, rcwa_cplx, rcwa_cplx, C.c_int, C.c_void_p]
    _FP = C.POINTER(C.c_float)
    lib.rcwa_mlp_create.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                    C.POINTER(C.c_void_p)]
    lib.rcwa_mlp_destroy.argtypes = [C.c_void_p]
    lib.rcwa_mlp_destroy.restype = None
    lib.rcwa_mlp_param_count.argtypes = [C.c_void_p]
    lib.rcwa_mlp_param_count.restype = C.c_longlong
    lib.rcwa_mlp_get_params.argtypes = [C.c_void_p, _FP]
    lib.rcwa_mlp_set_params.argtypes = [C.c_void_p, _FP]
    lib.rcwa_mlp_set_data.argtypes = [C.c_void_p, _FP, _FP, C.c_int]
    lib.rcwa_mlp_train.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_ulonglong, _FP]
    lib.rcwa_mlp_loss_grad.argtypes = [C.c_void_p, _FP, _FP, C.c_int, _DP, _FP]
    lib.rcwa_mlp_predict_fp32.argtypes = [C.c_void_p, _FP, C.c_int, _FP]
    lib.rcwa_mlp_predict.argtypes = [C.c_void_p, _FP, C.c_int, _FP]
    lib.rcwa_mlp_nn_distance.argtypes = [C.c_void_p, _FP, C.c_int, C.c_int, _FP]
    lib.rcwa_plan_schedule.argtypes = [C.c_void_p, C.c_int, _IP]
    lib.rcwa_tuner_create.argtypes = [C.POINTER(C.c_void_p)]
    lib.rcwa_tuner_destroy.argtypes = [C.c_void_p]
    lib.rcwa_tuner_destroy.restype = None
    lib.rcwa_tuner_set_sms.argtypes = [C.c_void_p, C.c_int]
    lib.rcwa_tuner_candidates.argtypes = [C.c_int, C.c_int, _IP]
    lib.rcwa_tuner_default.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    lib.rcwa_tuner_set.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.rcwa_tuner_get.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _IP]
    lib.rcwa_tuner_count.argtypes = [C.c_void_p]
    lib.rcwa_tuner_entry.argtypes = [C.c_void_p, C.c_int, _IP, _IP, _IP, _IP, _IP, _IP, _DP]
    lib.rcwa_tuner_save.argtypes = [C.c_void_p, C.c_char_p]
    lib.rcwa_tuner_load.argtypes = [C.c_void_p, C.c_char_p]
    lib.rcwa_engine_set_tuner.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.rcwa_tuner_measure.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, _IP, _DP]
    lib.rcwa_set_qr_sweep_limit.argtypes = [C.c_int]
    lib.rcwa_set_eig_cluster.argtypes = [C.c_int]
    lib.rcwa_eig_cluster_size.argtypes = [C.c_int, C.c_int]
    lib.rcwa_set_lu_cluster.argtypes = [C.c_int]
    lib.rcwa_plan_field_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _IP]
    lib.rcwa_plan_field.argtypes = [C.c_void_p, C.c_int, rcwa_cplx, rcwa_cplx, C.c_int, C.c_double, C.c_int, C.c_int,
                                    C.c_void_p]
    lib.rcwa_lu_cluster_size.argtypes = [C.c_int, C.c_int]
    lib.rcwa_plan_smatrix.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    _lib = lib
    return lib


def set_qr_sweep_limit(sweeps: int) -> None:
    """Cap the QR sweeps of every later eigensolve (0: the built-in budget);
    the failure-injection hook of the RCWA_ERR_NOCONV path."""
    rc = load().rcwa_set_qr_sweep_limit(int(sweeps))
    if rc:
        raise RcwaError(rc, "set_qr_sweep_limit")


def set_eig_cluster(ctas: int) -> None:
    """CTAs per matrix of the eigensolver's Hessenberg and Schur kernels for
    every later eigensolve (0: automatic, 1..8: forced)."""
    rc = load().rcwa_set_eig_cluster(int(ctas))
    if rc:
        raise RcwaError(rc, "set_eig_cluster")


def eig_cluster_size(n: int, batch: int) -> int:
    """The team size the current setting gives a batch of order-n matrices."""
    return int(load().rcwa_eig_cluster_size(int(n), int(batch)))


def set_lu_cluster(ctas: int) -> None:
    """CTAs per matrix of the LU panel step (0: automatic, 1..8: forced)."""
    rc = load().rcwa_set_lu_cluster(int(ctas))
    if rc:
        raise RcwaError(rc, "set_lu_cluster")


def lu_cluster_size(n: int, batch: int) -> int:
    """The LU panel team size the current setting gives a batch of order-n matrices."""
    return int(load().rcwa_lu_cluster_size(int(n), int(batch)))


def _d(a):
    return a.ctypes.data_as(_DP)


def _v(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_IP)


class RcwaError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"rcwa status {code} ({load().rcwa_status_string(code).decode()}) {msg}")


class Stack:
    """A layer stack on a common cell grid (owns its numpy buffers); mu, when
    given, is the relative permeability on the same grid (None: 1)."""

    def __init__(self, nHx, nHy, cx, cy, eps, thickness, mu=None):
        self.nHx, self.nHy = int(nHx), int(nHy)
        self.cx = np.ascontiguousarray(cx, dtype=np.float64)
        self.cy = np.ascontiguousarray(cy, dtype=np.float64)
        self.eps = np.ascontiguousarray(eps, dtype=np.complex128)
        assert self.eps.ndim == 3 and self.eps.shape[1:] == (self.cy.size - 1, self.cx.size - 1)
        self.thickness = np.ascontiguousarray(thickness, dtype=np.float64)
        assert self.thickness.size == self.eps.shape[0]
        self.mu = None if mu is None else np.ascontiguousarray(mu, dtype=np.complex128)
        assert self.mu is None or self.mu.shape == self.eps.shape

    @property
    def N(self):
        return (2 * self.nHx + 1) * (2 * self.nHy + 1)

    def c_struct(self):
        return rcwa_stack(self.nHx, self.nHy, self.cx.size, self.cy.size, self.cx.ctypes.data, self.cy.ctypes.data,
                          self.eps.shape[0], self.eps.ctypes.data, self.thickness.ctypes.data,
                          None if self.mu is None else self.mu.ctypes.data)


class TableStack:
    """A layer stack whose patterned layers are 2D Laurent coefficient tables
    (rcwa_table_stack): f2d [n_layers - 2, 4nHx + 1, 4nHy + 1], the uniform
    half-spaces' permittivities eps_half (2), thickness [n_layers]."""

    def __init__(self, nHx, nHy, Lx, Ly, eps_half, f2d, thickness):
        self.nHx, self.nHy = int(nHx), int(nHy)
        self.Lx, self.Ly = float(Lx), float(Ly)
        self.eps_half = np.ascontiguousarray(eps_half, dtype=np.complex128)
        self.f2d = np.ascontiguousarray(f2d, dtype=np.complex128)
        self.thickness = np.ascontiguousarray(thickness, dtype=np.float64)
        assert self.eps_half.shape == (2,)
        assert self.f2d.shape == (self.thickness.size - 2, 4 * self.nHx + 1, 4 * self.nHy + 1)

    @property
    def N(self):
        return (2 * self.nHx + 1) * (2 * self.nHy + 1)

    def c_struct(self):
        return rcwa_table_stack(self.nHx, self.nHy, self.Lx, self.Ly, self.thickness.size, self.eps_half.ctypes.data,
                                self.f2d.ctypes.data, self.thickness.ctypes.data)


class Engine:
    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.rcwa_engine_create(device, C.byref(h))
        if rc:
            raise RcwaError(rc, "engine_create")
        self.h = h
        # plans and networks of this engine: destroyed before the engine, whose
        # buffer pool and workspace cache they return their memory to
        self._children = weakref.WeakSet()

    def close(self):
        if self.h:
            for child in list(self._children):
                child.close()
            self.lib.rcwa_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self):
        return self.lib.rcwa_engine_last_error(self.h).decode()

    def _check(self, rc, what):
        if rc:
            raise RcwaError(rc, f"{what}: {self.last_error()}")

    def set_tuner(self, tuner, mode=RCWA_TUNING_AUTO):
        """Consult `tuner` (a Tuner) when plans are built; mode RCWA_TUNING_OFF,
        _TABLE or _AUTO (measure on a miss).  The engine keeps a reference."""
        self._tuner = tuner
        self._check(self.lib.rcwa_engine_set_tuner(self.h, tuner.h if tuner is not None else None, mode),
                    "engine_set_tuner")

    # -- batched solve ------------------------------------------------------
    @staticmethod
    def _pack(stacks: Sequence[Stack], points, pxy):
        kind = rcwa_table_stack if isinstance(stacks[0], TableStack) else rcwa_stack
        st = (kind * len(stacks))(*[s.c_struct() for s in stacks])
        pts = np.asarray(points, dtype=np.float64).reshape(-1, 4)
        cp = (rcwa_point * len(pts))(*[rcwa_point(int(p[0]), p[1], p[2], p[3]) for p in pts])
        pxy = np.ascontiguousarray(pxy, dtype=np.complex128)
        n_exc = pxy.shape[1]
        assert pxy.shape == (len(pts), n_exc, 2)
        return st, cp, pxy, n_exc

    def solve_batch(self, stacks, points, pxy, orders=True, precision=RCWA_PREC_FP64):
        """points: rows (stack, lambda, kx0, ky0); pxy: [n_pts][n_exc][2] complex.
        Returns R, T [n_pts, n_exc], per-order lists (REF, TRN) [n_pts] of
        [n_exc, N] arrays, status [n_pts]."""
        st, cp, pxy, n_exc = self._pack(stacks, points, pxy)
        npt = len(cp)
        R = np.zeros((npt, n_exc))
        T = np.zeros((npt, n_exc))
        Ns = [stacks[int(p.stack)].N for p in cp]
        tot = sum(Ns) * n_exc
        ref = np.zeros(max(tot, 1)) if orders else None
        trn = np.zeros(max(tot, 1)) if orders else None
        status = np.zeros(npt, dtype=np.int32)
        fn = self.lib.rcwa_engine_solve_tables if isinstance(stacks[0], TableStack) else self.lib.rcwa_engine_solve_batch
        rc = fn(self.h, st, len(stacks), cp, npt, n_exc, _v(pxy), precision, _d(R), _d(T),
                _d(ref) if orders else None, _d(trn) if orders else None, _i(status))
        if rc and not np.any(status):
            self._check(rc, "solve_batch")
        REF = TRN = None
        if orders:
            REF, TRN, o = [], [], 0
            for N in Ns:
                REF.append(ref[o:o + n_exc * N].reshape(n_exc, N))
                TRN.append(trn[o:o + n_exc * N].reshape(n_exc, N))
                o += n_exc * N
        return R, T, REF, TRN, status

    def plan(self, stacks, points, pxy, precision=RCWA_PREC_FP64):
        return Plan(self, stacks, points, pxy, precision)

    # -- stage entry points --------------------------------------------------
    def fourier1d(self, x, d, f, M):
        x = np.ascontiguousarray(x, dtype=np.float64)
        f = np.ascontiguousarray(f, dtype=np.complex128)
        out = np.zeros(M, dtype=np.complex128)
        self._check(self.lib.rcwa_fourier1d(self.h, _d(x), x.size, d, _v(f), M, _v(out)), "fourier1d")
        return out

    def fourier2d(self, cx, cy, f, nx, ny, opt):
        cx = np.ascontiguousarray(cx, dtype=np.float64)
        cy = np.ascontiguousarray(cy, dtype=np.float64)
        f = np.ascontiguousarray(f, dtype=np.complex128)
        out = np.zeros((nx * ny, nx * ny), dtype=np.complex128)
        self._check(self.lib.rcwa_fourier2d(self.h, _d(cx), cx.size, _d(cy), cy.size, _v(f), nx, ny, opt, _v(out)),
                    "fourier2d")
        return out

    def layer_solve(self, cx, cy, eps, nx, ny, alpha, beta, lam):
        cx = np.ascontiguousarray(cx, dtype=np.float64)
        cy = np.ascontiguousarray(cy, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.complex128)
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        beta = np.ascontiguousarray(beta, dtype=np.float64)
        n = 2 * nx * ny
        W = np.zeros((n, n), dtype=np.complex128)
        V = np.zeros((n, n), dtype=np.complex128)
        g = np.zeros(n, dtype=np.complex128)
        ev = np.zeros(n, dtype=np.complex128)
        self._check(self.lib.rcwa_layer_solve(self.h, _d(cx), cx.size, _d(cy), cy.size, _v(eps), nx, ny, _d(alpha),
                                              _d(beta), lam, _v(W), _v(V), _v(g), _v(ev)), "layer_solve")
        return W, V, g, ev

    def zgeev(self, A):
        A = np.ascontiguousarray(A, dtype=np.complex128)
        if A.ndim == 2:
            A = A[None]
        b, n, _ = A.shape
        w = np.zeros((b, n), dtype=np.complex128)
        VR = np.zeros((b, n, n), dtype=np.complex128)
        info = np.zeros(b, dtype=np.int32)
        rc = self.lib.rcwa_zgeev_batched(self.h, n, b, _v(A), _v(w), _v(VR), _i(info))
        if rc and not np.any(info):
            self._check(rc, "zgeev")
        return w, VR, info

    def zgemm(self, A, B, C=None, alpha=1.0, beta=0.0, precision=RCWA_PREC_FP64):
        """Batched D = alpha A B + beta C; (batch, M, K) x (batch, K, N)."""
        A, B = self._batch3(A, B)
        b, M, K = A.shape
        N = B.shape[2]
        Cm = None if C is None else self._batch3(C)[0]
        D = np.zeros((b, M, N), dtype=np.complex128)
        al, be = complex(alpha), complex(beta)
        self._check(self.lib.rcwa_zgemm_batched(self.h, M, N, K, b, _v(A), _v(B), _v(Cm), rcwa_cplx(al.real, al.imag),
                                                rcwa_cplx(be.real, be.imag), precision, _v(D)), "zgemm")
        return D

    @staticmethod
    def _batch3(*mats):
        out = [np.ascontiguousarray(m, dtype=np.complex128) for m in mats]
        return [m[None] if m.ndim == 2 else m for m in out]

    def slab_smatrix(self, W, V, gamma, W0, V0, lam, wz):
        """(Rud, Tuu) of z-uniform slabs: dtmm::RCWAScatterMatrix::compute_v2
        (rcwa/RCWAScatterMatrix.cpp:90-146).  Matrices (batch, n, n) or (n, n);
        gamma (batch, n); lam and wz scalars or (batch,)."""
        W, V, W0, V0 = self._batch3(W, V, W0, V0)
        b, n, _ = W.shape
        g = np.ascontiguousarray(np.broadcast_to(gamma, (b, n)), dtype=np.complex128)
        lam = np.ascontiguousarray(np.broadcast_to(np.asarray(lam, dtype=np.float64), (b,)))
        wz = np.ascontiguousarray(np.broadcast_to(np.asarray(wz, dtype=np.float64), (b,)))
        Rud = np.zeros((b, n, n), dtype=np.complex128)
        Tuu = np.zeros((b, n, n), dtype=np.complex128)
        st = np.zeros(b, dtype=np.int32)
        rc = self.lib.rcwa_slab_smatrix_batched(self.h, n, b, _v(W), _v(V), _v(g), _v(W0), _v(V0), _d(lam), _d(wz),
                                                _v(Rud), _v(Tuu), _i(st))
        if rc and not np.any(st):
            self._check(rc, "slab_smatrix")
        return Rud, Tuu, st

    def star_product(self, S, s):
        """Redheffer update of the running S-matrix ``S`` (dict Rud, Rdu, Tdd,
        Tuu) with slab ``s`` (dict rud, rdu, tdd, tuu) below it
        (core/RCWAIntegrator.cpp:57-67).  Returns the new dict and statuses."""
        Rud, Rdu, Tdd, Tuu = [m.copy() for m in self._batch3(S["Rud"], S["Rdu"], S["Tdd"], S["Tuu"])]
        rud, rdu, tdd, tuu = self._batch3(s["rud"], s["rdu"], s["tdd"], s["tuu"])
        b, n, _ = Rud.shape
        st = np.zeros(b, dtype=np.int32)
        rc = self.lib.rcwa_star_product_batched(self.h, n, b, _v(Rud), _v(Rdu), _v(Tdd), _v(Tuu), _v(rud), _v(rdu),
                                                _v(tdd), _v(tuu), _i(st))
        if rc and not np.any(st):
            self._check(rc, "star_product")
        return {"Rud": Rud, "Rdu": Rdu, "Tdd": Tdd, "Tuu": Tuu}, st

    def _integrate(self, fn, what, P, Q, nslab, lam, z0, z1):
        n = P.shape[1]
        out = {k: np.zeros((n, n), dtype=np.complex128) for k in ("Rud", "Rdu", "Tdd", "Tuu", "W0", "V0", "W1", "V1")}
        out["gam0"] = np.zeros(n, dtype=np.complex128)
        out["gam1"] = np.zeros(n, dtype=np.complex128)
        rc = fn(self.h, n, nslab, float(lam), float(z0), float(z1), _v(P), _v(Q),
                *[_v(out[k]) for k in ("Rud", "Rdu", "Tdd", "Tuu", "W0", "V0", "gam0", "W1", "V1", "gam1")])
        self._check(rc, what)
        return out

    @staticmethod
    def _samples(P, Q):
        P = np.ascontiguousarray(P, dtype=np.complex128)
        Q = np.ascontiguousarray(Q, dtype=np.complex128)
        if P.ndim != 3 or P.shape != Q.shape or P.shape[1] != P.shape[2]:
            raise ValueError("P, Q must be (samples, n, n)")
        return P, Q

    def rcwa_integrate(self, P, Q, lam, z0, z1):
        """RCWAIntegrator::compute (core/RCWAIntegrator.cpp:21-86) over sampled
        matrices: P, Q (nslab + 2, n, n) at z0, the slab midpoints and z1.
        Returns a dict with Rud, Rdu, Tdd, Tuu, W0, V0, gam0, W1, V1, gam1."""
        P, Q = self._samples(P, Q)
        if P.shape[0] < 2:
            raise ValueError("P, Q must be (nslab + 2, n, n)")
        return self._integrate(self.lib.rcwa_rcwa_integrate, "rcwa_integrate", P, Q, P.shape[0] - 2, lam, z0, z1)

    def redheffer_integrate(self, sample, n, lam, z0, z1, pe, max_intervals=100000):
        """RedhefferIntegrator::compute (core/RedhefferIntegrator.cpp:190-328):
        ``sample(z)`` returns the (n, n) matrices (P, Q) at depth z.  Returns
        the dict of rcwa_integrate plus N (accepted intervals) and n_eig."""
        failure = []

        def cb(user, z, Pp, Qp):
            try:
                P, Q = sample(z)
                for src, dst in ((P, Pp), (Q, Qp)):
                    a = np.ascontiguousarray(src, dtype=np.complex128)
                    if a.shape != (n, n):
                        raise ValueError("sampler returned shape %s" % (a.shape,))
                    C.memmove(dst, a.ctypes.data, a.nbytes)
                return 0
            except Exception as ex:  # reported after the call
                failure.append(ex)
                return 1

        fn = RCWA_SAMPLER(cb)
        out = {k: np.zeros((n, n), dtype=np.complex128) for k in ("Rud", "Rdu", "Tdd", "Tuu", "W0", "V0", "W1", "V1")}
        out["gam0"] = np.zeros(n, dtype=np.complex128)
        out["gam1"] = np.zeros(n, dtype=np.complex128)
        cnt = np.zeros(2, dtype=np.int32)
        rc = self.lib.rcwa_redheffer_integrate(
            self.h, n, float(lam), float(z0), float(z1), float(pe), int(max_intervals), fn, None,
            *[_v(out[k]) for k in ("Rud", "Rdu", "Tdd", "Tuu", "W0", "V0", "gam0", "W1", "V1", "gam1")],
            _i(cnt[0:1]), _i(cnt[1:2]))
        if failure:
            raise failure[0]
        self._check(rc, "redheffer_integrate")
        out["N"], out["n_eig"] = int(cnt[0]), int(cnt[1])
        return out

    def differential_integrate(self, P, Q, lam, z0, z1):
        """DifferentialIntegrator::compute (core/DifferentialIntegrator.cpp:21-133)
        over sampled matrices: P, Q (2 nslab + 1, n, n) at z0 + k dz/2.
        Returns the dict of rcwa_integrate."""
        P, Q = self._samples(P, Q)
        if P.shape[0] < 3 or P.shape[0] % 2 == 0:
            raise ValueError("P, Q must be (2 nslab + 1, n, n)")
        return self._integrate(self.lib.rcwa_differential_integrate, "differential_integrate", P, Q,
                               (P.shape[0] - 1) // 2, lam, z0, z1)

    def ofd_solve(self, setup, orders=True):
        """The rcwa_run computation for a setup object with the
        fields of rcwa_ofd_setup (layers with eps1..thickness, poles, freqs)."""
        L = len(setup.layers)
        lay = (rcwa_layer_spec * L)(*[rcwa_layer_spec(l.eps1, l.eps2, l.eps1i, l.eps2i, l.fill, l.fill_y,
                                                       l.thickness) for l in setup.layers])
        npo = len(setup.poles)
        pol = (rcwa_pole_spec * max(npo, 1))(*[rcwa_pole_spec(p.layer, p.side, p.einf, p.ae, p.be, p.ce)
                                               for p in setup.poles])
        fr = np.ascontiguousarray(setup.freqs, dtype=np.float64)
        py = setup.period_y if setup.period_y is not None else setup.period_x
        s = rcwa_ofd_setup(setup.nHx, setup.period_x, setup.nHy, py, L, lay, npo, pol, setup.theta, setup.phi,
                           fr.size, _d(fr))
        nf = fr.size
        nord = (2 * setup.nHx + 1) * (2 * setup.nHy + 1)
        R = np.zeros((nf, 2))
        T = np.zeros((nf, 2))
        oR = np.zeros((2, nf, nord)) if orders else None
        oT = np.zeros((2, nf, nord)) if orders else None
        st = np.zeros(nf, dtype=np.int32)
        rc = self.lib.rcwa_ofd_solve(self.h, C.byref(s), _d(R), _d(T), _d(oR) if orders else None,
                                     _d(oT) if orders else None, _i(st))
        if rc and not np.any(st):
            self._check(rc, "ofd_solve")
        return R, T, oR, oT, st


class Plan:
    """Inputs resident on the device; execute() enqueues the kernels only."""

    def __init__(self, eng: Engine, stacks, points, pxy, precision=RCWA_PREC_FP64):
        self.eng = eng
        self.stacks = stacks
        st, cp, pxy, n_exc = Engine._pack(stacks, points, pxy)
        self._keep = (st, cp, pxy)
        self.n_pts, self.n_exc = len(cp), n_exc
        self.Ns = [stacks[int(p.stack)].N for p in cp]
        h = C.c_void_p()
        fn = eng.lib.rcwa_plan_create_tables if isinstance(stacks[0], TableStack) else eng.lib.rcwa_plan_create
        rc = fn(eng.h, st, len(stacks), cp, len(cp), n_exc, _v(pxy), precision, C.byref(h))
        eng._check(rc, "plan_create")
        self.h = h
        eng._children.add(self)

    def execute(self, stream: Optional[int] = None):
        self.eng._check(self.eng.lib.rcwa_plan_execute(self.h, C.c_void_p(stream) if stream else None),
                        "plan_execute")

    def launch_count(self):
        return int(self.eng.lib.rcwa_plan_launch_count(self.h))

    def schedule(self):
        """Per chunk: dict of n, points, lu_interface, lu_tau, schur_crossover,
        product (0: 3xTF32 tensor cores, 1: FP64 tensor path)."""
        count = self.eng.lib.rcwa_plan_schedule(self.h, -1, None)
        out, v = [], (C.c_int * 6)()
        keys = ("n", "points", "lu_interface", "lu_tau", "schur_crossover", "product")
        for c in range(max(count, 0)):
            self.eng.lib.rcwa_plan_schedule(self.h, c, C.cast(v, _IP))
            out.append(dict(zip(keys, list(v))))
        return out

    def field(self, point, px, py, slice, coord, component, nres1=500):
        """One field component inside the stack (rcwa_plan_field): slice 0 XY
        at depth coord, 1 XZ at y = coord, 2 YZ at x = coord; component 0..5 =
        Ex, Ey, Ez, Hx, Hy, Hz.  Returns a (rows, nres1) complex array."""
        rows = np.zeros(1, dtype=np.int32)
        self.eng._check(self.eng.lib.rcwa_plan_field_rows(self.h, int(point), int(slice), int(nres1), _i(rows)),
                        "plan_field_rows")
        out = np.zeros((int(rows[0]), int(nres1)), dtype=np.complex128)
        px, py = complex(px), complex(py)
        self.eng._check(self.eng.lib.rcwa_plan_field(self.h, int(point), rcwa_cplx(px.real, px.imag),
                                                     rcwa_cplx(py.real, py.imag), int(slice), float(coord),
                                                     int(component), int(nres1), _v(out)), "plan_field")
        return out

    def rescatter(self, pxy):
        """New incident polarisations (n_pts, n_exc, 2) on the kept S-matrices."""
        pxy = np.ascontiguousarray(pxy, dtype=np.complex128).reshape(self.n_pts, self.n_exc, 2)
        self.eng._check(self.eng.lib.rcwa_plan_rescatter(self.h, _v(pxy)), "plan_rescatter")

    def smatrix(self, point):
        """(Rud, Tdd) of an executed single-chunk plan's point: the
        RCWASolver::Rud() / Tdd() matrices (rcwa/RCWASolver.h:141-142)."""
        n = 2 * self.Ns[point]
        Rud = np.zeros((n, n), dtype=np.complex128)
        Tdd = np.zeros((n, n), dtype=np.complex128)
        self.eng._check(self.eng.lib.rcwa_plan_smatrix(self.h, int(point), _v(Rud), _v(Tdd)), "plan_smatrix")
        return Rud, Tdd

    def set_profiling(self, on=True):
        self.eng._check(self.eng.lib.rcwa_plan_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def stage_times(self):
        """{stage name: milliseconds} of the last execution (profiling on)."""
        ms = np.zeros(64)
        n = self.eng.lib.rcwa_plan_stage_times(self.h, _d(ms), 64)
        return {self.eng.lib.rcwa_stage_name(i).decode(): float(ms[i]) for i in range(n)}

    def results(self, orders=False):
        R = np.zeros((self.n_pts, self.n_exc))
        T = np.zeros((self.n_pts, self.n_exc))
        tot = sum(self.Ns) * self.n_exc
        ref = np.zeros(max(tot, 1)) if orders else None
        trn = np.zeros(max(tot, 1)) if orders else None
        status = np.zeros(self.n_pts, dtype=np.int32)
        rc = self.eng.lib.rcwa_plan_results(self.h, _d(R), _d(T), _d(ref) if orders else None,
                                            _d(trn) if orders else None, _i(status))
        if rc and not np.any(status):
            self.eng._check(rc, "plan_results")
        return R, T, ref, trn, status

    def close(self):
        if self.h:
            self.eng.lib.rcwa_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _f(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The surrogate network of rcwa_mlp_* (training and inference on the GPU)."""

    def __init__(self, eng: Engine, n_in, n_hidden, n_layers, n_out, seed=0):
        self.eng = eng
        self.n_in, self.n_out = n_in, n_out
        self.dims = [n_in] + [n_hidden] * n_layers + [n_out]
        h = C.c_void_p()
        eng._check(eng.lib.rcwa_mlp_create(eng.h, n_in, n_hidden, n_layers, n_out, seed, C.byref(h)), "mlp_create")
        self.h = h
        eng._children.add(self)

    def param_count(self):
        return int(self.eng.lib.rcwa_mlp_param_count(self.h))

    def get_params(self):
        p = np.zeros(self.param_count(), dtype=np.float32)
        self.eng._check(self.eng.lib.rcwa_mlp_get_params(self.h, _f(p)), "mlp_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self.eng._check(self.eng.lib.rcwa_mlp_set_params(self.h, _f(p)), "mlp_set_params")

    def set_data(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        self.eng._check(self.eng.lib.rcwa_mlp_set_data(self.h, _f(X), _f(Y), X.shape[0]), "mlp_set_data")

    def train(self, epochs, batch, lr, seed=0):
        loss = np.zeros(epochs, dtype=np.float32)
        self.eng._check(self.eng.lib.rcwa_mlp_train(self.h, epochs, batch, lr, seed, _f(loss)), "mlp_train")
        return loss

    def loss_grad(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        loss = C.c_double()
        g = np.zeros(self.param_count(), dtype=np.float32)
        self.eng._check(self.eng.lib.rcwa_mlp_loss_grad(self.h, _f(X), _f(Y), X.shape[0], C.byref(loss), _f(g)),
                        "mlp_loss_grad")
        return loss.value, g

    def predict(self, X, tensor_cores=True):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], self.n_out), dtype=np.float32)
        fn = self.eng.lib.rcwa_mlp_predict if tensor_cores else self.eng.lib.rcwa_mlp_predict_fp32
        self.eng._check(fn(self.h, _f(X), X.shape[0], _f(Y)), "mlp_predict")
        return Y

    def nn_distance(self, X, skip_self=False):
        """Squared distance of every row of X to its nearest training row."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        d2 = np.zeros(X.shape[0], dtype=np.float32)
        self.eng._check(self.eng.lib.rcwa_mlp_nn_distance(self.h, _f(X), X.shape[0], 1 if skip_self else 0, _f(d2)),
                        "mlp_nn_distance")
        return d2

    def close(self):
        if self.h:
            self.eng.lib.rcwa_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tuner:
    """Schedule table of the engine's autotuner (host data; see rcwa_tuner_*).
    Decisions are named "lu", "schur" and "product"."""

    def __init__(self, lib=None):
        self.lib = lib or load()
        h = C.c_void_p()
        rc = self.lib.rcwa_tuner_create(C.byref(h))
        if rc:
            raise RcwaError(rc, "tuner_create")
        self.h = h

    @staticmethod
    def _op(op):
        return TUNE_OPS[op] if isinstance(op, str) else int(op)

    def set_sms(self, sms):
        if self.lib.rcwa_tuner_set_sms(self.h, sms):
            raise RcwaError(RCWA_ERR_INVALID, "tuner_set_sms")

    def candidates(self, op, n):
        c = (C.c_int * 4)()
        k = self.lib.rcwa_tuner_candidates(self._op(op), n, C.cast(c, _IP))
        if k < 0:
            raise RcwaError(RCWA_ERR_INVALID, "tuner_candidates")
        return list(c)[:k]

    def default(self, op, n, batch):
        return int(self.lib.rcwa_tuner_default(self.h, self._op(op), n, batch))

    def set(self, op, n, batch, choice):
        rc = self.lib.rcwa_tuner_set(self.h, self._op(op), n, batch, choice)
        if rc:
            raise RcwaError(rc, "tuner_set")

    def get(self, op, n, batch):
        """The recorded choice, or None."""
        c = C.c_int(-1)
        rc = self.lib.rcwa_tuner_get(self.h, self._op(op), n, batch, C.byref(c))
        if rc:
            raise RcwaError(rc, "tuner_get")
        return None if c.value < 0 else c.value

    def entries(self):
        names = {v: k for k, v in TUNE_OPS.items()}
        out = []
        for i in range(self.lib.rcwa_tuner_count(self.h)):
            op, n, cls, ch, nc = (C.c_int() for _ in range(5))
            cand = (C.c_int * 4)()
            ms = (C.c_double * 4)()
            self.lib.rcwa_tuner_entry(self.h, i, C.byref(op), C.byref(n), C.byref(cls), C.byref(ch), C.byref(nc),
                                      C.cast(cand, _IP), C.cast(ms, _DP))
            out.append({"op": names[op.value], "n": n.value, "batch_class": cls.value, "choice": ch.value,
                        "ms": {int(cand[k]): float(ms[k]) for k in range(nc.value)}})
        return out

    def save(self, path):
        rc = self.lib.rcwa_tuner_save(self.h, os.fsencode(path))
        if rc:
            raise RcwaError(rc, "tuner_save")

    def load(self, path):
        rc = self.lib.rcwa_tuner_load(self.h, os.fsencode(path))
        if rc:
            raise RcwaError(rc, "tuner_load")

    def measure(self, eng: Engine, op, n, batch):
        """Time every candidate now; returns (choice, {candidate: ms})."""
        ch = C.c_int(-1)
        ms = (C.c_double * 4)()
        eng._check(self.lib.rcwa_tuner_measure(eng.h, self.h, self._op(op), n, batch, C.byref(ch), C.cast(ms, _DP)),
                   "tuner_measure")
        cand = self.candidates(op, n)
        return ch.value, {c: float(ms[k]) for k, c in enumerate(cand)}

    def close(self):
        if self.h:
            self.lib.rcwa_tuner_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
