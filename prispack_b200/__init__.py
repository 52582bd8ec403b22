"""B200 solve phase for PrisPack: Python view of the C ABI (include/prism_solve.h).

The classes mirror the reference's C++ interface names and argument meaning
(HOST::CSRMatrix, IncompleteCholesky, IncompleteLU, IncompleteLDLT, CG, GMRES;
include/Preconditioner/BasePreconditon.h:34-145, include/Solver/BaseSolver.h:9-17),
so that code written against the reference reads the same.  All work runs in
``_lib/libprism_solve.so``; there is no CPU fallback: importing this package
without the built library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libprism_solve.so")

# ---- enums (include/prism_solve.h) ------------------------------------------------
PRISM_FP64, PRISM_FP32 = 0, 1
# float factor values and single-precision arithmetic inside the streamed triangular sweeps
PRISM_FP32_APPLY = 2
PRECOND_NONE, PRECOND_IC, PRECOND_ILUT, PRECOND_ILDLT, PRECOND_GMSLR, PRECOND_AMSED = range(6)
SOLVER_FCG, SOLVER_CG, SOLVER_FGMRES, SOLVER_GMRES = range(4)
LAUNCH_AUTO, LAUNCH_STREAM = range(2)
# reference spellings (include/Solver/CG.h:14-18, include/Solver/GMRES.h:15-18)
NormalCG, FlexibleCG = "NormalCG", "FlexibleCG"
NormalGMRES, FlexibleGMRES = "NormalGMRES", "FlexibleGMRES"
MAX_ITER_NUM_SOLVER = 500  # config/config.h:25

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_ZERO_PIVOT", 4: "ERR_NOT_SPD", 5: "ERR_NOT_READY",
          6: "ERR_TIMEOUT", 7: "ERR_NONFINITE", 8: "ERR_ALLOC", 9: "ERR_UNSUPPORTED", 10: "ERR_BAD_MATRIX"}


class PrismError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class SolveOpts(C.Structure):
    _fields_ = [("solver", C.c_int32), ("tol", C.c_double), ("max_iter", C.c_uint32), ("restart", C.c_uint32),
                ("x_ref", C.c_void_p), ("launch_mode", C.c_int32)]


class AmsedOpts(C.Structure):
    """prism_amsed_opts (include/prism_solve.h); defaults from prism_amsed_default_opts."""
    _fields_ = [("levels", C.c_int32), ("lanczos_steps", C.c_int32), ("low_rank", C.c_int32),
                ("eig_bound", C.c_double), ("lowrank_type", C.c_int32), ("lanczos_type", C.c_int32),
                ("reorder", C.c_int32), ("factor_tol", C.c_double), ("minsep", C.c_uint32), ("seed", C.c_uint64)]


# reference enum spellings (AMSEDPrecondition.h:53-72, MatrixReorderTools.h:14-18)
AMSEDBasic, AMSEDEigenvalueDeflation = 0, 1
UseClassicLanczos, UseRestartLanczos = 0, 1
MatrixReorderNo, MatrixReorderAMD, MatrixReorderRCM = 0, 1, 2


class SolveStats(C.Structure):
    _fields_ = [("num_iter", C.c_int32), ("converged", C.c_int32), ("final_error", C.c_double),
                ("true_rel_residual", C.c_double), ("precond_applies", C.c_uint32),
                ("spmv_count", C.c_uint32), ("device_ms", C.c_double), ("forward_error", C.c_double),
                ("host_syncs", C.c_uint32), ("graph_nodes", C.c_uint32)]


_lib = None
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p

# every exported symbol with its argument types (the C header, one to one)
_SIGS = {
    "prism_last_error": (C.c_char_p, []),
    "prism_version": (C.c_int32, []),
    "prism_kernel_launch_count": (C.c_uint64, []),
    "prism_selftest_wait_timeout": (C.c_int32, [C.c_int32, C.c_uint64, C.POINTER(C.c_int32)]),
    "prism_lowrank_block_run": (C.c_int32, [C.c_int32, C.c_uint32, C.c_uint32, C.c_uint32, _f64p, _f64p, _f64p, _f64p,
                                            C.c_int32]),
    "prism_selftest_stream_layout_capped": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, _vp, C.c_int32, C.c_int32,
                                                        C.c_int32, C.c_uint32, C.c_uint32, C.c_uint32, _f64p,
                                                        _f64p, C.POINTER(C.c_uint32)]),
    "prism_selftest_stream_layout": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, _vp, C.c_int32, C.c_int32,
                                                 C.c_int32, C.c_uint32, C.c_uint32, _f64p, _f64p]),
    "prism_stream_sweep_order": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, _vp, C.c_int32, C.c_int32, C.c_int32,
                                             C.c_uint32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "prism_stream_sweep_run": (C.c_int32, [C.c_int32, C.c_uint32, _u32p, _u32p, _f64p, _vp, C.c_int32, C.c_int32,
                                           C.c_int32, C.c_uint32, _f64p, _f64p]),
    "prism_precond_sweep_order": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_uint32), _vp, _vp, _vp, _vp, _vp,
                                              _vp, _vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "prism_precond_sweep_rhs_map": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_uint64), _vp,
                                                _vp, _vp]),
    "prism_stream_sweep_pair": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, _vp, C.c_int32, C.c_int32, C.c_int32,
                                            C.POINTER(C.c_uint64), _vp, _vp, _vp, C.POINTER(C.c_uint64), _vp, _vp,
                                            _vp]),
    "prism_mtx_read": (C.c_int32, [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                   C.POINTER(C.c_uint64), _vp, _vp, _vp]),
    "prism_mtx_read_dense": (C.c_int32, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), _vp]),
    "prism_laplacian_dims": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "prism_laplacian_fill": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                         C.c_double, _u32p, _u32p, _f64p]),
    "prism_create": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, C.c_int32, C.POINTER(_vp)]),
    "prism_destroy": (C.c_int32, [_vp]),
    "prism_set_stream": (C.c_int32, [_vp, _vp]),
    "prism_dims": (C.c_int32, [_vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    "prism_spmv_device": (C.c_int32, [_vp, _vp, _vp]),
    "prism_spmv_shape": (C.c_int32, [_vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "prism_spmv": (C.c_int32, [_vp, _f64p, _f64p]),
    "prism_set_precond_none": (C.c_int32, [_vp]),
    "prism_set_precond_ic": (C.c_int32, [_vp, C.c_double, C.c_int32]),
    "prism_set_precond_ildlt": (C.c_int32, [_vp, C.c_double, C.c_int32]),
    "prism_set_precond_ilut": (C.c_int32, [_vp, C.c_uint32, C.c_double, C.c_int32]),
    "prism_precond_nnz": (C.c_int32, [_vp, C.POINTER(C.c_uint64)]),
    "prism_precond_type": (C.c_int32, [_vp, C.POINTER(C.c_int32)]),
    "prism_precond_factor": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                         _vp, _vp, _vp, _vp]),
    "prism_precond_levels": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_uint32)]),
    "prism_factor_create": (C.c_int32, [C.c_int32, C.c_uint32, _u32p, _u32p, _f64p, C.c_double, C.c_uint32,
                                        C.c_int32, C.POINTER(_vp)]),
    "prism_factor_destroy": (C.c_int32, [_vp]),
    "prism_factor_get": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                     _vp, _vp, _vp, _vp]),
    "prism_factor_info": (C.c_int32, [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "prism_set_precond_factor": (C.c_int32, [_vp, _vp]),
    "prism_precond_sweep_device": (C.c_int32, [_vp, C.c_int32, _vp, _vp, C.c_int32]),
    "prism_precond_sweep_info": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "prism_amsed_default_opts": (None, [C.POINTER(AmsedOpts)]),
    "prism_set_precond_amsed": (C.c_int32, [_vp, C.POINTER(AmsedOpts), C.c_int32]),
    "prism_factor_create_amsed": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, C.POINTER(AmsedOpts), C.c_int32,
                                              C.POINTER(_vp)]),
    "prism_amsed_info": (C.c_int32, [_vp, C.POINTER(C.c_uint32), _vp, _vp, _vp, C.POINTER(C.c_uint64)]),
    "prism_amsed_perm": (C.c_int32, [_vp, _vp]),
    "prism_amsed_dom_ptr": (C.c_int32, [_vp, C.c_int32, _vp]),
    "prism_amsed_block": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                      _vp, _vp, _vp, _vp]),
    "prism_amsed_coupling": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64),
                                         _vp, _vp, _vp]),
    "prism_amsed_lowrank": (C.c_int32, [_vp, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), _vp, _vp]),
    "prism_gmslr_default_opts": (None, [C.POINTER(AmsedOpts)]),
    "prism_set_precond_gmslr": (C.c_int32, [_vp, C.POINTER(AmsedOpts), C.c_int32]),
    "prism_factor_create_gmslr": (C.c_int32, [C.c_uint32, _u32p, _u32p, _f64p, C.POINTER(AmsedOpts), C.c_int32,
                                              C.POINTER(_vp)]),
    "prism_gmslr_block": (C.c_int32, [_vp, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_uint32),
                                      C.POINTER(C.c_uint64), _vp, _vp, _vp, _vp]),
    "prism_residual_norms_noalloc": (C.c_int32, [C.c_int32, C.c_uint32, _vp, _vp, _vp, _vp, _vp, C.c_uint32,
                                                 C.c_uint64, _vp, _vp]),
    "prism_apply_batched_device": (C.c_int32, [_vp, C.c_uint32, _vp, _vp, C.c_uint64]),
    "prism_solve_batched_device": (C.c_int32, [_vp, C.POINTER(SolveOpts), C.c_uint32, _vp, _vp, C.c_uint64,
                                               C.POINTER(SolveStats)]),
    "prism_solve_batched": (C.c_int32, [_vp, C.POINTER(SolveOpts), C.c_uint32, _f64p, _f64p, C.c_uint64,
                                        C.POINTER(SolveStats)]),
    "prism_solve_segments_device": (C.c_int32, [_vp, C.POINTER(SolveOpts), C.c_uint32, _u32p, _vp, _vp,
                                                C.POINTER(SolveStats)]),
    "prism_solve_segments": (C.c_int32, [_vp, C.POINTER(SolveOpts), C.c_uint32, _u32p, _f64p, _f64p,
                                         C.POINTER(SolveStats)]),
    "prism_update_values": (C.c_int32, [_vp, _f64p]),
    "prism_refactor": (C.c_int32, [_vp]),
    "prism_update_values_device": (C.c_int32, [_vp, _vp]),
    "prism_adjoint_solve_device": (C.c_int32, [_vp, C.POINTER(SolveOpts), _vp, _vp, _vp, _vp, C.POINTER(SolveStats)]),
    "prism_adjoint_solve": (C.c_int32, [_vp, C.POINTER(SolveOpts), _f64p, _f64p, _f64p, _vp, C.POINTER(SolveStats)]),
    "prism_apply_device": (C.c_int32, [_vp, _vp, _vp]),
    "prism_apply": (C.c_int32, [_vp, _f64p, _f64p]),
    "prism_solve_device": (C.c_int32, [_vp, C.POINTER(SolveOpts), _vp, _vp, C.POINTER(SolveStats)]),
    "prism_solve": (C.c_int32, [_vp, C.POINTER(SolveOpts), _f64p, _f64p, C.POINTER(SolveStats)]),
}


def load() -> C.CDLL:
    """Loads the solve-phase library; raises if it was never built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m prispack_b200.build` (no CPU fallback exists)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def exported_symbols():
    return list(_SIGS)


def _check(rc: int):
    if rc != 0:
        raise PrismError(rc, load().prism_last_error().decode())


def kernel_launch_count() -> int:
    return int(load().prism_kernel_launch_count())


def selftest_wait_timeout(device: int = 0, wait_ns: int = 50_000_000) -> int:
    """Runs the bounded-wait self test; returns the device status the wait raised (6 = timeout)."""
    st = C.c_int32(-1)
    _check(load().prism_selftest_wait_timeout(device, wait_ns, C.byref(st)))
    return st.value


def lowrank_block_run(W, H, X, Y, *, tensor: bool, device: int = 0):
    """Y + W (H o (W^T X)) for W (nrem, rank), H (rank,), X and Y (nrem, k), k <= 64, on
    `device` (prism_lowrank_block_run): BF16 tensor cores when tensor, else FP64."""
    W = np.asarray(W, np.float64)
    nrem, rank = W.shape
    X = np.ascontiguousarray(X, np.float64)
    out = np.array(Y, np.float64, copy=True, order="C")
    _check(load().prism_lowrank_block_run(device, nrem, rank, X.shape[1], np.ascontiguousarray(W.T),
                                          np.ascontiguousarray(H, np.float64), X, out, int(bool(tensor))))
    return out


def selftest_stream_layout_capped(rowptr, col, val, in_, *, max_round_bytes: int, diag=None, op: int = 2,
                                  lower: bool = True, precision: int = 0, num_ctas: int = 4):
    """selftest_stream_layout with rounds cut short at max_round_bytes (the device layout's
    record cap; slab boundaries as the device layout chooses): (solution, largest record)."""
    rp = np.ascontiguousarray(rowptr, np.uint32)
    n = len(rp) - 1
    out = np.zeros(n)
    rec = C.c_uint32()
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    _check(load().prism_selftest_stream_layout_capped(n, rp, np.ascontiguousarray(col, np.uint32),
                                                      np.ascontiguousarray(val, np.float64),
                                                      d.ctypes.data if d is not None else None, op, int(lower),
                                                      precision, num_ctas, 0, max_round_bytes,
                                                      np.ascontiguousarray(in_, np.float64), out, C.byref(rec)))
    return out, rec.value


def selftest_stream_layout(rowptr, col, val, in_, *, diag=None, op: int = 2, lower: bool = True,
                           precision: int = 0, num_ctas: int = 4, rows_per_cta: int | None = None):
    """Host replay of the streamed round layout of the sweep kernel (no GPU): returns the
    sweep's solution as the kernel would compute it, or raises PrismError naming the flaw.
    rows_per_cta = 0 lets the layout choose the slab boundaries."""
    rp = np.ascontiguousarray(rowptr, np.uint32)
    n = len(rp) - 1
    rpc = rows_per_cta if rows_per_cta is not None else -(-n // num_ctas)
    out = np.zeros(n)
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    _check(load().prism_selftest_stream_layout(n, rp, np.ascontiguousarray(col, np.uint32),
                                               np.ascontiguousarray(val, np.float64),
                                               d.ctypes.data if d is not None else None, op, int(lower), precision,
                                               num_ctas, rpc, np.ascontiguousarray(in_, np.float64), out))
    return out


class SweepOrder:
    """The streamed sweep kernel's summation order (prism_stream_sweep_order): per row, its
    early positions eptr[r]:eptr[r+1] of (edep, ecoef) and its late ones kptr[r]:kptr[r+1]
    of (kdep, kcoef); a dependency of 0xFFFFFFFF is padding (coefficient 0)."""

    PAD = 0xFFFFFFFF

    def __init__(self, eptr, edep, ecoef, kptr, kdep, kcoef):
        self.eptr, self.edep, self.ecoef = eptr, edep, ecoef
        self.kptr, self.kdep, self.kcoef = kptr, kdep, kcoef
        self.diag, self.op, self.lower = None, None, None  # filled for a handle's sweep


def _fill_order(call, n):
    """Two-call fill of a SweepOrder: sizes first, then the arrays."""
    eptr = np.zeros(n + 1, np.uint32)
    kptr = np.zeros(n + 1, np.uint32)
    _check(call(eptr.ctypes.data, None, None, kptr.ctypes.data, None, None))
    ne, nk = int(eptr[-1]), int(kptr[-1])
    edep, ecoef = np.zeros(max(ne, 1), np.uint32), np.zeros(max(ne, 1))
    kdep, kcoef = np.zeros(max(nk, 1), np.uint32), np.zeros(max(nk, 1))
    _check(call(eptr.ctypes.data, edep.ctypes.data, ecoef.ctypes.data, kptr.ctypes.data, kdep.ctypes.data,
                kcoef.ctypes.data))
    return SweepOrder(eptr, edep[:ne], ecoef[:ne], kptr, kdep[:nk], kcoef[:nk])


def stream_sweep_order(rowptr, col, val, *, diag=None, op: int = 2, lower: bool = True, precision: int = 0,
                       num_ctas: int = 4) -> SweepOrder:
    """Summation order of the streamed sweep kernel for a gather-form triangular sweep (host only)."""
    rp = np.ascontiguousarray(rowptr, np.uint32)
    ci = np.ascontiguousarray(col, np.uint32)
    v = np.ascontiguousarray(val, np.float64)
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    n = len(rp) - 1
    lib = load()
    return _fill_order(lambda ep, ed, ec, kp, kd, kc: lib.prism_stream_sweep_order(
        n, rp, ci, v, d.ctypes.data if d is not None else None, op, int(lower), precision, num_ctas,
        ep, ed, ec, kp, kd, kc), n)


def stream_sweep_run(rowptr, col, val, in_, *, diag=None, op: int = 2, lower: bool = True, precision: int = 0,
                     num_ctas: int = 4, device: int = 0):
    """Runs the streamed sweep kernel alone on the GPU (same slabs as stream_sweep_order)."""
    rp = np.ascontiguousarray(rowptr, np.uint32)
    n = len(rp) - 1
    out = np.zeros(n)
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    _check(load().prism_stream_sweep_run(device, n, rp, np.ascontiguousarray(col, np.uint32),
                                         np.ascontiguousarray(val, np.float64),
                                         d.ctypes.data if d is not None else None, op, int(lower), precision,
                                         num_ctas, np.ascontiguousarray(in_, np.float64), out))
    return out


def stream_sweep_pair(rowptr, col, val, *, diag=None, op: int = 2, lower: bool = True, precision: int = 0):
    """Wavefront pairing of a gather-form sweep (prism_stream_sweep_pair, host only): the
    paired sweep (rowptr, col, val) and its right-hand side map (mptr, mdep, mcoef), with
    T^{-1} b = T'^{-1} (b - M b)."""
    rp = np.ascontiguousarray(rowptr, np.uint32)
    ci = np.ascontiguousarray(col, np.uint32)
    v = np.ascontiguousarray(val, np.float64)
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    n = len(rp) - 1
    lib = load()
    pn, mn = C.c_uint64(), C.c_uint64()
    dp = d.ctypes.data if d is not None else None
    _check(lib.prism_stream_sweep_pair(n, rp, ci, v, dp, op, int(lower), precision, C.byref(pn), None, None, None,
                                       C.byref(mn), None, None, None))
    prow = np.zeros(n + 1, np.uint32)
    pcol = np.zeros(max(pn.value, 1), np.uint32)
    pval = np.zeros(max(pn.value, 1))
    mptr = np.zeros(n + 1, np.uint32)
    mdep = np.zeros(max(mn.value, 1), np.uint32)
    mcoef = np.zeros(max(mn.value, 1))
    _check(lib.prism_stream_sweep_pair(n, rp, ci, v, dp, op, int(lower), precision, C.byref(pn), prow.ctypes.data,
                                       pcol.ctypes.data, pval.ctypes.data, C.byref(mn), mptr.ctypes.data,
                                       mdep.ctypes.data, mcoef.ctypes.data))
    return prow, pcol[:pn.value], pval[:pn.value], mptr, mdep[:mn.value], mcoef[:mn.value]


def read_mtx_dense(path: str):
    """A Matrix Market "array real" file (right-hand sides, HOST::ReadMtxTools::loadRightHand):
    returns an array of shape (cols, rows), one right-hand side per row."""
    lib = load()
    rows, cols = C.c_uint32(), C.c_uint32()
    bpath = os.fsencode(path)
    _check(lib.prism_mtx_read_dense(bpath, C.byref(rows), C.byref(cols), None))
    v = np.zeros(max(rows.value * cols.value, 1))
    _check(lib.prism_mtx_read_dense(bpath, C.byref(rows), C.byref(cols), v.ctypes.data))
    return v[:rows.value * cols.value].reshape(cols.value, rows.value)


def _ptr(t) -> int:
    """Device pointer of a torch CUDA tensor (float64, contiguous)."""
    import torch
    assert isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
    return t.data_ptr()


# =============================================================================
# CSR matrix (HOST::CSRMatrix<double>) and model problems
# =============================================================================
class CSRMatrix:
    """Host CSR with uint32 offsets/indices and double values, rows sorted."""

    def __init__(self, rowptr, col, val):
        self.rowptr = np.ascontiguousarray(rowptr, np.uint32)
        self.col = np.ascontiguousarray(col, np.uint32)
        self.val = np.ascontiguousarray(val, np.float64)

    @property
    def n(self) -> int:
        return len(self.rowptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def getRowNum(self) -> int:
        return self.n

    @classmethod
    def from_mtx(cls, path: str, base: int = 1, part: int = 0) -> "CSRMatrix":
        """A Matrix Market "coordinate" file (HOST::ReadMtxTools::loadMatrix,
        source/utils/TestTools/ReadMtxTools.cpp): symmetric files expanded, near-zero
        entries dropped, rows ordered by column; complex files: part 0 real, 1 imaginary.
        The matrix must be square to be solved."""
        lib = load()
        rows, cols, nnz = C.c_uint32(), C.c_uint32(), C.c_uint64()
        bpath = os.fsencode(path)
        _check(lib.prism_mtx_read(bpath, base, part, C.byref(rows), C.byref(cols), C.byref(nnz), None, None, None))
        rp = np.zeros(rows.value + 1, np.uint32)
        ci = np.zeros(max(nnz.value, 1), np.uint32)
        v = np.zeros(max(nnz.value, 1), np.float64)
        _check(lib.prism_mtx_read(bpath, base, part, C.byref(rows), C.byref(cols), C.byref(nnz), rp.ctypes.data,
                                  ci.ctypes.data, v.ctypes.data))
        m = cls(rp, ci[:nnz.value], v[:nnz.value])
        m.ncols = cols.value
        return m

    def write_mtx(self, path: str, symmetric: bool = False, comment: str = ""):
        """Writes the matrix as a Matrix Market "coordinate real" file (1-based; with
        symmetric=True only the lower triangle, as HOST::WriteMtxTools stores symmetric ones)."""
        rows = np.repeat(np.arange(self.n), np.diff(self.rowptr.astype(np.int64)))
        keep = rows >= self.col if symmetric else np.ones(len(rows), bool)
        with open(path, "w") as f:
            f.write(f"%%MatrixMarket matrix coordinate real {'symmetric' if symmetric else 'general'}\n")
            if comment:
                f.write(f"% {comment}\n")
            f.write(f"{self.n} {getattr(self, 'ncols', self.n)} {int(keep.sum())}\n")
            for r, c, v in zip(rows[keep], self.col[keep], self.val[keep]):
                f.write(f"{int(r) + 1} {int(c) + 1} {float(v)!r}\n")

    @classmethod
    def laplacian(cls, nx, ny, nz, alphax=0.0, alphay=0.0, alphaz=0.0, shift=0.0) -> "CSRMatrix":
        """generateLaplacianCSR (include/MatrixClass/ModelProblem.h:45-52)."""
        lib = load()
        n, nnz = C.c_uint32(), C.c_uint32()
        _check(lib.prism_laplacian_dims(nx, ny, nz, C.byref(n), C.byref(nnz)))
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        _check(lib.prism_laplacian_fill(nx, ny, nz, alphax, alphay, alphaz, shift, rp, ci, v))
        return cls(rp, ci, v)

    @classmethod
    def convection_diffusion(cls, nx, ny, nz, vx, vy, vz) -> "CSRMatrix":
        """Steady convection-diffusion -Laplace(u) + v . grad(u) on the unit cube,
        nx x ny x nz interior points (h = 1 / (n + 1) per axis, homogeneous
        Dirichlet boundaries), 7-point central differences for diffusion and
        first-order upwind differences for convection, scaled by h^2 per axis:
        along an axis with grid spacing h and velocity v, the upstream neighbour
        gets -(1 + h|v|), the downstream one -1, the diagonal 2 + h|v|.  A
        nonsymmetric M-matrix with the pattern (and the row ordering, x fastest)
        of generateLaplacianCSR(nx, ny, nz); the reference's generator offers
        central convection only (source/MatrixClass/ModelProblem.cpp:85-93)."""
        dims = (nx, ny, nz)
        vel = (float(vx), float(vy), float(vz))
        n = nx * ny * nz
        idx = np.arange(n, dtype=np.int64)
        coords = (idx % nx, (idx // nx) % ny, idx // (nx * ny))
        strides = (1, nx, nx * ny)
        rows, cols, vals = [idx], [idx], [np.zeros(n)]
        for d in range(3):
            if dims[d] == 1:
                continue
            h = 1.0 / (dims[d] + 1)
            c = abs(vel[d]) * h
            rows.append(idx)
            cols.append(idx)
            vals.append(np.full(n, 2.0 + c))
            for sgn in (-1, 1):
                ok = coords[d] + sgn >= 0 if sgn < 0 else coords[d] + sgn < dims[d]
                upstream = (sgn < 0) == (vel[d] > 0)   # neighbour the flow comes from
                w = -(1.0 + c) if upstream and vel[d] != 0.0 else -1.0
                rows.append(idx[ok])
                cols.append(idx[ok] + sgn * strides[d])
                vals.append(np.full(int(ok.sum()), w))
        r = np.concatenate(rows)
        cc = np.concatenate(cols)
        v = np.concatenate(vals)
        key = r * n + cc
        order = np.argsort(key, kind="stable")
        key, v = key[order], v[order]
        uk, start = np.unique(key, return_index=True)
        vsum = np.add.reduceat(v, start)
        rr, ccol = uk // n, uk % n
        rowptr = np.zeros(n + 1, np.int64)
        np.add.at(rowptr, rr + 1, 1)
        return cls(np.cumsum(rowptr).astype(np.uint32), ccol.astype(np.uint32), vsum)

    @classmethod
    def block_diagonal(cls, blocks) -> tuple:
        """One CSR holding the given systems on its diagonal; returns (matrix, seg_ptr)."""
        rps, cols, vals, seg = [np.zeros(1, np.int64)], [], [], [0]
        for B in blocks:
            rps.append(B.rowptr[1:].astype(np.int64) + rps[-1][-1])
            cols.append(B.col.astype(np.int64) + seg[-1])
            vals.append(B.val)
            seg.append(seg[-1] + B.n)
        return (cls(np.concatenate(rps).astype(np.uint32), np.concatenate(cols).astype(np.uint32),
                    np.concatenate(vals)), np.array(seg, np.uint32))

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.rowptr), shape=(self.n, self.n))


def generateLaplacianCSR(nx, ny, nz, alphax=0.0, alphay=0.0, alphaz=0.0, shift=0.0) -> CSRMatrix:
    return CSRMatrix.laplacian(nx, ny, nz, alphax, alphay, alphaz, shift)


# =============================================================================
# Host-only incomplete factorisation (no device needed)
# =============================================================================
class HostFactor:
    """prism_factor: an IC / ILUT / ILDLT factor built on the host, bit-exact
    with the reference's setup(), attachable to any DeviceSystem of the same size."""

    def __init__(self, A: CSRMatrix, kind: int, *, tol: float = 1e-3, lfill: int = 20, precision: int = PRISM_FP64):
        self.lib = load()
        self.kind = kind
        h = _vp()
        _check(self.lib.prism_factor_create(kind, A.n, A.rowptr, A.col, A.val, tol, lfill, precision, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.prism_factor_destroy(self.h)
            self.h = None

    def arrays(self, which: int = 0):
        n, nnz = C.c_uint32(), C.c_uint64()
        _check(self.lib.prism_factor_get(self.h, which, C.byref(n), C.byref(nnz), None, None, None, None))
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        d = np.zeros(n.value, np.float64)
        _check(self.lib.prism_factor_get(self.h, which, C.byref(n), C.byref(nnz), rp.ctypes.data, ci.ctypes.data,
                                         v.ctypes.data, d.ctypes.data))
        return rp, ci, v, d

    def info(self):
        m, lo, up = C.c_uint64(), C.c_uint32(), C.c_uint32()
        _check(self.lib.prism_factor_info(self.h, C.byref(m), C.byref(lo), C.byref(up)))
        return {"mnnz": m.value, "lower_levels": lo.value, "upper_levels": up.value}


def amsed_opts(**kw) -> AmsedOpts:
    o = AmsedOpts()
    load().prism_amsed_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class HostAmsed:
    """AMSED / MSLR setup built on the host (prism_factor_create_amsed): the HID
    permutation, level structure, block factors and low-rank terms; attachable
    to a DeviceSystem of the same size and exportable for parity checks."""

    def __init__(self, A: CSRMatrix, opts: AmsedOpts | None = None, precision: int = PRISM_FP64, **kw):
        self.lib = load()
        self.opts = opts if opts is not None else amsed_opts(**kw)
        h = _vp()
        _check(self.lib.prism_factor_create_amsed(A.n, A.rowptr, A.col, A.val, C.byref(self.opts), precision,
                                                  C.byref(h)))
        self.h = h
        self.n = A.n

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.prism_factor_destroy(self.h)
            self.h = None

    def info(self) -> dict:
        nlev, mnnz = C.c_uint32(), C.c_uint64()
        _check(self.lib.prism_amsed_info(self.h, C.byref(nlev), None, None, None, C.byref(mnnz)))
        L = nlev.value
        lev_ptr = np.zeros(L + 1, np.uint32)
        ncomps = np.zeros(L, np.uint32)
        ranks = np.zeros(L, np.uint32)
        _check(self.lib.prism_amsed_info(self.h, C.byref(nlev), lev_ptr.ctypes.data, ncomps.ctypes.data,
                                         ranks.ctypes.data, C.byref(mnnz)))
        return {"nlev": L, "lev_ptr": lev_ptr, "ncomps": ncomps, "ranks": ranks, "mnnz": mnnz.value}

    def perm(self):
        p = np.zeros(self.n, np.uint32)
        _check(self.lib.prism_amsed_perm(self.h, p.ctypes.data))
        return p

    def dom_ptr(self, level: int):
        nc = int(self.info()["ncomps"][level])
        d = np.zeros(nc + 1, np.uint32)
        _check(self.lib.prism_amsed_dom_ptr(self.h, level, d.ctypes.data))
        return d

    def block(self, level: int, block: int):
        n, nnz = C.c_uint32(), C.c_uint64()
        _check(self.lib.prism_amsed_block(self.h, level, block, C.byref(n), C.byref(nnz), None, None, None, None))
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        d = np.zeros(n.value, np.float64)
        _check(self.lib.prism_amsed_block(self.h, level, block, C.byref(n), C.byref(nnz), rp.ctypes.data,
                                          ci.ctypes.data, v.ctypes.data, d.ctypes.data))
        return rp, ci, v, d

    def coupling(self, level: int, which: int = 0):
        nr, nnz = C.c_uint32(), C.c_uint64()
        _check(self.lib.prism_amsed_coupling(self.h, level, which, C.byref(nr), C.byref(nnz), None, None, None))
        rp = np.zeros(nr.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        _check(self.lib.prism_amsed_coupling(self.h, level, which, C.byref(nr), C.byref(nnz), rp.ctypes.data,
                                             ci.ctypes.data, v.ctypes.data))
        return rp, ci, v

    def lowrank(self, level: int):
        r, nrem = C.c_uint32(), C.c_uint32()
        _check(self.lib.prism_amsed_lowrank(self.h, level, C.byref(r), C.byref(nrem), None, None))
        W = np.zeros(r.value * nrem.value, np.float64)
        H = np.zeros(r.value, np.float64)
        _check(self.lib.prism_amsed_lowrank(self.h, level, C.byref(r), C.byref(nrem), W.ctypes.data, H.ctypes.data))
        return W.reshape(r.value, nrem.value).T.copy() if r.value else W.reshape(nrem.value, 0), H


def gmslr_opts(**kw) -> AmsedOpts:
    o = AmsedOpts()
    load().prism_gmslr_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class HostGmslr(HostAmsed):
    """GMSLR setup built on the host (prism_factor_create_gmslr)."""

    is_gmslr = True

    def __init__(self, A: CSRMatrix, opts: AmsedOpts | None = None, precision: int = PRISM_FP64, **kw):
        self.lib = load()
        self.opts = opts if opts is not None else gmslr_opts(**kw)
        h = _vp()
        _check(self.lib.prism_factor_create_gmslr(A.n, A.rowptr, A.col, A.val, C.byref(self.opts), precision,
                                                  C.byref(h)))
        self.h = h
        self.n = A.n

    def gmslr_block(self, level: int, block: int, which: int):
        n, nnz = C.c_uint32(), C.c_uint64()
        _check(self.lib.prism_gmslr_block(self.h, level, block, which, C.byref(n), C.byref(nnz), None, None, None,
                                          None))
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        d = np.zeros(n.value, np.float64)
        _check(self.lib.prism_gmslr_block(self.h, level, block, which, C.byref(n), C.byref(nnz), rp.ctypes.data,
                                          ci.ctypes.data, v.ctypes.data, d.ctypes.data))
        return rp, ci, v, d


# =============================================================================
# Device operator: one C-ABI handle (A on the GPU + preconditioner + workspace)
# =============================================================================
class DeviceSystem:
    """A resident on one device, its preconditioner and Krylov workspace."""

    def __init__(self, A: CSRMatrix, device: int = 0):
        self.lib = load()
        self.A = A
        h = _vp()
        _check(self.lib.prism_create(A.n, A.rowptr, A.col, A.val, device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.prism_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n(self) -> int:
        return self.A.n

    @property
    def nnz(self) -> int:
        return int(self.A.rowptr[-1])

    def set_stream(self, stream_ptr: int):
        _check(self.lib.prism_set_stream(self.h, stream_ptr))

    # y = A x
    def spmv(self, x):
        if hasattr(x, "is_cuda"):
            import torch
            y = torch.empty_like(x)
            _check(self.lib.prism_spmv_device(self.h, _ptr(x), _ptr(y)))
            return y
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.n)
        _check(self.lib.prism_spmv(self.h, x, y))
        return y

    def spmv_shape(self) -> tuple:
        """(lanes per row, rows per pass) of the SpMV kernel the handle chose at creation."""
        g, u = C.c_int32(), C.c_int32()
        _check(self.lib.prism_spmv_shape(self.h, C.byref(g), C.byref(u)))
        return g.value, u.value

    def spmv_into(self, x, y):
        """y = A x on CUDA tensors (y preallocated; no allocation in the call)."""
        _check(self.lib.prism_spmv_device(self.h, _ptr(x), _ptr(y)))
        return y

    # ---- preconditioner -------------------------------------------------------
    def set_precond(self, kind: int, *, tol: float = 1e-3, lfill: int = 20, precision: int = PRISM_FP64):
        if kind == PRECOND_NONE:
            _check(self.lib.prism_set_precond_none(self.h))
        elif kind == PRECOND_IC:
            _check(self.lib.prism_set_precond_ic(self.h, tol, precision))
        elif kind == PRECOND_ILDLT:
            _check(self.lib.prism_set_precond_ildlt(self.h, tol, precision))
        elif kind == PRECOND_ILUT:
            _check(self.lib.prism_set_precond_ilut(self.h, lfill, tol, precision))
        else:
            raise PrismError(9, f"preconditioner kind {kind} not available")

    def set_amsed(self, opts: AmsedOpts | None = None, precision: int = PRISM_FP64, **kw):
        o = opts if opts is not None else amsed_opts(**kw)
        _check(self.lib.prism_set_precond_amsed(self.h, C.byref(o), precision))

    def attach(self, factor):
        _check(self.lib.prism_set_precond_factor(self.h, factor.h))

    def precond_nnz(self) -> int:
        v = C.c_uint64()
        _check(self.lib.prism_precond_nnz(self.h, C.byref(v)))
        return v.value

    def precond_levels(self, sweep: int) -> int:
        v = C.c_uint32()
        _check(self.lib.prism_precond_levels(self.h, sweep, C.byref(v)))
        return v.value

    def precond_factor(self, which: int = 0):
        """Stored factor arrays in the reference layout: (rowptr, col, val, diag)."""
        n, nnz = C.c_uint32(), C.c_uint64()
        _check(self.lib.prism_precond_factor(self.h, which, C.byref(n), C.byref(nnz), None, None, None, None))
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        d = np.zeros(n.value, np.float64)
        _check(self.lib.prism_precond_factor(self.h, which, C.byref(n), C.byref(nnz), rp.ctypes.data,
                                             ci.ctypes.data, v.ctypes.data, d.ctypes.data))
        return rp, ci, v, d

    def sweep_device(self, sweep: int, vin, vout, prepare: int = 1):
        """One triangular sweep alone on torch CUDA tensors (kernel timing).
        prepare: 1 mark pending + sweep, 0 sweep only, 2 mark pending only."""
        _check(self.lib.prism_precond_sweep_device(self.h, sweep, _ptr(vin), _ptr(vout), int(prepare)))

    def sweep_info(self, sweep: int) -> dict:
        n, nnz, vb, lv, kk = C.c_uint32(), C.c_uint64(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(self.lib.prism_precond_sweep_info(self.h, sweep, C.byref(n), C.byref(nnz), C.byref(vb), C.byref(lv),
                                                 C.byref(kk)))
        return {"n": n.value, "nnz": nnz.value, "value_bytes": vb.value, "levels": lv.value,
                "kernel": {1: "level-order", 2: "slab", 3: "stream"}.get(kk.value, "?")}

    def sweep_order(self, sweep: int) -> SweepOrder:
        """Summation order of one of the preconditioner's sweeps when it runs the streamed kernel
        (prism_precond_sweep_order); raises PrismError otherwise."""
        n, op, lower = C.c_uint32(), C.c_int32(), C.c_int32()
        _check(self.lib.prism_precond_sweep_order(self.h, sweep, C.byref(n), None, None, None, None, None, None,
                                                  None, None, None))
        lib, h = self.lib, self.h
        diag = np.zeros(max(n.value, 1))
        o = _fill_order(lambda ep, ed, ec, kp, kd, kc: lib.prism_precond_sweep_order(
            h, sweep, C.byref(n), ep, ed, ec, kp, kd, kc, diag.ctypes.data, C.byref(op), C.byref(lower)), n.value)
        o.diag, o.op, o.lower = diag[:n.value], op.value, bool(lower.value)
        # a paired sweep's right-hand side map (empty when the sweep runs unpaired)
        paired, mn = C.c_int32(), C.c_uint64()
        _check(lib.prism_precond_sweep_rhs_map(h, sweep, C.byref(paired), C.byref(mn), None, None, None))
        o.mptr = np.zeros(n.value + 1, np.uint32)
        o.mdep = np.zeros(max(mn.value, 1), np.uint32)
        o.mcoef = np.zeros(max(mn.value, 1))
        if paired.value:
            _check(lib.prism_precond_sweep_rhs_map(h, sweep, C.byref(paired), C.byref(mn), o.mptr.ctypes.data,
                                                   o.mdep.ctypes.data, o.mcoef.ctypes.data))
        o.mdep, o.mcoef = o.mdep[:mn.value], o.mcoef[:mn.value]
        o.paired = bool(paired.value)
        return o

    def apply(self, vec):
        """out = M^{-1} vec (MInvSolve(vecIN, vecOUT))."""
        if hasattr(vec, "is_cuda"):
            import torch
            out = torch.empty_like(vec)
            _check(self.lib.prism_apply_device(self.h, _ptr(vec), _ptr(out)))
            return out
        vec = np.ascontiguousarray(vec, np.float64)
        out = np.zeros(self.n)
        _check(self.lib.prism_apply(self.h, vec, out))
        return out

    # ---- solve ------------------------------------------------------------------
    def update_values(self, val):
        """New values of A on the same pattern (host array or CUDA tensor)."""
        if hasattr(val, "is_cuda"):
            _check(self.lib.prism_update_values_device(self.h, _ptr(val.contiguous())))
        else:
            _check(self.lib.prism_update_values(self.h, np.ascontiguousarray(val, np.float64)))

    def refactor(self):
        """IC / ILDLT: the factor recomputed on the device for A's current values, on its own
        pattern, in the host factorisation's operation order (prism_refactor)."""
        _check(self.lib.prism_refactor(self.h))

    def adjoint(self, g, x=None, *, solver=SOLVER_FCG, tol=1e-10, max_iter=1000, restart=0):
        """lambda = A^{-T} g and, with x given, dL/dA on A's pattern (-lambda_i x_j);
        returns (lambda, grad_val or None, SolveStats)."""
        opts = SolveOpts(solver, tol, max_iter, restart, None)
        st = SolveStats()
        if hasattr(g, "is_cuda"):
            import torch
            gc = g.contiguous()
            lam = torch.empty_like(gc)
            gv = None
            if x is not None:
                x = x.contiguous()
                gv = torch.empty(self.nnz, dtype=torch.float64, device=gc.device)
            _check(self.lib.prism_adjoint_solve_device(self.h, C.byref(opts), _ptr(gc),
                                                       _ptr(x) if x is not None else None, _ptr(lam),
                                                       _ptr(gv) if gv is not None else None, C.byref(st)))
            return lam, gv, st
        gh = np.ascontiguousarray(g, np.float64)
        lam = np.zeros(self.n)
        gv = np.zeros(self.nnz) if x is not None else None
        xh = np.ascontiguousarray(x, np.float64) if x is not None else np.zeros(self.n)
        _check(self.lib.prism_adjoint_solve(self.h, C.byref(opts), gh, xh, lam,
                                            gv.ctypes.data if gv is not None else None, C.byref(st)))
        return lam, gv, st

    def apply_batched(self, V):
        """M^{-1} applied to each row of V (shape (k, n), k <= 64): column-major blocks
        with leading dimension n, on the device (torch CUDA tensor) or the host."""
        if hasattr(V, "is_cuda"):
            import torch
            assert V.dim() == 2 and V.shape[1] == self.n
            Vc = V.contiguous()
            out = torch.empty_like(Vc)
            _check(self.lib.prism_apply_batched_device(self.h, Vc.shape[0], _ptr(Vc), _ptr(out), self.n))
            return out
        import torch
        return self.apply_batched(torch.from_numpy(np.ascontiguousarray(V, np.float64)).cuda()).cpu().numpy()

    def solve_batched(self, B, X=None, *, solver=SOLVER_FCG, tol=1e-8, max_iter=1000) -> tuple:
        """Solves A x_c = b_c for the k rows of B (shape (k, n), k <= 64) in one block
        solve; returns (X, [SolveStats] * k).  Device tensors or host arrays."""
        opts = SolveOpts(solver, tol, max_iter, 0, None)
        if hasattr(B, "is_cuda"):
            import torch
            Bc = B.contiguous()
            k = Bc.shape[0]
            Xc = torch.zeros_like(Bc) if X is None else X.contiguous()
            st = (SolveStats * k)()
            _check(self.lib.prism_solve_batched_device(self.h, C.byref(opts), k, _ptr(Bc), _ptr(Xc), self.n, st))
            return Xc, list(st)
        Bh = np.ascontiguousarray(B, np.float64)
        k = Bh.shape[0]
        Xh = np.zeros_like(Bh) if X is None else np.array(X, np.float64, copy=True)
        st = (SolveStats * k)()
        _check(self.lib.prism_solve_batched(self.h, C.byref(opts), k, Bh.reshape(-1), Xh.reshape(-1), self.n, st))
        return Xh, list(st)

    def solve_segments(self, seg_ptr, b, x=None, *, solver=SOLVER_FCG, tol=1e-8, max_iter=1000) -> tuple:
        """Solves the independent systems on the diagonal blocks [seg_ptr[s], seg_ptr[s+1])
        of A at once; returns (x, [SolveStats] per system).  Device tensors or host arrays."""
        sp = np.ascontiguousarray(seg_ptr, np.uint32)
        nseg = len(sp) - 1
        opts = SolveOpts(solver, tol, max_iter, 0, None)
        st = (SolveStats * nseg)()
        if hasattr(b, "is_cuda"):
            import torch
            bc = b.contiguous()
            xc = torch.zeros_like(bc) if x is None else x
            _check(self.lib.prism_solve_segments_device(self.h, C.byref(opts), nseg, sp, _ptr(bc), _ptr(xc), st))
            return xc, list(st)
        bh = np.ascontiguousarray(b, np.float64)
        xh = np.zeros(self.n) if x is None else np.array(x, np.float64, copy=True)
        _check(self.lib.prism_solve_segments(self.h, C.byref(opts), nseg, sp, bh, xh, st))
        return xh, list(st)

    def solve(self, b, x=None, *, solver=SOLVER_FCG, tol=1e-8, max_iter=1000, restart=0, x_ref=None,
              launch_mode=LAUNCH_AUTO) -> tuple:
        """x (in/out initial guess) solved in place; returns (x, SolveStats).  x_ref (same kind
        as b: a CUDA tensor or a host array): a reference solution whose forward error the
        stats then report (stats.forward_error, else -1).  launch_mode (GMRES solvers):
        LAUNCH_AUTO runs each restart cycle as one CUDA graph, LAUNCH_STREAM as plain
        launches with a host read after every Arnoldi step."""
        opts = SolveOpts(solver, tol, max_iter, restart, None, launch_mode)
        st = SolveStats()
        if hasattr(b, "is_cuda"):
            import torch
            if x is None:
                x = torch.zeros_like(b)
            if x_ref is not None:
                opts.x_ref = _ptr(x_ref)
            _check(self.lib.prism_solve_device(self.h, C.byref(opts), _ptr(b), _ptr(x), C.byref(st)))
            return x, st
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n) if x is None else np.array(x, np.float64, copy=True)
        if x_ref is not None:
            xr = np.ascontiguousarray(x_ref, np.float64)
            opts.x_ref = xr.ctypes.data
        _check(self.lib.prism_solve(self.h, C.byref(opts), b, x, C.byref(st)))
        return x, st


# =============================================================================
# Reference-named wrappers (BasePrecondition / BaseSolver mirror)
# =============================================================================
class _Triangular:
    kind = PRECOND_NONE

    def __init__(self, system: DeviceSystem, precision: int = PRISM_FP64):
        self.system = system
        self.precision = precision
        self._ready = False

    def isReady(self) -> bool:
        return self._ready

    def MInvSolve(self, vec):
        self.setup()
        return self.system.apply(vec)

    def getPreconditionNonZeroCount(self) -> int:
        self.setup()
        return self.system.precond_nnz()

    def getPreconditionFillinRatio(self) -> float:
        return self.getPreconditionNonZeroCount() / self.system.A.nnz


class IncompleteCholesky(_Triangular):
    """IncompleteCholesky<Low, double>(A, threshold) (IncompleteCholesky.cpp:11-33)."""
    kind = PRECOND_IC

    def __init__(self, system, threshold, precision=PRISM_FP64):
        super().__init__(system, precision)
        self.threshold = threshold

    def setup(self):
        if not self._ready:
            self.system.set_precond(PRECOND_IC, tol=self.threshold, precision=self.precision)
            self._ready = True


class IncompleteLDLT(_Triangular):
    """IncompleteLDLT<Low, double>(A, tol) (IncompleteLDLT.cpp)."""
    kind = PRECOND_ILDLT

    def __init__(self, system, tolerance, precision=PRISM_FP64):
        super().__init__(system, precision)
        self.tolerance = tolerance

    def setup(self):
        if not self._ready:
            self.system.set_precond(PRECOND_ILDLT, tol=self.tolerance, precision=self.precision)
            self._ready = True


class IncompleteLU(_Triangular):
    """IncompleteLU<Low, double>(A, lfill, tolerance) (IncompleteLU.cpp:12-35)."""
    kind = PRECOND_ILUT

    def __init__(self, system, lfill, tolerance, precision=PRISM_FP64):
        super().__init__(system, precision)
        self.lfill = lfill
        self.tolerance = tolerance

    def setup(self):
        if not self._ready:
            self.system.set_precond(PRECOND_ILUT, tol=self.tolerance, lfill=self.lfill, precision=self.precision)
            self._ready = True


class CG:
    """CG<double>(n, precond, CGType, tol, maxIter) (source/Solver/CG.cpp:11-31)."""

    def __init__(self, problemSize, precond=None, cgType=FlexibleCG, tol=1e-8, maxIter=1000):
        self.n = problemSize
        self.precond = precond
        self.cgType = cgType
        self.tol = tol
        self.maxIter = maxIter
        self.stats = None

    def solve(self, system: DeviceSystem, b, x):
        if self.precond is not None:
            self.precond.setup()
        else:
            system.set_precond(PRECOND_NONE)
        kind = SOLVER_FCG if self.cgType == FlexibleCG else SOLVER_CG
        x_out, self.stats = system.solve(b, x, solver=kind, tol=self.tol, max_iter=self.maxIter)
        return x_out

    def getNumIter(self):
        return self.stats.num_iter

    def getError(self):
        return self.stats.final_error

    def getConvergence(self):
        return bool(self.stats.converged)


class GMRES:
    """GMRES<double>(n, precond, tol, GMRESType) + setRestart (source/Solver/GMRES.cpp:11-70)."""

    def __init__(self, problemSize, precond=None, tolerance=1e-7, gmresType=FlexibleGMRES):
        self.n = problemSize
        self.precond = precond
        self.tol = tolerance
        self.gmresType = gmresType
        self.restart = 0
        self.stats = None

    def setRestart(self, restart: bool, m: int):
        self.restart = m if restart else 0

    def solve(self, system: DeviceSystem, b, x):
        if self.precond is not None:
            self.precond.setup()
        elif self.gmresType == FlexibleGMRES:
            raise PrismError(5, "FlexibleGMRES must use a preconditioner")
        else:
            system.set_precond(PRECOND_NONE)
        kind = SOLVER_FGMRES if self.gmresType == FlexibleGMRES else SOLVER_GMRES
        x_out, self.stats = system.solve(b, x, solver=kind, tol=self.tol, restart=self.restart)
        return x_out

    def getNumIter(self):
        return self.stats.num_iter

    def getError(self):
        return self.stats.final_error

    def getConvergence(self):
        return bool(self.stats.converged)


class AMSEDPrecondition:
    """AMSEDPrecondition<Low, double>(A, levelNum, lanczosSteps, lowRankSize, eigCorrectBound,
    localReorderType, lowRankType, lanczosType) (AMSEDPrecondition.cpp:60-79)."""

    def __init__(self, system: DeviceSystem, levelNum, lanczosSteps, lowRankSize, eigCorrectBound=0.8,
                 localReorderType=MatrixReorderRCM, lowRankType=AMSEDEigenvalueDeflation,
                 lanczosType=UseClassicLanczos, precision=PRISM_FP64, seed=20241116):
        self.system = system
        self.opts = amsed_opts(levels=levelNum, lanczos_steps=lanczosSteps, low_rank=lowRankSize,
                               eig_bound=eigCorrectBound, reorder=localReorderType, lowrank_type=lowRankType,
                               lanczos_type=lanczosType, seed=seed)
        self.precision = precision
        self.host = None

    def setup(self):
        if self.host is None:
            self.host = HostAmsed(self.system.A, self.opts, self.precision)
            self.system.attach(self.host)

    def MInvSolve(self, vec):
        self.setup()
        return self.system.apply(vec)

    def getPreconditionNonZeroCount(self):
        self.setup()
        return self.host.info()["mnnz"]


class GMSLRPrecondition:
    """GMSLRPrecondition<Low, double>(A, levelNum, lanczosSteps, lowRankSize, localReorderType)
    (GMSLRDPrecondition.cpp:41-55)."""

    def __init__(self, system: DeviceSystem, levelNum, lanczosSteps=20, lowRankSize=12,
                 localReorderType=MatrixReorderRCM, precision=PRISM_FP64):
        self.system = system
        self.opts = gmslr_opts(levels=levelNum, lanczos_steps=lanczosSteps, low_rank=lowRankSize,
                               reorder=localReorderType)
        self.precision = precision
        self.host = None

    def setup(self):
        if self.host is None:
            self.host = HostGmslr(self.system.A, self.opts, self.precision)
            self.system.attach(self.host)

    def MInvSolve(self, vec):
        self.setup()
        return self.system.apply(vec)

    def getPreconditionNonZeroCount(self):
        self.setup()
        return self.host.info()["mnnz"]
