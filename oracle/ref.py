"""ctypes view of the reference's own CPU classes, compiled from its sources.

Test infrastructure only: the parity tests, the golden-fixture generator and
the CPU-baseline arm of bench.py load this; the product never does.

``oracle/Makefile`` (target ``ref``) compiles PrisPack's CSRMatrix, COOMatrix,
ModelProblem, IncompleteCholesky, IncompleteLDLT, IncompleteLU, CG and GMRES
sources together with ``ref_shim/ref_capi.cpp`` into

* ``_ref/libprism_ref.so``       -- parity build (no fast-math, no FMA contraction)
* ``_ref/libprism_ref_fast.so``  -- the reference's Release flags (timing only)

Both are absent where the reference sources were never available; callers
check :func:`available` first.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[str, C.CDLL] = {}

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

KIND_IC, KIND_ILUT, KIND_ILDLT = 1, 2, 3


def lib_path(fast: bool = False) -> str:
    return os.path.join(_HERE, "_ref", "libprism_ref_fast.so" if fast else "libprism_ref.so")


def available(fast: bool = False) -> bool:
    return os.path.exists(lib_path(fast))


def load(fast: bool = False) -> C.CDLL:
    key = "fast" if fast else "parity"
    if key in _LIBS:
        return _LIBS[key]
    lib = C.CDLL(lib_path(fast))
    vp = C.c_void_p
    lib.ref_csr_laplacian.restype = vp
    lib.ref_csr_laplacian.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
    lib.ref_csr_poisson.restype = vp
    lib.ref_csr_poisson.argtypes = [C.c_uint]
    lib.ref_csr_from_arrays.restype = vp
    lib.ref_csr_from_arrays.argtypes = [C.c_uint, _u32p, _u32p, _f64p]
    lib.ref_csr_dims.argtypes = [vp, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    lib.ref_read_mtx.restype = vp
    lib.ref_read_mtx.argtypes = [C.c_char_p, C.c_int]
    lib.ref_csr_copy.argtypes = [vp, _u32p, _u32p, _f64p]
    lib.ref_csr_free.argtypes = [vp]
    lib.ref_spmv.argtypes = [vp, _f64p, _f64p]
    lib.ref_precond_create.restype = vp
    lib.ref_precond_create.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_int]
    lib.ref_precond_setup.argtypes = [vp]
    lib.ref_precond_free.argtypes = [vp]
    lib.ref_precond_mnnz.restype = C.c_uint
    lib.ref_precond_mnnz.argtypes = [vp]
    lib.ref_precond_factor_dims.argtypes = [vp, C.c_int, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    lib.ref_precond_factor_copy.argtypes = [vp, C.c_int, _u32p, _u32p, _f64p, C.c_void_p]
    lib.ref_precond_apply.argtypes = [vp, C.c_uint, _f64p]
    lib.ref_cg_solve.argtypes = [vp, vp, C.c_int, C.c_double, C.c_uint, _f64p, _f64p,
                                 C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.ref_gmres_solve.argtypes = [vp, vp, C.c_int, C.c_uint, C.c_double, _f64p, _f64p,
                                    C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.ref_omp_max_threads.restype = C.c_int
    lib.ref_set_seed.argtypes = [C.c_uint]
    lib.ref_amsed_create.restype = vp
    lib.ref_amsed_create.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.ref_amsed_info.argtypes = [vp, C.POINTER(C.c_uint), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_uint)]
    lib.ref_amsed_perm.argtypes = [vp, C.c_void_p]
    lib.ref_amsed_dom_ptr.argtypes = [vp, C.c_int, C.c_void_p]
    lib.ref_amsed_block.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ref_rcm.argtypes = [C.c_uint, _u32p, _u32p, _u32p]
    lib.ref_gmslr_create.restype = vp
    lib.ref_gmslr_create.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.ref_gmslr_info.argtypes = [vp, C.POINTER(C.c_uint), C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_uint), C.POINTER(C.c_double)]
    lib.ref_gmslr_perm.argtypes = [vp, C.c_void_p]
    lib.ref_gmslr_block.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint), C.POINTER(C.c_uint),
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ref_amsed_lowrank.argtypes = [vp, C.c_int, C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.c_void_p, C.c_void_p]
    _LIBS[key] = lib
    return lib


class RefCSR:
    """HOST::CSRMatrix<double> owned through the shim."""

    def __init__(self, handle: int, lib: C.CDLL):
        self.h = handle
        self.lib = lib

    @classmethod
    def laplacian(cls, nx, ny, nz, ax=0.0, ay=0.0, az=0.0, shift=0.0, fast=False):
        lib = load(fast)
        return cls(lib.ref_csr_laplacian(nx, ny, nz, ax, ay, az, shift), lib)

    @classmethod
    def from_mtx(cls, path, part=0, fast=False):
        """HOST::ReadMtxTools<double>::loadMatrix of a Matrix Market file (part 1: a complex
        file's imaginary part)."""
        lib = load(fast)
        return cls(lib.ref_read_mtx(os.fsencode(path), part), lib)

    @classmethod
    def from_arrays(cls, rowptr, col, val, fast=False):
        lib = load(fast)
        n = len(rowptr) - 1
        return cls(lib.ref_csr_from_arrays(n, np.ascontiguousarray(rowptr, np.uint32),
                                           np.ascontiguousarray(col, np.uint32),
                                           np.ascontiguousarray(val, np.float64)), lib)

    def dims(self):
        n, nnz = C.c_uint(), C.c_uint()
        self.lib.ref_csr_dims(self.h, C.byref(n), C.byref(nnz))
        return n.value, nnz.value

    def arrays(self):
        n, nnz = self.dims()
        rp = np.zeros(n + 1, np.uint32)
        ci = np.zeros(nnz, np.uint32)
        v = np.zeros(nnz, np.float64)
        self.lib.ref_csr_copy(self.h, rp, ci, v)
        return rp, ci, v

    def spmv(self, x):
        n, _ = self.dims()
        y = np.zeros(n, np.float64)
        self.lib.ref_spmv(self.h, np.ascontiguousarray(x, np.float64), y)
        return y

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_csr_free(self.h)
            self.h = None


class RefPrecond:
    """IncompleteCholesky / IncompleteLU / IncompleteLDLT<low, double> through the shim."""

    def __init__(self, A: RefCSR, kind: int, low_precision: bool, tol: float, lfill: int = 0):
        self.A = A
        self.lib = A.lib
        self.kind = kind
        self.h = self.lib.ref_precond_create(A.h, kind, int(low_precision), tol, lfill)
        if not self.h:
            raise ValueError("bad preconditioner kind")

    def setup(self) -> int:
        return self.lib.ref_precond_setup(self.h)

    def factor(self, which: int = 0):
        n, nnz = C.c_uint(), C.c_uint()
        self.lib.ref_precond_factor_dims(self.h, which, C.byref(n), C.byref(nnz))
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        d = np.zeros(n.value, np.float64)
        self.lib.ref_precond_factor_copy(self.h, which, rp, ci, v, d.ctypes.data_as(C.c_void_p))
        return rp, ci, v, d

    def apply(self, vec):
        out = np.array(vec, dtype=np.float64, copy=True)
        self.lib.ref_precond_apply(self.h, len(out), out)
        return out

    def mnnz(self) -> int:
        return self.lib.ref_precond_mnnz(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_precond_free(self.h)
            self.h = None


def cg_solve(A: RefCSR, P: RefPrecond | None, b, x0=None, tol=1e-8, maxit=1000, flexible=True):
    n, _ = A.dims()
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
    it, err, conv = C.c_int(), C.c_double(), C.c_int()
    A.lib.ref_cg_solve(A.h, P.h if P else None, int(flexible), tol, maxit,
                       np.ascontiguousarray(b, np.float64), x, C.byref(it), C.byref(err), C.byref(conv))
    return x, it.value, err.value, bool(conv.value)


def gmres_solve(A: RefCSR, P: RefPrecond | None, b, x0=None, tol=1e-8, restart=50, flexible=True):
    n, _ = A.dims()
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
    it, err, conv = C.c_int(), C.c_double(), C.c_int()
    A.lib.ref_gmres_solve(A.h, P.h if P else None, int(flexible), restart, tol,
                          np.ascontiguousarray(b, np.float64), x, C.byref(it), C.byref(err), C.byref(conv))
    return x, it.value, err.value, bool(conv.value)


KIND_AMSED = 5


class RefAmsed(RefPrecond):
    """AMSEDPrecondition<low, double>(A, levels, lanczosSteps, lowRankSize, eigCorrectBound,
    localReorderType, lowRankType, lanczosType) through the shim (METIS stand-in, seeded
    Lanczos start vector: base seed + call index, the product's convention)."""

    def __init__(self, A: RefCSR, levels, lanczos_steps, low_rank, eig_bound=0.8, reorder=2, lowrank_type=1,
                 lanczos_type=0, low_precision=False, seed=20241116):
        self.A = A
        self.lib = A.lib
        self.kind = KIND_AMSED
        self.seed = seed
        self.h = self.lib.ref_amsed_create(A.h, levels, lanczos_steps, low_rank, eig_bound, reorder, lowrank_type,
                                           lanczos_type, int(low_precision))

    def setup(self) -> int:
        self.lib.ref_set_seed(self.seed)
        return self.lib.ref_precond_setup(self.h)

    def info(self):
        nlev, mnnz = C.c_uint(), C.c_uint()
        self.lib.ref_amsed_info(self.h, C.byref(nlev), None, None, None, C.byref(mnnz))
        L = nlev.value
        lev_ptr = np.zeros(L + 1, np.uint32)
        ncomps = np.zeros(L, np.uint32)
        ranks = np.zeros(L, np.uint32)
        self.lib.ref_amsed_info(self.h, C.byref(nlev), lev_ptr.ctypes.data, ncomps.ctypes.data, ranks.ctypes.data,
                                C.byref(mnnz))
        return {"nlev": L, "lev_ptr": lev_ptr, "ncomps": ncomps, "ranks": ranks, "mnnz": mnnz.value}

    def perm(self):
        n, _ = self.A.dims()
        p = np.zeros(n, np.uint32)
        self.lib.ref_amsed_perm(self.h, p.ctypes.data)
        return p

    def dom_ptr(self, level):
        nc = int(self.info()["ncomps"][level])
        d = np.zeros(nc + 1, np.uint32)
        self.lib.ref_amsed_dom_ptr(self.h, level, d.ctypes.data)
        return d

    def block(self, level, block):
        n, nnz = C.c_uint(), C.c_uint()
        self.lib.ref_amsed_block(self.h, level, block, C.byref(n), C.byref(nnz), None, None, None, None)
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value, np.float64)
        d = np.zeros(n.value, np.float64)
        self.lib.ref_amsed_block(self.h, level, block, C.byref(n), C.byref(nnz), rp.ctypes.data, ci.ctypes.data,
                                 v.ctypes.data, d.ctypes.data)
        return rp, ci, v, d

    def lowrank(self, level):
        r, nrem = C.c_uint(), C.c_uint()
        self.lib.ref_amsed_lowrank(self.h, level, C.byref(r), C.byref(nrem), None, None)
        W = np.zeros(r.value * nrem.value)
        H = np.zeros(r.value)
        self.lib.ref_amsed_lowrank(self.h, level, C.byref(r), C.byref(nrem), W.ctypes.data, H.ctypes.data)
        return W.reshape(r.value, nrem.value).T.copy(), H


def rcm(rowptr, col):
    """rcmReorderCSR: perm[new] = old (vendored genrcm)."""
    n = len(rowptr) - 1
    p = np.zeros(n, np.uint32)
    load().ref_rcm(n, np.ascontiguousarray(rowptr, np.uint32), np.ascontiguousarray(col, np.uint32), p)
    return p


KIND_GMSLR = 4


class RefGmslr(RefPrecond):
    """GMSLRPrecondition<low, double>(A, levelNum, lanczosSteps, lowRankSize, localReorderType)."""

    def __init__(self, A: RefCSR, levels, lanczos_steps=20, low_rank=12, reorder=2, low_precision=False):
        self.A = A
        self.lib = A.lib
        self.kind = KIND_GMSLR
        self.h = self.lib.ref_gmslr_create(A.h, levels, lanczos_steps, low_rank, reorder, int(low_precision))

    def info(self):
        nlev, mnnz, wmax = C.c_uint(), C.c_uint(), C.c_double()
        self.lib.ref_gmslr_info(self.h, C.byref(nlev), None, None, None, C.byref(mnnz), C.byref(wmax))
        L = nlev.value
        lev_ptr = np.zeros(L + 1, np.uint32)
        ncomps = np.zeros(L, np.uint32)
        ranks = np.zeros(L, np.uint32)
        self.lib.ref_gmslr_info(self.h, C.byref(nlev), lev_ptr.ctypes.data, ncomps.ctypes.data, ranks.ctypes.data,
                                C.byref(mnnz), C.byref(wmax))
        return {"nlev": L, "lev_ptr": lev_ptr, "ncomps": ncomps, "ranks": ranks, "mnnz": mnnz.value,
                "w_max_abs": wmax.value}

    def perm(self):
        n, _ = self.A.dims()
        p = np.zeros(n, np.uint32)
        self.lib.ref_gmslr_perm(self.h, p.ctypes.data)
        return p

    def block(self, level, block, which):
        n, nnz = C.c_uint(), C.c_uint()
        self.lib.ref_gmslr_block(self.h, level, block, which, C.byref(n), C.byref(nnz), None, None, None, None)
        rp = np.zeros(n.value + 1, np.uint32)
        ci = np.zeros(nnz.value, np.uint32)
        v = np.zeros(nnz.value)
        d = np.zeros(n.value)
        self.lib.ref_gmslr_block(self.h, level, block, which, C.byref(n), C.byref(nnz), rp.ctypes.data,
                                 ci.ctypes.data, v.ctypes.data, d.ctypes.data)
        return rp, ci, v, d
