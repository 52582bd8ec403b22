"""ctypes binding of the C oracle (oracle.c) -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
bench.py as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


class _AmsedLevel(C.Structure):
    _fields_ = [("ncomps", C.c_uint32), ("dom_ptr", C.c_void_p),
                ("blk_rp", C.c_void_p), ("blk_ci", C.c_void_p), ("blk_val", C.c_void_p), ("blk_diag", C.c_void_p),
                ("e_rp", C.c_void_p), ("e_ci", C.c_void_p), ("e_val", C.c_void_p),
                ("rank", C.c_uint32), ("W", C.c_void_p), ("H", C.c_void_p),
                ("blk_rp1", C.c_void_p), ("blk_ci1", C.c_void_p), ("blk_val1", C.c_void_p),
                ("f_rp", C.c_void_p), ("f_ci", C.c_void_p), ("f_val", C.c_void_p),
                ("sweep_lo", C.c_void_p), ("sweep_up", C.c_void_p)]


class _SweepOrder(C.Structure):
    _fields_ = [("n", C.c_uint32), ("op", C.c_int), ("lower", C.c_int),
                ("eptr", C.c_void_p), ("edep", C.c_void_p), ("ecoef", C.c_void_p),
                ("kptr", C.c_void_p), ("kdep", C.c_void_p), ("kcoef", C.c_void_p), ("diag", C.c_void_p),
                ("mptr", C.c_void_p), ("mdep", C.c_void_p), ("mcoef", C.c_void_p)]


class _Amsed(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nlev", C.c_uint32), ("gmslr", C.c_int), ("single", C.c_int),
                ("pperm", C.c_void_p), ("lev_ptr", C.c_void_p), ("levels", C.c_void_p)]


class _Precond(C.Structure):
    _fields_ = [("kind", C.c_int), ("n", C.c_uint32),
                ("rp0", C.c_void_p), ("ci0", C.c_void_p), ("v0", C.c_void_p),
                ("rp1", C.c_void_p), ("ci1", C.c_void_p), ("v1", C.c_void_p),
                ("diag", C.c_void_p), ("amsed", C.c_void_p)]


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = [os.path.join(_HERE, f) for f in ("oracle.c", "oracle.h")]
    if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in src):
        subprocess.run(["/usr/bin/gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-shared",
                        "-o", path, os.path.join(_HERE, "oracle.c"), "-lm"], check=True)
    return path


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        _LIB.orc_laplacian.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, _u32p, _u32p, _f64p]
        _LIB.orc_spmv.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, _f64p, _f64p]
        _LIB.orc_sweep_f32.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, C.c_void_p, C.c_int, C.c_int, _f64p, _f64p]
        _LIB.orc_pair_rhs.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, _f64p, _f64p]
        _LIB.orc_sweep_ordered.argtypes = [C.c_uint32, C.c_int, C.c_int, C.c_int, _u32p, _u32p, _f64p, _u32p, _u32p,
                                           _f64p, C.c_void_p, _f64p, _f64p]
        _LIB.orc_precond_apply.argtypes = [C.POINTER(_Precond), _f64p]
        _LIB.orc_refactor.argtypes = [C.c_uint32, C.c_int, _u32p, _u32p, _f64p, _u32p, _u32p, C.c_int, _f64p, _f64p]
        _LIB.orc_refactor.restype = C.c_int
        _LIB.orc_amsed_apply.argtypes = [C.POINTER(_Amsed), _f64p]
        _LIB.orc_cg.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, C.POINTER(_Precond), C.c_int, C.c_double,
                                C.c_uint32, _f64p, _f64p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                C.POINTER(C.c_int32)]
        _LIB.orc_gmres.argtypes = [C.c_uint32, _u32p, _u32p, _f64p, C.POINTER(_Precond), C.c_int, C.c_uint32,
                                   C.c_double, _f64p, _f64p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                   C.POINTER(C.c_int32)]
    return _LIB


def laplacian(nx, ny, nz, ax=0.0, ay=0.0, az=0.0, shift=0.0):
    n = nx * ny * nz
    cap = 7 * n
    rp = np.zeros(n + 1, np.uint32)
    ci = np.zeros(cap, np.uint32)
    v = np.zeros(cap, np.float64)
    lib().orc_laplacian(nx, ny, nz, ax, ay, az, shift, rp, ci, v)
    nnz = int(rp[-1])
    return rp, ci[:nnz].copy(), v[:nnz].copy()


def spmv(rp, ci, v, x):
    y = np.zeros(len(rp) - 1)
    lib().orc_spmv(len(rp) - 1, rp, ci, v, np.ascontiguousarray(x, np.float64), y)
    return y


def sweep_f32(rp, ci, v, b, *, diag=None, op=2, lower=True):
    """Gather-form triangular sweep in single precision in the reference's order
    (each row summed in stored order); returns the float results widened to double."""
    rp = np.ascontiguousarray(rp, np.uint32)
    out = np.zeros(len(rp) - 1)
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    lib().orc_sweep_f32(len(rp) - 1, rp, np.ascontiguousarray(ci, np.uint32), np.ascontiguousarray(v, np.float64),
                        d.ctypes.data if d is not None else None, int(op), int(bool(lower)),
                        np.ascontiguousarray(b, np.float64), out)
    return out


def refactor(kind, A_rowptr, A_col, A_val, lt_rowptr, lt_col, *, single=False):
    """IC (kind 1) / ILDLT (kind 3) factor values on the pattern (lt_rowptr, lt_col) for the
    matrix values A_val: returns (status, lt_val, D)."""
    n = len(A_rowptr) - 1
    lt_val = np.zeros(max(len(lt_col), 1))
    D = np.zeros(max(n, 1))
    rc = lib().orc_refactor(n, int(kind), np.ascontiguousarray(A_rowptr, np.uint32),
                            np.ascontiguousarray(A_col, np.uint32), np.ascontiguousarray(A_val, np.float64),
                            np.ascontiguousarray(lt_rowptr, np.uint32),
                            np.ascontiguousarray(lt_col if len(lt_col) else np.zeros(1), np.uint32),
                            int(bool(single)), lt_val, D)
    return rc, lt_val[:len(lt_col)], D[:n]


def pair_rhs(mptr, mdep, mcoef, b):
    """A paired sweep's right-hand side: b_r - sum m b_dep in stored order, one fma each."""
    n = len(mptr) - 1
    out = np.zeros(n)
    u = lambda a: np.ascontiguousarray(a if len(a) else np.zeros(1), np.uint32)
    f = lambda a: np.ascontiguousarray(a if len(a) else np.zeros(1), np.float64)
    lib().orc_pair_rhs(n, u(mptr), u(mdep), f(mcoef), np.ascontiguousarray(b, np.float64), out)
    return out


def sweep_ordered(order, b, *, diag=None, op=2, lower=True, single=True):
    """Gather-form triangular sweep in the streamed kernel's summation order.  `order`
    carries eptr/edep/ecoef and kptr/kdep/kcoef (per row: early then late positions,
    padding 0xFFFFFFFF); float arithmetic when single, else double.  An order of a paired
    sweep (paired true, with mptr/mdep/mcoef) maps the right-hand side first (pair_rhs)."""
    n = len(order.eptr) - 1
    if getattr(order, "paired", False):
        b = pair_rhs(order.mptr, order.mdep, order.mcoef, b)
    out = np.zeros(n)
    d = np.ascontiguousarray(diag, np.float64) if diag is not None else None
    u = lambda a: np.ascontiguousarray(a if len(a) else np.zeros(1), np.uint32)
    f = lambda a: np.ascontiguousarray(a if len(a) else np.zeros(1), np.float64)
    lib().orc_sweep_ordered(n, int(bool(single)), int(op), int(bool(lower)), u(order.eptr), u(order.edep),
                            f(order.ecoef), u(order.kptr), u(order.kdep), f(order.kcoef),
                            d.ctypes.data if d is not None else None, np.ascontiguousarray(b, np.float64), out)
    return out


class Precond:
    """Factor arrays in the reference's stored layout (kind 1 IC, 2 ILUT, 3 ILDLT)."""

    def __init__(self, kind, n, f0=None, f1=None, diag=None):
        self.keep = []
        s = _Precond()
        s.kind = kind
        s.n = n

        def ptr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            self.keep.append(a)
            return a.ctypes.data

        if f0 is not None:
            s.rp0, s.ci0, s.v0 = ptr(f0[0], np.uint32), ptr(f0[1], np.uint32), ptr(f0[2], np.float64)
        if f1 is not None:
            s.rp1, s.ci1, s.v1 = ptr(f1[0], np.uint32), ptr(f1[1], np.uint32), ptr(f1[2], np.float64)
        s.diag = ptr(diag, np.float64)
        self.s = s

    def apply(self, vec):
        out = np.array(vec, np.float64, copy=True)
        lib().orc_precond_apply(C.byref(self.s), out)
        return out


def cg(rp, ci, v, b, P=None, x0=None, tol=1e-8, maxit=1000, flexible=True):
    n = len(rp) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
    it, err, conv = C.c_int32(), C.c_double(), C.c_int32()
    lib().orc_cg(n, rp, ci, v, C.byref(P.s) if P else None, int(flexible), tol, maxit,
                 np.ascontiguousarray(b, np.float64), x, C.byref(it), C.byref(err), C.byref(conv))
    return x, it.value, err.value, bool(conv.value)


def gmres(rp, ci, v, b, P=None, x0=None, tol=1e-8, restart=50, flexible=True):
    n = len(rp) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64, copy=True)
    it, err, conv = C.c_int32(), C.c_double(), C.c_int32()
    lib().orc_gmres(n, rp, ci, v, C.byref(P.s) if P else None, int(flexible), restart, tol,
                    np.ascontiguousarray(b, np.float64), x, C.byref(it), C.byref(err), C.byref(conv))
    return x, it.value, err.value, bool(conv.value)


class Amsed:
    """An AMSED/MSLR (or GMSLR) hierarchy for the oracle, from any exporter
    with the HostAmsed interface (info/perm/dom_ptr/block/coupling/lowrank;
    GMSLR: gmslr_block)."""

    def __init__(self, src):
        gmslr = bool(getattr(src, "is_gmslr", False))
        self.keep = []
        inf = src.info()
        nlev = inf["nlev"]
        n = int(inf["lev_ptr"][-1])

        def arr(a, dt):
            a = np.ascontiguousarray(a, dt)
            self.keep.append(a)
            return a.ctypes.data

        def ptrs(lst):
            a = (C.c_void_p * max(len(lst), 1))(*lst)
            self.keep.append(a)
            return C.cast(a, C.c_void_p).value

        levels = (_AmsedLevel * nlev)()
        for l in range(nlev):
            L = levels[l]
            dom = src.dom_ptr(l)
            L.ncomps = len(dom) - 1
            L.dom_ptr = arr(dom, np.uint32)
            nblk = 1 if l == nlev - 1 else L.ncomps
            rps, cis, vals, diags, rps1, cis1, vals1 = [], [], [], [], [], [], []
            for b in range(nblk):
                if gmslr:
                    rp, ci, v, d = src.gmslr_block(l, b, 0)
                    rp1, ci1, v1, _ = src.gmslr_block(l, b, 1)
                    rps1.append(arr(rp1, np.uint32)); cis1.append(arr(ci1, np.uint32)); vals1.append(arr(v1, np.float64))
                else:
                    rp, ci, v, d = src.block(l, b)
                rps.append(arr(rp, np.uint32)); cis.append(arr(ci, np.uint32))
                vals.append(arr(v, np.float64)); diags.append(arr(d, np.float64))
            L.blk_rp, L.blk_ci, L.blk_val, L.blk_diag = ptrs(rps), ptrs(cis), ptrs(vals), ptrs(diags)
            if gmslr:
                L.blk_rp1, L.blk_ci1, L.blk_val1 = ptrs(rps1), ptrs(cis1), ptrs(vals1)
            if l < nlev - 1:
                erp, eci, ev = src.coupling(l, 0)
                L.e_rp, L.e_ci, L.e_val = arr(erp, np.uint32), arr(eci, np.uint32), arr(ev, np.float64)
                if gmslr:
                    frp, fci, fv = src.coupling(l, 2)
                    L.f_rp, L.f_ci, L.f_val = arr(frp, np.uint32), arr(fci, np.uint32), arr(fv, np.float64)
                    continue
                W, H = src.lowrank(l)
                L.rank = len(H)
                if L.rank:
                    L.W = arr(np.asfortranarray(W).ravel(order="F"), np.float64)
                    L.H = arr(H, np.float64)
        self.levels = levels
        s = _Amsed()
        s.n, s.nlev = n, nlev
        s.gmslr = int(gmslr)
        s.pperm = arr(src.perm(), np.uint32)
        s.lev_ptr = arr(inf["lev_ptr"], np.uint32)
        s.levels = C.cast(levels, C.c_void_p).value
        self.s = s
        self.n = n

    def apply(self, vec):
        out = np.array(vec, np.float64, copy=True)
        lib().orc_amsed_apply(C.byref(self.s), out)
        return out

    def use_sweep_orders(self, orders, single=True):
        """Block solves as kernel-order sweeps: orders[2 l] / orders[2 l + 1] are level l's lower
        and upper sweeps (objects with eptr/edep/ecoef/kptr/kdep/kcoef/diag/op/lower, such as a
        device system's sweep_order()); `single` selects float arithmetic."""
        def arr(a, dt):
            a = np.ascontiguousarray(a if len(a) else np.zeros(1), dt)
            self.keep.append(a)
            return a.ctypes.data

        for l in range(self.s.nlev):
            for which, o in (("sweep_lo", orders[2 * l]), ("sweep_up", orders[2 * l + 1])):
                so = _SweepOrder()
                so.n, so.op, so.lower = len(o.eptr) - 1, int(o.op), int(bool(o.lower))
                so.eptr, so.edep, so.ecoef = arr(o.eptr, np.uint32), arr(o.edep, np.uint32), arr(o.ecoef, np.float64)
                so.kptr, so.kdep, so.kcoef = arr(o.kptr, np.uint32), arr(o.kdep, np.uint32), arr(o.kcoef, np.float64)
                so.diag = arr(o.diag, np.float64)
                if getattr(o, "paired", False):
                    so.mptr, so.mdep, so.mcoef = arr(o.mptr, np.uint32), arr(o.mdep, np.uint32), arr(o.mcoef, np.float64)
                self.keep.append(so)
                setattr(self.levels[l], which, C.cast(C.pointer(so), C.c_void_p).value)
        self.s.single = int(bool(single))

    def precond(self) -> "Precond":
        P = Precond(5, self.n)
        P.s.amsed = C.cast(C.pointer(self.s), C.c_void_p).value
        P.keep.append(self)
        return P
