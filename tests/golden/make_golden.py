"""Generates the golden fixtures in this directory from the reference itself.

Runs the reference's own CPU classes (compiled from its sources by
``oracle/Makefile`` target ``ref`` into ``oracle/_ref/libprism_ref.so``, the
parity build) on seeded model problems and stores their outputs:

* CSR arrays of generateLaplacianCSR,
* stored factor arrays of IncompleteCholesky / IncompleteLDLT / IncompleteLU
  (both <double,double> and <float,double>), full arrays for small cases and
  SHA-256 digests for the 64x64 case,
* MInvSolve outputs on a seeded vector,
* CG (FlexibleCG, NormalCG) and GMRES (FlexibleGMRES with restart) results:
  iteration count, reported error, convergence flag and solution.

* Matrix Market files read by HOST::ReadMtxTools (section ``mtx``): small
  files written here (mtx/*.mtx: general with explicit zeros, comments,
  duplicates and unsorted entries, symmetric, skew-symmetric, complex,
  hermitian, rectangular, a right-hand-side array) and the CSR arrays the
  reference's reader makes of them (mtx_cases.npz).

* AMSED / MSLR and GMSLR hierarchies (permutation, level pointers, block
  factor digests, low-rank spectra), their MInvSolve on a seeded vector and a
  preconditioned FCG / FGMRES solve.

Usage (needs the reference sources, i.e. only where oracle/_ref was built):
    make -C oracle ref && python tests/golden/make_golden.py [basic] [amsed] [gmslr]
(no argument regenerates every section; a named section updates only its own
files and manifest entries).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import ref  # noqa: E402

# (name, (nx, ny, nz, alphax, alphay, alphaz, shift), symmetric, full arrays?)
CASES = [
    ("lap2d_8", (8, 8, 1, 0.0, 0.0, 0.0, 0.0), True, True),
    ("lap3d_6", (6, 6, 6, 0.0, 0.0, 0.0, 0.0), True, True),
    ("conv2d_16", (16, 16, 1, 0.3, -0.2, 0.0, 0.0), False, True),
    ("lap2d_64", (64, 64, 1, 0.0, 0.0, 0.0, 0.0), True, False),
]
SEED = 20241116
AMSED_SEED = 20241116
# (name, grid, levels, lanczos steps, low rank, lowrank type (0 MSLR, 1 deflation), FP32 factors,
#  Lanczos type (0 classic, 1 restarted Krylov-Schur))
AMSED_CASES = [
    ("amsed_12c_mslr", (12, 12, 12), 3, 30, 16, 0, False, 0),
    ("amsed_16c_defl32", (16, 16, 16), 3, 40, 20, 1, True, 0),
    ("amsed_40sq_l4", (40, 40, 1), 4, 30, 16, 0, False, 0),
    ("amsed_14x11x9_restart", (14, 11, 9), 3, 30, 16, 0, False, 1),
    ("amsed_20c_defl_restart32", (20, 20, 20), 3, 30, 16, 1, True, 1),
]
# (name, grid with convection, levels, lanczos steps, low rank, FP32 factors)
GMSLR_CASES = [
    ("gmslr_16c_conv", (16, 16, 16, 0.3, 0.1, 0.0, 0.0), 3, 20, 12, False),
    ("gmslr_40sq_conv32", (40, 40, 1, 0.2, -0.3, 0.0, 0.0), 4, 20, 12, True),
    ("gmslr_12c_lap", (12, 12, 12, 0.0, 0.0, 0.0, 0.0), 2, 20, 12, False),
]


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def rhs(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


def main(sections):
    if not ref.available():
        raise SystemExit("oracle/_ref/libprism_ref.so not built: run `make -C oracle ref` where the reference exists")
    path = os.path.join(HERE, "manifest.json")
    manifest = {}
    if os.path.exists(path) and set(sections) != {"basic", "amsed", "gmslr", "mtx"}:
        with open(path) as f:
            manifest = json.load(f)
    if "basic" in sections:
        basic(manifest)
    if "amsed" in sections:
        amsed_section(manifest)
    if "gmslr" in sections:
        gmslr_section(manifest)
    if "mtx" in sections:
        mtx_section(manifest)
    manifest["_seed"] = SEED
    manifest["_generator"] = "tests/golden/make_golden.py via oracle/_ref/libprism_ref.so (reference sources, parity flags)"
    with open(path, "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("wrote", ", ".join(sections))


def basic(manifest):
    for name, grid, sym, full in CASES:
        A = ref.RefCSR.laplacian(*grid)
        rp, ci, v = A.arrays()
        n = len(rp) - 1
        b = rhs(n, SEED)
        probe = rhs(n, SEED + 1)
        out = {"rowptr": rp, "col": ci, "val": v, "b": b, "probe": probe}
        meta = {"grid": grid, "n": n, "nnz": int(rp[-1]), "A_sha": digest(rp, ci, v), "precond": {}}
        precs = []
        if sym:
            precs += [("ic_1e-3", ref.KIND_IC, 1e-3, 0), ("ic_1e-2", ref.KIND_IC, 1e-2, 0),
                      ("ic_0", ref.KIND_IC, 0.0, 0), ("ildlt_1e-3", ref.KIND_ILDLT, 1e-3, 0)]
        precs += [("ilut_20_1e-2", ref.KIND_ILUT, 1e-2, 20), ("ilut_5_1e-3", ref.KIND_ILUT, 1e-3, 5)]
        for pname, kind, tol, lfill in precs:
            for low in (False, True):
                key = f"{pname}_{'fp32' if low else 'fp64'}"
                P = ref.RefPrecond(A, kind, low, tol, lfill)
                rc = P.setup()
                if rc != 0:
                    meta["precond"][key] = {"setup_rc": rc}
                    continue
                f0 = P.factor(0)
                entry = {"setup_rc": 0, "mnnz": P.mnnz(), "kind": kind, "tol": tol, "lfill": lfill,
                         "f0_sha": digest(f0[0], f0[1], f0[2]), "nnz0": int(f0[0][-1])}
                if kind == ref.KIND_ILDLT:
                    entry["diag_sha"] = digest(f0[3])
                if kind == ref.KIND_ILUT:
                    f1 = P.factor(1)
                    entry["f1_sha"] = digest(f1[0], f1[1], f1[2])
                    entry["diag_sha"] = digest(f1[3])
                    entry["nnz1"] = int(f1[0][-1])
                if full:
                    out[f"{key}.f0_rowptr"], out[f"{key}.f0_col"], out[f"{key}.f0_val"] = f0[0], f0[1], f0[2]
                    if kind == ref.KIND_ILDLT:
                        out[f"{key}.diag"] = f0[3]
                    if kind == ref.KIND_ILUT:
                        out[f"{key}.f1_rowptr"], out[f"{key}.f1_col"], out[f"{key}.f1_val"] = f1[0], f1[1], f1[2]
                        out[f"{key}.diag"] = f1[3]
                out[f"{key}.apply"] = P.apply(probe)
                # solvers
                if sym and kind in (ref.KIND_IC, ref.KIND_ILDLT):
                    for flex in (True, False):
                        x, it, err, conv = ref.cg_solve(A, P, b, tol=1e-8, maxit=1000, flexible=flex)
                        tag = f"{key}.cg_{'flex' if flex else 'normal'}"
                        out[f"{tag}.x"] = x
                        entry[tag] = {"iters": it, "err": err, "conv": conv}
                x, it, err, conv = ref.gmres_solve(A, P, b, tol=1e-8, restart=20, flexible=True)
                out[f"{key}.fgmres20.x"] = x
                entry[f"{key}.fgmres20"] = {"iters": it, "err": err, "conv": conv}
                meta["precond"][key] = entry
        # unpreconditioned solvers
        if sym:
            x, it, err, conv = ref.cg_solve(A, None, b, tol=1e-8, maxit=1000, flexible=True)
            out["none.cg.x"] = x
            meta["none.cg"] = {"iters": it, "err": err, "conv": conv}
        x, it, err, conv = ref.gmres_solve(A, None, b, tol=1e-8, restart=30, flexible=False)
        out["none.gmres30.x"] = x
        meta["none.gmres30"] = {"iters": it, "err": err, "conv": conv}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        manifest[name] = meta


def amsed_section(manifest):
    """AMSED / MSLR (reference AMSEDPrecondition behind the METIS stand-in)."""
    amsed = {}
    for name, grid, levels, steps, rank, ltype, low, lanczos in AMSED_CASES:
        A = ref.RefCSR.laplacian(*grid)
        rp, ci, v = A.arrays()
        n = len(rp) - 1
        R = ref.RefAmsed(A, levels, steps, rank, 0.8, 2, ltype, lanczos, low, seed=AMSED_SEED)
        assert R.setup() == 0
        inf = R.info()
        entry = {"grid": grid, "levels": levels, "lanczos_steps": steps, "low_rank": rank, "lowrank_type": ltype,
                 "lanczos_type": lanczos, "fp32": low, "seed": AMSED_SEED, "nlev": inf["nlev"], "lev_ptr": inf["lev_ptr"].tolist(),
                 "ncomps": inf["ncomps"].tolist(), "ranks": inf["ranks"].tolist(), "mnnz": inf["mnnz"],
                 "perm_sha": digest(R.perm()), "blocks": {}}
        for lv in range(inf["nlev"]):
            entry["blocks"][str(lv)] = {"dom_ptr": R.dom_ptr(lv).tolist()}
            nb = 1 if lv == inf["nlev"] - 1 else int(inf["ncomps"][lv])
            entry["blocks"][str(lv)]["sha"] = [digest(*R.block(lv, b)[:3]) +
                                               ("" if lv == inf["nlev"] - 1 else digest(R.block(lv, b)[3]))
                                               for b in range(nb)]
            if lv < inf["nlev"] - 1 and inf["ranks"][lv] > 0:
                W, H = R.lowrank(lv)
                entry["blocks"][str(lv)]["H"] = sorted(H.tolist())
        probe = rhs(n, SEED + 1)
        b = rhs(n, SEED)
        out = {"probe": probe, "b": b, "apply": R.apply(probe)}
        x, it, err, conv = ref.cg_solve(A, R, b, tol=1e-10, maxit=500, flexible=True)
        out["cg.x"] = x
        entry["cg"] = {"iters": it, "err": err, "conv": conv}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        amsed[name] = entry
    manifest["_amsed"] = amsed


def gmslr_section(manifest):
    """GMSLR (reference GMSLRPrecondition behind the METIS stand-in): ILUT blocks,
    F coupling; its low-rank W is identically zero (dhseqr with COMPZ='V' on a
    zero Z), which the entry records as w_max_abs."""
    gm = {}
    for name, grid, levels, steps, rank, low in GMSLR_CASES:
        A = ref.RefCSR.laplacian(*grid)
        n = A.dims()[0]
        R = ref.RefGmslr(A, levels, steps, rank, 2, low)
        assert R.setup() == 0
        inf = R.info()
        entry = {"grid": grid, "levels": levels, "lanczos_steps": steps, "low_rank": rank, "fp32": low,
                 "nlev": inf["nlev"], "lev_ptr": inf["lev_ptr"].tolist(), "ncomps": inf["ncomps"].tolist(),
                 "ranks": inf["ranks"].tolist(), "mnnz": inf["mnnz"], "w_max_abs": inf["w_max_abs"],
                 "perm_sha": digest(R.perm()), "blocks": {}}
        for lv in range(inf["nlev"]):
            nb = 1 if lv == inf["nlev"] - 1 else int(inf["ncomps"][lv])
            entry["blocks"][str(lv)] = [[digest(*R.block(lv, b, w)) for w in (0, 1)] for b in range(nb)]
        probe = rhs(n, SEED + 1)
        b = rhs(n, SEED)
        out = {"probe": probe, "b": b, "apply": R.apply(probe)}
        x, it, err, conv = ref.gmres_solve(A, R, b, tol=1e-10, restart=30, flexible=True)
        out["fgmres30.x"] = x
        entry["fgmres30"] = {"iters": it, "err": err, "conv": conv}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        gm[name] = entry
    manifest["_gmslr"] = gm


def write_mtx_fixtures(d: str):
    """Small Matrix Market files exercising what ReadMtxTools handles (seeded)."""
    os.makedirs(d, exist_ok=True)
    rng = np.random.default_rng(SEED + 7)

    def entries(n, m, k, lower=None):
        rows = rng.integers(0, n, k)
        cols = rng.integers(0, m, k)
        if lower == "incl":
            rows, cols = np.maximum(rows, cols), np.minimum(rows, cols)
        elif lower == "strict":
            keep = rows != cols
            rows, cols = np.maximum(rows, cols)[keep], np.minimum(rows, cols)[keep]
        return rows, cols

    files = {}
    # general, 1-based, explicit zeros (exact and below 10 eps), duplicates, unsorted, comments, blank lines
    r, c = entries(30, 30, 160)
    v = rng.standard_normal(len(r))
    v[::17] = 0.0
    v[5::23] = 1e-16
    lines = ["%%MatrixMarket matrix coordinate real general", "% seeded fixture", "%",
             f"30 30 {len(r) + 3}"]
    for i, (a, b, x) in enumerate(zip(r, c, v)):
        lines.append(f"{a + 1} {b + 1} {float(x)!r}")
        if i == 40:
            lines.append("")
            lines.append("% a comment between entries")
    lines += [f"{r[0] + 1} {c[0] + 1} 2.5", "7 7 -3.25", "30 1 4e-3"]  # a duplicate and extra entries
    files["general"] = "\n".join(lines) + "\n"
    # symmetric (lower triangle with diagonal), keyword case mixed as some writers do
    r, c = entries(25, 25, 90, lower="incl")
    v = rng.standard_normal(len(r))
    files["symmetric"] = "\n".join(["%%MatrixMarket Matrix Coordinate Real Symmetric", f"25 25 {len(r)}"] +
                                    [f"{a + 1} {b + 1} {float(x)!r}" for a, b, x in zip(r, c, v)]) + "\n"
    # skew-symmetric (strictly lower)
    r, c = entries(20, 20, 70, lower="strict")
    v = rng.standard_normal(len(r))
    files["skew"] = "\n".join(["%%MatrixMarket matrix coordinate real skew-symmetric", f"20 20 {len(r)}"] +
                               [f"{a + 1} {b + 1} {float(x)!r}" for a, b, x in zip(r, c, v)]) + "\n"
    # complex general: real and imaginary parts, some zero in one part only
    r, c = entries(18, 18, 60)
    re, im = rng.standard_normal(len(r)), rng.standard_normal(len(r))
    re[::7] = 0.0
    im[3::5] = 0.0
    files["complex"] = "\n".join(["%%MatrixMarket matrix coordinate complex general", f"18 18 {len(r)}"] +
                                  [f"{a + 1} {b + 1} {float(x)!r} {float(y)!r}" for a, b, x, y in zip(r, c, re, im)]) + "\n"
    # hermitian: taken as stored
    r, c = entries(16, 16, 40, lower="incl")
    re, im = rng.standard_normal(len(r)), rng.standard_normal(len(r))
    files["hermitian"] = "\n".join(["%%MatrixMarket matrix coordinate complex hermitian", f"16 16 {len(r)}"] +
                                    [f"{a + 1} {b + 1} {float(x)!r} {float(y)!r}" for a, b, x, y in zip(r, c, re, im)]) + "\n"
    # rectangular general
    r, c = entries(12, 21, 50)
    v = rng.standard_normal(len(r))
    files["rect"] = "\n".join(["%%MatrixMarket matrix coordinate real general", f"12 21 {len(r)}"] +
                               [f"{a + 1} {b + 1} {float(x)!r}" for a, b, x in zip(r, c, v)]) + "\n"
    # right-hand sides: 30 x 2 array, column order
    vals = rng.standard_normal(60)
    files["rhs"] = "\n".join(["%%MatrixMarket matrix array real general", "% two right-hand sides", "30 2"] +
                              [repr(float(x)) for x in vals]) + "\n"
    for name, text in files.items():
        with open(os.path.join(d, f"{name}.mtx"), "w") as f:
            f.write(text)
    return files


def mtx_section(manifest):
    d = os.path.join(HERE, "mtx")
    write_mtx_fixtures(d)
    out = {}
    for name, parts in (("general", (0,)), ("symmetric", (0,)), ("skew", (0,)), ("complex", (0, 1)),
                        ("hermitian", (0, 1)), ("rect", (0,))):
        for part in parts:
            A = ref.RefCSR.from_mtx(os.path.join(d, f"{name}.mtx"), part)
            rp, ci, v = A.arrays()
            out[f"{name}.{part}.rowptr"], out[f"{name}.{part}.col"], out[f"{name}.{part}.val"] = rp, ci, v
    np.savez_compressed(os.path.join(HERE, "mtx_cases.npz"), **out)
    manifest["_mtx"] = {"files": sorted(os.listdir(d)), "reader": "HOST::ReadMtxTools<double>::loadMatrix"}


if __name__ == "__main__":
    main(sys.argv[1:] or ["basic", "amsed", "gmslr", "mtx"])
