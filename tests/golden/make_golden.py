"""Generates the golden fixtures in tests/golden/ by running the compiled CPS
reference (oracle/_ref/cpsref, built by oracle/build_ref.sh from the reference
sources).  Run from the repository root:  python tests/golden/make_golden.py

Inputs are re-created from seeds by cps_public_b200.fields (a SHA-256 of each
input is stored so a drifting generator is caught); outputs are stored in full.
OMP_NUM_THREADS=1 makes the reference's reductions sequential.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cps_public_b200 import fields  # noqa: E402
from oracle import refrun  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, action, dims, ls, eps, seed, mass, extra parameters)
CASES = [
    ("wilson_4x4x4x4", "wilson", (4, 4, 4, 4), 1, 0.3, 11, 0.1, {}),
    ("wilson_aprd_4x4x4x4", "wilson", (4, 4, 4, 4), 1, 0.3, 12, 0.1, {"bc_t": 1}),
    ("dwf_4x4x4x4_ls4", "dwf", (4, 4, 4, 4), 4, 0.2, 21, 0.05, {"m5": 1.8}),
    ("mobius_4x4x4x4_ls4", "mobius", (4, 4, 4, 4), 4, 0.2, 31, 0.05, {"m5": 1.8, "b": 1.5, "c": 0.5}),
]

SHIFTS = [0.0, 0.01, 0.1]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).hexdigest()


def gen_case(name, action, dims, ls, eps, seed, mass, extra):
    u = fields.random_gauge(dims, eps, seed)
    nsites = int(np.prod(dims)) // 2 * ls
    src = fields.random_source(nsites, seed)
    kw = dict(ls=ls, mass=mass, threads=1, **extra)
    rec = {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "ls": ls, "eps": eps,
           "seed": seed, "mass": mass}
    for k, v in extra.items():
        rec[k] = v
    full = action == "wilson"
    dsl = [(0, 0), (0, 1), (1, 0), (1, 1)] if full else [(1, 0), (0, 1)]
    for cb, dag in dsl:
        _, _, r = refrun.run(refrun.OP_DSLASH, action, dims, u, [src], cb=cb, dag=dag, **kw)
        rec[f"dslash_cb{cb}_dag{dag}"] = r
    if "bc_t" in extra:
        return rec
    for dag in (0, 1):
        _, _, r = refrun.run(refrun.OP_MATPC, action, dims, u, [src], dag=dag, **kw)
        rec[f"matpc_dag{dag}"] = r
    _, rp, r = refrun.run(refrun.OP_MDAGM, action, dims, u, [src], **kw)
    rec["mdagm"] = r
    rec["mdagm_dot"] = rp[0]
    it, rp, r = refrun.run(refrun.OP_INVCG, action, dims, u, [src, np.zeros_like(src)],
                           stop_rsd=1e-10, max_iter=5000, **kw)
    rec["cg_sol"] = r
    rec["cg_iters"] = it
    rec["cg_true_res"] = rp[0]
    ns = len(SHIFTS) if full else 2
    it, rp, r = refrun.run(refrun.OP_MINVCG, action, dims, u, [src], shifts=SHIFTS[:ns],
                           extra=[np.full(ns, 1e-9), np.ones(ns)], max_iter=5000, **kw)
    rec["minvcg_shifts"] = np.array(SHIFTS[:ns])
    rec["minvcg_sol"] = r.reshape(ns, -1)
    rec["minvcg_iters"] = it
    rec["minvcg_rsd"] = rp[:ns].copy()
    if action == "mobius":
        for dag in (0, 1):
            _, _, r = refrun.run(refrun.OP_M5INV, action, dims, u, [src], dag=dag, **kw)
            rec[f"m5inv_dag{dag}"] = r
        for cb, dag in [(1, 0), (0, 1)]:
            _, _, r = refrun.run(refrun.OP_MOBIUS_D4, action, dims, u, [src], cb=cb, dag=dag, **kw)
            rec[f"d4_cb{cb}_dag{dag}"] = r
    return rec


def gen_wilson_8x8x8x8_cg():
    """The reference's own CPU-runnable benchmark case: Wilson 8^4, eps 0.3,
    mass 0.1, Gaussian source on the odd checkerboard, stop_rsd 1e-10."""
    dims = (8, 8, 8, 8)
    u = fields.random_gauge(dims, 0.3, 100)
    src = fields.random_source(int(np.prod(dims)) // 2, 100)
    it, rp, r = refrun.run(refrun.OP_INVCG, "wilson", dims, u, [src, np.zeros_like(src)],
                           mass=0.1, stop_rsd=1e-10, max_iter=5000, threads=1)
    return {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "eps": 0.3,
            "seed": 100, "mass": 0.1, "cg_sol": r, "cg_iters": it, "cg_true_res": rp[0]}


def matinv_inputs(rec):
    """Full-lattice source and initial guess of the MatInv fixtures: Gaussian
    checkerboards from seed+500..503 (the guess scaled by 0.01)."""
    dims = tuple(int(d) for d in rec["dims"])
    n = int(np.prod(dims)) // 2 * int(rec.get("ls", 1))
    seed = int(rec["seed"])
    src = np.concatenate([fields.random_source(n, seed + 500), fields.random_source(n, seed + 501)])
    guess = 0.01 * np.concatenate([fields.random_source(n, seed + 502), fields.random_source(n, seed + 503)])
    return src, guess


def gen_matinv(name, action, dims, ls, eps, seed, mass, extra):
    """DiracOp*::MatInv (full-lattice solve, source preserved) of the case."""
    u = fields.random_gauge(dims, eps, seed)
    base = {"dims": np.array(dims), "ls": ls, "seed": seed}
    src, guess = matinv_inputs(base)
    it, rp, out = refrun.run(refrun.OP_MATINV, action, dims, u, [src, guess], ls=ls, mass=mass,
                             stop_rsd=1e-10, max_iter=5000, threads=1, **extra)
    rec = {"gauge_sha": sha(u), "matinv_src_sha": sha(src), "matinv_guess_sha": sha(guess), "dims": np.array(dims),
           "ls": ls, "eps": eps, "seed": seed, "mass": mass, "matinv_sol": out, "matinv_true_res": rp[0]}
    for k, v in extra.items():
        rec[k] = v
    return rec


FCONVERT_CASES = [("wilson", (4, 4, 4, 6), 1, 0, {}), ("dwf", (4, 4, 4, 6), 4, 0, {"m5": 1.8}),
                  ("mobius", (4, 4, 4, 6), 4, 1, {"m5": 1.8, "b": 1.5, "c": 0.5})]


def coded_field(dims, ls):
    """Full fermion field whose site i carries i + c/32 in component c."""
    n = int(np.prod(dims)) * ls
    return (np.arange(n)[:, None] + np.arange(24)[None, :] / 32.0).reshape(-1)


def gen_fconvert():
    """Lattice::Fconvert as site permutations: perm[j] = canonical site that
    lands at position j (CANONICAL -> order) and its inverse direction."""
    rec = {}
    for action, dims, ls, order, extra in FCONVERT_CASES:
        u = fields.random_gauge(dims, 0.2, 7)
        v = coded_field(dims, ls)
        for direction in (0, 1):
            _, _, out = refrun.run(refrun.OP_FCONVERT, action, dims, u, [v], ls=ls, order=order,
                                   direction=direction, threads=1, **extra)
            site = out.reshape(-1, 24)
            perm = np.floor(site[:, 0]).astype(np.int32)
            assert np.array_equal(site - perm[:, None], np.tile(np.arange(24) / 32.0, (len(perm), 1)))
            rec[f"{action}_dir{direction}"] = perm
    return rec


MINRESEXT_DEGREE = 4


def minresext_inputs(rec):
    """Source and previous solutions of the MinResExt fixtures (seed+600.. Gaussian)."""
    dims = tuple(int(d) for d in rec["dims"])
    n = int(np.prod(dims)) // 2 * int(rec.get("ls", 1))
    seed = int(rec["seed"])
    phi = fields.random_source(n, seed + 600)
    prev = [fields.random_source(n, seed + 601 + i) for i in range(MINRESEXT_DEGREE)]
    return phi, prev


def gen_minresext(name, action, dims, ls, eps, seed, mass, extra):
    """DiracOp::MinResExt: the guess psi in full, the orthonormalised previous
    solutions and their MatPcDagMatPc images as SHA-256 digests."""
    u = fields.random_gauge(dims, eps, seed)
    base = {"dims": np.array(dims), "ls": ls, "seed": seed}
    phi, prev = minresext_inputs(base)
    _, _, pay = refrun.run(refrun.OP_MINRESEXT, action, dims, u, [phi] + prev, ls=ls, mass=mass,
                           degree=MINRESEXT_DEGREE, threads=1, **extra)
    n = phi.size
    d = MINRESEXT_DEGREE
    rec = {"gauge_sha": sha(u), "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed, "mass": mass,
           "psi": pay[:n], "v_sha": sha(pay[n:(1 + d) * n]), "vm_sha": sha(pay[(1 + d) * n:])}
    for k, v in extra.items():
        rec[k] = v
    return rec


def main_minresext():
    for case in CASES:
        if "bc_t" in case[7]:
            continue
        rec = gen_minresext(*case)
        np.savez_compressed(os.path.join(OUT, "minresext_" + case[0] + ".npz"), **rec)
        print("wrote minresext_" + case[0])


def main():
    if not refrun.available():
        sys.exit("oracle/_ref/cpsref missing: run oracle/build_ref.sh first")
    for case in CASES:
        rec = gen_case(*case)
        np.savez_compressed(os.path.join(OUT, case[0] + ".npz"), **rec)
        print("wrote", case[0])
    np.savez_compressed(os.path.join(OUT, "wilson_8x8x8x8_cg.npz"), **gen_wilson_8x8x8x8_cg())
    print("wrote wilson_8x8x8x8_cg")
    main_matinv()
    main_fconvert()
    main_minresext()
    main_pc()
    main_dminus()
    main_zmobius()
    main_cg16()


# Mobius with the non-default preconditioners ZMOB_PC_ORIG (0) and ZMOB_PC_SYM1 (1)
PC_CASES = [
    ("mobius_orig_4x4x4x4_ls4", "mobius", (4, 4, 4, 4), 4, 0.2, 35, 0.05, {"m5": 1.8, "b": 1.5, "c": 0.5, "pc_type": 0}),
    ("mobius_sym1_4x4x4x4_ls8", "mobius", (4, 4, 4, 4), 8, 0.2, 36, 0.03, {"m5": 1.8, "b": 2.0, "c": 1.0, "pc_type": 1}),
]


def main_pc():
    for case in PC_CASES:
        # the hop, M5^-1 and D4 do not depend on the preconditioner: not stored again
        rec = {k: v for k, v in gen_case(*case).items() if not k.startswith(("dslash_", "m5inv_", "d4_"))}
        np.savez_compressed(os.path.join(OUT, case[0] + ".npz"), **rec)
        np.savez_compressed(os.path.join(OUT, "matinv_" + case[0] + ".npz"), **gen_matinv(*case))
        print("wrote", case[0], "and matinv_" + case[0])


# zMobius (complex per-slice b_s, c_s: b_s = b + 0.3 z, c_s = c + 0.2 z' with
# complex Gaussian z, z' from the case seed), SYM2
ZMOBIUS_CASES = [("zmobius_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 37, 0.04, 1.5, 0.5),
                 ("zmobius_orig_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 38, 0.04, 1.5, 0.5, 0),
                 ("zmobius_sym1_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 39, 0.04, 1.5, 0.5, 1),
                 # ZMOB_PC_SYM1_MIT (3), SYM2_MIT (4), SYM3 (5): operators and CG only
                 ("zmobius_sym1mit_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 40, 0.04, 1.5, 0.5, 3),
                 ("zmobius_sym2mit_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 41, 0.04, 1.5, 0.5, 4),
                 ("zmobius_sym3_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 42, 0.04, 1.5, 0.5, 5)]


def zmobius_coefficients(ls, seed, b, c):
    rng = np.random.default_rng(seed + 900)
    zb = b + 0.3 * (rng.standard_normal(ls) + 1j * rng.standard_normal(ls))
    zc = c + 0.2 * (rng.standard_normal(ls) + 1j * rng.standard_normal(ls))
    return zb, zc


def gen_zmobius(name, dims, ls, eps, seed, mass, b, c, pc_type=2):
    """DiracOpZMobius MatPc / MatPcDag / MatPcDagMatPc, InvCg, FmatEvlMInv and (for
    SYM2) the zmobius_m5inv / zmobius_dslash_4 kernels on complex coefficients."""
    u = fields.random_gauge(dims, eps, seed)
    src = fields.random_source(int(np.prod(dims)) // 2 * ls, seed)
    zb, zc = zmobius_coefficients(ls, seed, b, c)
    kw = dict(ls=ls, mass=mass, m5=1.8, b=b, c=c, zb=zb, zc=zc, pc_type=pc_type, threads=1)
    rec = {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed,
           "mass": mass, "m5": 1.8, "zb": zb, "zc": zc, "pc_type": pc_type}
    for dag in (0, 1):
        _, _, rec[f"matpc_dag{dag}"] = refrun.run(refrun.OP_MATPC, "zmobius", dims, u, [src], dag=dag, **kw)
        if pc_type == 2:
            _, _, rec[f"m5inv_dag{dag}"] = refrun.run(refrun.OP_M5INV, "zmobius", dims, u, [src], dag=dag, **kw)
    for cb, dag in ([(1, 0), (0, 1)] if pc_type == 2 else []):
        _, _, rec[f"d4_cb{cb}_dag{dag}"] = refrun.run(refrun.OP_MOBIUS_D4, "zmobius", dims, u, [src], cb=cb,
                                                      dag=dag, **kw)
    full, guess = matinv_inputs({"dims": np.array(dims), "ls": ls, "seed": seed})
    if pc_type == 2:  # DiracOpZMobius::Dminus of the full MatInv-fixture source (odd half first)
        rec["dminus_src_sha"] = sha(full)
        _, _, rec["dminus_out"] = refrun.run(refrun.OP_DMINUS, "zmobius", dims, u, [full], **kw)
    if pc_type in (0, 2):  # DiracOpZMobius::MatInv and Fzmobius::FmatInv(dminus = 1) from a nonzero guess
        rec["matinv_src_sha"], rec["matinv_guess_sha"] = sha(full), sha(guess)
        it, rp, rec["zmatinv_sol"] = refrun.run(refrun.OP_MATINV, "zmobius", dims, u, [full, guess],
                                                stop_rsd=1e-10, max_iter=5000, **kw)
        rec["zmatinv_iters"], rec["zmatinv_true_res"] = it, rp[0]
        it, rp, rec["zfmatinv_sol"] = refrun.run(refrun.OP_FMATINV, "zmobius", dims, u, [full, guess],
                                                 stop_rsd=1e-10, max_iter=5000, dminus=1, **kw)
        rec["zfmatinv_iters"], rec["zfmatinv_true_res"] = it, rp[0]
    _, rp, rec["mdagm"] = refrun.run(refrun.OP_MDAGM, "zmobius", dims, u, [src], **kw)
    rec["mdagm_dot"] = rp[0]
    it, rp, rec["cg_sol"] = refrun.run(refrun.OP_INVCG, "zmobius", dims, u, [src, np.zeros_like(src)],
                                       stop_rsd=1e-10, max_iter=5000, **kw)
    rec["cg_iters"], rec["cg_true_res"] = it, rp[0]
    if pc_type >= 3:
        return rec
    ns = 2
    it, rp, r = refrun.run(refrun.OP_MINVCG, "zmobius", dims, u, [src], shifts=SHIFTS[:ns],
                           extra=[np.full(ns, 1e-9), np.ones(ns)], max_iter=5000, **kw)
    rec["minvcg_shifts"] = np.array(SHIFTS[:ns])
    rec["minvcg_sol"] = r.reshape(ns, -1)
    rec["minvcg_iters"] = it
    rec["minvcg_rsd"] = rp[:ns].copy()
    return rec


def main_zmobius():
    for case in ZMOBIUS_CASES:
        np.savez_compressed(os.path.join(OUT, case[0] + ".npz"), **gen_zmobius(*case))
        print("wrote", case[0])


DMINUS_CASES = [("mobius_4x4x4x4_ls4", (4, 4, 4, 4), 4, 0.2, 31, 0.05, 1.5, 0.5),
                ("mobius_b2c1_4x4x4x4_ls8", (4, 4, 4, 4), 8, 0.2, 33, 0.02, 2.0, 1.0)]


def gen_dminus(name, dims, ls, eps, seed, mass, b, c):
    """DiracOpMobius::Dminus of the MatInv source, and Lattice::FmatInv with
    dminus = 1 (Dminus applied to the source, then MatInv) from the MatInv guess."""
    u = fields.random_gauge(dims, eps, seed)
    base = {"dims": np.array(dims), "ls": ls, "seed": seed}
    src, guess = matinv_inputs(base)
    kw = dict(ls=ls, mass=mass, m5=1.8, b=b, c=c, threads=1)
    _, _, dm = refrun.run(refrun.OP_DMINUS, "mobius", dims, u, [src], **kw)
    it, rp, sol = refrun.run(refrun.OP_FMATINV, "mobius", dims, u, [src, guess], stop_rsd=1e-10, max_iter=5000,
                             dminus=1, **kw)
    return {"gauge_sha": sha(u), "matinv_src_sha": sha(src), "matinv_guess_sha": sha(guess),
            "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed, "mass": mass, "m5": 1.8, "b": b, "c": c,
            "dminus_out": dm, "fmatinv_sol": sol, "fmatinv_true_res": rp[0], "fmatinv_iters": it}


def main_dminus():
    for case in DMINUS_CASES:
        np.savez_compressed(os.path.join(OUT, "dminus_" + case[0] + ".npz"), **gen_dminus(*case))
        print("wrote dminus_" + case[0])


def main_matinv():
    for case in CASES:
        if "bc_t" in case[7]:
            continue
        rec = gen_matinv(*case)
        np.savez_compressed(os.path.join(OUT, "matinv_" + case[0] + ".npz"), **rec)
        print("wrote matinv_" + case[0])


def main_fconvert():
    np.savez_compressed(os.path.join(OUT, "fconvert_4x4x4x6.npz"), **gen_fconvert())
    print("wrote fconvert_4x4x4x6")


# CG at the 8^4 x Ls 16 volume, where a whole CPS solve still takes well under
# a minute: the solution is pinned by the SHA-256 of its bytes (the oracle
# restates CPS bit for bit), with its norm and inner products with four seeded
# vectors kept as a readable digest.
CG16_CASES = [("cg_dwf_8x8x8x8_ls16", "dwf", (8, 8, 8, 8), 16, 0.2, 60, 0.1, {"m5": 1.8}),
              ("cg_mobius_8x8x8x8_ls16", "mobius", (8, 8, 8, 8), 16, 0.2, 61, 0.1, {"m5": 1.8, "b": 1.5, "c": 0.5})]
DIGEST_SEEDS = (1000, 1001, 1002, 1003)


def solution_digest(x, nsites):
    return np.array([float(x @ x)] + [float(x @ fields.random_source(nsites, s)) for s in DIGEST_SEEDS])


def gen_cg16(name, action, dims, ls, eps, seed, mass, extra):
    u = fields.random_gauge(dims, eps, seed)
    nsites = int(np.prod(dims)) // 2 * ls
    src = fields.random_source(nsites, seed)
    it, rp, r = refrun.run(refrun.OP_INVCG, action, dims, u, [src, np.zeros_like(src)], ls=ls, mass=mass,
                           stop_rsd=1e-10, max_iter=5000, threads=1, **extra)
    rec = {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed,
           "mass": mass, "cg_iters": it, "cg_true_res": rp[0], "cg_sol_sha": sha(r),
           "cg_sol_digest": solution_digest(r, nsites)}
    for k, v in extra.items():
        rec[k] = v
    return rec


# MInvCG (MULTI) at the same volume: four shifts, each solution pinned the same way
MINVCG16_CASE = ("minvcg_dwf_8x8x8x8_ls16", "dwf", (8, 8, 8, 8), 16, 0.2, 62, 0.1, {"m5": 1.8})
MINVCG16_SHIFTS = (1e-3, 0.05, 0.4, 2.0)


def gen_minvcg16(name, action, dims, ls, eps, seed, mass, extra):
    u = fields.random_gauge(dims, eps, seed)
    nsites = int(np.prod(dims)) // 2 * ls
    src = fields.random_source(nsites, seed)
    ns = len(MINVCG16_SHIFTS)
    it, rp, r = refrun.run(refrun.OP_MINVCG, action, dims, u, [src], ls=ls, mass=mass, shifts=MINVCG16_SHIFTS,
                           extra=[np.full(ns, 1e-10), np.ones(ns)], max_iter=5000, threads=1, **extra)
    sols = r.reshape(ns, -1)
    rec = {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed,
           "mass": mass, "minvcg_shifts": np.array(MINVCG16_SHIFTS), "minvcg_iters": it,
           "minvcg_rsd": rp[:ns].copy(), "minvcg_sol_sha": np.array([sha(x) for x in sols]),
           "minvcg_sol_digest": np.stack([solution_digest(x, nsites) for x in sols])}
    for k, v in extra.items():
        rec[k] = v
    return rec


# zMobius (SYM2, complex b_s, c_s from zmobius_coefficients) CG at the same volume
ZCG16_CASE = ("cg_zmobius_8x8x8x8_ls16", (8, 8, 8, 8), 16, 0.2, 63, 0.1, 1.5, 0.5)


def gen_zcg16(name, dims, ls, eps, seed, mass, b, c):
    u = fields.random_gauge(dims, eps, seed)
    nsites = int(np.prod(dims)) // 2 * ls
    src = fields.random_source(nsites, seed)
    zb, zc = zmobius_coefficients(ls, seed, b, c)
    it, rp, r = refrun.run(refrun.OP_INVCG, "zmobius", dims, u, [src, np.zeros_like(src)], ls=ls, mass=mass, m5=1.8,
                           b=b, c=c, zb=zb, zc=zc, pc_type=2, stop_rsd=1e-10, max_iter=5000, threads=1)
    return {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed,
            "mass": mass, "m5": 1.8, "zb": zb, "zc": zc, "pc_type": 2, "cg_iters": it, "cg_true_res": rp[0],
            "cg_sol_sha": sha(r), "cg_sol_digest": solution_digest(r, nsites)}


# The benchmark lattice itself (bench.py's fields: DWF 16^3x32, Ls 16, m_f 0.01,
# M5 1.8, links eps 0.2 seed 2024, Gaussian source seed 2025): one Dslash
# (cb 1, dag 0) and one MatPcDagMatPc of the compiled reference, each output
# pinned by its SHA-256 and digest, and the fused dot.
BENCH16_CASE = ("bench_dwf_16x16x16x32_ls16", "dwf", (16, 16, 16, 32), 16, 0.2, 2024, 2025, 0.01)


def gen_bench16(name, action, dims, ls, eps, seed, src_seed, mass):
    u = fields.random_gauge(dims, eps, seed)
    nsites = int(np.prod(dims)) // 2 * ls
    src = fields.random_source(nsites, src_seed)
    _, _, d = refrun.run(refrun.OP_DSLASH, action, dims, u, [src], ls=ls, mass=mass, m5=1.8, cb=1, dag=0,
                         threads=1)
    _, rp, m = refrun.run(refrun.OP_MDAGM, action, dims, u, [src], ls=ls, mass=mass, m5=1.8, threads=1)
    return {"gauge_sha": sha(u), "src_sha": sha(src), "dims": np.array(dims), "ls": ls, "eps": eps, "seed": seed,
            "src_seed": src_seed, "mass": mass, "m5": 1.8,
            "dslash_sha": sha(d), "dslash_digest": solution_digest(d, nsites),
            "mdagm_sha": sha(m), "mdagm_digest": solution_digest(m, nsites), "mdagm_dot": rp[0]}


def main_bench16():
    np.savez_compressed(os.path.join(OUT, BENCH16_CASE[0] + ".npz"), **gen_bench16(*BENCH16_CASE))
    print("wrote", BENCH16_CASE[0])


def main_cg16():
    for case in CG16_CASES:
        np.savez_compressed(os.path.join(OUT, case[0] + ".npz"), **gen_cg16(*case))
        print("wrote", case[0])
    np.savez_compressed(os.path.join(OUT, MINVCG16_CASE[0] + ".npz"), **gen_minvcg16(*MINVCG16_CASE))
    print("wrote", MINVCG16_CASE[0])
    np.savez_compressed(os.path.join(OUT, ZCG16_CASE[0] + ".npz"), **gen_zcg16(*ZCG16_CASE))
    print("wrote", ZCG16_CASE[0])


if __name__ == "__main__":
    if "--matinv" in sys.argv:
        main_matinv()
    elif "--fconvert" in sys.argv:
        main_fconvert()
    elif "--minresext" in sys.argv:
        main_minresext()
    elif "--dminus" in sys.argv:
        main_dminus()
    elif "--pc" in sys.argv:
        main_pc()
    elif "--zmobius" in sys.argv:
        main_zmobius()
    elif "--cg16" in sys.argv:
        main_cg16()
    elif "--bench16" in sys.argv:
        main_bench16()
    else:
        main()
