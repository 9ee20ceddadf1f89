"""Pins the C oracle (oracle/cps_oracle.c) against golden vectors produced by
the compiled CPS reference (tests/golden/make_golden.py).  Agreement is bit for
bit: the oracle issues the reference's floating-point operations in order."""
import numpy as np
import pytest

from oracle import oracle
from tests.golden_util import load

CASES = ["wilson_4x4x4x4", "dwf_4x4x4x4_ls4", "mobius_4x4x4x4_ls4"]
# Mobius with ZMOB_PC_ORIG and ZMOB_PC_SYM1 (no hop fixtures: the hop does not
# depend on the preconditioner)
PC_CASES = ["mobius_orig_4x4x4x4_ls4", "mobius_sym1_4x4x4x4_ls8"]


def make_op(rec, u, action):
    kw = dict(ls=int(rec["ls"]), mass=float(rec["mass"]))
    for k in ("m5", "b", "c", "bc_t", "pc_type"):
        if k in rec:
            kw[k] = float(rec[k]) if k in ("m5", "b", "c") else int(rec[k])
    return oracle.Op(action, tuple(rec["dims"]), u, **kw)


@pytest.mark.parametrize("name", CASES + ["wilson_aprd_4x4x4x4"])
def test_dslash_bitexact(name):
    rec, u, src = load(name)
    op = make_op(rec, u, name.split("_")[0])
    keys = [k for k in rec if k.startswith("dslash_")]
    assert keys
    for k in keys:
        cb, dag = int(k[9]), int(k[-1])
        np.testing.assert_array_equal(op.dslash(src, cb, dag), rec[k], err_msg=k)


@pytest.mark.parametrize("name", CASES + PC_CASES)
def test_matpc_mdagm_bitexact(name):
    rec, u, src = load(name)
    op = make_op(rec, u, name.split("_")[0])
    for dag in (0, 1):
        np.testing.assert_array_equal(op.matpc(src, dag), rec[f"matpc_dag{dag}"])
    out, dot = op.mdagm(src)
    np.testing.assert_array_equal(out, rec["mdagm"])
    assert dot == float(rec["mdagm_dot"])


@pytest.mark.parametrize("name", CASES + PC_CASES)
def test_invcg_bitexact(name):
    rec, u, src = load(name)
    op = make_op(rec, u, name.split("_")[0])
    sol, it, tr = op.invcg(src, 1e-10, 5000)
    assert it == int(rec["cg_iters"])
    assert tr == float(rec["cg_true_res"])
    np.testing.assert_array_equal(sol, rec["cg_sol"])


@pytest.mark.parametrize("name", CASES + PC_CASES)
def test_minvcg_bitexact(name):
    rec, u, src = load(name)
    op = make_op(rec, u, name.split("_")[0])
    shifts = list(rec["minvcg_shifts"])
    sols, it, rsd = op.minvcg(src, shifts, [1e-9] * len(shifts))
    assert it == int(rec["minvcg_iters"])
    np.testing.assert_array_equal(rsd, rec["minvcg_rsd"])
    for i in range(len(shifts)):
        np.testing.assert_array_equal(sols[i], rec["minvcg_sol"][i])


def test_mobius_m5inv_d4_bitexact():
    rec, u, src = load("mobius_4x4x4x4_ls4")
    op = make_op(rec, u, "mobius")
    for dag in (0, 1):
        np.testing.assert_array_equal(op.m5inv(src, dag), rec[f"m5inv_dag{dag}"])
    for cb, dag in [(1, 0), (0, 1)]:
        np.testing.assert_array_equal(op.mobius_d4(src, cb, dag), rec[f"d4_cb{cb}_dag{dag}"])


def test_wilson_8x8x8x8_cg_config():
    """The reference's CPU-runnable benchmark case (Wilson 8^4 CG to 1e-10)."""
    rec, u, src = load("wilson_8x8x8x8_cg")
    op = oracle.Op("wilson", (8, 8, 8, 8), u, mass=0.1)
    sol, it, tr = op.invcg(src, 1e-10, 5000)
    assert it == int(rec["cg_iters"])
    assert tr == float(rec["cg_true_res"]) and tr <= 1e-10
    np.testing.assert_array_equal(sol, rec["cg_sol"])


@pytest.mark.parametrize("name", ["cg_dwf_8x8x8x8_ls16", "cg_mobius_8x8x8x8_ls16"])
def test_cg_8x8x8x8_ls16_bitexact(name):
    """DWF and Mobius (SYM2) InvCg at 8^4 x Ls 16, m_f 0.1, to 1e-10 (175-200
    iterations): iteration count, true residual and the solution's bytes."""
    from tests.golden.make_golden import solution_digest
    from tests.golden_util import sha
    rec, u, src = load(name)
    op = make_op(rec, u, name.split("_")[1])
    sol, it, tr = op.invcg(src, 1e-10, 5000)
    assert it == int(rec["cg_iters"])
    assert tr == float(rec["cg_true_res"]) and tr <= 1e-10
    np.testing.assert_array_equal(solution_digest(sol, op.n // 24), rec["cg_sol_digest"])
    assert sha(sol) == str(rec["cg_sol_sha"])


def test_zmobius_cg_8x8x8x8_ls16_bitexact():
    """zMobius (SYM2, complex b_s, c_s) InvCg at 8^4 x Ls 16, m_f 0.1, to 1e-10
    (421 iterations): iteration count, true residual and the solution's bytes."""
    from tests.golden.make_golden import solution_digest
    from tests.golden_util import sha
    rec, u, src = load("cg_zmobius_8x8x8x8_ls16")
    op = oracle.Op("mobius", tuple(rec["dims"]), u, ls=int(rec["ls"]), mass=float(rec["mass"]),
                   m5=float(rec["m5"]), bs=list(rec["zb"]), cs=list(rec["zc"]), pc_type=int(rec["pc_type"]))
    sol, it, tr = op.invcg(src, 1e-10, 5000)
    assert it == int(rec["cg_iters"])
    assert tr == float(rec["cg_true_res"]) and tr <= 1e-10
    np.testing.assert_array_equal(solution_digest(sol, op.n // 24), rec["cg_sol_digest"])
    assert sha(sol) == str(rec["cg_sol_sha"])


def test_minvcg_8x8x8x8_ls16_bitexact():
    """DWF MInvCG (MULTI, shifts 1e-3..2, 1e-10 each) at 8^4 x Ls 16: iteration
    count, the reported residuals and every solution's bytes."""
    from tests.golden.make_golden import solution_digest
    from tests.golden_util import sha
    rec, u, src = load("minvcg_dwf_8x8x8x8_ls16")
    op = make_op(rec, u, "dwf")
    shifts = list(rec["minvcg_shifts"])
    sols, it, rsd = op.minvcg(src, shifts, [1e-10] * len(shifts))
    assert it == int(rec["minvcg_iters"])
    np.testing.assert_array_equal(rsd, rec["minvcg_rsd"])
    for k, x in enumerate(sols):
        np.testing.assert_array_equal(solution_digest(x, op.n // 24), rec["minvcg_sol_digest"][k])
        assert sha(x) == str(rec["minvcg_sol_sha"][k])


@pytest.mark.parametrize("name", CASES + PC_CASES)
def test_matinv_bitexact(name):
    """DiracOp*::MatInv (full-lattice solve with source preparation and
    even/odd reconstruction) from a nonzero initial guess."""
    from tests.golden_util import load_matinv
    rec, u, src, guess = load_matinv(name)
    op = make_op(rec, u, name.split("_")[0])
    out, it, tr = op.matinv(src, guess, stop_rsd=1e-10, max_iter=5000)
    np.testing.assert_array_equal(out, rec["matinv_sol"])
    assert tr == float(rec["matinv_true_res"])


DMINUS_CASES = ["mobius_4x4x4x4_ls4", "mobius_b2c1_4x4x4x4_ls8"]


@pytest.mark.parametrize("name", DMINUS_CASES)
def test_dminus_fmatinv_bitexact(name):
    """DiracOpMobius::Dminus, and Lattice::FmatInv with dminus = 1 (Dminus of
    the source, then MatInv) from a nonzero initial guess."""
    from tests.golden_util import load_dminus
    rec, u, src, guess = load_dminus(name)
    op = make_op(rec, u, "mobius")
    np.testing.assert_array_equal(op.dminus(src), rec["dminus_out"])
    out, it, tr = op.fmatinv(src, guess, dminus=1, stop_rsd=1e-10, max_iter=5000)
    np.testing.assert_array_equal(out, rec["fmatinv_sol"])
    assert tr == float(rec["fmatinv_true_res"]) and it == int(rec["fmatinv_iters"])


@pytest.mark.parametrize("action,order", [("wilson", "wilson"), ("dwf", "wilson"), ("mobius", "4d_ee")])
def test_fermion_convert_matches_reference(action, order):
    """Lattice::Fconvert (CANONICAL <-> WILSON / 5-D checkerboard /
    DWF_4D_EOPREC_EE) as recorded from the compiled reference: the oracle's
    permutation moves every site exactly where CPS puts it, both directions."""
    import os
    from tests.golden.make_golden import FCONVERT_CASES, coded_field
    rec = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "fconvert_4x4x4x6.npz")))
    dims, ls = [(c[1], c[2]) for c in FCONVERT_CASES if c[0] == action][0]
    v = coded_field(dims, ls)
    for direction in (0, 1):
        out = oracle.fermion_convert(v, dims, ls, order, inverse=bool(direction)).reshape(-1, 24)
        perm = rec[f"{action}_dir{direction}"]
        np.testing.assert_array_equal(np.floor(out[:, 0]).astype(np.int32), perm)
        np.testing.assert_array_equal(out, coded_field(dims, ls).reshape(-1, 24)[perm])


@pytest.mark.parametrize("name", CASES)
def test_minresext_bitexact(name):
    """DiracOp::MinResExt (chronological initial guess): the guess, the
    orthonormalised previous solutions and their MatPcDagMatPc images."""
    import os
    from tests.golden.make_golden import minresext_inputs
    from tests.golden_util import sha
    rec = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"minresext_{name}.npz")))
    from cps_public_b200 import fields
    u = fields.random_gauge(tuple(int(d) for d in rec["dims"]), float(rec["eps"]), int(rec["seed"]))
    assert sha(u) == str(rec["gauge_sha"])
    op = make_op(rec, u, name.split("_")[0])
    phi, prev = minresext_inputs(rec)
    psi, v, vm, err = op.minresext(phi, prev)
    np.testing.assert_array_equal(psi, rec["psi"])
    assert sha(np.concatenate(v)) == str(rec["v_sha"]) and sha(np.concatenate(vm)) == str(rec["vm_sha"])


ZMOBIUS_CASES = ["zmobius_4x4x4x4_ls4", "zmobius_orig_4x4x4x4_ls4", "zmobius_sym1_4x4x4x4_ls4",
                 "zmobius_sym1mit_4x4x4x4_ls4", "zmobius_sym2mit_4x4x4x4_ls4", "zmobius_sym3_4x4x4x4_ls4"]


@pytest.mark.parametrize("name", ZMOBIUS_CASES)
def test_zmobius_bitexact(name):
    """zMobius with complex per-slice b_s, c_s (DiracOpZMobius; SYM2, ORIG, SYM1,
    SYM1_MIT, SYM2_MIT, SYM3): the zmobius_m5inv / zmobius_dslash_4 kernels,
    MatPc, MatPcDag, MatPcDagMatPc, InvCg and MInvCG against the compiled
    reference.  SYM3's CG is compared to 1e-10: the reference multiplies GJP's
    b_s, c_s by kappa_b i and divides them back around every operator call
    (zmobius_m-sym3.h), which is not exact, and its next kappa computation
    (reset_mobius_arg) reads the drifted values."""
    rec, u, src = load(name)
    op = oracle.Op("mobius", tuple(rec["dims"]), u, ls=int(rec["ls"]), mass=float(rec["mass"]),
                   m5=float(rec["m5"]), bs=list(rec["zb"]), cs=list(rec["zc"]), pc_type=int(rec["pc_type"]))
    for dag in (0, 1):
        if f"m5inv_dag{dag}" in rec:
            np.testing.assert_array_equal(op.m5inv(src, dag), rec[f"m5inv_dag{dag}"])
        np.testing.assert_array_equal(op.matpc(src, dag), rec[f"matpc_dag{dag}"])
    for cb, dag in [(1, 0), (0, 1)]:
        if f"d4_cb{cb}_dag{dag}" in rec:
            np.testing.assert_array_equal(op.mobius_d4(src, cb, dag), rec[f"d4_cb{cb}_dag{dag}"])
    out, dot = op.mdagm(src)
    np.testing.assert_array_equal(out, rec["mdagm"])
    assert dot == float(rec["mdagm_dot"])
    sol, it, tr = op.invcg(src, 1e-10, 5000)
    if int(rec["pc_type"]) == 5:
        assert abs(it - int(rec["cg_iters"])) <= 20 and tr <= 1e-10
        assert np.linalg.norm(sol - rec["cg_sol"]) <= 1e-10 * np.linalg.norm(rec["cg_sol"])
    else:
        assert it == int(rec["cg_iters"]) and tr == float(rec["cg_true_res"])
        np.testing.assert_array_equal(sol, rec["cg_sol"])
    if "minvcg_sol" in rec:
        shifts = list(rec["minvcg_shifts"])
        sols, it, rsd = op.minvcg(src, shifts, [1e-9] * len(shifts))
        assert it == int(rec["minvcg_iters"])
        for i in range(len(shifts)):
            np.testing.assert_array_equal(sols[i], rec["minvcg_sol"][i])
    from tests.golden.make_golden import matinv_inputs
    from tests.golden_util import sha
    full, guess = matinv_inputs(rec)
    if "dminus_out" in rec:  # DiracOpZMobius::Dminus
        assert sha(full) == str(rec["dminus_src_sha"])
        np.testing.assert_array_equal(op.zdminus(full), rec["dminus_out"])
    if "zmatinv_sol" in rec:  # DiracOpZMobius::MatInv and Fzmobius::FmatInv(dminus = 1)
        assert sha(full) == str(rec["matinv_src_sha"]) and sha(guess) == str(rec["matinv_guess_sha"])
        out, it, tr = op.zmatinv(full, guess)
        np.testing.assert_array_equal(out, rec["zmatinv_sol"])
        assert it == int(rec["zmatinv_iters"]) and tr == float(rec["zmatinv_true_res"])
        out, it, tr = op.zfmatinv(full, guess, dminus=1)
        np.testing.assert_array_equal(out, rec["zfmatinv_sol"])
        assert it == int(rec["zfmatinv_iters"]) and tr == float(rec["zfmatinv_true_res"])


def test_bench_lattice_bitexact():
    """The benchmark lattice (DWF 16^3x32, Ls 16, bench.py's links and first
    source): the oracle's Dslash and MatPcDagMatPc equal the compiled
    reference's bit for bit (SHA-256 of the outputs) and so does the dot."""
    import os

    from cps_public_b200 import fields
    from tests.golden_util import GOLDEN, sha
    rec = dict(np.load(os.path.join(GOLDEN, "bench_dwf_16x16x16x32_ls16.npz")))
    dims, ls = tuple(int(d) for d in rec["dims"]), int(rec["ls"])
    u = fields.random_gauge(dims, float(rec["eps"]), int(rec["seed"]))
    src = fields.random_source(int(np.prod(dims)) // 2 * ls, int(rec["src_seed"]))
    assert sha(u) == str(rec["gauge_sha"]) and sha(src) == str(rec["src_sha"])
    op = oracle.Op("dwf", dims, u, ls=ls, mass=float(rec["mass"]), m5=float(rec["m5"]))
    assert sha(op.dslash(src, 1, 0)) == str(rec["dslash_sha"])
    out, dot = op.mdagm(src)
    assert sha(out) == str(rec["mdagm_sha"])
    assert dot == float(rec["mdagm_dot"])
