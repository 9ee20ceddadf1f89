"""Properties of the operators that hold independently of any golden vector,
checked on the C oracle (CPU): Dslash's dag form is its adjoint (and the
Wilson hop gamma_5-hermitian), MatPcDag is the adjoint of MatPc and
MatPcDagMatPc is Hermitian and positive, for every action and every
preconditioner; zMobius with constant coefficients is Mobius; Dminus is
linear (tolerances at rounding level, 1e-13 relative).  The solvers solve:
InvCg's solution meets its tolerance against an independently formed
residual, MInvCG's MULTI solutions each solve their shifted system, SINGLE
returns the alpha-weighted sum of the MULTI solutions, and the Wilson and DWF
full-lattice MatInv solves M x = b on both checkerboards."""
import numpy as np
import pytest

from cps_public_b200 import fields
from oracle import oracle

DIMS = (4, 4, 4, 4)
ZB = [1.5 + 0.3j, 1.4 - 0.2j, 1.6 + 0.1j, 1.5 - 0.05j]
ZC = [0.5 - 0.1j, 0.45 + 0.2j, 0.55, 0.5 + 0.05j]


def cdot(a, b):
    """conj(a) . b over complex pairs."""
    a = a.reshape(-1, 2)
    b = b.reshape(-1, 2)
    return complex(np.sum(a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]), np.sum(a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]))


def make(kind):
    u = fields.random_gauge(DIMS, 0.2, 7)
    action, pc = kind
    if action == "wilson":
        return oracle.Op("wilson", DIMS, u, mass=0.1)
    if action == "dwf":
        return oracle.Op("dwf", DIMS, u, ls=4, mass=0.05)
    if action == "mobius":
        return oracle.Op("mobius", DIMS, u, ls=4, mass=0.05, pc_type=pc)
    return oracle.Op("mobius", DIMS, u, ls=4, mass=0.05, pc_type=pc, bs=ZB, cs=ZC)


KINDS = [("wilson", 2), ("dwf", 2)] + [("mobius", pc) for pc in (0, 1, 2)] + [("zmobius", pc) for pc in range(6)]


@pytest.mark.parametrize("kind", KINDS, ids=[f"{a}-pc{p}" for a, p in KINDS])
def test_matpcdag_is_adjoint_and_mdagm_hermitian_positive(kind):
    op = make(kind)
    n = op.n // 24
    x, y = fields.random_source(n, 1), fields.random_source(n, 2)
    lhs, rhs = cdot(y, op.matpc(x, 0)), cdot(op.matpc(y, 1), x)
    assert abs(lhs - rhs) <= 1e-13 * abs(lhs)
    ax, dot = op.mdagm(x)
    ay, _ = op.mdagm(y)
    assert abs(cdot(x, ay) - cdot(ax, y)) <= 1e-13 * abs(cdot(x, ay))
    xax = cdot(x, ax)
    assert xax.real > 0 and abs(xax.imag) <= 1e-13 * xax.real
    # the fused norm is |MatPc x|^2
    mx = op.matpc(x, 0)
    assert abs(dot - float(mx @ mx)) <= 1e-13 * dot


@pytest.mark.parametrize("pc", [0, 1, 2])
def test_zmobius_constant_coefficients_are_mobius(pc):
    u = fields.random_gauge(DIMS, 0.2, 8)
    m = oracle.Op("mobius", DIMS, u, ls=4, mass=0.05, b=1.5, c=0.5, pc_type=pc)
    z = oracle.Op("mobius", DIMS, u, ls=4, mass=0.05, pc_type=pc, bs=[1.5] * 4, cs=[0.5] * 4)
    x = fields.random_source(m.n // 24, 3)
    a, da = m.mdagm(x)
    b, db = z.mdagm(x)
    assert np.linalg.norm(a - b) <= 1e-14 * np.linalg.norm(a) and abs(da - db) <= 1e-14 * da


@pytest.mark.parametrize("action", ["mobius", "zmobius"])
def test_dminus_is_linear(action):
    op = make((action, 2))
    n = 2 * (op.n // 24)
    x, y = fields.random_source(n, 4), fields.random_source(n, 5)
    f = op.dminus if action == "mobius" else op.zdminus
    lhs = f(0.7 * x - 1.3 * y)
    rhs = 0.7 * f(x) - 1.3 * f(y)
    assert np.linalg.norm(lhs - rhs) <= 1e-13 * np.linalg.norm(rhs)


def shifted_residual(op, x, b, shift):
    ax, _ = op.mdagm(x)
    return np.linalg.norm(ax + shift * x - b) / np.linalg.norm(b)


@pytest.mark.parametrize("kind", [("wilson", 2), ("dwf", 2), ("mobius", 2), ("zmobius", 2)], ids=lambda k: k[0])
def test_invcg_solves_the_system(kind):
    op = make(kind)
    b = fields.random_source(op.n // 24, 6)
    x, it, true_res = op.invcg(b, stop_rsd=1e-10)
    res = shifted_residual(op, x, b, 0.0)
    assert 0 < it < 5000 and res < 2e-10
    assert abs(true_res - res) <= 1e-3 * res


@pytest.mark.parametrize("action", ["wilson", "dwf"])
def test_minvcg_multi_solves_every_shift_and_single_is_their_sum(action):
    op = make((action, 2))
    b = fields.random_source(op.n // 24, 7)
    shifts = [1e-3, 0.05, 0.4, 2.0]
    alpha = [0.7, -0.2, 1.3, 0.45]
    xs, _, rs = op.minvcg(b, shifts, [1e-10] * 4, ms_type=0)
    for x, s, r in zip(xs, shifts, rs):
        # the reported residual is the iterated absolute one; the true relative residual follows it
        assert shifted_residual(op, x, b, s) < 3e-10
        assert r < 1e-10 * np.linalg.norm(b)
    (xsum,), _, _ = op.minvcg(b, shifts, [1e-10] * 4, ms_type=1, alpha=alpha)
    ref = sum(a * x for a, x in zip(alpha, xs))
    assert np.linalg.norm(xsum - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("action", ["wilson", "dwf"])
def test_matinv_solves_the_full_lattice_system(action):
    """MatInv solves M x = b on both checkerboards with M = 1 - kappa D
    (d_op_wilson.C:257-334, d_op_dwf.C:316-507); kappa = 1/(2(m + 4)) for Wilson
    (d_op_wilson.C:134-137), 1/(2(4 + a5_inv - M5)) for DWF (dwf_init.C:97-98).
    Full vectors are odd half first; Dslash(in, cb) reads checkerboard cb and
    writes the other one.  The even half is rebuilt exactly, the odd half is
    the CG solution."""
    op = make((action, 2))
    kappa = 1 / (2 * (0.1 + 4)) if action == "wilson" else 1 / (2 * (4 + 1.0 - 1.8))
    n = op.n
    b = np.concatenate([fields.random_source(n // 24, 8), fields.random_source(n // 24, 9)])
    x, it, _ = op.matinv(b, stop_rsd=1e-12)
    xo, xe = x[:n], x[n:]
    ro = xo - kappa * op.dslash(xe, 0, 0)
    re = xe - kappa * op.dslash(xo, 1, 0)
    assert np.linalg.norm(ro - b[:n]) <= 1e-10 * np.linalg.norm(b[:n])
    assert np.linalg.norm(re - b[n:]) <= 1e-13 * np.linalg.norm(b[n:])


def gamma5(v):
    """gamma_5 = diag(1, 1, -1, -1) over spins in CPS's chiral basis (spin slowest in a site)."""
    w = v.reshape(-1, 4, 3, 2).copy()
    w[:, 2:] *= -1
    return w.reshape(-1)


@pytest.mark.parametrize("kind", [("wilson", 2), ("dwf", 2), ("mobius", 2)], ids=lambda k: k[0])
def test_dslash_dag_is_the_adjoint(kind):
    """<y, D(cb) x> = <D^dag(1 - cb) y, x> for the hop of every action; the
    Wilson hop is also gamma_5-hermitian, D^dag = gamma_5 D gamma_5, bit for bit
    (the 5-D operators are hermitian only together with the reflection
    s -> Ls - 1 - s, which moves a field to the other 5-D checkerboard)."""
    op = make(kind)
    n = op.n // 24
    x, y = fields.random_source(n, 1), fields.random_source(n, 2)
    for cb in (0, 1):
        lhs, rhs = cdot(y, op.dslash(x, cb, 0)), cdot(op.dslash(y, 1 - cb, 1), x)
        assert abs(lhs - rhs) <= 1e-13 * abs(lhs)
        if kind[0] == "wilson":
            np.testing.assert_array_equal(op.dslash(x, cb, 1), gamma5(op.dslash(gamma5(x), cb, 0)))
