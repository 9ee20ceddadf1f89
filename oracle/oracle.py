"""ctypes front end of the C oracle (oracle/cps_oracle.c). TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module;
the product never does.  Vectors are float64 numpy arrays in CPS checkerboard
order; the gauge field is passed in CANONICAL order and converted here.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(
                os.path.join(HERE, "cps_oracle.c")):
            build()
        _lib = C.CDLL(LIB)
    return _lib


_dp = C.POINTER(C.c_double)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class MobiusParams(C.Structure):
    _fields_ = [("ls", C.c_int), ("mass", C.c_double), ("m5", C.c_double), ("a5_inv", C.c_double),
                ("b", (C.c_double * 2) * 64), ("c", (C.c_double * 2) * 64), ("pc_type", C.c_int)]


class OpStruct(C.Structure):
    _fields_ = [("action", C.c_int), ("dims", C.c_int * 4), ("ls", C.c_int), ("mass", C.c_double),
                ("m5", C.c_double), ("a5_inv", C.c_double), ("u", _dp), ("mob", MobiusParams)]


ACTIONS = {"wilson": 0, "dwf": 1, "mobius": 2}


class Op:
    """A CPS fermion operator on the CPU: ``Op('dwf', dims, gauge_canonical, ls=16, mass=0.01)``."""

    def __init__(self, action, dims, gauge_canonical, ls=1, mass=0.1, m5=1.8, a5_inv=1.0, b=1.5,
                 c=0.5, pc_type=2, bs=None, cs=None, bc_t=0):
        self.action = ACTIONS[action] if isinstance(action, str) else action
        self.dims = tuple(int(d) for d in dims)
        self.ls = 1 if self.action == 0 else int(ls)
        self.dims_c = (C.c_int * 4)(*self.dims)
        self.uw = np.empty(len(gauge_canonical))
        ucan = np.array(gauge_canonical, np.float64)
        if bc_t:
            lib().orc_bondcond_t(_p(ucan), self.dims_c)
        lib().orc_canon_to_wilson(_p(self.uw), _p(ucan), self.dims_c)
        s = OpStruct()
        s.action = self.action
        s.dims = self.dims_c
        s.ls = self.ls
        s.mass = mass
        s.m5 = m5
        s.a5_inv = a5_inv
        s.u = _p(self.uw)
        s.mob.ls = self.ls
        s.mob.mass = mass
        s.mob.m5 = m5
        s.mob.a5_inv = a5_inv
        s.mob.pc_type = pc_type
        for i in range(min(self.ls, 64)):
            bb = bs[i] if bs is not None else complex(b)
            cc = cs[i] if cs is not None else complex(c)
            s.mob.b[i][0], s.mob.b[i][1] = bb.real, bb.imag
            s.mob.c[i][0], s.mob.c[i][1] = cc.real, cc.imag
        self.s = s
        self.n = 24 * int(np.prod(self.dims)) // 2 * self.ls

    def _v(self, x):
        x = np.ascontiguousarray(x, np.float64)
        assert x.size == self.n, (x.size, self.n)
        return x

    def dslash(self, x, cb, dag):
        out = np.zeros(self.n)
        lib().orc_dslash(C.byref(self.s), _p(out), _p(self._v(x)), cb, dag)
        return out

    def matpc(self, x, dag=0):
        out = np.zeros(self.n)
        rc = lib().orc_matpc(C.byref(self.s), _p(out), _p(self._v(x)), dag)
        if rc:
            raise ValueError("preconditioner not restated in the oracle")
        return out

    def mdagm(self, x):
        out = np.zeros(self.n)
        dot = C.c_double(0)
        rc = lib().orc_mdagm(C.byref(self.s), _p(out), _p(self._v(x)), C.byref(dot))
        if rc:
            raise ValueError("preconditioner not restated in the oracle")
        return out, dot.value

    def m5inv(self, x, dag=0):
        assert self.action == 2
        out = self._v(x).copy()
        lib().orc_mobius_m5inv(_p(out), dag, self.dims_c, C.byref(self.s.mob))
        return out

    def mobius_d4(self, x, cb, dag):
        assert self.action == 2
        out = np.zeros(self.n)
        lib().orc_mobius_dslash_4(_p(out), _p(self.uw), _p(self._v(x)), cb, dag, self.dims_c,
                                  C.byref(self.s.mob))
        return out

    def invcg(self, src, stop_rsd=1e-10, max_iter=5000, guess=None):
        sol = np.zeros(self.n) if guess is None else self._v(guess).copy()
        tr = C.c_double(0)
        hist = np.zeros(max(max_iter, 1))
        it = lib().orc_invcg(C.byref(self.s), _p(sol), _p(self._v(src)), C.c_double(stop_rsd),
                             max_iter, C.byref(tr), _p(hist))
        return sol, it, tr.value

    def minvcg(self, src, shifts, rsd, ms_type=0, alpha=None, max_iter=5000):
        ns = len(shifts)
        nvec = 1 if ms_type == 1 else ns
        sols = [np.zeros(self.n) for _ in range(ns)]
        ptrs = (_dp * ns)(*[_p(s) for s in sols])
        src = self._v(src)
        # chi_norm: the sequential sum FmatEvlMInv passes in (lattice/f_dwf_base/f_dwf_base.C:248)
        chi_norm = _seqsum(src)
        rs = np.array(rsd, np.float64)
        sh = np.array(shifts, np.float64)
        al = np.ones(ns) if alpha is None else np.array(alpha, np.float64)
        it = lib().orc_minvcg(C.byref(self.s), ptrs, _p(src), C.c_double(chi_norm), _p(sh), ns,
                              _p(rs), ms_type, _p(al), max_iter)
        return sols[:nvec], it, rs


    def matinv(self, src_full, guess_full=None, stop_rsd=1e-10, max_iter=5000):
        """DiracOp*::MatInv on a full vector (2 checkerboards; Wilson/DWF odd
        half first, Mobius even half first); returns (solution, iterations, true_res)."""
        src = np.ascontiguousarray(src_full, np.float64)
        assert src.size == 2 * self.n
        out = np.zeros(2 * self.n) if guess_full is None else np.array(guess_full, np.float64)
        tr = C.c_double(0)
        it = lib().orc_matinv(C.byref(self.s), _p(out), _p(src), C.c_double(stop_rsd), max_iter, C.byref(tr))
        return out, it, tr.value


    def dminus(self, x_full):
        """DiracOpMobius::Dminus on a full vector (4-D-even half first)."""
        x = np.ascontiguousarray(x_full, np.float64)
        assert self.action == 2 and x.size == 2 * self.n
        out = np.zeros(2 * self.n)
        rc = lib().orc_mobius_dminus(C.byref(self.s), _p(out), _p(x))
        assert rc == 0
        return out

    def zdminus(self, x_full):
        """DiracOpZMobius::Dminus on a full vector (odd half first), complex c_s."""
        x = np.ascontiguousarray(x_full, np.float64)
        assert self.action == 2 and x.size == 2 * self.n
        out = np.zeros(2 * self.n)
        rc = lib().orc_zmobius_dminus(C.byref(self.s), _p(out), _p(x))
        assert rc == 0
        return out

    def zmatinv(self, src_full, guess_full=None, stop_rsd=1e-10, max_iter=5000):
        """DiracOpZMobius::MatInv on a full vector (solve checkerboard first);
        returns (solution, iterations, true_res)."""
        src = np.ascontiguousarray(src_full, np.float64)
        assert self.action == 2 and src.size == 2 * self.n
        out = np.zeros(2 * self.n) if guess_full is None else np.array(guess_full, np.float64)
        tr = C.c_double(0)
        it = lib().orc_zmobius_matinv(C.byref(self.s), _p(out), _p(src), C.c_double(stop_rsd), max_iter,
                                      C.byref(tr))
        assert it >= 0
        return out, it, tr.value

    def zfmatinv(self, src_full, guess_full=None, dminus=0, stop_rsd=1e-10, max_iter=5000):
        """Fzmobius::FmatInv (f_zmobius.C:70-130): the source (Dminus of it for
        dminus = 1) times 2 kappa_b(s), then DiracOpZMobius::MatInv; dminus = -1
        returns Dminus(source) without a solve (iterations 0)."""
        if dminus == -1:
            return self.zdminus(src_full), 0, 0.0
        src = self.zdminus(src_full) if dminus == 1 else np.array(src_full, np.float64)
        assert lib().orc_zmobius_scale_2kb(C.byref(self.s), _p(src)) == 0
        return self.zmatinv(src, guess_full, stop_rsd, max_iter)

    def fmatinv(self, src_full, guess_full=None, dminus=0, stop_rsd=1e-10, max_iter=5000):
        """Lattice::FmatInv(..., dminus): Fmobius applies Dminus to the source
        before MatInv (f_mobius.C:45-117); the other actions ignore the flag."""
        src = self.dminus(src_full) if (dminus and self.action == 2) else src_full
        return self.matinv(src, guess_full, stop_rsd, max_iter)

    def minresext(self, phi, prev):
        """DiracOp::MinResExt: returns (psi, orthonormalised prev, MatPcDagMatPc of them, guess residual)."""
        deg = len(prev)
        v = [np.array(x, np.float64) for x in prev]
        vm = [np.zeros(self.n) for _ in range(deg)]
        psi = np.zeros(self.n)
        vp = (_dp * max(deg, 1))(*[_p(x) for x in v]) if deg else (_dp * 1)()
        vmp = (_dp * max(deg, 1))(*[_p(x) for x in vm]) if deg else (_dp * 1)()
        err = lib().orc_minresext(C.byref(self.s), _p(psi), _p(self._v(phi)), vp, vmp, deg)
        return psi, v, vm, err


def _seqsum(x: np.ndarray) -> float:
    return float(np.cumsum(x * x)[-1])


def _setup():
    L = lib()
    L.orc_dslash.restype = C.c_int
    L.orc_matpc.restype = C.c_int
    L.orc_matinv.restype = C.c_int
    L.orc_minresext.restype = C.c_double
    L.orc_mobius_dminus.restype = C.c_int
    L.orc_zmobius_dminus.restype = C.c_int
    L.orc_zmobius_matinv.restype = C.c_int
    L.orc_zmobius_scale_2kb.restype = C.c_int
    L.orc_mdagm.restype = C.c_int
    L.orc_invcg.restype = C.c_int
    L.orc_invcg.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_int, C.POINTER(C.c_double), _dp]
    L.orc_minvcg.restype = C.c_int
    L.orc_minvcg.argtypes = [C.c_void_p, C.POINTER(_dp), _dp, C.c_double, _dp, C.c_int, _dp, C.c_int,
                             _dp, C.c_int]


_setup()


def fermion_convert(v, dims, ls=1, order="wilson", inverse=False):
    """Lattice::Fconvert between CANONICAL and the checkerboarded orders, as a
    permutation of 24-real sites.  TEST INFRASTRUCTURE ONLY.

    CANONICAL: slice s (slowest), then site x + lx*(y + ly*(z + lz*t)).
    order "wilson": each slice first to [odd | even] 4-D halves
    (FcanonToWilson, lattice/convert/convert_func.C:429-495); for ls > 1 the
    5-D checkerboard of FdwfBase::Fconvert (convert.C:700-755): the first half
    holds the sites with x+y+z+t+s odd (slice by slice), the second half the
    others.
    order "4d_ee" (DWF_4D_EOPREC_EE, convert.C:793-830): the 4-D even half of
    every slice, then the 4-D odd half of every slice.
    inverse=True maps the checkerboarded order back to CANONICAL.
    """
    lx, ly, lz, lt = dims
    vol = lx * ly * lz * lt
    h = vol // 2
    t, z, y, x = np.meshgrid(np.arange(lt), np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    par = ((x + y + z + t) % 2).reshape(-1)                   # canonical site -> 4-D parity
    cbi = (x // 2 + (lx // 2) * (y + ly * (z + lz * t))).reshape(-1)
    dst = np.empty((ls, vol), np.int64)
    for s in range(ls):
        if order == "wilson" and ls > 1:
            half = ((par + s) % 2 == 0).astype(np.int64)     # 5-D odd sites first
        elif order == "wilson":
            half = (par == 0).astype(np.int64)               # 4-D odd sites first
        else:
            half = (par == 1).astype(np.int64)               # 4-D even sites first
        dst[s] = half * (ls * h) + s * h + cbi
    v = np.asarray(v, np.float64).reshape(ls * vol, 24)
    out = np.empty_like(v)
    if inverse:
        out[:] = v[dst.reshape(-1)]
    else:
        out[dst.reshape(-1)] = v
    return out.reshape(-1)
