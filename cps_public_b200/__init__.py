"""cps_public_b200 -- B200-native CPS fermion-matrix hot path.

Python front end of libcpsb200.so, mirroring the CPS interfaces it replaces:

* ``Gauge``        resident gauge field (the gauge half of the DiracOp constructor)
* ``DiracOp``      Dslash / MatPc / MatPcDag / MatPcDagMatPc / InvCg / MInvCG for the
                   Wilson, DWF and Mobius actions (cps_pp/include/util/dirac_op.h)
* ``fmat_evl_inv`` / ``fmat_evl_minv`` / ``fmat_inv``  the Lattice::FmatEvlInv /
                   FmatEvlMInv / FmatInv entry points (cps_pp/include/util/lattice.h:942,976,1114)

All compute runs in the CUDA library; this module only marshals numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (DWF, F16, F32, F64, MOBIUS, MULTI, ORDER_CANONICAL, ORDER_WILSON, SINGLE,  # noqa: F401
                   WILSON, ZMOBIUS, CgArg, CpsbError, DiracParams, SolveResult, check, ptr)

_initialised = None


def init(device: int = 0) -> None:
    global _initialised
    lib = _lib.load()
    check(lib.cpsb_init(device), "cpsb_init")
    _initialised = device


def mem_info():
    lib = _lib.load()
    f, t = C.c_ulonglong(), C.c_ulonglong()
    check(lib.cpsb_mem_info(C.byref(f), C.byref(t)), "cpsb_mem_info")
    return f.value, t.value


class Gauge:
    """A gauge field resident on the device (CANONICAL or WILSON order input)."""

    def __init__(self, u: np.ndarray, dims, order: int = ORDER_CANONICAL, bc_t: int = 0):
        if _initialised is None:
            init(0)
        lib = _lib.load()
        self.dims = tuple(int(d) for d in dims)
        u = np.ascontiguousarray(u, np.float64)
        vol = int(np.prod(self.dims))
        if u.size != vol * 72:
            raise ValueError(f"gauge field has {u.size} reals, expected {vol * 72}")
        h = C.c_void_p()
        d = (C.c_int * 4)(*self.dims)
        check(lib.cpsb_gauge_load(C.byref(h), ptr(u), d, order, bc_t), "cpsb_gauge_load")
        self.h = h
        self.n4cb = vol // 2

    def free(self):
        if self.h:
            _lib.load().cpsb_gauge_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


ACTION_NAMES = {"wilson": WILSON, "dwf": DWF, "mobius": MOBIUS, "zmobius": ZMOBIUS}


class DiracOp:
    """Device fermion operator with the CPS DiracOp interface.

    ``DiracOp(gauge, 'dwf', mass=0.01, ls=16, m5=1.8)``; vectors are float64 numpy
    arrays in CPS checkerboard order (sites x 24).
    """

    def __init__(self, gauge: Gauge, action="wilson", mass=0.1, ls=1, m5=1.8, a5_inv=1.0, b=1.5, c=0.5,
                 pc_type=2, bs=None, cs=None):
        """zMobius ('zmobius') takes the complex per-slice coefficients bs, cs (ls each)."""
        self.gauge = gauge
        self.p = DiracParams()
        self.p.action = ACTION_NAMES[action] if isinstance(action, str) else int(action)
        self.p.ls = 1 if self.p.action == WILSON else int(ls)
        self.p.mass = mass
        self.p.m5 = m5
        self.p.a5_inv = a5_inv
        self.p.mobius_b = b
        self.p.mobius_c = c
        self.p.pc_type = pc_type
        if self.p.action == ZMOBIUS:
            if bs is None or cs is None or len(bs) != self.p.ls or len(cs) != self.p.ls:
                raise ValueError("zmobius needs bs and cs with ls entries each")
            # (re, im) pairs, kept alive with the operator
            self._zb = np.ascontiguousarray(np.stack([np.real(bs), np.imag(bs)], 1).reshape(-1), np.float64)
            self._zc = np.ascontiguousarray(np.stack([np.real(cs), np.imag(cs)], 1).reshape(-1), np.float64)
            self.p.zmobius_b = ptr(self._zb)
            self.p.zmobius_c = ptr(self._zc)
        self.n = gauge.n4cb * self.p.ls * 24

    def _v(self, x):
        x = np.ascontiguousarray(x, np.float64)
        if x.size != self.n:
            raise ValueError(f"vector has {x.size} reals, expected {self.n}")
        return x

    def Dslash(self, x, cb, dag):
        out = np.empty(self.n)
        check(_lib.load().cpsb_dslash(self.gauge.h, C.byref(self.p), ptr(out), ptr(self._v(x)), cb, dag),
              "cpsb_dslash")
        return out

    def MatPc(self, x):
        out = np.empty(self.n)
        check(_lib.load().cpsb_matpc(self.gauge.h, C.byref(self.p), ptr(out), ptr(self._v(x)), 0), "cpsb_matpc")
        return out

    def MatPcDag(self, x):
        out = np.empty(self.n)
        check(_lib.load().cpsb_matpc(self.gauge.h, C.byref(self.p), ptr(out), ptr(self._v(x)), 1), "cpsb_matpc")
        return out

    def MatPcDagMatPc(self, x):
        """Returns (M^dag M x, |M x|^2)."""
        out = np.empty(self.n)
        dot = C.c_double()
        check(_lib.load().cpsb_mdagm(self.gauge.h, C.byref(self.p), ptr(out), ptr(self._v(x)), C.byref(dot)),
              "cpsb_mdagm")
        return out, dot.value

    def DslashPrec(self, x, cb, dag, precision):
        """Dslash with fields and links stored in `precision` (F64, F32 or F16)."""
        out = np.empty(self.n)
        check(_lib.load().cpsb_dslash_ex(self.gauge.h, C.byref(self.p), precision, ptr(out), ptr(self._v(x)),
                                         cb, dag), "cpsb_dslash_ex")
        return out

    def MatPcDagMatPcPrec(self, x, precision):
        """MatPcDagMatPc with fields and links stored in `precision`; returns (out, |M x|^2)."""
        out = np.empty(self.n)
        dot = C.c_double()
        check(_lib.load().cpsb_mdagm_ex(self.gauge.h, C.byref(self.p), precision, ptr(out), ptr(self._v(x)),
                                        C.byref(dot)), "cpsb_mdagm_ex")
        return out, dot.value

    def InvCg(self, src, stop_rsd=1e-10, max_num_iter=5000, precision=F64, guess=None, reliable_delta=0.1,
              batch=0):
        """Solves M^dag M x = src; returns (x, SolveResult)."""
        x = np.zeros(self.n) if guess is None else self._v(guess).copy()
        a = CgArg(stop_rsd, max_num_iter, precision, reliable_delta, batch)
        r = SolveResult()
        rc = check(_lib.load().cpsb_invcg(self.gauge.h, C.byref(self.p), C.byref(a), ptr(x),
                                          ptr(self._v(src)), C.byref(r)), "cpsb_invcg")
        r.rc = rc
        return x, r

    def InvCgMulti(self, srcs, stop_rsd=1e-10, max_num_iter=5000, precision=F64, reliable_delta=0.1, batch=0):
        n = len(srcs)
        xs = [np.zeros(self.n) for _ in range(n)]
        bs = [self._v(s) for s in srcs]
        xp = (_lib._dp * n)(*[ptr(x) for x in xs])
        bp = (_lib._dp * n)(*[ptr(b) for b in bs])
        a = CgArg(stop_rsd, max_num_iter, precision, reliable_delta, batch)
        res = (SolveResult * n)()
        check(_lib.load().cpsb_invcg_multi(self.gauge.h, C.byref(self.p), C.byref(a), n, xp, bp, res),
              "cpsb_invcg_multi")
        return xs, list(res)

    def MatInv(self, src_full, guess_full=None, stop_rsd=1e-10, max_num_iter=5000, precision=F64,
               reliable_delta=0.1, batch=0):
        """Full-lattice solve M out = in (DiracOp*::MatInv); vectors hold both
        checkerboards (Wilson/DWF odd half first, Mobius even half first).
        Returns (out, SolveResult of the preconditioned CG)."""
        src = np.ascontiguousarray(src_full, np.float64)
        if src.size != 2 * self.n:
            raise ValueError(f"full vector has {src.size} reals, expected {2 * self.n}")
        out = np.zeros(2 * self.n) if guess_full is None else np.array(guess_full, np.float64)
        a = CgArg(stop_rsd, max_num_iter, precision, reliable_delta, batch)
        r = SolveResult()
        rc = check(_lib.load().cpsb_matinv(self.gauge.h, C.byref(self.p), C.byref(a), ptr(out), ptr(src),
                                           C.byref(r)), "cpsb_matinv")
        r.rc = rc
        return out, r

    def Dminus(self, x_full):
        """DiracOpMobius::Dminus on a full vector (4-D-even half first), or for
        zMobius DiracOpZMobius::Dminus (odd half first, complex c_s)."""
        x = np.ascontiguousarray(x_full, np.float64)
        if x.size != 2 * self.n:
            raise ValueError(f"full vector has {x.size} reals, expected {2 * self.n}")
        out = np.empty(2 * self.n)
        check(_lib.load().cpsb_dminus(self.gauge.h, C.byref(self.p), ptr(out), ptr(x)), "cpsb_dminus")
        return out

    def FmatInv(self, src_full, guess_full=None, dminus=0, stop_rsd=1e-10, max_num_iter=5000, precision=F64,
                reliable_delta=0.1, batch=0):
        """Lattice::FmatInv(..., dminus): for Mobius with dminus the source is
        replaced by Dminus(source) before MatInv; other actions ignore dminus."""
        src = np.ascontiguousarray(src_full, np.float64)
        if src.size != 2 * self.n:
            raise ValueError(f"full vector has {src.size} reals, expected {2 * self.n}")
        out = np.zeros(2 * self.n) if guess_full is None else np.array(guess_full, np.float64)
        a = CgArg(stop_rsd, max_num_iter, precision, reliable_delta, batch)
        r = SolveResult()
        rc = check(_lib.load().cpsb_fmatinv(self.gauge.h, C.byref(self.p), C.byref(a), ptr(out), ptr(src),
                                            int(dminus), C.byref(r)), "cpsb_fmatinv")
        r.rc = rc
        return out, r

    def MinResExt(self, phi, prev):
        """DiracOp::MinResExt: chronological guess from previous solutions.
        Returns (psi, orthonormalised prev, MatPcDagMatPc of them, |phi - A psi|/|phi|)."""
        deg = len(prev)
        v = [np.array(self._v(x), np.float64) for x in prev]
        vm = [np.zeros(self.n) for _ in range(deg)]
        psi = np.zeros(self.n)
        vp = (_lib._dp * max(deg, 1))(*[ptr(x) for x in v])
        vmp = (_lib._dp * max(deg, 1))(*[ptr(x) for x in vm])
        res = C.c_double()
        check(_lib.load().cpsb_minresext(self.gauge.h, C.byref(self.p), ptr(psi), ptr(self._v(phi)), vp, vmp, deg,
                                         C.byref(res)), "cpsb_minresext")
        return psi, v, vm, res.value

    def MInvCG(self, src, shifts, rsd, ms_type=MULTI, alpha=None, max_num_iter=5000, precision=F64):
        ns = len(shifts)
        nvec = 1 if ms_type == SINGLE else ns
        xs = [np.zeros(self.n) for _ in range(nvec)]
        xp = (_lib._dp * nvec)(*[ptr(x) for x in xs])
        rs = np.array(rsd, np.float64)
        sh = np.array(shifts, np.float64)
        al = np.ones(ns) if alpha is None else np.array(alpha, np.float64)
        a = CgArg(float(np.min(rs)), max_num_iter, precision, 0.1, 0)
        r = SolveResult()
        rc = check(_lib.load().cpsb_minvcg(self.gauge.h, C.byref(self.p), C.byref(a), xp, ptr(self._v(src)),
                                           ptr(sh), ns, ptr(rs), ms_type, ptr(al), C.byref(r)), "cpsb_minvcg")
        r.rc = rc
        return xs, r, rs

    def MInvCGMulti(self, srcs, shifts, rsd, ms_type=MULTI, alpha=None, max_num_iter=5000, precision=F64):
        """Batched MInvCG over the source vectors srcs (the pseudofermions of one
        RHMC evaluation), sharing the shifts; rsd: per shift, or per vector and
        shift (nvec x nshift).  Returns (xs[q][s], results[q], rsd[q][s])."""
        nvec, ns = len(srcs), len(shifts)
        nsol = 1 if ms_type == SINGLE else ns
        xs = [[np.zeros(self.n) for _ in range(nsol)] for _ in range(nvec)]
        xp = (_lib._dp * (nvec * nsol))(*[ptr(x) for row in xs for x in row])
        bs = [self._v(b) for b in srcs]
        bp = (_lib._dp * nvec)(*[ptr(b) for b in bs])
        rs = np.ascontiguousarray(np.broadcast_to(np.asarray(rsd, np.float64), (nvec, ns)), np.float64)
        sh = np.array(shifts, np.float64)
        al = np.ones(ns) if alpha is None else np.array(alpha, np.float64)
        a = CgArg(float(np.min(rs)), max_num_iter, precision, 0.1, 0)
        res = (SolveResult * nvec)()
        rc = check(_lib.load().cpsb_minvcg_multi(self.gauge.h, C.byref(self.p), C.byref(a), nvec, xp, bp, ptr(sh), ns,
                                                 ptr(rs), ms_type, ptr(al), res), "cpsb_minvcg_multi")
        out = list(res)
        for r in out:
            r.rc = rc
        return xs, out, rs


def fmat_evl_inv(op: DiracOp, f_in, cg_arg: dict, f_out=None):
    """Lattice::FmatEvlInv: returns (iterations, f_out, true_res)."""
    x, r = op.InvCg(f_in, cg_arg.get("stop_rsd", 1e-10), cg_arg.get("max_num_iter", 5000),
                    cg_arg.get("precision", F64), guess=f_out)
    return r.iters, x, r.true_rsd


def fmat_inv(op: DiracOp, f_in, cg_arg: dict, f_out=None, dminus=0):
    """Lattice::FmatInv (lattice.h:1114, dminus form :1127): full-lattice solve;
    returns (iterations, f_out, true_res)."""
    out, r = op.FmatInv(f_in, f_out, dminus, cg_arg.get("stop_rsd", 1e-10), cg_arg.get("max_num_iter", 5000),
                        cg_arg.get("precision", F64))
    return r.iters, out, r.true_rsd


def fmat_evl_minv(op: DiracOp, f_in, shifts, cg_args, ms_type=MULTI, alpha=None):
    """Lattice::FmatEvlMInv: returns (iterations, solutions, per-shift residuals)."""
    rsd = [a.get("stop_rsd", 1e-10) for a in cg_args]
    xs, r, rs = op.MInvCG(f_in, shifts, rsd, ms_type, alpha, cg_args[0].get("max_num_iter", 5000),
                          cg_args[0].get("precision", F64))
    return r.iters, xs, rs


class Server:
    """Request loop for concurrent solves (cpsb_serve_*).

    ``srv = Server(slots=4)``; ``rid = srv.submit(op, [b0, b1], stop_rsd=1e-10, precision=F16)``;
    ``xs, results, latency_ms = srv.wait(rid)``.  Admission is by the server's HBM
    budget (``hbm_fraction`` of the free device memory, capped at ``hbm_bytes``).
    """

    def __init__(self, slots: int = 4, hbm_fraction: float = 0.9, hbm_bytes: int = 0):
        if _initialised is None:
            init(0)
        h = C.c_void_p()
        check(_lib.load().cpsb_serve_create(C.byref(h), slots, hbm_fraction, hbm_bytes), "cpsb_serve_create")
        self.h = h
        self._live = {}

    def submit(self, op: DiracOp, srcs, stop_rsd=1e-10, max_num_iter=5000, precision=F64, guesses=None,
               reliable_delta=0.1, batch=0) -> int:
        bs = [op._v(s) for s in srcs]
        xs = [np.zeros(op.n) if guesses is None else op._v(g).copy() for g in (guesses or [None] * len(bs))]
        a = CgArg(stop_rsd, max_num_iter, precision, reliable_delta, batch)
        xp = (_lib._dp * len(xs))(*[ptr(x) for x in xs])
        bp = (_lib._dp * len(bs))(*[ptr(b) for b in bs])
        rid = C.c_ulonglong()
        check(_lib.load().cpsb_serve_submit(self.h, op.gauge.h, C.byref(op.p), C.byref(a), len(bs), xp, bp,
                                            C.byref(rid)), "cpsb_serve_submit")
        self._live[rid.value] = (xs, bs, xp, bp, op)  # keep the buffers alive until wait()
        return rid.value

    def submit_minvcg(self, op: DiracOp, src, shifts, rsd, ms_type=MULTI, alpha=None, max_num_iter=5000,
                      precision=F64) -> int:
        """Queues a multishift solve (DiracOp::MInvCG); collect it with wait_minvcg."""
        ns = len(shifts)
        nvec = 1 if ms_type == SINGLE else ns
        xs = [np.zeros(op.n) for _ in range(nvec)]
        b = op._v(src)
        rs = np.array(rsd, np.float64)
        sh = np.array(shifts, np.float64)
        al = np.ones(ns) if alpha is None else np.array(alpha, np.float64)
        a = CgArg(float(np.min(rs)), max_num_iter, precision, 0.1, 0)
        xp = (_lib._dp * nvec)(*[ptr(x) for x in xs])
        rid = C.c_ulonglong()
        check(_lib.load().cpsb_serve_submit_minvcg(self.h, op.gauge.h, C.byref(op.p), C.byref(a), xp, ptr(b), ptr(sh),
                                                   ns, ptr(rs), ms_type, ptr(al), C.byref(rid)),
              "cpsb_serve_submit_minvcg")
        self._live[rid.value] = (xs, b, xp, rs, sh, al, op)
        return rid.value

    def wait_minvcg(self, rid: int):
        """Returns (solutions, SolveResult, per-shift residuals, latency in ms)."""
        xs, rs = self._live[rid][0], self._live[rid][3]
        res = (SolveResult * 1)()
        lat = C.c_double()
        rc = _lib.load().cpsb_serve_wait(self.h, rid, res, C.byref(lat))
        self._live.pop(rid, None)
        check(rc, "cpsb_serve_wait")
        return xs, res[0], rs, lat.value

    def done(self, rid: int) -> bool:
        d = C.c_int()
        check(_lib.load().cpsb_serve_poll(self.h, rid, C.byref(d)), "cpsb_serve_poll")
        return bool(d.value)

    def wait(self, rid: int):
        """Returns (solutions, [SolveResult per RHS], latency in ms); raises on error."""
        xs = self._live[rid][0]
        res = (SolveResult * len(xs))()
        lat = C.c_double()
        rc = _lib.load().cpsb_serve_wait(self.h, rid, res, C.byref(lat))
        self._live.pop(rid, None)
        check(rc, "cpsb_serve_wait")
        return xs, list(res), lat.value

    def stats(self) -> dict:
        st = _lib.ServeStats()
        check(_lib.load().cpsb_serve_stats(self.h, C.byref(st)), "cpsb_serve_stats")
        return st.as_dict()

    def close(self):
        if self.h:
            _lib.load().cpsb_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
