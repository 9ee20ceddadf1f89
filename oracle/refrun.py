"""Runner for the compiled CPS reference (oracle/_ref/cpsref). TEST INFRASTRUCTURE ONLY.

Each call writes a request file, runs the reference executable in a fresh
process (CPS keeps its lattice in global singletons) and parses the response.
The wire format is documented in oracle/ref_harness.C.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CPSREF = os.path.join(HERE, "_ref", "cpsref")
# CPS built with the B200 bridge linked in (oracle/build_dropin.py)
CPSREF_B200 = os.path.join(HERE, "_ref", "cpsref_b200")

OP_DSLASH, OP_MATPC, OP_MDAGM, OP_INVCG, OP_MINVCG, OP_M5INV, OP_MOBIUS_D4, OP_BENCH, OP_MATINV, OP_FCONVERT, \
    OP_MINRESEXT, OP_DMINUS, OP_FMATINV, OP_FMATEVLINV = 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14
ACTIONS = {"wilson": 0, "dwf": 1, "mobius": 2, "zmobius": 3}


def available(binary=CPSREF) -> bool:
    return os.access(binary, os.X_OK)


def run(op, action, dims, gauge, vectors=(), ls=1, cb=0, dag=0, mass=0.1, m5=1.8, a5_inv=1.0,
        b=1.5, c=0.5, stop_rsd=1e-10, max_iter=5000, shifts=(), ms_type=0, pc_type=2,
        bc_t=0, extra=(), reps=0, threads=None, timeout=3600, order=0, direction=0, degree=0, dminus=0, zb=None, zc=None, binary=CPSREF, bridge_prec=(-1, -1)):
    """Run one reference operation; returns (iters, rpar[64], payload array).
    zMobius (action "zmobius") takes the complex per-slice coefficients zb, zc (ls each).
    binary: CPSREF, or CPSREF_B200 with bridge_prec the bridge's inner precisions
    (FmatEvlInv / FmatInv, FmatEvlMInv; -1 keeps its default)."""
    if not available(binary):
        raise RuntimeError(f"{os.path.basename(binary)} not built (oracle/build_ref.sh, oracle/build_dropin.py)")
    hdr = np.zeros(32, np.int64)
    par = np.zeros(32, np.float64)
    hdr[0] = op
    hdr[1] = ACTIONS[action] if isinstance(action, str) else action
    hdr[2:6] = dims
    hdr[6] = ls
    hdr[7] = cb
    hdr[8] = dag
    hdr[9] = max_iter
    hdr[10] = len(shifts)
    hdr[11] = ms_type
    hdr[12] = pc_type
    hdr[13] = bc_t
    hdr[14] = reps
    hdr[15] = order
    hdr[16] = direction
    hdr[17] = degree
    hdr[18] = dminus
    hdr[19], hdr[20] = bridge_prec
    par[0] = mass
    par[1] = m5
    par[2] = a5_inv
    par[3] = b
    par[4] = c
    par[5] = stop_rsd
    for i, s in enumerate(shifts):
        par[8 + i] = s
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as td:
        req = os.path.join(td, "req.bin")
        rsp = os.path.join(td, "rsp.bin")
        with open(req, "wb") as f:
            f.write(hdr.tobytes())
            f.write(par.tobytes())
            if hdr[1] == 3:
                for z in (zb, zc):
                    z = np.asarray(z, np.complex128)
                    assert z.size == ls
                    f.write(np.ascontiguousarray(np.stack([z.real, z.imag], 1).reshape(-1), np.float64).tobytes())
            f.write(np.ascontiguousarray(gauge, np.float64).tobytes())
            for v in vectors:
                f.write(np.ascontiguousarray(v, np.float64).tobytes())
            for v in extra:
                f.write(np.ascontiguousarray(v, np.float64).tobytes())
        p = subprocess.run([binary, req, rsp], capture_output=True, text=True, env=env,
                           timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"cpsref failed ({p.returncode}): {p.stderr[-2000:]}")
        raw = open(rsp, "rb").read()
    rhdr = np.frombuffer(raw[:64], np.int64)
    rpar = np.frombuffer(raw[64:64 + 512], np.float64)
    payload = np.frombuffer(raw[576:], np.float64).copy()
    return int(rhdr[0]), rpar.copy(), payload
