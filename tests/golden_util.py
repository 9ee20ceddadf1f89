"""Loads a golden fixture and re-creates its inputs from the stored seeds."""
import hashlib
import os

import numpy as np

from cps_public_b200 import fields

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).hexdigest()


def load(name):
    """Returns (record dict, gauge in CANONICAL order, source vector)."""
    rec = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    dims = tuple(int(d) for d in rec["dims"])
    ls = int(rec.get("ls", 1))
    u = fields.random_gauge(dims, float(rec["eps"]), int(rec["seed"]))
    src = fields.random_source(int(np.prod(dims)) // 2 * ls, int(rec["seed"]))
    assert sha(u) == str(rec["gauge_sha"]), "gauge generator drifted from the fixture"
    assert sha(src) == str(rec["src_sha"]), "source generator drifted from the fixture"
    return rec, u, src


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def load_matinv(name):
    """MatInv fixture: (record, gauge, full source, full initial guess)."""
    from tests.golden.make_golden import matinv_inputs
    rec = dict(np.load(os.path.join(GOLDEN, "matinv_" + name + ".npz")))
    dims = tuple(int(d) for d in rec["dims"])
    u = fields.random_gauge(dims, float(rec["eps"]), int(rec["seed"]))
    src, guess = matinv_inputs(rec)
    assert sha(u) == str(rec["gauge_sha"]), "gauge generator drifted from the fixture"
    assert sha(src) == str(rec["matinv_src_sha"]) and sha(guess) == str(rec["matinv_guess_sha"])
    return rec, u, src, guess


def load_dminus(name):
    """Dminus / FmatInv(dminus = 1) fixture: (record, gauge, full source, full initial guess)."""
    from tests.golden.make_golden import matinv_inputs
    rec = dict(np.load(os.path.join(GOLDEN, "dminus_" + name + ".npz")))
    dims = tuple(int(d) for d in rec["dims"])
    u = fields.random_gauge(dims, float(rec["eps"]), int(rec["seed"]))
    src, guess = matinv_inputs(rec)
    assert sha(u) == str(rec["gauge_sha"]), "gauge generator drifted from the fixture"
    assert sha(src) == str(rec["matinv_src_sha"]) and sha(guess) == str(rec["matinv_guess_sha"])
    return rec, u, src, guess
