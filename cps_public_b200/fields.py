"""Seeded synthetic gauge fields and sources, and CPS storage-order helpers.

Gauge links follow the benchmark recipe U = reunitarise(exp(i*eps*H)) with H a
Hermitian traceless 3x3 matrix built from complex Gaussian entries.  Random
numbers come from numpy's counter-based Philox generator keyed by the seed, so
a field is a pure function of (dims, eps, seed).

Storage orders (CPS, reference paths relative to cps_pp/):

* CANONICAL gauge (``Lattice::GaugeField()``): site ``x+lx*(y+ly*(z+lz*t))``,
  then the 4 links mu=x,y,z,t, each a row-major 3x3 complex matrix
  (src/util/lattice/convert/convert_func.C:397-405).
* WILSON gauge: even 4-D sites first, site index ``x/2 + lx/2*(y+ly*(z+lz*t))``
  within a parity, and each 3x3 matrix stored transposed, element (row,col) at
  ``r + 2*(row + 3*col)`` (convert_func.C:371-374, :403-405;
  d_op_wilson/noarch/wilson_dslash.C:54).
* Checkerboarded fermion: 24 reals per site, ``r + 2*(colour + 3*spin)``
  (wilson_dslash.C:60), sites in the same half-lattice order.  A 5-D vector is
  Ls consecutive 4-D checkerboard slices.
"""
from __future__ import annotations

import numpy as np


def _rng(seed: int, stream: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=[int(seed) & (2**64 - 1), int(stream)]))


def reunitarise(u: np.ndarray) -> np.ndarray:
    """Project (..., 3, 3) complex matrices onto SU(3) by Gram-Schmidt on rows.

    Row 0 is normalised, row 1 is orthogonalised against it and normalised,
    and row 2 is set to conj(row0 x row1), which fixes det = 1.
    """
    r0 = u[..., 0, :]
    r0 = r0 / np.linalg.norm(r0, axis=-1, keepdims=True)
    r1 = u[..., 1, :]
    r1 = r1 - np.sum(np.conj(r0) * r1, axis=-1, keepdims=True) * r0
    r1 = r1 / np.linalg.norm(r1, axis=-1, keepdims=True)
    r2 = np.conj(np.cross(r0, r1))
    return np.stack([r0, r1, r2], axis=-2)


def random_gauge(dims, eps: float, seed: int) -> np.ndarray:
    """Gauge field in CANONICAL order as a float64 array of shape (V*4*18,).

    dims = (lx, ly, lz, lt).  Each link is reunitarise(exp(i*eps*H)) with
    H = (A + A^dagger)/2 - tr/3, A having N(0,1) real and imaginary parts.
    """
    lx, ly, lz, lt = (int(d) for d in dims)
    n = lx * ly * lz * lt * 4
    g = _rng(seed, 1)
    a = g.standard_normal((n, 3, 3)) + 1j * g.standard_normal((n, 3, 3))
    h = 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))
    tr = np.trace(h, axis1=-2, axis2=-1).real / 3.0
    h = h - tr[:, None, None] * np.eye(3)[None]
    lam, vec = np.linalg.eigh(h)
    ph = np.exp(1j * eps * lam)
    u = np.einsum("nik,nk,njk->nij", vec, ph, np.conj(vec))
    u = reunitarise(u)
    out = np.empty((n, 3, 3, 2), dtype=np.float64)
    out[..., 0] = u.real
    out[..., 1] = u.imag
    return out.reshape(-1)


def random_source(nsites: int, seed: int, stream: int = 2) -> np.ndarray:
    """Checkerboard spinor field of ``nsites`` sites with N(0,1) real and
    imaginary parts, shape (nsites*24,), float64."""
    return _rng(seed, stream).standard_normal(nsites * 24)


def point_source(dims, ls: int, site, spin: int, colour: int, cb: int = 1,
                 five_d_parity: bool = True) -> np.ndarray:
    """Unit point source on one checkerboard, embedded in 5-D.

    The source sits at 4-D site ``site`` on the s-slices 0 and Ls-1 (chirality
    projected as in CPS's 4-D->5-D map, lattice/f_dwf_base/f_dwf_base.C:961:
    upper spins on s=0, lower spins on s=Ls-1).  Slices whose 4-D parity does
    not match the site get nothing.  For the 4-D-preconditioned (Mobius)
    layout pass five_d_parity=False.
    """
    lx, ly, lz, lt = dims
    x, y, z, t = site
    n4cb = lx * ly * lz * lt // 2
    v = np.zeros((ls, n4cb, 24))
    p4 = (x + y + z + t) % 2
    idx = x // 2 + (lx // 2) * (y + ly * (z + lz * t))
    for s in (0, ls - 1):
        slice_par = (s + cb) % 2 if five_d_parity else cb
        if slice_par != p4:
            continue
        if (spin < 2 and s == 0) or (spin >= 2 and s == ls - 1):
            v[s, idx, 2 * (colour + 3 * spin)] = 1.0
    return v.reshape(-1)


def canonical_to_wilson_gauge(u_can: np.ndarray, dims) -> np.ndarray:
    """CANONICAL -> WILSON gauge order (even sites first, links transposed)."""
    lx, ly, lz, lt = dims
    vol = lx * ly * lz * lt
    u = u_can.reshape(lt, lz, ly, lx, 4, 3, 3, 2)
    t, z, y, x = np.meshgrid(np.arange(lt), np.arange(lz), np.arange(ly), np.arange(lx),
                             indexing="ij")
    par = (x + y + z + t) % 2
    idx = x // 2 + (lx // 2) * (y + ly * (z + lz * t)) + (vol // 2) * par
    out = np.empty((vol, 4, 3, 3, 2))
    # transposed storage: out[..., col, row] = U[row, col]
    out[idx.reshape(-1)] = np.swapaxes(u.reshape(vol, 4, 3, 3, 2), 2, 3)
    return out.reshape(-1)


def site_parity_index(dims):
    """(parity, cb-index) of every canonical 4-D site, as two int arrays."""
    lx, ly, lz, lt = dims
    t, z, y, x = np.meshgrid(np.arange(lt), np.arange(lz), np.arange(ly), np.arange(lx),
                             indexing="ij")
    par = ((x + y + z + t) % 2).reshape(-1)
    idx = (x // 2 + (lx // 2) * (y + ly * (z + lz * t))).reshape(-1)
    return par, idx
