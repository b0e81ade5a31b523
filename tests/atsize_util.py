"""Compact summaries of a full-size state, for parity at the configs' sizes.

A 256^3 MHD state is 2.5 GB; a committed fixture holds instead, for every
array (the NVAR primitive and conserved variables and the face fields):

* one 8-byte BLAKE2b digest of each outermost plane's bytes (z-planes in
  3-D, y-rows in 2-D): equal digests on every plane mean a bit-identical
  state;
* per plane the sum, the sum of |x| and max |x| (size-independent checks of
  a state that is not bit-identical);
* the values on a strided lattice of cells and on the x-line through the
  grid centre, for relative L-infinity per variable.

Arrays are indexed ``[var, z, y, x]`` (cells) or ``[dir][z, y, x]`` (faces),
the layout of the reference dump and of ``Solver.download``.
"""
from __future__ import annotations

import hashlib

import numpy as np


def _planes(a: np.ndarray, ndim: int) -> np.ndarray:
    """View of one array (z, y, x) as a stack of outermost planes."""
    if ndim == 3:
        return a
    return a[0]            # 2-D: (1, ny, nx) -> rows along y


def plane_digests(a: np.ndarray, ndim: int) -> np.ndarray:
    pl = _planes(np.ascontiguousarray(a, dtype="<f8"), ndim)
    out = np.empty(pl.shape[0], np.uint64)
    for p in range(pl.shape[0]):
        h = hashlib.blake2b(np.ascontiguousarray(pl[p]).tobytes(), digest_size=8)
        out[p] = np.frombuffer(h.digest(), "<u8")[0]
    return out


def _stride(shape, ndim):
    nz, ny, nx = shape
    target = 16 if ndim == 3 else 64          # ~4096 sampled cells
    return tuple(max(1, n // target) for n in (nz, ny, nx))


def summarize(V: np.ndarray, U: np.ndarray, Bs, ndim: int) -> dict:
    """Summary arrays of one state (see the module docstring)."""
    arrays = [V[nv] for nv in range(V.shape[0])] + [U[nv] for nv in range(U.shape[0])]
    arrays += list(Bs)
    nz, ny, nx = V.shape[1:]
    sz, sy, sx = _stride((nz, ny, nx), ndim)
    oz, oy, ox = (sz // 3, sy // 3, sx // 3)
    out = {"digest": np.stack([plane_digests(a, ndim) for a in arrays])}
    sums, abss, maxs, samp, line = [], [], [], [], []
    for a in arrays:
        pl = _planes(a, ndim).reshape(_planes(a, ndim).shape[0], -1)
        sums.append(pl.sum(axis=1))
        abss.append(np.abs(pl).sum(axis=1))
        maxs.append(np.abs(pl).max(axis=1))
        samp.append(a[oz::sz, oy::sy, ox::sx].ravel())
        line.append(a[nz // 2, ny // 2, :].copy())
    out.update(psum=np.array(sums), pabs=np.array(abss), pmax=np.array(maxs),
               sample=np.array(samp), line=np.array(line))
    return out


def compare(got: dict, ref: dict, nvar: int) -> dict:
    """Per array: whether every plane is bit-identical, and the relative
    L-infinity difference on the sample and the centre line together."""
    narr = ref["digest"].shape[0]
    same = [bool(np.array_equal(got["digest"][a], ref["digest"][a])) for a in range(narr)]
    rel = []
    for a in range(narr):
        g = np.concatenate([got["sample"][a], got["line"][a]])
        r = np.concatenate([ref["sample"][a], ref["line"][a]])
        scale = np.abs(r).max()
        rel.append(float(np.abs(g - r).max() / scale) if scale > 0 else float(np.abs(g).max()))
    psum_rel = []
    for a in range(narr):
        scale = ref["pabs"][a].max()
        d = np.abs(got["psum"][a] - ref["psum"][a]).max()
        psum_rel.append(float(d / scale) if scale > 0 else float(d))
    return {"bitwise": same, "rel_linf": rel, "plane_sum_rel": psum_rel,
            "names": array_names(nvar, narr - 2 * nvar)}


def array_names(nvar: int, nface: int) -> list:
    return ([f"V{nv}" for nv in range(nvar)] + [f"U{nv}" for nv in range(nvar)]
            + [f"Bs{d}" for d in range(nface)])
