"""Seeded synthetic initial conditions for the Godunov-step workloads.

The reference ships no benchmark data; its test problems build initial
conditions in a user ``Init``/``InitDomain`` pair (e.g.
``Test_Problems/MHD/Orszag_Tang/init.cpp:60-154``).  These generators stand in
for that with random Fourier-mode fields (integer wave vectors with
``0 < |k| <= kmax``, uniform amplitudes and phases) evaluated exactly at cell
centres, faces or edges by a separable complex contraction.

Every generator returns a :class:`PrimState`: primitive cell variables in the
structure-of-arrays layout ``V[nv, k, j, i]`` (i fastest) and the face-normal
magnetic field on the left faces of each cell (``Bs[d][k, j, i]`` is the field
at ``x_d = i_d - 1/2``), which is the layout of ``Data::Vc``/``Data::Vs``
interiors in the reference (``Src/Array.hpp:476-479``,
``Src/boundary.cpp:30-45``).  Cell-centred field components along active
directions are the face averages ``0.5*(Bs(i) + Bs(i+1))``, the same formula
the reference applies at start-up (``Src/MHD/CT/ct_field_average.cpp:175-178``).
"""
from __future__ import annotations

import dataclasses
import struct

import numpy as np

# Variable indices of the MHD/RMHD modules (Src/MHD/mhd.hpp:21-33).
RHO, VX1, VX2, VX3, BX1, BX2, BX3, PRS = range(8)
# HD module (Src/HD/hd.hpp:21-34): RHO, MX1..3, ENG.
HD_PRS = 4

PHYS_HD, PHYS_MHD, PHYS_RMHD = 0, 1, 2
PHYS_NAMES = {PHYS_HD: "HD", PHYS_MHD: "MHD", PHYS_RMHD: "RMHD"}


@dataclasses.dataclass
class PrimState:
    physics: int
    ndim: int
    shape: tuple          # (nx, ny, nz); nz == 1 in 2-D
    gamma: float
    V: np.ndarray         # (nvar, nz, ny, nx) float64
    Bs: list              # ndim arrays (nz, ny, nx) float64 (MHD/RMHD); [] for HD
    xbeg: tuple = (0.0, 0.0, 0.0)
    xend: tuple = (1.0, 1.0, 1.0)

    @property
    def nvar(self) -> int:
        return self.V.shape[0]

    @property
    def ncells(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    def copy(self) -> "PrimState":
        return PrimState(self.physics, self.ndim, tuple(self.shape), self.gamma,
                         self.V.copy(), [b.copy() for b in self.Bs],
                         tuple(self.xbeg), tuple(self.xend))


# ---------------------------------------------------------------------------
# Random Fourier modes
# ---------------------------------------------------------------------------

def _kvectors(ndim: int, kmax: int) -> np.ndarray:
    r = np.arange(-kmax, kmax + 1)
    grids = np.meshgrid(*([r] * ndim), indexing="ij")
    k = np.stack([g.ravel() for g in grids], axis=1)
    k2 = (k * k).sum(axis=1)
    return k[(k2 > 0) & (k2 <= kmax * kmax)]


class ModeField:
    """Sum of cosines ``sum_k a_k cos(2 pi k.x + phi_k)`` on the unit box."""

    def __init__(self, rng: np.random.Generator, ndim: int, kmax: int = 4):
        self.ndim = ndim
        self.kmax = kmax
        self.k = _kvectors(ndim, kmax)
        self.amp = rng.uniform(0.0, 1.0, size=len(self.k))
        self.phase = rng.uniform(0.0, 2.0 * np.pi, size=len(self.k))

    def _coeff(self, deriv):
        c = 0.5 * self.amp * np.exp(1j * self.phase)
        if deriv is not None:
            c = c * (2j * np.pi * self.k[:, deriv])
        return c

    def evaluate(self, shape, shift, deriv=None) -> np.ndarray:
        """Field (or its derivative along ``deriv``) at ``x_d = (i_d + shift_d)/n_d``.

        Returns an array shaped ``(nz, ny, nx)`` (``(1, ny, nx)`` in 2-D).
        """
        kmax = self.kmax
        nk = 2 * kmax + 1
        coeff = self._coeff(deriv)
        dims = list(shape[: self.ndim])
        spec = np.zeros([nk] * self.ndim, dtype=np.complex128)
        idx = tuple((self.k[:, d] + kmax) for d in range(self.ndim))
        np.add.at(spec, idx, coeff)
        # phase factors e^{2 pi i k x} per direction, x = (i + s)/n
        ph = []
        for d in range(self.ndim):
            x = (np.arange(dims[d]) + shift[d]) / dims[d]
            kk = np.arange(-kmax, kmax + 1)
            ph.append(np.exp(2j * np.pi * np.outer(kk, x)))   # (nk, n_d)
        if self.ndim == 2:
            # spec[kx, ky]
            t = np.einsum("ab,ai->bi", spec, ph[0])          # (ky, nx)
            f = np.einsum("bi,bj->ji", t, ph[1])             # (ny, nx)
            out = 2.0 * f.real
            return out[None, :, :]
        t = np.einsum("abc,ai->bci", spec, ph[0])             # (ky, kz, nx)
        t = np.einsum("bci,bj->cji", t, ph[1])                # (kz, ny, nx)
        f = np.einsum("cji,ck->kji", t, ph[2])                # (nz, ny, nx)
        return 2.0 * f.real


def _face_average(Bs: np.ndarray, axis: int) -> np.ndarray:
    # 0.5*(B(i) + B(i+1)) with periodic wrap; axis given in (k, j, i) order
    return 0.5 * (Bs + np.roll(Bs, -1, axis=axis))


_AXIS = {0: 2, 1: 1, 2: 0}   # direction -> numpy axis of (nz, ny, nx)


def _shape3(n, ndim):
    if ndim == 2:
        return (int(n[0]), int(n[1]), 1)
    return (int(n[0]), int(n[1]), int(n[2]))


def _curl_face_B_2d(Az_nodes: np.ndarray, dx: float, dy: float):
    """Face field from a corner vector potential A_z(i-1/2, j-1/2).

    Bx(i-1/2, j) = (Az(i-1/2, j+1/2) - Az(i-1/2, j-1/2))/dy
    By(i, j-1/2) = -(Az(i+1/2, j-1/2) - Az(i-1/2, j-1/2))/dx
    (the discrete curl of ``Src/vector_curl.cpp`` on a Cartesian grid).
    """
    Az = Az_nodes[0]
    Bx = (np.roll(Az, -1, axis=0) - Az) / dy
    By = -(np.roll(Az, -1, axis=1) - Az) / dx
    return Bx[None], By[None]


def _curl_face_B_3d(A, dx, dy, dz):
    """Face field from edge vector potential components.

    A[0] = Ax at (i, j-1/2, k-1/2); A[1] = Ay at (i-1/2, j, k-1/2);
    A[2] = Az at (i-1/2, j-1/2, k).  Arrays are (nz, ny, nx).
    """
    Ax, Ay, Az = A
    r = lambda a, ax: np.roll(a, -1, axis=ax)
    Bx = (r(Az, 1) - Az) / dy - (r(Ay, 0) - Ay) / dz
    By = (r(Ax, 0) - Ax) / dz - (r(Az, 2) - Az) / dx
    Bz = (r(Ay, 2) - Ay) / dx - (r(Ax, 1) - Ax) / dy
    return Bx, By, Bz


# ---------------------------------------------------------------------------
# Workload generators
# ---------------------------------------------------------------------------

def mhd2d_turbulence(n=(256, 256), seed=0, gamma=5.0 / 3.0, amp_rho=0.2,
                     mach=1.0, beta=1.0) -> PrimState:
    """2-D ideal MHD on [0,1]^2, periodic.

    rho = 1 + amp_rho * f/max|f| (f a random |k|<=4 mode sum), p = 1,
    velocity from a random stream function scaled to rms Mach ``mach``,
    face B = discrete curl of a random corner A_z scaled to plasma beta.
    """
    rng = np.random.default_rng(seed)
    nx, ny, nz = _shape3(n, 2)
    shp = (nx, ny, nz)
    dx, dy = 1.0 / nx, 1.0 / ny
    frho, fpsi, faz = ModeField(rng, 2), ModeField(rng, 2), ModeField(rng, 2)
    f = frho.evaluate(shp, (0.5, 0.5))
    rho = 1.0 + amp_rho * f / np.abs(f).max()
    prs = np.ones_like(rho)
    vx = fpsi.evaluate(shp, (0.5, 0.5), deriv=1)
    vy = -fpsi.evaluate(shp, (0.5, 0.5), deriv=0)
    cs2 = gamma * prs / rho
    m = np.sqrt(np.mean((vx * vx + vy * vy) / cs2))
    vx *= mach / m
    vy *= mach / m
    Az = faz.evaluate(shp, (0.0, 0.0))
    Bx, By = _curl_face_B_2d(Az, dx, dy)
    b2 = np.mean(_face_average(Bx, 2) ** 2 + _face_average(By, 1) ** 2)
    s = np.sqrt(2.0 * prs.mean() / beta / b2)
    Bx, By = Bx * s, By * s
    V = np.zeros((8, nz, ny, nx))
    V[RHO], V[VX1], V[VX2], V[PRS] = rho, vx, vy, prs
    V[BX1] = _face_average(Bx, 2)
    V[BX2] = _face_average(By, 1)
    return PrimState(PHYS_MHD, 2, shp, gamma, V, [Bx, By])


def mhd3d_blast(n=(256, 256, 256), seed=0, gamma=5.0 / 3.0, p_amb=0.1,
                p_in=10.0, radius=0.1, beta=0.1, v_rms=0.1) -> PrimState:
    """3-D ideal MHD blast on [0,1]^3, periodic.

    rho = 1, p = p_amb with p = p_in inside a centred sphere of ``radius``;
    uniform B of strength sqrt(2 p_amb/beta) along a seeded unit vector;
    divergence-free random velocity (curl of a random vector potential with
    |k| <= 4) at rms ``v_rms``.
    """
    rng = np.random.default_rng(seed)
    nx, ny, nz = _shape3(n, 3)
    shp = (nx, ny, nz)
    u = rng.normal(size=3)
    u /= np.linalg.norm(u)
    psi = [ModeField(rng, 3) for _ in range(3)]
    c = (0.5, 0.5, 0.5)
    # v = curl(psi), analytic at cell centres
    d = lambda a, ax: psi[a].evaluate(shp, c, deriv=ax)
    vx = d(2, 1) - d(1, 2)
    vy = d(0, 2) - d(2, 0)
    vz = d(1, 0) - d(0, 1)
    s = v_rms / np.sqrt(np.mean(vx * vx + vy * vy + vz * vz))
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    r2 = ((x[None, None, :] - 0.5) ** 2 + (y[None, :, None] - 0.5) ** 2
          + (z[:, None, None] - 0.5) ** 2)
    prs = np.where(r2 < radius * radius, p_in, p_amb)
    B0 = np.sqrt(2.0 * p_amb / beta)
    V = np.zeros((8, nz, ny, nx))
    V[RHO] = 1.0
    V[VX1], V[VX2], V[VX3] = vx * s, vy * s, vz * s
    V[PRS] = prs
    Bs = [np.full((nz, ny, nx), B0 * u[dd]) for dd in range(3)]
    for dd in range(3):
        V[BX1 + dd] = _face_average(Bs[dd], _AXIS[dd])
    return PrimState(PHYS_MHD, 3, shp, gamma, V, Bs)


def mhd3d_turbulence(n=(32, 32, 32), seed=0, gamma=5.0 / 3.0, amp_rho=0.2,
                     mach=1.0, beta=1.0) -> PrimState:
    """3-D analogue of :func:`mhd2d_turbulence` (random A at cell edges)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = _shape3(n, 3)
    shp = (nx, ny, nz)
    frho = ModeField(rng, 3)
    psi = [ModeField(rng, 3) for _ in range(3)]
    fa = [ModeField(rng, 3) for _ in range(3)]
    c = (0.5, 0.5, 0.5)
    f = frho.evaluate(shp, c)
    rho = 1.0 + amp_rho * f / np.abs(f).max()
    prs = np.ones_like(rho)
    d = lambda a, ax: psi[a].evaluate(shp, c, deriv=ax)
    vx, vy, vz = d(2, 1) - d(1, 2), d(0, 2) - d(2, 0), d(1, 0) - d(0, 1)
    cs2 = gamma * prs / rho
    m = np.sqrt(np.mean((vx * vx + vy * vy + vz * vz) / cs2))
    A = [fa[0].evaluate(shp, (0.5, 0.0, 0.0)),
         fa[1].evaluate(shp, (0.0, 0.5, 0.0)),
         fa[2].evaluate(shp, (0.0, 0.0, 0.5))]
    Bs = list(_curl_face_B_3d(A, 1.0 / nx, 1.0 / ny, 1.0 / nz))
    bc = [_face_average(Bs[dd], _AXIS[dd]) for dd in range(3)]
    b2 = np.mean(bc[0] ** 2 + bc[1] ** 2 + bc[2] ** 2)
    sb = np.sqrt(2.0 * prs.mean() / beta / b2)
    Bs = [b * sb for b in Bs]
    V = np.zeros((8, nz, ny, nx))
    V[RHO], V[PRS] = rho, prs
    V[VX1], V[VX2], V[VX3] = vx * mach / m, vy * mach / m, vz * mach / m
    for dd in range(3):
        V[BX1 + dd] = _face_average(Bs[dd], _AXIS[dd])
    return PrimState(PHYS_MHD, 3, shp, gamma, V, Bs)


def hd_turbulence(n=(64, 64), seed=0, gamma=5.0 / 3.0, amp_rho=0.2,
                  mach=1.0) -> PrimState:
    """Hydrodynamics (NVAR=5: rho, vx, vy, vz, p) random flow, 2-D or 3-D."""
    ndim = len(n)
    rng = np.random.default_rng(seed)
    shp = _shape3(n, ndim)
    nx, ny, nz = shp
    c = (0.5,) * ndim
    f = ModeField(rng, ndim).evaluate(shp, c)
    rho = 1.0 + amp_rho * f / np.abs(f).max()
    prs = np.ones_like(rho)
    V = np.zeros((5, nz, ny, nx))
    if ndim == 2:
        psi = ModeField(rng, 2)
        vx = psi.evaluate(shp, c, deriv=1)
        vy = -psi.evaluate(shp, c, deriv=0)
        vz = np.zeros_like(vx)
    else:
        psi = [ModeField(rng, 3) for _ in range(3)]
        d = lambda a, ax: psi[a].evaluate(shp, c, deriv=ax)
        vx, vy, vz = d(2, 1) - d(1, 2), d(0, 2) - d(2, 0), d(1, 0) - d(0, 1)
    cs2 = gamma * prs / rho
    m = np.sqrt(np.mean((vx * vx + vy * vy + vz * vz) / cs2))
    V[0], V[1], V[2], V[3], V[4] = rho, vx * mach / m, vy * mach / m, vz * mach / m, prs
    return PrimState(PHYS_HD, ndim, shp, gamma, V, [])


def rmhd3d_turbulence(n=(192, 192, 192), seed=0, gamma=4.0 / 3.0,
                      amp_rho=0.5, p0=0.1, lorentz_max=10.0,
                      sigma=1.0, cone=None) -> PrimState:
    """3-D special-relativistic MHD, periodic.

    rho = 1 + amp_rho * f/max|f|, p = p0; the velocity direction comes from a
    random |k|<=4 field and its magnitude is remapped pointwise so that the
    Lorentz factor is log-uniform in [1, lorentz_max] (rank mapping of |v|),
    its direction that of the random field plus ``cone`` times its mean norm
    along a seeded bulk direction;
    B is the discrete curl of a random edge vector potential scaled to
    magnetisation sigma = <B^2>/<rho h> (h = 1 + gamma/(gamma-1) p/rho).
    """
    rng = np.random.default_rng(seed)
    shp = _shape3(n, 3)
    nx, ny, nz = shp
    c = (0.5, 0.5, 0.5)
    f = ModeField(rng, 3).evaluate(shp, c)
    rho = 1.0 + amp_rho * f / np.abs(f).max()
    prs = np.full_like(rho, p0)
    w = [ModeField(rng, 3).evaluate(shp, c) for _ in range(3)]
    mag = np.sqrt(w[0] ** 2 + w[1] ** 2 + w[2] ** 2)
    # rank-map |w| onto a log-uniform Lorentz factor distribution
    order = np.argsort(mag, axis=None)
    q = np.empty(mag.size)
    q[order] = (np.arange(mag.size) + 0.5) / mag.size
    lor = np.exp(q * np.log(lorentz_max)).reshape(mag.shape)
    vabs = np.sqrt(1.0 - 1.0 / (lor * lor))
    # directions inside a cone around a seeded bulk direction (random
    # directions at Gamma ~ 10 make head-on collisions with relative Lorentz
    # factors of hundreds, which the reference scheme itself cannot advance)
    e = rng.normal(size=3)
    e /= np.linalg.norm(e)
    if cone is None:          # all velocities along the bulk direction
        unit = [np.full(mag.shape, e[q]) for q in range(3)]
    else:
        d = [w[q] + cone * mag.mean() * e[q] for q in range(3)]
        dmag = np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
        unit = [dq / np.maximum(dmag, 1e-300) for dq in d]
    fa = [ModeField(rng, 3) for _ in range(3)]
    A = [fa[0].evaluate(shp, (0.5, 0.0, 0.0)),
         fa[1].evaluate(shp, (0.0, 0.5, 0.0)),
         fa[2].evaluate(shp, (0.0, 0.0, 0.5))]
    Bs = list(_curl_face_B_3d(A, 1.0 / nx, 1.0 / ny, 1.0 / nz))
    bc = [_face_average(Bs[dd], _AXIS[dd]) for dd in range(3)]
    b2 = np.mean(bc[0] ** 2 + bc[1] ** 2 + bc[2] ** 2)
    h = 1.0 + gamma / (gamma - 1.0) * prs / rho
    sb = np.sqrt(sigma * np.mean(rho * h) / b2)
    Bs = [b * sb for b in Bs]
    V = np.zeros((8, nz, ny, nx))
    V[RHO], V[PRS] = rho, prs
    for dd in range(3):
        V[VX1 + dd] = vabs * unit[dd]
        V[BX1 + dd] = _face_average(Bs[dd], _AXIS[dd])
    return PrimState(PHYS_RMHD, 3, shp, gamma, V, Bs)


# ---------------------------------------------------------------------------
# Binary IC file (read by the reference problem file under oracle/ref)
# ---------------------------------------------------------------------------

IC_MAGIC = b"GPIC"


def write_ic(path: str, st: PrimState) -> None:
    nx, ny, nz = st.shape
    with open(path, "wb") as fh:
        fh.write(IC_MAGIC)
        fh.write(struct.pack("<7i", 1, st.physics, st.ndim, nx, ny, nz, st.nvar))
        fh.write(struct.pack("<7d", st.gamma, *st.xbeg, *st.xend))
        fh.write(np.ascontiguousarray(st.V, dtype="<f8").tobytes())
        for b in st.Bs:
            fh.write(np.ascontiguousarray(b, dtype="<f8").tobytes())


def read_ic(path: str) -> PrimState:
    with open(path, "rb") as fh:
        buf = fh.read()
    assert buf[:4] == IC_MAGIC
    ver, phys, ndim, nx, ny, nz, nvar = struct.unpack_from("<7i", buf, 4)
    vals = struct.unpack_from("<7d", buf, 32)
    off = 32 + 56
    ncell = nx * ny * nz
    V = np.frombuffer(buf, "<f8", nvar * ncell, off).reshape(nvar, nz, ny, nx).copy()
    off += 8 * nvar * ncell
    Bs = []
    if phys != PHYS_HD:
        for _ in range(ndim):
            Bs.append(np.frombuffer(buf, "<f8", ncell, off).reshape(nz, ny, nx).copy())
            off += 8 * ncell
    return PrimState(phys, ndim, (nx, ny, nz), vals[0], V, Bs,
                     tuple(vals[1:4]), tuple(vals[4:7]))
