"""CPU oracle for the MHIT36 timestep hot path (TEST INFRASTRUCTURE ONLY).

This module is the checker, never the product: only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may import it.  It is a float64 NumPy restatement of
one rank of the reference timestep loop, ``multi/main.f90:456-1042`` (aroccon/MHIT36_mixedp),
with periodic indexing in place of the cuDecomp halo planes (on one rank a halo plane is the
periodic neighbour, ``multi/main.f90:352-364``).  ``numpy.fft`` (pocketfft) stands in for the
cuFFT 1-D plans of ``multi/main.f90:187-205`` (closed library; parity at that boundary is
pinned only through the golden vectors in ``tests/golden``).

Array convention: a field is a C-ordered ``(nz, ny, nx)`` float64 array, i.e. Fortran
``(nx, ny, nz)`` x-fastest, with no halo -- the layout of the reference's field files
(``multi/readwrite.f90:28-46``).  ``a[k, j, i]`` is the reference's ``a(i+1, j+2, k+2)``
(local index with the halo plane at 1).

Evaluation order follows the Fortran expressions term by term so that the oracle and the
reference round alike (Fortran evaluates ``a*b*c`` as ``(a*b)*c`` and unary minus binds
looser than ``*``).

Reference geometry.  The reference labels the owned y/z plane with 0-based global index g by
``x(jg)`` with ``jg = piX%lo + j - 1`` and the local (halo-shifted) index ``j = g + 2``, so
y/z tables are read one entry further on than x tables (``multi/main.f90:327-331,709-714``);
the last plane reads one entry past the end of ``x``/``mysin``/``mycos``.  The oracle extends
the tables by one accumulated step (``x(n+1) = x(n) + dx``), which equals the periodic value
for the integer forcing wavenumbers the reference uses.  ``yz_shift=0`` gives the
grid-aligned variant.  The tracer interpolation uses the same shifted labelling
(``multi/particles.f90:95-117``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

ENUM = 1.0e-16  # multi/readinput.f90:49 (enum=1.e-16, a double literal of a real constant)


# ----------------------------------------------------------------------------------------
# parameters  (multi/readinput.f90:14-49, multi/module.f90:1-19)
# ----------------------------------------------------------------------------------------
@dataclasses.dataclass
class Params:
    nx: int = 64
    ny: int = 0
    nz: int = 0
    dt: float = 5e-4
    mu: float = 0.006
    rho: float = 1.0
    f1: float = 1.0
    f2: float = 1.0
    f3: float = 1.0
    k0: float = 2.0
    radius: float = 0.5
    sigma: float = 1.0
    epsr: float = 1.0
    phiflag: int = 0
    partflag: int = 0
    poisson: str = "fp64"          # "fp64" | "fp32" (multi/main.f90:844,853-912) | "fp32_refined"
    #                                | "fp32_incremental"
    laplacian: str = "exact"       # "exact" k^2 (multi/main.f90:889) | "modified" (2-2cos)/dx^2
    yz_shift: int = 1              # 1: reference labelling of y/z planes, 0: grid aligned
    interp: str = "linear1d"       # "linear1d" (multi/particles.f90:114-117) | "trilinear"
    acdi_clamp: int = 0            # 1: also clamp phi >= 0 before the log (opt-in deviation)

    def __post_init__(self):
        if self.ny == 0:
            self.ny = self.nx
        if self.nz == 0:
            self.nz = self.nx

    # derived constants, multi/readinput.f90:114-124
    @property
    def lx(self):
        return 8.0 * math.atan(1.0)

    @property
    def dx(self):
        return self.lx / self.nx

    @property
    def dxi(self):
        return 1.0 / self.dx

    @property
    def ddxi(self):
        return 1.0 / self.dx / self.dx

    @property
    def rhoi(self):
        return 1.0 / self.rho

    @property
    def eps(self):
        return self.epsr * self.dx

    @property
    def epsi(self):
        return 1.0 / self.eps


def grid_coords(n, dx):
    """x(1..n+1) accumulated as in multi/main.f90:210-214 (x(i)=x(i-1)+dx), 0-based."""
    x = np.zeros(n + 1)
    acc = 0.0
    for i in range(1, n + 1):
        acc = acc + dx
        x[i] = acc
    return x


def forcing_tables(p: Params):
    """mysin/mycos of multi/main.f90:244-250, as read along each axis.

    Returns (sx, cx, sy, cy, sz, cz): per-axis tables indexed by the 0-based global index.
    x reads mysin(i); y/z read mysin(jg)/mysin(kg), one entry on (reference labelling).
    """
    out = []
    for axis, n in enumerate((p.nx, p.ny, p.nz)):
        xc = grid_coords(n, p.dx)
        off = 0 if axis == 0 else p.yz_shift
        s = np.array([math.sin(p.k0 * xc[g + off] + p.dx / 2) for g in range(n)])
        c = np.array([math.cos(p.k0 * xc[g + off] + p.dx / 2) for g in range(n)])
        out += [s, c]
    return tuple(out)


def wavenumbers(n):
    """kx of multi/main.f90:234-240 with twoPi/lx == 1 exactly (lx = 8*atan(1))."""
    k = np.zeros(n)
    for i in range(n):
        k[i] = i if i < n // 2 else i - n
    return k


# periodic neighbours ------------------------------------------------------------------
def xp(a):
    return np.roll(a, -1, axis=2)


def xm(a):
    return np.roll(a, 1, axis=2)


def yp(a):
    return np.roll(a, -1, axis=1)


def ym(a):
    return np.roll(a, 1, axis=1)


def zp(a):
    return np.roll(a, -1, axis=0)


def zm(a):
    return np.roll(a, 1, axis=0)


# ----------------------------------------------------------------------------------------
# state
# ----------------------------------------------------------------------------------------
@dataclasses.dataclass
class State:
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    rhsu_o: np.ndarray
    rhsv_o: np.ndarray
    rhsw_o: np.ndarray
    p: np.ndarray
    phi: np.ndarray | None = None
    rhsphi_o: np.ndarray | None = None
    part: np.ndarray | None = None   # (np, 12) table, multi/particles.f90:15-22 (0-based cols)
    p32: np.ndarray | None = None    # fp32_incremental: the FP32 pressure predictor (0 at start)
    alpha: float = 1.0               # Euler on the first step, multi/main.f90:440-441
    beta: float = 0.0
    gumax: float = 1.0               # multi/main.f90:442
    nstep: int = 0


def new_state(p: Params, u, v, w, phi=None, part=None) -> State:
    z = lambda: np.zeros_like(u)
    st = State(u=u.copy(), v=v.copy(), w=w.copy(), rhsu_o=z(), rhsv_o=z(), rhsw_o=z(), p=z())
    if p.phiflag:
        st.phi = phi.copy()
        st.rhsphi_o = z()
    if p.partflag:
        st.part = part.copy()
    if p.poisson == "fp32_incremental":
        st.p32 = np.zeros(u.shape, dtype=np.float32)
    return st


# ----------------------------------------------------------------------------------------
# step pieces
# ----------------------------------------------------------------------------------------
def tracer_step(p: Params, st: State):
    """multi/main.f90:477-508: interpolate (particles.f90:88-119), AB2, wrap (364-380), shift."""
    part = st.part
    u_p, v_p, w_p = interpolate(p, st.u, st.v, st.w, part[:, 1], part[:, 2], part[:, 3])
    part[:, 4] = u_p
    part[:, 5] = v_p
    part[:, 6] = w_p
    for j in range(3):  # multi/main.f90:481-486
        part[:, 1 + j] = part[:, 1 + j] + p.dt * (st.alpha * part[:, 4 + j] - st.beta * part[:, 8 + j])
    lx = p.lx
    for j in range(3):  # multi/particles.f90:372-376
        part[:, 1 + j] = part[:, 1 + j] - lx * np.floor(part[:, 1 + j] / lx)
    for j in range(3):  # multi/main.f90:504-508
        part[:, 8 + j] = part[:, 4 + j]


def interpolate(p: Params, u, v, w, xq, yq, zq):
    """Velocity at tracer positions.

    linear1d: multi/particles.f90:96-117 -- per-component 1-D linear interpolation along the
    component's own axis at the left node.  Local y/z index ``1+floor(y/dx)`` is global plane
    ``floor(y/dx) - yz_shift`` (the halo plane at local index 1).
    trilinear: full trilinear interpolation at the staggered face positions of the same
    labelling (u at x=(i-1/2)dx, y=(j+s)dx, z=(k+s)dx; v, w alike), s = yz_shift.
    """
    nx, ny, nz, dx = p.nx, p.ny, p.nz, p.dx
    s = p.yz_shift
    if p.interp == "linear1d":
        ix = np.floor(xq / dx)
        iy = np.floor(yq / dx)
        iz = np.floor(zq / dx)
        tx = xq / dx - ix
        ty = yq / dx - iy
        tz = zq / dx - iz
        ix = ix.astype(np.int64)
        iy = iy.astype(np.int64)
        iz = iz.astype(np.int64)
        i0 = np.mod(ix, nx)
        i1 = np.mod(ix + 1, nx)
        j0 = np.mod(iy - s, ny)
        j1 = np.mod(iy - s + 1, ny)
        k0 = np.mod(iz - s, nz)
        k1 = np.mod(iz - s + 1, nz)
        up = (1.0 - tx) * u[k0, j0, i0] + tx * u[k0, j0, i1]
        vp = (1.0 - ty) * v[k0, j0, i0] + ty * v[k0, j1, i0]
        wp = (1.0 - tz) * w[k0, j0, i0] + tz * w[k1, j0, i0]
        return up, vp, wp
    # trilinear
    def tri(f, ox, oy, oz):
        fx = xq / dx - ox
        fy = yq / dx - oy
        fz = zq / dx - oz
        ix = np.floor(fx)
        iy = np.floor(fy)
        iz = np.floor(fz)
        tx = fx - ix
        ty = fy - iy
        tz = fz - iz
        ix = ix.astype(np.int64)
        iy = iy.astype(np.int64)
        iz = iz.astype(np.int64)
        a0, a1 = np.mod(ix, nx), np.mod(ix + 1, nx)
        b0, b1 = np.mod(iy, ny), np.mod(iy + 1, ny)
        c0, c1 = np.mod(iz, nz), np.mod(iz + 1, nz)
        c00 = (1.0 - tx) * f[c0, b0, a0] + tx * f[c0, b0, a1]
        c10 = (1.0 - tx) * f[c0, b1, a0] + tx * f[c0, b1, a1]
        c01 = (1.0 - tx) * f[c1, b0, a0] + tx * f[c1, b0, a1]
        c11 = (1.0 - tx) * f[c1, b1, a0] + tx * f[c1, b1, a1]
        c0_ = (1.0 - ty) * c00 + ty * c10
        c1_ = (1.0 - ty) * c01 + ty * c11
        return (1.0 - tz) * c0_ + tz * c1_
    up = tri(u, -0.5, s, s)
    vp = tri(v, 0.0, s - 0.5, s)
    wp = tri(w, 0.0, s, s - 0.5)
    return up, vp, wp


def phase_step(p: Params, st: State):
    """ACDI transport, multi/main.f90:522-636 (psi, RHS, normals, sharpening, AB2)."""
    phi = st.phi
    u, v, w = st.u, st.v, st.w
    eps, epsi, dxi, ddxi = p.eps, p.epsi, p.dxi, p.ddxi
    # :522-534
    val = np.minimum(phi, 1.0)
    if p.acdi_clamp:
        val = np.maximum(val, 0.0)
    psidi = eps * np.log((val + ENUM) / (1.0 - val + ENUM))
    tanh_psi = np.tanh(0.5 * psidi * epsi)
    gamma = 1.0 * st.gumax  # :536
    # :537-564
    rhsphi = (-((xp(u) * 0.5 * (xp(phi) + phi) - u * 0.5 * (phi + xm(phi))) * dxi)
              - (yp(v) * 0.5 * (yp(phi) + phi) - v * 0.5 * (phi + ym(phi))) * dxi
              - (zp(w) * 0.5 * (zp(phi) + phi) - w * 0.5 * (phi + zm(phi))) * dxi
              + gamma * (eps * (xp(phi) - 2.0 * phi + xm(phi)) * ddxi
                         + eps * (yp(phi) - 2.0 * phi + ym(phi)) * ddxi
                         + eps * (zp(phi) - 2.0 * phi + zm(phi)) * ddxi))
    normx = xp(psidi) - xm(psidi)
    normy = yp(psidi) - ym(psidi)
    normz = zp(psidi) - zm(psidi)
    # :582-593
    normag = 1.0 / (np.sqrt(normx * normx + normy * normy + normz * normz) + ENUM)
    normx = normx * normag
    normy = normy * normag
    normz = normz * normag
    # :596-618
    fx = 0.25 * (1.0 - tanh_psi * tanh_psi) * normx
    fy = 0.25 * (1.0 - tanh_psi * tanh_psi) * normy
    fz = 0.25 * (1.0 - tanh_psi * tanh_psi) * normz
    rhsphi = rhsphi - gamma * ((xp(fx) - xm(fx)) * 0.5 * dxi
                               + (yp(fy) - ym(fy)) * 0.5 * dxi
                               + (zp(fz) - zm(fz)) * 0.5 * dxi)
    # :621-630
    st.phi = phi + p.dt * (st.alpha * rhsphi - st.beta * st.rhsphi_o)
    st.rhsphi_o = rhsphi


def momentum_rhs(p: Params, st: State, tables):
    """Momentum RHS, multi/main.f90:658-717 (advection, diffusion, ABC forcing)."""
    u, v, w = st.u, st.v, st.w
    dxi, ddxi, rhoi, mu = p.dxi, p.ddxi, p.rhoi, p.mu
    sx, cx, sy, cy, sz, cz = tables
    up_, um_ = xp(u), xm(u)
    h11 = (up_ + u) * (up_ + u) - (u + um_) * (u + um_)
    h12 = (yp(u) + u) * (yp(v) + xm(yp(v))) - (u + ym(u)) * (v + xm(v))
    h13 = (zp(u) + u) * (zp(w) + xm(zp(w))) - (u + zm(u)) * (w + xm(w))
    h21 = (xp(u) + xp(ym(u))) * (xp(v) + v) - (u + ym(u)) * (v + xm(v))
    h22 = (yp(v) + v) * (yp(v) + v) - (v + ym(v)) * (v + ym(v))
    h23 = (zp(w) + ym(zp(w))) * (zp(v) + v) - (w + ym(w)) * (v + zm(v))
    h31 = (xp(w) + w) * (xp(u) + xp(zm(u))) - (w + xm(w)) * (u + zm(u))
    h32 = (yp(v) + yp(zm(v))) * (yp(w) + w) - (v + zm(v)) * (w + ym(w))
    h33 = (zp(w) + w) * (zp(w) + w) - (w + zm(w)) * (w + zm(w))
    h11 = h11 * 0.25 * dxi
    h12 = h12 * 0.25 * dxi
    h13 = h13 * 0.25 * dxi
    h21 = h21 * 0.25 * dxi
    h22 = h22 * 0.25 * dxi
    h23 = h23 * 0.25 * dxi
    h31 = h31 * 0.25 * dxi
    h32 = h32 * 0.25 * dxi
    h33 = h33 * 0.25 * dxi
    rhsu = -(h11 + h12 + h13)
    rhsv = -(h21 + h22 + h23)
    rhsw = -(h31 + h32 + h33)
    h11 = mu * (xp(u) - 2.0 * u + xm(u)) * ddxi
    h12 = mu * (yp(u) - 2.0 * u + ym(u)) * ddxi
    h13 = mu * (zp(u) - 2.0 * u + zm(u)) * ddxi
    h21 = mu * (xp(v) - 2.0 * v + xm(v)) * ddxi
    h22 = mu * (yp(v) - 2.0 * v + ym(v)) * ddxi
    h23 = mu * (zp(v) - 2.0 * v + zm(v)) * ddxi
    h31 = mu * (xp(w) - 2.0 * w + xm(w)) * ddxi
    h32 = mu * (yp(w) - 2.0 * w + ym(w)) * ddxi
    h33 = mu * (zp(w) - 2.0 * w + zm(w)) * ddxi
    rhsu = rhsu + (h11 + h12 + h13) * rhoi
    rhsv = rhsv + (h21 + h22 + h23) * rhoi
    rhsw = rhsw + (h31 + h32 + h33) * rhoi
    # ABC forcing, :712-714 (tables broadcast along their own axis)
    SX, CX = sx[None, None, :], cx[None, None, :]
    SY, CY = sy[None, :, None], cy[None, :, None]
    SZ, CZ = sz[:, None, None], cz[:, None, None]
    rhsu = rhsu + p.f3 * SZ + p.f2 * CY
    rhsv = rhsv + p.f1 * SX + p.f3 * CZ
    rhsw = rhsw + p.f2 * SY + p.f1 * CX
    return rhsu, rhsv, rhsw


def surface_tension(p: Params, phi):
    """Chemical-potential force at cell centres, multi/main.f90:721-743."""
    eps, epsi, dxi, ddxi, sigma = p.eps, p.epsi, p.dxi, p.ddxi, p.sigma
    chempot = (phi * (1.0 - phi) * (1.0 - 2.0 * phi) * epsi
               - eps * (xp(phi) + xm(phi) + yp(phi) + ym(phi) + zp(phi) + zm(phi) - 6.0 * phi) * ddxi)
    fxst = 6.0 * sigma * chempot * 0.5 * (xp(phi) - xm(phi)) * dxi
    fyst = 6.0 * sigma * chempot * 0.5 * (yp(phi) - ym(phi)) * dxi
    fzst = 6.0 * sigma * chempot * 0.5 * (zp(phi) - zm(phi)) * dxi
    return fxst, fyst, fzst


def momentum_step(p: Params, st: State, tables):
    """u* and rhs_o, multi/main.f90:658-802."""
    rhsu, rhsv, rhsw = momentum_rhs(p, st, tables)
    if p.phiflag:  # :760-780
        fxst, fyst, fzst = surface_tension(p, st.phi)
        rhsu = rhsu + 0.5 * (xm(fxst) + fxst) * p.rhoi
        rhsv = rhsv + 0.5 * (ym(fyst) + fyst) * p.rhoi
        rhsw = rhsw + 0.5 * (zm(fzst) + fzst) * p.rhoi
    a, b, dt = st.alpha, st.beta, p.dt
    st.u = st.u + dt * (a * rhsu - b * st.rhsu_o)
    st.v = st.v + dt * (a * rhsv - b * st.rhsv_o)
    st.w = st.w + dt * (a * rhsw - b * st.rhsw_o)
    st.rhsu_o, st.rhsv_o, st.rhsw_o = rhsu, rhsv, rhsw
    st.alpha, st.beta = 1.5, 0.5  # :801-802


def poisson_rhs(p: Params, u, v, w):
    """rho/dt * div u*, multi/main.f90:833-848 (FP64)."""
    c = p.rho * p.dxi / p.dt
    rhsp = c * (xp(u) - u)
    rhsp = rhsp + c * (yp(v) - v)
    rhsp = rhsp + c * (zp(w) - w)
    return rhsp


def k2_table(p: Params):
    """k^2 on the half spectrum (nz, ny, nx//2+1) in FP64, multi/main.f90:884-890.

    The cells are cubes of side dx = lx/nx, so an axis of n cells is n dx long: its wavenumber of
    index k is k nx/n (2 pi/lx = 1) and its modified symbol (2 - 2 cos(2 pi k/n))/dx^2.  On the
    reference's cubic box these reduce to the integer k and (2 - 2 cos(k dx))/dx^2."""
    kx = wavenumbers(p.nx)[: p.nx // 2 + 1].copy()
    kx[p.nx // 2] = -(p.nx // 2)   # kx(nx/2+1) = (nx/2 - nx)
    ky = wavenumbers(p.ny)
    kz = wavenumbers(p.nz)
    if p.laplacian == "modified":
        # (2 - 2 cos(k h)) / dx^2 per axis, h = lx/n: the symbol of the 7-point staggered Laplacian
        mx = (2.0 - 2.0 * np.cos(kx * (p.lx / p.nx))) * p.ddxi
        my = (2.0 - 2.0 * np.cos(ky * (p.lx / p.ny))) * p.ddxi
        mz = (2.0 - 2.0 * np.cos(kz * (p.lx / p.nz))) * p.ddxi
        return mx[None, None, :] + my[None, :, None] + mz[:, None, None]
    kx, ky, kz = kx * (p.nx / p.nx), ky * (p.nx / p.ny), kz * (p.nx / p.nz)
    return kx[None, None, :] ** 2 + ky[None, :, None] ** 2 + kz[:, None, None] ** 2


def poisson_solve(p: Params, rhsp):
    """Spectral solve of lap(p) = rhsp, multi/main.f90:851-913.

    fp64: the intended FP64 semantics.  fp32: rhs cast to FP32 (:844), FP32 transforms,
    the divide in FP64 and rounded back (complex(4)/real(8) promotes, :890), FP32 pressure.
    """
    n = p.nx * p.ny * p.nz
    k2 = k2_table(p)
    with np.errstate(divide="ignore", invalid="ignore"):
        if p.poisson == "fp64":
            hat = np.fft.rfftn(rhsp, axes=(0, 1, 2))
            hat = -hat / k2 / float(n)
            hat[0, 0, 0] = 0.0
            pr = np.fft.irfftn(hat, s=rhsp.shape, axes=(0, 1, 2), norm="forward")
            return pr
        if p.poisson in ("fp32", "fp32_refined"):
            p32 = solve32(p, rhsp)
            if p.poisson == "fp32":
                return p32
            # one FP64 residual sweep: r = rhs - L_h p32 in FP64, L_h delta = r in FP32
            q = p32.astype(np.float64)
            delta = solve32(p, rhsp - laplacian7(p, q))
            return q + delta.astype(np.float64)
    raise ValueError(p.poisson)


def solve32(p: Params, rhs):
    """The FP32 branch's solve (multi/main.f90:844-912): rhs rounded to FP32, FP32 transforms,
    the divide in FP64 rounded back (complex(4)/real(8) promotes, :890), FP32 pressure."""
    n = p.nx * p.ny * p.nz
    with np.errstate(divide="ignore", invalid="ignore"):
        hat = fft3_r2c_f32(rhs.astype(np.float32))
        hat = (-(hat.astype(np.complex128)) / k2_table(p) / float(n)).astype(np.complex64)
    hat[0, 0, 0] = 0.0
    return fft3_c2r_f32(hat, rhs.shape)


def laplacian7(p: Params, q):
    """The 7-point Laplacian L_h q (the operator whose symbol the modified divide uses), summed
    per axis as (q+ - 2 q + q-) ddxi."""
    return ((xp(q) - 2.0 * q + xm(q)) * p.ddxi + (yp(q) - 2.0 * q + ym(q)) * p.ddxi
            + (zp(q) - 2.0 * q + zm(q)) * p.ddxi)


def poisson_solve_incremental(p: Params, rhsp, pred32):
    """One FP32 solve for the increment over the previous step's pressure (needs the modified
    Laplacian).  r = rhs - L_h q in FP64 with q the FP32 predictor, L_h delta = r in FP32, and
    s = q + delta in FP64.  Returns (s, the pressure the projection uses; fl32(s), the next
    step's predictor)."""
    if p.laplacian != "modified":
        raise ValueError("fp32_incremental needs the modified Laplacian")
    q = pred32.astype(np.float64)
    delta = solve32(p, rhsp - laplacian7(p, q))
    s = q + delta.astype(np.float64)
    return s, s.astype(np.float32)


def fft3_r2c_f32(a32):
    """Unnormalised 3-D R2C in single precision (rounded to complex64 after each axis)."""
    h = np.fft.rfft(a32.astype(np.float64), axis=2).astype(np.complex64)
    h = np.fft.fft(h.astype(np.complex128), axis=1).astype(np.complex64)
    h = np.fft.fft(h.astype(np.complex128), axis=0).astype(np.complex64)
    return h


def fft3_c2r_f32(h, shape):
    """Unnormalised 3-D C2R in single precision (rounded to complex64 after each axis)."""
    h = np.fft.ifft(h.astype(np.complex128), axis=0, norm="forward").astype(np.complex64)
    h = np.fft.ifft(h.astype(np.complex128), axis=1, norm="forward").astype(np.complex64)
    r = np.fft.irfft(h.astype(np.complex128), n=shape[2], axis=2, norm="forward")
    return r.astype(np.float32)


def correct(p: Params, st: State, pr):
    """Projection, mean removal and max, multi/main.f90:942-1003 (one rank, ranks=1)."""
    c = p.dt / p.rho
    pr = pr.astype(np.float64)
    u = st.u - c * (pr - xm(pr)) * p.dxi
    v = st.v - c * (pr - ym(pr)) * p.dxi
    w = st.w - c * (pr - zm(pr)) * p.dxi
    n = (p.nx, p.ny, p.nz)
    um = np.sum(u) / n[0] / n[1] / n[2]
    vm = np.sum(v) / n[0] / n[1] / n[2]
    wm = np.sum(w) / n[0] / n[1] / n[2]
    st.u = u - um
    st.v = v - vm
    st.w = w - wm
    uc, vc, wc = st.u.max(), st.v.max(), st.w.max()
    st.gumax = max(wc, max(uc, vc))
    st.p = pr
    return (um, vm, wm)


def step(p: Params, st: State, tables=None):
    """One timestep of multi/main.f90:456-1007 on one rank."""
    if tables is None:
        tables = forcing_tables(p)
    if p.partflag:
        tracer_step(p, st)
    if p.phiflag:
        phase_step(p, st)
    momentum_step(p, st, tables)
    rhsp = poisson_rhs(p, st.u, st.v, st.w)
    if p.poisson == "fp32_incremental":
        pr, st.p32 = poisson_solve_incremental(p, rhsp, st.p32)
    else:
        pr = poisson_solve(p, rhsp)
    means = correct(p, st, pr)
    st.nstep += 1
    return means


def run(p: Params, st: State, nsteps: int):
    tables = forcing_tables(p)
    for _ in range(nsteps):
        step(p, st, tables)
    return st


# ----------------------------------------------------------------------------------------
# diagnostics
# ----------------------------------------------------------------------------------------
def divergence(p: Params, u, v, w):
    """Discrete divergence at cell centres (the operator of multi/main.f90:841-843 / (rho/dt))."""
    return (xp(u) - u) * p.dxi + (yp(v) - v) * p.dxi + (zp(w) - w) * p.dxi


def dissipation(u, v, w, nu, dx):
    """2 nu <S_ij S_ij>, post/compute_diss/main.f90:72-117 (central differences)."""
    h = 0.5 / dx
    dudx = (xp(u) - xm(u)) * h
    dudy = (yp(u) - ym(u)) * h
    dudz = (zp(u) - zm(u)) * h
    dvdx = (xp(v) - xm(v)) * h
    dvdy = (yp(v) - ym(v)) * h
    dvdz = (zp(v) - zm(v)) * h
    dwdx = (xp(w) - xm(w)) * h
    dwdy = (yp(w) - ym(w)) * h
    dwdz = (zp(w) - zm(w)) * h
    s12 = 0.5 * (dudy + dvdx)
    s13 = 0.5 * (dudz + dwdx)
    s23 = 0.5 * (dvdz + dwdy)
    e = np.sum(dudx ** 2 + dvdy ** 2 + dwdz ** 2 + 2.0 * (s12 ** 2 + s13 ** 2 + s23 ** 2))
    n = u.size
    return 2.0 * nu * e / n


def kinetic_energy(u, v, w):
    return 0.5 * float(np.mean(u * u + v * v + w * w))


def energy_spectrum(u, v, w, nbins):
    """Shell-summed kinetic-energy spectrum E(k) = 1/2 sum_{round|kappa| = k} |u_kappa|^2 (+ v, w),
    u_kappa = rfftn(u)/N over the x-half spectrum (weight 2 for 0 < kx < nx/2), kappa in units of
    2 pi/Lx: kappa_y = m_y nx/ny, kappa_z = m_z nx/nz.  The reference has no 3-D spectrum tool;
    this is the definition the library's mhit_energy_spectrum restates (sum E = KE, Parseval)."""
    nz, ny, nx = u.shape
    ntot = float(u.size)
    kx = np.arange(nx // 2 + 1, dtype=np.float64)
    ky = np.fft.fftfreq(ny, 1.0 / ny) * (nx / ny)
    kz = np.fft.fftfreq(nz, 1.0 / nz) * (nx / nz)
    kk = np.sqrt(kx[None, None, :] ** 2 + (ky[None, :, None] ** 2 + kz[:, None, None] ** 2))
    shell = np.rint(kk).astype(np.int64)
    wgt = np.where((kx == 0) | (2 * kx == nx), 0.5, 1.0)[None, None, :]
    e = np.zeros(shell.shape)
    for f in (u, v, w):
        c = np.fft.rfftn(f) / ntot
        e += wgt * (c.real ** 2 + c.imag ** 2)
    keep = shell < nbins
    return np.bincount(shell[keep].ravel(), weights=e[keep].ravel(), minlength=nbins)[:nbins]


def taylor_green(p: Params):
    """Taylor-Green start, multi/main.f90:324-337 (u at x(i)-dx/2, reference y/z labelling)."""
    xs = grid_coords(p.nx, p.dx)
    ys = grid_coords(p.ny, p.dx)
    zs = grid_coords(p.nz, p.dx)
    s = p.yz_shift
    X = xs[: p.nx]
    Y = ys[s: s + p.ny]
    Z = zs[s: s + p.nz]
    u = (np.sin(X - p.dx / 2)[None, None, :] * np.cos(Y)[None, :, None] * np.cos(Z)[:, None, None])
    v = (-np.cos(X)[None, None, :] * np.sin(Y - p.dx / 2)[None, :, None] * np.cos(Z)[:, None, None])
    w = np.zeros_like(u)
    return u, v, w


def single_drop(p: Params):
    """Centred drop, multi/main.f90:370-382 (reference y/z labelling)."""
    xs = grid_coords(p.nx, p.dx)
    ys = grid_coords(p.ny, p.dx)
    zs = grid_coords(p.nz, p.dx)
    s = p.yz_shift
    X = xs[: p.nx]
    Y = ys[s: s + p.ny]
    Z = zs[s: s + p.nz]
    lx = p.lx
    pos = ((X - lx / 2) ** 2.0)[None, None, :] + ((Y - lx / 2) ** 2.0)[None, :, None]
    pos = pos + ((Z - lx / 2) ** 2.0)[:, None, None]
    return 0.5 * (1.0 - np.tanh((np.sqrt(pos) - p.radius) / 2 / p.eps))


# ---------------------------------------------------------------------- droplet labelling
def neighbour_offsets(connectivity):
    """(dz, dy, dx) of the 6 face or 26 face/edge/corner neighbours
    (post/unionfind_periodic/main.f90:33-48)."""
    if connectivity == 6:
        return [(0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)]
    if connectivity == 26:
        return [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1) if (a, b, c) != (0, 0, 0)]
    raise ValueError("connectivity must be 6 or 26")


def label_components(phi, thresh=0.5, connectivity=6):
    """Periodic connected components of phi >= thresh by min-label propagation, the algorithm of
    post/unionfind_periodic/main.f90:137-258: every masked cell starts with its own index and
    takes the minimum over itself and its masked neighbours (periodic wrap) until nothing changes.
    Arrays are (nz, ny, nx), x fastest; the starting index is the flat cell index (the reference's
    includes its halo planes), so each component ends labelled with its smallest cell index.
    Returns the label array with -1 for background."""
    n = phi.size
    mask = phi >= thresh
    big = np.int64(n)
    lab = np.where(mask, np.arange(n, dtype=np.int64).reshape(phi.shape), big)
    offs = neighbour_offsets(connectivity)
    while True:
        new = lab
        for dz, dy, dx in offs:
            # value at (k+dz, j+dy, i+dx), periodic
            new = np.minimum(new, np.roll(lab, shift=(-dz, -dy, -dx), axis=(0, 1, 2)))
        new = np.where(mask, new, big)
        if np.array_equal(new, lab):
            break
        lab = new
    return np.where(mask, lab, -1)


def drop_statistics(lab, u, v, w, lx=2 * math.pi):
    """Per component (ordered by label): cells, volume = cells dx^3, centre = circular mean of the
    cell centres per axis, mean u, v, w (post/unionfind_periodic/main.f90:276-336, :425-436).
    Cell centres accumulate x(1) = dx/2, x(i) = x(i-1) + dx as the reference does (:294-298);
    sums are in float64 (the reference accumulates the velocities in default REAL)."""
    nz, ny, nx = lab.shape
    pi = 4.0 * math.atan(1.0)
    dx = lx / nx
    sel = lab >= 0
    roots = np.unique(lab[sel])
    ids = np.searchsorted(roots, lab[sel])
    nd = len(roots)
    kk, jj, ii = np.nonzero(sel)
    cells = np.bincount(ids, minlength=nd)
    out = {"label": roots, "cells": cells, "volume": cells.astype(np.float64) * dx * dx * dx}
    for name, idx, na in (("x", ii, nx), ("y", jj, ny), ("z", kk, nz)):
        per = na * dx
        xs = np.empty(na)
        x = dx / 2.0
        for i in range(na):
            if i > 0:
                x = x + dx
            xs[i] = x
        s = np.bincount(ids, weights=np.sin(2.0 * pi * xs / per)[idx], minlength=nd)
        c = np.bincount(ids, weights=np.cos(2.0 * pi * xs / per)[idx], minlength=nd)
        ctr = per * np.arctan2(s, c) / (2.0 * pi)
        out[name] = np.where(ctr < 0.0, ctr + per, ctr)
    for name, f in (("u", u), ("v", v), ("w", w)):
        out[name] = np.bincount(ids, weights=f[sel], minlength=nd) / cells
    return out


def reference_test_sphere(nx):
    """The synthetic sphere of post/unionfind_periodic/main.f90:124-129 (readf = .false.):
    phi = 1 at 1-based (i, j, k) with (i-cx)^2+(j-cy)^2+(k-cz)^2 <= r2, cx = nx/4, cy = nx/3,
    cz = nx/2, r2 = (nx/10)^2 in integer arithmetic; phi = 0 elsewhere.  (nz, ny, nx) array."""
    cx, cy, cz, r2 = nx // 4, nx // 3, nx // 2, (nx // 10) ** 2
    i = np.arange(1, nx + 1)
    d2 = (i[None, None, :] - cx) ** 2 + (i[None, :, None] - cy) ** 2 + (i[:, None, None] - cz) ** 2
    return np.where(d2 <= r2, 1.0, 0.0), (cx, cy, cz, r2)
