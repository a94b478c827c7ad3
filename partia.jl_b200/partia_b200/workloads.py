"""Seeded synthetic particle sets and sample geometries of the benchmark
configurations (numpy PCG64 streams; the reference publishes no datasets).

C1  uniform box, gather, rho + Shepard A on a 64^3 cell-centre grid
C2  Plummer sphere, symmetric, rho, grad rho, div A, curl A on a 128^3 grid
C3  Gaussian clumps + background, scatter, column density on a 1024^2 beam
C4  the C3 model at N = 1e6 on a 512^2 beam (adjoint workload)
C5  exponential disc + Plummer halo, float32, rho, grad rho, curl v, z^2
"""
from __future__ import annotations

import math

import numpy as np

M4_SUPPORT = 2.0


def plummer_density(r, a=0.1, M=1.0):
    return 3.0 * M / (4.0 * math.pi * a ** 3) * (1.0 + (r / a) ** 2) ** -2.5


def _plummer_radii(rng, n, a, rmax):
    out = np.empty(0)
    while len(out) < n:
        u = rng.random(2 * (n - len(out)) + 16)
        u = u[u > 0]
        r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        out = np.concatenate([out, r[r <= rmax]])
    return out[:n]


def _isotropic(rng, n):
    cz = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    s = np.sqrt(1.0 - cz * cz)
    return s * np.cos(phi), s * np.sin(phi), cz


def uniform_c1(n=100_000, seed=0):
    """C1 particles; rho must still be filled by the density sum."""
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    m = np.full(n, 1.0 / n)
    h = np.full(n, 1.2 * (1.0 / n / 1.0) ** (1.0 / 3.0))
    A = np.sin(2 * math.pi * x) * np.cos(2 * math.pi * y) * z
    return dict(x=x, y=y, z=z, m=m, h=h, A=A)


def plummer_c2(n=2_000_000, seed=1, a=0.1):
    """C2: Plummer sphere (a = 0.1, truncated at 10a), equal masses summing to 1,
    h = 1.2 (m / rho_P)^(1/3), rho = rho_P(r), A = (-y, x, 0.1 z) + 0.01 N(0,1)."""
    rng = np.random.default_rng(seed)
    r = _plummer_radii(rng, n, a, 10 * a)
    ux, uy, uz = _isotropic(rng, n)
    x, y, z = r * ux, r * uy, r * uz
    m = np.full(n, 1.0 / n)
    rho = plummer_density(r, a)
    h = 1.2 * (m / rho) ** (1.0 / 3.0)
    noise = 0.01 * rng.standard_normal((3, n))
    Ax, Ay, Az = -y + noise[0], x + noise[1], 0.1 * z + noise[2]
    return dict(x=x, y=y, z=z, m=m, h=h, rho=rho, Ax=Ax, Ay=Ay, Az=Az)


def clumps(n, seed, nclump=64, frac_clump=0.9):
    """C3/C4 positions: 90% in 64 isotropic Gaussian clumps (centres U[0,1)^3,
    sigma log-uniform in [0.005, 0.05], counts multinomial with Dirichlet(1)
    weights), 10% uniform in [0,1)^3; equal masses summing to 1."""
    rng = np.random.default_rng(seed)
    nc = int(round(frac_clump * n))
    w = rng.dirichlet(np.ones(nclump))
    counts = rng.multinomial(nc, w)
    cen = rng.random((nclump, 3))
    sig = np.exp(rng.uniform(math.log(0.005), math.log(0.05), nclump))
    lab = np.repeat(np.arange(nclump), counts)
    pos = cen[lab] + sig[lab, None] * rng.standard_normal((nc, 3))
    bg = rng.random((n - nc, 3))
    p = np.concatenate([pos, bg])
    return dict(x=np.ascontiguousarray(p[:, 0]), y=np.ascontiguousarray(p[:, 1]),
                z=np.ascontiguousarray(p[:, 2]), m=np.full(n, 1.0 / n))


def disc_halo_c5(n=64_000_000, seed=4, frac_disc=0.7, rd=0.2, zd=0.02, a_halo=0.3, dtype=np.float32):
    """C5 positions (float32 by default): frac_disc of the particles in an
    exponential disc (surface density ~ exp(-R/rd), so R ~ Gamma(2, rd);
    sech^2(z/zd) vertical profile, z = zd atanh(2u - 1); uniform azimuth), the
    rest in a Plummer halo (scale a_halo, truncated at 10 a_halo); equal masses
    summing to 1.  Fields: the disc rotation velocity
    v = (-y, x, 0) (x^2 + y^2 + 0.01)^(-3/4) and the scalar z^2.  h and rho
    come from density_h."""
    rng = np.random.default_rng(seed)
    nd = int(round(frac_disc * n))
    R = rng.gamma(2.0, rd, nd)
    u = rng.random(nd)
    u = np.clip(u, 1e-12, 1.0 - 1e-12)
    zdisc = zd * np.arctanh(2.0 * u - 1.0)
    phi = rng.uniform(0.0, 2.0 * math.pi, nd)
    r = _plummer_radii(rng, n - nd, a_halo, 10 * a_halo)
    ux, uy, uz = _isotropic(rng, n - nd)
    x = np.concatenate([R * np.cos(phi), r * ux])
    y = np.concatenate([R * np.sin(phi), r * uy])
    z = np.concatenate([zdisc, r * uz])
    fac = (x * x + y * y + 0.01) ** -0.75
    out = dict(x=x, y=y, z=z, m=np.full(n, 1.0 / n), vx=-y * fac, vy=x * fac, vz=np.zeros(n), z2=z * z)
    return {k: np.ascontiguousarray(v, dtype=dtype) for k, v in out.items()}


def density_h(d, iters=3, eta=1.2, device=0):
    """Smoothing lengths and densities from the density sum (the clump
    configurations' recipe): h0 = eta (m / rho0)^(1/3) with rho0 the mean
    density (total mass over the unit cube), then `iters` rounds of
    rho = sum_b m_b W(|x - x_b|, h) (gather at the particles, M4) and
    h = eta (m / rho)^(1/3).  Runs on the GPU through the library; returns
    (h, rho) with rho the last density sum."""
    from . import _lib as L
    from .engine import Context
    x, y, z, m = d["x"], d["y"], d["z"], d["m"]
    rho0 = float(np.sum(m))
    h = eta * (m / rho0) ** (1.0 / 3.0)
    ctx = Context(device)
    rho = None
    try:
        for _ in range(iters):
            ctx.set_particles(x, y, z, m, h, np.ones_like(m))
            ctx.build(want_perm=False)
            rho = ctx.density(x, y, z, strategy=L.PSB_GATHER, hmode=L.PSB_H_PER_SAMPLE, hs=h)
            h = eta * (m / rho) ** (1.0 / 3.0)
    finally:
        ctx.close()
    return h, rho


def cell_centre_axis(n, lo=0.0, hi=1.0):
    d = (hi - lo) / n
    return (lo + 0.5 * d, hi - 0.5 * d, n)


# ---- oriented frames (src/julia/Frames/) -----------------------------------------
def qmul(a, b):
    """Hamilton product of quaternions (s, v1, v2, v3)."""
    s1, x1, y1, z1 = a
    s2, x2, y2, z2 = b
    return (s1 * s2 - x1 * x2 - y1 * y2 - z1 * z2,
            s1 * x2 + x1 * s2 + y1 * z2 - z1 * y2,
            s1 * y2 - x1 * z2 + y1 * s2 + z1 * x2,
            s1 * z2 + x1 * y2 - y1 * x2 + z1 * s2)


class Frame:
    """Frame(x, f0, u0) with rotate!, frame_right/up/forward
    (Frames/struct/Frame.jl:42-90, Frames/operations/rotation.jl:15-26,87-113)."""

    def __init__(self, x, f0, u0):
        f0 = np.asarray(f0, dtype=float)
        u0 = np.asarray(u0, dtype=float)
        nf, nu = math.hypot(*f0), math.hypot(*u0)
        if nf == 0 or nu == 0:
            raise ValueError("f0 and u0 must be nonzero.")
        f0 = f0 * (1.0 / nf)
        u0 = u0 * (1.0 / nu)
        if abs(float(np.dot(f0, u0))) > math.sqrt(np.finfo(float).eps):
            raise ValueError("f0 and u0 must be orthogonal.")
        r0 = np.cross(f0, u0)
        self.x = np.asarray(x, dtype=float)
        self.f0, self.u0, self.r0 = f0, u0, r0 / np.linalg.norm(r0)
        self.Q = (1.0, 0.0, 0.0, 0.0)

    @staticmethod
    def _rotation(axis, angle):
        n = axis / np.linalg.norm(axis)
        c, s = math.cos(angle * 0.5), math.sin(angle * 0.5)
        return (c, s * n[0], s * n[1], s * n[2])

    def rotate(self, yaw, pitch, roll):
        """rotate!(frame, yaw, pitch, roll): Q = Q * Qyaw(u0) * Qpitch(r0) * Qroll(f0)."""
        Q = qmul(qmul(qmul(self.Q, self._rotation(self.u0, yaw)), self._rotation(self.r0, pitch)),
                 self._rotation(self.f0, roll))
        nq = math.sqrt(sum(q * q for q in Q))
        self.Q = tuple(q / nq for q in Q)

    def _rot(self, v):
        q = self.Q
        qc = (q[0], -q[1], -q[2], -q[3])
        r = qmul(qmul(q, (0.0, v[0], v[1], v[2])), qc)
        return np.array(r[1:])

    def right(self):
        return self._rot(self.r0)

    def up(self):
        return self._rot(self.u0)

    def forward(self):
        return self._rot(self.f0)

    def as_array(self):
        """{x0,y0,z0, rx,ry,rz, ux,uy,uz, fx,fy,fz} for psb_interp_box / psb_interp_beam."""
        return np.concatenate([self.x, self.right(), self.up(), self.forward()])


def c3_frame():
    """Frame(x=0, f0=-z, u0=+y), rotated 30 deg about z, then 45 deg about x."""
    fr = Frame((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0))
    fr.rotate(0.0, 0.0, -math.pi / 6)
    fr.rotate(0.0, math.pi / 4, 0.0)
    return fr


def plane_coordinates(frame_arr, xparams, yparams):
    """_cartesian_plane_coordinates (Grids/grids/coordinate.jl:37-73), column-major."""
    x0, r, u = frame_arr[0:3], frame_arr[3:6], frame_arr[6:9]
    (xmin, xmax, nx), (ymin, ymax, ny) = xparams, yparams
    dx = (xmax - xmin) / float(nx - 1)
    dy = (ymax - ymin) / float(ny - 1)
    xi = xmin + np.arange(nx, dtype=float) * dx
    eta = ymin + np.arange(ny, dtype=float) * dy
    XI, ETA = np.meshgrid(xi, eta, indexing="ij")
    XI, ETA = XI.ravel(order="F"), ETA.ravel(order="F")
    return tuple(x0[c] + XI * r[c] + ETA * u[c] for c in range(3))


def box_coordinates(frame_arr, xparams, yparams, zparams):
    """_cartesian_box_coordinates (Grids/grids/coordinate.jl:93-151), column-major."""
    x0, r, u, f = frame_arr[0:3], frame_arr[3:6], frame_arr[6:9], frame_arr[9:12]
    (xmin, xmax, nx), (ymin, ymax, ny), (zmin, zmax, nz) = xparams, yparams, zparams
    dx = (xmax - xmin) / float(nx - 1)
    dy = (ymax - ymin) / float(ny - 1)
    dz = (zmax - zmin) / float(nz - 1)
    xi = xmin + np.arange(nx, dtype=float) * dx
    eta = ymin + np.arange(ny, dtype=float) * dy
    zeta = zmin + np.arange(nz, dtype=float) * dz
    XI, ETA, ZE = np.meshgrid(xi, eta, zeta, indexing="ij")
    XI, ETA, ZE = (a.ravel(order="F") for a in (XI, ETA, ZE))
    return tuple(x0[c] + XI * r[c] + ETA * u[c] + ZE * f[c] for c in range(3))
