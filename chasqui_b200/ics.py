"""Initial conditions for the workloads the reference's own problem generators cannot produce,
in the reference layout, plus the reference restart format used to hand them to any
reference-compatible reader.

  blast_noise : 3D MHD blast on [-0.5, 0.5]^3 with seeded uniform relative density noise
                (the reference's Blast, src/pgen.hpp:114-135, has no noise).
  cpaw_oblique: circularly polarised Alfven wave along an arbitrary lattice wavevector
                2*pi*(m1, m2, m3) on the unit box (the reference's CPAW, src/pgen.hpp:54-91,
                rotates only in x-y). B comes from a periodic vector potential on edges plus
                the uniform parallel field on faces, so div B = 0 to round-off.
  orszag_tang : the reference's Orszag-Tang set-up (src/pgen.hpp:94-111) with an optional
                pressure rescale to a target plasma beta.

Primitive -> conserved conversion follows src/pgen.hpp:286-300 (face-averaged centred B,
E = p/(gamma-1) + rho v^2/2 + B^2/2, entropy rho * p / rho^gamma) with the same operation
order. Noise: U = splitmix64(seed, n) / 2^53 for the active cell n in C order (k, j, i),
rho = 1 + amp * (2 U - 1) — the same counter-based stream as the device generator
(chq_init_problem), so host and device blasts are bitwise identical; ghost cells are filled
later by the boundary kernel, exactly as after the reference's Initialize().
"""
from __future__ import annotations

import math
import struct

import numpy as np


class Grid:
    def __init__(self, nx1, nx2, nx3, ng, x1min, x1max, x2min, x2max, x3min, x3max):
        self.nx1, self.nx2, self.nx3, self.ng = nx1, nx2, nx3, ng
        self.ni = nx1 + 2 * ng
        self.nj = nx2 + 2 * ng if nx2 > 1 else 1
        self.nk = nx3 + 2 * ng if nx3 > 1 else 1
        self.is_, self.js = ng, (ng if nx2 > 1 else 0)
        self.ks = ng if nx3 > 1 else 0
        self.two_d, self.three_d = nx2 > 1, nx3 > 1
        self.x1min, self.x2min, self.x3min = x1min, x2min, x3min
        self.dx1 = (x1max - x1min) / nx1
        self.dx2 = (x2max - x2min) / nx2
        self.dx3 = (x3max - x3min) / nx3

    # cell-centre and face coordinates (src/mesh.hpp:66-71), as 1-D arrays over all indices
    def x1v(self, n=None):
        i = np.arange(self.ni if n is None else n)
        return self.x1min + (i - self.is_ + 0.5) * self.dx1

    def x2v(self, n=None):
        j = np.arange(self.nj if n is None else n)
        return self.x2min + (j - self.js + 0.5) * self.dx2

    def x3v(self, n=None):
        k = np.arange(self.nk if n is None else n)
        return self.x3min + (k - self.ks + 0.5) * self.dx3

    def x1f(self, n=None):
        i = np.arange(self.ni + 1 if n is None else n)
        return self.x1min + (i - self.is_) * self.dx1

    def x2f(self, n=None):
        j = np.arange(self.nj + 1 if n is None else n)
        return self.x2min + (j - self.js) * self.dx2

    def x3f(self, n=None):
        k = np.arange(self.nk + 1 if n is None else n)
        return self.x3min + (k - self.ks) * self.dx3


def _conserve(g: Grid, d, vx, vy, vz, p, b1, b2, b3, gamma):
    """u0 (6, nk, nj, ni) from primitives on cells and face fields (src/pgen.hpp:286-300)."""
    gm1 = gamma - 1.0
    bx = 0.5 * (b1[:, :, :-1] + b1[:, :, 1:])[: g.nk, : g.nj]
    by = (0.5 * (b2[:, :-1, :] + b2[:, 1:, :]) if g.two_d else b2[:, :-1, :])[: g.nk, :, : g.ni]
    bz = (0.5 * (b3[:-1] + b3[1:]) if g.three_d else b3[:-1])[:, : g.nj, : g.ni]
    u = np.empty((6, g.nk, g.nj, g.ni))
    u[0] = d
    u[1] = d * vx
    u[2] = d * vy
    u[3] = d * vz
    u[4] = p / gm1 + 0.5 * d * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz)
    s = p / np.power(d, gamma)
    u[5] = d * s
    return u


def splitmix_uniform(seed: int, idx: np.ndarray) -> np.ndarray:
    """splitmix64 of (seed, idx) -> uniform doubles in [0, 1) from the top 53 bits."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx.astype(np.uint64) + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def blast_noise(n: int, seed: int = 20261203, amp: float = 1e-3, pres_in: float = 10.0, pres_out: float = 0.1,
                radius: float = 0.1, b0: float = 1.0, angle_deg: float = 45.0, gamma: float = 5.0 / 3.0, ng: int = 3):
    g = Grid(n, n, n, ng, -0.5, 0.5, -0.5, 0.5, -0.5, 0.5)
    ang = angle_deg * math.pi / 180.0
    bx, by = b0 * math.cos(ang), b0 * math.sin(ang)
    if abs(bx) < 1e-14 * b0:
        bx = 0.0
    if abs(by) < 1e-14 * b0:
        by = 0.0
    shp_f = (g.nk + 1, g.nj + 1, g.ni + 1)
    b1 = np.full(shp_f, bx)
    b2 = np.full(shp_f, by)
    b3 = np.zeros(shp_f)
    x, y, z = g.x1v(), g.x2v(), g.x3v()
    r = np.sqrt(x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2)
    p = np.where(r < radius, pres_in, pres_out)
    d = np.ones((g.nk, g.nj, g.ni))
    if amp != 0.0:
        noise = splitmix_uniform(seed, np.arange(n * n * n, dtype=np.uint64)).reshape(n, n, n)
        d[g.ks:g.ks + n, g.js:g.js + n, g.is_:g.is_ + n] = 1.0 + amp * (2.0 * noise - 1.0)
    zero = np.zeros_like(d)
    u = _conserve(g, d, zero, zero, zero, p, b1, b2, b3, gamma)
    return g, u, b1, b2, b3


def _curl_faces(g: Grid, A):
    """Face fields from a vector potential sampled at edge centres (src/pgen.hpp:30-50)."""
    xf, yf, zf = g.x1f(), g.x2f(), g.x3f()
    xv, yv, zv = g.x1v(g.ni + 1), g.x2v(g.nj + 1), g.x3v(g.nk + 1)
    idx, idy, idz = 1.0 / g.dx1, 1.0 / g.dx2, 1.0 / g.dx3
    X = lambda a: a[None, None, :]
    Y = lambda a: a[None, :, None]
    Z = lambda a: a[:, None, None]
    xf1 = g.x1f(g.ni + 2)[1:]
    yf1 = g.x2f(g.nj + 2)[1:]
    zf1 = g.x3f(g.nk + 2)[1:]
    b1 = np.zeros((g.nk + 1, g.nj + 1, g.ni + 1))
    if g.two_d:
        b1 = b1 + (A(2, X(xf), Y(yf1), Z(zv)) - A(2, X(xf), Y(yf), Z(zv))) * idy
    if g.three_d:
        b1 = b1 - (A(1, X(xf), Y(yv), Z(zf1)) - A(1, X(xf), Y(yv), Z(zf))) * idz
    b2 = -(A(2, X(xf1), Y(yf), Z(zv)) - A(2, X(xf), Y(yf), Z(zv))) * idx
    if g.three_d:
        b2 = b2 + (A(0, X(xv), Y(yf), Z(zf1)) - A(0, X(xv), Y(yf), Z(zf))) * idz
    b3 = (A(1, X(xf1), Y(yv), Z(zf)) - A(1, X(xf), Y(yv), Z(zf))) * idx
    if g.two_d:
        b3 = b3 - (A(0, X(xv), Y(yf1), Z(zf)) - A(0, X(xv), Y(yf), Z(zf))) * idy
    shp = (g.nk + 1, g.nj + 1, g.ni + 1)
    return (np.broadcast_to(b1, shp).copy(), np.broadcast_to(b2, shp).copy(), np.broadcast_to(b3, shp).copy())


def cpaw_oblique(n: int, m=(1, 1, 1), dens: float = 1.0, pres: float = 0.1, b_par: float = 1.0, amp: float = 0.1,
                 gamma: float = 5.0 / 3.0, ng: int = 3):
    """CPAW with wavevector 2 pi m on [0,1]^3; period T = lambda / v_A, lambda = 1/|m|."""
    g = Grid(n, n, n, ng, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    m = np.asarray(m, dtype=float)
    nrm = np.linalg.norm(m)
    e1 = m / nrm
    # e2 perpendicular to e1 (prefer the x-y plane), e3 = e1 x e2 (right handed)
    t = np.array([0.0, 0.0, 1.0]) if abs(e1[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    e2 = np.cross(t, e1)
    e2 /= np.linalg.norm(e2)
    e3 = np.cross(e1, e2)
    k = 2.0 * math.pi * nrm

    def s_of(x, y, z):
        return (x * e1[0] + y * e1[1] + z * e1[2])

    def A(c, x, y, z):
        s = s_of(x, y, z)
        return (amp / k) * (np.sin(k * s) * e2[c] + np.cos(k * s) * e3[c])

    b1, b2, b3 = _curl_faces(g, A)
    b1 += b_par * e1[0]
    b2 += b_par * e1[1]
    b3 += b_par * e1[2]
    x, y, z = g.x1v()[None, None, :], g.x2v()[None, :, None], g.x3v()[:, None, None]
    s = s_of(x, y, z)
    fac = -amp / math.sqrt(dens)
    vt2, vt3 = fac * np.sin(k * s), fac * np.cos(k * s)
    vx = vt2 * e2[0] + vt3 * e3[0]
    vy = vt2 * e2[1] + vt3 * e3[1]
    vz = vt2 * e2[2] + vt3 * e3[2]
    shp = (g.nk, g.nj, g.ni)
    d = np.full(shp, dens)
    p = np.full(shp, pres)
    u = _conserve(g, d, np.broadcast_to(vx, shp), np.broadcast_to(vy, shp), np.broadcast_to(vz, shp), p,
                  b1, b2, b3, gamma)
    period = (1.0 / nrm) / (b_par / math.sqrt(dens))
    return g, u, b1, b2, b3, period


def orszag_tang(n: int, beta: float | None = None, gamma: float = 5.0 / 3.0, ng: int = 3):
    """Orszag-Tang (src/pgen.hpp:94-111); with beta, p is rescaled to beta * B0^2 / 2."""
    g = Grid(n, n, 1, ng, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0)
    b0 = 1.0 / math.sqrt(4.0 * math.pi)

    def A(c, x, y, z):
        if c != 2:
            return np.zeros(np.broadcast_shapes(np.shape(x), np.shape(y), np.shape(z)))
        return b0 / (2.0 * math.pi) * np.cos(2.0 * math.pi * y) + b0 / (4.0 * math.pi) * np.cos(4.0 * math.pi * x)

    b1, b2, b3 = _curl_faces(g, A)
    shp = (g.nk, g.nj, g.ni)
    x, y = g.x1v()[None, None, :], g.x2v()[None, :, None]
    d = np.full(shp, 25.0 / (36.0 * math.pi))
    vx = np.broadcast_to(-np.sin(2.0 * math.pi * y), shp)
    vy = np.broadcast_to(np.sin(2.0 * math.pi * x), shp)
    p0 = 5.0 / (12.0 * math.pi) if beta is None else beta * b0 * b0 / 2.0
    p = np.full(shp, p0)
    u = _conserve(g, d, vx, vy, np.zeros(shp), p, b1, b2, b3, gamma)
    return g, u, b1, b2, b3


# ---- reference restart format (src/restart.hpp:11-56) ------------------------------------
_HDR = struct.Struct("<6i d i 4x")   # magic nx1 nx2 nx3 ng cycle | time | real_size | pad: 40 bytes
MAGIC = 0x43485351


def write_restart(fname: str, g: Grid, u, b1, b2, b3, time: float = 0.0, cycle: int = 0) -> None:
    with open(fname, "wb") as f:
        f.write(_HDR.pack(MAGIC, g.nx1, g.nx2, g.nx3, g.ng, cycle, time, 8))
        for a in (u, b1, b2, b3):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


def read_restart(fname: str):
    with open(fname, "rb") as f:
        magic, nx1, nx2, nx3, ng, cycle, time, rs = _HDR.unpack(f.read(_HDR.size))
        if magic != MAGIC:
            raise ValueError("not a Chasqui restart file: " + fname)
        if rs != 8:
            raise ValueError("restart file precision is not double")
        ni = nx1 + 2 * ng
        nj = nx2 + 2 * ng if nx2 > 1 else 1
        nk = nx3 + 2 * ng if nx3 > 1 else 1
        nc = 6 * nk * nj * ni
        nf = (nk + 1) * (nj + 1) * (ni + 1)
        data = np.frombuffer(f.read(8 * (nc + 3 * nf)), dtype="<f8")
    u = data[:nc].reshape(6, nk, nj, ni).copy()
    bs = [data[nc + q * nf: nc + (q + 1) * nf].reshape(nk + 1, nj + 1, ni + 1).copy() for q in range(3)]
    return dict(nx=(nx1, nx2, nx3), ng=ng, cycle=cycle, time=time, u=u, b1=bs[0], b2=bs[1], b3=bs[2])
