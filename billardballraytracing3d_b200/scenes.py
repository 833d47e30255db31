"""Seeded synthetic scenes and ray sources in the reference's patch format.

The reference ships no geometry: its patches come from the external IFGF-RP
pipeline as one whitespace-separated ``.txt`` file per patch, read by
``SurfacePatch::load_patch_file`` (include/ScatObjects/SurfacePatch.hpp:313-371).
This module builds closed obstacles (spheres and rotated ellipsoids) as
cubed-sphere patch sets in that format, with exact node positions, exact
first derivatives and exact outward unit normals, plus the ray sources the
benchmark workloads use.

Determinism: every number is produced with IEEE-754 double ``+ - * /`` and
``sqrt`` only (elementwise numpy, no BLAS, no reductions, no libm
transcendental).  Cosines and sines come from a fixed Taylor evaluation, so a
scene generated on any x86-64 or aarch64 host is bit-identical; the random
streams come from numpy's PCG64, which is platform independent.

Geometry choices (the reference leaves them open):
  * cubed sphere, gnomonic map: a face is the cube square [-1,1]^2, cut into
    m x m equal squares; a patch's parameter square [-1,1]^2 maps linearly
    onto one of those squares and the cube point is projected to the sphere;
  * interpolation nodes: Chebyshev-Lobatto points, ascending, the same set
    for u and v;
  * node layout: row-major, flat index i*jmax + j with i the u index
    (SurfacePatch.hpp:549); zoneID = obstacle * 100000 + patch index.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# deterministic trigonometry (fixed Taylor series; IEEE ops only)
# ---------------------------------------------------------------------------
_PI = 3.141592653589793
_HALF_PI = 1.5707963267948966
_QUARTER_PI = 0.7853981633974483
_TWO_PI = 6.283185307179586

# 1/k! for the even and odd Taylor terms, as exact quotients evaluated once.
_INV_FACT = [1.0]
for _k in range(1, 30):
    _INV_FACT.append(_INV_FACT[-1] / float(_k))


_COS_COEF = [(-1.0) ** n * _INV_FACT[2 * n] for n in range(14)]      # (-1)^n / (2n)!
_SIN_COEF = [(-1.0) ** n * _INV_FACT[2 * n + 1] for n in range(13)]  # (-1)^n / (2n+1)!


def _cos_small(x):
    """cos(x) for |x| <= pi/4: Horner in x^2 over 14 Taylor terms (floats or arrays)."""
    x2 = x * x
    c = _COS_COEF[-1]
    for a in reversed(_COS_COEF[:-1]):
        c = c * x2 + a
    return c


def _sin_small(x):
    """sin(x) for |x| <= pi/4: x times Horner in x^2 over 13 Taylor terms."""
    x2 = x * x
    s = _SIN_COEF[-1]
    for a in reversed(_SIN_COEF[:-1]):
        s = s * x2 + a
    return s * x


def det_sincos(theta):
    """(sin, cos) of theta (float or float64 array) with IEEE ops only.

    Reduction: theta -> r in [-pi/4, pi/4] plus a quadrant, using a fixed
    two-constant Cody-Waite split of pi/2.  Accurate to a few ulp for
    |theta| < 1e4, which covers every use here (angles below 2*pi).
    """
    th = np.asarray(theta, dtype=np.float64)
    q = np.floor(th / _HALF_PI + 0.5)
    # pi/2 = C1 + C2 with C1 holding 33 bits so q*C1 is exact for |q| < 2^20
    c1 = 1.5707963267341256
    c2 = 6.077100506506192e-11
    r = (th - q * c1) - q * c2
    s = _sin_small(r)
    c = _cos_small(r)
    qi = np.mod(q.astype(np.int64), 4)
    sin_out = np.where(qi == 0, s, np.where(qi == 1, c, np.where(qi == 2, -s, -c)))
    cos_out = np.where(qi == 0, c, np.where(qi == 1, -s, np.where(qi == 2, -c, s)))
    if np.ndim(theta) == 0:
        return float(sin_out), float(cos_out)
    return sin_out, cos_out


def det_cos(theta):
    return det_sincos(theta)[1]


def det_sin(theta):
    return det_sincos(theta)[0]


def cheb_lobatto(n: int) -> np.ndarray:
    """Ascending Chebyshev-Lobatto nodes -cos(pi k/(n-1)), exactly antisymmetric."""
    if n < 2:
        raise ValueError("need at least 2 nodes")
    x = np.empty(n)
    for k in range(n):
        if 2 * k < n - 1:
            x[k] = -det_cos(_PI * float(k) / float(n - 1))
        elif 2 * k == n - 1:
            x[k] = 0.0
        else:
            x[k] = -x[n - 1 - k]
    x[0], x[-1] = -1.0, 1.0
    return x


# ---------------------------------------------------------------------------
# patches
# ---------------------------------------------------------------------------
@dataclass
class Patch:
    """One patch file's payload (SurfacePatch::Data, SurfacePatch.hpp:59-89)."""
    imax: int
    jmax: int
    zone_id: int
    u_nodes: np.ndarray
    v_nodes: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    dxdu: np.ndarray
    dydu: np.ndarray
    dzdu: np.ndarray
    dxdv: np.ndarray
    dydv: np.ndarray
    dzdv: np.ndarray
    dS: np.ndarray
    nu_x: np.ndarray
    nu_y: np.ndarray
    nu_z: np.ndarray
    kmax: int = 1
    mask: np.ndarray = None
    edge_flags: Tuple[int, int, int, int] = None

    FIELDS = ("x", "y", "z", "dxdu", "dydu", "dzdu", "dxdv", "dydv", "dzdv",
              "dS", "nu_x", "nu_y", "nu_z")

    def __post_init__(self):
        n = self.imax * self.jmax * self.kmax
        if self.mask is None:
            self.mask = np.ones(n, dtype=np.int64)
        for f in self.FIELDS:
            a = np.ascontiguousarray(getattr(self, f), dtype=np.float64).reshape(-1)
            if a.size != n:
                raise ValueError(f"field {f} has {a.size} values, expected {n}")
            setattr(self, f, a)
        self.u_nodes = np.ascontiguousarray(self.u_nodes, dtype=np.float64)
        self.v_nodes = np.ascontiguousarray(self.v_nodes, dtype=np.float64)


# Face frames (normal axis, t1, t2) with t1 x t2 = normal, so the (u, v)
# orientation is outward on every face.
_FACES = (
    ((1, 0, 0), (0, 1, 0), (0, 0, 1)),
    ((-1, 0, 0), (0, 0, 1), (0, 1, 0)),
    ((0, 1, 0), (0, 0, 1), (1, 0, 0)),
    ((0, -1, 0), (1, 0, 0), (0, 0, 1)),
    ((0, 0, 1), (1, 0, 0), (0, 1, 0)),
    ((0, 0, -1), (0, 1, 0), (1, 0, 0)),
)


def _matvec(q, a):
    """q (3x3 nested floats) times a (tuple of 3 arrays), fixed summation order."""
    return tuple((q[r][0] * a[0] + q[r][1] * a[1]) + q[r][2] * a[2] for r in range(3))


def obstacle_patches(obstacle: int, center: Sequence[float], semi_axes: Sequence[float],
                     rotation, m: int, n_nodes: int) -> List[Patch]:
    """6*m*m cubed-sphere patches of the ellipsoid c + Q diag(A) s, |s| = 1.

    A sphere of radius R is semi_axes = (R, R, R) with rotation = None.
    """
    nodes = cheb_lobatto(n_nodes)
    uu = np.repeat(nodes, n_nodes)        # u index i is the slow one: idx = i*jmax + j
    vv = np.tile(nodes, n_nodes)
    A = [float(a) for a in semi_axes]
    c = [float(v) for v in center]
    q = rotation if rotation is not None else ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0))
    patches = []
    for f, (nrm, t1, t2) in enumerate(_FACES):
        for pa in range(m):
            for pb in range(m):
                a0 = -1.0 + 2.0 * float(pa) / float(m)
                a1 = -1.0 + 2.0 * float(pa + 1) / float(m)
                b0 = -1.0 + 2.0 * float(pb) / float(m)
                b1 = -1.0 + 2.0 * float(pb + 1) / float(m)
                am, ah = 0.5 * (a0 + a1), 0.5 * (a1 - a0)
                bm, bh = 0.5 * (b0 + b1), 0.5 * (b1 - b0)
                a = am + ah * uu
                b = bm + bh * vv
                w = tuple(float(nrm[k]) + a * float(t1[k]) + b * float(t2[k]) for k in range(3))
                r = np.sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2])
                s = tuple(w[k] / r for k in range(3))
                st1 = (s[0] * float(t1[0]) + s[1] * float(t1[1])) + s[2] * float(t1[2])
                st2 = (s[0] * float(t2[0]) + s[1] * float(t2[1])) + s[2] * float(t2[2])
                s_u = tuple(ah * ((float(t1[k]) - s[k] * st1) / r) for k in range(3))
                s_v = tuple(bh * ((float(t2[k]) - s[k] * st2) / r) for k in range(3))
                loc = tuple(A[k] * s[k] for k in range(3))
                loc_u = tuple(A[k] * s_u[k] for k in range(3))
                loc_v = tuple(A[k] * s_v[k] for k in range(3))
                nloc = tuple(s[k] / A[k] for k in range(3))
                X = _matvec(q, loc)
                X = tuple(c[k] + X[k] for k in range(3))
                Xu = _matvec(q, loc_u)
                Xv = _matvec(q, loc_v)
                nw = _matvec(q, nloc)
                nl = np.sqrt((nw[0] * nw[0] + nw[1] * nw[1]) + nw[2] * nw[2])
                nu = tuple(nw[k] / nl for k in range(3))
                cr = (Xu[1] * Xv[2] - Xu[2] * Xv[1],
                      Xu[2] * Xv[0] - Xu[0] * Xv[2],
                      Xu[0] * Xv[1] - Xu[1] * Xv[0])
                dS = np.sqrt((cr[0] * cr[0] + cr[1] * cr[1]) + cr[2] * cr[2])
                idx = (f * m + pa) * m + pb
                patches.append(Patch(
                    imax=n_nodes, jmax=n_nodes, zone_id=obstacle * 100000 + idx,
                    u_nodes=nodes.copy(), v_nodes=nodes.copy(),
                    x=X[0], y=X[1], z=X[2],
                    dxdu=Xu[0], dydu=Xu[1], dzdu=Xu[2],
                    dxdv=Xv[0], dydv=Xv[1], dzdv=Xv[2],
                    dS=dS, nu_x=nu[0], nu_y=nu[1], nu_z=nu[2]))
    return patches


# ---------------------------------------------------------------------------
# patch files (SurfacePatch::load_patch_file's format, SurfacePatch.hpp:313-371)
# ---------------------------------------------------------------------------
def _fmt(a) -> str:
    return " ".join(repr(float(v)) for v in a)


def write_patch_file(path: str, p: Patch) -> None:
    """Write one patch: header, u/v nodes, x y z, mask, 6 derivative fields,
    dS, 3 normal fields, then the optional sharp-edge block."""
    with open(path, "w") as fh:
        fh.write(f"{p.imax} {p.jmax} {p.kmax} {p.zone_id}\n")
        fh.write(_fmt(p.u_nodes) + "\n")
        fh.write(_fmt(p.v_nodes) + "\n")
        for f in ("x", "y", "z"):
            fh.write(_fmt(getattr(p, f)) + "\n")
        fh.write(" ".join(str(int(v)) for v in p.mask) + "\n")
        for f in ("dxdu", "dydu", "dzdu", "dxdv", "dydv", "dzdv", "dS", "nu_x", "nu_y", "nu_z"):
            fh.write(_fmt(getattr(p, f)) + "\n")
        if p.edge_flags is not None:
            fh.write(" ".join(str(int(v)) for v in p.edge_flags) + "\n")


def write_scene_dir(directory: str, patches: Sequence[Patch], prefix: str = "patch_") -> List[str]:
    """One file per patch; zero-padded names so the reference's sorted
    directory scan (RayTracingDriver.hpp:353-361) keeps this order."""
    os.makedirs(directory, exist_ok=True)
    paths = []
    for k, p in enumerate(patches):
        path = os.path.join(directory, f"{prefix}{k:06d}.txt")
        write_patch_file(path, p)
        paths.append(path)
    return paths


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def scene_two_spheres() -> List[Patch]:
    """Two unit spheres at (+-1.5, 0, 0); 6 x 4 x 4 = 96 patches each on 5x5 nodes."""
    out = []
    for k, cx in enumerate((-1.5, 1.5)):
        out += obstacle_patches(k, (cx, 0.0, 0.0), (1.0, 1.0, 1.0), None, m=4, n_nodes=5)
    return out


def tetrahedron_centers(edge: float = 2.5):
    """Vertices of a regular tetrahedron with the given edge, centred at the origin,
    one vertex at (+,+,+)."""
    s = edge / (2.0 * math.sqrt(2.0))
    return [(s, s, s), (s, -s, -s), (-s, s, -s), (-s, -s, s)]


def scene_tetra_spheres(m: int = 8, n_nodes: int = 7) -> List[Patch]:
    """Four unit spheres on a regular tetrahedron of edge 2.5; 6 x 8 x 8 = 384
    patches each on 7x7 nodes (degree 6)."""
    out = []
    for k, c in enumerate(tetrahedron_centers(2.5)):
        out += obstacle_patches(k, c, (1.0, 1.0, 1.0), None, m=m, n_nodes=n_nodes)
    return out


def _quat_rotation(rng) -> Tuple[Tuple[float, float, float], ...]:
    """Uniform random rotation: a rejection-sampled point of the unit 4-ball,
    normalised to S^3, turned into a rotation matrix."""
    while True:
        qv = rng.random(4) * 2.0 - 1.0
        n2 = ((qv[0] * qv[0] + qv[1] * qv[1]) + qv[2] * qv[2]) + qv[3] * qv[3]
        if 1e-6 < n2 <= 1.0:
            break
    n = math.sqrt(float(n2))
    w, x, y, z = (float(v) / n for v in qv)
    return ((1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w)),
            (2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w)),
            (2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)))


def random_ellipsoids(rng, count: int, box: float = 6.0, gap: float = 0.2,
                      axis_lo: float = 0.2, axis_hi: float = 1.2, max_tries: int = 100000):
    """`count` ellipsoids: semi-axes U[axis_lo, axis_hi], random rotation,
    centres rejection-sampled in [-box, box]^3 so that bounding spheres keep
    at least `gap` between them."""
    objs = []
    tries = 0
    while len(objs) < count:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place the ellipsoids")
        axes = tuple(float(v) for v in axis_lo + (axis_hi - axis_lo) * rng.random(3))
        rot = _quat_rotation(rng)
        rad = max(axes)
        cen = tuple(float(v) for v in (rng.random(3) * 2.0 - 1.0) * (box - rad))
        ok = True
        for (c2, a2, _) in objs:
            d2 = ((cen[0] - c2[0]) ** 2 + (cen[1] - c2[1]) ** 2) + (cen[2] - c2[2]) ** 2
            lim = rad + max(a2) + gap
            if d2 < lim * lim:
                ok = False
                break
        if ok:
            objs.append((cen, axes, rot))
    return objs


def scene_ellipsoids(seed: int = 2024, count: int = 16, m: int = 8, n_nodes: int = 7) -> List[Patch]:
    """16 random ellipsoids (semi-axes U[0.2,1.2], seeded rotations, centres in
    [-6,6]^3 with gap >= 0.2), 6 x 8 x 8 = 384 patches each, degree 6."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k, (cen, axes, rot) in enumerate(random_ellipsoids(rng, count)):
        out += obstacle_patches(k, cen, axes, rot, m=m, n_nodes=n_nodes)
    return out


# ---------------------------------------------------------------------------
# rays
# ---------------------------------------------------------------------------
def plane_grid(corner0, corner1, nx: int, ny: int) -> np.ndarray:
    """PlaneSourceDriver::build_plane_grid (PlaneSourceDriver.hpp:190-243),
    same arithmetic, returned as an (nx*ny, 3) array."""
    c0 = [float(v) for v in corner0]
    c1 = [float(v) for v in corner1]
    scale = max(1.0, *(abs(v) for v in c0 + c1))
    tol = 1e-9 * scale
    matches = [a for a in range(3) if abs(c0[a] - c1[a]) < tol]
    if len(matches) != 1:
        raise ValueError("corner0 and corner1 must agree in exactly one coordinate "
                         f"to define an axis-aligned plane (got {len(matches)} matching coordinates)")
    const = matches[-1]
    axa, axb = [a for a in range(3) if a != const]
    ga = [c0[axa] if nx == 1 else c0[axa] + (c1[axa] - c0[axa]) * float(i) / float(nx - 1) for i in range(nx)]
    gb = [c0[axb] if ny == 1 else c0[axb] + (c1[axb] - c0[axb]) * float(j) / float(ny - 1) for j in range(ny)]
    pts = np.empty((nx * ny, 3))
    pts[:, const] = c0[const]
    pts[:, axa] = np.repeat(np.array(ga), ny)
    pts[:, axb] = np.tile(np.array(gb), nx)
    return pts


def cone_rays(n: int, seed: int, plane_z: float, half_extent: float, cone_half_deg: float,
              axis_sign: float = -1.0) -> Tuple[np.ndarray, np.ndarray]:
    """n rays: origins uniform on [-h,h]^2 in the plane z = plane_z, unit
    directions uniform in solid angle within a cone of half-angle
    cone_half_deg about (0, 0, axis_sign)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.random((n, 4))
    o = np.empty((n, 3))
    o[:, 0] = -half_extent + (2.0 * half_extent) * u[:, 0]
    o[:, 1] = -half_extent + (2.0 * half_extent) * u[:, 1]
    o[:, 2] = plane_z
    cos_max = det_cos(cone_half_deg * (_PI / 180.0))
    mu = 1.0 - u[:, 2] * (1.0 - cos_max)
    st = np.sqrt(np.maximum(0.0, 1.0 - mu * mu))
    sp, cp = det_sincos(_TWO_PI * u[:, 3])
    d = np.empty((n, 3))
    d[:, 0] = st * cp
    d[:, 1] = st * sp
    d[:, 2] = axis_sign * mu
    return o, d


# ---------------------------------------------------------------------------
# named workloads
# ---------------------------------------------------------------------------
def multi_scene_workload(n_scenes: int, seed: int = 77, max_obstacles: int = 32, min_rays: int = 16384,
                         max_rays: int = 1 << 20):
    """Independent scenes of uneven size (the batched multi-scene case): each
    has a seeded count of 1..max_obstacles spheres or ellipsoids (semi-axes
    U[0.2,1.2], random rotations, centres in [-6,6]^3 with gap >= 0.2), each
    obstacle 6*4*4 = 96 or 6*8*8 = 384 patches of degree 4 (5x5 nodes) or 6
    (7x7), coarse grid 17x17, and a log-uniform count of rays in
    [min_rays, max_rays] from z = 8 over [-6,6]^2 in a 20-degree cone, <= 100
    bounces, Newton tolerance 1e-12.  Returns a list of
    (patches, origins, dirs, max_bounces, coarse_n, newton_tol)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(n_scenes):
        count = int(rng.integers(1, max_obstacles + 1))
        objs = random_ellipsoids(rng, count)
        patches = []
        for j, (cen, axes, rot) in enumerate(objs):
            if rng.random() < 0.5:   # sphere
                r = axes[0]
                axes, rot = (r, r, r), None
            m = 4 if rng.random() < 0.5 else 8
            nn = 5 if rng.random() < 0.5 else 7
            patches += obstacle_patches(j, cen, axes, rot, m=m, n_nodes=nn)
        n_rays = int(round(np.exp(rng.uniform(np.log(min_rays), np.log(max_rays)))))
        o, d = cone_rays(n_rays, int(rng.integers(1, 1 << 30)), 8.0, 6.0, 20.0)
        out.append((patches, o, d, 100, 17, 1e-12))
    return out


def workload(name: str, n_rays: int = None):
    """(patches, origins, dirs, max_bounces, coarse_n, newton_tol) of a named workload.

    two_spheres   : 2 spheres x 96 patches (5x5), 128x128 plane grid on z=4 over
                    [-3,3]^2, direction (0.3,0,-1), <=20 bounces, coarse n=9, tol 1e-12
    tetra_spheres : 4 spheres x 384 patches (7x7) on a tetrahedron of edge 2.5,
                    1024^2 seeded origins on [-3,3]^2 at z=5, 10 deg cone about -z,
                    <=200 bounces, coarse n=17, tol 1e-12
    ellipsoids    : 16 ellipsoids x 384 patches (7x7), 4M rays from z=8 over
                    [-6,6]^2 in a 20 deg cone, <=100 bounces, coarse n=17, tol 1e-12
    """
    if name == "two_spheres":
        pts = plane_grid((-3.0, -3.0, 4.0), (3.0, 3.0, 4.0), 128, 128)
        if n_rays is not None:
            pts = pts[:n_rays]
        dirs = np.tile(np.array([0.3, 0.0, -1.0]), (pts.shape[0], 1))
        return scene_two_spheres(), pts, dirs, 20, 9, 1e-12
    if name == "tetra_spheres":
        n = 1024 * 1024 if n_rays is None else n_rays
        o, d = cone_rays(n, 1234, 5.0, 3.0, 10.0)
        return scene_tetra_spheres(), o, d, 200, 17, 1e-12
    if name == "ellipsoids":
        n = 4 * 1024 * 1024 if n_rays is None else n_rays
        o, d = cone_rays(n, 4321, 8.0, 6.0, 20.0)
        return scene_ellipsoids(), o, d, 100, 17, 1e-12
    raise KeyError(name)
