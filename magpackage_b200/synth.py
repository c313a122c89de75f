"""Seeded synthetic tetrahedral meshes and region layouts.

The reference ships no assembly benchmark meshes, so every workload is a
jittered box: ``nx x ny x nz`` hexahedra, each split into the 6 Kuhn
tetrahedra (one per ordering of the three axes, all sharing the (0,0,0)-(1,1,1)
diagonal, so the split is conforming). Nodes are jittered by U(-j h, +j h) per
coordinate from a seeded PCG64 stream; boundary nodes move only tangentially
so the box keeps its faces.

Layout (MATLAB-compatible memory order):
  P  float64 (Nn, 3)  == MATLAB [3 x Nn] column-major
  T  int32   (Ne, 4)  0-based node ids == MATLAB [4 x Ne] (1-based there)
Node (i,j,k) has id i + (nx+1)(j + (ny+1)k); hexahedra are numbered the same
way and element 6h+t is tetrahedron t of hexahedron h.

Region tags (1-based, like MATLAB RegionTags): 1 air, 2 iron, 3 aluminium,
4 coil. The workloads:
  cube_layout    -- unit cube; iron = centre 0.4^3 block; aluminium = slab
                    z in [0.1, 0.2]; tagging by element centroid.
  ecore_layout   -- 0.4 x 0.4 x 0.2 m box with an E-shaped iron core (three
                    legs joined by two yokes) and a rectangular coil box around
                    the centre leg.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

AIR, IRON, ALUMINIUM, COIL = 1, 2, 3, 4

_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


@dataclass
class BoxMesh:
    P: np.ndarray  # (Nn, 3) float64
    T: np.ndarray  # (Ne, 4) int32, 0-based
    shape: tuple
    size: tuple

    @property
    def num_nodes(self):
        return self.P.shape[0]

    @property
    def num_elements(self):
        return self.T.shape[0]

    def centroids(self) -> np.ndarray:
        c = np.zeros((self.num_elements, 3))
        for a in range(4):
            c += self.P[self.T[:, a]]
        return c * 0.25


def kuhn_box(nx: int, ny: int | None = None, nz: int | None = None, size=(1.0, 1.0, 1.0),
             jitter: float = 0.1, seed: int = 0) -> BoxMesh:
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    sx, sy, sz = (float(s) for s in size)
    hx, hy, hz = sx / nx, sy / ny, sz / nz
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    # node id = i + (nx+1)*(j + (ny+1)*k): order arrays with i fastest
    ii, jj, kk = (a.transpose(2, 1, 0).ravel() for a in (ii, jj, kk))
    P = np.stack([ii * hx, jj * hy, kk * hz], axis=1)
    if jitter:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter, jitter, size=P.shape) * np.array([hx, hy, hz])
        d[(ii == 0) | (ii == nx), 0] = 0.0
        d[(jj == 0) | (jj == ny), 1] = 0.0
        d[(kk == 0) | (kk == nz), 2] = 0.0
        P = P + d
    hi, hj, hk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    hi, hj, hk = (a.transpose(2, 1, 0).ravel().astype(np.int64) for a in (hi, hj, hk))
    sxn, syn = nx + 1, (nx + 1) * (ny + 1)
    base = hi + sxn * hj + syn * hk
    step = np.array([1, sxn, syn], dtype=np.int64)
    T = np.empty((hi.size, 6, 4), dtype=np.int64)
    for t, perm in enumerate(_PERMS):
        v = base.copy()
        T[:, t, 0] = v
        for a in range(3):
            v = v + step[perm[a]]
            T[:, t, a + 1] = v
    T = T.reshape(-1, 4)
    if T.max() >= 2 ** 31:
        raise ValueError("mesh too large for int32 node ids")
    return BoxMesh(P=P, T=T.astype(np.int32), shape=(nx, ny, nz), size=(sx, sy, sz))


def cube_layout(mesh: BoxMesh, iron=(0.3, 0.7), al_z=(0.1, 0.2)) -> np.ndarray:
    """Config-1 style tags: iron centre block, aluminium slab, air elsewhere."""
    c = mesh.centroids() / np.array(mesh.size)
    tags = np.full(mesh.num_elements, AIR, dtype=np.int32)
    in_al = (c[:, 2] >= al_z[0]) & (c[:, 2] <= al_z[1])
    tags[in_al] = ALUMINIUM
    in_fe = np.all((c >= iron[0]) & (c <= iron[1]), axis=1)
    tags[in_fe] = IRON
    return tags


def random_box_layout(mesh: BoxMesh, rng: np.random.Generator) -> np.ndarray:
    """Per-instance iron block and aluminium slab at seeded random positions."""
    c = mesh.centroids() / np.array(mesh.size)
    lo = rng.uniform(0.15, 0.45, size=3)
    ext = rng.uniform(0.2, 0.4, size=3)
    z0 = rng.uniform(0.02, 0.1)
    tags = np.full(mesh.num_elements, AIR, dtype=np.int32)
    tags[(c[:, 2] >= z0) & (c[:, 2] <= z0 + 0.1)] = ALUMINIUM
    tags[np.all((c >= lo) & (c <= lo + ext), axis=1)] = IRON
    return tags


def ecore_layout(mesh: BoxMesh):
    """E-core iron region and coil box in a 0.4 x 0.4 x 0.2 m box.

    Returns (tags, coil_mask). The core lies in the x-y plane between
    z = 0.06 and z = 0.14 m: three legs along y (x in [0.08,0.12], [0.18,0.22],
    [0.28,0.32]) joined by yokes (y in [0.06,0.10] and [0.30,0.34]); the coil is
    the box x in [0.13,0.17] U [0.23,0.27], y in [0.12,0.28] around the centre leg.
    """
    c = mesh.centroids()
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    slab = (z >= 0.06) & (z <= 0.14)
    legs = ((x >= 0.08) & (x <= 0.12)) | ((x >= 0.18) & (x <= 0.22)) | ((x >= 0.28) & (x <= 0.32))
    leg_span = (y >= 0.06) & (y <= 0.34)
    yokes = (((y >= 0.06) & (y <= 0.10)) | ((y >= 0.30) & (y <= 0.34))) & (x >= 0.08) & (x <= 0.32)
    iron = slab & ((legs & leg_span) | yokes)
    coil = slab & (((x > 0.13) & (x < 0.17)) | ((x > 0.23) & (x < 0.27))) & (y > 0.12) & (y < 0.28)
    tags = np.full(mesh.num_elements, AIR, dtype=np.int32)
    tags[iron] = IRON
    tags[coil & ~iron] = COIL
    return tags, coil & ~iron


# Coil of the transient workload: a rectangular winding around the E-core's centre
# leg. In the x-z plane it is the ring between the outer box [0.13,0.27]x[0.01,0.19]
# and the window [0.17,0.23]x[0.05,0.15] (the window holds the leg with a gap);
# along y it spans [0.12,0.28], its current fading linearly over the first and last
# 0.02 m.
COIL_OUTER = ((0.13, 0.27), (0.01, 0.19))
COIL_WINDOW = ((0.17, 0.23), (0.05, 0.15))
COIL_Y = (0.12, 0.28)
COIL_RAMP = 0.02


def ecore_coil_layout(mesh: BoxMesh) -> np.ndarray:
    """Tags for the transient workload: E-core iron, ring coil around the centre leg, air."""
    tags, _ = ecore_layout(mesh)
    tags[tags == COIL] = AIR
    c = mesh.centroids()
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    (ox0, ox1), (oz0, oz1) = COIL_OUTER
    (wx0, wx1), (wz0, wz1) = COIL_WINDOW
    outer = (x > ox0) & (x < ox1) & (z > oz0) & (z < oz1)
    window = (x > wx0) & (x < wx1) & (z > wz0) & (z < wz1)
    ring = outer & ~window & (y > COIL_Y[0]) & (y < COIL_Y[1])
    tags[ring & (tags == AIR)] = COIL
    return tags


def _ring_phi(x, z):
    """0 outside the ring's outer box, 1 in the window, linear across the 0.04 m wall."""
    (ox0, ox1), (oz0, oz1) = COIL_OUTER
    w = COIL_WINDOW[0][0] - ox0
    d = np.minimum(np.minimum(x - ox0, ox1 - x), np.minimum(z - oz0, oz1 - z))
    return np.clip(d / w, 0.0, 1.0), w


def _ramp_integral(y):
    """X(y) = integral from 0 to y of the coil's axial profile chi (0 -> 1 -> 0 along y)."""
    y0, y1 = COIL_Y
    r = COIL_RAMP
    y = np.clip(np.asarray(y, dtype=np.float64), y0, y1)
    up = np.minimum(y - y0, r)
    X = up * up / (2 * r)                                   # rising ramp
    X = X + np.clip(y - (y0 + r), 0.0, (y1 - r) - (y0 + r))  # plateau
    down = np.clip(y - (y1 - r), 0.0, r)
    return X + down - down * down / (2 * r)                 # falling ramp


def coil_edge_values(P: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """Edge values t_e of a current vector potential T = w phi(x, z) chi(y) e_y.

    J = curl T = w chi (-d phi/dz, 0, d phi/dx) has unit magnitude in the ring
    walls (where chi = 1), circulates around the centre leg and vanishes in the
    window. t_e = w phi(midpoint) (X(y_b) - X(y_a)) with X the antiderivative of
    chi: on edges inside the window (phi = 1) that is the exact increment of a
    potential, so the discrete current, the element curl of t, is exactly zero
    there, and being a curl it is exactly divergence-free everywhere.
    """
    a, b = P[edges[:, 0]], P[edges[:, 1]]
    mid = 0.5 * (a + b)
    phi, w = _ring_phi(mid[:, 0], mid[:, 2])
    return w * phi * (_ramp_integral(b[:, 1]) - _ramp_integral(a[:, 1]))


def standard_materials(iron_nonlinear: bool = True):
    """Material map used by the workloads: air/aluminium/coil linear, iron Froehlich."""
    from .material import NU0, create_linear_nu, create_nonlinear, froehlich_bh

    iron = create_nonlinear(*froehlich_bh()) if iron_nonlinear else create_linear_nu(NU0 / 1000.0)
    return {AIR: create_linear_nu(NU0), IRON: iron, ALUMINIUM: create_linear_nu(NU0),
            COIL: create_linear_nu(NU0)}


SIGMA_AL = 3.526e7


def frequency_sweep_sizes(count: int = 64, n_min: int = 8, n_max: int = 48) -> list[int]:
    """Tetrahedra of each instance of frequency_sweep_instances (6 n_k^3), without building
    the meshes."""
    out = []
    for k in range(count):
        t = k / max(count - 1, 1)
        n = int(round(n_min + (n_max - n_min) * t))
        out.append(6 * n ** 3)
    return out


def frequency_sweep_instances(count: int = 64, n_min: int = 8, n_max: int = 48, f_min: float = 10.0,
                              f_max: float = 1e4, seed: int = 0):
    """Independent jittered cubes of uneven size for the batched complex workload.

    Instance k has n_k = round(n_min + (n_max - n_min) k / (count - 1)) hexahedra per
    side (6 tetrahedra each), its own seeded jitter and region boxes, and frequency
    f_k = f_min * (f_max / f_min)^(k / (count - 1)). Yields (mesh, tags, nu, sigma, omega).
    """
    from .material import NU0

    rng = np.random.default_rng(seed)
    for k in range(count):
        t = k / max(count - 1, 1)
        n = int(round(n_min + (n_max - n_min) * t))
        mesh = kuhn_box(n, seed=seed * 1000 + k)
        tags = random_box_layout(mesh, rng)
        nu = np.where(tags == IRON, NU0 / 1000.0, NU0)
        sigma = np.where(tags == ALUMINIUM, SIGMA_AL, 0.0)
        omega = 2.0 * np.pi * f_min * (f_max / f_min) ** t
        yield mesh, tags, nu, sigma, omega
