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


def standard_materials(iron_nonlinear: bool = True):
    """Material map used by the workloads: air/aluminium/coil linear, iron Froehlich."""
    from .material import NU0, create_linear_nu, create_nonlinear, froehlich_bh

    iron = create_nonlinear(*froehlich_bh()) if iron_nonlinear else create_linear_nu(NU0 / 1000.0)
    return {AIR: create_linear_nu(NU0), IRON: iron, ALUMINIUM: create_linear_nu(NU0),
            COIL: create_linear_nu(NU0)}


SIGMA_AL = 3.526e7


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
