"""Material tables for the assembly kernels (host-side setup).

Restates the reference's material handling that produces the kernel inputs:

* ``create_linear`` -- src/MaterialLib.m:58-63.
* ``create_nonlinear`` -- src/MaterialLib.m:65-125: sort/unique the B-H samples,
  nu = H/B (nu(1) = nu(2) when B(1) = 0), append the vacuum-guide point
  (B^2_end + 0.1, nu_end + (nu0 - nu_end)/(2 B_end^2) * 0.1, capped at nu0),
  MaxBSq = last B^2, then a monotone piecewise-cubic Hermite table nu(B^2).
* ``pchip`` -- MATLAB's pchip as called at MaterialLib.m:117. MATLAB is absent,
  so this follows its published algorithm (Fritsch-Carlson slopes with the
  scaled weighted harmonic mean, shape-preserving three-point end slopes,
  coefficients highest power first).
* ``pack_material_data`` -- src/Assembler.m:270-304: the eight SoA arrays the
  Jacobian kernel reads, indexed by tag-1, plus the concatenated breaks and
  coefficients.
* ``froehlich_bh`` -- the synthetic iron curve B = mu0 H + 1.8 H / (150 + |H|)
  on H = 0 plus 199 log-spaced points in [1, 2e5] A/m.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MU0 = 4.0 * np.pi * 1e-7
NU0 = 1.0 / MU0


@dataclass
class Material:
    kind: str  # 'Linear' | 'Nonlinear'
    nu0: float = NU0
    nu_linear: float = NU0
    breaks: np.ndarray | None = None
    coefs: np.ndarray | None = None  # [pieces x 4], highest power first
    max_bsq: float = 1e10
    extra: dict = field(default_factory=dict)


def create_linear(mu_r: float) -> Material:
    """MaterialLib.createLinear (MaterialLib.m:58-63)."""
    return Material(kind="Linear", nu0=1.0 / MU0, nu_linear=1.0 / (mu_r * MU0))


def create_linear_nu(nu: float) -> Material:
    """A linear material given directly by its reluctivity."""
    return Material(kind="Linear", nu0=1.0 / MU0, nu_linear=float(nu))


def _sgn(v):
    return int(v > 0) - int(v < 0)


def pchip(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Piecewise cubic Hermite coefficients [n-1 x 4] (highest power first)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = x.size
    if n < 2:
        raise ValueError("pchip needs at least two points")
    h = np.diff(x)
    if np.any(h <= 0):
        raise ValueError("pchip breaks must be strictly increasing")
    dl = np.diff(y) / h
    d = np.zeros(n)
    if n == 2:
        d[:] = dl[0]
    else:
        for k in range(n - 2):
            if _sgn(dl[k]) * _sgn(dl[k + 1]) > 0:
                hs = h[k] + h[k + 1]
                w1 = (h[k] + hs) / (3 * hs)
                w2 = (hs + h[k + 1]) / (3 * hs)
                a, b = abs(dl[k]), abs(dl[k + 1])
                dmax, dmin = max(a, b), min(a, b)
                d[k + 1] = dmin / (w1 * (dl[k] / dmax) + w2 * (dl[k + 1] / dmax))

        def end(h1, h2, d1, d2):
            s = ((2 * h1 + h2) * d1 - h1 * d2) / (h1 + h2)
            if _sgn(s) != _sgn(d1):
                return 0.0
            if _sgn(d1) != _sgn(d2) and abs(s) > abs(3 * d1):
                return 3 * d1
            return s

        d[0] = end(h[0], h[1], dl[0], dl[1])
        d[-1] = end(h[-1], h[-2], dl[-1], dl[-2])
    a = (dl - d[:-1]) / h
    b = (d[1:] - dl) / h
    return np.stack([(b - a) / h, 2 * a - b, d[:-1], y[:-1]], axis=1)


def create_nonlinear(b_curve, h_curve) -> Material:
    """MaterialLib.createNonlinear (MaterialLib.m:65-125)."""
    b = np.abs(np.asarray(b_curve, dtype=np.float64).ravel())
    h = np.abs(np.asarray(h_curve, dtype=np.float64).ravel())
    order = np.argsort(b, kind="stable")
    b, h = b[order], h[order]
    # unique(B, 'last'): sorted distinct values, index of the last occurrence
    last = np.r_[b[1:] != b[:-1], True]
    b_u, h_u = b[last], h[last]
    bsq = b_u ** 2
    nu = np.zeros_like(b_u)
    nz = b_u > 1e-12
    nu[nz] = h_u[nz] / b_u[nz]
    if not nz[0]:
        nu[0] = nu[1] if b_u.size > 1 else NU0
    if bsq.size > 2:
        b_end, nu_end = b_u[-1], nu[-1]
        slope = (NU0 - nu_end) / (2 * b_end ** 2)
        bsq_new = bsq[-1] + 0.1
        nu_new = min(nu_end + slope * 0.1, NU0)
        bsq = np.r_[bsq, bsq_new]
        nu = np.r_[nu, nu_new]
    mat = Material(kind="Nonlinear", nu0=NU0, nu_linear=NU0, max_bsq=float(bsq.max()))
    if bsq.size > 1:
        mat.coefs = pchip(bsq, nu)
        mat.breaks = bsq.copy()
    else:
        mat.coefs = np.array([[0.0, 0.0, 0.0, nu[0]]])
        mat.breaks = np.r_[bsq, bsq + 1.0]
    mat.extra["B_data"], mat.extra["H_data"] = b_u, h_u
    return mat


def froehlich_bh(n_points: int = 200, h_max: float = 2e5):
    """Froehlich iron curve B = mu0 H + 1.8 H/(150 + |H|) on 0 + log-spaced H."""
    h = np.r_[0.0, np.logspace(0.0, np.log10(h_max), n_points - 1)]
    b = MU0 * h + 1.8 * h / (150.0 + np.abs(h))
    return b, h


@dataclass
class PackedMaterials:
    """The eight arrays of Assembler.packMaterialData, index = tag - 1."""

    lin: np.ndarray
    is_non: np.ndarray
    max_b: np.ndarray
    breaks: np.ndarray
    coefs: np.ndarray
    start: np.ndarray
    count: np.ndarray
    coe_start: np.ndarray

    def as_tuple(self):
        return (self.lin, self.is_non, self.max_b, self.breaks, self.coefs, self.start,
                self.count, self.coe_start)


def pack_material_data(matlib: dict) -> PackedMaterials:
    """Assembler.packMaterialData (Assembler.m:270-304); keys are 1-based tags."""
    keys = sorted(k for k in matlib)
    max_tag = max(keys)
    n = max_tag + 1
    lin, is_non, max_b = np.zeros(n), np.zeros(n), np.zeros(n)
    start, count, coe_start = np.zeros(n), np.zeros(n), np.zeros(n)
    brk_parts, coe_parts = [], []
    b_ptr = c_ptr = 0
    for tag in keys:
        if tag <= 0:
            continue
        m = matlib[tag]
        if m.kind == "Linear":
            lin[tag - 1] = m.nu_linear
            is_non[tag - 1] = 0.0
        else:
            lin[tag - 1] = m.nu0
            is_non[tag - 1] = 1.0
            max_b[tag - 1] = m.max_bsq if m.max_bsq is not None else 1e10
            nb, nc = m.breaks.size, m.coefs.size
            start[tag - 1], count[tag - 1], coe_start[tag - 1] = b_ptr, nb - 1, c_ptr
            brk_parts.append(m.breaks.astype(np.float64))
            coe_parts.append(np.ascontiguousarray(m.coefs, dtype=np.float64).ravel())
            b_ptr += nb
            c_ptr += nc
    breaks = np.concatenate(brk_parts) if brk_parts else np.zeros(0)
    coefs = np.concatenate(coe_parts) if coe_parts else np.zeros(0)
    return PackedMaterials(lin, is_non, max_b, breaks, coefs, start, count, coe_start)
