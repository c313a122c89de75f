"""Reference-element data for first-order Nedelec tetrahedra.

Restates the two MATLAB helpers whose outputs the reference passes to its MEX
kernels on every assembly call (Assembler.m:30-32,191-193):

* ``get_quadrature_data('tet', order)`` -- src/utils/get_quadrature_data.m:1-32.
  Order <= 1 is the centroid rule (w = 1/6); otherwise the 4-point rule with the
  reference's 8-digit literals a = 0.58541020, b = 0.13819660 and w = 1/24.
* ``nedelec_tet_p1(q_pts)`` -- src/shape_functions/nedelec_tet_p1.m:1-51 with
  the Lagrange P1 data of src/shape_functions/lagrange_tet_p1.m:1-39. Whitney
  values ``W_e = L_i grad(L_j) - L_j grad(L_i)`` and constant reference curls
  ``2 grad(L_i) x grad(L_j)`` for the local edges (1,2),(1,3),(1,4),(2,3),(2,4),(3,4).

Both arrays are returned flattened in MATLAB column-major order, so entry
(basis i, component c, point q) sits at ``i + 6*c + 18*q`` exactly as the MEX
kernels index them (assemble_curl_curl_kernel_mex.cpp:72-82).
"""
from __future__ import annotations

import numpy as np

LOCAL_EDGES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
_GRAD = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def get_quadrature_data(elem_type: str = "tet", order: int = 2):
    """Return ``(q_pts [3 x nq], q_w [nq])`` (get_quadrature_data.m:18-28)."""
    if elem_type.lower() != "tet":
        raise ValueError(f"Unsupported element type: {elem_type}")
    if order <= 1:
        return np.array([[0.25], [0.25], [0.25]]), np.array([1.0 / 6.0])
    a, b = 0.58541020, 0.13819660
    q_pts = np.array([[a, b, b, b], [b, a, b, b], [b, b, a, b]])
    return q_pts, np.full(4, 1.0 / 24.0)


def _lagrange_values(q_pts: np.ndarray) -> np.ndarray:
    xi, eta, zeta = q_pts
    # lagrange_tet_p1.m:20-24; N1 evaluated left to right as in MATLAB
    return np.stack([((1.0 - xi) - eta) - zeta, xi, eta, zeta])


def nedelec_tet_p1(q_pts: np.ndarray):
    """Return ``(val_ref, curl_ref)``, each flattened [6 x 3 x nq] column-major."""
    q_pts = np.asarray(q_pts, dtype=np.float64)
    nq = q_pts.shape[1]
    lam = _lagrange_values(q_pts)
    val = np.zeros((6, 3, nq))
    curl = np.zeros((6, 3, nq))
    for e, (i, j) in enumerate(LOCAL_EDGES):
        gi, gj = _GRAD[i], _GRAD[j]
        # val(e,c,p) = Li(p)*Gj(c) - Lj(p)*Gi(c)   (nedelec_tet_p1.m:39-44)
        val[e] = gj[:, None] * lam[i][None, :] - gi[:, None] * lam[j][None, :]
        curl[e] = (2.0 * np.cross(gi, gj))[:, None]
    return val.flatten(order="F"), curl.flatten(order="F")


def reference_data(order: int = 2):
    """Quadrature weights plus basis values and curls, as Assembler.m prepares them."""
    q_pts, q_w = get_quadrature_data("tet", order)
    val, curl = nedelec_tet_p1(q_pts)
    return q_w, val, curl
