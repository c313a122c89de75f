"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Two CPU implementations of the reference's element-assembly path:

* ``RefMex`` -- the reference's own MEX kernels (src/mex/assemble_*_kernel_mex.cpp)
  compiled unchanged into oracle/_ref/libref_mex.so by oracle/Makefile.
* ``Port``   -- the C restatement in oracle/port (libmagoracle.so), which also
  restates Mesh.generateEdges, MATLAB sparse() and pchip.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the reference results to compare with or the timed CPU baseline; the product path
never imports it. Inputs follow the reference's MEX boundary (Assembler.m):
column-major doubles with 1-based indices.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libref_mex.so")
PORT_SO = os.path.join(HERE, "libmagoracle.so")

_dp = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_i8p = C.POINTER(C.c_int8)


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# Where the reference tree is read when the oracle is built: $REF_ROOT, else the
# read-only mount of the reference in the build container.
REFERENCE_TREE = os.environ.get("REF_ROOT", "/root/reference")


def build(quiet: bool = True) -> None:
    """Build the oracle libraries (make -C oracle); the reference's own kernels too when
    its tree is present."""
    import subprocess

    args = ["make", "-C", HERE]
    if os.path.isdir(os.path.join(REFERENCE_TREE, "src", "mex")):
        args.append(f"REF_ROOT={REFERENCE_TREE}")
    out = subprocess.run(args, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)


@dataclass
class MexInputs:
    """Arguments exactly as Assembler.m passes them to the MEX gateways."""

    P: np.ndarray      # [3 x Nn] doubles (stored (Nn,3) C-order)
    T: np.ndarray      # [4 x Ne] 1-based doubles
    Dofs: np.ndarray   # [6 x Ne] 1-based doubles
    Signs: np.ndarray  # [6 x Ne] +-1 doubles
    Tags: np.ndarray   # [Ne] doubles

    @property
    def ne(self):
        return self.T.shape[0]

    @property
    def nn(self):
        return self.P.shape[0]


def _split(a):
    """Column-major real and imaginary parts of a 2-D array; None for a real array."""
    a = np.asarray(a)
    re = _f64(np.real(a).T.ravel())
    return re, (_f64(np.imag(a).T.ravel()) if np.iscomplexobj(a) else None)


def mex_inputs(P, T0, t2e0, sign, tags) -> MexInputs:
    """Convert 0-based int mesh arrays to the reference's double/1-based layout."""
    return MexInputs(P=_f64(P), T=_f64(np.asarray(T0) + 1), Dofs=_f64(np.asarray(t2e0) + 1),
                     Signs=_f64(sign), Tags=_f64(tags))


class _Lib:
    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)


class Port(_Lib):
    """The C restatement (oracle/port)."""

    def __init__(self, path: str = PORT_SO):
        super().__init__(path)
        L = self.lib
        L.oracle_generate_edges.restype = C.c_int64
        L.oracle_sparse_csr.restype = C.c_int64
        L.oracle_sparse_vec.restype = C.c_int
        L.oracle_pchip.restype = C.c_int

    def generate_edges(self, T0: np.ndarray):
        """Mesh.generateEdges on a 0-based (Ne,4) int array -> 0-based edges, t2e, sign."""
        T1 = np.ascontiguousarray(T0, dtype=np.int32) + 1
        ne = T1.shape[0]
        cap = 6 * ne
        edges = np.zeros((cap, 2), dtype=np.int32)
        t2e = np.zeros((ne, 6), dtype=np.int32)
        sign = np.zeros((ne, 6), dtype=np.int8)
        E = self.lib.oracle_generate_edges(T1.ctypes.data_as(_i32p), C.c_int64(ne),
                                           edges.ctypes.data_as(_i32p), C.c_int64(cap),
                                           t2e.ctypes.data_as(_i32p), sign.ctypes.data_as(_i8p))
        return edges[:E] - 1, t2e - 1, sign

    def jacobian(self, m: MexInputs, sol, qw, curl, packed, calc_j=True):
        ne = m.ne
        nK = 36 * ne if calc_j else 0
        I, J, V = (np.zeros(max(nK, 1)) for _ in range(3))
        Ri, Rv = np.zeros(6 * ne), np.zeros(6 * ne)
        pk = [_f64(a) for a in packed.as_tuple()]
        sol, qw, curl = _f64(sol), _f64(qw), _f64(curl)
        self.lib.oracle_jacobian(_d(m.P), _d(m.T), C.c_int64(ne), _d(m.Dofs), _d(m.Signs),
                                 _d(m.Tags), _d(sol), _d(qw), C.c_int(qw.size), _d(curl),
                                 *[_d(a) for a in pk], C.c_int(int(calc_j)), _d(I), _d(J), _d(V),
                                 _d(Ri), _d(Rv))
        return I[:nK], J[:nK], V[:nK], Ri, Rv

    def material_eval(self, bsq, tags, packed):
        """(nu, dnu/d|B|^2) at |B|^2 = bsq for 1-based tags (MexMaterialUtils.hpp:24-87)."""
        bsq, tags = _f64(bsq), _f64(tags)
        pk = [_f64(a) for a in packed.as_tuple()]
        nu, dnu = np.zeros(bsq.size), np.zeros(bsq.size)
        self.lib.oracle_material_eval(_d(bsq), _d(tags), C.c_int64(bsq.size), *[_d(a) for a in pk], _d(nu),
                                      _d(dnu))
        return nu, dnu

    def curl_curl(self, m: MexInputs, nu, qw, curl):
        ne = m.ne
        I, J, V = (np.zeros(36 * ne) for _ in range(3))
        nu, qw, curl = _f64(nu), _f64(qw), _f64(curl)
        self.lib.oracle_curl_curl(_d(m.P), _d(m.T), C.c_int64(ne), _d(m.Dofs), _d(m.Signs),
                                  _d(nu), _d(qw), C.c_int(qw.size), _d(curl), _d(I), _d(J), _d(V))
        return I, J, V

    def mass(self, m: MexInputs, coeffs, qw, val):
        ne = m.ne
        I, J, V = (np.zeros(36 * ne) for _ in range(3))
        qw, val = _f64(qw), _f64(val)
        cf = None if coeffs is None else _f64(coeffs)
        ncf = 0 if cf is None else cf.size
        self.lib.oracle_mass(_d(m.P), _d(m.T), C.c_int64(ne), _d(m.Dofs), _d(m.Signs), _d(cf),
                             C.c_int64(ncf), _d(qw), C.c_int(qw.size), _d(val), _d(I), _d(J), _d(V))
        return I, J, V

    def source(self, m: MexInputs, js, qw, val):
        ne = m.ne
        I, V = np.zeros(6 * ne), np.zeros(6 * ne)
        js, qw, val = _f64(js), _f64(qw), _f64(val)
        self.lib.oracle_source(_d(m.P), _d(m.T), C.c_int64(ne), _d(m.Dofs), _d(m.Signs), _d(js),
                               _d(qw), C.c_int(qw.size), _d(val), _d(I), _d(V))
        return I, V

    def winding(self, m: MexInputs, coil_id, dir_field, uni_dir, scale, qw, val):
        """assemble_winding_kernel_mex.cpp:13-127; dir_field [Ne x 3] or None (uniform direction)."""
        ne = m.ne
        I, V = np.zeros(6 * ne), np.zeros(6 * ne)
        qw, val, ud = _f64(qw), _f64(val), _f64(uni_dir)
        df = None if dir_field is None else _f64(dir_field)
        self.lib.oracle_winding(_d(m.P), _d(m.T), C.c_int64(ne), _d(m.Dofs), _d(m.Signs), _d(m.Tags),
                                C.c_double(coil_id), _d(df), _d(ud), C.c_double(scale), _d(qw),
                                C.c_int(qw.size), _d(val), _d(I), _d(V))
        return I, V

    def hbfem(self, m: MexInputs, sol, D, P, qw, curl, packed, calc_j=True, scalings=None):
        """assemble_hbfem_kernel_mex restated with the coefficient offsets passed.

        sol: complex [Ndof, K]; D: complex [N, K]; P: complex [K, N]. Returns
        (I, J, V, R_rows, R_cols, R_re, R_im) in the gateway's layout."""
        ne, (ndof, K), N = m.ne, sol.shape, D.shape[0]
        sr, si = _split(sol)  # column-major [Ndof x K]; a real input has no imaginary part
        dr, di = _split(D)    # [N x K]
        pr, pi = _split(P)    # [K x N]
        sc = _f64(np.ones(K) if scalings is None else scalings)
        pk = [_f64(a) for a in packed.as_tuple()]
        qw, curl = _f64(qw), _f64(curl)
        nK = 36 * K * ne if calc_j else 0
        I, J, V = (np.zeros(max(nK, 1)) for _ in range(3))
        Rr, Rc, Rre, Rim = (np.zeros(6 * K * ne) for _ in range(4))
        self.lib.oracle_hbfem(_d(m.P), _d(m.T), C.c_int64(ne), _d(m.Dofs), _d(m.Signs), _d(m.Tags), _d(sr),
                              _d(si), C.c_int64(ndof), C.c_int(K), _d(dr), _d(di), _d(pr), _d(pi), C.c_int(N),
                              _d(qw), C.c_int(qw.size), _d(curl), *[_d(a) for a in pk], C.c_int(int(calc_j)),
                              _d(sc), _d(I), _d(J), _d(V), _d(Rr), _d(Rc), _d(Rre), _d(Rim))
        return I[:nK], J[:nK], V[:nK], Rr, Rc, Rre, Rim

    def sparse_csr(self, I, J, V, N, drop_zeros=True):
        I, J, V = _f64(I), _f64(J), _f64(V)
        n = I.size
        nnz = self.lib.oracle_sparse_csr(_d(I), _d(J), _d(V), C.c_int64(n), C.c_int64(N),
                                         C.c_int(int(drop_zeros)), None, None, None)
        if nnz < 0:
            raise ValueError("sparse: index out of range")
        rp = np.zeros(N + 1, dtype=np.int64)
        ci = np.zeros(max(nnz, 1), dtype=np.int32)
        vv = np.zeros(max(nnz, 1))
        self.lib.oracle_sparse_csr(_d(I), _d(J), _d(V), C.c_int64(n), C.c_int64(N),
                                   C.c_int(int(drop_zeros)), rp.ctypes.data_as(_i64p),
                                   ci.ctypes.data_as(_i32p), _d(vv))
        return rp, ci[:nnz], vv[:nnz]

    def sparse_vec(self, Ridx, Rval, N):
        Ridx, Rval = _f64(Ridx), _f64(Rval)
        out = np.zeros(N)
        if self.lib.oracle_sparse_vec(_d(Ridx), _d(Rval), C.c_int64(Ridx.size), C.c_int64(N),
                                      _d(out)) != 0:
            raise ValueError("sparse vector: index out of range")
        return out

    def pchip(self, x, y):
        x, y = _f64(x), _f64(y)
        coefs = np.zeros((x.size - 1, 4))
        if self.lib.oracle_pchip(_d(x), _d(y), C.c_int64(x.size), _d(coefs)) != 0:
            raise ValueError("pchip failed")
        return coefs


class RefMex(_Lib):
    """The reference's own MEX kernels, compiled unchanged (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        for f in ("ref_jacobian", "ref_curl_curl", "ref_mass", "ref_source", "ref_hbfem"):
            getattr(L, f).restype = C.c_int
        L.ref_last_error.restype = C.c_char_p
        self.last_seconds = 0.0

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def jacobian(self, m: MexInputs, sol, qw, curl, packed, calc_j=True):
        ne = m.ne
        nK = 36 * ne if calc_j else 0
        I, J, V = (np.empty(max(nK, 1)) for _ in range(3))
        Ri, Rv = np.empty(6 * ne), np.empty(6 * ne)
        pk = [_f64(a) for a in packed.as_tuple()]
        sol, qw, curl = _f64(sol), _f64(qw), _f64(curl)
        secs = C.c_double(0)
        nmat = pk[0].size
        rc = self.lib.ref_jacobian(
            _d(m.P), C.c_size_t(m.nn), _d(m.T), C.c_size_t(ne), _d(m.Dofs), _d(m.Signs),
            _d(m.Tags), _d(sol), C.c_size_t(sol.size), _d(qw), C.c_size_t(qw.size), _d(curl),
            _d(pk[0]), _d(pk[1]), _d(pk[2]), C.c_size_t(nmat), _d(pk[3]), C.c_size_t(pk[3].size),
            _d(pk[4]), C.c_size_t(pk[4].size), _d(pk[5]), _d(pk[6]), _d(pk[7]),
            C.c_int(int(calc_j)), _d(I), _d(J), _d(V), _d(Ri), _d(Rv), C.byref(secs))
        self._check(rc)
        self.last_seconds = secs.value
        return I[:nK], J[:nK], V[:nK], Ri, Rv

    def curl_curl(self, m: MexInputs, nu, qw, curl):
        ne = m.ne
        I, J, V = (np.empty(36 * ne) for _ in range(3))
        nu, qw, curl = _f64(nu), _f64(qw), _f64(curl)
        secs = C.c_double(0)
        rc = self.lib.ref_curl_curl(_d(m.P), C.c_size_t(m.nn), _d(m.T), C.c_size_t(ne), _d(m.Dofs),
                                    _d(m.Signs), _d(nu), _d(qw), C.c_size_t(qw.size), _d(curl),
                                    _d(I), _d(J), _d(V), C.byref(secs))
        self._check(rc)
        self.last_seconds = secs.value
        return I, J, V

    def mass(self, m: MexInputs, coeffs, qw, val):
        ne = m.ne
        I, J, V = (np.empty(36 * ne) for _ in range(3))
        qw, val = _f64(qw), _f64(val)
        cf = None if coeffs is None else _f64(coeffs)
        secs = C.c_double(0)
        rc = self.lib.ref_mass(_d(m.P), C.c_size_t(m.nn), _d(m.T), C.c_size_t(ne), _d(m.Dofs),
                               _d(m.Signs), _d(cf), C.c_size_t(0 if cf is None else cf.size),
                               _d(qw), C.c_size_t(qw.size), _d(val), _d(I), _d(J), _d(V),
                               C.byref(secs))
        self._check(rc)
        self.last_seconds = secs.value
        return I, J, V

    def source(self, m: MexInputs, js, qw, val):
        ne = m.ne
        I, V = np.empty(6 * ne), np.empty(6 * ne)
        js, qw, val = _f64(js), _f64(qw), _f64(val)
        secs = C.c_double(0)
        rc = self.lib.ref_source(_d(m.P), C.c_size_t(m.nn), _d(m.T), C.c_size_t(ne), _d(m.Dofs),
                                 _d(m.Signs), _d(js), _d(qw), C.c_size_t(qw.size), _d(val),
                                 _d(I), _d(V), C.byref(secs))
        self._check(rc)
        self.last_seconds = secs.value
        return I, V

    def winding(self, m: MexInputs, coil_id, dir_field, uni_dir, scale, qw, val):
        ne = m.ne
        I, V = np.empty(6 * ne), np.empty(6 * ne)
        qw, val, ud = _f64(qw), _f64(val), _f64(uni_dir)
        df = None if dir_field is None else _f64(dir_field)
        secs = C.c_double(0)
        rc = self.lib.ref_winding(_d(m.P), C.c_size_t(m.nn), _d(m.T), C.c_size_t(ne), _d(m.Dofs), _d(m.Signs),
                                  _d(m.Tags), C.c_double(coil_id), _d(df), _d(ud), C.c_double(scale), _d(qw),
                                  C.c_size_t(qw.size), _d(val), _d(I), _d(V), C.byref(secs))
        self._check(rc)
        self.last_seconds = secs.value
        return I, V


    def hbfem(self, m: MexInputs, sol, D, P, qw, curl, packed, calc_j=True, scalings=None):
        """The reference gateway (22 inputs). It leaves the spline coefficient offsets unset,
        so only linear materials are defined; the caller must not pass nonlinear ones."""
        ne, (ndof, K), N = m.ne, sol.shape, D.shape[0]
        if np.any(np.asarray(packed.is_non) != 0):
            raise ValueError("the reference HBFEM gateway is undefined for nonlinear materials")
        sr, si = _split(sol)
        dr, di = _split(D)
        pr, pi = _split(P)
        sc = _f64(np.ones(K) if scalings is None else scalings)
        pk = [_f64(a) for a in packed.as_tuple()]
        qw, curl = _f64(qw), _f64(curl)
        nK = 36 * K * ne if calc_j else 0
        I, J, V = (np.zeros(max(nK, 1)) for _ in range(3))
        Rr, Rc, Rre, Rim = (np.zeros(6 * K * ne) for _ in range(4))
        secs = C.c_double(0)
        nmat = pk[0].size
        z = C.c_size_t
        rc = self.lib.ref_hbfem(
            _d(m.P), z(m.nn), _d(m.T), z(ne), _d(m.Dofs), _d(m.Signs), _d(m.Tags), _d(sr), _d(si), z(ndof), z(K),
            _d(dr), _d(di), _d(pr), _d(pi), z(N), _d(qw), z(qw.size), _d(curl), _d(pk[0]), _d(pk[1]), _d(pk[2]),
            z(nmat), _d(pk[3]), z(pk[3].size), _d(pk[4]), z(pk[4].size), _d(pk[5]), _d(pk[6]),
            C.c_int(int(calc_j)), _d(sc), _d(I), _d(J), _d(V), _d(Rr), _d(Rc), _d(Rre), _d(Rim), C.byref(secs))
        self._check(rc)
        self.last_seconds = secs.value
        return I[:nK], J[:nK], V[:nK], Rr, Rc, Rre, Rim


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def element_b(P, T0, dofs0, sign, sol):
    """PostProcessor.computeElementB (src/post/PostProcessor.m:64-126), restated in numpy.

    Per element: J = [x2-x1, x3-x1, x4-x1] and detJ by first-row cofactors
    (src/utils/compute_jacobian_tet.m:14-28); reference curls C_ref(e,:) =
    2 * cross(grad L_i, grad L_j) for the local edges (1,2),(1,3),(1,4),(2,3),(2,4),(3,4)
    (src/shape_functions/nedelec_tet_p1.m:28-51); C_phy = (C_ref * J') / detJ;
    B = C_phy' * (A(dofs) .* signs). MATLAB evaluates the two products with BLAS, whose
    summation order is unspecified, so this restatement pins B to rounding level, not to
    the bit. P (Nn,3), T0 (Ne,4) and dofs0 (Ne,6) 0-based, sign (Ne,6) +-1, sol [Ndof].
    Returns B (Ne,3) and, per element, the bound sum_e |C_phy(e,:)| |a_e| that scales its
    rounding error.
    """
    P = np.asarray(P, dtype=np.float64)
    T0 = np.asarray(T0, dtype=np.int64)
    G = np.array([[-1.0, -1.0, -1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    pairs = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))
    C_ref = np.array([2.0 * np.cross(G[i], G[j]) for i, j in pairs])  # (6, 3)
    x1, x2, x3, x4 = (P[T0[:, k]] for k in range(4))
    d1, d2, d3 = x2 - x1, x3 - x1, x4 - x1
    J = np.stack([d1, d2, d3], axis=2)  # J[:, r, c] = d_c[r]
    det = (d1[:, 0] * (d2[:, 1] * d3[:, 2] - d2[:, 2] * d3[:, 1])
           - d1[:, 1] * (d2[:, 0] * d3[:, 2] - d2[:, 2] * d3[:, 0])
           + d1[:, 2] * (d2[:, 0] * d3[:, 1] - d2[:, 1] * d3[:, 0]))
    C_phy = np.einsum("ec,nrc->ner", C_ref, J) * (1.0 / det)[:, None, None]  # (Ne, 6, 3)
    dofs0 = np.asarray(dofs0, dtype=np.int64)
    a = np.where(dofs0 >= 0, np.asarray(sol, dtype=np.float64)[np.maximum(dofs0, 0)], 0.0) * sign
    B = np.einsum("ner,ne->nr", C_phy, a)
    scale = np.einsum("ner,ne->nr", np.abs(C_phy), np.abs(a))
    return B, scale
