"""The oracle pinned against the reference: golden vectors and the compiled MEX.

CPU only. The C restatement in oracle/port must reproduce, bit for bit, the
outputs that the reference's own MEX kernels produced for the committed
fixtures (tests/golden/*.npz), and, when oracle/_ref is built, the live
reference kernels on fresh seeded inputs.
"""
import numpy as np
import pytest
from conftest import bits_equal, load_golden, packed_from_golden

from magpackage_b200 import material, quadrature, synth
from oracle.oracle import mex_inputs


@pytest.mark.parametrize("name", ["one_hex", "cube3"])
def test_port_matches_golden(oracle_port, name):
    d = load_golden(name)
    e, t2e, sign = oracle_port.generate_edges(d["T0"])
    assert np.array_equal(e, d["edges"]) and np.array_equal(t2e, d["t2e"]) and np.array_equal(sign, d["sign"])
    m = mex_inputs(d["P"], d["T0"], t2e, sign, d["tags"])
    pk = packed_from_golden(d)
    I, J, V, Ri, Rv = oracle_port.jacobian(m, d["sol"], d["qw"], d["curl"], pk, True)
    assert bits_equal(I, d["jac_I"]) and bits_equal(J, d["jac_J"])
    assert bits_equal(V, d["jac_V"]) and bits_equal(Ri, d["jac_Ridx"]) and bits_equal(Rv, d["jac_Rval"])
    _, _, _, Ri0, Rv0 = oracle_port.jacobian(m, d["sol"], d["qw"], d["curl"], pk, False)
    assert bits_equal(Rv0, d["res_only_Rval"]) and bits_equal(Ri0, d["res_only_Ridx"])
    _, _, Vk = oracle_port.curl_curl(m, d["cc_nu"], d["qw"], d["curl"])
    assert bits_equal(Vk, d["cc_V"])
    _, _, Vm = oracle_port.mass(m, d["mass_sigma"], d["qw"], d["val"])
    assert bits_equal(Vm, d["mass_V"])
    _, _, Vm1 = oracle_port.mass(m, None, d["qw"], d["val"])
    assert bits_equal(Vm1, d["mass1_V"])
    Is, Vs = oracle_port.source(m, d["src_js"], d["qw"], d["val"])
    assert bits_equal(Is, d["src_I"]) and bits_equal(Vs, d["src_V"])
    for field, key in ((None, "u"), (d["win_field"], "f")):
        Iw, Vw = oracle_port.winding(m, float(d["win_coil"]), field, d["win_dir"], float(d["win_scale"]), d["qw"],
                                     d["val"])
        assert bits_equal(Iw, d[f"win_{key}_I"]) and bits_equal(Vw, d[f"win_{key}_V"])


def test_unit_tet_known_answer(oracle_port):
    """tests/test_mex_assembly.m:32-73: the unit tetrahedron, Nu = 500."""
    d = load_golden("unit_tet")
    m = mex_inputs(d["P"], np.array([[0, 1, 2, 3]]), np.arange(6)[None, :],
                   np.array([[1, -1, 1, -1, 1, -1]]), np.array([1]))
    I, J, V = oracle_port.curl_curl(m, np.array([500.0]), d["qw"], d["curl"])
    assert bits_equal(V, d["V"]) and bits_equal(I, d["I"]) and bits_equal(J, d["J"])
    # the reference's MATLAB-vs-MEX bound
    K = np.zeros((6, 6))
    np.add.at(K, (I.astype(int) - 1, J.astype(int) - 1), V)
    assert np.allclose(K, K.T, rtol=0, atol=1e-13)


def test_quadrature_tables_match_reference_inputs():
    d = load_golden("cube3")
    qw, val, curl = quadrature.reference_data(2)
    assert bits_equal(qw, d["qw"]) and bits_equal(val, d["val"]) and bits_equal(curl, d["curl"])
    q1, w1 = quadrature.get_quadrature_data("tet", 1)
    assert w1[0] == 1.0 / 6.0 and q1.shape == (3, 1)


@pytest.mark.parametrize("n", [1, 2, 5])
def test_edges_counts_and_order(oracle_port, n):
    mesh = synth.kuhn_box(n, seed=n)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    assert edges.shape[0] == 7 * n ** 3 + 9 * n ** 2 + 3 * n
    key = edges[:, 0].astype(np.int64) * mesh.num_nodes + edges[:, 1]
    assert np.all(np.diff(key) > 0) and np.all(edges[:, 0] < edges[:, 1])
    a = mesh.T[:, [0, 0, 0, 1, 1, 2]]
    b = mesh.T[:, [1, 2, 3, 2, 3, 3]]
    assert np.array_equal(sign, np.where(a < b, 1, -1))
    assert np.array_equal(edges[t2e, 0], np.minimum(a, b)) and np.array_equal(edges[t2e, 1], np.maximum(a, b))


def test_sparse_semantics(oracle_port):
    import scipy.sparse as sp

    rng = np.random.default_rng(0)
    n = 50
    I = rng.integers(0, n + 1, 2000).astype(float)  # includes invalid 0 indices
    J = rng.integers(0, n + 1, 2000).astype(float)
    V = rng.normal(size=2000)
    V[::7] = 0.0
    rp, ci, vv = oracle_port.sparse_csr(I, J, V, n, drop_zeros=True)
    ok = (I > 0) & (J > 0)
    S = sp.coo_matrix((V[ok], (I[ok] - 1, J[ok] - 1)), shape=(n, n)).tocsr()
    S.sum_duplicates()
    S.eliminate_zeros()
    assert np.array_equal(rp, S.indptr) and np.array_equal(ci, S.indices)
    assert np.allclose(vv, S.data, rtol=1e-15, atol=0)
    # duplicates summing to exactly zero disappear; kept only without dropping
    I2, J2, V2 = np.array([1.0, 1, 2, 0]), np.array([1.0, 1, 2, 2]), np.array([1.5, -1.5, 2.0, 9.0])
    rp, ci, vv = oracle_port.sparse_csr(I2, J2, V2, 2, drop_zeros=True)
    assert rp.tolist() == [0, 0, 1] and ci.tolist() == [1] and vv.tolist() == [2.0]
    rp, ci, vv = oracle_port.sparse_csr(I2, J2, V2, 2, drop_zeros=False)
    assert rp.tolist() == [0, 1, 2] and vv.tolist() == [0.0, 2.0]


def test_pchip_restatements_agree(oracle_port):
    from scipy.interpolate import PchipInterpolator

    b, h = material.froehlich_bh()
    mat = material.create_nonlinear(b, h)
    x = mat.breaks
    y = np.r_[mat.coefs[:, 3], np.polyval(mat.coefs[-1], x[-1] - x[-2])]
    c_port = oracle_port.pchip(x, y)
    assert bits_equal(c_port, material.pchip(x, y))
    # interpolant values against scipy (MATLAB's own bits are not available here)
    S = PchipInterpolator(x, y)
    xs = np.concatenate([np.linspace(x[k], x[k + 1], 7) for k in range(x.size - 1)])
    k = np.clip(np.searchsorted(x, xs, side="right") - 1, 0, x.size - 2)
    t = xs - x[k]
    c = mat.coefs[k]
    mine = ((c[:, 0] * t + c[:, 1]) * t + c[:, 2]) * t + c[:, 3]
    assert np.allclose(mine, S(xs), rtol=1e-12, atol=0)
    assert mat.breaks.size == 201 and mat.max_bsq == x[-1]


def test_create_nonlinear_vacuum_point():
    b, h = material.froehlich_bh()
    mat = material.create_nonlinear(b, h)
    nu = mat.coefs[:, 3]
    assert nu[0] == nu[1]  # MaterialLib.m:87
    bu = mat.extra["B_data"]
    nu_end = mat.extra["H_data"][-1] / bu[-1]
    expect = min(nu_end + (material.NU0 - nu_end) / (2 * bu[-1] ** 2) * 0.1, material.NU0)
    last = np.polyval(mat.coefs[-1], mat.breaks[-1] - mat.breaks[-2])
    assert abs(last - expect) <= 1e-9 * expect
    assert mat.breaks[-1] == bu[-1] ** 2 + 0.1


def test_port_matches_live_reference(oracle_port, oracle_ref):
    mesh = synth.kuhn_box(5, 4, 3, seed=9)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    m = mex_inputs(mesh.P, mesh.T, t2e, sign, tags)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    sol = np.random.default_rng(3).normal(0, 0.05, edges.shape[0])
    for cj in (True, False):
        r = oracle_ref.jacobian(m, sol, qw, curl, pk, cj)
        p = oracle_port.jacobian(m, sol, qw, curl, pk, cj)
        assert all(bits_equal(x, y) for x, y in zip(r, p))
    nu = np.random.default_rng(4).uniform(100, 1e6, mesh.num_elements)
    assert bits_equal(oracle_ref.curl_curl(m, nu, qw, curl)[2], oracle_port.curl_curl(m, nu, qw, curl)[2])
    sig = np.where(tags == synth.ALUMINIUM, synth.SIGMA_AL, 0.0)
    assert bits_equal(oracle_ref.mass(m, sig, qw, val)[2], oracle_port.mass(m, sig, qw, val)[2])
    js = np.random.default_rng(5).normal(size=(mesh.num_elements, 3))
    assert bits_equal(oracle_ref.source(m, js, qw, val)[1], oracle_port.source(m, js, qw, val)[1])
    # winding: coil region present or absent, uniform or per-element direction, missing dofs
    m.Dofs[::7, 2] = 0.0
    field = np.random.default_rng(6).normal(size=(mesh.num_elements, 3))
    for coil in (float(synth.ALUMINIUM), float(synth.IRON), 99.0):
        for f in (None, field):
            r = oracle_ref.winding(m, coil, f, (0.0, 0.6, -0.8), 4.0e5, qw, val)
            p = oracle_port.winding(m, coil, f, (0.0, 0.6, -0.8), 4.0e5, qw, val)
            assert bits_equal(r[0], p[0]) and bits_equal(r[1], p[1])


def _hbfem_case(oracle_port, iron_nonlinear, n=(4, 3, 3), seed=11, harmonics=(0, 1, 3), imag=True):
    from magpackage_b200.hbfem import AFT

    mesh = synth.kuhn_box(*n, seed=seed)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    m = mex_inputs(mesh.P, mesh.T, t2e, sign, tags)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials(iron_nonlinear))
    aft = AFT(harmonics)
    rng = np.random.default_rng(seed)
    E, K = edges.shape[0], len(harmonics)
    sol = rng.normal(0, 0.05, (E, K)) + (1j * rng.normal(0, 0.05, (E, K)) if imag else 0.0)
    return mesh, m, qw, curl, pk, aft, sol


@pytest.mark.parametrize("imag", [True, False])
def test_hbfem_port_matches_reference_on_linear_materials(oracle_port, oracle_ref, imag):
    """assemble_hbfem_kernel_mex compiled unchanged (defined for linear materials only:
    it leaves the spline coefficient offsets unset) against the restatement, bit for bit."""
    mesh, m, qw, curl, pk, aft, sol = _hbfem_case(oracle_port, False, imag=imag)
    D = aft.D if imag else np.real(aft.D)
    P = aft.P if imag else np.real(aft.P)
    sc = np.array([1.0, 2.5, -0.75])
    for cj in (True, False):
        r = oracle_ref.hbfem(m, sol, D, P, qw, curl, pk, cj, sc)
        p = oracle_port.hbfem(m, sol, D, P, qw, curl, pk, cj, sc)
        assert all(bits_equal(x, y) for x, y in zip(r, p))
        assert np.abs(p[5]).max() > 0


def test_hbfem_single_dc_harmonic_is_the_static_residual(oracle_port):
    """With the harmonic set {0} and one time sample (D = P = 1) the harmonic-balance
    residual is the static Newton residual of the Jacobian kernel on nonlinear iron (the
    two kernels order the same products differently, so they agree to rounding)."""
    from magpackage_b200.hbfem import AFT

    mesh, m, qw, curl, pk, _, sol = _hbfem_case(oracle_port, True, harmonics=(0,), imag=False)
    aft = AFT([0], n_time_steps=1)
    assert aft.D.shape == (1, 1) and aft.P[0, 0] == 1.0
    E = sol.shape[0]
    x = np.real(sol[:, 0]) * 40.0  # drive the iron through the spline's interior and knee
    _, _, _, Rr, Rc, Rre, Rim = oracle_port.hbfem(m, x[:, None], aft.D, aft.P, qw, curl, pk, False)
    hb = oracle_port.sparse_vec(Rr, Rre, E)
    _, _, _, Ri, Rv = oracle_port.jacobian(m, x, qw, curl, pk, False)
    st = oracle_port.sparse_vec(Ri, Rv, E)
    assert np.abs(hb - st).max() <= 1e-13 * np.abs(st).max()
    assert np.all(Rim == 0.0)


def uniform_field_edges(P, edges, B0):
    """Edge dofs of A = B0 x x / 2 (curl A = B0): the line integral along each global edge,
    oriented from its first to its second node, exact for a linear field."""
    p, q = P[edges[:, 0]], P[edges[:, 1]]
    return 0.5 * np.einsum("ij,ij->i", np.cross(B0, 0.5 * (p + q)), q - p)


def test_element_b_restatement_patch_test(oracle_port):
    """PostProcessor.computeElementB restated: a uniform field is reproduced in every
    element (Nedelec elements contain the constant curls exactly)."""
    from oracle.oracle import element_b

    mesh = synth.kuhn_box(5, 4, 3, seed=7)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    B0 = np.array([0.3, -1.2, 0.7])
    sol = uniform_field_edges(mesh.P, edges, B0)
    B, scale = element_b(mesh.P, mesh.T, t2e, sign, sol)
    assert np.all(np.abs(B - B0) <= 1e-12 * scale)
    # a gradient field (edge differences of a nodal potential) has zero curl
    phi = np.random.default_rng(3).normal(size=mesh.num_nodes)
    B, scale = element_b(mesh.P, mesh.T, t2e, sign, phi[edges[:, 1]] - phi[edges[:, 0]])
    assert np.all(np.abs(B) <= 1e-12 * scale)


def test_mlp_oracle_gradient_matches_finite_differences(monkeypatch):
    """The MLP oracle's backward pass (oracle/mlp_ref.py), which the GPU gradient kernels
    are checked against, pinned by central differences of its own loss
    L = sum_i s/2 (y_i - t_i)^2 with the BF16 rounding switched off (the backward pass
    treats each rounding as the identity, so without it the two must agree to
    finite-difference accuracy)."""
    from magpackage_b200.mlp import init_params
    from oracle import mlp_ref

    monkeypatch.setattr(mlp_ref, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(8)
    p = init_params(2).astype(np.float64)
    p[256:320] = rng.normal(0, 0.1, 64)
    x = rng.normal(0, 1, (37, 4))
    t = rng.normal(0, 1, 37)
    s = 0.5

    def loss(q):
        y, _ = mlp_ref.forward(q, x)
        return float(np.sum(0.5 * s * (y - t) ** 2))

    _, g = mlp_ref.gradient(p, x, t, s)
    assert g.shape == (mlp_ref.NPARAMS,)
    # a few parameters of every block: W1, b1, W2, b2, W3, b3, w4, b4
    starts = [0, 256, 320, 4416, 4480, 8576, 8640, 8704]
    idx = sorted({int(i) for st, en in zip(starts, starts[1:] + [mlp_ref.NPARAMS])
                  for i in rng.integers(st, en, size=6)})
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        fd = (loss(q1) - loss(q2)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * (1.0 + abs(fd)), (i, fd, g[i])
