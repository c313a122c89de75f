"""GPU parity: the sm_100a path against the oracle, bit for bit.

Every CSR produced on the GPU is compared with the oracle's restatement of
MATLAB's sparse() applied to the reference MEX triplets (the compiled
reference when oracle/_ref is present, its pinned C restatement otherwise):
row_ptr/col_idx must be identical and every value identical bit for bit
(tolerance 0; the required bound is 1e-12 relative per nonzero).
"""
import ctypes as C

import numpy as np
import pytest
import torch
from conftest import bits_equal, load_golden, packed_from_golden

from magpackage_b200 import _lib, material, quadrature, synth
from magpackage_b200.assembler import Assembler, DofHandler, Mesh
from magpackage_b200.plan import AssemblyPlan, generate_edges
from oracle.oracle import mex_inputs

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # required bound per nonzero; the tests below demand exact equality


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().cpu().numpy()


def make_case(port, P, T, tags):
    edges, t2e, sign = port.generate_edges(T)
    return edges, t2e, sign, mex_inputs(P, T, t2e, sign, tags)


def oracle_matrix(port, I, J, V, n, drop):
    return port.sparse_csr(I, J, V, n, drop_zeros=drop)


def assert_csr_equal(rp, ci, vals, ref):
    rrp, rci, rv = ref
    assert np.array_equal(host(rp), rrp), "row_ptr differs"
    assert np.array_equal(host(ci), rci), "col_idx differs"
    v = host(vals)
    assert bits_equal(v, rv), f"values differ: max rel {np.max(np.abs(v - rv) / np.maximum(np.abs(rv), 1e-300))}"


# ---- topology ----------------------------------------------------------------------

@pytest.mark.parametrize("n", [1, 3, 8])
def test_generate_edges_matches_oracle(oracle_port, n):
    mesh = synth.kuhn_box(n, n + 1, max(n - 1, 1), seed=n)
    edges, t2e, sign = generate_edges(mesh.T)
    e0, t0, s0 = oracle_port.generate_edges(mesh.T)
    assert np.array_equal(host(edges), e0) and np.array_equal(host(t2e), t0) and np.array_equal(host(sign), s0)


def test_generate_edges_rejects_bad_nodes():
    T = np.array([[0, 1, 2, 2]], dtype=np.int32)  # repeated node
    with pytest.raises(_lib.MagError):
        generate_edges(T)


# ---- golden fixtures through the handle path ------------------------------------------

@pytest.mark.parametrize("name", ["one_hex", "cube3"])
def test_jacobian_matches_golden(oracle_port, name):
    d = load_golden(name)
    E = d["edges"].shape[0]
    plan = AssemblyPlan(d["P"], d["T0"], d["t2e"], E, d["tags"], d["sign"])
    assert plan.info.signs_derived == 1
    plan.set_materials(packed_from_golden(d))
    vals, res = plan.jacobian(dev(d["sol"]))
    ref = oracle_matrix(oracle_port, d["jac_I"], d["jac_J"], d["jac_V"], E, drop=False)
    assert_csr_equal(plan.row_ptr, plan.col_idx, vals, ref)
    assert bits_equal(host(res), oracle_port.sparse_vec(d["jac_Ridx"], d["jac_Rval"], E))
    # residual-only pass (CalcJ = false)
    _, res0 = plan.jacobian(dev(d["sol"]), calc_j=False)
    assert bits_equal(host(res0), oracle_port.sparse_vec(d["res_only_Ridx"], d["res_only_Rval"], E))
    # MATLAB storage: exact zeros dropped
    rp2, ci2, v2 = plan.drop_zeros(vals)
    assert_csr_equal(rp2, ci2, v2, oracle_matrix(oracle_port, d["jac_I"], d["jac_J"], d["jac_V"], E, True))


@pytest.mark.parametrize("name", ["one_hex", "cube3"])
def test_stiffness_mass_source_match_golden(oracle_port, name):
    d = load_golden(name)
    E = d["edges"].shape[0]
    plan = AssemblyPlan(d["P"], d["T0"], d["t2e"], E, d["tags"], d["sign"])
    I, J = d["jac_I"], d["jac_J"]
    k = plan.stiffness(dev(d["cc_nu"]))
    assert_csr_equal(plan.row_ptr, plan.col_idx, k, oracle_matrix(oracle_port, I, J, d["cc_V"], E, False))
    m = plan.mass(dev(d["mass_sigma"]))
    assert_csr_equal(plan.row_ptr, plan.col_idx, m, oracle_matrix(oracle_port, I, J, d["mass_V"], E, False))
    rp2, ci2, v2 = plan.drop_zeros(m)
    assert_csr_equal(rp2, ci2, v2, oracle_matrix(oracle_port, I, J, d["mass_V"], E, True))
    m1 = plan.mass(None)
    assert_csr_equal(plan.row_ptr, plan.col_idx, m1, oracle_matrix(oracle_port, I, J, d["mass1_V"], E, False))
    f = plan.source(dev(d["src_js"]))
    assert bits_equal(host(f), oracle_port.sparse_vec(d["src_I"], d["src_V"], E))


def test_unit_tet_known_answer_on_gpu():
    """tests/test_mex_assembly.m:32-73 through the MEX-compatible entry point."""
    d = load_golden("unit_tet")
    L = _lib.lib()
    P = np.ascontiguousarray(d["P"])
    T = np.array([1.0, 2, 3, 4])
    dofs = np.arange(1.0, 7.0)
    signs = np.array([1.0, -1, 1, -1, 1, -1])
    nu = np.array([500.0])
    I, J, V = np.zeros(36), np.zeros(36), np.zeros(36)
    qw, curl = np.ascontiguousarray(d["qw"]), np.ascontiguousarray(d["curl"])
    _lib.check(L.mag_mex_curl_curl(_lib.dptr(P), 4, _lib.dptr(T), 1, _lib.dptr(dofs), _lib.dptr(signs),
                                   _lib.dptr(nu), _lib.dptr(qw), qw.size, _lib.dptr(curl), _lib.dptr(I),
                                   _lib.dptr(J), _lib.dptr(V)))
    assert bits_equal(V, d["V"]) and bits_equal(I, d["I"]) and bits_equal(J, d["J"])


@pytest.mark.parametrize("name", ["one_hex", "cube3"])
def test_mex_entry_points_match_golden(name):
    d = load_golden(name)
    L = _lib.lib()
    m = mex_inputs(d["P"], d["T0"], d["t2e"], d["sign"], d["tags"])
    ne, nn, E = m.ne, m.nn, d["edges"].shape[0]
    pk = [np.ascontiguousarray(a, dtype=np.float64) for a in packed_from_golden(d).as_tuple()]
    qw, curl, val = (np.ascontiguousarray(d[k]) for k in ("qw", "curl", "val"))
    sol = np.ascontiguousarray(d["sol"])
    for cj in (1, 0):
        I, J, V = (np.zeros(36 * ne) for _ in range(3))
        Ri, Rv = np.zeros(6 * ne), np.zeros(6 * ne)
        p = _lib.dptr
        _lib.check(L.mag_mex_jacobian(p(m.P), nn, p(m.T), ne, p(m.Dofs), p(m.Signs), p(m.Tags), p(sol), E,
                                      p(qw), qw.size, p(curl), p(pk[0]), p(pk[1]), p(pk[2]), pk[0].size,
                                      p(pk[3]), pk[3].size, p(pk[4]), pk[4].size, p(pk[5]), p(pk[6]),
                                      p(pk[7]), cj, p(I), p(J), p(V), p(Ri), p(Rv)))
        if cj:
            assert bits_equal(I, d["jac_I"]) and bits_equal(J, d["jac_J"]) and bits_equal(V, d["jac_V"])
            assert bits_equal(Ri, d["jac_Ridx"]) and bits_equal(Rv, d["jac_Rval"])
        else:
            assert bits_equal(Rv, d["res_only_Rval"])
    I, J, V = (np.zeros(36 * ne) for _ in range(3))
    nu = np.ascontiguousarray(d["cc_nu"])
    _lib.check(L.mag_mex_curl_curl(p(m.P), nn, p(m.T), ne, p(m.Dofs), p(m.Signs), p(nu), p(qw), qw.size,
                                   p(curl), p(I), p(J), p(V)))
    assert bits_equal(V, d["cc_V"])
    sig = np.ascontiguousarray(d["mass_sigma"])
    _lib.check(L.mag_mex_mass(p(m.P), nn, p(m.T), ne, p(m.Dofs), p(m.Signs), p(sig), ne, p(qw), qw.size,
                              p(val), p(I), p(J), p(V)))
    assert bits_equal(V, d["mass_V"])
    _lib.check(L.mag_mex_mass(p(m.P), nn, p(m.T), ne, p(m.Dofs), p(m.Signs), None, 0, p(qw), qw.size,
                              p(val), p(I), p(J), p(V)))
    assert bits_equal(V, d["mass1_V"])


# ---- fresh seeded meshes against the live oracle ------------------------------------------

def _nonlinear_case(oracle_port, n, seed, scale=0.02):
    mesh = synth.kuhn_box(n, seed=seed)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign, m = make_case(oracle_port, mesh.P, mesh.T, tags)
    E = edges.shape[0]
    rng = np.random.default_rng(seed)
    sol = rng.normal(0, scale, E) * 10.0 ** rng.uniform(-1.5, 0.5, E)
    return mesh, tags, edges, t2e, sign, m, E, sol


@pytest.mark.parametrize("n,seed", [(6, 1), (13, 2)])
def test_jacobian_random_meshes(oracle_port, n, seed):
    mesh, tags, edges, t2e, sign, m, E, sol = _nonlinear_case(oracle_port, n, seed)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    plan.set_materials(pk)
    vals, res = plan.jacobian(dev(sol))
    assert_csr_equal(plan.row_ptr, plan.col_idx, vals, oracle_matrix(oracle_port, I, J, V, E, False))
    assert bits_equal(host(res), oracle_port.sparse_vec(Ri, Rv, E))
    assert plan.nnz == 115 * n ** 3 + 45 * n ** 2 + 3 * n


def test_config1_assembler_surface(oracle_port):
    """Config 1 (20^3 cube): K(nu) and M(sigma) through the Assembler mirror, MATLAB storage."""
    mesh_s = synth.kuhn_box(20, seed=0)
    tags = synth.cube_layout(mesh_s)
    mesh = Mesh(mesh_s.P, mesh_s.T, tags)
    dh = DofHandler(mesh)
    dh.distribute_dofs()
    asm = Assembler(mesh, dh)
    nu_map = {synth.AIR: material.NU0, synth.IRON: material.NU0 / 1000.0, synth.ALUMINIUM: material.NU0}
    sig_map = {synth.ALUMINIUM: synth.SIGMA_AL}
    K = asm.assemble_stiffness(nu_map)
    M = asm.assemble_mass_weighted(sig_map)
    e0, t0, s0 = oracle_port.generate_edges(mesh_s.T)
    m = mex_inputs(mesh_s.P, mesh_s.T, t0, s0, tags)
    qw, val, curl = quadrature.reference_data(2)
    E = e0.shape[0]
    assert E == 59660 and dh.NumGlobalDofs == E
    Ik, Jk, Vk = oracle_port.curl_curl(m, asm.expand_material_map(nu_map), qw, curl)
    assert_csr_equal(K.row_ptr, K.col_idx, K.values, oracle_matrix(oracle_port, Ik, Jk, Vk, E, True))
    Im, Jm, Vm = oracle_port.mass(m, asm.expand_material_map(sig_map), qw, val)
    assert_csr_equal(M.row_ptr, M.col_idx, M.values, oracle_matrix(oracle_port, Im, Jm, Vm, E, True))
    assert M.nnz < K.nnz  # only rows touching aluminium survive zero dropping


def test_reduced_domain_dofs(oracle_port):
    """DofHandler.distributeDofs with target regions: dofs only on active edges (DofHandler.m:72-105)."""
    mesh_s = synth.kuhn_box(7, seed=3)
    tags = synth.cube_layout(mesh_s)
    mesh = Mesh(mesh_s.P, mesh_s.T, tags)
    dh = DofHandler(mesh)
    dofs = host(dh.distribute_dofs(target_region_tags=[synth.IRON, synth.ALUMINIUM]))
    assert (dofs < 0).any() and dh.NumGlobalDofs < mesh.Edges.shape[0]
    sign = host(mesh.T2E_Sign)
    m = mex_inputs(mesh_s.P, mesh_s.T, dofs, sign, tags)
    sol = np.random.default_rng(0).normal(0, 0.02, dh.NumGlobalDofs)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    asm = Assembler(mesh, dh, matlab_storage=True)
    Jm, R = asm.assemble_jacobian(sol, synth.standard_materials())
    assert_csr_equal(Jm.row_ptr, Jm.col_idx, Jm.values, oracle_matrix(oracle_port, I, J, V, dh.NumGlobalDofs, True))
    assert bits_equal(host(R), oracle_port.sparse_vec(Ri, Rv, dh.NumGlobalDofs))


def test_generic_quadrature_path(oracle_port):
    """Non-standard curl table and non-uniform weights take the general per-point loop."""
    mesh, tags, edges, t2e, sign, m, E, sol = _nonlinear_case(oracle_port, 4, 5)
    qw = np.array([0.05, 0.04, 0.045, 0.0316666])
    _, val, curl = quadrature.reference_data(2)
    curl = curl.copy()
    curl[18 * 2: 18 * 3] *= 0.5  # one point with a scaled curl
    pk = material.pack_material_data(synth.standard_materials())
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    plan.set_quadrature(qw, curl, val)
    plan.set_materials(pk)
    vals, res = plan.jacobian(dev(sol))
    assert_csr_equal(plan.row_ptr, plan.col_idx, vals, oracle_matrix(oracle_port, I, J, V, E, False))
    assert bits_equal(host(res), oracle_port.sparse_vec(Ri, Rv, E))
    nu = np.random.default_rng(1).uniform(1e2, 1e6, mesh.num_elements)
    _, _, Vk = oracle_port.curl_curl(m, nu, qw, curl)
    k = plan.stiffness(dev(nu))
    assert_csr_equal(plan.row_ptr, plan.col_idx, k, oracle_matrix(oracle_port, I, J, Vk, E, False))
    # uniform weights with the standard table take the fast path; same bits as the oracle
    qw2, val2, curl2 = quadrature.reference_data(2)
    plan.set_quadrature(qw2, curl2, val2)
    vals2, _ = plan.jacobian(dev(sol))
    I2, J2, V2, _, _ = oracle_port.jacobian(m, sol, qw2, curl2, pk, True)
    assert_csr_equal(plan.row_ptr, plan.col_idx, vals2, oracle_matrix(oracle_port, I2, J2, V2, E, False))


def test_explicit_signs_are_honoured(oracle_port):
    """Signs that differ from the Mesh.m rule are stored and applied as given."""
    mesh, tags, edges, t2e, sign, m, E, sol = _nonlinear_case(oracle_port, 3, 8)
    flipped = sign.copy()
    flipped[::5] *= -1
    m2 = mex_inputs(mesh.P, mesh.T, t2e, flipped, tags)
    pk = material.pack_material_data(synth.standard_materials())
    qw, val, curl = quadrature.reference_data(2)
    I, J, V, Ri, Rv = oracle_port.jacobian(m2, sol, qw, curl, pk, True)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, flipped)
    assert plan.info.signs_derived == 0
    plan.set_materials(pk)
    vals, res = plan.jacobian(dev(sol))
    assert_csr_equal(plan.row_ptr, plan.col_idx, vals, oracle_matrix(oracle_port, I, J, V, E, False))
    assert bits_equal(host(res), oracle_port.sparse_vec(Ri, Rv, E))


def test_async_calls_on_side_streams_and_mag_sync(oracle_port):
    """The handle API only enqueues: two handles assembling on two streams, each waited for
    with mag_sync, give the same bits as a call on the current stream."""
    mesh = synth.kuhn_box(5, seed=4)
    tags = synth.cube_layout(mesh)
    packed = material.pack_material_data(synth.standard_materials())
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    E = edges.shape[0]
    sol = torch.as_tensor(np.random.default_rng(9).normal(0, 0.05, E), device="cuda")
    plans = [AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign) for _ in range(2)]
    for p in plans:
        p.set_materials(packed)
    v0, r0 = plans[0].jacobian(sol)
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in range(2)]
    out = []
    for p, s in zip(plans, streams):
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            vals, res = p.new_values(), p.new_vector()
        p.jacobian(sol, vals, res, stream=s)
        out.append((vals, res, s))
    for vals, res, s in out:
        _lib.sync(s)
        assert torch.equal(vals, v0) and torch.equal(res, r0)
    for p in plans:
        p.close()


def test_deterministic_repeat(oracle_port):
    mesh, tags, edges, t2e, sign, m, E, sol = _nonlinear_case(oracle_port, 10, 4)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    plan.set_materials(material.pack_material_data(synth.standard_materials()))
    s = dev(sol)
    v1, r1 = plan.jacobian(s)
    v2, r2 = plan.jacobian(s)
    assert torch.equal(v1.view(torch.int64), v2.view(torch.int64))
    assert torch.equal(r1.view(torch.int64), r2.view(torch.int64))


# ---- analytic properties ----------------------------------------------------------------

def test_gradient_null_space_and_symmetry(oracle_port):
    """A = grad(phi) (edge differences of a nodal field) has zero curl: R = 0, K A = 0."""
    mesh, tags, edges, t2e, sign, m, E, _ = _nonlinear_case(oracle_port, 8, 6)
    phi = np.random.default_rng(2).normal(size=mesh.num_nodes)
    a = phi[edges[:, 1]] - phi[edges[:, 0]]
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    nu = np.where(tags == synth.IRON, material.NU0 / 1000, material.NU0)
    k = plan.stiffness(dev(nu))
    A = torch.sparse_csr_tensor(plan.row_ptr, plan.col_idx.long(), k, size=(E, E))
    ka = A @ dev(a)
    scale = torch.sparse_csr_tensor(plan.row_ptr, plan.col_idx.long(), k.abs(), size=(E, E)) @ dev(np.abs(a))
    assert float((ka.abs() / scale.clamp_min(1e-300)).max()) < 1e-9
    plan.set_materials(material.pack_material_data(synth.standard_materials()))
    _, r = plan.jacobian(dev(a), calc_j=False)
    assert float(r.abs().max()) < 1e-9 * float(scale.max())
    # K is symmetric bit for bit for linear materials
    Kd = A.to_dense()
    assert torch.equal(Kd, Kd.T)


def test_jacobian_matches_finite_differences(oracle_port):
    mesh, tags, edges, t2e, sign, m, E, sol = _nonlinear_case(oracle_port, 5, 9, scale=0.05)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    plan.set_materials(material.pack_material_data(synth.standard_materials()))
    x = dev(sol)
    vals, _ = plan.jacobian(x)
    Jm = torch.sparse_csr_tensor(plan.row_ptr, plan.col_idx.long(), vals, size=(E, E))
    d = dev(np.random.default_rng(1).normal(size=E)) * 1e-3 * x.abs().mean()
    eps = 1e-3
    _, rp = plan.jacobian(x + eps * d, calc_j=False)
    _, rm = plan.jacobian(x - eps * d, calc_j=False)
    fd = (rp - rm) / (2 * eps)
    jd = Jm @ d
    assert float((fd - jd).norm() / jd.norm()) < 1e-5


# ---- errors are reported, not dereferenced ------------------------------------------------

def test_errors_are_reported(oracle_port):
    mesh = synth.kuhn_box(2, seed=0)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    E = edges.shape[0]
    bad = tags.copy()
    bad[3] = 0
    with pytest.raises(_lib.MagError) as ei:
        AssemblyPlan(mesh.P, mesh.T, t2e, E, bad, sign)
    assert ei.value.code == -2
    flat = mesh.P.copy()
    flat[mesh.T[0, 3]] = flat[mesh.T[0, 0]]  # collapse an element
    with pytest.raises(_lib.MagError) as ei:
        AssemblyPlan(flat, mesh.T, t2e, E, tags, sign)
    assert ei.value.code in (-3, -2)
    dofs = t2e.copy()
    dofs[0, 0] = E + 5
    with pytest.raises(_lib.MagError):
        AssemblyPlan(mesh.P, mesh.T, dofs, E, tags, sign)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    with pytest.raises(_lib.MagError):  # materials not set
        plan.jacobian(dev(np.zeros(E)))
    plan.set_materials(material.pack_material_data({1: material.create_linear(1.0)}))
    with pytest.raises(_lib.MagError) as ei:  # tags 2, 3 have no entry
        plan.jacobian(dev(np.zeros(E)))
    assert ei.value.code == -2


# ---- the three Jacobian schedules ------------------------------------------------------------

SCHEDULES = (_lib.SCHEDULE_TILE_BLOCKS, _lib.SCHEDULE_SHARED_ROW_BLOCKS, _lib.SCHEDULE_NZ_ROW_BLOCKS,
             _lib.SCHEDULE_ROW_BLOCKS, _lib.SCHEDULE_TWO_PASS)


def available(plan):
    """The schedules this mesh supports (the tile and nonzero-pass ones need rows of at most
    31 entries and off-diagonal entries of at most two contributions)."""
    out = []
    for sch in SCHEDULES:
        if sch == _lib.SCHEDULE_TILE_BLOCKS and plan.info.tile_blocks == 0:
            continue
        if sch == _lib.SCHEDULE_NZ_ROW_BLOCKS and plan.info.nz_pass == 0:
            continue
        out.append(sch)
    return out


@pytest.mark.parametrize("n,seed", [(13, 21), (30, 22)])
def test_schedules_agree_bit_for_bit(oracle_port, n, seed):
    """Tile blocks (default), the row-block variants and the two-pass kernels give the same
    bits as each other and as the oracle, with and without the Jacobian, on the fast and the
    general quadrature path."""
    mesh, tags, edges, t2e, sign, m, E, sol = _nonlinear_case(oracle_port, n, seed)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    assert plan.info.schedule == _lib.SCHEDULE_TILE_BLOCKS
    assert plan.info.nz_pass == 1 and plan.info.tile_colors == 2
    # 4x4x4-node tiles: each element is evaluated about 1.5 times (1 + 2/4 for interior tiles)
    assert 1.0 < plan.info.tile_evals_per_elem < 1.75
    pk = material.pack_material_data(synth.standard_materials())
    plan.set_materials(pk)
    x = dev(sol)
    qw, val, curl = quadrature.reference_data(2)
    qw2 = np.array([0.05, 0.04, 0.045, 0.0316666])
    refs = {}
    for name, w in (("std", qw), ("general", qw2)):
        I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, w, curl, pk, True)
        _, _, _, Ri0, Rv0 = oracle_port.jacobian(m, sol, w, curl, pk, False)
        refs[name] = (oracle_matrix(oracle_port, I, J, V, E, False), oracle_port.sparse_vec(Ri, Rv, E),
                      oracle_port.sparse_vec(Ri0, Rv0, E))
    for name, w in (("std", qw), ("general", qw2)):
        plan.set_quadrature(w, curl, val)
        mat, vec, vec0 = refs[name]
        for sch in available(plan):
            plan.set_schedule(sch)
            v, r = plan.jacobian(x)
            _, r0 = plan.jacobian(x, calc_j=False)
            plan.check()
            assert_csr_equal(plan.row_ptr, plan.col_idx, v, mat)
            assert bits_equal(host(r), vec), (name, sch)
            assert bits_equal(host(r0), vec0), (name, sch)


# ---- batched complex K + j*omega*M ----------------------------------------------------------

def test_batched_complex_matches_oracle(oracle_port):
    """Several uneven meshes in one graph-captured launch: the real part equals the
    oracle's assembled K bit for bit, the imaginary part equals omega times the
    oracle's assembled M (MATLAB forms K + 1j*omega*M from the two matrices)."""
    from magpackage_b200.plan import ComplexBatch

    cases = list(synth.frequency_sweep_instances(count=4, n_min=2, n_max=9, seed=3))
    plans, nus, sigmas, refs = [], [], [], []
    qw, val, curl = quadrature.reference_data(2)
    for mesh, tags, nu, sigma, omega in cases:
        edges, t2e, sign, m = make_case(oracle_port, mesh.P, mesh.T, tags)
        E = edges.shape[0]
        plans.append(AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign))
        nus.append(dev(nu))
        sigmas.append(dev(sigma))
        I, J, Vk = oracle_port.curl_curl(m, nu, qw, curl)
        _, _, Vm = oracle_port.mass(m, sigma, qw, val)
        refs.append((oracle_matrix(oracle_port, I, J, Vk, E, False), oracle_matrix(oracle_port, I, J, Vm, E, False),
                     omega))
    batch = ComplexBatch(plans, nus, sigmas, [c[4] for c in cases])
    chosen, times, name = batch.tuning()
    assert 0 <= chosen < len(times) and times[chosen] == times[times > 0].min() and name
    assert np.all(times > 0)  # every variant, row blocks and tile blocks, ran on these meshes
    for variant in [chosen] + [v for v in range(len(times)) if v != chosen]:
        batch.select(variant)
        for rep in range(2):  # graph replay is repeatable
            vals = batch.assemble()
            torch.cuda.synchronize()
            for plan, v, (kref, mref, omega) in zip(plans, vals, refs):
                assert_csr_equal(plan.row_ptr, plan.col_idx, v.real.contiguous(), kref)
                im = host(v.imag.contiguous())
                assert bits_equal(im, omega * mref[2]), variant
    batch.close()


def test_batched_complex_unit_sigma_and_negative_omega(oracle_port):
    """A mesh without sigma (sigma = 1: every block conducts and takes the M pass) and
    non-uniform quadrature weights (the kernels' general per-point sums), one whose conductor
    covers only a few blocks, and a negative omega: every variant equals the oracle bit for bit."""
    from magpackage_b200.plan import ComplexBatch

    qw4, val, curl = quadrature.reference_data(2)
    plans, nus, sigmas, refs, omegas = [], [], [], [], []
    for k, (nx, ny, nz) in enumerate(((6, 5, 4), (11, 9, 8))):
        mesh = synth.kuhn_box(nx, ny, nz, seed=11 + k)
        tags = synth.cube_layout(mesh)
        edges, t2e, sign, m = make_case(oracle_port, mesh.P, mesh.T, tags)
        E = edges.shape[0]
        rng = np.random.default_rng(20 + k)
        nu = rng.uniform(0.5, 2.0, mesh.num_elements) * material.NU0
        sigma = None if k == 0 else np.where(tags == synth.IRON, 1e6, 0.0)
        qw = np.array([0.05, 0.04, 0.045, 0.0316666]) if k == 0 else qw4
        I, J, Vk = oracle_port.curl_curl(m, nu, qw, curl)
        _, _, Vm = oracle_port.mass(m, np.ones(mesh.num_elements) if sigma is None else sigma, qw, val)
        plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
        plan.set_quadrature(qw, curl, val)
        plans.append(plan)
        nus.append(dev(nu))
        sigmas.append(None if sigma is None else dev(sigma))
        omegas.append(-2 * np.pi * 60.0 if k == 1 else 2 * np.pi * 400.0)
        refs.append((oracle_matrix(oracle_port, I, J, Vk, E, False), oracle_matrix(oracle_port, I, J, Vm, E, False)))
    batch = ComplexBatch(plans, nus, sigmas, omegas)
    _, times, _ = batch.tuning()
    assert np.all(times > 0)
    for variant in range(len(times)):
        batch.select(variant)
        vals = batch.assemble()
        torch.cuda.synchronize()
        for plan, v, (kref, mref), omega in zip(plans, vals, refs, omegas):
            assert_csr_equal(plan.row_ptr, plan.col_idx, v.real.contiguous(), kref)
            assert bits_equal(host(v.imag.contiguous()), omega * mref[2]), variant
    batch.close()


def test_batched_complex_slot_and_row_paths(oracle_port):
    """A batch mixing a mesh whose off-diagonal entries have at most two contributions (slot
    path), one where a dof shared by two edges breaks that bound (row phase) and one with
    rows of more than 31 entries (slot path, wide positions) is exact on every variant."""
    from magpackage_b200.plan import ComplexBatch

    qw, val, curl = quadrature.reference_data(2)
    plans, nus, sigmas, refs, omegas = [], [], [], [], []
    for kind in ("box", "merged", "pinwheel"):
        if kind == "pinwheel":
            P, T = _pinwheel()
            tags = np.where(np.arange(T.shape[0]) % 3 == 0, synth.ALUMINIUM, synth.AIR).astype(np.int32)
        else:
            mesh = synth.kuhn_box(5, 4, 3, seed=4)
            P, T, tags = mesh.P, mesh.T, synth.cube_layout(mesh)
        edges, t2e, sign = oracle_port.generate_edges(T)
        E = edges.shape[0]
        merged = kind == "merged"
        dofs = np.where(t2e == 1, 0, t2e).astype(np.int32) if merged else t2e
        m = mex_inputs(P, T, dofs, sign, tags)
        rng = np.random.default_rng(7 + len(plans))
        nu = rng.uniform(0.5, 2.0, T.shape[0]) * material.NU0
        sigma = np.where(tags == synth.ALUMINIUM, synth.SIGMA_AL, 0.0)
        plan = AssemblyPlan(P, T, dofs, E, tags, sign)
        assert plan.info.nz_pass == (0 if merged else 1)
        assert plan.info.wide_positions == (1 if kind == "pinwheel" else 0)
        I, J, Vk = oracle_port.curl_curl(m, nu, qw, curl)
        _, _, Vm = oracle_port.mass(m, sigma, qw, val)
        plans.append(plan)
        nus.append(dev(nu))
        sigmas.append(dev(sigma))
        omegas.append(2 * np.pi * (50.0 + 25.0 * len(plans)))
        refs.append((oracle_matrix(oracle_port, I, J, Vk, E, False), oracle_matrix(oracle_port, I, J, Vm, E, False)))
    batch = ComplexBatch(plans, nus, sigmas, omegas)
    _, times, _ = batch.tuning()
    # the tile-block variants need a tile plan on every mesh: the merged-dof and pinwheel
    # meshes have none, so only the row-block variants run here
    assert np.all(times[:4] > 0) and np.all(times[4:] < 0)
    for variant in range(4):
        batch.select(variant)
        vals = batch.assemble()
        torch.cuda.synchronize()
        for plan, v, (kref, mref), omega in zip(plans, vals, refs, omegas):
            assert_csr_equal(plan.row_ptr, plan.col_idx, v.real.contiguous(), kref)
            assert bits_equal(host(v.imag.contiguous()), omega * mref[2]), variant
    batch.close()


# ---- wide rows ---------------------------------------------------------------------------

def _pinwheel(n_blades=12, seed=0):
    """n tetrahedra around one edge (nodes 0, 1 on the axis, a ring of n nodes): that edge's
    CSR row has 3n + 1 entries, more than the compact 31-slot position format holds."""
    rng = np.random.default_rng(seed)
    ang = 2 * np.pi * np.arange(n_blades) / n_blades
    ring = np.stack([np.cos(ang), np.sin(ang), 0.5 + 0.05 * rng.normal(size=n_blades)], axis=1)
    P = np.vstack([[0.0, 0.0, 0.0], [0.0, 0.0, 1.0], ring])
    T = np.array([[0, 1, 2 + i, 2 + (i + 1) % n_blades] for i in range(n_blades)], dtype=np.int32)
    # orient every tetrahedron positively
    for e in range(T.shape[0]):
        a, b, c, d = P[T[e]]
        if np.dot(np.cross(b - a, c - a), d - a) < 0:
            T[e, [2, 3]] = T[e, [3, 2]]
    return P, T


def test_wide_rows_match_oracle_on_every_schedule(oracle_port):
    P, T = _pinwheel()
    tags = np.where(np.arange(T.shape[0]) % 2 == 0, synth.IRON, synth.AIR).astype(np.int32)
    edges, t2e, sign, m = make_case(oracle_port, P, T, tags)
    E = edges.shape[0]
    pk = material.pack_material_data(synth.standard_materials())
    sol = np.random.default_rng(7).normal(0, 0.5, E)
    qw, val, curl = quadrature.reference_data(2)
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    ref = oracle_matrix(oracle_port, I, J, V, E, False)
    plan = AssemblyPlan(P, T, t2e, E, tags, sign)
    assert plan.info.wide_positions == 1 and plan.info.max_row_nnz > 31 and plan.info.nz_pass == 1
    plan.set_materials(pk)
    x = dev(sol)
    assert plan.info.tile_blocks == 0  # wide rows: the tile schedule is not offered
    for sch in available(plan):
        plan.set_schedule(sch)
        v, r = plan.jacobian(x)
        plan.check()
        assert_csr_equal(plan.row_ptr, plan.col_idx, v, ref)
        assert bits_equal(host(r), oracle_port.sparse_vec(Ri, Rv, E)), sch
    K = plan.stiffness(dev(np.full(T.shape[0], 800.0)))
    Ik, Jk, Vk = oracle_port.curl_curl(m, np.full(T.shape[0], 800.0), qw, curl)
    assert_csr_equal(plan.row_ptr, plan.col_idx, K, oracle_matrix(oracle_port, Ik, Jk, Vk, E, False))


# ---- the nonzero-pass schedule's preconditions ----------------------------------------------

def test_nz_schedule_rows_without_incidences_and_merged_dofs(oracle_port):
    """Dofs that no element uses give empty CSR rows, which the nonzero pass skips; dofs shared
    by two edges give off-diagonal entries with more than two contributions, which it cannot
    place: the plan reports it unavailable and the default schedule stays exact."""
    mesh = synth.kuhn_box(5, 4, 3, seed=4)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    E = edges.shape[0]
    pk = material.pack_material_data(synth.standard_materials())
    qw, val, curl = quadrature.reference_data(2)
    # (a) three unused dofs at the end
    n = E + 3
    m = mex_inputs(mesh.P, mesh.T, t2e, sign, tags)
    sol = np.random.default_rng(5).normal(0, 0.05, n)
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, n, tags, sign)
    plan.set_materials(pk)
    assert plan.info.nz_pass == 1
    plan.set_schedule(_lib.SCHEDULE_NZ_ROW_BLOCKS)
    v, r = plan.jacobian(dev(sol))
    assert_csr_equal(plan.row_ptr, plan.col_idx, v, oracle_matrix(oracle_port, I, J, V, n, False))
    assert bits_equal(host(r), oracle_port.sparse_vec(Ri, Rv, n))
    # (b) two edges through the corner node that share no element, (0,1) and (0,6), carry
    # one dof: entries coupling it with the diagonal edge from the corner get four
    # contributions
    assert list(edges[0]) == [0, 1] and list(edges[1]) == [0, 6]
    assert not set(np.where(t2e == 0)[0]) & set(np.where(t2e == 1)[0])
    dofs = np.where(t2e == 1, 0, t2e).astype(np.int32)
    m2 = mex_inputs(mesh.P, mesh.T, dofs, sign, tags)
    I, J, V, Ri, Rv = oracle_port.jacobian(m2, sol[:E], qw, curl, pk, True)
    plan2 = AssemblyPlan(mesh.P, mesh.T, dofs, E, tags, sign)
    plan2.set_materials(pk)
    assert plan2.info.nz_pass == 0 and plan2.info.shared_blocks > 0
    assert plan2.info.schedule == _lib.SCHEDULE_SHARED_ROW_BLOCKS
    with pytest.raises(_lib.MagError):
        plan2.set_schedule(_lib.SCHEDULE_NZ_ROW_BLOCKS)
    v, r = plan2.jacobian(dev(sol[:E]))
    assert_csr_equal(plan2.row_ptr, plan2.col_idx, v, oracle_matrix(oracle_port, I, J, V, E, False))
    assert bits_equal(host(r), oracle_port.sparse_vec(Ri, Rv, E))


def test_stiffness_nonzero_pass_matches_oracle(oracle_port):
    """K(nu) under the nonzero-pass schedule (one launch, no scratch) equals the oracle's
    curl-curl sparse() and the two-pass assembly, on the standard and a general quadrature,
    on a box and on a mesh with rows of more than 31 entries."""
    qw, val, curl = quadrature.reference_data(2)
    qw2 = np.array([0.05, 0.04, 0.045, 0.0316666])
    cases = []
    mesh = synth.kuhn_box(7, 5, 6, seed=13)
    cases.append((mesh.P, mesh.T, synth.cube_layout(mesh)))
    P, T = _pinwheel(n_blades=14, seed=2)
    cases.append((P, T, np.full(T.shape[0], synth.AIR, dtype=np.int32)))
    for P, T, tags in cases:
        edges, t2e, sign, m = make_case(oracle_port, P, T, tags)
        E = edges.shape[0]
        nu = np.random.default_rng(T.shape[0]).uniform(0.2, 5.0, T.shape[0]) * material.NU0
        plan = AssemblyPlan(P, T, t2e, E, tags, sign)
        assert plan.info.schedule in (_lib.SCHEDULE_TILE_BLOCKS, _lib.SCHEDULE_NZ_ROW_BLOCKS)
        for w in (qw, qw2):
            plan.set_quadrature(w, curl, val)
            I, J, V = oracle_port.curl_curl(m, nu, w, curl)
            ref = oracle_matrix(oracle_port, I, J, V, E, False)
            if plan.info.tile_blocks:
                plan.set_schedule(_lib.SCHEDULE_TILE_BLOCKS)
                assert_csr_equal(plan.row_ptr, plan.col_idx, plan.stiffness(dev(nu)), ref)
            plan.set_schedule(_lib.SCHEDULE_NZ_ROW_BLOCKS)
            k_nz = plan.stiffness(dev(nu))
            assert_csr_equal(plan.row_ptr, plan.col_idx, k_nz, ref)
            plan.set_schedule(_lib.SCHEDULE_TWO_PASS)
            assert torch.equal(plan.stiffness(dev(nu)), k_nz)


def test_tile_schedule_absent_dofs(oracle_port):
    """Edges without a dof (-1, as DofHandler gives outside the target regions) on the tile
    schedule: the absent columns' values go to the row's diagonal slot, which the row phase
    overwrites; Jacobian, residual and K(nu) equal the oracle bit for bit."""
    mesh = synth.kuhn_box(10, 9, 8, seed=6)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    E = edges.shape[0]
    dofs = np.where(t2e % 5 == 3, -1, t2e).astype(np.int32)
    m = mex_inputs(mesh.P, mesh.T, dofs, sign, tags)
    sol = np.random.default_rng(3).normal(0, 0.05, E)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    plan = AssemblyPlan(mesh.P, mesh.T, dofs, E, tags, sign)
    plan.set_materials(pk)
    assert plan.info.schedule == _lib.SCHEDULE_TILE_BLOCKS
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    v, r = plan.jacobian(dev(sol))
    plan.check()
    assert_csr_equal(plan.row_ptr, plan.col_idx, v, oracle_matrix(oracle_port, I, J, V, E, False))
    assert bits_equal(host(r), oracle_port.sparse_vec(Ri, Rv, E))
    nu = np.random.default_rng(4).uniform(0.2, 5.0, mesh.num_elements) * material.NU0
    Ik, Jk, Vk = oracle_port.curl_curl(m, nu, qw, curl)
    assert_csr_equal(plan.row_ptr, plan.col_idx, plan.stiffness(dev(nu)), oracle_matrix(oracle_port, Ik, Jk, Vk, E, False))
    plan.check()
    plan.close()


def test_tile_schedule_shuffled_numbering_and_unused_dofs(oracle_port):
    """The tile schedule on a mesh whose node and element numbering is shuffled (a block's
    rows are then scattered over the CSR in short runs) with three unused dofs at the end
    (rows without incidences, whose residual is 0): Jacobian, residual-only pass and K(nu)
    equal the oracle bit for bit, and a repeated call gives the same bits."""
    base = synth.kuhn_box(9, 8, 7, seed=4)
    rng = np.random.default_rng(4)
    perm = rng.permutation(base.num_nodes)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    P = base.P[perm]
    T = inv[base.T][rng.permutation(base.num_elements)].astype(np.int32)
    mesh = synth.BoxMesh(P=P, T=T, shape=base.shape, size=base.size)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign, m = make_case(oracle_port, P, T, tags)
    E = edges.shape[0]
    n = E + 3
    sol = np.random.default_rng(9).normal(0, 0.05, n) * 10.0 ** np.random.default_rng(8).uniform(-1.5, 0.5, n)
    pk = material.pack_material_data(synth.standard_materials())
    qw, val, curl = quadrature.reference_data(2)
    plan = AssemblyPlan(P, T, t2e, n, tags, sign)
    plan.set_materials(pk)
    assert plan.info.schedule == _lib.SCHEDULE_TILE_BLOCKS and plan.info.tile_colors == 2
    x = dev(sol)
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    v, r = plan.jacobian(x)
    _, r0 = plan.jacobian(x, calc_j=False)
    plan.check()
    assert_csr_equal(plan.row_ptr, plan.col_idx, v, oracle_matrix(oracle_port, I, J, V, n, False))
    rr = oracle_port.sparse_vec(Ri, Rv, n)
    assert bits_equal(host(r), rr) and bits_equal(host(r0), rr)
    assert np.all(host(r)[E:] == 0.0)
    v2, r2 = plan.jacobian(x)
    assert torch.equal(v.view(torch.int64), v2.view(torch.int64)) and torch.equal(r.view(torch.int64),
                                                                                   r2.view(torch.int64))
    for variant in (1, 2, 3, 0):  # every launch shape gives the same bits
        plan.set_tile_variant(variant)
        v3, r3 = plan.jacobian(x)
        plan.check()
        assert torch.equal(v.view(torch.int64), v3.view(torch.int64)), variant
        assert torch.equal(r.view(torch.int64), r3.view(torch.int64)), variant
    with pytest.raises(_lib.MagError):
        plan.set_tile_variant(4)
    for waves in (0, 2, 1):  # every staging depth too
        plan.set_tile_prefetch(waves)
        v3, r3 = plan.jacobian(x)
        plan.check()
        assert torch.equal(v.view(torch.int64), v3.view(torch.int64)), waves
    with pytest.raises(_lib.MagError):
        plan.set_tile_prefetch(3)
    # the autotuner times all 12 pairs, keeps one, and leaves the same bits in its outputs
    vt, rt = plan.new_values(), plan.new_vector()
    variant, depth, times = plan.tune(x, vt, rt, reps=2)
    plan.check()
    assert 0 <= variant < 4 and 0 <= depth < 3 and np.all(times > 0) and times[variant, depth] == times.min()
    assert torch.equal(v.view(torch.int64), vt.view(torch.int64)) and torch.equal(r.view(torch.int64),
                                                                                    rt.view(torch.int64))
    v4, _ = plan.jacobian(x)
    assert torch.equal(v.view(torch.int64), v4.view(torch.int64))
    plan.set_schedule(_lib.SCHEDULE_TWO_PASS)
    with pytest.raises(_lib.MagError):  # the tuner is for the tile schedule only
        plan.tune(x, vt, rt)
    plan.set_schedule(_lib.SCHEDULE_TILE_BLOCKS)
    nu = np.random.default_rng(5).uniform(0.2, 5.0, T.shape[0]) * material.NU0
    Ik, Jk, Vk = oracle_port.curl_curl(m, nu, qw, curl)
    assert_csr_equal(plan.row_ptr, plan.col_idx, plan.stiffness(dev(nu)), oracle_matrix(oracle_port, Ik, Jk, Vk, n, False))
    plan.check()
    plan.close()
