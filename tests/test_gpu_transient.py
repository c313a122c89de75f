"""Newton-driver pieces on the GPU: element nu, CSR algebra, PCG, the coil source, the
seeded tangent, and the learned warm start against the plain one (magpackage_b200/transient.py)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from magpackage_b200 import _lib, synth
from magpackage_b200.material import pack_material_data
from magpackage_b200.plan import AssemblyPlan, generate_edges
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _plan(n=6, seed=3):
    mesh = synth.kuhn_box(n, seed=seed)
    tags = synth.cube_layout(mesh)
    edges, t2e, _ = generate_edges(mesh.T)
    E = edges.shape[0]
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags)
    pk = pack_material_data(synth.standard_materials())
    plan.set_materials(pk)
    return mesh, tags, edges.cpu().numpy(), plan, pk


def _scipy(plan, vals):
    rp, ci = plan.row_ptr.cpu().numpy(), plan.col_idx.cpu().numpy()
    return sp.csr_matrix((vals.cpu().numpy(), ci, rp), shape=(plan.num_dofs, plan.num_dofs))


def test_element_nu_matches_oracle():
    mesh, tags, edges, plan, pk = _plan()
    rng = np.random.default_rng(0)
    # spread |B| over the whole table, including extrapolation beyond its last break
    x = torch.as_tensor(rng.normal(0, 1, plan.num_dofs) * np.exp(rng.uniform(-8, 1, plan.num_dofs)) * 0.05,
                        device="cuda")
    _, bsq = plan.element_b(x, want_vec=False)
    nu = torch.empty(plan.num_elements, dtype=torch.float64, device="cuda")
    dnu = torch.empty_like(nu)
    _lib.check(_lib.lib().mag_element_nu(plan._h, _ptr(x), _ptr(nu), _ptr(dnu), _lib.stream_ptr()))
    nu_ref, dnu_ref = Port().material_eval(bsq.cpu().numpy(), tags, pk)
    assert np.array_equal(nu.cpu().numpy(), nu_ref)
    assert np.array_equal(dnu.cpu().numpy(), dnu_ref)
    iron = tags == synth.IRON
    assert np.unique(nu.cpu().numpy()[iron]).size > 10  # the spline, not a constant, was exercised


def test_spmv_and_dirichlet_match_scipy():
    _, _, _, plan, _ = _plan(7)
    L = _lib.lib()
    rng = np.random.default_rng(1)
    vals = torch.as_tensor(rng.normal(size=plan.nnz), device="cuda")
    x = torch.as_tensor(rng.normal(size=plan.num_dofs), device="cuda")
    y = torch.empty_like(x)
    _lib.check(L.mag_csr_spmv(plan.num_dofs, _ptr(plan.row_ptr), _ptr(plan.col_idx), _ptr(vals), _ptr(x), _ptr(y),
                              _lib.stream_ptr()))
    A = _scipy(plan, vals)
    assert np.allclose(y.cpu().numpy(), A @ x.cpu().numpy(), rtol=1e-13, atol=1e-13)
    fixed = (rng.random(plan.num_dofs) < 0.2).astype(np.uint8)
    rhs = torch.as_tensor(rng.normal(size=plan.num_dofs), device="cuda")
    rhs0 = rhs.cpu().numpy().copy()
    fd = torch.as_tensor(fixed, device="cuda")
    _lib.check(L.mag_csr_apply_dirichlet(plan.num_dofs, _ptr(plan.row_ptr), _ptr(plan.col_idx), _ptr(vals),
                                         _ptr(fd), _ptr(rhs), _lib.stream_ptr()))
    free = sp.diags((1 - fixed).astype(float))
    ref = (free @ A @ free + sp.diags(fixed.astype(float))).toarray()
    assert np.array_equal(_scipy(plan, vals).toarray(), ref)
    rhs0[fixed == 1] = 0.0
    assert np.array_equal(rhs.cpu().numpy(), rhs0)


def test_pcg_solves_spd_system_deterministically():
    mesh, tags, edges, plan, _ = _plan(8)
    L = _lib.lib()
    nu = torch.as_tensor(np.where(tags == synth.IRON, 80.0, 8e5), device="cuda")
    K = plan.stiffness(nu)
    M = plan.mass(None)
    dK = _scipy(plan, K).diagonal().mean()
    dM = _scipy(plan, M).diagonal().mean()
    A = K + (1e-2 * dK / dM) * M  # positive definite and well conditioned (the mass term lifts grad modes)
    rng = np.random.default_rng(2)
    b = torch.as_tensor(rng.normal(size=plan.num_dofs), device="cuda")
    h = C.c_void_p()
    _lib.check(L.mag_pcg_create(plan.num_dofs, C.byref(h)))
    sols = []
    try:
        for _ in range(2):
            x = torch.zeros_like(b)
            it, rel, st = C.c_int(), C.c_double(), C.c_int()
            _lib.check(L.mag_pcg_solve(h, _ptr(plan.row_ptr), _ptr(plan.col_idx), _ptr(A), _ptr(b), _ptr(x), 1e-10,
                                       100000, C.byref(it), C.byref(rel), C.byref(st), _lib.stream_ptr()))
            assert st.value == 1 and rel.value <= 1e-10 and it.value > 10
            sols.append(x.cpu().numpy())
    finally:
        L.mag_pcg_destroy(h)
    As = _scipy(plan, A)
    bn = b.cpu().numpy()
    assert np.linalg.norm(As @ sols[0] - bn) <= 2e-10 * np.linalg.norm(bn)
    assert np.array_equal(sols[0], sols[1])


def test_pcg_auxiliary_space_cuts_iterations():
    """Curl-curl with a tiny mass shift: the gradient space turns ~10^4 Jacobi iterations into hundreds."""
    from magpackage_b200.transient import TransientConfig, TransientProblem

    prob = TransientProblem(TransientConfig(nx=12, ny=12, nz=6, steps=1))
    try:
        rng = np.random.default_rng(3)
        vals, _ = prob.plan.jacobian(torch.zeros(prob.num_dofs, dtype=torch.float64, device="cuda"))
        A = vals + prob.reg * prob.m_reg
        prob.dirichlet(A, None)
        xt = torch.as_tensor(rng.normal(size=prob.num_dofs), device="cuda") * prob.free
        b = prob.spmv(A, xt)
        prob._A.copy_(A)
        x = torch.zeros_like(b)
        it_aux, rel, st = prob.solve(prob._A, b, x)
        assert st == 1
        res_aux = float(torch.linalg.vector_norm(prob.spmv(A, x) - b) / torch.linalg.vector_norm(b))
        _lib.check(prob.lib.mag_pcg_set_aux(prob._pcg, 0, None, None, None, None, None, None, None))
        x2 = torch.zeros_like(b)
        it_jac, _, _ = prob.solve(prob._A, b, x2)
        assert res_aux < 1e-8
        assert it_aux * 4 < it_jac, (it_aux, it_jac)
    finally:
        prob.close()


def test_coil_source_is_discretely_divergence_free():
    from magpackage_b200.transient import TransientConfig, TransientProblem

    prob = TransientProblem(TransientConfig(nx=20, ny=20, nz=10, steps=2))
    try:
        F = prob.source(0.005).cpu().numpy()  # peak current
        e = prob.edges
        div = np.zeros(prob.mesh.num_nodes)
        np.add.at(div, e[:, 1], F)
        np.add.at(div, e[:, 0], -F)
        assert np.abs(F).max() > 0
        assert np.abs(div).max() <= 1e-10 * np.abs(F).max()
        jm = torch.linalg.vector_norm(prob.j_unit, dim=1).cpu().numpy()
        coil = prob.tags == synth.COIL
        assert jm[prob.tags == synth.IRON].max() <= 1e-9 * jm.max()  # no current in the core
        assert jm[coil].sum() > 0.8 * jm.sum()  # the current flows in the winding
        assert 0.7 < np.median(jm[coil & (jm > 0.5)]) < 1.3
    finally:
        prob.close()


def test_seeded_jacobian_with_unit_scale_is_the_jacobian():
    mesh, tags, edges, plan, _ = _plan(6)
    L = _lib.lib()
    rng = np.random.default_rng(5)
    x = torch.as_tensor(rng.normal(0, 0.02, plan.num_dofs), device="cuda")
    v0, r0 = plan.jacobian(x)
    ones = torch.ones(plan.num_elements, dtype=torch.float64, device="cuda")
    v1, r1 = plan.new_values(), plan.new_vector()
    _lib.check(L.mag_assemble_jacobian_seeded(plan._h, _ptr(x), _ptr(ones), _ptr(v1), _ptr(r1), _lib.stream_ptr()))
    assert torch.equal(r0, r1)  # the residual is the unseeded one, bit for bit
    assert torch.allclose(v0, v1, rtol=1e-13, atol=1e-12 * float(v0.abs().max()))
    # a seed nu equal to the element's own nu keeps the tangent where it is (beta = 1)
    nu = torch.empty(plan.num_elements, dtype=torch.float64, device="cuda")
    _lib.check(L.mag_element_nu(plan._h, _ptr(x), _ptr(nu), None, _lib.stream_ptr()))
    beta = torch.empty_like(nu)
    _lib.check(L.mag_seed_midpoint(plan._h, _ptr(x), _ptr(nu), 4.0, _ptr(beta), _lib.stream_ptr()))
    from magpackage_b200.material import NU0

    iron = torch.as_tensor(tags == synth.IRON, device="cuda")
    # where nu is below its clamp at nu0 the table is invertible and the midpoint is the state itself
    inv = iron & (nu < NU0 * (1 - 1e-12))
    assert int(inv.sum()) > 20
    assert torch.allclose(beta[inv], torch.ones_like(beta[inv]), rtol=1e-6)
    assert torch.all(beta[~iron] == 1.0)


def test_learned_warm_start_beats_plain():
    """The config-4 time discretisation (dt = 1e-4, 200 steps) on a 20 x 20 x 10 box: plain warm
    start on every step; an MLP trained on steps 1-100 seeds the first Jacobian of steps
    101-200. Every step of every mode reaches the same RHS-relative tolerance; the learned
    seed needs fewer Newton iterations and fewer assemblies than the plain warm start, and
    seeding with the converged nu (the bound for any predictor) does better still."""
    from magpackage_b200.transient import TransientConfig, compare

    out = compare(TransientConfig(nx=20, ny=20, nz=10), epochs=120, batch=8192, lr=2e-3)
    p, l, i = out["plain"], out["learned"], out["ideal"]
    assert p["converged"] and l["converged"] and i["converged"]
    assert max(p["max_res_over_tol"], l["max_res_over_tol"], i["max_res_over_tol"]) <= 1.0
    print({k: (out[k]["newton"], out[k]["assemblies"], round(out[k]["gpu_ms"])) for k in ("plain", "learned", "ideal")})
    assert out["train"]["loss_last"] < 0.5 * out["train"]["loss_first"]
    assert l["newton"] < p["newton"] and l["assemblies"] < p["assemblies"]
    assert i["newton"] <= l["newton"]
    assert l["nu_rel_err_median"] < 0.05


def test_seeded_jacobian_tile_schedule_equals_two_pass():
    """The seeded Jacobian through the tile schedule (one launch, no scratch) equals the
    two-pass element kernel + row reduction bit for bit, with scales spread over the trust
    region, the residual included."""
    mesh, tags, edges, plan, _ = _plan(9, seed=7)
    assert plan.info.schedule == _lib.SCHEDULE_TILE_BLOCKS
    L = _lib.lib()
    rng = np.random.default_rng(11)
    x = torch.as_tensor(rng.normal(0, 0.05, plan.num_dofs), device="cuda")
    beta = torch.as_tensor(rng.uniform(0.8, 1.25, plan.num_elements), device="cuda")
    out = {}
    for sch in (_lib.SCHEDULE_TILE_BLOCKS, _lib.SCHEDULE_TWO_PASS):
        plan.set_schedule(sch)
        v, r = plan.new_values(), plan.new_vector()
        _lib.check(L.mag_assemble_jacobian_seeded(plan._h, _ptr(x), _ptr(beta), _ptr(v), _ptr(r),
                                                  _lib.stream_ptr()))
        plan.check()
        out[sch] = (v, r)
    (v1, r1), (v2, r2) = out[_lib.SCHEDULE_TILE_BLOCKS], out[_lib.SCHEDULE_TWO_PASS]
    assert torch.equal(v1.view(torch.int64), v2.view(torch.int64))
    assert torch.equal(r1.view(torch.int64), r2.view(torch.int64))
    plan.close()
