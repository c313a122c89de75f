"""Parity at the benchmark configurations' own sizes.

The smaller parity tests pin every schedule on meshes up to 30^3; these run the default
path on the full meshes of the workloads: the 60^3 (1.296M tets, 25.0M nonzeros) and 110^3
(7.986M tets, 153.6M nonzeros, where int32 row pointers and the block planner are at
their largest) Froehlich Jacobians, the 64-mesh complex frequency batch, and the E-core
transient box (40x40x20, 192k tets) after one Newton-converged step. Each compares the
CSR pattern bit for bit and reports the per-nonzero maximum relative error and the
Frobenius relative error against the oracle (the restated MATLAB sparse() of the
reference MEX triplets); the bound is bit equality (the required bound is 1e-12 relative per nonzero).
"""
import json

import numpy as np
import pytest
import torch
from conftest import bits_equal

from magpackage_b200 import material, quadrature, synth
from magpackage_b200.plan import AssemblyPlan, ComplexBatch, generate_edges
from oracle.oracle import mex_inputs

pytestmark = pytest.mark.gpu


def parity_report(name, vals, ref, res=None, ref_res=None):
    v, r = np.asarray(vals, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    nz = r != 0
    rel = np.abs(v[nz] - r[nz]) / np.abs(r[nz])
    out = {"case": name, "nnz": int(v.size), "bit_equal": bits_equal(v, r),
           "max_rel": float(rel.max()) if rel.size else 0.0,
           "frobenius_rel": float(np.linalg.norm(v - r) / max(np.linalg.norm(r), 1e-300))}
    if res is not None:
        a, b = np.asarray(res), np.asarray(ref_res)
        bz = b != 0
        out["residual_bit_equal"] = bits_equal(a, b)
        out["residual_max_rel"] = float((np.abs(a[bz] - b[bz]) / np.abs(b[bz])).max()) if bz.any() else 0.0
    print("parity " + json.dumps(out))
    return out


@pytest.mark.parametrize("n", [60, 110])
def test_froehlich_jacobian_at_workload_size(oracle_port, n):
    """Configs 2 and 5: the bench's own mesh, layout and state (seeded like bench.py)."""
    mesh = synth.kuhn_box(n, seed=0)
    tags = synth.cube_layout(mesh)
    packed = material.pack_material_data(synth.standard_materials())
    edges, t2e, sign = generate_edges(mesh.T)
    E = int(edges.shape[0])
    assert E == 7 * n ** 3 + 9 * n ** 2 + 3 * n
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    plan.set_materials(packed)
    assert plan.nnz == 115 * n ** 3 + 45 * n ** 2 + 3 * n
    sol = np.random.default_rng(1).normal(0.0, 1e-3, E)
    vals, res = plan.jacobian(torch.as_tensor(sol, device="cuda"))
    rp, ci = plan.row_ptr.cpu().numpy(), plan.col_idx.cpu().numpy()
    vals, res = vals.cpu().numpy(), res.cpu().numpy()
    plan.close()
    del plan
    torch.cuda.empty_cache()
    e0, t0, s0 = oracle_port.generate_edges(mesh.T)
    assert np.array_equal(t0, t2e.cpu().numpy())
    m = mex_inputs(mesh.P, mesh.T, t0, s0, tags)
    qw, val, curl = quadrature.reference_data(2)
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, packed, True)
    del m
    rrp, rci, rv = oracle_port.sparse_csr(I, J, V, E, drop_zeros=False)
    del I, J, V
    rres = oracle_port.sparse_vec(Ri, Rv, E)
    assert np.array_equal(rp, rrp), "row_ptr differs"
    assert np.array_equal(ci, rci), "col_idx differs"
    rep = parity_report(f"jacobian_{n}", vals, rv, res, rres)
    assert rep["bit_equal"] and rep["residual_bit_equal"]


def test_frequency_batch_at_workload_size(oracle_port):
    """Config 3: all 64 meshes (8^3 .. 48^3) in one graph-captured launch; the largest
    instance and three others against the oracle's K and omega*M."""
    qw, val, curl = quadrature.reference_data(2)
    cases = list(synth.frequency_sweep_instances(count=64, seed=0))
    plans, nus, sigmas, omegas, keep = [], [], [], [], []
    for mesh, tags, nu, sigma, omega in cases:
        edges, t2e, sign = generate_edges(mesh.T)
        plans.append(AssemblyPlan(mesh.P, mesh.T, t2e, int(edges.shape[0]), tags, sign))
        nus.append(torch.as_tensor(nu, device="cuda"))
        sigmas.append(torch.as_tensor(sigma, device="cuda"))
        omegas.append(omega)
    assert sum(c[0].num_elements for c in cases) > 12_000_000
    batch = ComplexBatch(plans, nus, sigmas, omegas)
    chosen, times, _ = batch.tuning()
    # the tuned variant and the fastest of the other family (row blocks 0-3, tile blocks 4-5)
    other = [v for v in range(len(times)) if (v >= 4) != (chosen >= 4) and times[v] > 0]
    variants = [chosen] + ([min(other, key=lambda v: times[v])] if other else [])
    refs = {}
    for k in (0, 21, 42, 63):
        mesh, tags, nu, sigma, omega = cases[k]
        e0, t0, s0 = oracle_port.generate_edges(mesh.T)
        E = e0.shape[0]
        m = mex_inputs(mesh.P, mesh.T, t0, s0, tags)
        I, J, Vk = oracle_port.curl_curl(m, nu, qw, curl)
        _, _, Vm = oracle_port.mass(m, sigma, qw, val)
        krp, kci, kv = oracle_port.sparse_csr(I, J, Vk, E, drop_zeros=False)
        _, _, mv = oracle_port.sparse_csr(I, J, Vm, E, drop_zeros=False)
        assert np.array_equal(plans[k].row_ptr.cpu().numpy(), krp)
        assert np.array_equal(plans[k].col_idx.cpu().numpy(), kci)
        refs[k] = (kv, omega * mv)
    for variant in variants:
        batch.select(variant)
        vals = [v.cpu().numpy() for v in batch.assemble()]
        for k, (kv, omv) in refs.items():
            re = parity_report(f"batch_v{variant}_{k}_K", vals[k].real.copy(), kv)
            im = parity_report(f"batch_v{variant}_{k}_omegaM", vals[k].imag.copy(), omv)
            assert re["bit_equal"] and im["bit_equal"], variant
    batch.close()
    for p in plans:
        p.close()


def test_transient_box_after_one_step(oracle_port):
    """Config 4 (the E-core box, 40x40x20 hexahedra x6): one backward-Euler step at the
    source peak, Newton to ||R|| <= 1e-8 max(||F||, 1) from A = 0; the Jacobian and residual
    at the converged state (saturated iron) against the oracle."""
    from magpackage_b200.transient import TransientConfig, TransientProblem

    cfg = TransientConfig()
    prob = TransientProblem(cfg)
    assert prob.mesh.num_elements == 192_000
    x0 = torch.zeros(prob.num_dofs, dtype=torch.float64, device="cuda")
    x, st = prob.step(x0, 0.25 / cfg.freq, 1)
    assert st.converged and st.res <= st.tol_abs
    iron_nu = prob.element_nu(x)[torch.as_tensor(prob.tags == synth.IRON, device="cuda")]
    assert float(iron_nu.max()) > 10 * float(iron_nu.min())  # the step reached the nonlinear range
    xs = x.cpu().numpy()
    vals, res = prob.plan.jacobian(x)
    vals, res = vals.cpu().numpy(), res.cpu().numpy()
    mesh = prob.mesh
    e0, t0, s0 = oracle_port.generate_edges(mesh.T)
    E = e0.shape[0]
    m = mex_inputs(mesh.P, mesh.T, t0, s0, prob.tags)
    qw, val, curl = quadrature.reference_data(2)
    packed = material.pack_material_data(synth.standard_materials())
    I, J, V, Ri, Rv = oracle_port.jacobian(m, xs, qw, curl, packed, True)
    rrp, rci, rv = oracle_port.sparse_csr(I, J, V, E, drop_zeros=False)
    assert np.array_equal(prob.rp.cpu().numpy(), rrp) and np.array_equal(prob.ci.cpu().numpy(), rci)
    rep = parity_report("transient_box_step", vals, rv, res, oracle_port.sparse_vec(Ri, Rv, E))
    assert rep["bit_equal"] and rep["residual_bit_equal"]
    prob.close()
