"""Right-hand-side kernels on the GPU against the oracle, bit for bit: the winding vector
(assemble_winding_kernel_mex.cpp) and the source vector (assemble_source_kernel_mex.cpp),
through the MEX-compatible entry points (golden fixtures of the reference) and the mesh
handle (sparse(I(valid), 1, V(valid), Ndof, 1) of the oracle's pairs)."""
import numpy as np
import pytest
import torch
from conftest import bits_equal, load_golden

from magpackage_b200 import _lib, quadrature, synth
from magpackage_b200.assembler import Assembler, DofHandler, Mesh, Winding
from magpackage_b200.plan import AssemblyPlan
from oracle.oracle import mex_inputs

pytestmark = pytest.mark.gpu


def _mex_winding(L, m, coil, field, udir, scale, qw, val):
    p = _lib.dptr
    ne = m.ne
    I, V = np.zeros(6 * ne), np.zeros(6 * ne)
    f = None if field is None else np.ascontiguousarray(field, dtype=np.float64)
    u = np.ascontiguousarray(udir, dtype=np.float64)
    _lib.check(L.mag_mex_winding(p(m.P), m.nn, p(m.T), ne, p(m.Dofs), p(m.Signs), p(m.Tags), float(coil), p(f),
                                 p(u), float(scale), p(qw), qw.size, p(val), p(I), p(V)))
    return I, V


@pytest.mark.parametrize("name", ["one_hex", "cube3"])
def test_mex_winding_and_source_match_golden(name):
    d = load_golden(name)
    L = _lib.lib()
    m = mex_inputs(d["P"], d["T0"], d["t2e"], d["sign"], d["tags"])
    qw, val = np.ascontiguousarray(d["qw"]), np.ascontiguousarray(d["val"])
    for field, key in ((None, "u"), (d["win_field"], "f")):
        I, V = _mex_winding(L, m, d["win_coil"], field, d["win_dir"], d["win_scale"], qw, val)
        assert bits_equal(I, d[f"win_{key}_I"]) and bits_equal(V, d[f"win_{key}_V"])
    js = np.ascontiguousarray(d["src_js"])
    I, V = np.zeros(6 * m.ne), np.zeros(6 * m.ne)
    p = _lib.dptr
    _lib.check(L.mag_mex_source(p(m.P), m.nn, p(m.T), m.ne, p(m.Dofs), p(m.Signs), p(js), p(qw), qw.size, p(val),
                                p(I), p(V)))
    assert bits_equal(I, d["src_I"]) and bits_equal(V, d["src_V"])


def _vector(port, I, V, n):
    k = I > 0
    return port.sparse_vec(I[k], V[k], n)


@pytest.mark.parametrize("coil", [synth.IRON, synth.ALUMINIUM, 77])
def test_winding_vector_matches_oracle(oracle_port, coil):
    mesh = synth.kuhn_box(7, 6, 5, seed=21)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    E = edges.shape[0]
    dofs = t2e.copy()
    rng = np.random.default_rng(coil)
    dofs[rng.random(dofs.shape) < 0.05] = -1  # edges without an unknown
    m = mex_inputs(mesh.P, mesh.T, dofs, sign, tags)
    qw, val, curl = quadrature.reference_data(2)
    plan = AssemblyPlan(mesh.P, mesh.T, dofs, E, tags, sign)
    field = rng.normal(size=(mesh.num_elements, 3))
    udir = np.array([0.2, 0.9, -0.4])
    for f in (None, field):
        I, V = oracle_port.winding(m, float(coil), f, udir, 3.3e5, qw, val)
        ref = _vector(oracle_port, I, V, E)
        got = plan.winding(coil, udir, 3.3e5, dir_field=None if f is None else torch.as_tensor(f, device="cuda"))
        assert bits_equal(got.cpu().numpy(), ref)
        assert (np.abs(ref).max() > 0) == (coil != 77)
        Ig, Vg = _mex_winding(_lib.lib(), m, coil, f, udir, 3.3e5, qw, val)
        assert bits_equal(Ig, I) and bits_equal(Vg, V)


def test_assembler_winding_surface(oracle_port):
    mesh_s = synth.kuhn_box(6, seed=2)
    tags = synth.cube_layout(mesh_s)
    mesh = Mesh(mesh_s.P, mesh_s.T, tags)
    dh = DofHandler(mesh)
    dh.distribute_dofs()
    asm = Assembler(mesh, dh)
    w1 = Winding.create("A", synth.IRON, 120, 0.5, 2e-3, (0, 0, 2.0))
    w2 = Winding.create("B", synth.ALUMINIUM, 40, 0.1, 1e-3, (1.0, 1.0, 0))
    assert np.allclose(np.linalg.norm(w1.Direction), 1.0) and np.allclose(np.linalg.norm(w2.Direction), 1.0)
    w2.set_direction_field(np.random.default_rng(1).normal(size=(mesh.num_elements, 3)))
    C = asm.assemble_winding([w1, w2])
    assert C.shape == (dh.NumGlobalDofs, 2)
    dofs, signs = (torch.as_tensor(a).cpu().numpy() for a in dh.pack_for_kernel())
    m = mex_inputs(mesh_s.P, mesh_s.T, dofs, signs, tags)
    qw, val, curl = quadrature.reference_data(2)
    for k, w in enumerate((w1, w2)):
        I, V = oracle_port.winding(m, float(w.RegionID), w.DirectionField, w.Direction, w.Turns / w.CrossSectionArea,
                                   qw, val)
        assert bits_equal(C[:, k].cpu().numpy(), _vector(oracle_port, I, V, dh.NumGlobalDofs))
    with pytest.raises(ValueError):
        w2.set_direction_field(np.zeros((3, 3)))
        asm.assemble_winding(w2)


@pytest.mark.parametrize("flip", [False, True])
def test_element_b_matches_postprocessor(oracle_port, flip):
    """mag_element_b against PostProcessor.computeElementB restated (PostProcessor.m:64-126):
    B per element within 1e-12 of its rounding scale (MATLAB's BLAS products have no fixed
    summation order, so this is a tolerance, not a bit comparison), |B|^2 = B.B bit for bit;
    with the mesh's own signs and with explicitly flipped ones."""
    from oracle.oracle import element_b
    from test_oracle import uniform_field_edges

    mesh = synth.kuhn_box(9, 7, 8, seed=5)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = oracle_port.generate_edges(mesh.T)
    if flip:
        sign = sign.copy()
        sign[::3] *= -1
    E = edges.shape[0]
    plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, tags, sign)
    rng = np.random.default_rng(4)
    for sol in (rng.normal(0, 1e-2, E), uniform_field_edges(mesh.P, edges, np.array([0.2, 0.5, -1.1]))):
        b, bsq = plan.element_b(torch.as_tensor(sol, device="cuda"))
        b, bsq = b.cpu().numpy(), bsq.cpu().numpy()
        B, scale = element_b(mesh.P, mesh.T, t2e, sign, sol)
        assert np.all(np.abs(b - B) <= 1e-12 * scale + 1e-300)
        assert bits_equal(bsq, (b[:, 0] * b[:, 0] + b[:, 1] * b[:, 1]) + b[:, 2] * b[:, 2])
    plan.close()
