"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own MEX element kernels (src/mex/*.cpp compiled unchanged
into oracle/_ref/libref_mex.so by oracle/Makefile) on small inputs and stores
inputs + outputs as .npz. The reference tree is only needed to (re)generate;
the committed fixtures travel with the tests.

Cases:
  unit_tet   -- the reference's known-answer case (tests/test_mex_assembly.m:32-73):
                unit tetrahedron, Dofs 1..6, Signs [1 -1 1 -1 1 -1], Nu = 500.
  one_hex    -- one hexahedron split into 6 tetrahedra, iron (Froehlich spline).
  cube3      -- 3x3x3 jittered Kuhn cube with the air/iron/aluminium layout and a
                random edge field large enough to drive the iron spline through
                its interior pieces, the extrapolation branch and the clamps.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from magpackage_b200 import material, quadrature, synth  # noqa: E402
from oracle.oracle import Port, RefMex, build, mex_inputs  # noqa: E402


def run_case(name, P, T0, tags, matlib, sol_scale, seed, sigma, js_iron):
    port, ref = Port(), RefMex()
    edges, t2e, sign = port.generate_edges(T0)
    E = edges.shape[0]
    m = mex_inputs(P, T0, t2e, sign, tags)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(matlib)
    rng = np.random.default_rng(seed)
    # log-spread magnitudes: elements land in interior pieces, past maxBSq and in the clamps
    sol = rng.normal(0.0, 1.0, E) * sol_scale * 10.0 ** rng.uniform(-2.0, 0.5, E)
    out = {}
    I, J, V, Ri, Rv = ref.jacobian(m, sol, qw, curl, pk, True)
    out.update(jac_I=I, jac_J=J, jac_V=V, jac_Ridx=Ri, jac_Rval=Rv)
    _, _, _, Ri0, Rv0 = ref.jacobian(m, sol, qw, curl, pk, False)
    out.update(res_only_Ridx=Ri0, res_only_Rval=Rv0)
    nu = np.where(tags == synth.IRON, material.NU0 / 1000.0, material.NU0)
    _, _, Vk = ref.curl_curl(m, nu, qw, curl)
    sig = np.where(tags == synth.ALUMINIUM, synth.SIGMA_AL, 0.0)
    _, _, Vm = ref.mass(m, sig, qw, val)
    _, _, Vm1 = ref.mass(m, None, qw, val)
    js = np.zeros((T0.shape[0], 3))
    js[tags == synth.IRON] = js_iron
    Is, Vs = ref.source(m, js, qw, val)
    out.update(cc_nu=nu, cc_V=Vk, mass_sigma=sig, mass_V=Vm, mass1_V=Vm1, src_js=js, src_I=Is,
               src_V=Vs)
    # winding vector of the iron region: uniform direction, then a per-element direction field
    wdir, wscale = np.array([0.3, -0.5, 0.8]), 250.0 / 2.5e-3
    wfield = rng.normal(0.0, 1.0, (T0.shape[0], 3))
    Iu, Vu = ref.winding(m, float(synth.IRON), None, wdir, wscale, qw, val)
    If, Vf = ref.winding(m, float(synth.IRON), wfield, wdir, wscale, qw, val)
    out.update(win_coil=np.array(float(synth.IRON)), win_dir=wdir, win_scale=np.array(wscale),
               win_field=wfield, win_u_I=Iu, win_u_V=Vu, win_f_I=If, win_f_V=Vf)
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"), P=P, T0=T0, tags=tags, edges=edges, t2e=t2e, sign=sign,
        sol=sol, qw=qw, curl=curl, val=val, mat_lin=pk.lin, mat_isnon=pk.is_non, mat_maxb=pk.max_b,
        mat_brk=pk.breaks, mat_coe=pk.coefs, mat_start=pk.start, mat_cnt=pk.count,
        mat_coestart=pk.coe_start, **out)
    print(f"{name}: Ne={T0.shape[0]} E={E}")


def unit_tet():
    ref = RefMex()
    P = np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    m = mex_inputs(P, np.array([[0, 1, 2, 3]]), np.arange(6)[None, :], np.array([[1, -1, 1, -1, 1, -1]]),
                   np.array([1]))
    qw, val, curl = quadrature.reference_data(2)
    I, J, V = ref.curl_curl(m, np.array([500.0]), qw, curl)
    np.savez_compressed(os.path.join(HERE, "unit_tet.npz"), P=P, I=I, J=J, V=V, qw=qw, curl=curl)
    print("unit_tet: 36 triplets")


def main():
    build()
    unit_tet()
    iron_mats = {synth.IRON: material.create_nonlinear(*material.froehlich_bh())}
    hexm = synth.kuhn_box(1, jitter=0.0)
    run_case("one_hex", hexm.P, hexm.T, np.full(6, synth.IRON, dtype=np.int32),
             {**iron_mats, synth.AIR: material.create_linear_nu(material.NU0)}, 0.8, 11, None,
             (1e6, 0, 0))
    mesh = synth.kuhn_box(3, seed=5)
    tags = synth.cube_layout(mesh)
    tags[:18] = synth.IRON  # iron at the cube corner too, so several iron elements see large fields
    run_case("cube3", mesh.P, mesh.T, tags, synth.standard_materials(), 0.12, 7, None, (3e5, -1e5, 2e5))


if __name__ == "__main__":
    main()
