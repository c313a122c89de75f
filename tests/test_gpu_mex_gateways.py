"""The MEX gateways run end to end (test mx runtime, libmagasm on the GPU) against the
oracle: the reference's triplet outputs bit for bit, and with the optional trailing
argument MATLAB's sparse() of those triplets (Assembler.m:37-38, 52-53, 205-215) in its
compressed-column storage, bit for bit.
"""
import numpy as np
import pytest
from conftest import bits_equal
from mex_host.gateway import Gateway, GatewayError, build

from magpackage_b200 import material, quadrature, synth
from oracle.oracle import mex_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gateways(tmp_path_factory):
    d = tmp_path_factory.mktemp("mex")
    return {k: Gateway(build(f"assemble_{k}_kernel_mex", d))
            for k in ("jacobian", "curl_curl", "mass", "source", "winding")}


def _case(port, n, seed, drop_dofs=0.0):
    mesh = synth.kuhn_box(n, n + 1, n, seed=seed)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = port.generate_edges(mesh.T)
    m = mex_inputs(mesh.P, mesh.T, t2e, sign, tags)
    E = edges.shape[0]
    rng = np.random.default_rng(seed)
    if drop_dofs:  # dof 0 = no unknown on that edge (the (I > 0) & (J > 0) filter drops it)
        gone = rng.random(E) < drop_dofs
        m.Dofs[gone[t2e]] = 0.0
    sol = rng.normal(0, 0.02, E) * 10.0 ** rng.uniform(-1.5, 0.5, E)
    return m, E, sol, tags


def _valid(I, J, V):
    k = (I > 0) & (J > 0)
    return I[k], J[k], V[k]


def _matlab_sparse(port, I, J, V, N):
    """Compressed-column storage of sparse(I, J, V, N, N): the CSR of the transpose."""
    I, J, V = _valid(I, J, V)
    return port.sparse_csr(J, I, V, N, drop_zeros=True)


def _assert_sparse(out, ref, N):
    jc, ir, pr = ref
    assert out["sparse"] and out["m"] == N and out["n"] == N
    assert np.array_equal(out["jc"], jc), "column pointers differ"
    assert np.array_equal(out["ir"], ir), "row indices differ"
    assert bits_equal(out["pr"], pr), "values differ"


def _jac_args(m, sol, pk, qw, curl, calc_j):
    return (m.P, m.T, m.Dofs, m.Signs, m.Tags, sol, qw, curl, *pk.as_tuple(), float(calc_j))


@pytest.mark.parametrize("n,seed,drop", [(4, 3, 0.0), (7, 5, 0.1)])
def test_jacobian_gateway(gateways, oracle_port, n, seed, drop):
    m, E, sol, _ = _case(oracle_port, n, seed, drop)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
    gw = gateways["jacobian"]
    # 17 inputs: the reference's triplets, unchanged
    out = gw(5, *_jac_args(m, sol, pk, qw, curl, True))
    for o, ref in zip(out, (I, J, V, Ri, Rv)):
        assert not o["sparse"] and bits_equal(o["pr"], ref)
    # 18th input: J_mat = sparse(I,J,V,Ndof,Ndof), R_mat = sparse(R_idx,1,R_val,Ndof,1)
    Jm, Rm = gw(2, *_jac_args(m, sol, pk, qw, curl, True), 1.0)
    _assert_sparse(Jm, _matlab_sparse(oracle_port, I, J, V, E), E)
    k = Ri > 0
    r = oracle_port.sparse_vec(Ri[k], Rv[k], E)
    nzr = np.flatnonzero(r != 0.0)
    assert Rm["sparse"] and Rm["m"] == E and Rm["n"] == 1
    assert np.array_equal(Rm["jc"], [0, nzr.size]) and np.array_equal(Rm["ir"], nzr)
    assert bits_equal(Rm["pr"], r[nzr])
    # the transposition matters: the nonlinear blocks are not bit-symmetric
    rrp, rci, rv = oracle_port.sparse_csr(*_valid(I, J, V), E, drop_zeros=True)
    if np.array_equal(rrp, Jm["jc"]) and np.array_equal(rci, Jm["ir"]):
        assert not bits_equal(rv, Jm["pr"])
    # calcJ = 0: J_mat = [], same residual
    Jm0, Rm0 = gw(2, *_jac_args(m, sol, pk, qw, curl, False), 1.0)
    assert not Jm0["sparse"] and Jm0["m"] == 0 and Jm0["n"] == 0
    assert np.array_equal(Rm0["ir"], Rm["ir"]) and bits_equal(Rm0["pr"], Rm["pr"])
    # a zero flag keeps the triplet outputs
    assert len(gw(5, *_jac_args(m, sol, pk, qw, curl, True), 0.0)) == 5


def test_curl_curl_and_mass_gateways(gateways, oracle_port):
    m, E, _, tags = _case(oracle_port, 6, 11, 0.05)
    qw, val, curl = quadrature.reference_data(2)
    rng = np.random.default_rng(4)
    ne = m.ne
    nu = rng.uniform(0.5, 2.0, ne) * material.NU0
    I, J, V = oracle_port.curl_curl(m, nu, qw, curl)
    args = (m.P, m.T, m.Dofs, m.Signs, nu, qw, curl)
    out = gateways["curl_curl"](3, *args)
    assert all(bits_equal(o["pr"], r) for o, r in zip(out, (I, J, V)))
    (K,) = gateways["curl_curl"](1, *args, float(E))
    _assert_sparse(K, _matlab_sparse(oracle_port, I, J, V, E), E)
    sig = rng.uniform(1e6, 6e7, ne) * (tags == synth.ALUMINIUM)
    for coeffs in (sig, None):
        I, J, V = oracle_port.mass(m, coeffs if coeffs is not None else np.zeros(0), qw, val)
        args = (m.P, m.T, m.Dofs, m.Signs, coeffs, qw, val)
        out = gateways["mass"](3, *args)
        assert all(bits_equal(o["pr"], r) for o, r in zip(out, (I, J, V)))
        (M,) = gateways["mass"](1, *args, float(E))
        _assert_sparse(M, _matlab_sparse(oracle_port, I, J, V, E), E)
        structural = oracle_port.sparse_csr(*_valid(I, J, V), E, drop_zeros=False)[0][-1]
        # sigma = 0 outside the aluminium: those couplings sum to exact zeros, which sparse() drops
        assert (M["pr"].size < structural) == (coeffs is not None)


def test_gateway_errors_and_empty_mesh(gateways, oracle_port):
    m, E, sol, _ = _case(oracle_port, 2, 1)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    bad = m.Dofs.copy()
    bad[0, 0] = E + 1  # beyond numel(SolA)
    with pytest.raises(GatewayError, match="MagPackage:GPU"):
        gateways["jacobian"](2, m.P, m.T, bad, m.Signs, m.Tags, sol, qw, curl, *pk.as_tuple(), 1.0, 1.0)
    with pytest.raises(GatewayError, match="MagPackage:GPU"):
        gateways["curl_curl"](1, m.P, m.T, bad, m.Signs, np.ones(m.ne), qw, curl, float(E))
    # an empty mesh gives an all-zero N x N sparse and a zero residual
    P0, T0 = np.zeros((0, 3)), np.zeros((0, 4))
    Jm, Rm = gateways["jacobian"](2, P0, T0, np.zeros((0, 6)), np.zeros((0, 6)), np.zeros(0), np.zeros(5), qw,
                                  curl, *pk.as_tuple(), 1.0, 1.0)
    assert Jm["sparse"] and Jm["m"] == 5 and np.array_equal(Jm["jc"], np.zeros(6)) and Jm["pr"].size == 0
    assert Rm["sparse"] and Rm["pr"].size == 0
    (K,) = gateways["mass"](1, P0, T0, np.zeros((0, 6)), np.zeros((0, 6)), None, qw, val, 7.0)
    assert K["sparse"] and K["n"] == 7 and K["pr"].size == 0


def test_source_and_winding_gateways(gateways, oracle_port):
    m, E, _, tags = _case(oracle_port, 5, 8, 0.05)
    qw, val, curl = quadrature.reference_data(2)
    rng = np.random.default_rng(9)
    js = rng.normal(size=(m.ne, 3)) * (tags == synth.IRON)[:, None]
    I, V = oracle_port.source(m, js, qw, val)
    out = gateways["source"](2, m.P, m.T, m.Dofs, m.Signs, js, qw, val)
    assert bits_equal(out[0]["pr"], I) and bits_equal(out[1]["pr"], V)
    with pytest.raises(GatewayError, match="MagPackage:Dim"):
        gateways["source"](2, m.P, m.T, m.Dofs, m.Signs, js[:-1], qw, val)
    field = rng.normal(size=(m.ne, 3))
    for f in (None, field):
        I, V = oracle_port.winding(m, float(synth.IRON), f, (0.0, 0.0, 1.0), 5e4, qw, val)
        out = gateways["winding"](2, m.P, m.T, m.Dofs, m.Signs, m.Tags, float(synth.IRON), f,
                                  np.array([0.0, 0.0, 1.0]), 5e4, qw, val)
        assert bits_equal(out[0]["pr"], I) and bits_equal(out[1]["pr"], V)


def test_gateway_mesh_cache_reuse_and_invalidation(gateways, oracle_port):
    """The MEX entry points keep the converted mesh between calls. A repeated call (the
    Newton loop's case) returns the same bits from the cached mesh; a coordinate changed in
    place, a tag changed in place and a dof array changed in place (same addresses, same
    sizes) are each converted afresh, so every result equals the oracle's for the arrays as
    they are at that call."""
    import ctypes as C

    from magpackage_b200 import _lib

    L = _lib.lib()
    _lib.check(L.mag_mex_cache_clear())
    m, E, sol, _ = _case(oracle_port, 5, 21)
    qw, val, curl = quadrature.reference_data(2)
    pk = material.pack_material_data(synth.standard_materials())
    gw = gateways["jacobian"]

    def check_against_oracle():
        I, J, V, Ri, Rv = oracle_port.jacobian(m, sol, qw, curl, pk, True)
        Jm, Rm = gw(2, *_jac_args(m, sol, pk, qw, curl, True), 1.0)
        _assert_sparse(Jm, _matlab_sparse(oracle_port, I, J, V, E), E)
        out = gw(5, *_jac_args(m, sol, pk, qw, curl, True))
        for o, ref in zip(out, (I, J, V, Ri, Rv)):
            assert bits_equal(o["pr"], ref)
        return Jm["pr"].copy()

    first = check_against_oracle()
    assert bits_equal(check_against_oracle(), first)  # from the cache
    # a node moved in place (interior node, small move keeps every element valid)
    node = int(m.T[len(m.T) // 2, 0]) - 1
    m.P[node] += np.array([1e-3, -2e-3, 1.5e-3]) / 5
    moved = check_against_oracle()
    assert not bits_equal(moved, first)
    # a region tag changed in place: iron <-> air somewhere
    k = int(np.flatnonzero(m.Tags == synth.IRON)[0])
    m.Tags[k] = float(synth.AIR)
    check_against_oracle()
    # a dof removed in place (0 = no unknown on that edge)
    m.Dofs[3, 2] = 0.0
    check_against_oracle()
    # the curl-curl gateway shares the cached mesh (no tags needed) and stays exact
    nu = np.random.default_rng(2).uniform(0.5, 2.0, m.ne) * material.NU0
    I, J, Vk = oracle_port.curl_curl(m, nu, qw, curl)
    out = gateways["curl_curl"](3, m.P, m.T, m.Dofs, m.Signs, nu, qw, curl)
    assert bits_equal(out[2]["pr"], Vk)
    _lib.check(L.mag_mex_cache_clear())
