"""Host-side logic that needs no GPU: synthetic meshes, material maps and packing."""
import numpy as np
import pytest

from magpackage_b200 import material, synth
from magpackage_b200.assembler import Assembler, DofHandler, Mesh


@pytest.mark.parametrize("n", [1, 3, 6])
def test_kuhn_box_counts_and_orientation(n):
    mesh = synth.kuhn_box(n, seed=2)
    assert mesh.num_nodes == (n + 1) ** 3 and mesh.num_elements == 6 * n ** 3
    v = mesh.P[mesh.T]
    det = np.linalg.det(np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=2))
    # the six Kuhn tetrahedra tile each hexahedron (volumes add up to the box)
    assert abs(np.abs(det).sum() / 6.0 - 1.0) < 1e-12
    assert np.all(np.abs(det) > 0)


def test_kuhn_box_boundary_stays_flat():
    mesh = synth.kuhn_box(4, seed=1, jitter=0.1)
    for c in range(3):
        on = np.isclose(mesh.P[:, c], 0.0) | np.isclose(mesh.P[:, c], 1.0)
        assert on.sum() == 2 * 25  # two faces of 5x5 nodes per axis


def test_cube_layout_regions():
    mesh = synth.kuhn_box(20, seed=0)
    tags = synth.cube_layout(mesh)
    frac = np.bincount(tags, minlength=4)[1:] / tags.size
    assert abs(frac[1] - 0.4 ** 3) < 0.02 and abs(frac[2] - 0.1) < 0.03


def test_expand_material_map_forms():
    tags = np.array([1, 2, 2, 3], dtype=np.int32)
    mesh = Mesh(np.zeros((4, 3)), np.array([[0, 1, 2, 3]] * 4), tags)
    a = Assembler(mesh, DofHandler(mesh))
    assert np.array_equal(a.expand_material_map({2: 5.0, 3: 7.0}), [0, 5, 5, 7])
    assert np.array_equal(a.expand_material_map(2.5), [2.5] * 4)
    assert np.array_equal(a.expand_material_map(np.array([1.0, 2, 3, 4])), [1, 2, 3, 4])
    assert np.array_equal(a.expand_material_map(np.array([10.0, 20, 30])), [10, 20, 20, 30])
    with pytest.raises(ValueError):
        a.expand_material_map(np.ones((2, 2)))


def test_pack_material_data_layout():
    b, h = material.froehlich_bh()
    lib = {1: material.create_linear(1.0), 3: material.create_nonlinear(b, h),
           4: material.create_nonlinear(b[:50], h[:50])}
    pk = material.pack_material_data(lib)
    assert pk.lin.size == 5  # maxTag + 1, index = tag - 1
    assert pk.is_non.tolist() == [0, 0, 1, 1, 0]
    assert pk.lin[0] == 1.0 / material.MU0 and pk.lin[2] == material.NU0
    assert pk.start[2] == 0 and pk.count[2] == lib[3].breaks.size - 1
    assert pk.start[3] == lib[3].breaks.size and pk.coe_start[3] == lib[3].coefs.size
    assert pk.breaks.size == lib[3].breaks.size + lib[4].breaks.size
    assert np.array_equal(pk.coefs[:4], lib[3].coefs[0])


def test_frequency_sweep_sizes_match_the_instances():
    """The sizes the rank split is computed from are the instances' element counts."""
    from magpackage_b200 import synth

    sizes = synth.frequency_sweep_sizes(count=5, n_min=2, n_max=10)
    got = [m.num_elements for m, *_ in synth.frequency_sweep_instances(count=5, n_min=2, n_max=10)]
    assert sizes == got
    assert len(synth.frequency_sweep_sizes()) == 64 and sum(synth.frequency_sweep_sizes()) == 12_848_640


@pytest.mark.parametrize("harmonics,n", [((0, 1, 3, 5), None), ((1, 3, 5), None), ((1, 7), 15), ((0, 2), 5)])
def test_aft_round_trip_of_real_signals(harmonics, n):
    """AFT (src/utils/AFT.m:19-86 restated): a real time signal x = Re(D X) made of the
    listed harmonics goes back to X through P (a DC coefficient keeps its real part), and
    the sample count follows the reference's rule."""
    from magpackage_b200.hbfem import AFT

    aft = AFT(harmonics, n)
    h = np.asarray(harmonics)
    want_n = max(32, 1 << int(np.ceil(np.log2(2 * h.max() + 1)))) if n is None else max(n, 2 * h.max() + 1)
    assert aft.num_time_steps == want_n
    assert aft.D.shape == (want_n, len(h)) and aft.P.shape == (len(h), want_n)
    rng = np.random.default_rng(2)
    X = rng.normal(size=len(h)) + 1j * rng.normal(size=len(h))
    x = np.real(aft.D @ X)
    back = aft.P @ x
    want = np.where(h == 0, np.real(X), X)
    np.testing.assert_allclose(back, want, rtol=0, atol=1e-12)
