"""mag_mex_jacobian_noalloc against mag_mex_jacobian, through the C ABI.

The allocation-free entry point serves callers that cannot allocate device
memory themselves (for example a MEX function working on mxGPUArray buffers
that MATLAB's allocator owns). It must give the same triplets and residual
pairs as the regular MEX-compatible entry point, call after call, even though
every call reuses the same static device array. This file is collected last
so that a run stopping at the first failure has already run everything else.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from magpackage_b200 import _lib, material, quadrature, synth
from magpackage_b200.plan import generate_edges

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 32768


def _p(t):
    return C.c_void_p(t.data_ptr())


def _inputs(n=12, seed=4):
    mesh = synth.kuhn_box(n, seed=seed)
    tags = synth.cube_layout(mesh)
    edges, t2e, sign = generate_edges(mesh.T)
    E = int(edges.shape[0])
    host = {
        "P": np.ascontiguousarray(mesh.P, dtype=np.float64),
        "T": np.ascontiguousarray(mesh.T + 1, dtype=np.float64),
        "Dofs": np.ascontiguousarray(t2e.cpu().numpy() + 1, dtype=np.float64),
        "Signs": np.ascontiguousarray(sign.cpu().numpy(), dtype=np.float64),
        "Tags": np.ascontiguousarray(tags, dtype=np.float64),
    }
    pk = [np.ascontiguousarray(a, dtype=np.float64)
          for a in material.pack_material_data(synth.standard_materials()).as_tuple()]
    qw, _, curl = quadrature.reference_data(2)
    return mesh.num_nodes, mesh.num_elements, E, host, pk, qw, curl


def _regular(nn, ne, E, h, pk, qw, curl, sol):
    L = _lib.lib()
    p = _lib.dptr
    I, J, V = (np.zeros(36 * ne) for _ in range(3))
    Ri, Rv = np.zeros(6 * ne), np.zeros(6 * ne)
    _lib.check(L.mag_mex_jacobian(p(h["P"]), nn, p(h["T"]), ne, p(h["Dofs"]), p(h["Signs"]), p(h["Tags"]),
                                  p(sol), E, p(qw), qw.size, p(curl), p(pk[0]), p(pk[1]), p(pk[2]),
                                  pk[0].size, p(pk[3]), pk[3].size, p(pk[4]), pk[4].size, p(pk[5]),
                                  p(pk[6]), p(pk[7]), 1, p(I), p(J), p(V), p(Ri), p(Rv)))
    return I, J, V, Ri, Rv


def _noalloc(nn, ne, E, d, pk, qw, curl, d_sol, out, stream_ptr):
    L = _lib.lib()
    p = _lib.dptr
    return L.mag_mex_jacobian_noalloc(
        _p(d["P"]), nn, _p(d["T"]), ne, _p(d["Dofs"]), _p(d["Signs"]), _p(d["Tags"]), _p(d_sol), E,
        p(qw), qw.size, p(curl), p(pk[0]), p(pk[1]), p(pk[2]), pk[0].size, p(pk[3]), pk[3].size,
        p(pk[4]), pk[4].size, p(pk[5]), p(pk[6]), p(pk[7]), 1, _p(out["I"]), _p(out["J"]), _p(out["V"]),
        _p(out["Ri"]), _p(out["Rv"]), stream_ptr)


def test_noalloc_matches_regular_entry_on_consecutive_calls():
    nn, ne, E, h, pk, qw, curl = _inputs()
    assert ne <= MAX_ELEMENTS
    d = {k: torch.as_tensor(v, device="cuda") for k, v in h.items()}
    out = {k: torch.empty(36 * ne if k in "IJV" else 6 * ne, dtype=torch.float64, device="cuda")
           for k in ("I", "J", "V", "Ri", "Rv")}
    rng = np.random.default_rng(7)
    stream = _lib.stream_ptr()
    for call in range(2):  # two calls in a row share the static scratch
        sol = rng.normal(0.0, 0.05, E) * 10.0 ** rng.uniform(-1.5, 0.5, E)
        ref = _regular(nn, ne, E, h, pk, qw, curl, sol)
        d_sol = torch.as_tensor(sol, device="cuda")
        for t in out.values():
            t.fill_(np.nan)
        _lib.check(_noalloc(nn, ne, E, d, pk, qw, curl, d_sol, out, stream))
        got = [out[k].cpu().numpy() for k in ("I", "J", "V", "Ri", "Rv")]
        for name, g, r in zip(("I", "J", "V", "R_idx", "R_val"), got, ref):
            # same tolerance as the other parity tests: exact equality
            assert np.array_equal(g, r), f"call {call}: {name} differs"


def test_noalloc_rejects_oversized_input():
    nn, ne, E, h, pk, qw, curl = _inputs(n=2)
    d = {k: torch.as_tensor(v, device="cuda") for k, v in h.items()}
    out = {k: torch.empty(36, dtype=torch.float64, device="cuda") for k in ("I", "J", "V", "Ri", "Rv")}
    d_sol = torch.zeros(E, dtype=torch.float64, device="cuda")
    rc = _noalloc(nn, MAX_ELEMENTS + 1, E, d, pk, qw, curl, d_sol, out, _lib.stream_ptr())
    assert rc == -7
    assert b"at most 32768 elements" in _lib.load().mag_last_error()
