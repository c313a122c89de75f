"""Device-resident assembly plan: one ``mag_mesh`` handle of libmagasm.

An ``AssemblyPlan`` owns the mesh copy, the CSR pattern and the incidence plan
that the fixed-order reduction walks. Assembly calls write into caller-provided
(or freshly allocated) torch CUDA tensors on the current stream and do not
synchronise, so they can be captured in CUDA graphs and timed with events.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .material import PackedMaterials
from .quadrature import reference_data


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class AssemblyPlan:
    def __init__(self, P, T, cell_dofs, num_dofs: int, tags, signs=None, stream=None):
        self._lib = _lib.lib()
        dev = torch.device("cuda")
        self.P = torch.as_tensor(np.ascontiguousarray(P) if isinstance(P, np.ndarray) else P,
                                 dtype=torch.float64, device=dev).contiguous()
        self.T = torch.as_tensor(T, dtype=torch.int32, device=dev).contiguous()
        self.dofs = torch.as_tensor(cell_dofs, dtype=torch.int32, device=dev).contiguous()
        self.tags = torch.as_tensor(tags, dtype=torch.int32, device=dev).contiguous()
        sg = None if signs is None else torch.as_tensor(signs, dtype=torch.int8, device=dev).contiguous()
        self.num_dofs = int(num_dofs)
        self.num_elements = int(self.T.shape[0])
        h = C.c_void_p()
        _lib.check(self._lib.mag_mesh_create(_ptr(self.P), self.P.shape[0], _ptr(self.T),
                                             self.num_elements, _ptr(self.dofs), _ptr(sg),
                                             _ptr(self.tags), self.num_dofs, C.byref(h),
                                             _lib.stream_ptr(stream)))
        self._h = h
        info = _lib.MeshInfo()
        _lib.check(self._lib.mag_mesh_get_info(self._h, C.byref(info)))
        self.info = info
        self.nnz = int(info.nnz)
        self._row_ptr = self._col_idx = None
        self._materials_key = None
        qw, val, curl = reference_data(2)
        self.set_quadrature(qw, curl, val)

    # ---- setup -----------------------------------------------------------
    def set_quadrature(self, qw, curl_ref, val_ref):
        qw = np.ascontiguousarray(qw, dtype=np.float64)
        curl_ref = np.ascontiguousarray(curl_ref, dtype=np.float64)
        val_ref = np.ascontiguousarray(val_ref, dtype=np.float64)
        _lib.check(self._lib.mag_mesh_set_quadrature(self._h, _lib.dptr(qw), qw.size,
                                                     _lib.dptr(curl_ref), _lib.dptr(val_ref)))

    def set_materials(self, packed: PackedMaterials, key=None):
        if key is not None and key == self._materials_key:
            return
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in packed.as_tuple()]
        nb, nc = a[3].size, a[4].size
        if nb == 0:
            a[3] = np.zeros(1)
        if nc == 0:
            a[4] = np.zeros(1)
        _lib.check(self._lib.mag_mesh_set_materials(
            self._h, _lib.dptr(a[0]), _lib.dptr(a[1]), _lib.dptr(a[2]), a[0].size, _lib.dptr(a[3]),
            nb, _lib.dptr(a[4]), nc, _lib.dptr(a[5]), _lib.dptr(a[6]), _lib.dptr(a[7])))
        self._keep = a
        self._materials_key = key

    def set_schedule(self, schedule: int):
        """Jacobian schedule: one of _lib.SCHEDULE_* (all give the same bits)."""
        _lib.check(self._lib.mag_mesh_set_option(self._h, 1, int(schedule)))
        info = _lib.MeshInfo()
        _lib.check(self._lib.mag_mesh_get_info(self._h, C.byref(info)))
        self.info = info

    def set_tile_variant(self, variant: int):
        """Launch shape of the tile schedule's Jacobian kernel (MAG_OPTION_TILE_VARIANT)."""
        _lib.check(self._lib.mag_mesh_set_option(self._h, 2, int(variant)))

    def set_tile_prefetch(self, waves: int):
        """Staging depth of the tile schedule in waves of resident CTAs (MAG_OPTION_TILE_PREFETCH)."""
        _lib.check(self._lib.mag_mesh_set_option(self._h, 3, int(waves)))

    def tune(self, sol, vals, res, reps: int = 3, stream=None):
        """Time every launch shape x staging depth of the tile Jacobian on this state and keep the
        fastest (mag_mesh_tune); returns (variant, depth, times_ms[4][3]). vals and res hold the
        Jacobian and residual at sol afterwards."""
        times = np.zeros(12)
        v, d = C.c_int(), C.c_int()
        _lib.check(self._lib.mag_mesh_tune(self._h, _ptr(sol), _ptr(vals), _ptr(res), int(reps),
                                           times.ctypes.data_as(C.c_void_p), C.byref(v), C.byref(d),
                                           _lib.stream_ptr(stream)))
        return v.value, d.value, times.reshape(4, 3)

    def check(self, stream=None):
        """Synchronise and raise if a bounded device-side wait gave up."""
        _lib.check(self._lib.mag_mesh_check(self._h, _lib.stream_ptr(stream)))

    # ---- pattern -----------------------------------------------------------
    def _pattern(self):
        if self._row_ptr is None:
            rp = torch.empty(self.num_dofs + 1, dtype=torch.int64, device="cuda")
            ci = torch.empty(max(self.nnz, 1), dtype=torch.int32, device="cuda")
            _lib.check(self._lib.mag_mesh_pattern(self._h, _ptr(rp), _ptr(ci), _lib.stream_ptr()))
            self._row_ptr, self._col_idx = rp, ci[: self.nnz]
        return self._row_ptr, self._col_idx

    @property
    def row_ptr(self):
        return self._pattern()[0]

    @property
    def col_idx(self):
        return self._pattern()[1]

    def new_values(self):
        return torch.empty(self.nnz, dtype=torch.float64, device="cuda")

    def new_vector(self):
        return torch.empty(self.num_dofs, dtype=torch.float64, device="cuda")

    # ---- assembly (structural CSR values, current stream, asynchronous) ----
    def jacobian(self, sol, vals=None, res=None, calc_j: bool = True, stream=None):
        if calc_j and vals is None:
            vals = self.new_values()
        if res is None:
            res = self.new_vector()
        _lib.check(self._lib.mag_assemble_jacobian(self._h, _ptr(sol), _ptr(vals) if calc_j else None,
                                                   _ptr(res), int(calc_j), _lib.stream_ptr(stream)))
        return (vals if calc_j else None), res

    def stiffness(self, nu_e, vals=None, stream=None):
        vals = self.new_values() if vals is None else vals
        _lib.check(self._lib.mag_assemble_stiffness(self._h, _ptr(nu_e), _ptr(vals),
                                                    _lib.stream_ptr(stream)))
        return vals

    def mass(self, sigma_e=None, vals=None, stream=None):
        vals = self.new_values() if vals is None else vals
        _lib.check(self._lib.mag_assemble_mass(self._h, _ptr(sigma_e), _ptr(vals),
                                               _lib.stream_ptr(stream)))
        return vals

    def source(self, js, out=None, stream=None):
        out = self.new_vector() if out is None else out
        _lib.check(self._lib.mag_assemble_source(self._h, _ptr(js), _ptr(out), _lib.stream_ptr(stream)))
        return out

    def winding(self, coil_id: int, direction=None, scale: float = 1.0, dir_field=None, out=None, stream=None):
        """Coil current vector of the elements tagged coil_id (mag_assemble_winding):
        dir_field [Ne, 3] on the device, else the uniform host direction."""
        out = self.new_vector() if out is None else out
        d = None if direction is None else np.ascontiguousarray(np.asarray(direction, dtype=np.float64).ravel()[:3])
        if dir_field is None and (d is None or d.size != 3):
            raise ValueError("winding needs a 3-vector direction or an [Ne, 3] direction field")
        _lib.check(self._lib.mag_assemble_winding(self._h, int(coil_id), _ptr(dir_field), _lib.dptr(d),
                                                  float(scale), _ptr(out), _lib.stream_ptr(stream)))
        return out

    def element_b(self, sol, want_vec: bool = True, stream=None):
        b = torch.empty((self.num_elements, 3), dtype=torch.float64, device="cuda") if want_vec else None
        bsq = torch.empty(self.num_elements, dtype=torch.float64, device="cuda")
        _lib.check(self._lib.mag_element_b(self._h, _ptr(sol), _ptr(b), _ptr(bsq),
                                           _lib.stream_ptr(stream)))
        return b, bsq

    def drop_zeros(self, vals):
        """MATLAB sparse() storage of (row_ptr, col_idx, vals): exact zeros removed."""
        rp, ci = self._pattern()
        rp2 = torch.empty_like(rp)
        ci2 = torch.empty_like(ci) if ci.numel() else torch.empty(1, dtype=torch.int32, device="cuda")
        v2 = torch.empty_like(vals)
        nnz = C.c_int64()
        _lib.check(self._lib.mag_csr_drop_zeros(_ptr(rp), _ptr(ci), _ptr(vals), self.num_dofs, _ptr(rp2),
                                                _ptr(ci2), _ptr(v2), C.byref(nnz), _lib.stream_ptr()))
        n = nnz.value
        return rp2, ci2[:n], v2[:n]

    # ---- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.mag_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_edges(T):
    """Mesh.generateEdges (src/Mesh.m:114-138) on the GPU.

    T: (Ne, 4) 0-based node ids (torch CUDA or numpy). Returns (edges (E,2),
    t2e (Ne,6), sign (Ne,6) int8) as CUDA tensors, edges 0-based and ordered
    lexicographically by (min, max) node like MATLAB's unique(sort(rows)).
    """
    L = _lib.lib()
    T = torch.as_tensor(T, dtype=torch.int32, device="cuda").contiguous()
    ne = T.shape[0]
    nn = int(T.max().item()) + 1
    edges = torch.empty((6 * ne, 2), dtype=torch.int32, device="cuda")
    t2e = torch.empty((ne, 6), dtype=torch.int32, device="cuda")
    sign = torch.empty((ne, 6), dtype=torch.int8, device="cuda")
    E = C.c_int64()
    _lib.check(L.mag_generate_edges(_ptr(T), ne, nn, _ptr(edges), _ptr(t2e), _ptr(sign), C.byref(E),
                                    _lib.stream_ptr()))
    return edges[: E.value], t2e, sign


class ComplexBatch:
    """K_i(nu_i) + j*omega_i*M_i(sigma_i) for many meshes in one graph-captured launch.

    plans: AssemblyPlan per mesh; nus / sigmas: per-element CUDA float64 tensors
    (a sigma may be None: sigma = 1); omegas: rad/s. ``values[i]`` holds mesh i's
    complex128 CSR values on its structural pattern after ``assemble()``.
    """

    def __init__(self, plans, nus, sigmas, omegas, stream=None):
        self._lib = _lib.lib()
        n = len(plans)
        self.plans = list(plans)
        self.nus = [t.contiguous() for t in nus]
        self.sigmas = [None if t is None else t.contiguous() for t in sigmas]
        self.values = [torch.empty(p.nnz, dtype=torch.complex128, device="cuda") for p in plans]
        H = (C.c_void_p * n)(*[p._h.value for p in plans])
        NU = (C.c_void_p * n)(*[t.data_ptr() for t in self.nus])
        SG = (C.c_void_p * n)(*[0 if t is None else t.data_ptr() for t in self.sigmas])
        VA = (C.c_void_p * n)(*[t.data_ptr() for t in self.values])
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        h = C.c_void_p()
        _lib.check(self._lib.mag_batch_create(H, n, NU, SG, _lib.dptr(om), VA, C.byref(h),
                                              _lib.stream_ptr(stream)))
        self._h = h
        self.omegas = om

    def assemble(self, stream=None):
        _lib.check(self._lib.mag_batch_assemble(self._h, _lib.stream_ptr(stream)))
        return self.values

    def select(self, variant: int):
        """Replay `variant` from now on instead of the tuned one."""
        _lib.check(self._lib.mag_batch_select(self._h, int(variant)))

    def tuning(self):
        nv = self._lib.mag_batch_variants()
        chosen = C.c_int()
        times = np.zeros(nv)
        name = C.create_string_buffer(128)
        _lib.check(self._lib.mag_batch_tuning(self._h, C.byref(chosen), _lib.dptr(times), name, 128))
        return chosen.value, times, name.value.decode()

    def close(self):
        if getattr(self, "_h", None):
            self._lib.mag_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
