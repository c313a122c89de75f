"""Host-side mirror of the reference's assembly interface, backed by the GPU.

Mirrors the MATLAB classes a caller of the hot path uses, with the same method
names (snake_case), argument meaning and error behaviour:

* ``Mesh``       -- src/Mesh.m (P, T, RegionTags; ``generate_edges`` =
                    Mesh.generateEdges, :114-138, run on the GPU).
* ``DofHandler`` -- src/DofHandler.m, Nedelec branch of ``distributeDofs``
                    (:72-105): dofs on the edges touched by the active regions,
                    numbered in edge order; ``pack_for_kernel`` (:124-130).
* ``Assembler``  -- src/Assembler.m: ``assemble_stiffness`` (:26-39),
                    ``assemble_mass`` (:41-57), ``assemble_mass_weighted``
                    (:59-76), ``assemble_source`` (:78-97), ``assemble_winding``
                    (:134-180), ``assemble_jacobian`` (:182-231),
                    ``expand_material_map`` (:240-268) and ``pack_material_data``
                    (:270-304).
* ``Winding``    -- src/Winding.m (coil region, turns, cross-section, unit
                    direction or a per-element direction field).

Indices are 0-based here (the reference's are 1-based). Matrices come back as
``CSR`` objects holding CUDA tensors. With ``matlab_storage=True`` (default)
exact zeros are dropped as MATLAB's sparse() does; ``False`` keeps the fixed
structural pattern, which is what a Newton loop wants.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .material import PackedMaterials, pack_material_data
from .plan import AssemblyPlan, generate_edges


@dataclass
class CSR:
    row_ptr: torch.Tensor  # int64 [n+1]
    col_idx: torch.Tensor  # int32 [nnz]
    values: torch.Tensor   # float64 / complex128 [nnz]
    shape: tuple

    @property
    def nnz(self):
        return int(self.col_idx.numel())

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.values.cpu().numpy(), self.col_idx.cpu().numpy(),
                              self.row_ptr.cpu().numpy()), shape=self.shape)

    def matvec(self, x: torch.Tensor) -> torch.Tensor:
        A = torch.sparse_csr_tensor(self.row_ptr, self.col_idx.to(torch.int64), self.values,
                                    size=self.shape)
        return A @ x


@dataclass
class Winding:
    """src/Winding.m: a coil on region RegionID. ``create`` normalises the direction
    as the constructor does (Winding.m:18-31); DirectionField [Ne, 3], when set, takes
    precedence over Direction in the assembly."""

    Name: str
    RegionID: int
    Turns: float
    Resistance: float
    CrossSectionArea: float
    Direction: np.ndarray
    DirectionField: np.ndarray | None = None

    @classmethod
    def create(cls, name, region_id, turns, resistance, area, direction):
        d = np.asarray(direction, dtype=np.float64).ravel()[:3]
        n = float(np.linalg.norm(d))
        return cls(name, int(region_id), float(turns), float(resistance), float(area),
                   d / n if n > 0 else np.zeros(3))

    def set_direction_field(self, field):
        self.DirectionField = None if field is None else np.asarray(field, dtype=np.float64)


class Mesh:
    def __init__(self, P, T, region_tags):
        self.P = np.ascontiguousarray(P, dtype=np.float64)          # (Nn, 3)
        self.T = np.ascontiguousarray(T, dtype=np.int32)            # (Ne, 4), 0-based
        self.RegionTags = np.ascontiguousarray(region_tags, dtype=np.int32)
        if self.T.ndim != 2 or self.T.shape[1] != 4 or self.P.ndim != 2 or self.P.shape[1] != 3:
            raise ValueError("Mesh expects P (Nn,3) and T (Ne,4)")
        if self.RegionTags.shape[0] != self.T.shape[0]:
            raise ValueError("RegionTags must have one entry per element")
        self.Edges = self.T2E = self.T2E_Sign = None

    @property
    def num_nodes(self):
        return self.P.shape[0]

    @property
    def num_elements(self):
        return self.T.shape[0]

    def generate_edges(self):
        """Mesh.generateEdges: lexicographic edge ids, T2E, orientation signs."""
        if self.Edges is not None:
            return
        if self.T.max(initial=-1) >= self.num_nodes or self.T.min(initial=0) < 0:
            raise ValueError("T references a node outside P")
        self.Edges, self.T2E, self.T2E_Sign = generate_edges(self.T)


class DofHandler:
    def __init__(self, mesh: Mesh):
        self.Mesh = mesh
        self.NumGlobalDofs = 0
        self.cell_dofs = None
        self.entity_map = None

    def distribute_dofs(self, target_region_tags=None):
        """Nedelec dofs on the edges of the active elements (DofHandler.m:72-105)."""
        m = self.Mesh
        m.generate_edges()
        t2e = m.T2E
        if target_region_tags is None:
            active_edges = None
            n_edges = int(m.Edges.shape[0])
            emap = torch.arange(n_edges, dtype=torch.int32, device=t2e.device)
            nd = n_edges
        else:
            act = torch.as_tensor(np.isin(m.RegionTags, np.asarray(target_region_tags)),
                                  device=t2e.device)
            active_edges = torch.unique(t2e[act].ravel())
            emap = torch.full((int(m.Edges.shape[0]),), -1, dtype=torch.int32, device=t2e.device)
            emap[active_edges.long()] = torch.arange(active_edges.numel(), dtype=torch.int32,
                                                     device=t2e.device)
            nd = int(active_edges.numel())
        self.entity_map = emap
        self.cell_dofs = emap[t2e.long()].contiguous()
        self.NumGlobalDofs = nd
        return self.cell_dofs

    def pack_for_kernel(self):
        return self.cell_dofs, self.Mesh.T2E_Sign


class Assembler:
    def __init__(self, mesh: Mesh, dof_handler: DofHandler, matlab_storage: bool = True):
        self.Mesh = mesh
        self.DofHandler = dof_handler
        self.matlab_storage = matlab_storage
        self._plan = None

    # ---- helpers -------------------------------------------------------------
    @property
    def plan(self) -> AssemblyPlan:
        if self._plan is None:
            if self.DofHandler.cell_dofs is None:
                self.DofHandler.distribute_dofs()
            dofs, signs = self.DofHandler.pack_for_kernel()
            self._plan = AssemblyPlan(self.Mesh.P, self.Mesh.T, dofs, self.DofHandler.NumGlobalDofs,
                                      self.Mesh.RegionTags, signs)
        return self._plan

    def expand_material_map(self, map_or_array, tags=None) -> np.ndarray:
        """Per-element coefficients from a {tag: value} map or a numeric array."""
        tags = self.Mesh.RegionTags if tags is None else tags
        n = tags.shape[0]
        if isinstance(map_or_array, dict):
            vec = np.zeros(n)
            for k, v in map_or_array.items():
                if np.isscalar(v):
                    vec[tags == int(k)] = v
            return vec
        a = np.asarray(map_or_array, dtype=np.float64)
        if a.ndim == 0 or a.size == 1:
            return np.full(n, float(a.ravel()[0]))
        if a.ndim == 1 or 1 in a.shape:
            a = a.ravel()
            return a.copy() if a.size == n else a[tags - 1]
        raise ValueError("Assembler:InvalidInput: Invalid material array format.")

    @staticmethod
    def pack_material_data(matlib) -> PackedMaterials:
        return pack_material_data(matlib)

    def _out(self, vals) -> CSR:
        p = self.plan
        n = self.DofHandler.NumGlobalDofs
        if self.matlab_storage:
            rp, ci, v = p.drop_zeros(vals)
            return CSR(rp, ci, v, (n, n))
        return CSR(p.row_ptr, p.col_idx, vals, (n, n))

    def _dev(self, a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")

    # ---- Assembler.m surface --------------------------------------------------
    def assemble_stiffness(self, material_map) -> CSR:
        nu = self._dev(self.expand_material_map(material_map))
        return self._out(self.plan.stiffness(nu))

    def assemble_mass(self) -> CSR:
        return self._out(self.plan.mass(None))

    def assemble_mass_weighted(self, coeff_map) -> CSR:
        sigma = self._dev(self.expand_material_map(coeff_map))
        return self._out(self.plan.mass(sigma))

    def assemble_source(self, source_map) -> torch.Tensor:
        n = self.Mesh.num_elements
        js = np.zeros((n, 3))
        if isinstance(source_map, dict):
            for k, v in source_map.items():
                js[self.Mesh.RegionTags == int(k)] = np.asarray(v, dtype=np.float64).ravel()[:3]
        else:
            a = np.asarray(source_map, dtype=np.float64)
            if a.size == 3:
                js[:] = a.ravel()
            elif a.shape == (n, 3):
                js = a
            else:
                raise ValueError("Source must be [3x1] or [Ne x 3].")
        return self.plan.source(self._dev(js))

    def assemble_winding(self, winding) -> torch.Tensor:
        """Coil vector C [num_dofs] of one Winding (Turns / CrossSectionArea times its
        direction, Assembler.m:157-166), or [num_dofs, k] for a list (:175-178)."""
        if isinstance(winding, (list, tuple)):
            return torch.stack([self.assemble_winding(w) for w in winding], dim=1)
        scale = winding.Turns / winding.CrossSectionArea
        field = None
        if winding.DirectionField is not None and np.size(winding.DirectionField):
            f = np.asarray(winding.DirectionField, dtype=np.float64)
            if f.shape != (self.Mesh.num_elements, 3):
                raise ValueError("DirectionField must be [Ne x 3]")
            field = self._dev(f)
        return self.plan.winding(winding.RegionID, winding.Direction, scale, dir_field=field)

    def assemble_jacobian(self, solution_a, matlib, calc_j: bool = True):
        p = self.plan
        p.set_materials(pack_material_data(matlib), key=id(matlib))
        sol = solution_a if isinstance(solution_a, torch.Tensor) else self._dev(solution_a)
        vals, res = p.jacobian(sol.contiguous(), calc_j=calc_j)
        return (self._out(vals) if calc_j else None), res
