"""Transient nonlinear A-formulation on the GPU, with an optional learned warm start.

Restates the Newton loop of TransientSolver.solve (src/solver/TransientSolver.m:
138-266) for the pure-A case on top of the assembly kernels:

  R(x) = R_nu(x) + M_sigma (x - x_prev)/dt - F(t) + reg M_reg x        (:294-300, :177-180)
  J(x) = J_nu(x) + M_sigma/dt + reg M_reg                               (:154, :170, :177-179)

with reg = RegScaleRel * mean(|diag J|) taken from the first Newton matrix of a run
started at A = 0 (:168-175), Dirichlet elimination on the box boundary (:189,
BoundaryCondition.m:81-112), and the reference's backtracking line search with
residual-only assemblies (:218-246). The linear solve stands in for MUMPS
(LinearSolver.m:22-46) with the library's preconditioned CG, timed apart.

Convergence is RHS-relative, ||R_bc|| <= tol * max(||F_bc||, 1), instead of the
reference's test relative to the first-iteration residual (:198-207): that test
gets stricter the better the initial guess, so it cannot compare warm starts.

Warm starts of step t (x_0 = x_{t-1} in all modes, TransientSolver.m:159):
  plain    -- every Newton iteration uses the tangent at the current iterate;
  learned  -- the MLP predicts each nonlinear element's nu_e at the end of step t
              from |B|_{t-1}, |B|_{t-2}, |J(t)| and the material id (as the ratio
              nu_t / nu(|B|_{t-1}), multiplied onto the exactly evaluated nu at
              x_{t-1}, so its error scales with the step's change); inverting the
              element's B-H table turns it into a predicted |B_hat_e|, and the FIRST
              Jacobian of the step is evaluated at the midpoint state
              (|B_{t-1}| + |B_hat|)/2 (per element, along B_{t-1}) -- a secant-like
              tangent over the step, the scale kept in a trust region [1/1.25, 1.25] --
              while its residual stays the true R(x_{t-1}).
              Later iterations are plain Newton to the same tolerance, so a bad
              prediction costs iterations, never accuracy;
  ideal    -- the same seeding with the converged nu of the step (a bound on what
              any predictor can gain; needs the plain run's solutions).
A seed that solves K(nu_hat) x = F for a new starting point (a Picard step) was
measured and rejected: in saturated iron a 1% error in nu moves that start
further from the solution than x_{t-1} is.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, synth
from .material import NU0, pack_material_data
from .plan import AssemblyPlan, generate_edges


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


@dataclass
class TransientConfig:
    nx: int = 40
    ny: int = 40
    nz: int = 20
    size: tuple = (0.4, 0.4, 0.2)
    jitter: float = 0.1
    seed: int = 4
    j_peak: float = 2e6        # A/m^2
    freq: float = 50.0         # Hz
    dt: float = 1e-4
    steps: int = 200
    sigma_iron: float = 0.0    # S/m; the workload names no conductivity (laminated core)
    tol: float = 1e-8
    max_newton: int = 50
    max_line_search: int = 10
    reg_rel: float = 1e-5      # TransientSolver.RegScaleRel
    cg_rtol: float = 1e-10
    cg_max: int = 20000
    seed_max_scale: float = 1.25  # trust region of the seeded tangent's flux-density scale


@dataclass
class StepStats:
    step: int
    mode: str
    newton: int = 0            # Newton iterations (Jacobian assemblies)
    residual_only: int = 0     # line-search residual assemblies
    solves: int = 0
    cg_iters: int = 0
    gpu_ms: float = 0.0        # whole step, device clock
    solve_ms: float = 0.0
    assembly_ms: float = 0.0
    mlp_ms: float = 0.0
    res: float = 0.0
    tol_abs: float = 0.0
    converged: bool = False
    nu_rel_err: float = float("nan")
    nu_rel_err_max: float = float("nan")
    res_history: list = field(default_factory=list)  # ||R_bc|| at each Newton iteration

    @property
    def assemblies(self):
        return self.newton + self.residual_only


class _Timer:
    """Device-time accumulator of event pairs on the current stream."""

    def __init__(self):
        self.pairs = []

    def start(self):
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    def stop(self, e0, key):
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record()
        self.pairs.append((key, e0, e1))

    def collect(self):
        torch.cuda.synchronize()
        out = {}
        for k, a, b in self.pairs:
            out[k] = out.get(k, 0.0) + a.elapsed_time(b)
        self.pairs = []
        return out


class TransientProblem:
    """E-core transient workload: mesh, matrices, boundary, coil current, Newton."""

    def __init__(self, cfg: TransientConfig | None = None):
        self.cfg = cfg = cfg or TransientConfig()
        mesh = synth.kuhn_box(cfg.nx, cfg.ny, cfg.nz, size=cfg.size, jitter=cfg.jitter, seed=cfg.seed)
        self.mesh = mesh
        self.tags = synth.ecore_coil_layout(mesh)
        edges_d, t2e, _sign = generate_edges(mesh.T)
        edges = edges_d.cpu().numpy()
        E = int(edges.shape[0])
        self.edges, self.num_dofs = edges, E
        self.plan = AssemblyPlan(mesh.P, mesh.T, t2e, E, self.tags)
        self.plan.set_materials(pack_material_data(synth.standard_materials()))
        dev = torch.device("cuda")
        self.lib = _lib.lib()
        self.rp, self.ci = self.plan.row_ptr, self.plan.col_idx
        # boundary: edges with both end nodes on one face of the box
        P = mesh.P
        lo, hi = P.min(0), P.max(0)
        on = np.concatenate([np.isclose(P, lo[None, :]), np.isclose(P, hi[None, :])], axis=1)
        fixed = np.any(on[edges[:, 0]] & on[edges[:, 1]], axis=1)
        self.fixed = torch.as_tensor(fixed.astype(np.uint8), device=dev)
        self.free = torch.as_tensor(~fixed, device=dev)
        # unit coil current per element: curl of the interpolated current potential
        t_edge = torch.as_tensor(synth.coil_edge_values(P, edges), dtype=torch.float64, device=dev)
        jb, _ = self.plan.element_b(t_edge)
        self.j_unit = jb.contiguous()
        self.iron = torch.as_tensor(np.flatnonzero(self.tags == synth.IRON).astype(np.int32), device=dev)
        self.iron_rows = torch.arange(self.iron.numel(), dtype=torch.int32, device=dev)
        sigma = np.where(self.tags == synth.IRON, cfg.sigma_iron, 0.0)
        self.has_sigma = bool(np.any(sigma != 0.0))
        self.m_sigma = self.plan.mass(torch.as_tensor(sigma, dtype=torch.float64, device=dev)) \
            if self.has_sigma else None
        self.m_reg = self.plan.mass(None)
        # regularisation scale from the first Newton matrix of a run started at A = 0
        # (TransientSolver.m:168-175 with x_prev = 0)
        vals0, _ = self.plan.jacobian(torch.zeros(E, dtype=torch.float64, device=dev))
        if self.has_sigma:
            vals0 = vals0 + self.m_sigma / cfg.dt
        d = self._diag(vals0).abs()
        d = d[d > 0]
        self.reg = float(d.mean()) * cfg.reg_rel if d.numel() else cfg.reg_rel
        h = C.c_void_p()
        _lib.check(self.lib.mag_pcg_create(E, C.byref(h)))
        self._pcg = h
        a0 = vals0 + self.reg * self.m_reg
        self.dirichlet(a0, None)
        self._setup_aux(a0, fixed, on)
        # the system matrix lives in one buffer, so the solver's captured iteration graph stays valid
        self._A = torch.empty(self.plan.nnz, dtype=torch.float64, device=dev)

    # ---- small helpers -----------------------------------------------------
    def source_scale(self, t: float) -> float:
        return self.cfg.j_peak * float(np.sin(2.0 * np.pi * self.cfg.freq * t))

    def spmv(self, vals, x, out=None):
        out = torch.empty_like(x) if out is None else out
        _lib.check(self.lib.mag_csr_spmv(self.num_dofs, _ptr(self.rp), _ptr(self.ci), _ptr(vals), _ptr(x),
                                         _ptr(out), _lib.stream_ptr()))
        return out

    def dirichlet(self, vals, rhs):
        _lib.check(self.lib.mag_csr_apply_dirichlet(self.num_dofs, _ptr(self.rp), _ptr(self.ci), _ptr(vals),
                                                    _ptr(self.fixed), _ptr(rhs), _lib.stream_ptr()))

    def solve(self, vals, b, x):
        it, rel, st = C.c_int(), C.c_double(), C.c_int()
        _lib.check(self.lib.mag_pcg_solve(self._pcg, _ptr(self.rp), _ptr(self.ci), _ptr(vals), _ptr(b), _ptr(x),
                                          self.cfg.cg_rtol, self.cfg.cg_max, C.byref(it), C.byref(rel),
                                          C.byref(st), _lib.stream_ptr()))
        return it.value, rel.value, st.value

    def source(self, t: float):
        js = (self.j_unit * self.source_scale(t)).contiguous()
        return self.plan.source(js)

    def element_bmag(self, x):
        _, bsq = self.plan.element_b(x, want_vec=False)
        return torch.sqrt(bsq)

    def element_nu(self, x, out=None):
        out = torch.empty(self.plan.num_elements, dtype=torch.float64, device="cuda") if out is None else out
        _lib.check(self.lib.mag_element_nu(self.plan._h, _ptr(x), _ptr(out), None, _lib.stream_ptr()))
        return out

    def residual(self, x, x_prev, F, calc_j: bool, bscale=None):
        """(J_sys values or None, R_sys) before boundary elimination; bscale seeds the tangent."""
        if bscale is not None:
            vals, r = self.plan.new_values(), self.plan.new_vector()
            _lib.check(self.lib.mag_assemble_jacobian_seeded(self.plan._h, _ptr(x), _ptr(bscale), _ptr(vals),
                                                             _ptr(r), _lib.stream_ptr()))
        else:
            vals, r = self.plan.jacobian(x, calc_j=calc_j)
        if self.has_sigma:
            r = r + self.spmv(self.m_sigma, x - x_prev) / self.cfg.dt
            if calc_j:
                vals = vals + self.m_sigma / self.cfg.dt
        r = r - F
        return vals, r

    def _regularise(self, vals, r, x):
        if self.reg > 0.0:
            vals.add_(self.m_reg, alpha=self.reg)
            r.add_(self.spmv(self.m_reg, x), alpha=self.reg)

    # ---- one time step -------------------------------------------------------
    def step(self, x_prev, t: float, step: int, mode: str = "plain", seed_nu=None) -> tuple:
        """Newton solve of one backward-Euler step; returns (x, StepStats).

        seed_nu: predicted per-element reluctivity [Ne] (float64, device; <= 0 where
        there is no prediction); the first Jacobian is then taken at the midpoint
        between x_prev's and the predicted flux density (mag_seed_midpoint).
        """
        cfg = self.cfg
        st = StepStats(step=step, mode=mode)
        tm = _Timer()
        e_step = tm.start()
        F = self.source(t)
        Fb = F.clone()
        Fb[self.free.logical_not()] = 0.0
        st.tol_abs = cfg.tol * max(float(torch.linalg.vector_norm(Fb)), 1.0)
        x = x_prev.clone()
        bscale = None
        if seed_nu is not None:
            bscale = torch.empty(self.plan.num_elements, dtype=torch.float64, device="cuda")
            _lib.check(self.lib.mag_seed_midpoint(self.plan._h, _ptr(x), _ptr(seed_nu), cfg.seed_max_scale,
                                                  _ptr(bscale), _lib.stream_ptr()))
        for it_n in range(1, cfg.max_newton + 1):
            e0 = tm.start()
            vals, r = self.residual(x, x_prev, F, True, bscale if it_n == 1 else None)
            tm.stop(e0, "assembly")
            st.newton += 1
            self._regularise(vals, r, x)
            self._A.copy_(vals)
            self.dirichlet(self._A, r)
            norm_res = float(torch.linalg.vector_norm(r))
            st.res = norm_res
            st.res_history.append(norm_res)
            if norm_res <= st.tol_abs:
                st.converged = True
                break
            dx = torch.zeros_like(x)
            e0 = tm.start()
            cg_it, _, _ = self.solve(self._A, -r, dx)
            tm.stop(e0, "solve")
            st.solves += 1
            st.cg_iters += cg_it
            alpha = 1.0
            for k in range(cfg.max_line_search + 1):
                a_try = alpha * 0.5 ** k
                x_try = x + a_try * dx
                e0 = tm.start()
                _, r_try = self.residual(x_try, x_prev, F, False)
                tm.stop(e0, "assembly")
                st.residual_only += 1
                if self.reg > 0.0:
                    r_try.add_(self.spmv(self.m_reg, x_try), alpha=self.reg)
                r_try[self.free.logical_not()] = 0.0
                res_try = float(torch.linalg.vector_norm(r_try))
                if res_try < norm_res or (it_n == 1 and k < 3):
                    alpha = a_try
                    break
                if res_try > norm_res * 10:
                    alpha = alpha * 0.1
            x = x + alpha * dx
        tm.stop(e_step, "step")
        t_ = tm.collect()
        st.gpu_ms = t_.get("step", 0.0)
        st.solve_ms = t_.get("solve", 0.0)
        st.assembly_ms = t_.get("assembly", 0.0)
        return x, st

    def _setup_aux(self, a0, fixed, on):
        """Gradient auxiliary space of the CG preconditioner (free edges x interior nodes)."""
        import scipy.sparse as sp

        E, e = self.num_dofs, self.edges
        interior = ~np.any(on, axis=1)
        node_map = np.full(interior.size, -1, dtype=np.int64)
        node_map[interior] = np.arange(int(interior.sum()))
        rows = np.r_[np.arange(E), np.arange(E)]
        cols = node_map[np.r_[e[:, 0], e[:, 1]]]
        vals = np.r_[-np.ones(E), np.ones(E)]
        keep = (cols >= 0) & ~fixed[rows]
        ni = int(interior.sum())
        G = sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(E, ni))
        Gt = G.T.tocsr()
        A = sp.csr_matrix((a0.cpu().numpy(), self.ci.cpu().numpy(), self.rp.cpu().numpy()), shape=(E, E))
        dn = (Gt @ A @ G).diagonal()
        dn_inv = np.where(dn > 0, 1.0 / np.where(dn > 0, dn, 1.0), 0.0)
        dev = torch.device("cuda")

        def up(a, dt):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)

        self._aux = [up(G.indptr, torch.int64), up(G.indices, torch.int32), up(G.data, torch.float64),
                     up(Gt.indptr, torch.int64), up(Gt.indices, torch.int32), up(Gt.data, torch.float64),
                     up(dn_inv, torch.float64)]
        _lib.check(self.lib.mag_pcg_set_aux(self._pcg, ni, *[_ptr(t) for t in self._aux]))

    def _diag(self, vals):
        n = self.num_dofs
        rows = torch.repeat_interleave(torch.arange(n, device="cuda"), self.rp[1:] - self.rp[:-1])
        return vals[rows == self.ci.long()]

    def close(self):
        if getattr(self, "_pcg", None):
            self.lib.mag_pcg_destroy(self._pcg)
            self._pcg = None
        self.plan.close()


@dataclass
class RunRecord:
    stats: list = field(default_factory=list)
    bmag: list = field(default_factory=list)   # per step: |B| of the nonlinear elements (float32)
    nu: list = field(default_factory=list)     # per step: converged nu of the nonlinear elements
    x: list = field(default_factory=list)      # (step, solution) pairs kept on request


def features(prob: TransientProblem, b1, b2, t: float) -> torch.Tensor:
    """MLP inputs of the nonlinear elements for step time t: |B|_{t-1}, |B|_{t-2}, |J(t)|, material id."""
    n = prob.iron.numel()
    f = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    f[:, 0] = b1
    f[:, 1] = b2
    f[:, 2] = abs(prob.source_scale(t))
    f[:, 3] = float(synth.IRON)
    return f


def run(prob: TransientProblem, first: int, last: int, x_prev, b_hist, mode: str = "plain", predictor=None,
        keep_x=(), record: RunRecord | None = None, reference_x=None) -> RunRecord:
    """Steps first..last (1-based). b_hist = (|B|_{first-1}, |B|_{first-2}) of the nonlinear elements.

    mode: "plain", "learned" (needs predictor) or "ideal" (needs reference_x: step -> converged x).
    """
    rec = record or RunRecord()
    cfg = prob.cfg
    b1, b2 = b_hist
    x = x_prev
    ir = prob.iron.long()
    for s in range(first, last + 1):
        t = s * cfg.dt
        seed = None
        mlp_ms = 0.0
        if mode == "learned":
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            seed = torch.zeros(prob.plan.num_elements, dtype=torch.float64, device="cuda")
            ratio = torch.empty(prob.iron.numel(), dtype=torch.float64, device="cuda")
            predictor.predict_nu(features(prob, b1, b2, t), prob.iron_rows, ratio, nu_min=1e-3, nu_max=1e3)
            seed[ir] = prob.element_nu(x)[ir] * ratio
            e1.record()
            e1.synchronize()
            mlp_ms = e0.elapsed_time(e1)
        elif mode == "ideal":
            seed = torch.zeros(prob.plan.num_elements, dtype=torch.float64, device="cuda")
            seed[ir] = prob.element_nu(reference_x[s])[ir]
        x_new, st = prob.step(x, t, s, mode, seed)
        st.mlp_ms = mlp_ms
        st.gpu_ms += mlp_ms
        bm = prob.element_bmag(x_new)[ir].float()
        nu_c = prob.element_nu(x_new)[ir]
        if seed is not None:
            rel = (seed[ir] - nu_c).abs() / nu_c
            st.nu_rel_err = float(rel.mean())
            st.nu_rel_err_max = float(rel.max())
        rec.stats.append(st)
        rec.bmag.append(bm)
        rec.nu.append(nu_c.float())
        if s in keep_x:
            rec.x.append((s, x_new.clone()))
        b2, b1 = b1, bm
        x = x_new
    return rec


def training_set(prob: TransientProblem, rec: RunRecord, first: int, last: int):
    """(features, nu_t / nu_{t-1}) pairs of steps first..last from a plain run recorded from step 1.

    The network learns the step's change of reluctivity; the seed multiplies it onto the
    reluctivity evaluated exactly at x_{t-1}, so its error scales with the change, not with nu.
    """
    cfg = prob.cfg
    n = prob.iron.numel()
    zero = torch.zeros(n, dtype=torch.float32, device="cuda")
    nu0 = prob.element_nu(torch.zeros(prob.num_dofs, dtype=torch.float64, device="cuda"))[prob.iron.long()]
    fs, ys = [], []
    for s in range(first, last + 1):
        b1 = rec.bmag[s - 2] if s >= 2 else zero
        b2 = rec.bmag[s - 3] if s >= 3 else zero
        fs.append(features(prob, b1, b2, s * cfg.dt))
        prev = rec.nu[s - 2].double() if s >= 2 else nu0
        ys.append(rec.nu[s - 1].double() / prev)
    return torch.cat(fs), torch.cat(ys)


def summarize(stats) -> dict:
    keys = ("newton", "residual_only", "solves", "cg_iters")
    out = {k: int(sum(getattr(s, k) for s in stats)) for k in keys}
    out["assemblies"] = int(sum(s.assemblies for s in stats))
    for k in ("gpu_ms", "solve_ms", "assembly_ms", "mlp_ms"):
        out[k] = float(sum(getattr(s, k) for s in stats))
    out["steps"] = len(stats)
    out["converged"] = all(s.converged for s in stats)
    out["max_res_over_tol"] = float(max(s.res / s.tol_abs for s in stats))
    errs = [s.nu_rel_err for s in stats if s.nu_rel_err == s.nu_rel_err]
    out["nu_rel_err_mean"] = float(np.mean(errs)) if errs else None
    out["nu_rel_err_median"] = float(np.median(errs)) if errs else None
    errs = [s.nu_rel_err_max for s in stats if s.nu_rel_err_max == s.nu_rel_err_max]
    out["nu_rel_err_max"] = float(np.max(errs)) if errs else None
    return out


def compare(cfg: TransientConfig | None = None, train_steps: int | None = None, epochs: int = 10,
            seed: int = 0, log=None, ideal: bool = True, batch: int = 32768, lr: float = 4e-3) -> dict:
    """Plain run over all steps; train on the first half; rerun the second half learned (and ideal)."""
    from .mlp import NuPredictor

    cfg = cfg or TransientConfig()
    half = train_steps or cfg.steps // 2
    prob = TransientProblem(cfg)
    try:
        n = prob.iron.numel()
        zero = torch.zeros(n, dtype=torch.float32, device="cuda")
        x0 = torch.zeros(prob.num_dofs, dtype=torch.float64, device="cuda")
        t0 = time.perf_counter()
        plain = run(prob, 1, cfg.steps, x0, (zero, zero), "plain",
                    keep_x=tuple(range(half, cfg.steps + 1)) if ideal else (half,))
        wall_plain = time.perf_counter() - t0
        if log:
            log(f"plain: {summarize(plain.stats)} ({wall_plain:.1f} s)")
        feats, nu = training_set(prob, plain, 1, half)
        pred = NuPredictor(seed=seed)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        hist = pred.fit(feats, nu, epochs=epochs, batch=batch, lr=lr, seed=seed)
        e1.record()
        e1.synchronize()
        train_ms = e0.elapsed_time(e1)
        xs = dict(plain.x)
        x_half = xs[half]
        b_hist = (plain.bmag[half - 1], plain.bmag[half - 2] if half >= 2 else zero)
        # the second half again without a seed, after warm-up, for a like-for-like device time
        plain2 = run(prob, half + 1, cfg.steps, x_half, b_hist, "plain")
        learned = run(prob, half + 1, cfg.steps, x_half, b_hist, "learned", pred)
        ideal_rec = run(prob, half + 1, cfg.steps, x_half, b_hist, "ideal", reference_x=xs) if ideal else None
        out = {
            "config": {"mesh": [cfg.nx, cfg.ny, cfg.nz], "elements": int(prob.plan.num_elements),
                       "dofs": int(prob.num_dofs), "nonlinear_elements": int(n), "steps": cfg.steps,
                       "dt": cfg.dt, "train_steps": half, "tol": cfg.tol, "reg": prob.reg,
                       "sigma_iron": cfg.sigma_iron},
            "plain_first": summarize(plain.stats[:half]),
            "plain": summarize(plain2.stats),
            "learned": summarize(learned.stats),
            "ideal": summarize(ideal_rec.stats) if ideal else None,
            "train": {"samples": int(feats.shape[0]), "epochs": epochs, "batch": batch, "lr": lr,
                      "loss_first": hist[0],
                      "loss_last": hist[-1], "gpu_ms": train_ms},
            # the whole cost of the learned warm start on steps 101-200: its steps plus the
            # training on steps 1-100, against the plain warm start's steps
            "net_gpu_ms": {"plain": summarize(plain2.stats)["gpu_ms"],
                           "learned_with_training": summarize(learned.stats)["gpu_ms"] + train_ms},
            "per_step": {"plain": [s.newton for s in plain2.stats],
                         "learned": [s.newton for s in learned.stats],
                         "ideal": [s.newton for s in ideal_rec.stats] if ideal else None},
        }
        pred.mlp.close()
        return out
    finally:
        prob.close()
