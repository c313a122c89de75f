"""Harmonic-balance (HBFEM) assembly: the AFT operators and the assembly call.

``AFT`` restates src/utils/AFT.m:19-86: harmonics h_k, N time samples
(default max(32, 2^ceil(log2(2 max h + 1))), at least 2 max h + 1), the
frequency-to-time matrix D[t, k] = exp(i h_k theta_t) and the time-to-frequency
matrix P[k, t] = f_k exp(-i h_k theta_t) with f = 1/N for h = 0 and 2/N otherwise,
theta_t = 2 pi t / N.

``assemble_hbfem`` is the GPU counterpart of assemble_hbfem_kernel_mex
(src/mex/assemble_hbfem_kernel_mex.cpp:26-258), the call HBFEMSolver makes through
Assembler.assembleHBFEM (HBFEMSolver.m:78,96; the wrapper itself is absent from the
reference). It returns the harmonic residual [K, Ndof] (complex) and, on request,
the DC-reluctivity curl-curl block on the mesh's CSR pattern; harmonic k's Jacobian
block is Scalings[k] times that block (HBFEMSolver assembles them block-diagonally).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


class AFT:
    def __init__(self, harmonics, n_time_steps=None, base_freq: float = 50.0):
        self.harmonics = np.asarray(harmonics, dtype=np.int64).ravel()
        max_h = int(self.harmonics.max())
        min_steps = 2 * max_h + 1
        if n_time_steps is None:
            n = max(32, 1 << int(np.ceil(np.log2(min_steps))))
        else:
            n = max(int(n_time_steps), min_steps)
        self.num_time_steps = n
        self.base_freq = float(base_freq)
        theta = np.arange(n) * (2.0 * np.pi / n)
        h = self.harmonics[None, :]
        self.D = np.exp(1j * h * theta[:, None])                                  # [N, K]
        f = np.where(self.harmonics == 0, 1.0 / n, 2.0 / n)
        self.P = f[:, None] * np.exp(-1j * self.harmonics[:, None] * theta[None, :])  # [K, N]

    @property
    def num_harmonics(self):
        return self.harmonics.size

    def device_operators(self):
        """D and P split into real / imaginary float64 CUDA tensors in the library's layout
        (D as [K][N], P as [N][K]); made once and kept."""
        if getattr(self, "_dev", None) is None:
            dev = torch.device("cuda")

            def t(a):
                return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)

            self._dev = (t(np.real(self.D).T), t(np.imag(self.D).T), t(np.real(self.P).T), t(np.imag(self.P).T))
        return self._dev


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def assemble_hbfem(plan, sol, aft: AFT, calc_j: bool = True, stream=None):
    """Harmonic residual and DC Jacobian block for the harmonic field sol [Ndof, K] (complex):
    a host array, or a CUDA tensor (complex128 [Ndof, K], or a (re, im) pair of float64
    [K, Ndof] tensors in the library's layout, which is used as is).

    Returns (R complex [K, Ndof] on the GPU, vals [nnz] float64 or None)."""
    L = _lib.lib()
    K, N = aft.num_harmonics, aft.num_time_steps
    dev = torch.device("cuda")
    if isinstance(sol, tuple):
        sr, si = sol
    elif isinstance(sol, torch.Tensor):
        sr = torch.real(sol).T.contiguous().to(torch.float64)  # [K][Ndof]
        si = torch.imag(sol).T.contiguous().to(torch.float64) if sol.is_complex() else None
    else:
        sol = np.asarray(sol)
        sr = torch.as_tensor(np.ascontiguousarray(np.real(sol).T), dtype=torch.float64, device=dev)  # [K][Ndof]
        si = torch.as_tensor(np.ascontiguousarray(np.imag(sol).T), dtype=torch.float64, device=dev)
    if sr.shape != (K, plan.num_dofs) or not sr.is_cuda or (si is not None and si.shape != sr.shape):
        raise ValueError("harmonic field must be [Ndof, K] for the AFT's K harmonics")
    dr, di, pr, pi = aft.device_operators()
    rre = torch.empty((K, plan.num_dofs), dtype=torch.float64, device=dev)
    rim = torch.empty_like(rre)
    vals = plan.new_values() if calc_j else None
    _lib.check(L.mag_assemble_hbfem(plan._h, _ptr(sr), _ptr(si), K, _ptr(dr), _ptr(di), _ptr(pr), _ptr(pi), N,
                                    _ptr(vals), _ptr(rre), _ptr(rim), _lib.stream_ptr(stream)))
    return torch.complex(rre, rim), vals
