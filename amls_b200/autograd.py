"""Thin torch.autograd.Function over the AMLS solve and the adjoint
sensitivity kernel, used to check the gradient of sum_k w_k lambda_k with
respect to the per-element moduli E_e and densities rho_e against finite
differences.  The forward assembles K = sum_e E_e Kbar and
M = sum_e rho_e Mbar on the host, solves on the GPU (refined to FP64
accuracy) and returns sum_k w_k lambda_k; the backward returns the adjoint
gradient from amls_sensitivities (simple eigenvalues only).
"""
from __future__ import annotations

import numpy as np
import torch

from . import cases
from .solver import AmlsOptions, AmlsSolver


class WeightedEigenvalueSum(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E: torch.Tensor, rho: torch.Tensor, solver: AmlsSolver, pencil: cases.Pencil,
                weights: np.ndarray, opt: AmlsOptions):
        Ev = E.detach().cpu().double().numpy()
        rv = rho.detach().cpu().double().numpy()
        n = pencil.n
        K = cases._assemble(pencil.dofmap, pencil.Kbar, Ev, n)
        M = cases._assemble(pencil.dofmap, pencil.Mbar, rv, n)
        sol = solver.solve(K, M, opt)
        p = cases.Pencil(K, M, dofmap=pencil.dofmap, Kbar=pencil.Kbar, Mbar=pencil.Mbar, E=Ev,
                         rho=rv)
        sens = solver.sensitivities(p, weights=weights)
        ctx.save_for_backward(torch.from_numpy(sens["gE"]), torch.from_numpy(sens["gRho"]))
        value = float(np.dot(weights[sens["simple"]], sol.theta[sens["simple"]]))
        return torch.tensor(value, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad):
        gE, gR = ctx.saved_tensors
        return grad * gE, grad * gR, None, None, None, None
