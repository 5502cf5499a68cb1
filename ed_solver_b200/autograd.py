"""torch.autograd binding of the adjoint entry points.

``ImpurityGreen.apply(theta, problem)`` returns the ground-state energy E0 and
the Green functions G_c(i w_n) of one (N_up, N_dn) sector as functions of the
model parameters theta (a float64 CPU tensor, one value per entry of
``problem.params``).  The forward pass runs the device solve (FP64 Lanczos
with a residual-converged eigenvector, then one compute_dynamic chain per
channel); the backward pass calls edk_grad_green, which differentiates E0
(Hellmann-Feynman), the Lanczos chains (reverse mode with checkpointed replay)
and the eigenvector (conjugate-gradient adjoint solve).  Nothing here computes
on the CPU: the library is the only path.
"""
from __future__ import annotations

import dataclasses
from typing import List, Sequence, Tuple

import numpy as np
import torch

from . import edk
from .model import AIMModel


@dataclasses.dataclass
class GreenProblem:
    """What ImpurityGreen differentiates.

    chains: (site, spin, dagger) per Green channel (dagger=True: particle part).
    """
    ctx: "edk.Context"
    model: AIMModel
    params: List[Tuple[int, int, int, int]]
    sector: Tuple[int, int]
    chains: Sequence[Tuple[int, int, bool]]
    nitergreen: int
    wn: np.ndarray
    tolerance: float = 1e-13
    residual_tol: float = 1e-11
    nitermax: int = 1000
    cg_tol: float = 1e-11

    def values(self) -> np.ndarray:
        """The current parameter values of the model (the point theta0)."""
        m = self.model
        out = []
        for kind, i, j, spin in self.params:
            s = 0 if spin == 2 else spin
            if kind == edk.PARAM_U:
                out.append(m.u[i, j])
            else:
                out.append({edk.PARAM_EC: m.ec, edk.PARAM_EB: m.eb, edk.PARAM_VBC: m.vbc}[kind][s, i, j])
        return np.array(out, np.float64)

    def model_at(self, theta: np.ndarray) -> AIMModel:
        """The model with every listed parameter set to theta."""
        m = self.model
        for p, t, t0 in zip(self.params, theta, self.values()):
            m = edk.perturb(m, p, float(t) - float(t0))
        return m


class ImpurityGreen(torch.autograd.Function):
    @staticmethod
    def forward(fctx, theta: torch.Tensor, problem: GreenProblem):
        model = problem.model_at(theta.detach().cpu().numpy())
        h = edk.Hamiltonian(problem.ctx, model, *problem.sector)
        r = h.lanczos_e0("f64", tolerance=problem.tolerance, residual_tol=problem.residual_tol,
                         nitermax=problem.nitermax)
        psi = h.lanczos_gs(r["vecp"][0])
        e0 = float(r["E"][0])
        G = []
        for site, spin, dag in problem.chains:
            phi, ts = h.apply_c(psi, site, spin, dag)
            ht = edk.Hamiltonian(problem.ctx, model, *ts)
            g, _, _, _ = ht.green_chain(phi, problem.nitergreen, e0, 1 if dag else 2, problem.wn, cutoff_dynamic=0.0)
            G.append(g)
            ht.close()
        fctx.saved = (h, psi, e0, problem)
        return torch.tensor(e0, dtype=torch.float64), torch.tensor(np.array(G), dtype=torch.complex128)

    @staticmethod
    def backward(fctx, gE0, gG):
        h, psi, e0, problem = fctx.saved
        gb = gG.detach().cpu().numpy() if gG is not None else np.zeros((len(problem.chains), len(problem.wn)),
                                                                         np.complex128)
        e0bar = float(gE0) if gE0 is not None else 0.0
        grad, _, _ = h.grad_green(psi, e0, list(problem.chains), problem.nitergreen, problem.wn, gb, problem.params,
                                  e0bar=e0bar, cg_tol=problem.cg_tol)
        return torch.tensor(grad, dtype=torch.float64), None
