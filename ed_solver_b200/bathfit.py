"""Bath fit: the caller of the gradients.

The reference fits the bath parameters to a target hybridisation between DMFT
iterations (hybrid2bath, ed_solver/bath_class_hybrid.f90:919-1133):
  * bath2hybrid (bath_class_hybrid.f90:587-903), branch without the cluster
    perturbation extension: Delta(i w_n) = Vcb (i w_n - Eb_Nambu)^-1 Vbc over
    the Nambu matrices of Nambu_Eb / Nambu_Vbc (bath_class.f90:956-1022), a
    2nc x 2nc function (for a normal bath: diag(Delta_up(i w), -conj Delta_dn(i w)));
  * distance_func -> diff_correl (correl_class.f90:1061-1145), default options
    (no symmetry penalty, no frequency window, every element weighted 1):
      d = sum_{n <= fit_nw} sum_{ab} |Delta_t - Delta_b|^weight_expo
          / (|w_n - w_1| + fit_shift)^fit_weight_power,   divided by fit_nw * N^2;
  * a quasi-Newton minimiser over the bath vector (minimize_func_wrapper with
    FIT_METH = MINIMIZE, tools_minimization_wrapping.f90:125-399, whose
    minimize_civelli, conj_grad_civelli.f90:7, builds its gradient by finite
    differences of size search_step).

Here the distance has an exact gradient (the adjoint of Delta with respect to
the bath levels, hybridisations and pairings), and the minimiser is BFGS with
that gradient and a backtracking line search; it stops when the distance falls
below dist_max or after niter_search_max iterations (the reference's
Niter_search_max counts function calls).  `fit_green` closes the loop through
the impurity solver on the device instead: it fits the bath so that the
impurity Green function of the solve matches a target, with the gradients from
the adjoint entry points (edk_grad_green through autograd.ImpurityGreen).

Parameter vector of a star bath (the independent elements bath2vec collects,
bath_class_vec.f90:27-68, for diagonal Eb and one hybridisation per bath site
and orbital): bath levels eps_k, then the non-zero V_kc, then (Nambu) the
pairings P_k; spin-symmetric.
"""
from __future__ import annotations

import dataclasses
from typing import Optional, Tuple

import numpy as np

from .model import AIMModel, NambuModel

FIT_WEIGHT_POWER = 0.5     # fit_weight_power (dmft_ed_solver_variables.h:6)
FIT_SHIFT = 0.01           # fit_shift (:7)
WEIGHT_EXPO = 2.0          # weight_expo (:38)
FIT_NW = 650               # fit_nw (:33)
NITER_SEARCH_MAX = 100     # Niter_search_max (:10)
DIST_MAX = 1e-10           # dist_max (:12)


@dataclasses.dataclass
class StarBath:
    """A star bath: levels eps (nb,), hybridisations V (nb, nc) with a fixed
    non-zero pattern, optional s-wave pairings P (nb,), spin-symmetric."""
    eps: np.ndarray
    V: np.ndarray
    P: Optional[np.ndarray] = None

    @property
    def mask(self) -> np.ndarray:
        return self.V != 0

    def vec(self) -> np.ndarray:
        parts = [self.eps, self.V[self.mask]]
        if self.P is not None:
            parts.append(self.P)
        return np.concatenate(parts).astype(np.float64)

    def with_vec(self, x: np.ndarray, mask: Optional[np.ndarray] = None) -> "StarBath":
        mask = self.mask if mask is None else mask
        nb = len(self.eps)
        nv = int(mask.sum())
        V = np.zeros_like(self.V)
        V[mask] = x[nb:nb + nv]
        P = None if self.P is None else np.array(x[nb + nv:nb + nv + nb])
        return StarBath(np.array(x[:nb]), V, P)

    @staticmethod
    def of(model) -> "StarBath":
        base = model.base if isinstance(model, NambuModel) else model
        P = np.diag(model.pb).copy() if isinstance(model, NambuModel) else None
        return StarBath(np.diag(base.eb[0]).copy(), base.vbc[0].copy(), P)

    def apply(self, model):
        """The model with this bath (both spins)."""
        base = model.base if isinstance(model, NambuModel) else model
        b = dataclasses.replace(base, eb=base.eb.copy(), vbc=base.vbc.copy())
        for s in range(2):
            b.eb[s] = np.diag(self.eps)
            b.vbc[s] = self.V
        if isinstance(model, NambuModel):
            return NambuModel(b, np.diag(self.P if self.P is not None else np.zeros(len(self.eps))), model.pvbc,
                              model.on_fly)
        return b


def nambu_hybrid(bath: StarBath, wn: np.ndarray) -> np.ndarray:
    """Delta(i w_n) (nw, 2nc, 2nc) = Vcb (i w_n - Eb_Nambu)^-1 Vbc (bath2hybrid)."""
    nb, nc = bath.V.shape
    ebn = np.zeros((2 * nb, 2 * nb))
    ebn[:nb, :nb] = np.diag(bath.eps)
    ebn[nb:, nb:] = -np.diag(bath.eps)
    if bath.P is not None:
        ebn[:nb, nb:] = np.diag(bath.P)
        ebn[nb:, :nb] = np.diag(bath.P)
    vbn = np.zeros((2 * nb, 2 * nc))
    vbn[:nb, :nc] = bath.V
    vbn[nb:, nc:] = -bath.V
    eye = np.eye(2 * nb)
    out = np.empty((len(wn), 2 * nc, 2 * nc), np.complex128)
    for n, w in enumerate(wn):
        out[n] = vbn.T @ np.linalg.solve(1j * w * eye - ebn, vbn)
    return out


def _weights(wn: np.ndarray, fit_shift: float, power: float) -> np.ndarray:
    shift = fit_shift if abs(fit_shift) >= 1e-10 else abs(wn[0])
    return 1.0 / (np.abs(wn - wn[0]) + shift) ** power


def distance(d_bath: np.ndarray, d_target: np.ndarray, wn: np.ndarray, fit_shift=FIT_SHIFT,
             power=FIT_WEIGHT_POWER, expo=WEIGHT_EXPO) -> float:
    """diff_correl with the default options (correl_class.f90:1061-1128)."""
    nw = d_bath.shape[0]
    N = d_bath.shape[1]
    w = _weights(wn[:nw], fit_shift, power)
    s = (np.abs(d_target[:nw] - d_bath) ** expo).sum(axis=(1, 2))
    return float(abs((s * w).sum()) / (nw * N * N))


def distance_and_grad(bath: StarBath, d_target: np.ndarray, wn: np.ndarray, fit_nw=FIT_NW, fit_shift=FIT_SHIFT,
                      power=FIT_WEIGHT_POWER) -> Tuple[float, np.ndarray]:
    """Distance (weight_expo = 2) and its exact gradient with respect to the
    bath vector, from the resolvent R = (i w - Eb_N)^-1:
    dDelta = dVn^T R Vn + Vn^T R dVn + Vn^T R dEb_N R Vn."""
    nw = min(fit_nw, len(wn))
    wn = wn[:nw]
    nb, nc = bath.V.shape
    mask = bath.mask
    ebn = np.zeros((2 * nb, 2 * nb))
    ebn[:nb, :nb] = np.diag(bath.eps)
    ebn[nb:, nb:] = -np.diag(bath.eps)
    if bath.P is not None:
        ebn[:nb, nb:] = np.diag(bath.P)
        ebn[nb:, :nb] = np.diag(bath.P)
    vbn = np.zeros((2 * nb, 2 * nc))
    vbn[:nb, :nc] = bath.V
    vbn[nb:, nc:] = -bath.V
    N = 2 * nc
    w = _weights(wn, fit_shift, power) / (nw * N * N)
    eye = np.eye(2 * nb)
    nv = int(mask.sum())
    g = np.zeros(nb + nv + (nb if bath.P is not None else 0))
    d = 0.0
    kv = np.argwhere(mask)
    for n, om in enumerate(wn):
        R = np.linalg.inv(1j * om * eye - ebn)
        RV = R @ vbn
        D = vbn.T @ RV
        E = D - d_target[n]                       # Delta_b - Delta_t
        d += w[n] * float((np.abs(E) ** 2).sum())
        # dd/dDelta (real-parameter chain rule): 2 w Re(conj(E) . dDelta)
        A = 2.0 * w[n] * np.conj(E)               # (N, N)
        # Vn^T R dEb_N R Vn (R is complex symmetric): d/dEb_N[p,q] = (RV A RV^T)[p,q]
        M = RV @ A @ RV.T
        for k in range(nb):
            g[k] += float(np.real(M[k, k] - M[nb + k, nb + k]))
        if bath.P is not None:
            for k in range(nb):
                g[nb + nv + k] += float(np.real(M[k, nb + k] + M[nb + k, k]))
        # d/dVn[p, a]: dVn^T R Vn gives (RV A^T)[p,a], Vn^T R dVn gives (RV A)[p,a]
        GV = RV @ A.T + RV @ A
        for q, (k, c) in enumerate(kv):
            g[nb + q] += float(np.real(GV[k, c] - GV[nb + k, nc + c]))
    return d, g


def fit_hybrid(bath0: StarBath, d_target: np.ndarray, wn: np.ndarray, fit_nw=FIT_NW, niter=NITER_SEARCH_MAX,
               dist_max=DIST_MAX, fit_shift=FIT_SHIFT, power=FIT_WEIGHT_POWER):
    """hybrid2bath: BFGS on the distance with its exact gradient.  Returns
    (fitted bath, final distance, iterations)."""
    x = bath0.vec()
    mask = bath0.mask

    def fg(v):
        return distance_and_grad(bath0.with_vec(v, mask), d_target, wn, fit_nw, fit_shift, power)

    f, g = fg(x)
    H = np.eye(len(x))
    it = 0
    for it in range(1, niter + 1):
        if f < dist_max:
            break
        p = -H @ g
        if g @ p >= 0:
            H = np.eye(len(x))
            p = -g
        t, f_new, g_new = 1.0, None, None
        for _ in range(40):
            xn = x + t * p
            f_new, g_new = fg(xn)
            if f_new <= f + 1e-4 * t * (g @ p):
                break
            t *= 0.5
        s, yv = xn - x, g_new - g
        x, f, g = xn, f_new, g_new
        sy = s @ yv
        if sy > 1e-300:
            rho = 1.0 / sy
            I = np.eye(len(x))
            H = (I - rho * np.outer(s, yv)) @ H @ (I - rho * np.outer(yv, s)) + rho * np.outer(s, s)
    return bath0.with_vec(x, mask), f, it


def fit_green(ctx, model: AIMModel, G_target: np.ndarray, sector, wn: np.ndarray, nitergreen: int = 200,
              steps: int = 20, lr: float = 0.5):
    """Fit the bath so that the impurity Green function of the (N_up, N_dn)
    sector's ground state (spin up, site 0, particle + hole chains) matches
    G_target on wn, with the gradients of the device adjoint (edk_grad_green).
    Returns (fitted model, loss history)."""
    import torch
    from . import edk
    from .autograd import GreenProblem, ImpurityGreen
    params = [p for p in edk.star_params(model) if p[0] in (edk.PARAM_EB, edk.PARAM_VBC)]
    prob = GreenProblem(ctx=ctx, model=model, params=params, sector=tuple(sector),
                        chains=[(0, 0, True), (0, 0, False)], nitergreen=nitergreen, wn=np.asarray(wn))
    theta = torch.tensor(prob.values(), dtype=torch.float64, requires_grad=True)
    target = torch.tensor(np.asarray(G_target), dtype=torch.complex128)
    opt = torch.optim.LBFGS([theta], lr=lr, max_iter=steps, line_search_fn="strong_wolfe")
    hist = []

    def closure():
        opt.zero_grad()
        _, G = ImpurityGreen.apply(theta, prob)
        loss = (torch.abs(G.sum(0) - target) ** 2).mean()
        loss.backward()
        hist.append(float(loss.detach()))
        return loss

    opt.step(closure)
    return prob.model_at(theta.detach().numpy()), hist
