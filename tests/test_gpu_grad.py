"""Adjoint entry points against the oracle's operators and central finite differences.

Bounds: <a|dH/dtheta|b> equals a.(H_theta b) from the oracle's matvec of the
model with only that parameter set (1e-12 relative); dE0/dtheta and the
vector-Jacobian product of E0 + G(i w_n) match central differences with
h = 1e-5 on FP64 solves to 1e-5 of the largest component.
"""
import numpy as np
import pytest
import torch

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.autograd import GreenProblem, ImpurityGreen
from ed_solver_b200.model import AIMModel, matsubara, star_model, workload

pytestmark = pytest.mark.gpu

H_FD = 1e-5


def _zero_like(m: AIMModel) -> AIMModel:
    return AIMModel(nc=m.nc, nb=m.nb, ec=np.zeros_like(m.ec), eb=np.zeros_like(m.eb), vbc=np.zeros_like(m.vbc),
                    u=np.zeros_like(m.u), jj=np.zeros_like(m.jj), jhund=0.0, cutoff=m.cutoff)


def test_dh_bilinear_matches_the_oracle_operators(ctx):
    rng = np.random.default_rng(21)
    m = star_model(-1.0, 3.0, rng.uniform(-1, 1, 4), rng.uniform(0.2, 0.6, 4), orbital_of_bath=[0, 1, 1, 0], nc=2)
    m.ec[:, 0, 1] = m.ec[:, 1, 0] = 0.3
    m.eb[:, 0, 2] = m.eb[:, 2, 0] = 0.25
    params = [(edk.PARAM_EC, 0, 0, 0), (edk.PARAM_EC, 1, 1, 2), (edk.PARAM_EC, 0, 1, 2), (edk.PARAM_EB, 3, 3, 1),
              (edk.PARAM_EB, 0, 2, 2), (edk.PARAM_EB, 0, 2, 1), (edk.PARAM_VBC, 1, 1, 2), (edk.PARAM_VBC, 0, 0, 0),
              (edk.PARAM_U, 0, 0, 0), (edk.PARAM_U, 0, 1, 0)]
    for sec in [(3, 3), (2, 4)]:
        h = edk.Hamiltonian(ctx, m, *sec)
        a = rng.normal(size=h.dim)
        b = rng.normal(size=h.dim)
        got = h.dh_bilinear(torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda"), params)
        for q, p in enumerate(params):
            mq = edk.perturb(_zero_like(m), p, 1.0)
            ref = a @ O.OracleH(mq, *sec).hmult(b)
            assert abs(got[q] - ref) <= 1e-12 * max(1.0, abs(ref)), (sec, p, got[q], ref)


def _ground_state(ctx, m, sec):
    h = edk.Hamiltonian(ctx, m, *sec)
    r = h.lanczos_e0("f64", tolerance=1e-14, residual_tol=1e-11)
    return h, h.lanczos_gs(r["vecp"][0]), float(r["E"][0])


def test_grad_e0_against_central_differences(ctx):
    w = workload("c1")
    params = edk.star_params(w.model)
    h, psi, e0 = _ground_state(ctx, w.model, (4, 4))
    g = h.grad_e0(psi, params)
    fd = []
    for p in params:
        ep = _ground_state(ctx, edk.perturb(w.model, p, H_FD), (4, 4))[2]
        em = _ground_state(ctx, edk.perturb(w.model, p, -H_FD), (4, 4))[2]
        fd.append((ep - em) / (2 * H_FD))
    fd = np.array(fd)
    assert np.abs(g - fd).max() <= 1e-5 * np.abs(fd).max()


def _loss(ctx, m, sec, chains, nit, wn, gbar, e0bar):
    h, psi, e0 = _ground_state(ctx, m, sec)
    val = e0bar * e0
    for c, (site, spin, dag) in enumerate(chains):
        phi, ts = h.apply_c(psi, site, spin, dag)
        ht = edk.Hamiltonian(ctx, m, *ts)
        G, _, _, _ = ht.green_chain(phi, nit, e0, 1 if dag else 2, wn, cutoff_dynamic=0.0)
        val += float(np.sum((np.conj(gbar[c]) * G).real))
    return val


def test_grad_green_against_central_differences(ctx):
    """All 16 parameters of the ns=8 star model; particle and hole chains of
    spin up, 80 steps, 64 Matsubara frequencies, random cotangents."""
    w = workload("c1")
    m = w.model
    sec = (4, 4)
    params = edk.star_params(m)
    chains = [(0, 0, True), (0, 0, False)]
    nit = 80
    wn = matsubara(w.beta, 64)
    rng = np.random.default_rng(5)
    gbar = rng.normal(size=(2, 64)) + 1j * rng.normal(size=(2, 64))
    e0bar = 0.7
    h, psi, e0 = _ground_state(ctx, m, sec)
    grad, G, st = h.grad_green(psi, e0, chains, nit, wn, gbar, params, e0bar=e0bar, cg_tol=1e-12)
    assert st["reverse_steps"] == 2 * nit and st["cg_iterations"] > 0 and st["cg_residual"] <= 1e-12
    fd = np.array([(_loss(ctx, edk.perturb(m, p, H_FD), sec, chains, nit, wn, gbar, e0bar) -
                    _loss(ctx, edk.perturb(m, p, -H_FD), sec, chains, nit, wn, gbar, e0bar)) / (2 * H_FD)
                   for p in params])
    assert np.abs(grad - fd).max() <= 1e-5 * np.abs(fd).max(), (grad, fd)


def test_autograd_function_matches_the_direct_vjp(ctx):
    w = workload("c1")
    m = w.model
    wn = matsubara(w.beta, 32)
    prob = GreenProblem(ctx=ctx, model=m, params=edk.star_params(m), sector=(4, 4),
                        chains=[(0, 1, True), (0, 1, False)], nitergreen=60, wn=wn)
    theta = torch.tensor(prob.values(), requires_grad=True)
    e0, G = ImpurityGreen.apply(theta, prob)
    loss = 0.3 * e0 + (G.real ** 2).sum() - G.imag.sum()
    loss.backward()
    # the same cotangents through the C-ABI
    Gd = G.detach().numpy()
    gbar = 2 * Gd.real - 1j * np.ones_like(Gd.real)
    h, psi, e0v = _ground_state(ctx, m, (4, 4))
    ref, _, _ = h.grad_green(psi, e0v, prob.chains, 60, wn, gbar, prob.params, e0bar=0.3)
    assert np.abs(theta.grad.numpy() - ref).max() <= 1e-8 * np.abs(ref).max()


def _oracle_loss(m, sec, chains, nit, wn, gbar, e0bar):
    """E0 and the chains' G from the oracle alone: the exact ground state (dense
    diagonalisation of the sector) and the oracle's FP64 compute_dynamic."""
    ho = O.OracleH(m, *sec)
    E, V = np.linalg.eigh(ho.dense())
    e0, psi = float(E[0]), V[:, 0]
    val = e0bar * e0
    for c, (site, spin, dag) in enumerate(chains):
        phi, ts = O.apply_c(m, *sec, site, spin, dag, psi)
        G, _, _ = O.green_chain(O.OracleH(m, *ts), phi, nit, e0, 1 if dag else 2, wn, cutoff_dynamic=0.0)
        val += float(np.sum((np.conj(gbar[c]) * G).real))
    return val


def test_grad_green_against_the_oracle_fp64_gradient(ctx):
    """The device adjoint of E0 + G (one-orbital star, ns = 6, sector (3,3)) against
    an FP64 reference gradient that involves no device code: central differences
    (h = 1e-5) of the oracle's own solve (dense ground state, compute_dynamic
    chains of 60 steps, 32 Matsubara points).  Bound 1e-6 of the largest
    component."""
    rng = np.random.default_rng(9)
    m = star_model(-0.8, 2.0, rng.uniform(-1, 1, 5), rng.uniform(0.2, 0.6, 5))
    sec = (3, 3)
    params = edk.star_params(m)
    chains = [(0, 0, True), (0, 0, False), (0, 1, True)]
    nit = 60
    wn = matsubara(30.0, 32)
    gbar = rng.normal(size=(3, 32)) + 1j * rng.normal(size=(3, 32))
    e0bar = 0.4
    h, psi, e0 = _ground_state(ctx, m, sec)
    grad, G, st = h.grad_green(psi, e0, chains, nit, wn, gbar, params, e0bar=e0bar, cg_tol=1e-13)
    ref = np.array([(_oracle_loss(edk.perturb(m, p, H_FD), sec, chains, nit, wn, gbar, e0bar) -
                     _oracle_loss(edk.perturb(m, p, -H_FD), sec, chains, nit, wn, gbar, e0bar)) / (2 * H_FD)
                    for p in params])
    assert np.abs(grad - ref).max() <= 1e-6 * np.abs(ref).max(), (grad, ref)
