"""The bath fit closing the loop through the device solver: the bath is fitted
so that the impurity G of the ground state matches a target G produced by the
solver at known bath parameters; the gradients come from edk_grad_green."""
import numpy as np
import pytest

from ed_solver_b200 import bathfit, edk
from ed_solver_b200.model import matsubara, star_model

pytestmark = pytest.mark.gpu


def test_fit_green_recovers_the_bath(ctx):
    truth = star_model(-1.0, 2.0, [-0.9, 0.1, 0.8], [0.45, 0.3, 0.5])
    wn = matsubara(20.0, 48)
    sector = (2, 2)
    h = edk.Hamiltonian(ctx, truth, *sector)
    r = h.lanczos_e0("f64", tolerance=1e-13, residual_tol=1e-11)
    psi = h.lanczos_gs(r["vecp"][0])
    G = 0.0
    for dag in (True, False):
        phi, ts = h.apply_c(psi, 0, 0, dag)
        g, *_ = edk.Hamiltonian(ctx, truth, *ts).green_chain(phi, 200, r["E"][0], 1 if dag else 2, wn,
                                                               cutoff_dynamic=0.0)
        G = G + g
    start = bathfit.StarBath(np.array([-0.8, 0.2, 0.9]), np.array([[0.4], [0.35], [0.45]])).apply(truth)
    fitted, hist = bathfit.fit_green(ctx, start, G, sector, wn, nitergreen=200, steps=40)
    # G of one sector does not fix the bath uniquely: the fit is judged by G
    assert hist[-1] < 1e-3 * hist[0]


def test_fit_then_solve_reproduces_g_bm(ctx):
    """The reference's own test/2b loop closed on the device: fit the bath to
    the deck's hybridisation (fixture of test/2b/delta1.inp, fit run to
    convergence), build the impurity model of the deck with it (two orbitals,
    eps = -5, U = 10, U' = 2, J = 0), solve at beta = 50, and compare G11 and
    G22 with the reference's output test/2b/bm/g_bm (2e-8)."""
    import math
    import os
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from test_bathfit import _deck_2b
    from ed_solver_b200.bathfit import StarBath, fit_hybrid
    from ed_solver_b200.model import star_model
    wn, D = _deck_2b()
    b0 = StarBath(np.array([0.5, -0.4]), np.array([[0.5, 0.0], [0.0, 0.7]]))
    bath, d, _ = fit_hybrid(b0, D, wn, fit_nw=200, niter=400, dist_max=1e-20, fit_shift=0.0, power=1.0)
    assert d < 1e-20
    m0 = star_model(-5.0, 10.0, [0.0, 0.0], [math.sqrt(0.2), math.sqrt(0.3)], orbital_of_bath=[0, 1], nc=2,
                    Uprime=2.0, J=0.0, cutoff=1e-8)
    m = bath.apply(m0)
    g = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "g_bm_2b.txt"))
    secs = [(a, b) for a in range(5) for b in range(5)]
    r = edk.solve(ctx, m, secs, 50.0, len(g), dtype="f64", neigen=40, tolerance=1e-13, demax0=50.0,
                  nitergreen=400, spins=(0,), pairs=[(0, 0), (1, 1)])
    assert np.abs(r["G"][0, 0] - (g[:, 1] + 1j * g[:, 2])).max() < 2e-8
    assert np.abs(r["G"][0, 1] - (g[:, 3] + 1j * g[:, 4])).max() < 2e-8
