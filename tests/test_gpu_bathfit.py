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
