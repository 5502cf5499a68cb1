"""Bath fit (hybrid2bath path): the Nambu hybridisation of a star bath, the
diff_correl distance, its exact gradient against central differences, and the
minimiser recovering a bath from its own hybridisation."""
import numpy as np
import pytest

from ed_solver_b200.bathfit import (StarBath, distance, distance_and_grad, fit_hybrid, nambu_hybrid)
from ed_solver_b200.model import matsubara


def _bath(pairing=False, seed=0):
    rng = np.random.default_rng(seed)
    nb, nc = 4, 1
    eps = rng.uniform(-1.5, 1.5, nb)
    V = rng.uniform(0.2, 0.6, (nb, nc))
    P = rng.uniform(0.05, 0.3, nb) if pairing else None
    return StarBath(eps, V, P)


def test_normal_bath_hybridisation_blocks():
    b = _bath()
    wn = matsubara(20.0, 16)
    D = nambu_hybrid(b, wn)
    up = np.array([np.sum(b.V[:, 0] ** 2 / (1j * w - b.eps)) for w in wn])
    assert np.allclose(D[:, 0, 0], up, atol=1e-14)
    assert np.allclose(D[:, 1, 1], -np.conj(up), atol=1e-14)
    assert np.abs(D[:, 0, 1]).max() == 0.0


def test_distance_formula():
    b, b2 = _bath(seed=1), _bath(seed=2)
    wn = matsubara(20.0, 32)
    D1, D2 = nambu_hybrid(b, wn), nambu_hybrid(b2, wn)
    w = 1.0 / (np.abs(wn - wn[0]) + 0.01) ** 0.5
    ref = sum(w[n] * (np.abs(D2[n] - D1[n]) ** 2).sum() for n in range(32)) / (32 * 4)
    assert distance(D1, D2, wn) == pytest.approx(ref, rel=1e-13)
    assert distance_and_grad(b, D2, wn)[0] == pytest.approx(ref, rel=1e-12)


@pytest.mark.parametrize("pairing", [False, True])
def test_gradient_against_central_differences(pairing):
    b = _bath(pairing, seed=3)
    target = nambu_hybrid(_bath(pairing, seed=4), matsubara(20.0, 40))
    wn = matsubara(20.0, 40)
    f, g = distance_and_grad(b, target, wn)
    x = b.vec()
    h = 1e-6
    for i in range(len(x)):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (distance_and_grad(b.with_vec(xp), target, wn)[0] - distance_and_grad(b.with_vec(xm), target, wn)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-6 * max(1.0, abs(fd)), (i, g[i], fd)


@pytest.mark.parametrize("pairing", [False, True])
def test_fit_recovers_a_bath_from_its_hybridisation(pairing):
    # well separated levels: near-degenerate poles are not resolved by any fit
    truth = StarBath(np.array([-1.2, -0.3, 0.5, 1.3]), np.array([[0.3], [0.45], [0.25], [0.4]]),
                     np.array([0.1, 0.2, 0.15, 0.05]) if pairing else None)
    wn = matsubara(30.0, 100)
    target = nambu_hybrid(truth, wn)
    start = StarBath(truth.eps + 0.15, truth.V * 0.8, None if truth.P is None else truth.P * 1.5)
    d0 = distance(nambu_hybrid(start, wn), target, wn)
    fitted, d, it = fit_hybrid(start, target, wn, niter=200, dist_max=1e-14)
    assert d < 1e-12 < d0
    o = np.argsort(fitted.eps)
    assert np.allclose(fitted.eps[o], np.sort(truth.eps), atol=1e-4)
    assert np.allclose(np.abs(fitted.V[o]), np.abs(truth.V[np.argsort(truth.eps)]), atol=1e-4)


def _deck_2b():
    """The hybridisation the reference's two-orbital test deck fits its bath to
    (test/2b/delta1.inp, fixture written by tests/golden/make_golden.py), in
    the Nambu form of bath2hybrid: diag(D11, D22, -conj D11, -conj D22)."""
    import os
    d = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "delta_2b.txt"))
    wn = d[:, 0]
    d11, d22 = d[:, 1] + 1j * d[:, 2], d[:, 3] + 1j * d[:, 4]
    D = np.zeros((len(wn), 4, 4), complex)
    D[:, 0, 0], D[:, 1, 1] = d11, d22
    D[:, 2, 2], D[:, 3, 3] = -np.conj(d11), -np.conj(d22)
    return wn, D


def fit_deck_2b():
    """hybrid2bath on the test/2b deck with its fit options (test/2b/ED/ED.in:
    fit_nw=200, fit_weight_power=1, fit_shift=0, weight_expo=2, dist_max=1e-12):
    one bath level per orbital, started away from the answer."""
    wn, D = _deck_2b()
    b0 = StarBath(np.array([0.5, -0.4]), np.array([[0.5, 0.0], [0.0, 0.7]]))
    return fit_hybrid(b0, D, wn, fit_nw=200, niter=400, dist_max=1e-12, fit_shift=0.0, power=1.0)


def test_fit_recovers_the_2b_deck_bath():
    """The deck's hybridisation is analytic, V^2 = 0.2 and 0.3 at level 0
    (test/2b/test.py): the fit recovers that bath."""
    b, d, it = fit_deck_2b()
    assert d < 1e-12
    assert np.abs(b.eps).max() < 1e-5
    assert abs(b.V[0, 0] ** 2 - 0.2) < 1e-6 and abs(b.V[1, 1] ** 2 - 0.3) < 1e-6
