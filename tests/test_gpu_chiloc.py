"""chi~_loc on the device against the reference's own chi_tilde_loc_ (its C++
source compiled unmodified into oracle/_ref): random sector data at every
boundary case of (nup, ndn), frequency triples that take the
vanishing-denominator branches, and the physical vertex of a small model
built on the device (full ED + c+ matrices) against the one the oracle builds.
Tolerance: |d| <= 1e-9 max|chi| of the batch (FP64, another summation order)."""
import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk, vertex
from ed_solver_b200.model import star_model

pytestmark = pytest.mark.gpu

SITES = 3


def _need_ref():
    if O.ref_chiloc_lib() is None:
        pytest.fail("oracle/_ref/libchiloc_ref.so missing: build it with `make -C oracle ref` where the "
                    "reference sources are present")


def _random_inputs(rng, nup, ndn, degenerate):
    from math import comb
    E = [None] * 11
    for q, (du, dd) in enumerate(O.CHILOC_SECTORS):
        nu, nd = nup + du, ndn + dd
        if 0 <= nu <= SITES and 0 <= nd <= SITES:
            d = comb(SITES, nu) * comb(SITES, nd)
            e = np.round(rng.uniform(-2, 2, d), 1) if degenerate else rng.uniform(-2, 2, d)
            E[q] = np.sort(e)
    M = [None] * 14
    for m, (t, s, _) in enumerate(O.CHILOC_MATRICES):
        if E[t] is not None and E[s] is not None:
            x = rng.standard_normal((len(E[t]), len(E[s])))
            x[rng.random(x.shape) < 0.3] = 0.0
            M[m] = x
    return E, M


def _triples(beta):
    nu = lambda n: 1j * (2 * n + 1) * np.pi / beta
    return [
        (nu(0), nu(1), nu(2)),
        (nu(0), nu(1), -nu(1)),          # w2 + w3 = 0
        (nu(2), -nu(2), nu(0)),          # w1 + w2 = 0
        (nu(-3), nu(1), nu(0)),
        (nu(1), nu(-1), -nu(-1)),
    ]


@pytest.fixture(params=[False, True], ids=["split-kernel", "per-element-kernel"])
def kernel(request):
    edk.chiloc_set_kernel(request.param)
    yield request.param
    edk.chiloc_set_kernel(False)


@pytest.mark.parametrize("nup,ndn", [(1, 1), (0, 0), (SITES, SITES), (0, SITES), (SITES, 0), (1, 2), (2, 1),
                                     (2, 2), (1, SITES - 1)])
@pytest.mark.parametrize("degenerate", [False, True])
def test_random_sector_data_against_reference(ctx, kernel, nup, ndn, degenerate):
    _need_ref()
    rng = np.random.default_rng(100 * nup + 10 * ndn + degenerate)
    E, M = _random_inputs(rng, nup, ndn, degenerate)
    beta, eps = 7.0, 1e-5
    es = np.concatenate([e for e in E if e is not None])
    Z, gs = float(np.exp(-beta * (es - es.min())).sum()), float(es.min())
    w = _triples(beta)
    pd, pu = edk.chiloc(ctx, E, M, w, beta, Z, gs, SITES, nup, ndn, phi_eps=eps)
    rd = np.array([O.ref_chiloc(1, t, eps, beta, Z, gs, SITES, nup, ndn, E, M)[0] for t in w])
    ru = np.array([O.ref_chiloc(2, t, eps, beta, Z, gs, SITES, nup, ndn, E, M)[1] for t in w])
    assert np.abs(pd - rd).max() <= 1e-9 * max(1e-30, np.abs(rd).max())
    assert np.abs(pu - ru).max() <= 1e-9 * max(1e-30, np.abs(ru).max())


def test_full_ed_matches_dense_diagonalisation(ctx):
    m = star_model(-1.0, 2.0, [-0.5, 0.4, 0.9], [0.4, 0.3, 0.5])
    for nu, nd in [(2, 2), (1, 3), (0, 4)]:
        h = edk.Hamiltonian(ctx, m, nu, nd)
        E, V = h.full_ed()
        Hd = O.OracleH(m, nu, nd).dense()
        assert np.abs(E - np.linalg.eigvalsh(Hd)).max() < 1e-12 * max(1.0, np.abs(E).max())
        assert np.abs(Hd @ V - V * E).max() < 1e-10
        assert np.abs(V.T @ V - np.eye(h.dim)).max() < 1e-12


def test_physical_vertex_against_reference(ctx, kernel):
    """ns=4 star model, sector (2,2): device full ED + device c+ matrices +
    device chi~ against the oracle's dense ED + c+ matrices + the reference's
    chi_tilde_loc_ (eigenvector signs and degenerate rotations differ between
    the two diagonalisations; chi~ does not depend on them)."""
    _need_ref()
    m = star_model(-1.0, 2.0, [-0.6, 0.2, 0.7], [0.45, 0.3, 0.5])
    beta, eps = 8.0, 1e-5
    Ed, Md = vertex.vertex_inputs(ctx, m, 2, 2)
    Eo, Mo, _ = O.chiloc_inputs(m, 2, 2)
    Z, gs = vertex.partition(Eo, beta)
    w = _triples(beta)
    pd, pu = edk.chiloc(ctx, Ed, Md, w, beta, Z, gs, m.ns, 2, 2, phi_eps=eps)
    rd = np.array([O.ref_chiloc(1, t, eps, beta, Z, gs, m.ns, 2, 2, Eo, Mo)[0] for t in w])
    ru = np.array([O.ref_chiloc(2, t, eps, beta, Z, gs, m.ns, 2, 2, Eo, Mo)[1] for t in w])
    assert np.abs(pd - rd).max() <= 1e-9 * np.abs(rd).max()
    assert np.abs(pu - ru).max() <= 1e-9 * np.abs(ru).max()
