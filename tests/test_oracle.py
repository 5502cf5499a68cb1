"""The CPU oracle against an independent dense build, analytic limits and the
reference's own golden output (test/2b/bm/g_bm)."""
import math
import os

import numpy as np
import pytest

import oracle as O
from ed_solver_b200.model import star_model, matsubara, workload

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "g_bm_2b.txt")


def _models():
    rng = np.random.default_rng(11)
    m1 = star_model(-0.7, 2.0, rng.uniform(-1, 1, 4), rng.uniform(0.2, 0.6, 4))
    m2 = star_model(-1.0, 3.0, rng.uniform(-1, 1, 3), rng.uniform(0.2, 0.6, 3), orbital_of_bath=[0, 1, 1],
                    nc=2, J=0.5)
    m2.ec[:, 0, 1] = m2.ec[:, 1, 0] = 0.3
    m2.eb[:, 0, 2] = m2.eb[:, 2, 0] = 0.25
    return [m1, m2]


@pytest.mark.parametrize("mi", [0, 1])
def test_hmult_matches_second_quantised_build(mi):
    m = _models()[mi]
    for nu, nd in [(2, 2), (3, 2), (1, 3), (0, 2), (m.ns, 1)]:
        h = O.OracleH(m, nu, nd)
        A = h.dense()
        B = O.dense_sector_h(m, nu, nd)
        assert np.abs(A - B).max() < 1e-14
        assert np.abs(A - A.T).max() == 0.0


def test_split_form_is_the_matvec_without_the_jj_terms():
    """The restatement of HAIMupdo_multr_split (transposes, no -JJ terms)
    equals the restatement of HAIMupdo_multr with JJ set to zero, bit for bit,
    on a two-orbital model without Hund spin-flip terms; on a single-orbital
    model it equals the plain matvec; with |Jhund| > 1e-5 the reference STOPs
    (None)."""
    import dataclasses
    m = _models()[1]
    m.jhund = 0.0
    m0 = dataclasses.replace(m, jj=np.zeros_like(m.jj))
    rng = np.random.default_rng(4)
    for nu, nd in [(2, 2), (3, 2), (1, 3), (0, 2)]:
        x = rng.normal(size=O.OracleH(m, nu, nd).dim)
        ys = O.OracleH(m, nu, nd).hmult_split(x)
        assert np.array_equal(ys, O.OracleH(m0, nu, nd).hmult(x))
    h = O.OracleH(m, 2, 2)
    x = rng.normal(size=h.dim)
    assert not np.array_equal(h.hmult_split(x), h.hmult(x))
    m1 = _models()[0]
    h = O.OracleH(m1, 2, 3)
    x = rng.normal(size=h.dim)
    assert np.array_equal(h.hmult_split(x), h.hmult(x))
    assert O.OracleH(_models()[1], 2, 2).hmult_split(np.zeros(O.OracleH(_models()[1], 2, 2).dim)) is None


def test_tridiagonal_solver_against_numpy():
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 40):
        d = rng.normal(size=n)
        e = rng.uniform(0.1, 1.0, size=max(n - 1, 1))[:n - 1]
        w, z = O.tridiag_eig(d, e, vectors=True)
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        assert np.allclose(w, np.linalg.eigvalsh(T), atol=1e-12)
        assert np.allclose(T @ z, z * w, atol=1e-10)


def test_lanczos_e0_against_dense():
    m = _models()[1]
    h = O.OracleH(m, 3, 3)
    r = O.lanczos_e0(h, neigen=2, tolerance=1e-13)
    w = np.linalg.eigvalsh(h.dense())
    assert abs(r["E"][0] - w[0]) < 1e-10
    psi = O.lanczos_gs(h, r["vecp"][0])
    assert np.linalg.norm(h.hmult(psi) - w[0] * psi) < 1e-6


def test_noninteracting_limit_is_the_exact_resolvent():
    """U=0: G(iw) = 1/(iw - eps - sum V^2/(iw - eps_k)) for a single orbital."""
    rng = np.random.default_rng(5)
    eb, v = rng.uniform(-1, 1, 5), rng.uniform(0.2, 0.6, 5)
    m = star_model(-0.3, 0.0, eb, v)
    beta, nw = 30.0, 64
    wn = matsubara(beta, nw)
    gs, e0, z = O.ground_states(m, [(a, b) for a in range(7) for b in range(7)], beta, 200.0, neigen=8)
    G = O.green_impurity(m, gs, beta, nw, 60)[(0, 0)]
    iw = 1j * wn
    G0 = 1.0 / (iw - (-0.3) - (v[None, :] ** 2 / (iw[:, None] - eb[None, :])).sum(1))
    assert np.abs(G - G0).max() < 1e-6


def test_atomic_limit():
    """V=0, single site at half filling: G = 0.5/(iw - U/2) + 0.5/(iw + U/2) for eps=-U/2."""
    U, beta = 2.0, 40.0
    m = star_model(-U / 2, U, [0.1], [0.0])
    wn = matsubara(beta, 32)
    secs = [(a, b) for a in range(3) for b in range(3)]
    G = O.lehmann_green(m, secs, beta, wn)
    iw = 1j * wn
    assert np.abs(G - (0.5 / (iw - U / 2) + 0.5 / (iw + U / 2))).max() < 1e-8


def test_reference_golden_g_bm():
    """The two-orbital test of the reference (test/2b): G11 and G22 at beta=50."""
    g = np.loadtxt(GOLDEN)
    m = star_model(-5.0, 10.0, [0.0, 0.0], [math.sqrt(0.2), math.sqrt(0.3)], orbital_of_bath=[0, 1], nc=2,
                   Uprime=2.0, J=0.0, cutoff=1e-8)
    secs = [(a, b) for a in range(5) for b in range(5)]
    gs, e0, z = O.ground_states(m, secs, 50.0, 50.0, neigen=40, tolerance=1e-13)
    G = O.green_impurity(m, gs, 50.0, len(g), 400, pairs=[(0, 0), (1, 1), (0, 1)])
    assert np.abs(G[(0, 0)] - (g[:, 1] + 1j * g[:, 2])).max() < 2e-8
    assert np.abs(G[(1, 1)] - (g[:, 3] + 1j * g[:, 4])).max() < 2e-8
    assert np.abs(G[(0, 1)]).max() < 1e-12


def _model_2b():
    return star_model(-5.0, 10.0, [0.0, 0.0], [math.sqrt(0.2), math.sqrt(0.3)], orbital_of_bath=[0, 1], nc=2,
                      Uprime=2.0, J=0.0, cutoff=1e-8)


def test_reference_golden_g_bm_through_the_lehmann_branch():
    """Every sector of the test/2b model has at most 36 states, so the
    reference took compute_dynamic_full_ed there.  Its vertex-dump run keeps
    every eigenstate (dEmax0=10000, Neigen=500, test/2b/test.py:200), where the
    Lehmann sum is exact: the oracle's restatement of that branch reproduces
    G11 and G22."""
    g = np.loadtxt(GOLDEN)
    m = _model_2b()
    secs = [(a, b) for a in range(5) for b in range(5)]
    gs, e0, z = O.ground_states(m, secs, 50.0, 10000.0, neigen=500, tolerance=1e-13)
    assert len(gs) == 256
    G = O.green_impurity(m, gs, 50.0, len(g), 400, pairs=[(0, 0), (1, 1), (0, 1)],
                         reference_small_sectors=True)
    assert np.abs(G[(0, 0)] - (g[:, 1] + 1j * g[:, 2])).max() < 2e-8
    assert np.abs(G[(1, 1)] - (g[:, 3] + 1j * g[:, 4])).max() < 2e-8


def test_lehmann_branch_differs_from_the_continued_fraction_in_a_narrow_window():
    """With a narrow window (dEmax = 0.5) the Lehmann branch sums only the
    target-sector states the window kept, so it is not the exact G the
    continued fraction gives; zero when no target state is kept."""
    m = _model_2b()
    secs = [(a, b) for a in range(5) for b in range(5)]
    gs, e0, z = O.ground_states(m, secs, 50.0, 25.0, neigen=40, tolerance=1e-13)
    Gl = O.green_impurity(m, gs, 50.0, 64, 400, reference_small_sectors=True)[(0, 0)]
    Gc = O.green_impurity(m, gs, 50.0, 64, 400)[(0, 0)]
    assert np.abs(Gl - Gc).max() > 1e-3
    kept = {tuple(s["sector"]) for s in gs}
    wn = matsubara(50.0, 8)
    v, tsec = O.apply_c(m, *gs[0]["sector"], 0, 0, True, gs[0]["psi"])
    Gs = O.lehmann_small_sector(gs, tsec, v, gs[0]["E"], 1, wn)
    assert (tsec in kept) or np.all(Gs == 0)


def test_apply_c_is_a_signed_partial_permutation():
    m = _models()[1]
    rng = np.random.default_rng(2)
    h = O.OracleH(m, 2, 3)
    x = rng.normal(size=h.dim)
    for spin in (0, 1):
        for dag in (True, False):
            y, tsec = O.apply_c(m, 2, 3, 1, spin, dag, x)
            nz = np.abs(y) > 0
            assert set(np.round(np.abs(y[nz]), 12)) <= set(np.round(np.abs(x), 12))
            # c c+ + c+ c = 1 on the site: apply both orders and add
            if dag:
                y2, _ = O.apply_c(m, *tsec, 1, spin, False, y)
                z, _ = O.apply_c(m, 2, 3, 1, spin, False, x)
                z2, _ = O.apply_c(m, *( (1, 3) if spin == 0 else (2, 2)), 1, spin, True, z)
                assert np.allclose(y2 + z2, x)


def test_workload_shapes():
    assert O.binom(8, 4) ** 2 == 4900
    assert O.binom(14, 7) ** 2 == 11778624
    assert O.binom(16, 8) ** 2 == 165636900
    w = workload("c2")
    assert w.model.nc == 2 and w.model.nb == 8 and len(w.sectors) == 121
