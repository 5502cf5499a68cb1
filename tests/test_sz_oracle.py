"""The Nambu (Sz) restatement of HAIMsz (oracle/edk_oracle.c) pinned on the CPU:

* against an independent build of the physical Hamiltonian with pairing terms
  on the fixed-Sz subspace (explicit fermion operators, another orbital order):
  equal spectra after the energy shift, and equal Lehmann Green functions for
  c+ of either spin;
* U = 0: the sector's spectrum is the free-fermion one of the Nambu one-body
  matrix (lowest level = sum of the npart lowest one-particle levels);
* no pairing: the Nambu sector is the direct sum of the (N_up, N_dn) sectors
  with N_up + ns - N_dn = npart, whose oracle is pinned to the reference's
  golden output;
* the two term orders (tabulated HAIMsz_multr, HAIMsz_mult_fly_r) agree to
  rounding, and the tabulated CSR is the sequential one."""
import itertools
import math

import numpy as np
import pytest

import oracle as O
from ed_solver_b200.model import NambuModel, matsubara, nambu_star_model, nambu_workload, star_model


def _two_orbital(pvbc=False, on_fly=False):
    rng = np.random.default_rng(11)
    base = star_model([-1.2, -0.8], 2.5, rng.uniform(-1.5, 1.5, 3), rng.uniform(0.2, 0.5, 3),
                      orbital_of_bath=[0, 1, 1], nc=2, Uprime=1.3, J=0.0, cutoff=1e-8)
    base.ec[0, 0, 1] = base.ec[0, 1, 0] = 0.15
    base.ec[1, 0, 1] = base.ec[1, 1, 0] = 0.15
    base.eb[0, 0, 2] = base.eb[0, 2, 0] = 0.07
    base.eb[1, 0, 2] = base.eb[1, 2, 0] = 0.07
    pb = np.diag(rng.uniform(0.1, 0.3, 3))
    pb[0, 1] = pb[1, 0] = 0.05
    pv = None
    if pvbc:
        pv = np.zeros((2, 3, 2))
        pv[0, 0, 0] = 0.11
        pv[1, 2, 1] = -0.09
    return NambuModel(base, pb, pv, on_fly)


MODELS = {
    "star5": lambda: nambu_workload(5),
    "star5_fly": lambda: nambu_workload(5, on_fly=True),
    "two_orbital": lambda: _two_orbital(),
    "two_orbital_pvbc_fly": lambda: _two_orbital(pvbc=True, on_fly=True),
}


@pytest.mark.parametrize("name", sorted(MODELS))
def test_nambu_spectrum_equals_physical_with_pairing(name):
    m = MODELS[name]()
    for npart in range(0, 2 * m.ns + 1):
        oh = O.OracleSz(m, npart)
        assert oh.dim == O.binom(2 * m.ns, npart)
        Hn = oh.dense()
        assert np.array_equal(Hn, Hn.T)
        en = np.linalg.eigvalsh(Hn) + oh.shift
        ep = np.linalg.eigvalsh(O.dense_physical_sz(m, npart))
        assert np.abs(en - ep).max() < 1e-12 * max(1.0, np.abs(ep).max())


def test_energy_shift_is_the_down_diagonal():
    m = _two_orbital()
    assert O.OracleSz(m, 3).shift == pytest.approx(m.energy_shift, abs=1e-15)


def test_free_fermion_limit():
    m = nambu_workload(5)
    m.base.u[:] = 0.0
    eps = np.linalg.eigvalsh(O.nambu_one_body(m))
    for npart in (3, 5, 7):
        oh = O.OracleSz(m, npart)
        e = np.linalg.eigvalsh(oh.dense())
        assert e[0] == pytest.approx(eps[:npart].sum(), abs=1e-12)
        free = np.sort([sum(c) for c in itertools.combinations(eps, npart)])
        assert np.abs(e - free).max() < 1e-12


def test_no_pairing_is_the_direct_sum_of_updo_sectors():
    m = nambu_workload(5)
    m.pb[:] = 0.0
    ns = m.ns
    for npart in (3, 5, 6):
        e = np.linalg.eigvalsh(O.OracleSz(m, npart).dense()) + m.energy_shift
        parts = []
        for nup in range(ns + 1):
            ndn = nup + ns - npart
            if 0 <= ndn <= ns:
                parts.append(np.linalg.eigvalsh(O.OracleH(m.base, nup, ndn).dense()))
        ref = np.sort(np.concatenate(parts))
        assert np.abs(e - ref).max() < 1e-12


@pytest.mark.parametrize("name", ["star5", "two_orbital"])
def test_term_orders_agree(name):
    m = MODELS[name]()
    m_fly = NambuModel(m.base, m.pb, m.pvbc, on_fly=True)
    m_tab = NambuModel(m.base, m.pb, m.pvbc, on_fly=False)
    rng = np.random.default_rng(3)
    for npart in (m.ns - 1, m.ns):
        a, b = O.OracleSz(m_tab, npart), O.OracleSz(m_fly, npart)
        x = rng.standard_normal(a.dim)
        assert np.abs(a.hmult(x) - b.hmult(x)).max() < 1e-13 * np.abs(x).sum()


def test_tabulated_operator_is_sequential_csr():
    m = _two_orbital(pvbc=True)
    oh = O.OracleSz(m, m.ns)
    st, q, dg, ptr, tgt, val = oh.table()
    assert np.all(np.diff(st.astype(np.int64)) > 0)
    assert all(O.colex_rank(int(s)) == i for i, s in enumerate(st))
    x = np.random.default_rng(5).standard_normal(oh.dim)
    y = np.empty(oh.dim)
    for i in range(oh.dim):
        v = q[i] * x[i]
        v = v + dg[i] * x[i]
        for e in range(ptr[i], ptr[i + 1]):
            v = v + val[e] * x[tgt[e]]
        y[i] = v
    assert np.array_equal(y, oh.hmult(x))


def _lehmann_particle(E0, psi, Et, V, opm_psi, wn):
    """sum_m |<m|op|psi>|^2 / (i wn - (E_m - E0)) from eigenpairs (Et, V) of the target."""
    amp = V.T @ opm_psi
    return np.array([np.sum(amp ** 2 / (1j * w - (Et - E0))) for w in wn])


@pytest.mark.parametrize("spin", [0, 1])
def test_apply_c_green_function_equals_physical(spin):
    """Lehmann G of c+_{0,spin} from the sector ground state: Nambu (apply_Csz_updo)
    against the physical build (c+ as an explicit operator)."""
    m = _two_orbital()
    ns = m.ns
    npart = ns
    wn = np.array([0.3, 1.1, 2.7])
    oh = O.OracleSz(m, npart)
    E, V = np.linalg.eigh(oh.dense())
    psi = V[:, 0]
    phi, npt = oh.apply_c(psi, 0, spin, True)
    ot = O.OracleSz(m, npt)
    Et, Vt = np.linalg.eigh(ot.dense())
    Gn = _lehmann_particle(E[0], psi, Et, Vt, phi, wn)
    # physical side: c+_{imp 0, spin} between the Sz subspaces
    Hp = O.dense_physical_sz(m, npart)
    Ep, Vp = np.linalg.eigh(Hp)
    Hq = O.dense_physical_sz(m, npt)
    Eq, Vq = np.linalg.eigh(Hq)
    no = 2 * ns
    idx = lambda o, s: 2 * o + s

    def sz_states(npa):
        return [st for st in range(1 << no)
                if sum((st >> idx(o, 0)) & 1 for o in range(ns)) - sum((st >> idx(o, 1)) & 1 for o in range(ns))
                == npa - ns]
    src, tgt = sz_states(npart), sz_states(npt)
    rk = {s: i for i, s in enumerate(tgt)}
    Cmat = np.zeros((len(tgt), len(src)))
    p = idx(m.nb + 0, spin)
    for j, s in enumerate(src):
        if (s >> p) & 1:
            continue
        sg = -1 if bin(s & ((1 << p) - 1)).count("1") & 1 else 1
        Cmat[rk[s | (1 << p)], j] = sg
    assert Ep[0] == pytest.approx(E[0] + m.energy_shift, abs=1e-12)
    Gp = _lehmann_particle(Ep[0], Vp[:, 0], Eq, Vq, Cmat @ Vp[:, 0], wn)
    assert np.abs(Gn - Gp).max() < 1e-12


def test_projected_operator_splits_the_plain_one():
    """apply_Csz_N_updo(up) + the complementary projection = apply_Csz_updo(up)."""
    m = nambu_workload(4)
    oh = O.OracleSz(m, 4)
    x = np.random.default_rng(2).standard_normal(oh.dim)
    full, npt = oh.apply_c(x, 0, 0, True)
    proj, _ = oh.apply_c(x, 0, 0, True, projected=True)
    # the projected part lives on states whose hole orbital of site 0 is empty
    ot = O.OracleSz(m, npt)
    st = ot.table()[0]
    hole = np.array([(int(s) >> (m.ns + m.nb)) & 1 for s in st])
    assert np.array_equal(proj, np.where(hole == 0, full, 0.0))


def _ab_lehmann(m, beta, nw, demax0, proj_a, proj_b, spin=0):
    """G_AB = sum_s w_s [ sum_m <s|A|m><m|B+|s>/(iw - (E_m - E_s)) + <s|B+|m><m|A|s>/(iw + (E_m - E_s)) ]
    over the dense Nambu sectors, for A = (projected) c of spin `spin` on site 0, B likewise."""
    wn = matsubara(beta, nw)
    eig = {n: np.linalg.eigh(O.OracleSz(m, n).dense()) for n in range(2 * m.ns + 1)}
    e0 = min(w[0] for w, _ in eig.values())
    states = [(n, k) for n, (w, _) in eig.items() for k in range(len(w)) if w[k] <= e0 + demax0 / beta]
    z = sum(math.exp(-beta * (eig[n][0][k] - e0)) for n, k in states)
    g = np.zeros(nw, complex)
    for n, k in states:
        ws = math.exp(-beta * (eig[n][0][k] - e0)) / z
        psi, Es = eig[n][1][:, k], eig[n][0][k]
        for dagger, sgn in ((True, -1.0), (False, 1.0)):
            try:
                pa, npt = O.OracleSz(m, n).apply_c(psi, 0, spin, dagger, projected=proj_a)
                pb, _ = O.OracleSz(m, n).apply_c(psi, 0, spin, dagger, projected=proj_b)
            except ValueError:
                continue
            W, V = eig[npt]
            amp = (V.T @ pa) * (V.T @ pb)
            g += np.array([np.sum(amp / (1j * w + sgn * (W - Es))) for w in wn]) * ws
    return g, states, eig, e0, z


def test_green_ab_nambu_against_lehmann():
    """The oracle's compute_greenAB restatement (symmetric combinations, then
    (G_{A+B} - G_AA - G_BB)/2) equals the Lehmann sum <A ; B+> on the dense
    Nambu sectors of a 4-site superconducting model, for the GNF pair
    (A projected, B plain) and for A = B = c (where it is G itself)."""
    from ed_solver_b200.model import nambu_workload
    m = nambu_workload(4)
    beta, nw, demax0 = 20.0, 12, 2.0
    for proj_a, proj_b in ((True, False), (False, False)):
        g_ref, states, eig, e0, z = _ab_lehmann(m, beta, nw, demax0, proj_a, proj_b)
        gs = [dict(npart=n, E=float(eig[n][0][k]), psi=eig[n][1][:, k],
                   boltz=math.exp(-beta * (eig[n][0][k] - e0)) / z) for n, k in states]
        G = O.green_ab_nambu(m, gs, beta, nw, 200, spin=0, sites=[0], proj_a=proj_a, proj_b=proj_b,
                             cutoff_dynamic=0.0)[(0, 0)]
        assert np.abs(G - g_ref).max() < 1e-9 * max(1.0, np.abs(g_ref).max())
        assert np.abs(g_ref).max() > 1e-3
