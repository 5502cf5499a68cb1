"""The superconducting solve on Nambu sectors (sector scan, window, Nambu
Green functions through the device chains) against Lehmann sums over the
oracle's dense Nambu sectors."""
import math

import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import solver
from ed_solver_b200.model import matsubara, nambu_workload

pytestmark = pytest.mark.gpu


def _lehmann(m, beta, nw, demax0):
    """G_ab = sum_s w_s [ sum_m <s|b_a|m><m|b+_b|s>/(iw - (E_m - E_s)) + <s|b+_b|m><m|b_a|s>/(iw + (E_m - E_s)) ]."""
    ns2 = 2 * m.ns
    wn = matsubara(beta, nw)
    eig = {}
    for npart in range(ns2 + 1):
        eig[npart] = np.linalg.eigh(O.OracleSz(m, npart).dense())
    e0 = min(w[0] for w, _ in eig.values())
    demax = demax0 / beta
    states = [(n, k) for n, (w, _) in eig.items() for k in range(len(w)) if w[k] <= e0 + demax]
    z = sum(math.exp(-beta * (eig[n][0][k] - e0)) for n, k in states)

    def b_op(npart, orb, dagger, vec):
        nc = m.nc
        site, spin = (orb, 0) if orb < nc else (orb - nc, 1)
        # Nambu b+ on the hole orbital is the physical c of spin down
        return O.OracleSz(m, npart).apply_c(vec, site, spin, dagger if spin == 0 else not dagger)

    G = {}
    nc = m.nc
    for a in range(2 * nc):
        for b in range(2 * nc):
            g = np.zeros(nw, complex)
            for n, k in states:
                ws = math.exp(-beta * (eig[n][0][k] - e0)) / z
                psi = eig[n][1][:, k]
                Es = eig[n][0][k]
                if n + 1 <= ns2:
                    pa, _ = b_op(n, a, True, psi)
                    pb, _ = b_op(n, b, True, psi)
                    W, V = eig[n + 1]
                    amp = (V.T @ pa) * (V.T @ pb)
                    g += np.array([np.sum(amp / (1j * w - (W - Es))) for w in wn]) * ws
                if n - 1 >= 0:
                    ha, _ = b_op(n, a, False, psi)
                    hb, _ = b_op(n, b, False, psi)
                    W, V = eig[n - 1]
                    amp = (V.T @ ha) * (V.T @ hb)
                    g += np.array([np.sum(amp / (1j * w + (W - Es))) for w in wn]) * ws
            G[(a, b)] = g
    return G, e0, len(states)


def test_nambu_green_functions_against_lehmann(ctx):
    # a window holding one state per sector (the ground states of npart = 3 and 5);
    # neigen = 1: plain Lanczos returns converged ghost copies of a state when asked for more,
    # as the reference's does
    m = nambu_workload(4)
    beta, nw, demax0 = 20.0, 16, 2.0
    hc = solver.HCacheSz(ctx, m)
    gs, e0, z, shift = solver.ground_states_sz(hc, range(0, 2 * m.ns + 1), beta, demax0, neigen=1, tolerance=1e-13)
    G = solver.green_nambu(hc, gs, beta, nw, nitergreen=200, cutoff_dynamic=0.0)
    Go, e0o, nstates = _lehmann(m, beta, nw, demax0)
    assert len(gs) == nstates
    assert abs(e0 - e0o) < 1e-11
    assert abs(shift - m.energy_shift) < 1e-14
    for key in [(0, 0), (1, 1), (0, 1)]:
        assert np.abs(G[key] - Go[key]).max() < 1e-7 * max(1.0, np.abs(Go[key]).max()), key
    # the pairing makes the anomalous function non-zero
    assert np.abs(Go[(0, 1)]).max() > 1e-3
    hc.close()


@pytest.mark.parametrize("spin", [0, 1])
def test_gnf_channel_against_oracle(ctx, spin):
    """compute_greenAB in the Nambu basis with A = the projected c of
    apply_Csz_N_updo and B = c (the GNF channel of correlations_dyn_stat.h:96):
    the device chains from edk_apply_csz_ab's symmetric combinations against the
    oracle's restatement on the same states (1e-9)."""
    m = nambu_workload(5)
    beta, nw, demax0 = 20.0, 32, 2.0
    hc = solver.HCacheSz(ctx, m)
    gs, e0, z, shift = solver.ground_states_sz(hc, range(0, 2 * m.ns + 1), beta, demax0, neigen=1, tolerance=1e-13)
    G = solver.green_ab_nambu(hc, gs, beta, nw, 200, spin=spin, cutoff_dynamic=0.0)[(0, 0)]
    gso = [dict(npart=s["npart"], E=s["E"], psi=s["psi"].double().cpu().numpy(), boltz=s["boltz"]) for s in gs]
    Go = O.green_ab_nambu(m, gso, beta, nw, 200, spin=spin, cutoff_dynamic=0.0)[(0, 0)]
    assert np.abs(G - Go).max() < 1e-9 * max(1.0, np.abs(Go).max())
    assert np.abs(Go).max() > 1e-3
    hc.close()
