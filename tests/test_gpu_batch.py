"""Batched Green chains (edk_green_batch) against the oracle's compute_dynamic.

The items are the chains compute_greenAA issues (green_class_computeAA.f90:105-126):
for several eigenstates, every impurity site, spin and particle/hole part.  The
model has Kanamori interactions with Hund spin-flip and pair-hopping terms, so
the generic per-block H*v (with the Hund gathers) is exercised.
"""
import numpy as np
import pytest
import torch

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import matsubara, workload

pytestmark = pytest.mark.gpu

NITER = 120


def _items(ctx, sectors):
    w = workload("c2")
    m = w.model
    wn = matsubara(w.beta, 128)
    items, Gref = [], {}
    hs = {}
    weights = [0.6, 0.3, 0.1]
    for si, (nup, ndn) in enumerate(sectors):
        ho = O.OracleH(m, nup, ndn)
        r = O.lanczos_e0(ho)
        psi = O.lanczos_gs(ho, r["vecp"][0])
        e0 = r["E"][0]
        for site in range(m.nc):
            for spin in (0, 1):
                for dag, iph in ((True, 1), (False, 2)):
                    phi, ts = O.apply_c(m, nup, ndn, site, spin, dag, psi)
                    if ts not in hs:
                        hs[ts] = edk.Hamiltonian(ctx, m, *ts)
                    Go, _, _ = O.green_chain(O.OracleH(m, *ts), phi, NITER, e0, iph, wn)
                    out = site * 2 + spin
                    Gref[out] = Gref.get(out, 0) + weights[si] * Go
                    items.append(dict(h=hs[ts], phi=phi, e0=e0, iph=iph, weight=weights[si], out=out))
    ref = np.array([Gref[o] for o in range(2 * m.nc)])
    return items, ref, wn, hs


@pytest.mark.parametrize("mode", [0, 1])
def test_green_batch_fp64_against_oracle(ctx, mode):
    items, ref, wn, hs = _items(ctx, [(5, 5), (4, 5), (5, 4)])
    chains = [dict(it, start=torch.tensor(it["phi"], device="cuda")) for it in items]
    G, st = edk.green_batch(ctx, chains, NITER, wn, ref.shape[0], mode=mode, dtype="f64")
    assert st["chains"] == len(chains)
    assert 0 < st["steps"] <= NITER * len(chains)
    assert np.abs(G - ref).max() < 1e-9 * max(1.0, np.abs(ref).max())
    if mode == 0:
        assert st["block"] in (128, 256, 512) and st["rows"] in (1, 2, 4)
        # the tuned shape is cached on the context: a second call tunes nothing
        G2, st2 = edk.green_batch(ctx, chains, NITER, wn, ref.shape[0], mode=0, dtype="f64")
        assert st2["tuned_shapes"] == 0
        assert np.abs(G2 - G).max() == 0.0


def test_green_batch_fp32_against_oracle(ctx):
    # FP32 vectors, FP64 coefficients and continued fractions: |dG| <= 2e-5
    items, ref, wn, hs = _items(ctx, [(5, 5), (4, 5)])
    chains = [dict(it, start=torch.tensor(it["phi"], device="cuda", dtype=torch.float32)) for it in items]
    G, st = edk.green_batch(ctx, chains, NITER, wn, ref.shape[0], mode=0, dtype="f32")
    assert np.abs(G - ref).max() < 2e-5


def test_green_batch_rejects_bad_items(ctx):
    w = workload("c2")
    h = edk.Hamiltonian(ctx, w.model, 5, 5)
    x = torch.zeros(h.dim, dtype=torch.float64, device="cuda")
    wn = matsubara(w.beta, 8)
    with pytest.raises(edk.EdkError):
        edk.green_batch(ctx, [dict(h=h, start=x, e0=0.0, iph=3, out=0)], 10, wn, 1)
    with pytest.raises(edk.EdkError):
        edk.green_batch(ctx, [dict(h=h, start=x, e0=0.0, iph=1, out=2)], 10, wn, 1)
    # a zero start vector contributes nothing
    G, st = edk.green_batch(ctx, [dict(h=h, start=x, e0=0.0, iph=1, out=0)], 10, wn, 1)
    assert np.all(G == 0) and st["steps"] == 0
