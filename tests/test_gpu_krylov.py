"""Lanczos, c/c+ maps and Green chains on the device against the CPU oracle."""
import math

import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk, solver
from ed_solver_b200.model import star_model, workload, matsubara

pytestmark = pytest.mark.gpu


def test_lanczos_e0_and_vector_fp64(ctx):
    w = workload("c1")
    m = w.model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    ho = O.OracleH(m, 4, 4)
    r = h.lanczos_e0(nitermax=1000, neigen=1, tolerance=1e-12, check_every=4)
    ro = O.lanczos_e0(ho, nitermax=1000, neigen=1, tolerance=1e-12)
    assert abs(r["E"][0] - ro["E"][0]) <= 1e-11 * abs(ro["E"][0])
    # same start vector -> same Krylov coefficients early on
    n = min(20, r["niter"], ro["niter"])
    assert np.allclose(r["diag"][:n], ro["diag"][:n], rtol=1e-9, atol=1e-11)
    assert np.allclose(r["subdiag"][1:n], ro["subdiag"][1:n], rtol=1e-9, atol=1e-11)
    assert abs(r["niter"] - ro["niter"]) <= 2
    psi = h.lanczos_gs(r["vecp"][0]).cpu().numpy()
    psio = O.lanczos_gs(ho, ro["vecp"][0])
    s = np.sign(psi @ psio)
    assert np.abs(psi - s * psio).max() < 1e-7
    ev = np.linalg.eigvalsh(ho.dense()) if ho.dim <= 5000 else None
    if ev is not None:
        assert abs(r["E"][0] - ev[0]) < 1e-10
    res, nrm = h.residual(h.lanczos_gs(r["vecp"][0]), r["E"][0])
    assert abs(nrm - 1.0) < 1e-12 and res < 1e-6


def test_lanczos_neigen_window(ctx):
    m = workload("c2").model
    h = edk.Hamiltonian(ctx, m, 5, 5)
    ho = O.OracleH(m, 5, 5)
    r = h.lanczos_e0(neigen=3, tolerance=1e-10, demax=5.0)
    ro = O.lanczos_e0(ho, neigen=3, tolerance=1e-10, demax=5.0)
    k = min(len(r["E"]), len(ro["E"]))
    assert k >= 1
    assert np.allclose(r["E"][:k], ro["E"][:k], rtol=1e-10, atol=1e-10)


def test_lanczos_fp32_then_fp64_residual(ctx):
    import torch
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    e64 = h.lanczos_e0(dtype="f64")["E"][0]
    r = h.lanczos_e0(dtype="f32", tolerance=1e-7)
    assert abs(r["E"][0] - e64) < 1e-5 * abs(e64)
    psi = h.lanczos_gs(r["vecp"][0], dtype="f32")
    res, nrm = h.residual(psi.double(), r["E"][0])
    assert res < 1e-3


def test_zero_start_vector_is_an_error_not_a_fault(ctx):
    import torch
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    z = torch.zeros(h.dim, dtype=torch.float64, device="cuda")
    with pytest.raises(edk.EdkError) as ei:
        h.lanczos_e0(start=z)
    assert ei.value.code == edk.EDK_ERR_ZERO_START


def test_apply_c_bit_exact(ctx):
    import torch
    m = workload("c2").model
    rng = np.random.default_rng(4)
    for (nu, nd) in [(5, 5), (0, 3), (10, 2)]:
        h = edk.Hamiltonian(ctx, m, nu, nd)
        x = rng.normal(size=h.dim)
        xt = torch.tensor(x, device="cuda")
        for spin in (0, 1):
            for dag in (True, False):
                for site in (0, 1):
                    try:
                        yo, tsec = O.apply_c(m, nu, nd, site, spin, dag, x)
                    except ValueError:
                        continue
                    y, tsec2 = h.apply_c(xt, site, spin, dag)
                    assert tsec == tsec2
                    assert np.array_equal(y.cpu().numpy(), yo)
                y, _ = h.apply_c(xt, 0, spin, True, site2=1, sign2=1) if (nu if spin == 0 else nd) < m.ns else (None, None)
                if y is not None:
                    a, _ = O.apply_c(m, nu, nd, 0, spin, True, x)
                    b, _ = O.apply_c(m, nu, nd, 1, spin, True, x)
                    assert np.array_equal(y.cpu().numpy(), a + b)


def test_green_chain_against_oracle(ctx):
    import torch
    w = workload("c1")
    m = w.model
    ho = O.OracleH(m, 4, 4)
    ro = O.lanczos_e0(ho)
    psi = O.lanczos_gs(ho, ro["vecp"][0])
    e0 = ro["E"][0]
    wn = matsubara(w.beta, 256)
    for iph, dag in ((1, True), (2, False)):
        phi, tsec = O.apply_c(m, 4, 4, 0, 0, dag, psi)
        Go, dgo, sdo = O.green_chain(O.OracleH(m, *tsec), phi, 200, e0, iph, wn)
        ht = edk.Hamiltonian(ctx, m, *tsec)
        G, dg, sd, n = ht.green_chain(torch.tensor(phi, device="cuda"), 200, e0, iph, wn)
        assert n == len(dgo)
        assert np.allclose(dg[:30], dgo[:30], rtol=1e-9, atol=1e-10)
        assert np.abs(G - Go).max() < 1e-9


def test_cf_eval_against_oracle(ctx):
    rng = np.random.default_rng(8)
    chains = []
    for n in (1, 5, 50):
        chains.append(dict(diag=rng.normal(size=n), subdiag=np.concatenate([[0.0], rng.uniform(0.2, 1, n - 1)]),
                           e=-1.3, ph=1.0 if n % 2 else -1.0, scale=0.7))
    wn = matsubara(20.0, 64)
    G = edk.cf_eval(ctx, chains, wn)
    for c, g in zip(chains, G):
        td = c["ph"] * (c["diag"] - c["e"])
        ref = np.array([O.cf(td, c["subdiag"], 1j * x) for x in wn]) * c["scale"]
        assert np.abs(g - ref).max() < 1e-12


def test_full_green_c1_against_oracle_driver(ctx):
    w = workload("c1")
    m = w.model
    hc = solver.HCache(ctx, m)
    gs, e0, z = solver.ground_states(hc, w.sectors, w.beta, w.demax0)
    gso, e0o, zo = O.ground_states(m, w.sectors, w.beta, w.demax0)
    assert abs(e0 - e0o) < 1e-11 * abs(e0o)
    G = solver.green_impurity(hc, gs, w.beta, 256, w.nitergreen)[(0, 0)]
    Go = O.green_impurity(m, gso, w.beta, 256, w.nitergreen)[(0, 0)]
    assert np.abs(G - Go).max() < 1e-8
    d, n = hc.get((4, 4)).double_occ(gs[0]["psi"])
    assert abs(d - O.OracleH(m, 4, 4).double_occ(gso[0]["psi"])) < 1e-9


def test_reference_golden_through_the_device(ctx):
    import os
    g = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "g_bm_2b.txt"))
    m = star_model(-5.0, 10.0, [0.0, 0.0], [math.sqrt(0.2), math.sqrt(0.3)], orbital_of_bath=[0, 1], nc=2,
                   Uprime=2.0, J=0.0, cutoff=1e-8)
    hc = solver.HCache(ctx, m)
    secs = [(a, b) for a in range(5) for b in range(5)]
    gs, e0, z = solver.ground_states(hc, secs, 50.0, 50.0, neigen=40, tolerance=1e-13)
    G = solver.green_impurity(hc, gs, 50.0, len(g), 400, pairs=[(0, 0), (1, 1)])
    assert np.abs(G[(0, 0)] - (g[:, 1] + 1j * g[:, 2])).max() < 2e-8
    assert np.abs(G[(1, 1)] - (g[:, 3] + 1j * g[:, 4])).max() < 2e-8


def test_fast_row_kernel_krylov_ns14_against_oracle(ctx):
    """The ns=14 (7,7) sector (1.18e7 states) runs on the fast row kernel:
    Lanczos coefficients, the pass-2 vector (accumulated inside the fused step),
    the c+ map and a Green chain in FP64 against the oracle (1e-9); the FP32
    chain against the FP64 one (1e-5)."""
    import torch
    w = workload("c3")
    m = w.model
    nst = 40
    h = edk.Hamiltonian(ctx, m, 7, 7)
    ho = O.OracleH(m, 7, 7)
    r = h.lanczos_e0(nitermax=nst, tolerance=0.0, check_every=nst)
    ro = O.lanczos_e0(ho, nitermax=nst, tolerance=0.0)
    n = min(r["niter"], ro["niter"])
    assert n >= nst - 1
    assert np.allclose(r["diag"][:n], ro["diag"][:n], rtol=1e-9, atol=1e-10)
    assert np.allclose(r["subdiag"][1:n], ro["subdiag"][1:n], rtol=1e-9, atol=1e-10)
    psi = h.lanczos_gs(r["vecp"][0])
    psio = O.lanczos_gs(ho, r["vecp"][0])
    assert np.abs(psi.cpu().numpy() - psio).max() < 1e-8
    e0 = r["E"][0]
    phi, ts = h.apply_c(psi, 0, 0, True)
    wn = matsubara(w.beta, 128)
    ht = edk.Hamiltonian(ctx, m, *ts)
    G, _, _, _ = ht.green_chain(phi, nst, e0, 1, wn)
    Go, _, _ = O.green_chain(O.OracleH(m, *ts), phi.cpu().numpy(), nst, e0, 1, wn)
    assert np.abs(G - Go).max() < 1e-9
    G32, _, _, _ = ht.green_chain(phi.to(torch.float32), nst, e0, 1, wn)
    assert np.abs(G32 - G).max() < 1e-5


def test_block_lanczos_against_dense_ed(ctx):
    """Block_Lanczos_diagonalize: lowest eigenvalues with multiplicity against
    dense diagonalisation (1e-9), eigenvector residuals (1e-6).  The second
    model has two identical orbitals, so its levels come in degenerate pairs
    that a single-vector Lanczos would see once."""
    import torch
    rng = np.random.default_rng(4)
    eb = rng.uniform(-1, 1, 2)
    v = rng.uniform(0.2, 0.5, 2)
    sym = star_model(-1.5, 3.0, [eb[0], eb[1], eb[0], eb[1]], [v[0], v[1], v[0], v[1]],
                     orbital_of_bath=[0, 0, 1, 1], nc=2, J=0.4)
    for m, sec, p, ne in [(workload("c1").model, (4, 4), 3, 6), (sym, (3, 2), 2, 6)]:
        h = edk.Hamiltonian(ctx, m, *sec)
        ref = np.linalg.eigvalsh(O.OracleH(m, *sec).dense())[:ne]
        E, V, it, conv = h.block_lanczos(block=p, neigen=ne, nitermax=400, tolerance=1e-13, check_every=2)
        assert conv
        assert np.abs(E - ref).max() < 1e-9 * max(1.0, np.abs(ref).max()), (E, ref)
        for e in range(ne):
            r = h.hmult(V[e]) - E[e] * V[e]
            assert float(torch.linalg.norm(r)) < 1e-6
    assert abs(ref[1] - ref[0]) < 1e-9          # the symmetric model does have a degenerate ground level


def test_graph_replayed_steps_equal_plain_launches(ctx):
    """Pairs of fused steps replayed as a CUDA graph give the same Krylov
    coefficients, eigenvector and Green function, bit for bit, as plain
    launches (ns=8 and the ns=14 (7,7) sector, pass 1, pass 2 and a chain)."""
    import torch
    for name, sec in [("c1", (4, 4)), ("c3", (7, 7))]:
        w = workload(name)
        h = edk.Hamiltonian(ctx, w.model, *sec)
        res = []
        for g in (False, True):
            ctx.set_graphs(g)
            r = h.lanczos_e0("f64", nitermax=60, tolerance=0.0, check_every=7)
            psi = h.lanczos_gs(r["vecp"][0])
            phi, ts = h.apply_c(psi, 0, 0, True)
            ht = edk.Hamiltonian(ctx, w.model, *ts)
            G, dg, sd, n = ht.green_chain(phi, 41, r["E"][0], 1, matsubara(w.beta, 16))
            res.append((r["diag"], r["subdiag"], psi.cpu().numpy(), G, dg))
        ctx.set_graphs(True)
        for a, b in zip(res[0], res[1]):
            assert np.array_equal(a, b)


def test_timing_counts_graph_replays_as_their_launches(ctx):
    """Per-launch timing with graph replay on: a replay is timed as a whole and
    counted as its two fused steps, so the fused-step count equals the plain
    launches' count and the coefficients stay bit-identical."""
    w = workload("c3")
    h = edk.Hamiltonian(ctx, w.model, 7, 7)
    out = []
    for g in (False, True):
        ctx.set_graphs(g)
        ctx.timing(True)
        r = h.lanczos_e0("f64", nitermax=40, tolerance=0.0, check_every=40)
        n, ms, el = ctx.timing_report(2)
        ctx.timing(False)
        out.append((r["diag"], n, ms, el))
    ctx.set_graphs(True)
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] >= len(out[0][0]) - 1
    assert out[1][2] > 0.0 and out[1][3] == out[0][3]
