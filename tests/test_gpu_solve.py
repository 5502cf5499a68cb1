"""edk_solve (the driver behind the bench) against the oracle drivers, the
reference golden output, and mixed precision against FP64."""
import math
import os

import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import matsubara, star_model, workload

pytestmark = pytest.mark.gpu


def test_solve_fp64_matches_oracle_driver(ctx):
    w = workload("c1")
    m = w.model
    r = edk.solve(ctx, m, w.sectors, w.beta, 256, dtype="f64", nitergreen=w.nitergreen, spins=(0, 1))
    gso, e0o, zo = O.ground_states(m, w.sectors, w.beta, w.demax0)
    assert abs(r["e0"] - e0o) < 1e-11 * abs(e0o)
    Go_up = O.green_impurity(m, gso, w.beta, 256, w.nitergreen, spin=0)[(0, 0)]
    Go_dn = O.green_impurity(m, gso, w.beta, 256, w.nitergreen, spin=1)[(0, 0)]
    assert np.abs(r["G"][0, 0] - Go_up).max() < 1e-8
    assert np.abs(r["G"][1, 0] - Go_dn).max() < 1e-8
    assert r["residual"] < 1e-6
    assert abs(r["docc"][0] - O.OracleH(m, 4, 4).double_occ(gso[0]["psi"])) < 1e-9


def test_solve_reference_golden_g_bm(ctx):
    g = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "g_bm_2b.txt"))
    m = star_model(-5.0, 10.0, [0.0, 0.0], [math.sqrt(0.2), math.sqrt(0.3)], orbital_of_bath=[0, 1], nc=2,
                   Uprime=2.0, J=0.0, cutoff=1e-8)
    secs = [(a, b) for a in range(5) for b in range(5)]
    r = edk.solve(ctx, m, secs, 50.0, len(g), dtype="f64", neigen=40, tolerance=1e-13, demax0=50.0,
                  nitergreen=400, spins=(0,), pairs=[(0, 0), (1, 1), (0, 1)])
    assert np.abs(r["G"][0, 0] - (g[:, 1] + 1j * g[:, 2])).max() < 2e-8
    assert np.abs(r["G"][0, 1] - (g[:, 3] + 1j * g[:, 4])).max() < 2e-8
    assert np.abs(r["G"][0, 2]).max() < 1e-12


@pytest.mark.parametrize("fp32_sums", [False, True])
def test_mixed_precision_against_fp64(ctx, fp32_sums):
    """ns=14, (7,7): every sector of the solve has more than 2^20 states, so the
    mixed path runs FP32 vectors throughout, with the hop terms of H*v summed
    in FP64 or (fp32_sums) in FP32.  Bounds: |dE0/E0| <= 1e-8, max|dG| <= 1e-6
    against the FP64 solve."""
    w = workload("c3")
    # both paths converge the eigenvector (Ritz residual) so the comparison
    # measures the FP32 storage, not an under-converged FP64 ground state
    kw = dict(nitergreen=w.nitergreen, spins=(0, 1), tolerance=1e-12, residual_tol=1e-10)
    r64 = edk.solve(ctx, w.model, w.sectors, w.beta, 512, dtype="f64", **kw)
    r32 = edk.solve(ctx, w.model, w.sectors, w.beta, 512, dtype="f32", fp32_sums=fp32_sums, **kw)
    assert abs(r32["e0"] - r64["e0"]) <= 1e-8 * abs(r64["e0"])
    assert np.abs(r32["G"] - r64["G"]).max() <= 1e-6
    assert r32["residual"] < 1e-6
    assert r32["e0_lowprec"] != r32["e0"]          # the FP32 pass ran and was refined


def test_mixed_precision_keeps_small_sectors_fp64(ctx):
    """Sectors below 2^20 states run in FP64 in a mixed-precision solve: the
    result equals the FP64 solve exactly."""
    w = workload("c1")
    kw = dict(nitergreen=w.nitergreen, spins=(0, 1), tolerance=1e-12)
    r64 = edk.solve(ctx, w.model, w.sectors, w.beta, 256, dtype="f64", **kw)
    r32 = edk.solve(ctx, w.model, w.sectors, w.beta, 256, dtype="f32", **kw)
    assert r32["e0"] == r64["e0"] and r32["e0_lowprec"] == r32["e0"]
    assert np.array_equal(r32["G"], r64["G"])


def test_fp32_green_chain_small_sector(ctx):
    """FP32 chain storage on a small sector (FP64 arithmetic): the hole chain
    of ns=8 has a pole 0.06 from the Fermi level (|G| = 2 at the first
    Matsubara frequency), the worst conditioning among the workloads.
    Bound: max|dG| <= 2e-6 against the FP64 chain from the same state."""
    import torch
    w = workload("c1")
    h = edk.Hamiltonian(ctx, w.model, 4, 4)
    r = h.lanczos_e0("f64", tolerance=1e-12, residual_tol=1e-10)
    psi = h.lanczos_gs(r["vecp"][0])
    wn = matsubara(w.beta, 256)
    for dag, iph in ((True, 1), (False, 2)):
        phi, ts = h.apply_c(psi, 0, 0, dag)
        ht = edk.Hamiltonian(ctx, w.model, *ts)
        G64, *_ = ht.green_chain(phi, w.nitergreen, r["E"][0], iph, wn)
        G32, *_ = ht.green_chain(phi.to(torch.float32), w.nitergreen, r["E"][0], iph, wn)
        assert np.abs(G32 - G64).max() <= 2e-6


def test_solve_two_orbital_kanamori_all_sectors(ctx):
    """All 121 sectors of the two-orbital Kanamori model (Hund terms active)."""
    w = workload("c2")
    r = edk.solve(ctx, w.model, w.sectors, w.beta, 64, dtype="f64", nitergreen=100, spins=(0,),
                  pairs=[(0, 0), (1, 1), (0, 1)], tolerance=1e-10)
    secs = sorted(set(r["sectors"]))
    gso, e0o, zo = O.ground_states(w.model, secs, w.beta, w.demax0, tolerance=1e-10)
    assert abs(r["e0"] - e0o) < 1e-9 * abs(e0o)
    Go = O.green_impurity(w.model, gso, w.beta, 64, 100, spin=0, pairs=[(0, 0), (1, 1), (0, 1)])
    assert np.abs(r["G"][0, 0] - Go[(0, 0)]).max() < 1e-7
    assert np.abs(r["G"][0, 2] - Go[(0, 1)]).max() < 1e-7


def test_batched_chains_in_the_solve_equal_per_chain_runs(ctx):
    """ns=12 two-orbital Kanamori model, sectors (6,6), (5,6), (6,5) with three
    states each: the Green chains of these small sectors run in one persistent
    launch per spin (green_mode 0) or one by one (green_mode 1); G agrees to 1e-9."""
    w = workload("c4")
    kw = dict(dtype="f64", neigen=3, nitergreen=120, spins=(0, 1), pairs=[(0, 0), (1, 1), (0, 1)],
              tolerance=1e-11, demax0=w.demax0)
    secs = [(6, 6), (5, 6), (6, 5)]
    r0 = edk.solve(ctx, w.model, secs, w.beta, 128, green_mode=0, **kw)
    r1 = edk.solve(ctx, w.model, secs, w.beta, 128, green_mode=1, **kw)
    assert r0["nstates"] == r1["nstates"] and r0["e0"] == r1["e0"]
    assert r0["green_steps"] == r1["green_steps"]
    assert np.abs(r0["G"] - r1["G"]).max() < 1e-9 * max(1.0, np.abs(r1["G"]).max())


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_resume_from_gs_file_gives_the_same_green_function(ctx, tmp_path, dtype):
    """gs_out writes the window's eigenstates in GS.raw form; a solve started
    from that file (gs_in, no sector scan) gives the same E0, weights and G bit
    for bit.  ns=14 (7,7) for the mixed path (its FP32 vectors round-trip
    through FP64 exactly), ns=8 for FP64."""
    w = workload("c3" if dtype == "f32" else "c1")
    kw = dict(dtype=dtype, nitergreen=w.nitergreen if dtype == "f64" else 60, spins=(0, 1), tolerance=1e-12,
              residual_tol=1e-10)
    p = str(tmp_path / "GS.raw")
    r1 = edk.solve(ctx, w.model, w.sectors, w.beta, 64, gs_out=p, **kw)
    ents = edk.gs_read(p)
    assert len(ents) == r1["nstates"]
    assert ents[0]["val"] == r1["e0"] and (ents[0]["nup"], ents[0]["ndn"]) == w.sectors[0]
    r2 = edk.solve(ctx, w.model, w.sectors, w.beta, 64, gs_in=p, **kw)
    assert r2["lanczos_steps"] == 0
    assert r2["e0"] == r1["e0"] and r2["z"] == r1["z"]
    assert np.array_equal(r2["G"], r1["G"])


def test_sector_bound_file_restricts_the_scan(ctx, tmp_path):
    """With ed.sector_bound_file present only sectors within its bounds +/-
    iwindow are scanned, and the file is rewritten with the bounds of the
    states kept (two-orbital model, 121 sectors)."""
    w = workload("c2")
    kw = dict(dtype="f64", nitergreen=50, spins=(0,), pairs=[(0, 0)], tolerance=1e-10)
    full = edk.solve(ctx, w.model, w.sectors, w.beta, 16, **kw)
    nu, nd = full["sectors"][0]
    p = str(tmp_path / "ed.sector_bound_file")
    edk.sector_bounds_write(p, (nu, nu), (nd, nd))
    r = edk.solve(ctx, w.model, w.sectors, w.beta, 16, sector_bound_file=p, iwindow=1, **kw)
    assert r["lanczos_steps"] < full["lanczos_steps"]
    assert abs(r["e0"] - full["e0"]) < 1e-9 * abs(full["e0"])
    kept = set(r["sectors"])
    b = edk.sector_bounds_read(p)
    assert b[0] == (min(s[0] for s in kept), max(s[0] for s in kept))
    assert b[1] == (min(s[1] for s in kept), max(s[1] for s in kept))
    assert all(abs(s[0] - nu) <= 1 and abs(s[1] - nd) <= 1 for s in kept)


def _model_2b():
    return star_model(-5.0, 10.0, [0.0, 0.0], [math.sqrt(0.2), math.sqrt(0.3)], orbital_of_bath=[0, 1], nc=2,
                      Uprime=2.0, J=0.0, cutoff=1e-8)


def test_solve_reference_small_sectors_reproduce_g_bm(ctx):
    """reference_small_sectors on the test/2b deck, where every sector has at
    most 36 states and the reference's own run took the Lehmann branch with
    every eigenstate kept (dEmax0=10000, Neigen=500): G11 and G22 of g_bm."""
    g = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "g_bm_2b.txt"))
    secs = [(a, b) for a in range(5) for b in range(5)]
    r = edk.solve(ctx, _model_2b(), secs, 50.0, len(g), dtype="f64", neigen=500, tolerance=1e-13, demax0=10000.0,
                  nitergreen=400, spins=(0,), pairs=[(0, 0), (1, 1)], reference_small_sectors=True)
    assert r["nstates"] == 256
    assert np.abs(r["G"][0, 0] - (g[:, 1] + 1j * g[:, 2])).max() < 2e-8
    assert np.abs(r["G"][0, 1] - (g[:, 3] + 1j * g[:, 4])).max() < 2e-8


def test_solve_reference_small_sectors_narrow_window_against_oracle(ctx):
    """A narrow window (dEmax = 0.5): the Lehmann branch keeps only the target
    states in the window, so G differs from the exact continued fraction; the
    device solve equals the oracle's restatement of the branch (1e-10)."""
    m = _model_2b()
    secs = [(a, b) for a in range(5) for b in range(5)]
    kw = dict(neigen=40, tolerance=1e-13, demax0=25.0, nitergreen=400, spins=(0, 1), pairs=[(0, 0), (1, 1), (0, 1)])
    r = edk.solve(ctx, m, secs, 50.0, 128, dtype="f64", reference_small_sectors=True, **kw)
    rc = edk.solve(ctx, m, secs, 50.0, 128, dtype="f64", **kw)
    gs, e0, z = O.ground_states(m, secs, 50.0, 25.0, neigen=40, tolerance=1e-13)
    for spin in (0, 1):
        Go = O.green_impurity(m, gs, 50.0, 128, 400, spin=spin, pairs=[(0, 0), (1, 1), (0, 1)],
                              reference_small_sectors=True)
        for p, key in enumerate([(0, 0), (1, 1), (0, 1)]):
            assert np.abs(r["G"][spin, p] - Go[key]).max() < 1e-10
    assert np.abs(r["G"] - rc["G"]).max() > 1e-3


def test_mixed_precision_c2_all_sectors_fp32(ctx):
    """C2 (ns=10 Kanamori, 121 sectors, 512 points at beta=40) with FP32
    Krylov vectors in every sector of at least 1000 states (lowprec_min_dim),
    against the FP64 solve: |dE0/E0| <= 1e-8, |d docc| <= 1e-7 and
    max|dG| <= 1e-6."""
    w = workload("c2")
    kw = dict(nitergreen=w.nitergreen, spins=(0, 1), pairs=[(0, 0), (1, 1), (0, 1)], tolerance=1e-12,
              residual_tol=1e-10, demax0=w.demax0)
    r64 = edk.solve(ctx, w.model, w.sectors, w.beta, 512, dtype="f64", **kw)
    r32 = edk.solve(ctx, w.model, w.sectors, w.beta, 512, dtype="f32", lowprec_min_dim=1000, **kw)
    de = abs(r32["e0"] - r64["e0"]) / abs(r64["e0"])
    dd = np.abs(r32["docc"] - r64["docc"]).max()
    dg = np.abs(r32["G"] - r64["G"]).max()
    print(f"C2 mixed vs FP64: |dE0/E0| = {de:.3e}, |d docc| = {dd:.3e}, max|dG| = {dg:.3e}")
    assert r32["e0_lowprec"] != r32["e0"]          # FP32 passes ran and were refined
    assert de <= 1e-8 and dd <= 1e-7 and dg <= 1e-6


def test_mixed_precision_two_states_per_sector(ctx):
    """Mixed precision with neigen = 2 and a short FP32 pass 1 (eigenvalue
    tolerance 1e-5): every FP32 state of the sector is formed before any FP64
    refinement, and each refinement, which runs longer than that pass 1 (it
    also converges the Ritz residual), has its own coefficient buffers.  Each
    refined state is an eigenstate of the sector: its energy is one of the
    sector's exact lowest eigenvalues (oracle Lanczos, 1e-13) to 1e-8
    relative, the two differ, and the FP64 residual of the lower one is small.
    (States 2 and 3 of this sector lie 1.1e-3 apart; which of them the FP32
    pass resolves first is the pass's business, not the refinement's.)"""
    w = workload("c1")
    kw = dict(nitergreen=50, spins=(0,), tolerance=1e-12, neigen=2, demax0=100.0, nitermax=1000,
              tolerance_lowprec=1e-5)
    r32 = edk.solve(ctx, w.model, w.sectors, w.beta, 16, dtype="f32", lowprec_min_dim=1000, **kw)
    assert r32["nstates"] == 2
    exact = O.lanczos_e0(O.OracleH(w.model, 4, 4), nitermax=1000, neigen=4, tolerance=1e-13)["E"]
    for e in r32["energies"]:
        assert np.abs(exact - e).min() <= 1e-8 * abs(exact[0]), (e, exact)
    assert abs(r32["energies"][1] - r32["energies"][0]) > 0.1
    assert r32["residual"] < 1e-6


def test_c1_as_specified(ctx):
    """C1 as the configuration states it: ground state to |H psi - E psi| < 1e-12
    (Ritz residual), then G(i w_n) at 1024 Matsubara points, beta = 50, from
    200-step continued fractions.  The reference values come from the exact
    ground state (dense diagonalisation of the 4900-state sector) and the
    oracle's 200-step chains from it: the oracle's own Lanczos stops on the
    eigenvalue change alone, which leaves its vector converged only to about
    1e-7, too loose for a 1e-8 comparison."""
    import scipy.linalg as sla
    w = workload("c1")
    m = w.model
    r = edk.solve(ctx, m, w.sectors, w.beta, 1024, dtype="f64", nitergreen=200, spins=(0, 1), tolerance=1e-14,
                  residual_tol=1e-12)
    assert r["residual"] < 1e-11
    ho = O.OracleH(m, 4, 4)
    E, V = sla.eigh(ho.dense(), subset_by_index=[0, 0])
    e0, psi = float(E[0]), V[:, 0]
    assert abs(r["e0"] - e0) < 1e-12 * abs(e0)
    wn = matsubara(w.beta, 1024)
    for spin in (0, 1):
        Go = np.zeros(1024, complex)
        for dag, iph in ((True, 1), (False, 2)):
            phi, tsec = O.apply_c(m, 4, 4, 0, spin, dag, psi)
            G, _, _ = O.green_chain(O.OracleH(m, *tsec), phi, 200, e0, iph, wn)
            Go += G
        assert np.abs(r["G"][spin, 0] - Go).max() < 1e-8


@pytest.mark.parametrize("name,neigen", [("c2", 1), ("c4", 3)])
def test_batched_ground_states_equal_per_sector(ctx, name, neigen):
    """edk_solve_opts.batch_gs: the ground states of the small FP64 sectors in
    two persistent launches (pass 1 of every sector with its convergence test
    on the device, then pass 2) against the sector-by-sector solve.  With the
    step count fixed (tolerance 0, nitermax 60) both runs take the same steps:
    E0 and G agree to 1e-9.  With the eigenvalue tolerance both stop on it
    (the batched run checks every 8 steps, so it may take a few more): E0
    agrees to 1e-9 and G to 2e-6."""
    w = workload(name)
    pairs = [(0, 0)] if w.model.nc == 1 else [(0, 0), (1, 1)]
    kw = dict(neigen=neigen, nitergreen=100, spins=(0, 1), pairs=pairs, green_mode=1)
    for extra, tol_g in ((dict(tolerance=0.0, nitermax=60), 1e-9), (dict(tolerance=1e-11), 2e-6)):
        r0 = edk.solve(ctx, w.model, w.sectors, w.beta, 128, dtype="f64", **kw, **extra)
        r1 = edk.solve(ctx, w.model, w.sectors, w.beta, 128, dtype="f64", batch_gs=True, **kw, **extra)
        assert r1["nstates"] == r0["nstates"]
        assert list(r1["sectors"]) == list(r0["sectors"])
        assert abs(r1["e0"] - r0["e0"]) <= 1e-9 * abs(r0["e0"])
        assert np.abs(np.array(r1["energies"]) - np.array(r0["energies"])).max() <= 1e-9 * abs(r0["e0"])
        assert np.abs(r1["G"] - r0["G"]).max() <= tol_g * max(1.0, np.abs(r0["G"]).max()), \
            np.abs(r1["G"] - r0["G"]).max()
