"""Pass 2 from the Krylov vectors pass 1 kept on the device (keep_basis)
against pass 2 recomputing the recurrence (Lanczos_get_GS_sector's way)."""
import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import workload, nambu_workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tol", [("f64", 1e-13), ("f32", 2e-6)])
def test_stored_basis_matches_recompute(ctx, dtype, tol):
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    r0 = h.lanczos_e0(dtype=dtype, neigen=2, demax=50.0, tolerance=1e-10 if dtype == "f64" else 1e-6)
    r1 = h.lanczos_e0(dtype=dtype, neigen=2, demax=50.0, tolerance=1e-10 if dtype == "f64" else 1e-6,
                      keep_basis=True)
    # the stored-basis pass 1 runs the same recurrence (plain launches instead of graphs)
    assert r1["niter"] == r0["niter"]
    assert np.array_equal(r1["diag"], r0["diag"]) and np.array_equal(r1["subdiag"], r0["subdiag"])
    k = len(r1["E"])
    for j in range(k):
        ref = h.lanczos_gs(r0["vecp"][j], dtype=dtype).double().cpu().numpy()
        got = h.lanczos_gs(r1["vecp"][j], dtype=dtype, keep_basis=2 if j + 1 < k else 1)
        got = got.double().cpu().numpy()
        assert abs(np.linalg.norm(got) - 1.0) < 10 * tol
        assert np.abs(got - ref).max() < tol
    # released: a further keep_basis pass 2 recomputes, identical to the plain one
    again = h.lanczos_gs(r1["vecp"][0], dtype=dtype, keep_basis=1).double().cpu().numpy()
    plain = h.lanczos_gs(r0["vecp"][0], dtype=dtype).double().cpu().numpy()
    assert np.array_equal(again, plain)


def test_stored_basis_start_vector_and_oracle(ctx):
    import torch
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    ho = O.OracleH(m, 4, 4)
    g = np.random.default_rng(3).standard_normal(h.dim)
    start = torch.tensor(g, dtype=torch.float64, device=f"cuda:{ctx.device}")
    r = h.lanczos_e0(start=start, keep_basis=True)
    psi = h.lanczos_gs(r["vecp"][0], start=start, keep_basis=True).cpu().numpy()
    ref = h.lanczos_gs(r["vecp"][0], start=start).cpu().numpy()
    assert np.abs(psi - ref).max() < 1e-13
    ev, V = np.linalg.eigh(ho.dense())
    assert abs(r["E"][0] - ev[0]) < 1e-10
    # stopped on an eigenvalue change of 1e-12: the vector is good to ~sqrt of that
    s = np.sign(psi @ V[:, 0])
    assert np.abs(psi - s * V[:, 0]).max() < 1e-5


def test_stored_basis_other_start_recomputes(ctx):
    """A pass 2 whose start differs from pass 1's does not use the kept vectors."""
    import torch
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    r = h.lanczos_e0(keep_basis=True)
    g = np.random.default_rng(4).standard_normal(h.dim)
    start = torch.tensor(g, dtype=torch.float64, device=f"cuda:{ctx.device}")
    got = h.lanczos_gs(r["vecp"][0], start=start, keep_basis=True).cpu().numpy()
    ref = h.lanczos_gs(r["vecp"][0], start=start).cpu().numpy()
    assert np.array_equal(got, ref)


def test_stored_basis_nambu(ctx):
    m = nambu_workload(8)
    h = edk.HamiltonianSz(ctx, m, 8)
    r0 = h.lanczos_e0()
    r1 = h.lanczos_e0(keep_basis=True)
    assert np.array_equal(r1["diag"], r0["diag"])
    ref = h.lanczos_gs(r0["vecp"][0]).cpu().numpy()
    got = h.lanczos_gs(r1["vecp"][0], keep_basis=True).cpu().numpy()
    assert np.abs(got - ref).max() < 1e-13


@pytest.mark.parametrize("dtype,tol", [("f64", 1e-12), ("f32", 1e-6)])
def test_solve_pass2_from_kept_vectors_matches_recompute(ctx, dtype, tol):
    """edk_solve with pass 2 formed from the kept Krylov vectors (the default)
    and with the reference's recomputing pass 2 give the same E0 and G."""
    from ed_solver_b200.model import workload as wl
    w = wl("c1")
    kw = dict(dtype=dtype, nitermax=w.nitermax, nitergreen=60)
    a = edk.solve(ctx, w.model, w.sectors, w.beta, 64, **kw)
    b = edk.solve(ctx, w.model, w.sectors, w.beta, 64, recompute_pass2=True, **kw)
    assert abs(a["e0"] - b["e0"]) <= tol * abs(b["e0"])
    assert np.abs(a["G"] - b["G"]).max() <= tol * np.abs(b["G"]).max()
    assert a["lanczos_steps"] == b["lanczos_steps"]
