"""Failure statuses of the Krylov entry points, each made on the host and
each expected as a status with the context still usable afterwards (no GPU
fault).  The reference STOPs at these points: zero or broken-down Krylov
vectors (ed_solver/Lanczos_plain.h:85-91), zero continued-fraction
denominators (ed_solver/matrices_tridiag.f90:176-190); an allocation it
cannot make kills the process."""
import numpy as np
import pytest
import torch

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import star_model, workload

pytestmark = pytest.mark.gpu


def _after_ok(ctx):
    """The context still runs a normal pass afterwards."""
    w = workload("c1")
    h = edk.Hamiltonian(ctx, w.model, 4, 4)
    r = h.lanczos_e0()
    ro = O.lanczos_e0(O.OracleH(w.model, 4, 4))
    assert abs(r["E"][0] - ro["E"][0]) < 1e-10 * abs(ro["E"][0])


def test_nan_start_vector_is_not_finite(ctx):
    w = workload("c1")
    h = edk.Hamiltonian(ctx, w.model, 4, 4)
    v = torch.ones(h.dim, dtype=torch.float64, device="cuda:0")
    v[17] = float("nan")
    with pytest.raises(edk.EdkError) as e:
        h.lanczos_e0(start=v)
    assert e.value.code == edk.EDK_ERR_NOT_FINITE
    v[17] = float("inf")
    with pytest.raises(edk.EdkError) as e:
        h.lanczos_e0(start=v)
    assert e.value.code == edk.EDK_ERR_NOT_FINITE
    _after_ok(ctx)


def test_zero_start_vector(ctx):
    w = workload("c1")
    h = edk.Hamiltonian(ctx, w.model, 4, 4)
    v = torch.zeros(h.dim, dtype=torch.float64, device="cuda:0")
    with pytest.raises(edk.EdkError) as e:
        h.lanczos_e0(start=v)
    assert e.value.code == edk.EDK_ERR_ZERO_START
    _after_ok(ctx)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_eigenvector_start_exhausts_the_krylov_space(ctx, dtype):
    """Without hybridisation (V = 0) H is diagonal in the occupation basis, so
    a basis state is an exact eigenvector: beta_2 is exactly zero, the chain
    stops after one step with EDK_KRYLOV_EXHAUSTED, and its Ritz value is the
    state's diagonal energy."""
    rng = np.random.default_rng(3)
    m = star_model(-1.0, 2.0, rng.uniform(-1, 1, 7), np.zeros(7))
    h = edk.Hamiltonian(ctx, m, 4, 4)
    d = O.OracleH(m, 4, 4).dense()
    assert np.count_nonzero(d - np.diag(np.diag(d))) == 0
    i = 123
    v = torch.zeros(h.dim, dtype=torch.float64 if dtype == "f64" else torch.float32, device="cuda:0")
    v[i] = 0.5
    r = h.lanczos_e0(dtype, start=v, nitermax=50)
    assert r["status"] == edk.EDK_KRYLOV_EXHAUSTED
    assert r["niter"] == 1
    assert r["subdiag"][1] == 0.0
    # FP32 storage rounds the stored vector s = H v to FP32, and alpha is read from it
    tol = 1e-12 if dtype == "f64" else 1.2e-7
    assert abs(r["E"][0] - d[i, i]) < tol * max(1.0, abs(d[i, i]))
    _after_ok(ctx)


def test_workspace_cap_gives_nomem(ctx):
    """A host-side cap below the five Krylov vectors of the sector: the pass
    returns EDK_ERR_NOMEM before allocating; lifting the cap restores it."""
    w = workload("c1")
    h = edk.Hamiltonian(ctx, w.model, 4, 4)
    ctx.set_workspace_limit(5 * 8 * h.dim - 8)
    try:
        with pytest.raises(edk.EdkError) as e:
            h.lanczos_e0()
        assert e.value.code == edk.EDK_ERR_NOMEM
        assert "limit" in str(e.value)
        with pytest.raises(edk.EdkError) as e:
            edk.solve(ctx, w.model, w.sectors, w.beta, 16, dtype="f64", nitergreen=20)
        assert e.value.code == edk.EDK_ERR_NOMEM
        ctx.set_workspace_limit(5 * 8 * h.dim)
        h.lanczos_e0()
    finally:
        ctx.set_workspace_limit(0)
    _after_ok(ctx)
