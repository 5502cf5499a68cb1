"""Nambu (Sz) sectors on the device against the CPU oracle (HAIMsz restated in
oracle/edk_oracle.c): H*v FP64 bit-exact in both term orders, FP32 within the
output rounding, c / c+ bit-exact, Lanczos energies, Green chains, and the
hermiticity of H*v at 601M states (ns=16, the half-filled Nambu sector)."""
import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import NambuModel, matsubara, nambu_workload, star_model

pytestmark = pytest.mark.gpu


def _two_orbital(pvbc=False, on_fly=False):
    rng = np.random.default_rng(11)
    base = star_model([-1.2, -0.8], 2.5, rng.uniform(-1.5, 1.5, 5), rng.uniform(0.2, 0.5, 5),
                      orbital_of_bath=[0, 1, 1, 0, 1], nc=2, Uprime=1.3, J=0.0, cutoff=1e-8)
    base.ec[:, 0, 1] = base.ec[:, 1, 0] = 0.15
    base.eb[:, 0, 2] = base.eb[:, 2, 0] = 0.07
    pb = np.diag(rng.uniform(0.1, 0.3, 5))
    pb[0, 1] = pb[1, 0] = 0.05
    pv = None
    if pvbc:
        pv = np.zeros((2, 5, 2))
        pv[0, 0, 0] = 0.11
        pv[1, 2, 1] = -0.09
    return NambuModel(base, pb, pv, on_fly)


MODELS = {
    "star8": lambda: nambu_workload(8),
    "star8_fly": lambda: nambu_workload(8, on_fly=True),
    "two_orbital": lambda: _two_orbital(),
    "two_orbital_pvbc_fly": lambda: _two_orbital(pvbc=True, on_fly=True),
}


@pytest.fixture(params=[0, 1], ids=["compacted-rows", "whole-term-list"])
def kpath(request, ctx):
    ctx.set_kernel_path(request.param)
    yield request.param
    ctx.set_kernel_path(0)


@pytest.mark.parametrize("name", sorted(MODELS))
def test_hmult_fp64_bit_exact(ctx, kpath, name):
    import torch
    m = MODELS[name]()
    rng = np.random.default_rng(1)
    for npart in (0, 1, m.ns - 1, m.ns, m.ns + 2, 2 * m.ns):
        h = edk.HamiltonianSz(ctx, m, npart)
        ho = O.OracleSz(m, npart)
        assert h.dim == ho.dim
        assert h.energy_shift == ho.shift
        x = rng.normal(size=h.dim)
        y = h.hmult(torch.tensor(x, device="cuda")).cpu().numpy()
        assert np.array_equal(y, ho.hmult(x)), npart


def test_hmult_fp64_bit_exact_ns12(ctx, kpath):
    """ns=12 half-filled Nambu sector: 2.7M states, rows of up to 924 low halves."""
    import torch
    m = nambu_workload(12)
    h = edk.HamiltonianSz(ctx, m, 12)
    ho = O.OracleSz(m, 12)
    x = np.random.default_rng(4).normal(size=h.dim)
    y = h.hmult(torch.tensor(x, device="cuda")).cpu().numpy()
    assert np.array_equal(y, ho.hmult(x))


@pytest.mark.parametrize("name", ["star8", "two_orbital_pvbc_fly"])
def test_hmult_fp32(ctx, kpath, name):
    import torch
    m = MODELS[name]()
    h = edk.HamiltonianSz(ctx, m, m.ns)
    x = np.random.default_rng(7).normal(size=h.dim)
    y = h.hmult(torch.tensor(x, dtype=torch.float32, device="cuda")).double().cpu().numpy()
    y_ref = O.OracleSz(m, m.ns).hmult(x.astype(np.float32).astype(np.float64))
    # FP64 arithmetic on FP32-stored vectors: only the output rounding remains
    assert np.abs(y - y_ref).max() <= 1.2e-7 * np.abs(y_ref).max()


@pytest.mark.parametrize("projected", [False, True])
def test_apply_c_bit_exact(ctx, projected):
    import torch
    m = _two_orbital(pvbc=True)
    rng = np.random.default_rng(9)
    for npart in (m.ns - 1, m.ns):
        h = edk.HamiltonianSz(ctx, m, npart)
        ho = O.OracleSz(m, npart)
        x = rng.normal(size=h.dim)
        xd = torch.tensor(x, device="cuda")
        for site in range(m.nc):
            for spin in (0, 1):
                for dag in (True, False):
                    out, npt = h.apply_c(xd, site, spin, dag, projected=projected)
                    ref, npt_o = ho.apply_c(x, site, spin, dag, projected=projected)
                    assert npt == npt_o
                    assert np.array_equal(out.cpu().numpy(), ref), (site, spin, dag)


def test_apply_c_symmetric_combination(ctx):
    """(c_0 + sign2 c_1)|x>: the second operator's term added to the first's."""
    import torch
    m = _two_orbital()
    h = edk.HamiltonianSz(ctx, m, m.ns)
    ho = O.OracleSz(m, m.ns)
    x = np.random.default_rng(5).normal(size=h.dim)
    for sign2 in (1, -1):
        out, npt = h.apply_c(torch.tensor(x, device="cuda"), 0, 1, True, site2=1, sign2=sign2)
        a, _ = ho.apply_c(x, 0, 1, True)
        b, _ = ho.apply_c(x, 1, 1, True)
        assert np.array_equal(out.cpu().numpy(), a + sign2 * b)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_lanczos_ground_state_energy(ctx, dtype):
    """Nambu ground state of ns=8 (12870 states) against dense diagonalisation;
    the device eigenvector against the dense one."""
    import torch
    m = nambu_workload(8)
    h = edk.HamiltonianSz(ctx, m, m.ns)
    E = np.linalg.eigvalsh(O.OracleSz(m, m.ns).dense())
    r = h.lanczos_e0(dtype, tolerance=1e-12, residual_tol=1e-9 if dtype == "f64" else 0.0)
    tol = 1e-10 if dtype == "f64" else 1e-5
    assert abs(r["E"][0] - E[0]) < tol * max(1.0, abs(E[0]))
    if dtype == "f64":
        psi = h.lanczos_gs(r["vecp"][0])
        res, nrm = h.residual(psi, r["E"][0])
        assert res < 1e-7 and abs(nrm - 1.0) < 1e-12


def test_lanczos_matches_oracle_driver(ctx):
    """Pass 1 from the same start vector: the device alpha/beta follow the
    oracle's Lanczos_fast_diagonalize, and the lowest energy agrees."""
    m = _two_orbital(pvbc=True, on_fly=True)
    h = edk.HamiltonianSz(ctx, m, m.ns)
    ho = O.OracleSz(m, m.ns)
    ro = O.lanczos_e0(ho, nitermax=60, tolerance=1e-12)
    r = h.lanczos_e0("f64", nitermax=60, tolerance=1e-12, check_every=1)
    assert abs(r["E"][0] - ro["E"][0]) < 1e-11 * abs(ro["E"][0])
    n = min(12, len(ro["diag"]), len(r["diag"]))
    assert np.abs(r["diag"][:n] - ro["diag"][:n]).max() < 1e-10


@pytest.mark.parametrize("spin,dagger", [(0, True), (0, False), (1, True), (1, False)])
def test_green_chain_matches_oracle(ctx, spin, dagger):
    """compute_dynamic on the Nambu target sector from c[+]|GS>."""
    import torch
    m = nambu_workload(7)
    wn = matsubara(50.0, 64)
    h = edk.HamiltonianSz(ctx, m, m.ns)
    ho = O.OracleSz(m, m.ns)
    r = h.lanczos_e0("f64", tolerance=1e-12, residual_tol=1e-10)
    psi = h.lanczos_gs(r["vecp"][0])
    phi, npt = h.apply_c(psi, 0, spin, dagger)
    ht = edk.HamiltonianSz(ctx, m, npt)
    iph = 1 if dagger else 2
    G, dg, sd, n = ht.green_chain(phi, 150, r["E"][0], iph, wn)
    Go, dgo, sdo = O.green_chain(O.OracleSz(m, npt), phi.cpu().numpy(), 150, r["E"][0], iph, wn)
    assert n == len(dgo)
    assert np.abs(G - Go).max() < 1e-9 * max(1.0, np.abs(Go).max())


def test_block_lanczos_nambu(ctx):
    m = nambu_workload(6)
    h = edk.HamiltonianSz(ctx, m, m.ns)
    E = np.linalg.eigvalsh(O.OracleSz(m, m.ns).dense())
    Eb, V, it, conv = h.block_lanczos(block=2, neigen=3, nitermax=200, tolerance=1e-12)
    assert conv
    assert np.abs(Eb - E[:3]).max() < 1e-9
    for e in range(3):
        res, nrm = h.residual(V[e].contiguous(), Eb[e])
        assert res < 1e-5 * max(1.0, abs(Eb[e]))


def test_hermitian_at_ns16(ctx):
    """ns=16, npart=16: 601,080,390 states.  <a|H b> = <H a|b> and the FP64
    result does not depend on the launch (a size-independent check)."""
    import torch
    m = nambu_workload(16)
    h = edk.HamiltonianSz(ctx, m, 16)
    assert h.dim == 601080390
    g = torch.Generator(device="cuda").manual_seed(0)
    a = torch.randn(h.dim, dtype=torch.float64, device="cuda", generator=g)
    b = torch.randn(h.dim, dtype=torch.float64, device="cuda", generator=g)
    hb = h.hmult(b)
    lhs = float(torch.dot(a, hb))
    del hb
    ha = h.hmult(a)
    rhs = float(torch.dot(ha, b))
    ha2 = h.hmult(a)
    assert torch.equal(ha, ha2)
    scale = float(a.norm()) * float(ha.norm())
    assert abs(lhs - rhs) <= 1e-12 * scale
