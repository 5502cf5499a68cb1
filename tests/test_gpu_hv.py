"""H*v on the device against the CPU oracle: FP64 bit-exact, FP32 within tolerance."""
import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import star_model, workload

pytestmark = pytest.mark.gpu


def _models():
    rng = np.random.default_rng(21)
    m1 = star_model(-0.7, 2.0, rng.uniform(-1, 1, 5), rng.uniform(0.2, 0.6, 5))
    m2 = star_model(-1.0, 3.0, rng.uniform(-1, 1, 4), rng.uniform(0.2, 0.6, 4), orbital_of_bath=[0, 1, 1, 0],
                    nc=2, J=0.5)
    m2.ec[:, 0, 1] = m2.ec[:, 1, 0] = 0.3
    m2.eb[:, 0, 2] = m2.eb[:, 2, 0] = 0.25
    m3 = star_model([-1.2, -0.8, -1.0], 2.5, rng.uniform(-1, 1, 3), rng.uniform(0.2, 0.6, 3),
                    orbital_of_bath=[0, 1, 2], nc=3, J=0.3)
    return [m1, m2, m3]


SECTORS = [(3, 3), (2, 4), (4, 1), (0, 3), (5, 5), (1, 0)]


@pytest.fixture(params=[0, 1, 2], ids=["auto-kernel", "generic-kernel", "fast-kernel"])
def kpath(request, ctx):
    ctx.set_kernel_path(request.param)
    yield request.param
    ctx.set_kernel_path(0)


@pytest.mark.parametrize("mi", [0, 1, 2])
def test_hmult_fp64_bit_exact(ctx, kpath, mi):
    import torch
    m = _models()[mi]
    rng = np.random.default_rng(mi)
    for nu, nd in SECTORS:
        if nu > m.ns or nd > m.ns:
            continue
        h = edk.Hamiltonian(ctx, m, nu, nd)
        ho = O.OracleH(m, nu, nd)
        x = rng.normal(size=h.dim)
        y = h.hmult(torch.tensor(x, device="cuda")).cpu().numpy()
        y_ref = ho.hmult(x)
        assert np.array_equal(y, y_ref), (nu, nd, np.abs(y - y_ref).max())


@pytest.mark.parametrize("mi", [0, 1])
def test_hmult_fp32(ctx, kpath, mi):
    import torch
    m = _models()[mi]
    rng = np.random.default_rng(7)
    for nu, nd in [(3, 3), (2, 4)]:
        h = edk.Hamiltonian(ctx, m, nu, nd)
        x = rng.normal(size=h.dim)
        y = h.hmult(torch.tensor(x, dtype=torch.float32, device="cuda")).double().cpu().numpy()
        y_ref = O.OracleH(m, nu, nd).hmult(x.astype(np.float32).astype(np.float64))
        # FP64 arithmetic on FP32-stored vectors: only the output rounding remains
        assert np.abs(y - y_ref).max() <= 1.2e-7 * np.abs(y_ref).max()


def test_hmult_large_rows_c3_sector_bit_exact(ctx, kpath):
    """The ns=14 sector (3432 x 3432 rows): staged rows, packed up table, row schedule."""
    import torch
    m = workload("c3").model
    h = edk.Hamiltonian(ctx, m, 7, 7)
    ho = O.OracleH(m, 7, 7)
    rng = np.random.default_rng(3)
    x = rng.normal(size=h.dim)
    y = h.hmult(torch.tensor(x, device="cuda")).cpu().numpy()
    assert np.array_equal(y, ho.hmult(x))


def test_hmult_host_buffers(ctx):
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    x = np.random.default_rng(1).normal(size=h.dim)
    assert np.array_equal(h.hmult_host(x), O.OracleH(m, 4, 4).hmult(x))


def test_hmult_rejects_bad_sizes(ctx):
    import torch
    h = edk.Hamiltonian(ctx, workload("c1").model, 4, 4)
    with pytest.raises(edk.EdkError):
        edk.lib()  # loaded
        ctx.check(edk.lib().edk_hmult(h.h, 0, h.dim + 1, torch.zeros(1, device="cuda").data_ptr(),
                                      torch.zeros(1, device="cuda").data_ptr()), "size")


def test_tables_on_device_match_host_builder(ctx):
    m = workload("c2").model
    h = edk.Hamiltonian(ctx, m, 5, 4)
    for spin in (0, 1):
        p, t, v, d = h.table(spin)
        p2, t2, v2, d2 = edk.build_table(m, spin, 5 if spin == 0 else 4)
        assert np.array_equal(t, t2) and np.array_equal(v, v2) and np.array_equal(d, d2)


def test_hmult_misaligned_pointers_take_the_generic_path(ctx):
    """Vectors offset by one element (not 16-byte aligned) must still be exact."""
    import torch
    m = workload("c1").model
    h = edk.Hamiltonian(ctx, m, 4, 4)
    x = np.random.default_rng(5).normal(size=h.dim)
    xb = torch.zeros(h.dim + 1, dtype=torch.float64, device="cuda")
    xb[1:] = torch.tensor(x, device="cuda")
    yb = torch.zeros(h.dim + 1, dtype=torch.float64, device="cuda")
    h.hmult(xb[1:], out=yb[1:])
    assert np.array_equal(yb[1:].cpu().numpy(), O.OracleH(m, 4, 4).hmult(x))


def test_hmult_full_size_ns16_bit_exact(ctx):
    """The ns=16 half-filled sector (1.66e8 states), FP64, against the oracle."""
    import torch
    m = workload("c5").model
    h = edk.Hamiltonian(ctx, m, 8, 8)
    x = torch.rand(h.dim, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    y = h.hmult(x).cpu().numpy()
    ho = O.OracleH(m, 8, 8)
    assert np.array_equal(y, ho.hmult(x.cpu().numpy()))


@pytest.mark.parametrize("name,sec", [("c3", (7, 7)), ("c3", (8, 7))])
def test_hmult_fp32_large_sectors(ctx, kpath, name, sec):
    """FP32 H*v on sectors large enough for multi-row groups (R > 1) in both kernels."""
    import torch
    m = workload(name).model
    h = edk.Hamiltonian(ctx, m, *sec)
    x = np.random.default_rng(9).normal(size=h.dim)
    y = h.hmult(torch.tensor(x, dtype=torch.float32, device="cuda")).double().cpu().numpy()
    y_ref = O.OracleH(m, *sec).hmult(x.astype(np.float32).astype(np.float64))
    assert np.abs(y - y_ref).max() <= 1.2e-7 * np.abs(y_ref).max()


def test_every_fast_kernel_launch_shape_is_exact(ctx):
    """Each feasible launch shape of both fast row kernels (rows per group,
    block shape, kernel kind) on the ns=14 (7,7) and (8,7) sectors: FP64
    bit-exact, FP32 within the output rounding."""
    import torch
    m = workload("c3").model
    rng = np.random.default_rng(13)
    for sec in [(7, 7), (8, 7)]:
        h = edk.Hamiltonian(ctx, m, *sec)
        ho = O.OracleH(m, *sec)
        x = rng.normal(size=h.dim)
        y64 = ho.hmult(x)
        y32 = ho.hmult(x.astype(np.float32).astype(np.float64))
        xd = torch.tensor(x, device="cuda")
        xf = xd.to(torch.float32)
        n64, n32 = len(h.launch_shapes("f64")), len(h.launch_shapes("f32"))
        assert any(sh["kind"] == 1 for sh in h.launch_shapes("f32")), h.launch_shapes("f32")
        try:
            for i in range(max(n64, n32)):
                ctx.set_kernel_path(16 + i)
                assert np.array_equal(h.hmult(xd).cpu().numpy(), y64), (sec, i)
                yf = h.hmult(xf).double().cpu().numpy()
                assert np.abs(yf - y32).max() <= 1.2e-7 * np.abs(y32).max(), (sec, i)
        finally:
            ctx.set_kernel_path(0)


def test_fp32_hop_sums_every_launch_shape(ctx):
    """FP32 hop sums (edk_ctx_set_fp32_sums) at every launch shape on the
    ns=14 (7,7) and (8,7) sectors: H*v of the FP32-rounded input within
    2e-6 of the largest element of the oracle's FP64 H*v (eight FP32 products
    per spin summed in FP32 against the FP64 sums)."""
    import torch
    m = workload("c3").model
    rng = np.random.default_rng(17)
    ctx.set_fp32_sums(True, 1)
    try:
        for sec in [(7, 7), (8, 7)]:
            h = edk.Hamiltonian(ctx, m, *sec)
            ho = O.OracleH(m, *sec)
            x = rng.normal(size=h.dim).astype(np.float32)
            y = ho.hmult(x.astype(np.float64))
            xf = torch.tensor(x, device="cuda")
            n = len(h.launch_shapes("f32"))
            assert n > 0
            for i in range(n):
                ctx.set_kernel_path(16 + i)
                yf = h.hmult(xf).double().cpu().numpy()
                assert np.abs(yf - y).max() <= 2e-6 * np.abs(y).max(), (sec, i, h.launch_shapes("f32")[i])
    finally:
        ctx.set_kernel_path(0)
        ctx.set_fp32_sums(False)


def test_launch_shape_timed_once_per_sector_shape():
    """The fast kernel's launch shape is timed on the first H*v of a sector
    shape; a second Hamiltonian of the same shape in the same context reuses
    it (one launch per H*v) and gives the same bits."""
    import torch
    c = edk.Context(0)
    try:
        m = workload("c3").model
        x = torch.tensor(np.random.default_rng(3).normal(size=3432 * 3432), device="cuda")
        h1 = edk.Hamiltonian(c, m, 7, 7)
        n0 = c.launches
        y1 = h1.hmult(x)
        tuned = c.launches - n0
        assert tuned > 1                    # the feasible shapes were timed
        h2 = edk.Hamiltonian(c, m, 7, 7)
        n1 = c.launches
        y2 = h2.hmult(x)
        assert c.launches - n1 == 1
        assert torch.equal(y1, y2)
        h3 = edk.Hamiltonian(c, m, 7, 6)    # another shape: timed again
        n2 = c.launches
        h3.hmult(torch.zeros(h3.dim, dtype=torch.float64, device="cuda"))
        assert c.launches - n2 > 1
    finally:
        c.close()


@pytest.mark.parametrize("name,sec", [("c3", (7, 7)), ("c3", (7, 6)), ("c5", (9, 8)), ("c5", (8, 8))])
def test_lean_kernel_fp32_sums(ctx, name, sec):
    """The lean FP32 row kernels (kind 3: two rows staged interleaved by
    column, packed FP32x2 FMAs; kind 5: the same arithmetic in two passes,
    the down-spin hops from L2-resident column tiles) at each of their launch
    shapes: H*v of an
    FP32-rounded input within 2e-6 of the largest element of the oracle's
    FP64 H*v, and a 40-step Green chain whose Lanczos coefficients agree with
    the FP64 chain's to 2e-5 relative (FP32 vectors and hop sums against
    FP64 throughout)."""
    import torch
    m = workload(name).model
    ctx.set_fp32_sums(True, 1)
    try:
        h = edk.Hamiltonian(ctx, m, *sec)
        shapes = h.launch_shapes("f32")
        lean = [i for i, sh in enumerate(shapes) if sh["kind"] in (3, 5)]
        assert {shapes[i]["kind"] for i in lean} == {3, 5}, shapes
        rng = np.random.default_rng(5)
        x = rng.normal(size=h.dim).astype(np.float32)
        y = O.OracleH(m, *sec).hmult(x.astype(np.float64))
        xf = torch.tensor(x, device="cuda")
        ctx.set_kernel_path(0)
        start = torch.tensor(rng.normal(size=h.dim), device="cuda")
        wn = np.pi / 50.0 * (2 * np.arange(16) + 1)
        G64, a64, b64, n64 = h.green_chain(start, 40, 0.0, 1, wn)
        for i in lean:
            ctx.set_kernel_path(16 + i)
            yf = h.hmult(xf).double().cpu().numpy()
            assert np.abs(yf - y).max() <= 2e-6 * np.abs(y).max(), (sec, shapes[i])
            G32, a32, b32, n32 = h.green_chain(start.to(torch.float32), 40, 0.0, 1, wn)
            assert n32 == n64 == 40
            scale = np.abs(a64).max() + np.abs(b64).max()
            assert np.abs(a32 - a64).max() <= 2e-5 * scale, (sec, shapes[i], np.abs(a32 - a64).max())
            assert np.abs(b32 - b64).max() <= 2e-5 * scale, (sec, shapes[i], np.abs(b32 - b64).max())
            assert np.abs(G32 - G64).max() <= 2e-5 * np.abs(G64).max()
    finally:
        ctx.set_kernel_path(0)
        ctx.set_fp32_sums(False)


def _jj_model():
    """Two orbitals with U' and a density-density J (JJ) but no Hund spin-flip
    or pair-hop coupling (Jhund = 0): the split form applies (the reference
    STOPs in it only for |Jhund| > 1e-5) and differs from HAIMupdo_multr by
    the missing -JJ terms."""
    rng = np.random.default_rng(31)
    m = star_model(-1.0, 3.0, rng.uniform(-1, 1, 4), rng.uniform(0.2, 0.6, 4), orbital_of_bath=[0, 1, 1, 0],
                   nc=2, J=0.5)
    m.ec[:, 0, 1] = m.ec[:, 1, 0] = 0.3
    m.jhund = 0.0
    return m


@pytest.mark.parametrize("name,sec", [("c1", (4, 4)), ("c1", (3, 5)), ("jj", (3, 3)), ("jj", (2, 4)),
                                      ("c5", (8, 8))])
def test_hmult_split_fp64_bit_exact(ctx, name, sec):
    """edk_hmult_split (HAIMupdo_multr_split) against the oracle's restatement
    of the split form, bit for bit in FP64 (the ns=16 sector included); equal
    to edk_hmult where the model has no -JJ terms, different where it has."""
    import torch
    m = _jj_model() if name == "jj" else workload(name).model
    h = edk.Hamiltonian(ctx, m, *sec)
    ho = O.OracleH(m, *sec)
    x = np.random.default_rng(41).normal(size=h.dim)
    xd = torch.tensor(x, device="cuda")
    y = h.hmult_split(xd).cpu().numpy()
    y_ref = ho.hmult_split(x)
    assert np.array_equal(y, y_ref), np.abs(y - y_ref).max()
    if name == "jj":
        assert not np.array_equal(y, ho.hmult(x))
    else:
        assert np.array_equal(y, h.hmult(xd).cpu().numpy())
    # FP32 vectors: FP64 accumulation, the pass-1 partial sums stored in FP32
    xf = xd.to(torch.float32)
    yf = h.hmult_split(xf).double().cpu().numpy()
    y32 = ho.hmult_split(x.astype(np.float32).astype(np.float64))
    assert np.abs(yf - y32).max() <= 2.5e-7 * np.abs(y32).max()


def test_hmult_split_rejects_hund_models(ctx):
    """The reference STOPs in the split form when |Jhund| > 1e-5; the library
    returns EDK_ERR_UNSUPPORTED (and the oracle None)."""
    import torch
    m = workload("c2").model
    h = edk.Hamiltonian(ctx, m, 5, 5)
    assert O.OracleH(m, 5, 5).hmult_split(np.zeros(h.dim)) is None
    with pytest.raises(edk.EdkError) as e:
        h.hmult_split(torch.zeros(h.dim, dtype=torch.float64, device="cuda"))
    assert e.value.code == edk.EDK_ERR_UNSUPPORTED


def test_launch_shape_chosen_is_reported():
    """edk_h_launch_shape_chosen reports nothing before the first launch of a
    sector shape in a context and the timed choice after it, also on a second
    handle of the same sector shape."""
    import torch
    c = edk.Context(0)
    try:
        m = workload("c3").model
        h1 = edk.Hamiltonian(c, m, 7, 6)
        assert h1.launch_shape_chosen("f64", False) is None
        h1.hmult(torch.zeros(h1.dim, dtype=torch.float64, device="cuda"))
        s1 = h1.launch_shape_chosen("f64", False)
        assert s1 is not None and s1 in h1.launch_shapes("f64")
        h2 = edk.Hamiltonian(c, m, 7, 6)
        assert h2.launch_shape_chosen("f64", False) == s1
    finally:
        c.close()
