"""edk_cf_eval_noalloc (static device scratch, no allocation) against edk_cf_eval.

Both entry points are called through the C-ABI with the same host inputs; the
results must agree within 1e-12 (the bound the continued-fraction tests use),
on consecutive calls that share the static scratch array.
"""
import ctypes as C

import numpy as np
import pytest

from ed_solver_b200 import edk
from ed_solver_b200.model import matsubara

pytestmark = pytest.mark.gpu

TOL = 1e-12
SCRATCH_BYTES = 4194304


def _bind(name):
    f = getattr(edk.lib(), name)
    P, I32 = C.c_void_p, C.c_int32
    f.restype = C.c_int
    f.argtypes = [P, I32, I32, P, P, P, P, P, P, I32, P, P]
    return f


def _chains(seed, nchain, ld):
    rng = np.random.default_rng(seed)
    n = rng.integers(1, ld + 1, nchain).astype(np.int32)
    diag = rng.normal(size=(nchain, ld))
    sub = rng.uniform(0.2, 1.0, (nchain, ld))
    sub[:, 0] = 0.0
    e = rng.normal(size=nchain)
    ph = np.where(np.arange(nchain) % 2 == 0, 1.0, -1.0)
    scale = rng.uniform(0.1, 1.0, nchain)
    return n, diag, sub, e, ph, scale


def _call(name, ctx, n, diag, sub, e, ph, scale, wn):
    G = np.zeros((len(n), len(wn), 2))
    rc = _bind(name)(ctx.h, len(n), diag.shape[1], n.ctypes.data, diag.ctypes.data, sub.ctypes.data,
                     e.ctypes.data, ph.ctypes.data, scale.ctypes.data, len(wn), wn.ctypes.data, G.ctypes.data)
    return rc, G[..., 0] + 1j * G[..., 1]


@pytest.fixture(scope="module")
def nctx():
    c = edk.Context(0)
    yield c
    c.close()


def test_noalloc_matches_cf_eval_on_consecutive_calls(nctx):
    for seed, (nchain, ld, nw) in enumerate([(24, 300, 512), (7, 1200, 1024)]):
        args = _chains(seed, nchain, ld)
        wn = matsubara(40.0 + seed, nw)
        rc_ref, G_ref = _call("edk_cf_eval", nctx, *args, wn)
        rc, G = _call("edk_cf_eval_noalloc", nctx, *args, wn)
        assert rc_ref == 0 and rc == 0
        assert np.abs(G - G_ref).max() <= TOL * max(1.0, np.abs(G_ref).max())


def test_noalloc_allocates_nothing(nctx):
    """The device's free memory, torch's allocator counters and the current
    device are the same before and after a call (after a first call has
    resolved the array's address)."""
    import torch
    args = _chains(11, 16, 400)
    wn = matsubara(25.0, 256)
    rc0, G0 = _call("edk_cf_eval_noalloc", nctx, *args, wn)
    assert rc0 == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    stats0 = {k: v for k, v in torch.cuda.memory_stats(0).items() if k.endswith(".allocated") or "segment" in k}
    dev0 = torch.cuda.current_device()
    for _ in range(3):
        rc, G = _call("edk_cf_eval_noalloc", nctx, *args, wn)
        assert rc == 0
        assert np.array_equal(G, G0)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    stats1 = {k: v for k, v in torch.cuda.memory_stats(0).items() if k.endswith(".allocated") or "segment" in k}
    assert free1 == free0
    assert stats1 == stats0
    assert torch.cuda.current_device() == dev0


def test_noalloc_flag_cleared_between_calls(nctx):
    # a zero denominator sets the flag; the next call starts from a cleared flag
    n = np.array([1], np.int32)
    diag = np.array([[0.5]])
    sub = np.zeros((1, 1))
    one = np.ones(1)
    e = np.array([0.5])
    rc, _ = _call("edk_cf_eval_noalloc", nctx, n, diag, sub, e, one, one, np.zeros(1))
    assert rc == edk.EDK_ERR_CF_ZERO_DEN
    args = _chains(5, 10, 64)
    wn = matsubara(30.0, 128)
    rc_ref, G_ref = _call("edk_cf_eval", nctx, *args, wn)
    rc, G = _call("edk_cf_eval_noalloc", nctx, *args, wn)
    assert rc_ref == 0 and rc == 0
    assert np.abs(G - G_ref).max() <= TOL * max(1.0, np.abs(G_ref).max())


def test_noalloc_rejects_sizes_beyond_the_static_maximum(nctx):
    nchain, ld = 64, 4096                     # 2 x 64 x 4096 doubles alone exceed 4 MiB
    args = _chains(9, nchain, ld)
    wn = matsubara(10.0, 16)
    rc, _ = _call("edk_cf_eval_noalloc", nctx, *args, wn)
    assert rc == edk.EDK_ERR_INVALID
    msg = edk.lib().edk_ctx_last_error(nctx.h).decode()
    assert "scratch" in msg and str(SCRATCH_BYTES) in msg
    # the array is still usable afterwards
    args = _chains(10, 3, 50)
    rc_ref, G_ref = _call("edk_cf_eval", nctx, *args, wn)
    rc, G = _call("edk_cf_eval_noalloc", nctx, *args, wn)
    assert rc_ref == 0 and rc == 0
    assert np.abs(G - G_ref).max() <= TOL * max(1.0, np.abs(G_ref).max())
