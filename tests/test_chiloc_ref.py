"""The chi~_loc checker: the reference's own chi_tilde_loc_ compiled from its
C++ source (oracle/_ref), and the full-ED inputs the oracle builds for it."""
import os

import numpy as np
import pytest

import oracle as O
from ed_solver_b200.model import star_model

REF_SRC = os.path.join(os.environ.get("ED_SOLVER_REF", "/root/reference"), "ed_solver", "Chiloc_Wenhu_version3.cpp")


def _need_ref():
    if O.ref_chiloc_lib() is None and os.path.exists(REF_SRC):
        import subprocess
        subprocess.check_call(["make", "-s", "-C", os.path.dirname(O.__file__), "ref"])
        O._REF_CHILOC = None
    if O.ref_chiloc_lib() is None:
        pytest.skip("reference vertex kernel not built (reference sources absent)")


def _model():
    rng = np.random.default_rng(1)
    return star_model(-1.0, 2.0, rng.uniform(-1, 1, 3), rng.uniform(0.3, 0.6, 3))


def test_chiloc_inputs_sum_rule():
    """sum over targets of |<t|c+|s>|^2 = <s| c c+ |s> = 1 - <s|n|s> for every eigenstate s."""
    m = _model()
    E, M, V = O.chiloc_inputs(m, 2, 2)
    for mat, (t, s, spin) in enumerate(O.CHILOC_MATRICES):
        if M[mat] is None:
            continue
        nu, nd = 2 + O.CHILOC_SECTORS[s][0], 2 + O.CHILOC_SECTORS[s][1]
        h = O.OracleH(m, nu, nd)
        bit = m.nb
        st = O.basis(m.ns, nu if spin == 0 else nd)
        occ_sp = ((st >> np.uint64(bit)) & np.uint64(1)).astype(float)
        occ = np.kron(np.ones(h.ddn), occ_sp) if spin == 0 else np.kron(occ_sp, np.ones(h.dup))
        n_s = (V[s] ** 2 * occ[:, None]).sum(axis=0)
        assert np.allclose((M[mat] ** 2).sum(axis=0), 1.0 - n_s, atol=1e-12)


def test_reference_kernel_runs_and_is_real_at_symmetric_frequencies():
    """The compiled reference returns finite values; with w3 = conj(w1)... the
    DNDN and UPDN values of (w, -w) pairs are complex conjugates (real H)."""
    _need_ref()
    m = _model()
    E, M, V = O.chiloc_inputs(m, 2, 2)
    beta = 10.0
    es = np.concatenate([e for e in E if e is not None])
    Z, gs = float(np.exp(-beta * (es - es.min())).sum()), float(es.min())
    nu = lambda n: 1j * (2 * n + 1) * np.pi / beta
    w = (nu(0), nu(1), nu(-2))
    wc = tuple(-x for x in w)
    a = O.ref_chiloc(1, w, 1e-5, beta, Z, gs, m.ns, 2, 2, E, M)[0]
    b = O.ref_chiloc(1, wc, 1e-5, beta, Z, gs, m.ns, 2, 2, E, M)[0]
    assert np.isfinite(a) and abs(a - np.conj(b)) < 1e-12 * max(1.0, abs(a))
    a = O.ref_chiloc(2, w, 1e-5, beta, Z, gs, m.ns, 2, 2, E, M)[1]
    b = O.ref_chiloc(2, wc, 1e-5, beta, Z, gs, m.ns, 2, 2, E, M)[1]
    assert np.isfinite(a) and abs(a - np.conj(b)) < 1e-12 * max(1.0, abs(a))
