"""Python side of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Wraps ``oracle/_build/liborc.so`` (the C restatement in ``edk_oracle.c``) and
adds, in numpy:

* ``dense_sector_h``: an independent second-quantised build of the sector
  Hamiltonian (standard Jordan-Wigner algebra, Kanamori terms), used to pin the
  C restatement of HAIMupdo_multr element by element;
* the drivers that sit above the Krylov primitives in the reference:
  the sector scan and Boltzmann window of get_eigen_energies
  (ed_solver/solver.h:98-237, ed_solver/eigen_class.f90:322-450) and the
  Green-function loop of compute_greenAA (ed_solver/green_class_computeAA.f90:40-185,
  ed_solver/green_class_computeAA.h:101-302) with the symmetric combinations of
  ed_solver/green_class_compute_symmetric_combination.f90:39-138 and the
  off-diagonal reshuffle of ed_solver/green_class_compute_symmetric_combination_AA.h:10-60.

Only tests, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg import
this module; the product never does.  Parity of this oracle is pinned by the
reference's golden output test/2b/bm/g_bm (see tests/golden) plus analytic
limits and dense diagonalisation; the reference's gfortran start-vector table
is not reproducible, so its exact Lanczos coefficient sequence is unpinned.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
import sys
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(_HERE)
if _REPO not in sys.path:
    sys.path.insert(0, _REPO)

from ed_solver_b200.model import AIMModel, default_ran_tab, matsubara  # noqa: E402

_LIB = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liborc.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        d = C.c_double
        i32 = C.c_int
        i64 = C.c_int64
        L.orc_binom.restype = i64
        L.orc_binom.argtypes = [i32, i32]
        L.orc_basis.restype = i64
        L.orc_basis.argtypes = [i32, i32, P]
        L.orc_rank_table.argtypes = [i32, P]
        L.orc_h_new.restype = P
        L.orc_h_new.argtypes = [P, i32, i32]
        L.orc_h_free.argtypes = [P]
        for f in ("orc_h_dim", "orc_h_dup", "orc_h_ddn"):
            getattr(L, f).restype = i64
            getattr(L, f).argtypes = [P]
        L.orc_h_table.restype = i64
        L.orc_h_table.argtypes = [P, i32, P, P, P, P, P]
        L.orc_hmult.argtypes = [P, P, P]
        L.orc_hmult_split.argtypes = [P, P, P]
        L.orc_hmult_split.restype = C.c_int
        L.orc_tridiag_eig.restype = i32
        L.orc_tridiag_eig.argtypes = [i32, P, P, P, P]
        L.orc_fix_initial_vector.argtypes = [i64, P, P]
        L.orc_lanczos_e0.restype = i32
        L.orc_lanczos_e0.argtypes = [P, P, i32, i32, d, d, d, P, P, P, P, P, P]
        L.orc_lanczos_gs.restype = i32
        L.orc_lanczos_gs.argtypes = [P, P, i32, P, d, P]
        L.orc_apply_c.restype = i32
        L.orc_apply_c.argtypes = [i32, i32, i32, i32, i32, i32, i32, P, P]
        L.orc_cf.restype = i32
        L.orc_cf.argtypes = [i32, P, P, d, d, P, P]
        L.orc_green_chain.restype = i32
        L.orc_green_chain.argtypes = [P, P, i32, d, i32, i32, P, d, d, P, P, P]
        L.orc_double_occ.restype = d
        L.orc_double_occ.argtypes = [P, P, i32]
        L.orc_num_threads.restype = i32
        L.orc_lanczos_steps.restype = i32
        L.orc_lanczos_steps.argtypes = [P, P, i32, P, P]
        L.orc_h_new_sz.restype = P
        L.orc_h_new_sz.argtypes = [P, i32]
        L.orc_sz_shift.restype = d
        L.orc_sz_shift.argtypes = [P]
        L.orc_sz_table.restype = i64
        L.orc_sz_table.argtypes = [P, P, P, P, P, P, P]
        L.orc_apply_csz.restype = i32
        L.orc_apply_csz.argtypes = [P, i32, i32, i32, i32, P, P]
        L.orc_colex_rank.restype = i64
        L.orc_colex_rank.argtypes = [C.c_uint64]
        _LIB = L
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class _CModel(C.Structure):
    _fields_ = [("nc", C.c_int32), ("nb", C.c_int32), ("ec", C.c_void_p), ("eb", C.c_void_p),
                ("vbc", C.c_void_p), ("u", C.c_void_p), ("jj", C.c_void_p),
                ("jhund", C.c_double), ("cutoff", C.c_double)]


def _cmodel(m: AIMModel):
    arrs = m.arrays()
    cm = _CModel(m.nc, m.nb, *[a.ctypes.data for a in arrs], float(m.jhund), float(m.cutoff))
    return cm, arrs


# ---------------------------------------------------------------------------
# basis
# ---------------------------------------------------------------------------

def binom(n, k) -> int:
    return int(lib().orc_binom(n, k))


def basis(ns: int, np_: int) -> np.ndarray:
    out = np.zeros(max(binom(ns, np_), 1), dtype=np.uint64)
    n = lib().orc_basis(ns, np_, _p(out))
    return out[:n]


def rank_table(ns: int) -> np.ndarray:
    out = np.zeros(1 << ns, dtype=np.int32)
    lib().orc_rank_table(ns, _p(out))
    return out


# ---------------------------------------------------------------------------
# sector Hamiltonian
# ---------------------------------------------------------------------------

class OracleH:
    """new_H / Hmult__ / delete_H for one (N_up, N_dn) sector (HAIMupdo.f90:53-121,677-1195)."""

    def __init__(self, model: AIMModel, nup: int, ndn: int):
        self.model = model
        self.nup, self.ndn = nup, ndn
        cm, self._keep = _cmodel(model)
        self._cm = cm
        self.h = lib().orc_h_new(C.byref(cm), nup, ndn)
        if not self.h:
            raise ValueError("unsupported model")
        self.dim = int(lib().orc_h_dim(self.h))
        self.dup = int(lib().orc_h_dup(self.h))
        self.ddn = int(lib().orc_h_ddn(self.h))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_h_free(h)
            self.h = None

    def hmult(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.dim, dtype=np.float64)
        lib().orc_hmult(self.h, _p(x), _p(y))
        return y

    def hmult_split(self, x: np.ndarray) -> np.ndarray:
        """HAIMupdo_multr_split (HAIMupdo.f90:1221-1347): up hops, transpose,
        down hops as up hops, transpose back; no -JJ density terms.  None where
        the reference STOPs (|Jhund| > 1e-5)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.dim, dtype=np.float64)
        if lib().orc_hmult_split(self.h, _p(x), _p(y)) != 0:
            return None
        return y

    def table(self, spin: int):
        d = self.dup if spin == 0 else self.ddn
        nnz = int(lib().orc_h_table(self.h, spin, None, None, None, None, None))
        st = np.zeros(d, np.uint64)
        ptr = np.zeros(d + 1, np.int64)
        tgt = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros(max(nnz, 1), np.float64)
        diag = np.zeros(d, np.float64)
        lib().orc_h_table(self.h, spin, _p(st), _p(ptr), _p(tgt), _p(val), _p(diag))
        return st, ptr, tgt[:nnz], val[:nnz], diag

    def dense(self) -> np.ndarray:
        """Dense matrix built column by column from Hmult__ (ED_diago, ED_ARPACK.f90:620-626)."""
        H = np.zeros((self.dim, self.dim))
        e = np.zeros(self.dim)
        for i in range(self.dim):
            e[i] = 1.0
            H[:, i] = self.hmult(e)
            e[i] = 0.0
        return H

    def double_occ(self, psi: np.ndarray, site: int = 0) -> float:
        psi = np.ascontiguousarray(psi, dtype=np.float64)
        return float(lib().orc_double_occ(self.h, _p(psi), site))


def start_vector(dim: int, ran_tab: Optional[np.ndarray] = None) -> np.ndarray:
    tab = default_ran_tab() if ran_tab is None else np.ascontiguousarray(ran_tab, np.float64)
    v = np.empty(dim, dtype=np.float64)
    lib().orc_fix_initial_vector(dim, _p(tab), _p(v))
    return v


def tridiag_eig(d: np.ndarray, e: np.ndarray, vectors: bool = False):
    n = len(d)
    d = np.ascontiguousarray(d, np.float64)
    e = np.ascontiguousarray(e, np.float64) if n > 1 else np.zeros(1)
    w = np.empty(n)
    z = np.empty((n, n)) if vectors else None
    lib().orc_tridiag_eig(n, _p(d), _p(e), _p(w), _p(z) if vectors else None)
    if vectors:
        return w, z.T.copy()   # columns are eigenvectors
    return w


def lanczos_e0(h: OracleH, v0=None, nitermax=1000, neigen=1, tolerance=1e-12, demax=1e300,
               cutoff_min=1e-25):
    """Pass 1 (Lanczos_plain.f90:33-134). Returns dict with E, niter, diag, subdiag, vecp, conv."""
    if v0 is None:
        v0 = start_vector(h.dim)
    v0 = np.ascontiguousarray(v0, np.float64)
    nmax = max(1, min(h.dim - 1, nitermax))
    E = np.zeros(64)
    niter = np.zeros(1, np.int32)
    diag = np.zeros(nmax + 1)
    sub = np.zeros(nmax + 1)
    vecp = np.zeros(64 * (nmax + 1))
    conv = np.zeros(64, np.int32)
    k = lib().orc_lanczos_e0(h.h, _p(v0), nitermax, neigen, tolerance, demax, cutoff_min,
                             _p(E), _p(niter), _p(diag), _p(sub), _p(vecp), _p(conv))
    if k < 0:
        raise RuntimeError(f"orc_lanczos_e0 failed ({k})")
    it = int(niter[0])
    return dict(E=E[:k].copy(), niter=it, diag=diag[:it].copy(), subdiag=sub[:it].copy(),
                vecp=vecp[:k * it].reshape(k, it).copy(), conv=conv[:k].copy())


def lanczos_steps(h: OracleH, nsteps: int, v0=None):
    """Runs nsteps plain Lanczos iterations (CPU-baseline sample); returns (alpha, beta)."""
    if v0 is None:
        v0 = start_vector(h.dim)
    v0 = np.ascontiguousarray(v0, np.float64)
    d = np.zeros(nsteps + 2)
    s = np.zeros(nsteps + 2)
    n = lib().orc_lanczos_steps(h.h, _p(v0), nsteps, _p(d), _p(s))
    return d[:n], s[:n + 1]


def num_threads() -> int:
    return int(lib().orc_num_threads())


def lanczos_gs(h: OracleH, coef: np.ndarray, v0=None, cutoff_min=1e-25) -> np.ndarray:
    """Pass 2 (Lanczos_plain.f90:156-229)."""
    if v0 is None:
        v0 = start_vector(h.dim)
    v0 = np.ascontiguousarray(v0, np.float64)
    coef = np.ascontiguousarray(coef, np.float64)
    psi = np.empty(h.dim)
    lib().orc_lanczos_gs(h.h, _p(v0), len(coef), _p(coef), cutoff_min, _p(psi))
    return psi


def apply_c(model: AIMModel, nup: int, ndn: int, site: int, spin: int, dagger: bool,
            vec: np.ndarray) -> Tuple[np.ndarray, Tuple[int, int]]:
    """apply_Cupdo (apply_C.f90:497-653). Returns (vector, target sector)."""
    ns = model.ns
    tnup = nup + ((1 if dagger else -1) if spin == 0 else 0)
    tndn = ndn + ((1 if dagger else -1) if spin == 1 else 0)
    if not (0 <= tnup <= ns and 0 <= tndn <= ns):
        raise ValueError("target sector out of range")
    out = np.zeros(binom(ns, tnup) * binom(ns, tndn))
    vec = np.ascontiguousarray(vec, np.float64)
    lib().orc_apply_c(ns, model.nb, nup, ndn, site, spin, int(dagger), _p(vec), _p(out))
    return out, (tnup, tndn)


def cf(diag: np.ndarray, subdiag: np.ndarray, z: complex) -> complex:
    d = np.ascontiguousarray(diag, np.float64)
    s = np.ascontiguousarray(subdiag, np.float64)
    r = np.zeros(1)
    i = np.zeros(1)
    if lib().orc_cf(len(d), _p(d), _p(s), z.real, z.imag, _p(r), _p(i)):
        raise ZeroDivisionError("zero denominator in continued fraction")
    return complex(r[0], i[0])


def green_chain(h: OracleH, opm: np.ndarray, nitergreen: int, e0: float, iph: int,
                wn: np.ndarray, cutoff_dynamic=1e-8, cutoff_min=1e-25):
    """compute_dynamic_cpu (green_class_compute_dynamic.f90:191-334). Returns (G, diag, subdiag)."""
    opm = np.ascontiguousarray(opm, np.float64)
    wn = np.ascontiguousarray(wn, np.float64)
    G = np.zeros(2 * len(wn))
    nmax = max(1, min(nitergreen, h.dim))
    dg = np.zeros(nmax)
    sd = np.zeros(nmax)
    n = lib().orc_green_chain(h.h, _p(opm), nitergreen, e0, iph, len(wn), _p(wn),
                              cutoff_dynamic, cutoff_min, _p(G), _p(dg), _p(sd))
    return G[0::2] + 1j * G[1::2], dg[:n].copy(), sd[:n].copy()


# ---------------------------------------------------------------------------
# independent dense build (second quantisation, numpy) for small sectors
# ---------------------------------------------------------------------------

def dense_sector_h(model: AIMModel, nup: int, ndn: int) -> np.ndarray:
    """Sector Hamiltonian from explicit fermion operators, per-spin Jordan-Wigner.

    H = sum_s sum_{a!=b} t^s_ab c+_{a s} c_{b s} + sum_s sum_a t^s_aa n_{a s}
      + sum_c U_cc n_c,up n_c,dn + sum_{c<c'} U_cc' n_c n_c'
      - sum_{c<c'} J_cc' (n_c,up n_c',up + n_c,dn n_c',dn)
      + [spin flip  J c+_{c,up} c_{c',up} c+_{c',dn} c_{c,dn}  + h.c.]
      + [pair hop   J c+_{c,up} c_{c',up} c+_{c,dn} c_{c',dn}  for c != c']
    with the Hund terms active only when |jhund| > 1e-5 and U has an
    off-diagonal element.  The hopping matrix t^s collects Ec, Eb and Vbc in
    the bit layout of the library; off-diagonal entries with |t| <= cutoff
    are dropped, as tab_HAIM2 does.
    """
    nc, nb, ns = model.nc, model.nb, model.ns
    su = [s for s in range(1 << ns) if bin(s).count("1") == nup]
    sd = [s for s in range(1 << ns) if bin(s).count("1") == ndn]
    ru = {s: i for i, s in enumerate(su)}
    rd = {s: i for i, s in enumerate(sd)}
    dup = len(su)
    D = dup * len(sd)
    H = np.zeros((D, D))

    def tmat(spin):
        t = np.zeros((ns, ns))
        t[nb:, nb:] = model.ec[spin]
        t[:nb, :nb] = model.eb[spin]
        t[:nb, nb:] = model.vbc[spin]
        t[nb:, :nb] = model.vbc[spin].T
        for a in range(ns):
            for b in range(ns):
                if a != b and not (abs(t[a, b]) > model.cutoff):
                    t[a, b] = 0.0
        return t

    def hop(s, a, b):
        """c+_a c_b |s> with per-species JW sign; returns (sign, state) or None."""
        if not (s >> b) & 1:
            return None
        s1 = s & ~(1 << b)
        sg = -1 if bin(s1 >> (b + 1)).count("1") & 1 else 1
        if (s1 >> a) & 1:
            return None
        s2 = s1 | (1 << a)
        if bin(s2 >> (a + 1)).count("1") & 1:
            sg = -sg
        return sg, s2

    tt = [tmat(0), tmat(1)]
    U, JJ = model.u, model.jj
    offc = any(U[a, b] != 0 for a in range(nc) for b in range(nc) if a != b)
    hund = abs(model.jhund) > 1e-5 and offc
    occ = lambda s, p: (s >> p) & 1
    for iu, s_u in enumerate(su):
        for id_, s_d in enumerate(sd):
            i = iu + id_ * dup
            e = 0.0
            for a in range(ns):
                e += tt[0][a, a] * occ(s_u, a) + tt[1][a, a] * occ(s_d, a)
            for c in range(nc):
                e += U[c, c] * occ(s_u, nb + c) * occ(s_d, nb + c)
            for c in range(nc):
                for c2 in range(c + 1, nc):
                    n1 = occ(s_u, nb + c) + occ(s_d, nb + c)
                    n2 = occ(s_u, nb + c2) + occ(s_d, nb + c2)
                    if U[c, c2] != 0:
                        e += U[c, c2] * n1 * n2
                        e -= JJ[c, c2] * (occ(s_u, nb + c) * occ(s_u, nb + c2) +
                                          occ(s_d, nb + c) * occ(s_d, nb + c2))
            H[i, i] += e
            for spin, s, rk in ((0, s_u, ru), (1, s_d, rd)):
                t = tt[spin]
                for a in range(ns):
                    for b in range(ns):
                        if a == b or t[a, b] == 0:
                            continue
                        r = hop(s, a, b)
                        if r is None:
                            continue
                        sg, s2 = r
                        j = (rk[s2] + id_ * dup) if spin == 0 else (iu + rk[s2] * dup)
                        H[j, i] += t[a, b] * sg
            if hund:
                for c in range(nc):
                    for c2 in range(nc):
                        if c == c2 or U[c, c2] == 0:
                            continue
                        pc, pc2 = nb + c, nb + c2
                        # spin flip: up c2 -> c, down c -> c2
                        ru_ = hop(s_u, pc, pc2)
                        rd_ = hop(s_d, pc2, pc)
                        if ru_ and rd_:
                            j = ru[ru_[1]] + rd[rd_[1]] * dup
                            H[j, i] += JJ[c, c2] * ru_[0] * rd_[0]
                        # pair hop: up and down c2 -> c
                        ru_ = hop(s_u, pc, pc2)
                        rd_ = hop(s_d, pc, pc2)
                        if ru_ and rd_:
                            j = ru[ru_[1]] + rd[rd_[1]] * dup
                            H[j, i] += JJ[c, c2] * ru_[0] * rd_[0]
    return H


# ---------------------------------------------------------------------------
# Nambu (Sz) sectors: HAIMsz (ed_solver/HAIMsz.f90:51-1027)
# ---------------------------------------------------------------------------

class _CModelSz(C.Structure):
    _fields_ = [("base", _CModel), ("pb", C.c_void_p), ("pvbc", C.c_void_p), ("on_fly", C.c_int32)]


def _cmodel_sz(m):
    cm, arrs = _cmodel(m.base)
    pb = np.ascontiguousarray(m.pb, np.float64)
    pv = None if m.pvbc is None else np.ascontiguousarray(m.pvbc, np.float64)
    cs = _CModelSz(cm, pb.ctypes.data, None if pv is None else pv.ctypes.data, int(bool(m.on_fly)))
    return cs, (arrs, pb, pv)


class OracleSz:
    """new_HAIMsz / HAIMsz_mult for the sector of `npart` Nambu particles.

    Usable wherever the oracle drivers take an OracleH (Lanczos passes, Green
    chains): the C handle dispatches H*v to the Nambu operator."""

    def __init__(self, model, npart: int):
        self.model = model
        self.npart = npart
        cs, self._keep = _cmodel_sz(model)
        self._cs = cs
        self.h = lib().orc_h_new_sz(C.byref(cs), npart)
        if not self.h:
            raise ValueError("unsupported Nambu model or sector")
        self.dim = int(lib().orc_h_dim(self.h))
        self.shift = float(lib().orc_sz_shift(self.h))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_h_free(h)
            self.h = None

    def hmult(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.dim, dtype=np.float64)
        lib().orc_hmult(self.h, _p(x), _p(y))
        return y

    def table(self):
        """(states, QUART_INT_SZ, diagsz, ptr, tgt, val) of the tabulated operator."""
        d = self.dim
        nnz = int(lib().orc_sz_table(self.h, None, None, None, None, None, None))
        st = np.zeros(d, np.uint64)
        q = np.zeros(d)
        dg = np.zeros(d)
        ptr = np.zeros(d + 1, np.int64)
        tgt = np.zeros(max(nnz, 1), np.int64)
        val = np.zeros(max(nnz, 1))
        lib().orc_sz_table(self.h, _p(st), _p(q), _p(dg), _p(ptr), _p(tgt), _p(val))
        return st, q, dg, ptr, tgt[:nnz], val[:nnz]

    def dense(self) -> np.ndarray:
        H = np.zeros((self.dim, self.dim))
        e = np.zeros(self.dim)
        for i in range(self.dim):
            e[i] = 1.0
            H[:, i] = self.hmult(e)
            e[i] = 0.0
        return H

    def apply_c(self, vec: np.ndarray, site: int, spin: int, dagger: bool, projected: bool = False):
        """apply_Csz_updo / apply_Csz_N_updo (apply_C.f90:344-483): (vector, target npart)."""
        vec = np.ascontiguousarray(vec, np.float64)
        create = bool(dagger) if spin == 0 else not dagger
        npt = self.npart + (1 if create else -1)
        if not 0 <= npt <= 2 * self.model.ns:
            raise ValueError("target sector out of range")
        out = np.zeros(binom(2 * self.model.ns, npt))
        r = lib().orc_apply_csz(self.h, site, spin, int(bool(dagger)), int(bool(projected)), _p(vec), _p(out))
        if r != npt:
            raise ValueError("orc_apply_csz failed")
        return out, npt


def green_ab_nambu(model, gs, beta: float, nw: int, nitergreen: int, spin: int = 0, sites=None,
                   proj_a: bool = True, proj_b: bool = False, cutoff_dynamic=1e-8):
    """compute_greenAB in the Nambu basis (ed_solver/green_class_computeAB.f90:23-212)
    for A = c of one spin, projected (apply_Csz_N_updo, ed_solver/apply_C.f90:404-483)
    or not (apply_Csz_updo), and B likewise: chains from the symmetric
    combinations (A+_i + B+_j)|psi> (particle) and (A_i + B_j)|psi> (hole) of
    symmetric_combineAB (ed_solver/green_class_compute_symmetric_combination.f90:155-262,
    real H), and G_AB(i,j) = (G_{A_i+B_j} - G_{A_iA_i} - G_{B_jB_j}) / 2
    (reshuffle_vecAB, ed_solver/green_class_compute_symmetric_combination_AB.h:50-69).
    gs: list of dict(npart, E, psi, boltz).  Returns {(i, j): G}."""
    nc = model.nc
    sites = list(range(nc)) if sites is None else list(sites)
    wn = matsubara(beta, nw)
    keys = [("ab", i, j) for i in sites for j in sites] + [("aa", i, i) for i in sites] + \
           [("bb", j, j) for j in sites]
    raw = {k: np.zeros(nw, complex) for k in keys}
    cache = {}

    def H(n):
        if n not in cache:
            cache[n] = OracleSz(model, n)
        return cache[n]

    for st in gs:
        hs = H(st["npart"])
        psi = np.asarray(st["psi"], np.float64)
        for iph in (1, 2):
            dagger = iph == 1
            create = dagger if spin == 0 else not dagger
            npt = st["npart"] + (1 if create else -1)
            if not 0 <= npt <= 2 * model.ns:
                continue
            for (kind, i, j) in keys:
                pa, pb = {"ab": (proj_a, proj_b), "aa": (proj_a, proj_a), "bb": (proj_b, proj_b)}[kind]
                v, _ = hs.apply_c(psi, i, spin, dagger, projected=pa)
                if kind == "ab":
                    v = v + hs.apply_c(psi, j, spin, dagger, projected=pb)[0]
                G, _, _ = green_chain(H(npt), v, nitergreen, st["E"], iph, wn, cutoff_dynamic=cutoff_dynamic)
                raw[(kind, i, j)] += st["boltz"] * G
    return {(i, j): 0.5 * (raw[("ab", i, j)] - raw[("aa", i, i)] - raw[("bb", j, j)]) for i in sites for j in sites}


def colex_rank(state: int) -> int:
    return int(lib().orc_colex_rank(int(state)))


def nambu_one_body(model) -> Tuple[np.ndarray, np.ndarray]:
    """The Nambu one-body matrix over the 2*ns bits (numpy, from the physical
    parameters): returns (h, bits) with h[a, b] the coefficient of b+_a b_b.
    Down-spin entries enter particle-hole transformed: -t_dn^T."""
    m = model.base
    nc, nb, ns = m.nc, m.nb, m.ns
    h = np.zeros((2 * ns, 2 * ns))
    up = lambda o: o
    hole = lambda o: ns + o
    imp = lambda c: nb + c
    for a in range(nc):
        for b in range(nc):
            h[up(imp(a)), up(imp(b))] += m.ec[0, a, b]
            h[hole(imp(a)), hole(imp(b))] -= m.ec[1, b, a]
    for k in range(nb):
        for l in range(nb):
            h[up(k), up(l)] += m.eb[0, k, l]
            h[hole(k), hole(l)] -= m.eb[1, l, k]
            h[up(k), hole(l)] += model.pb[k, l]
            h[hole(l), up(k)] += model.pb[k, l]
        for c in range(nc):
            for (a, b, t) in ((up(k), up(imp(c)), m.vbc[0, k, c]), (hole(k), hole(imp(c)), -m.vbc[1, k, c])):
                h[a, b] += t
                h[b, a] += t
            if model.pvbc is not None:
                for (a, b, t) in ((hole(k), up(imp(c)), model.pvbc[0, k, c]),
                                  (up(k), hole(imp(c)), model.pvbc[1, k, c])):
                    h[a, b] += t
                    h[b, a] += t
    return h


def dense_physical_sz(model, npart: int) -> np.ndarray:
    """Physical Hamiltonian on the fixed-Sz subspace N_up - N_dn = npart - ns,
    built from explicit fermion operators in an ordering unrelated to the Nambu
    one (spin-orbital index 2*o + spin, Jordan-Wigner over that order):

    H = sum_s t^s_ab c+_as c_bs + sum_kl Pb(k,l) (c+_k,up c+_l,dn + h.c.)
      + sum_kc PVbc_1(k,c) (c+_c,up c+_k,dn + h.c.) + PVbc_2(k,c) (c+_k,up c+_c,dn + h.c.)
      + sum_c U_cc n_c,up n_c,dn + sum_{c<c'} U_cc' n_c n_c'

    with t^s collecting Ec, Eb, Vbc.  Its eigenvalues equal those of the Nambu
    sector plus the energy shift."""
    m = model.base
    nc, nb, ns = m.nc, m.nb, m.ns
    no = 2 * ns
    idx = lambda o, s: 2 * o + s
    states = [st for st in range(1 << no)
              if sum((st >> idx(o, 0)) & 1 for o in range(ns)) - sum((st >> idx(o, 1)) & 1 for o in range(ns))
              == npart - ns]
    rk = {st: i for i, st in enumerate(states)}
    D = len(states)
    H = np.zeros((D, D))

    def op(st, p, create):
        occ = (st >> p) & 1
        if occ == create:
            return None
        sg = -1 if bin(st & ((1 << p) - 1)).count("1") & 1 else 1
        return sg, st ^ (1 << p)

    def apply_seq(st, ops):
        sg = 1
        for p, cr in reversed(ops):
            r = op(st, p, cr)
            if r is None:
                return None
            sg *= r[0]
            st = r[1]
        return sg, st

    terms = []     # (coef, [(p, create), ...]) applied right to left
    imp = lambda c: nb + c
    for s in range(2):
        t = np.zeros((ns, ns))
        t[nb:, nb:] = m.ec[s]
        t[:nb, :nb] = m.eb[s]
        t[:nb, nb:] = m.vbc[s]
        t[nb:, :nb] = m.vbc[s].T
        for a in range(ns):
            for b in range(ns):
                if t[a, b] != 0:
                    terms.append((t[a, b], [(idx(a, s), 1), (idx(b, s), 0)]))
    for k in range(nb):
        for l in range(nb):
            p = model.pb[k, l]
            if p != 0:
                terms.append((p, [(idx(k, 0), 1), (idx(l, 1), 1)]))
                terms.append((p, [(idx(l, 1), 0), (idx(k, 0), 0)]))
    if model.pvbc is not None:
        for k in range(nb):
            for c in range(nc):
                p1, p2 = model.pvbc[0, k, c], model.pvbc[1, k, c]
                if p1 != 0:
                    terms.append((p1, [(idx(imp(c), 0), 1), (idx(k, 1), 1)]))
                    terms.append((p1, [(idx(k, 1), 0), (idx(imp(c), 0), 0)]))
                if p2 != 0:
                    terms.append((p2, [(idx(k, 0), 1), (idx(imp(c), 1), 1)]))
                    terms.append((p2, [(idx(imp(c), 1), 0), (idx(k, 0), 0)]))
    for j, st in enumerate(states):
        n = lambda o, s: (st >> idx(o, s)) & 1
        e = 0.0
        for c in range(nc):
            e += m.u[c, c] * n(imp(c), 0) * n(imp(c), 1)
            for c2 in range(c + 1, nc):
                e += m.u[c, c2] * (n(imp(c), 0) + n(imp(c), 1)) * (n(imp(c2), 0) + n(imp(c2), 1))
        H[j, j] += e
        for coef, ops in terms:
            r = apply_seq(st, ops)
            if r is None:
                continue
            H[rk[r[1]], j] += coef * r[0]
    return H


# ---------------------------------------------------------------------------
# drivers above the Krylov primitives
# ---------------------------------------------------------------------------

FULL_ED_SWITCH = 40   # ed_solver/Global_Variables.f90:23


def solve_sector(model: AIMModel, nup: int, ndn: int, neigen=1, nitermax=1000, tolerance=1e-12,
                 demax=1e300, ran_tab=None):
    """Eigenpairs of one sector as get_eigen_energies/get_GS would produce them.

    dim <= FULL_ED_SWITCH: dense diagonalisation (ED_diago, ED_ARPACK.f90:590-715);
    otherwise Lanczos pass 1 + pass 2.  Returns list of (E, psi).
    """
    h = OracleH(model, nup, ndn)
    if h.dim == 0:
        return h, []
    if h.dim <= FULL_ED_SWITCH:
        w, v = np.linalg.eigh(h.dense())
        j = min(h.dim, neigen)
        keep = [0]
        for i in range(1, j):
            if w[i] <= w[0] + demax:
                keep.append(i)
            else:
                break
        return h, [(float(w[i]), v[:, i].copy()) for i in keep]
    v0 = start_vector(h.dim, ran_tab)
    r = lanczos_e0(h, v0, nitermax=nitermax, neigen=neigen, tolerance=tolerance, demax=demax)
    out = []
    for k in range(len(r["E"])):
        psi = lanczos_gs(h, r["vecp"][k], v0)
        out.append((float(r["E"][k]), psi))
    return h, out


def ground_states(model: AIMModel, sectors: Sequence[Tuple[int, int]], beta: float, demax0: float,
                  neigen=1, nitermax=1000, tolerance=1e-12, ran_tab=None):
    """Sector scan + global Boltzmann window [E0, E0 + demax0/beta]
    (solver.h:98-237, eigen_sector_class.f90:274-470, dmft_ed_solver.f90:1468)."""
    demax = demax0 / beta
    found = []
    for (nu, nd) in sectors:
        h, states = solve_sector(model, nu, nd, neigen=neigen, nitermax=nitermax,
                                 tolerance=tolerance, demax=demax, ran_tab=ran_tab)
        if states:
            e_s = min(e for e, _ in states)
            for e, psi in states:
                if e <= e_s + demax:
                    found.append(dict(sector=(nu, nd), E=e, psi=psi))
    e0 = min(f["E"] for f in found)
    gs = [f for f in found if f["E"] <= e0 + demax]
    z = sum(math.exp(-beta * (f["E"] - e0)) for f in gs)
    for f in gs:
        f["boltz"] = math.exp(-beta * (f["E"] - e0)) / z
    return gs, e0, z


def lehmann_small_sector(gs, tsec, v: np.ndarray, e_psi: float, iph: int, wn: np.ndarray,
                         cutoff_dynamic=1e-8) -> np.ndarray:
    """compute_dynamic_full_ed (ed_solver/green_class_compute_dynamic.f90:77-165),
    the branch compute_dynamic takes for target sectors of at most FULL_ED_SWITCH
    states (:44-62): with v = A|psi> unnormalised, the sum over the states |n> of
    the target sector that the window kept of |<n|v>|^2 / (i w - ph (E_n - E_psi))
    (:150-154, fermionic sign -1); zero when |v|^2 < cutoff_dynamic (:116-122) or
    when no state of that sector is kept (iisector == 0, :143)."""
    out = np.zeros(len(wn), complex)
    if float(v @ v) < cutoff_dynamic:
        return out
    ph = 1.0 if iph == 1 else -1.0
    for n in gs:
        if tuple(n["sector"]) != tuple(tsec):
            continue
        amp = float(n["psi"] @ v) ** 2
        out += amp / (1j * wn - ph * (n["E"] - e_psi))
    return out


def green_impurity(model: AIMModel, gs, beta: float, nw: int, nitergreen: int, spin: int = 0,
                   pairs: Optional[Sequence[Tuple[int, int]]] = None, cutoff_dynamic=1e-8,
                   reference_small_sectors: bool = False):
    """G_ij(i w_n) for impurity orbitals of one spin, the (c, c+) channel of compute_greenAA.

    For each state |psi> with weight boltz: particle part with |phi> = (c+_i [+ c+_j])|psi>,
    hole part with (c_i [+ c_j])|psi> (real-H symmetric combination), then
    G_ij = (G_{i+j} - G_ii - G_jj) / 2 for i != j.  Returns dict {(i,j): array(nw)}.
    reference_small_sectors: target sectors of at most FULL_ED_SWITCH states take
    the Lehmann branch (lehmann_small_sector) as the reference does; otherwise
    every target sector runs the continued fraction.
    """
    nc = model.nc
    if pairs is None:
        pairs = [(i, i) for i in range(nc)]
    wn = matsubara(beta, nw)
    combos = sorted(set([(i, i) for (i, j) in pairs] + [(j, j) for (i, j) in pairs] +
                        [(min(i, j), max(i, j)) for (i, j) in pairs if i != j]))
    raw = {c: np.zeros(nw, complex) for c in combos}
    hcache: Dict[Tuple[int, int], OracleH] = {}
    for st in gs:
        nu, nd = st["sector"]
        psi = st["psi"]
        for iph in (1, 2):
            dagger = iph == 1
            for (i, j) in combos:
                vi, tsec = _try_apply(model, nu, nd, i, spin, dagger, psi)
                if vi is None:
                    continue
                if i != j:
                    vj, _ = _try_apply(model, nu, nd, j, spin, dagger, psi)
                    v = vi + vj
                else:
                    v = vi
                if tsec not in hcache:
                    hcache[tsec] = OracleH(model, *tsec)
                if reference_small_sectors and hcache[tsec].dim <= FULL_ED_SWITCH:
                    G = lehmann_small_sector(gs, tsec, v, st["E"], iph, wn, cutoff_dynamic)
                else:
                    G, _, _ = green_chain(hcache[tsec], v, nitergreen, st["E"], iph, wn,
                                          cutoff_dynamic=cutoff_dynamic)
                raw[(i, j)] += st["boltz"] * G
    out = {}
    for (i, j) in pairs:
        if i == j:
            out[(i, j)] = raw[(i, i)]
        else:
            a, b = min(i, j), max(i, j)
            out[(i, j)] = 0.5 * (raw[(a, b)] - raw[(a, a)] - raw[(b, b)])
    return out


def _try_apply(model, nu, nd, site, spin, dagger, psi):
    try:
        return apply_c(model, nu, nd, site, spin, dagger, psi)
    except ValueError:
        return None, None


def lehmann_green(model: AIMModel, sectors, beta: float, wn: np.ndarray, site=0, spin=0,
                  demax=None):
    """Exact finite-temperature G_ii(i w_n) by full diagonalisation of small sectors."""
    ns = model.ns
    eig = {}
    for (nu, nd) in sectors:
        H = dense_sector_h(model, nu, nd)
        w, v = np.linalg.eigh(H)
        eig[(nu, nd)] = (w, v)
    e0 = min(w[0] for w, _ in eig.values())
    z = 0.0
    G = np.zeros(len(wn), complex)
    for (nu, nd), (w, v) in eig.items():
        for n in range(len(w)):
            if demax is not None and w[n] > e0 + demax:
                continue
            z += math.exp(-beta * (w[n] - e0))
    for (nu, nd), (w, v) in eig.items():
        tnu, tnd = (nu + 1, nd) if spin == 0 else (nu, nd + 1)
        if (tnu, tnd) not in eig:
            continue
        wt, vt = eig[(tnu, tnd)]
        for n in range(len(w)):
            bn = math.exp(-beta * (w[n] - e0))
            for m in range(len(wt)):
                bm = math.exp(-beta * (wt[m] - e0))
                if bn < 1e-300 and bm < 1e-300:
                    continue
                phi, _ = apply_c(model, nu, nd, site, spin, True, v[:, n])
                amp = float(vt[:, m] @ phi) ** 2
                G += amp * (bn + bm) / (1j * wn - (wt[m] - w[n]))
    return G / z


# ---------------------------------------------------------------------------
# chi~_loc: the reference's own chi_tilde_loc_ (ed_solver/Chiloc_Wenhu_version3.cpp),
# compiled unmodified into oracle/_ref by `make -C oracle ref`
# ---------------------------------------------------------------------------

CHILOC_SECTORS = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (0, 2), (0, -2), (1, 1), (-1, 1), (1, -1), (-1, -1)]
# (target slot, source slot, spin) of the 14 c+ matrices, in the reference's argument order
CHILOC_MATRICES = [(1, 0, 0), (2, 0, 1), (7, 1, 1), (7, 2, 0), (5, 2, 1), (0, 3, 0), (8, 3, 1),
                   (0, 4, 1), (9, 4, 0), (2, 8, 0), (1, 9, 1), (4, 10, 0), (3, 10, 1), (4, 6, 1)]
_REF_CHILOC = None


def ref_chiloc_path():
    return os.path.join(_HERE, "_ref", "libchiloc_ref.so")


def ref_chiloc_lib():
    """The compiled reference (oracle/_ref/libchiloc_ref.so); None when it was not built."""
    global _REF_CHILOC
    if _REF_CHILOC is None and os.path.exists(ref_chiloc_path()):
        _REF_CHILOC = C.CDLL(ref_chiloc_path())
    return _REF_CHILOC


def ref_chiloc(op, w, phi_eps, beta, Z, gs_e, sites, nup, ndn, E, M):
    """chi_tilde_loc_ of the reference for one frequency triple w = (w1, w2, w3):
    E[11] energy arrays, M[14] c+ matrices (target x source).  Returns
    (pDNDN, pUPDN) as Python complex numbers."""
    L = ref_chiloc_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libchiloc_ref.so is not built (make -C oracle ref)")
    ci = lambda v: C.byref(C.c_int(int(v)))
    cd = lambda v: C.byref(C.c_double(float(v)))
    keep = []

    def cplx(z):
        a = np.array([z.real, z.imag], np.float64)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    def arr(a):
        a = np.ascontiguousarray(a if a is not None and np.size(a) else np.zeros(1), np.float64).reshape(-1)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    args = [ci(op), cplx(w[0]), cplx(w[1]), cplx(w[2]), cd(phi_eps), cd(beta), cd(Z), cd(gs_e), ci(sites),
            ci(nup), ci(ndn)]
    for q in range(11):
        args += [arr(E[q]), ci(0 if E[q] is None else len(E[q]))]
    args += [ci(0)] * 28
    for m in range(14):
        args.append(arr(M[m]))
    out_d = np.zeros(2)
    out_u = np.zeros(2)
    args += [out_d.ctypes.data_as(C.c_void_p), out_u.ctypes.data_as(C.c_void_p)]
    L.chi_tilde_loc_(*args)
    return complex(out_d[0], out_d[1]), complex(out_u[0], out_u[1])


def chiloc_inputs(model: AIMModel, nup: int, ndn: int, site: int = 0):
    """Full-ED eigenpairs of the 11 sectors around (nup, ndn) (dense Hmult__
    columns, numpy eigh) and the 14 c+ matrices <t|c+_{site,spin}|s> between
    their eigenbases (apply_Cupdo on every eigenvector), as the reference's
    vertex tool assembles them (four_leg_vertex_matrices, Chiloc_four_leg.f90:200-444).
    Returns (E[11] (None for sectors outside the space), M[14], V[11])."""
    ns = model.ns
    E, V = [None] * 11, [None] * 11
    for q, (du, dd) in enumerate(CHILOC_SECTORS):
        nu, nd = nup + du, ndn + dd
        if 0 <= nu <= ns and 0 <= nd <= ns:
            w, v = np.linalg.eigh(OracleH(model, nu, nd).dense())
            E[q], V[q] = w, v
    M = [None] * 14
    for m, (t, s, spin) in enumerate(CHILOC_MATRICES):
        if V[t] is None or V[s] is None:
            continue
        nu, nd = nup + CHILOC_SECTORS[s][0], ndn + CHILOC_SECTORS[s][1]
        cols = []
        for j in range(V[s].shape[1]):
            out, _ = apply_c(model, nu, nd, site, spin, True, V[s][:, j])
            cols.append(out)
        CV = np.stack(cols, axis=1)                     # c+ V_s in the target's Fock basis
        M[m] = V[t].T @ CV                               # target x source
    return E, M, V
