"""Drivers above the Krylov C-ABI, mirroring the reference's L4 layer.

* ``solve_sector``   - get_eigen_energies + get_GS for one sector
  (ed_solver/solver.h:98-237, ed_solver/Lanczos_plain.f90:33-229), with dense
  diagonalisation below FULL_ED_SWITCH (ed_solver/ED_ARPACK.f90:590-715);
* ``ground_states``  - the sector scan and global Boltzmann window
  (ed_solver/eigen_class.f90:322-450, ed_solver/dmft_ed_solver.f90:1468);
* ``green_impurity`` - compute_greenAA for the (c, c+) channel
  (ed_solver/green_class_computeAA.f90:40-185) with the real-H symmetric
  combinations (ed_solver/green_class_compute_symmetric_combination.f90:39-138)
  and the off-diagonal reshuffle (..._AA.h:10-60).

Every vector operation runs on the GPU through ``ed_solver_b200.edk``.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import edk
from .model import AIMModel, matsubara

FULL_ED_SWITCH = 40   # ed_solver/Global_Variables.f90:23


class HCache:
    """Keeps one device Hamiltonian per sector alive across calls."""

    def __init__(self, ctx: edk.Context, model: AIMModel):
        self.ctx, self.model = ctx, model
        self._h: Dict[Tuple[int, int], edk.Hamiltonian] = {}

    def get(self, sector) -> edk.Hamiltonian:
        sector = tuple(sector)
        if sector not in self._h:
            self._h[sector] = edk.Hamiltonian(self.ctx, self.model, *sector)
        return self._h[sector]

    def close(self):
        for h in self._h.values():
            h.close()
        self._h.clear()


def _dense(h: edk.Hamiltonian, dtype="f64"):
    """Dense H built column by column with Hmult__ on the device (ED_ARPACK.f90:620-626)."""
    import torch
    eye = torch.eye(h.dim, dtype=torch.float64, device=f"cuda:{h.ctx.device}")
    cols = [h.hmult(eye[i].contiguous()) for i in range(h.dim)]
    return torch.stack(cols, 1).cpu().numpy()


def solve_sector(hc: HCache, sector, neigen=1, nitermax=1000, tolerance=1e-12, demax=1e300,
                 dtype="f64", ran_tab=None, check_every=8):
    """Eigenpairs of one sector: list of dict(E, psi (device tensor), niter)."""
    import torch
    h = hc.get(sector)
    if h.dim == 0:
        return []
    if h.dim <= FULL_ED_SWITCH:
        H = _dense(h)
        w, v = np.linalg.eigh(H)
        j = min(h.dim, neigen)
        keep = [0] + [i for i in range(1, j) if w[i] <= w[0] + demax]
        dev = f"cuda:{h.ctx.device}"
        tdt = torch.float64 if dtype in ("f64", edk.EDK_F64) else torch.float32
        return [dict(E=float(w[i]), psi=torch.tensor(v[:, i], dtype=tdt, device=dev), niter=0) for i in keep]
    r = h.lanczos_e0(dtype=dtype, nitermax=nitermax, neigen=neigen, tolerance=tolerance, demax=demax,
                     ran_tab=ran_tab, check_every=check_every)
    out = []
    for k in range(len(r["E"])):
        psi = h.lanczos_gs(r["vecp"][k], dtype=dtype, ran_tab=ran_tab)
        out.append(dict(E=float(r["E"][k]), psi=psi, niter=r["niter"]))
    return out


def ground_states(hc: HCache, sectors, beta: float, demax0: float, neigen=1, nitermax=1000,
                  tolerance=1e-12, dtype="f64", ran_tab=None):
    demax = demax0 / beta
    found = []
    for sec in sectors:
        states = solve_sector(hc, sec, neigen=neigen, nitermax=nitermax, tolerance=tolerance,
                              demax=demax, dtype=dtype, ran_tab=ran_tab)
        if not states:
            continue
        es = min(s["E"] for s in states)
        for s in states:
            if s["E"] <= es + demax:
                found.append(dict(sector=tuple(sec), **s))
    e0 = min(f["E"] for f in found)
    gs = [f for f in found if f["E"] <= e0 + demax]
    z = sum(math.exp(-beta * (f["E"] - e0)) for f in gs)
    for f in gs:
        f["boltz"] = math.exp(-beta * (f["E"] - e0)) / z
    return gs, e0, z


def green_impurity(hc: HCache, gs, beta: float, nw: int, nitergreen: int, spin: int = 0,
                   pairs: Optional[Sequence[Tuple[int, int]]] = None, cutoff_dynamic=1e-8,
                   dtype=None):
    """G_ij(i w_n) of the impurity orbitals for one spin (compute_greenAA, (c,c+) channel)."""
    model = hc.model
    nc = model.nc
    if pairs is None:
        pairs = [(i, i) for i in range(nc)]
    wn = matsubara(beta, nw)
    combos = sorted(set([(i, i) for (i, j) in pairs] + [(j, j) for (i, j) in pairs] +
                        [(min(i, j), max(i, j)) for (i, j) in pairs if i != j]))
    raw = {c: np.zeros(nw, complex) for c in combos}
    ns = model.ns
    for st in gs:
        nu, nd = st["sector"]
        h_src = hc.get(st["sector"])
        psi = st["psi"]
        if dtype is not None:
            psi = psi.to(dtype)
        for iph in (1, 2):
            dagger = iph == 1
            d = 1 if dagger else -1
            tsec = (nu + d, nd) if spin == 0 else (nu, nd + d)
            if not (0 <= tsec[0] <= ns and 0 <= tsec[1] <= ns):
                continue
            h_t = hc.get(tsec)
            for (i, j) in combos:
                if i == j:
                    v, _ = h_src.apply_c(psi, i, spin, dagger)
                else:
                    v, _ = h_src.apply_c(psi, i, spin, dagger, site2=j, sign2=1)
                G, _, _, _ = h_t.green_chain(v, nitergreen, st["E"], iph, wn, cutoff_dynamic)
                raw[(i, j)] += st["boltz"] * G
    out = {}
    for (i, j) in pairs:
        if i == j:
            out[(i, j)] = raw[(i, i)]
        else:
            a, b = min(i, j), max(i, j)
            out[(i, j)] = 0.5 * (raw[(a, b)] - raw[(a, a)] - raw[(b, b)])
    return out


# ---------------------------------------------------------------------------
# Nambu (Sz) sectors: the superconducting branch of get_eigen_energies and
# compute_greenAA (AIM%bath%SUPER, force_sz_basis)
# ---------------------------------------------------------------------------

class HCacheSz:
    """One device Nambu Hamiltonian per sector (npart) kept alive across calls."""

    def __init__(self, ctx: edk.Context, model):
        self.ctx, self.model = ctx, model
        self._h: Dict[int, edk.HamiltonianSz] = {}

    def get(self, npart: int) -> edk.HamiltonianSz:
        if npart not in self._h:
            self._h[npart] = edk.HamiltonianSz(self.ctx, self.model, npart)
        return self._h[npart]

    def close(self):
        for h in self._h.values():
            h.close()
        self._h.clear()


def ground_states_sz(hc: HCacheSz, nparts, beta: float, demax0: float, neigen=1, nitermax=1000,
                     tolerance=1e-12, dtype="f64"):
    """Sector scan over Nambu sectors and the global window.  Energies stay
    those of the Nambu operator (solve_AIM shifts them back before get_GS and
    the Green functions, solver.f90:87-94); the physical E0 is e0 + shift (the
    same shift for every sector, so window and weights do not change)."""
    import torch
    demax = demax0 / beta
    found = []
    for npart in nparts:
        h = hc.get(npart)
        if h.dim == 0:
            continue
        if h.dim <= FULL_ED_SWITCH:
            w, v = np.linalg.eigh(_dense(h))
            j = min(h.dim, neigen)
            keep = [0] + [i for i in range(1, j) if w[i] <= w[0] + demax]
            dev = f"cuda:{h.ctx.device}"
            states = [dict(E=float(w[i]), psi=torch.tensor(v[:, i], device=dev)) for i in keep]
        else:
            r = h.lanczos_e0(dtype=dtype, nitermax=nitermax, neigen=neigen, tolerance=tolerance, demax=demax)
            states = [dict(E=float(r["E"][k]), psi=h.lanczos_gs(r["vecp"][k], dtype=dtype)) for k in range(len(r["E"]))]
        es = min(s["E"] for s in states)
        found += [dict(npart=npart, **s) for s in states if s["E"] <= es + demax]
    e0 = min(f["E"] for f in found)
    gs = [f for f in found if f["E"] <= e0 + demax]
    z = sum(math.exp(-beta * (f["E"] - e0)) for f in gs)
    for f in gs:
        f["boltz"] = math.exp(-beta * (f["E"] - e0)) / z
    shift = hc.get(gs[0]["npart"]).energy_shift
    return gs, e0, z, shift


def green_nambu(hc: HCacheSz, gs, beta: float, nw: int, nitergreen: int, orbs=None, cutoff_dynamic=1e-8):
    """G_ab(i w_n) over Nambu impurity orbitals (compute_greenAA on the Nambu
    AIM2): a, b in [0, 2nc), a < nc the up orbital, a >= nc the hole orbital
    (so G_{0,nc} is the anomalous function of site 0).  Particle chains from
    b+_a|psi>, hole chains from b_a|psi>; off-diagonal elements from the
    symmetric combination b_a + b_b (green_class_compute_symmetric_combination.f90:39-138):
    G_ab = (G_{a+b} - G_aa - G_bb) / 2.  Returns {(a, b): G}."""
    nc = hc.model.nc
    if orbs is None:
        orbs = list(range(2 * nc))
    wn = matsubara(beta, nw)
    pairs = [(a, a) for a in orbs] + [(a, b) for i, a in enumerate(orbs) for b in orbs[i + 1:]]
    raw = {p: np.zeros(nw, complex) for p in pairs}
    ns2 = 2 * hc.model.ns
    for st in gs:
        h_src = hc.get(st["npart"])
        for iph in (1, 2):
            dagger = iph == 1
            npt = st["npart"] + (1 if dagger else -1)
            if not 0 <= npt <= ns2:
                continue
            h_t = hc.get(npt)
            for (a, b) in pairs:
                v, _ = h_src.apply_b(st["psi"], a, dagger, orb2=(b if b != a else -1), sign2=1)
                G, _, _, _ = h_t.green_chain(v, nitergreen, st["E"], iph, wn, cutoff_dynamic)
                raw[(a, b)] += st["boltz"] * G
    out = {}
    for (a, b) in pairs:
        out[(a, b)] = raw[(a, b)] if a == b else 0.5 * (raw[(a, b)] - raw[(a, a)] - raw[(b, b)])
    return out


def green_ab_nambu(hc: HCacheSz, gs, beta: float, nw: int, nitergreen: int, spin: int = 0, sites=None,
                   proj_a: bool = True, proj_b: bool = False, cutoff_dynamic=1e-8):
    """compute_greenAB (green_class_computeAB.f90:23-212) in the Nambu basis for
    two impurity operators of one spin: A = c (projected: apply_Csz_N_updo,
    apply_C.f90:404-483) and B = c (apply_Csz_updo).  With A projected and B
    plain this is the GNF channel of correlations_dyn_stat.h:96.  For every
    state |psi> (weight boltz): particle chains from (A+_i + B+_j)|psi> and hole
    chains from (A_i + B_j)|psi> (symmetric_combineAB,
    green_class_compute_symmetric_combination.f90:155-262, real H), then
    G_AB(i, j) = (G_{A_i+B_j} - G_{A_i A_i} - G_{B_j B_j}) / 2
    (reshuffle_vecAB, green_class_compute_symmetric_combination_AB.h:50-69).
    Returns {(i, j): G} over the impurity sites."""
    nc = hc.model.nc
    if sites is None:
        sites = list(range(nc))
    wn = matsubara(beta, nw)
    keys = [("ab", i, j) for i in sites for j in sites] + [("aa", i, i) for i in sites] + \
           [("bb", j, j) for j in sites]
    raw = {k: np.zeros(nw, complex) for k in keys}
    ns2 = 2 * hc.model.ns
    for st in gs:
        h_src = hc.get(st["npart"])
        for iph in (1, 2):
            dagger = iph == 1
            create = dagger if spin == 0 else not dagger
            npt = st["npart"] + (1 if create else -1)
            if not 0 <= npt <= ns2:
                continue
            h_t = hc.get(npt)
            for (kind, i, j) in keys:
                pa, pb = {"ab": (proj_a, proj_b), "aa": (proj_a, proj_a), "bb": (proj_b, proj_b)}[kind]
                if kind == "ab":
                    v, _ = h_src.apply_c_ab(st["psi"], i, pa, j, pb, spin, dagger)
                else:
                    v, _ = h_src.apply_c(st["psi"], i, spin, dagger, projected=pa)
                G, _, _, _ = h_t.green_chain(v, nitergreen, st["E"], iph, wn, cutoff_dynamic)
                raw[(kind, i, j)] += st["boltz"] * G
    return {(i, j): 0.5 * (raw[("ab", i, j)] - raw[("aa", i, i)] - raw[("bb", j, j)])
            for i in sites for j in sites}
