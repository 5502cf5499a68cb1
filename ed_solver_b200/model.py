"""Anderson impurity model description and the synthetic configurations.

The model mirrors what the reference assembles into ``AIM_type``
(ed_solver/quantum_algebra_Anderson_Impurity_class.f90:12-87) and the globals
``JJmatrix``/``Jhund`` (ed_solver/Global_Variables.f90:55-56,
ed_solver/dmft_ed_solver.f90:185-206):

* per spin species, bath site k sits on bit k and impurity site c on bit nb+c;
* ``ec[s]`` (nc x nc) impurity quadratic part, ``eb[s]`` (nb x nb) bath
  quadratic part, ``vbc[s]`` (nb x nc) hybridisation, s = 0 (up), 1 (down);
* ``u`` (nc x nc): U(c,c) on-site, U(c,c') density-density between sites;
* ``jj`` (nc x nc) and the scalar gate ``jhund``: Hund terms (same-spin -J on
  the diagonal, spin flip and pair hopping), active when |jhund| > 1e-5 and U
  has an off-diagonal element (ed_solver/HAIMupdo.f90:1017,1087).

Kanamori parameters map onto the reference's convention as U(c,c)=U,
U(c,c')=U'=U-2J, JJ(c,c')=J (ed_solver/HAIMupdo.f90:798-829).

The five synthetic workloads are seeded restatements of the benchmark
configurations (numpy ``default_rng(seed)``, bath energies drawn before
hybridisations).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Tuple

import numpy as np


@dataclasses.dataclass
class AIMModel:
    nc: int
    nb: int
    ec: np.ndarray      # (2, nc, nc)
    eb: np.ndarray      # (2, nb, nb)
    vbc: np.ndarray     # (2, nb, nc)
    u: np.ndarray       # (nc, nc)
    jj: np.ndarray      # (nc, nc)
    jhund: float = 0.0
    cutoff: float = 1e-3    # cutoff_hamilt_param (reference default)

    @property
    def ns(self) -> int:
        return self.nc + self.nb

    def copy(self) -> "AIMModel":
        return AIMModel(self.nc, self.nb, self.ec.copy(), self.eb.copy(), self.vbc.copy(),
                        self.u.copy(), self.jj.copy(), float(self.jhund), float(self.cutoff))

    def arrays(self):
        """Contiguous float64 arrays in the layout the C-ABI expects."""
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        return f(self.ec), f(self.eb), f(self.vbc), f(self.u), f(self.jj)


def star_model(eps_imp, U, eps_bath, V, orbital_of_bath=None, nc=1, Uprime=None, J=0.0,
               cutoff=1e-3) -> AIMModel:
    """Star-geometry AIM: diagonal bath, each bath site hybridised with one orbital.

    ``eps_imp`` scalar or length-nc, ``eps_bath``/``V`` length-nb,
    ``orbital_of_bath[k]`` the impurity orbital bath site k couples to.
    """
    eps_bath = np.asarray(eps_bath, dtype=np.float64)
    V = np.asarray(V, dtype=np.float64)
    nb = len(eps_bath)
    if orbital_of_bath is None:
        orbital_of_bath = np.zeros(nb, dtype=int)
    eps_imp = np.broadcast_to(np.asarray(eps_imp, dtype=np.float64), (nc,))
    ec = np.zeros((2, nc, nc))
    eb = np.zeros((2, nb, nb))
    vbc = np.zeros((2, nb, nc))
    for s in range(2):
        ec[s][np.arange(nc), np.arange(nc)] = eps_imp
        eb[s][np.arange(nb), np.arange(nb)] = eps_bath
        for k in range(nb):
            vbc[s, k, orbital_of_bath[k]] = V[k]
    u = np.zeros((nc, nc))
    jj = np.zeros((nc, nc))
    up = U - 2.0 * J if Uprime is None else Uprime
    for a in range(nc):
        for b in range(nc):
            u[a, b] = U if a == b else up
            jj[a, b] = J
    return AIMModel(nc, nb, ec, eb, vbc, u, jj, jhund=float(J), cutoff=cutoff)


@dataclasses.dataclass
class NambuModel:
    """Superconducting AIM in the Nambu (Sz) basis: ``base`` plus the bath
    pairing ``pb`` (nb x nb, Pb(k,k') of bath_class.f90:956-986) and, when the
    reference's PAIRING_IMP_TO_BATH is on, the impurity-to-bath pairing
    ``pvbc`` (2, nb, nc) (bath_class.f90:998-1022).  ``on_fly`` selects the
    term order of HAIMsz_mult_fly_r (ed_solver/HAIMsz.f90:615-808) instead of
    the tabulated HAIMsz_multr (ed_solver/HAIMsz.f90:453-589); the on-the-fly
    order keeps every non-zero element (no cutoff_hamilt_param).

    The sector of ``npart`` Nambu particles in 2*ns orbitals holds the states
    with N_up + (ns - N_dn) = npart: up orbitals on bits 0..ns-1 as in one spin
    species of the (N_up, N_dn) basis, down holes on bits ns..2ns-1.
    Eigenvalues of the Nambu operator plus ``energy_shift`` are the physical
    energies (eigen_sector_class.f90:329).
    """
    base: AIMModel
    pb: np.ndarray
    pvbc: Optional[np.ndarray] = None
    on_fly: bool = False

    @property
    def nc(self) -> int:
        return self.base.nc

    @property
    def nb(self) -> int:
        return self.base.nb

    @property
    def ns(self) -> int:
        return self.base.ns

    @property
    def energy_shift(self) -> float:
        """energy_global_shift + energy_global_shift2: the down-spin diagonal of Ec and Eb."""
        m = self.base
        s1 = 0.0
        for c in range(m.nc):
            s1 += float(m.ec[1, c, c])
        s2 = 0.0
        for k in range(m.nb):
            s2 += float(m.eb[1, k, k])
        return s1 + s2


def nambu_star_model(eps_imp, U, eps_bath, V, delta, cutoff=1e-3, on_fly=False, pvbc=None) -> NambuModel:
    """One-orbital star AIM with an s-wave superconducting bath: Pb = diag(delta)."""
    base = star_model(eps_imp, U, eps_bath, V, cutoff=cutoff)
    delta = np.asarray(delta, dtype=np.float64)
    pb = np.diag(np.broadcast_to(delta, (base.nb,)).copy())
    return NambuModel(base, pb, None if pvbc is None else np.asarray(pvbc, np.float64), bool(on_fly))


def nambu_workload(ns: int, seed: int = 7, on_fly: bool = False) -> NambuModel:
    """Seeded one-orbital superconducting AIM with ns-1 bath sites: U=2 at half
    filling, bath levels uniform in [-2,2], hybridisations in [0.2,0.5], pairing
    amplitudes in [0.1,0.4] (numpy default_rng(seed), drawn in that order)."""
    rng = np.random.default_rng(seed)
    nb = ns - 1
    eb = rng.uniform(-2.0, 2.0, nb)
    v = rng.uniform(0.2, 0.5, nb)
    d = rng.uniform(0.1, 0.4, nb)
    return nambu_star_model(-1.0, 2.0, eb, v, d, on_fly=on_fly)


# --------------------------------------------------------------------------
# synthetic workloads
# --------------------------------------------------------------------------

@dataclasses.dataclass
class Workload:
    name: str
    model: AIMModel
    sectors: List[Tuple[int, int]]        # sectors scanned for the ground state
    beta: float
    nw: int
    nitermax: int = 1000
    nitergreen: int = 200
    neigen: int = 1
    tolerance: float = 1e-12
    demax0: float = 5.0                   # Boltzmann window dEmax = demax0 / beta
    description: str = ""


def _all_sectors(ns):
    return [(a, b) for a in range(ns + 1) for b in range(ns + 1)]


def workload(name: str) -> Workload:
    """The five synthetic configurations (seeded, shapes as specified)."""
    if name == "c1":
        rng = np.random.default_rng(0)
        eb = rng.uniform(-1.0, 1.0, 7)
        v = rng.uniform(0.2, 0.6, 7)
        m = star_model(-1.0, 2.0, eb, v)
        return Workload("c1", m, [(4, 4)], beta=50.0, nw=1024, nitergreen=200, neigen=1,
                        description="1 imp + 7 bath (ns=8), U=2, sector (4,4) D=4900")
    if name == "c2":
        rng = np.random.default_rng(1)
        eb = rng.uniform(-2.0, 2.0, 8)
        v = rng.uniform(0.1, 0.5, 8)
        U, J = 4.0, 0.7
        m = star_model(-(3 * U - 5 * J) / 2, U, eb, v, orbital_of_bath=[0] * 4 + [1] * 4, nc=2, J=J)
        return Workload("c2", m, _all_sectors(10), beta=40.0, nw=512, nitergreen=200, neigen=1,
                        description="2 orb + 8 bath (ns=10), Kanamori U=4 J=0.7, all 121 sectors")
    if name == "c3":
        rng = np.random.default_rng(2)
        eb = np.linspace(-2.0, 2.0, 13)
        v = 0.3 * (1.0 + 0.1 * rng.standard_normal(13))
        m = star_model(-1.5, 3.0, eb, v)
        return Workload("c3", m, [(7, 7)], beta=50.0, nw=512, nitergreen=300, neigen=1,
                        description="1 imp + 13 bath (ns=14), U=3, sector (7,7) D=1.18e7")
    if name == "c4":
        rng = np.random.default_rng(3)
        eb = rng.uniform(-2.0, 2.0, 10)
        v = rng.uniform(0.1, 0.5, 10)
        U, J = 3.5, 0.6
        m = star_model(-(3 * U - 5 * J) / 2, U, eb, v, orbital_of_bath=[0] * 5 + [1] * 5, nc=2, J=J)
        return Workload("c4", m, _all_sectors(12), beta=20.0, nw=512, nitergreen=200, neigen=3,
                        demax0=math.log(1e8),
                        description="2 orb + 10 bath (ns=12), U=3.5 J=0.6, beta=20, Boltzmann window 1e-8")
    if name == "c5":
        rng = np.random.default_rng(4)
        eb = rng.uniform(-2.0, 2.0, 15)
        v = rng.uniform(0.15, 0.45, 15)
        m = star_model(-1.25, 2.5, eb, v)
        return Workload("c5", m, [(8, 8)], beta=50.0, nw=512, nitergreen=300, neigen=1,
                        description="1 imp + 15 bath (ns=16), U=2.5, sector (8,8) D=1.66e8")
    raise KeyError(name)


def matsubara(beta: float, nw: int, fermionic: bool = True) -> np.ndarray:
    """Imaginary parts of the Matsubara axis (ed_solver/frequency_axis.f90:154-180):
    fermionic (2n-1)*pi/beta, bosonic 2n*pi/beta, n = 1..nw."""
    n = np.arange(1, nw + 1, dtype=np.float64)
    if fermionic:
        return (2.0 * math.pi / beta) * n - math.pi / beta
    return (2.0 * math.pi / beta) * n


# --------------------------------------------------------------------------
# start-vector table
# --------------------------------------------------------------------------

def default_ran_tab() -> np.ndarray:
    """The 10001-entry table behind the fixed Lanczos start vector.

    The reference fills ``ran_tab(0:10000)`` from gfortran ``random_number``
    (seed 1234567) rounded to 3 decimals (ed_solver/random.f90:684-704) and sets
    v(i) = ran_tab(modi(i,10000)) (ed_solver/rcvector_class.f90:43-60).  That
    generator is compiler-specific, so this library uses splitmix64 seeded with
    1234567, each draw mapped to [0,1) as (z >> 11) * 2**-53 and rounded to 3 decimals
    half away from zero as the reference's ANINT does.  A caller that
    holds the reference's own table passes it instead.
    """
    out = np.empty(10001, dtype=np.float64)
    x = 1234567
    mask = (1 << 64) - 1
    for i in range(10001):
        x = (x + 0x9E3779B97F4A7C15) & mask
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z = z ^ (z >> 31)
        u = (z >> 11) * (1.0 / 9007199254740992.0)
        out[i] = math.floor(u * 1000.0 + 0.5) / 1000.0   # ANINT: half away from zero
    return out
