"""Inputs of the local vertex chi~_loc on the device: full-ED eigenpairs of the
eleven sectors around (nup, ndn) (ED_diago, ED_ARPACK.f90:590-715) and the
fourteen c+ matrices between their eigenbases, as the reference's vertex tool
assembles them (four_leg_vertex_matrices, ed_solver/Chiloc_four_leg.f90:200-444).

The c+ images of every eigenvector come from the device c/c+ kernel
(edk_apply_c); the projection onto the target eigenbasis is a plain GEMM.
"""
from __future__ import annotations

import numpy as np

from . import edk

# sector offsets (d nup, d ndn) of the eleven slots, and (target, source, spin)
# of the fourteen matrices, in the order of chi_tilde_loc_'s arguments
SECTORS = [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (0, 2), (0, -2), (1, 1), (-1, 1), (1, -1), (-1, -1)]
MATRICES = [(1, 0, 0), (2, 0, 1), (7, 1, 1), (7, 2, 0), (5, 2, 1), (0, 3, 0), (8, 3, 1),
            (0, 4, 1), (9, 4, 0), (2, 8, 0), (1, 9, 1), (4, 10, 0), (3, 10, 1), (4, 6, 1)]


def vertex_inputs(ctx: edk.Context, model, nup: int, ndn: int, site: int = 0):
    """(E[11], M[14]): energies (None outside the Hilbert space) and c+ matrices."""
    import torch
    ns = model.ns
    E, V, H = [None] * 11, [None] * 11, [None] * 11
    for q, (du, dd) in enumerate(SECTORS):
        nu, nd = nup + du, ndn + dd
        if 0 <= nu <= ns and 0 <= nd <= ns:
            h = edk.Hamiltonian(ctx, model, nu, nd)
            E[q], V[q] = h.full_ed()
            H[q] = h
    dev = f"cuda:{ctx.device}"
    M = [None] * 14
    for m, (t, s, spin) in enumerate(MATRICES):
        if V[t] is None or V[s] is None:
            continue
        Vs = torch.tensor(V[s], device=dev)
        cols = [H[s].apply_c(Vs[:, j].contiguous(), site, spin, True)[0] for j in range(Vs.shape[1])]
        CV = torch.stack(cols, dim=1)                    # c+ V_s in the target's Fock basis
        M[m] = (torch.tensor(V[t], device=dev).T @ CV).cpu().numpy()
    return E, M


def partition(E, beta: float):
    """(Z, E_gs) over the sectors given, as the vertex tool normalises."""
    es = np.concatenate([e for e in E if e is not None])
    gs = es.min()
    return float(np.exp(-beta * (es - gs)).sum()), float(gs)
