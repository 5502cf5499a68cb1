"""Extracts the golden fixture from the reference's own test outputs.

Reads the reference's test/2b/bm/g_bm (1000 Matsubara rows x 8 columns: Re/Im
of G11, G12, G21, G22 of the two-orbital test at beta=50) and keeps the first
200 rows of G11 and G22 as tests/golden/g_bm_2b.txt; reads the deck's input
hybridisation test/2b/delta1.inp (the frequency, then Re/Im of Delta11,
Delta12, Delta21, Delta22) and keeps its first 200 rows of Delta11 and
Delta22 (fit_nw = 200 in test/2b/ED/ED.in) as tests/golden/delta_2b.txt.
Run in a container that has the reference checked out:

    python tests/golden/make_golden.py /path/to/reference

The model behind that output (test/2b/test.py:5-60, test/2b/PARAMS): two
orbitals, eps=-5, U=10, U'=2, J=0, beta=50, hybridisation Delta_11=0.2/iw,
Delta_22=0.3/iw, i.e. one bath level at 0 per orbital with V^2=0.2 and 0.3.
"""
import os
import sys

import numpy as np

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ED_SOLVER_REF", "/root/reference")
g = np.loadtxt(os.path.join(ref, "test", "2b", "bm", "g_bm"))
beta = 50.0
n = 200
wn = (2 * np.arange(1, n + 1) - 1) * np.pi / beta
out = np.column_stack([wn, g[:n, 0], g[:n, 1], g[:n, 6], g[:n, 7]])
here = os.path.dirname(os.path.abspath(__file__))
np.savetxt(os.path.join(here, "g_bm_2b.txt"), out, fmt="%.10f",
           header="wn ReG11 ImG11 ReG22 ImG22  (reference test/2b/bm/g_bm, first 200 rows)")
print("wrote", os.path.join(here, "g_bm_2b.txt"))
d = np.loadtxt(os.path.join(ref, "test", "2b", "delta1.inp"))
out = np.column_stack([d[:n, 0], d[:n, 1], d[:n, 2], d[:n, 7], d[:n, 8]])
np.savetxt(os.path.join(here, "delta_2b.txt"), out, fmt="%.12f",
           header="wn ReD11 ImD11 ReD22 ImD22  (reference test/2b/delta1.inp, first 200 rows)")
print("wrote", os.path.join(here, "delta_2b.txt"))
