"""C-ABI library: loads, exports every declared symbol, host-only entry points
bit-exact with the oracle (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle as O
from ed_solver_b200 import edk
from ed_solver_b200.model import workload, star_model, default_ran_tab

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            syms |= set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*\**(edk_\w+)\s*\(", txt, re.M))
    return syms


def test_library_exports_every_declared_symbol():
    L = C.CDLL(edk.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_fortran_module_binds_every_declared_symbol():
    """The ISO_C_BINDING module names every entry point of include/*.h (and
    nothing else) in its bind(C) interfaces."""
    f90 = open(os.path.join(ROOT, "ed_solver_b200", "fortran", "edk_fortran.f90")).read()
    bound = set(re.findall(r'bind\(C,\s*name="(edk_\w+)"\)', f90))
    assert bound == declared_symbols(), (declared_symbols() - bound, bound - declared_symbols())


def _header_arity():
    """Number of parameters of every declared entry point."""
    out = {}
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", f)).read(), flags=re.S)
        for name, args in re.findall(r"(?:^|\n)\s*(?:int|int64_t|const char \*)\s*\**(edk_\w+)\s*\(([^;]*?)\)\s*;",
                                     txt, re.S):
            a = args.strip()
            out[name] = 0 if a in ("", "void") else a.count(",") + 1
    return out


def test_fortran_interfaces_have_the_c_argument_counts():
    """Each bind(C) interface of the Fortran module declares as many dummy
    arguments as the C prototype has parameters."""
    f90 = open(os.path.join(ROOT, "ed_solver_b200", "fortran", "edk_fortran.f90")).read()
    f90 = re.sub(r"&\s*\n\s*&?", " ", f90)
    fort = {}
    for name, args, cname in re.findall(r"(?:function|subroutine)\s+(edk_\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(edk_\w+)\"\)",
                                        f90, re.I):
        a = args.strip()
        fort[cname] = 0 if not a else a.count(",") + 1
    arity = _header_arity()
    assert set(arity) == declared_symbols()
    bad = {k: (arity[k], fort.get(k)) for k in arity if fort.get(k) != arity[k]}
    assert not bad, bad


def test_basis_and_rank_bit_exact():
    for ns in (1, 4, 8, 11, 16):
        for np_ in range(ns + 1):
            assert np.array_equal(edk.basis(ns, np_), O.basis(ns, np_))
        assert np.array_equal(edk.rank_table(ns), O.rank_table(ns))


@pytest.mark.parametrize("name", ["c1", "c2", "c3", "c4"])
def test_tables_bit_exact(name):
    m = workload(name).model
    for spin in (0, 1):
        for np_ in range(m.ns + 1):
            p, t, v, d = edk.build_table(m, spin, np_)
            h = O.OracleH(m, np_, 0) if spin == 0 else O.OracleH(m, 0, np_)
            _, p2, t2, v2, d2 = h.table(spin)
            assert np.array_equal(p, p2) and np.array_equal(t, t2)
            assert np.array_equal(v, v2) and np.array_equal(d, d2)


def test_tables_with_cutoff_and_offdiagonal_blocks():
    rng = np.random.default_rng(4)
    m = star_model(-1.0, 3.0, rng.uniform(-1, 1, 4), [0.3, 0.0005, 0.2, 0.4], orbital_of_bath=[0, 1, 0, 1],
                   nc=2, J=0.4)
    m.ec[:, 0, 1] = m.ec[:, 1, 0] = 0.2
    m.eb[:, 1, 3] = m.eb[:, 3, 1] = -0.15
    m.vbc[1] *= 1.1   # spin-dependent hybridisation
    for spin in (0, 1):
        for np_ in range(m.ns + 1):
            p, t, v, d = edk.build_table(m, spin, np_)
            h = O.OracleH(m, np_, 0) if spin == 0 else O.OracleH(m, 0, np_)
            _, p2, t2, v2, d2 = h.table(spin)
            assert np.array_equal(t, t2) and np.array_equal(v, v2) and np.array_equal(d, d2)


def test_default_start_table_matches_python_restatement():
    assert np.array_equal(edk.default_ran_tab(), default_ran_tab())


def test_invalid_models_are_rejected():
    m = star_model(-1.0, 2.0, [0.1, 0.2], [0.3, 0.4])
    m.eb[0, 0, 1] = 0.5     # not symmetric
    with pytest.raises(edk.EdkError):
        edk.build_table(m, 0, 1)
    m2 = star_model(-1.0, 2.0, [0.1], [0.3], nc=1)
    m2.nc = 9               # more impurity sites than supported
    with pytest.raises(Exception):
        edk.build_table(m2, 0, 1)


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "ed_solver_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cpp", ".h")):
                txt = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in re.sub(r"#.*|//.*", "", txt).lower() or f == "__init__.py", f
