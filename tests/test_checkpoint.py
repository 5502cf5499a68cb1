"""GS.raw eigenstate checkpoints and ed.sector_bound_file (host-only C-ABI):
round trips are bit-exact, and the reader takes the list-directed layouts a
Fortran WRITE(UNIT,*) produces (line breaks inside vectors, repeat counts,
D exponents, .TRUE./.FALSE., quoted sector names, commas)."""
import os

import numpy as np
import pytest

from ed_solver_b200 import edk


def test_round_trip_is_bit_exact(tmp_path):
    rng = np.random.default_rng(0)
    v1 = rng.standard_normal(7)
    v1[2] = -0.0
    v1[3] = 1e-300
    v1[4] = -3.5e300
    ents = [
        dict(kind=0, norbs=8, nup=4, ndn=4, val=-9.321080867574677, converged=True, rank=1, vec=v1),
        dict(kind=0, norbs=8, nup=4, ndn=4, val=-9.3, converged=False, rank=2, vec=rng.standard_normal(5)),
        dict(kind=0, norbs=8, nup=3, ndn=4, val=np.nextafter(-9.0, 0.0), converged=True, rank=1, vec=np.zeros(0)),
        dict(kind=1, norbs=16, nup=8, ndn=-1, val=1.25, converged=True, rank=1, vec=rng.standard_normal(9)),
    ]
    p = str(tmp_path / "GS.raw")
    edk.gs_write(p, ents)
    back = edk.gs_read(p)
    assert len(back) == len(ents)
    for a, b in zip(ents, back):
        for k in ("kind", "norbs", "nup", "ndn", "rank"):
            assert a[k] == b[k]
        assert a["val"] == b["val"] and bool(a["converged"]) == b["converged"]
        assert np.array_equal(np.asarray(a["vec"]).view(np.uint64), b["vec"].view(np.uint64))
    # one eigensector per run of equal sectors: T, sector, states, F ... final F
    lines = open(p).read().split("\n")
    assert lines[0].strip() == "T" and lines[1].strip() == "updo"
    assert [l.strip() for l in lines[-3:]] == ["F", "F", ""]


def test_empty_list(tmp_path):
    p = str(tmp_path / "GS.raw")
    edk.gs_write(p, [])
    assert open(p).read().split() == ["F"]
    assert edk.gs_read(p) == []


FORTRAN_STYLE = """ T
 'updo'
           6
           3
           6
           2
 .TRUE.
  -4.1250000000000000
 T
           1
           4
   1.0000000000000000D-01, 2*-0.50000000000000000
  0.25E+00
 F
 T
 sz
          12
           6
 T
   3.0000000000000000     
 F
           2
           3
 3*7.0
 F
 F
"""


def test_reads_fortran_list_directed_layout(tmp_path):
    p = str(tmp_path / "GS.raw")
    with open(p, "w") as f:
        f.write(FORTRAN_STYLE)
    e = edk.gs_read(p)
    assert len(e) == 2
    assert (e[0]["kind"], e[0]["norbs"], e[0]["nup"], e[0]["ndn"]) == (0, 6, 3, 2)
    assert e[0]["val"] == -4.125 and e[0]["converged"] and e[0]["rank"] == 1
    assert np.array_equal(e[0]["vec"], [0.1, -0.5, -0.5, 0.25])
    assert (e[1]["kind"], e[1]["norbs"], e[1]["nup"]) == (1, 12, 6)
    assert e[1]["val"] == 3.0 and not e[1]["converged"] and e[1]["rank"] == 2
    assert np.array_equal(e[1]["vec"], [7.0, 7.0, 7.0])


@pytest.mark.parametrize("bad", [" T\n 'xyz'\n 1\n 1\n F\n", " T\n updo\n 6\n 3\n 6\n", "garbage\n"])
def test_malformed_files_are_rejected(tmp_path, bad):
    p = str(tmp_path / "GS.raw")
    with open(p, "w") as f:
        f.write(bad)
    with pytest.raises(edk.EdkError):
        edk.gs_read(p)


def test_missing_file_is_rejected(tmp_path):
    with pytest.raises(edk.EdkError):
        edk.gs_read(str(tmp_path / "nothing"))


def test_sector_bounds(tmp_path):
    p = str(tmp_path / "ed.sector_bound_file")
    edk.sector_bounds_write(p, (3, 5), (2, 4))
    assert edk.sector_bounds_read(p) == ((3, 5), (2, 4), (1000, -1000))
    with open(p, "w") as f:
        f.write("  3  5\n  2  4\n")          # no Sz record (READ ..., end=31)
    assert edk.sector_bounds_read(p) == ((3, 5), (2, 4), None)
    with open(p, "w") as f:
        f.write(" 1 2\n 3 4\n 5 6\n")
    assert edk.sector_bounds_read(p) == ((1, 2), (3, 4), (5, 6))
