"""The library's MPS reader (sp_read_mps) against the reference's own MPS tests
(crates/saddlepoint-io/src/lib.rs:327-381) and against the oracle's reader on every
Netlib fixture the reference ships: the same LP, array for array and bit for bit.
Host code only: these run without a GPU."""
import math

import numpy as np
import pytest

import oracle
from conftest import KNOWN_HARD, NETLIB, QUICK, SLOW, netlib_bytes
from test_oracle import MPS_SAMPLE

INF = math.inf


def sp():
    import saddlepoint_b200

    return saddlepoint_b200


def test_reads_all_sections():
    """io/src/lib.rs:361-375 on the library's reader."""
    p = sp().read_mps(MPS_SAMPLE)
    assert p.maximize
    assert list(p.c) == [-1.0, -2.0, 1.0]
    assert p.c0 == -3.5
    assert list(p.lc) == [1.5, 1.0, 7.0, 1.0]
    assert list(p.uc) == [4.0, INF, 7.0, 2.0]
    assert list(p.lv) == [0.0, -INF, -INF]
    assert list(p.uv) == [4.0, 1.0, INF]
    assert p.nnz == 6
    assert list(p.col_idx[p.row_ptr[2]:p.row_ptr[3]]) == [1, 2]
    assert list(p.values[p.row_ptr[2]:p.row_ptr[3]]) == [-1.0, 1.0]


def test_unknown_row_names_its_line():
    """io/src/lib.rs:377-381: the error names line 5."""
    with pytest.raises(sp().MpsError, match=r"^line 5: unknown row nope$"):
        sp().read_mps(b"NAME X\nROWS\n N obj\nCOLUMNS\n    x  nope  1\nENDATA\n")


@pytest.mark.parametrize("text,line,msg", [
    (b" x\n", 1, "data before the first section"),
    (b"NAME X\nFOO\n", 2, "unknown section FOO"),
    (b"NAME X\nQUADOBJ\n", 2, "section QUADOBJ is not supported"),
    (b"NAME X\nOBJSENSE\n    SIDEWAYS\n", 3, "bad OBJSENSE SIDEWAYS"),
    (b"ROWS\n N obj\n E r\n E r\n", 4, "duplicate row r"),
    (b"ROWS\n N obj\n X r\n", 3, "unknown row type X"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r  1.5e\n", 5, "bad number 1.5e"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r  0x10\n", 5, "bad number 0x10"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r  nan\n", 5, "bad number nan"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r\n", 5, "COLUMNS line needs a column and row/value pairs"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    M  'MARKER'  'FOO'\n", 5, "unknown marker FOO"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r  1\nBOUNDS\n UP B y 1\n", 7, "unknown column y"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r  1\nBOUNDS\n UP\n", 7, "malformed BOUNDS line"),
    (b"ROWS\n N obj\n E r\nCOLUMNS\n    x  r  1\nBOUNDS\n ZZ B x 1\n", 7, "unsupported bound type ZZ"),
])
def test_errors_name_line_and_cause(text, line, msg):
    with pytest.raises(sp().MpsError) as e:
        sp().read_mps(text)
    assert (e.value.line, e.value.msg) == (line, msg)
    with pytest.raises(ValueError, match=rf"^line {line}:"):
        oracle.read_mps(text)


def test_rules_of_ranges_bounds_sets_and_duplicates():
    text = b"""NAME RULES
ROWS
 N  obj
 N  other
 E  e1
 E  e2
 L  l1
 G  g1
COLUMNS
    x  obj  1  e1  2
    x  e1  3  other  9
    y  e2  1  l1  0.0
    y  g1  -1
    z  e1  5e-1  g1  inf
RHS
    R1  e1  1  e2  2
    R1  l1  3  g1  4
    R2  e1  100
RANGES
    G1  e1  2  e2  -3
    G1  l1  -4  g1  5
BOUNDS
 UP B1  x  -2
 LO B1  y  -1
 UP B1  y  -0.5
 BV B1  z
 FR B2  x
"""
    p = sp().read_mps(text)
    # e1: x twice (2 + 3, file order), z; l1's explicit 0.0 dropped
    assert list(p.row_ptr) == [0, 2, 3, 3, 5]
    assert list(p.col_idx) == [0, 2, 1, 1, 2]
    assert list(p.values) == [5.0, 0.5, 1.0, -1.0, INF]
    assert list(p.c) == [1.0, 0.0, 0.0]
    assert list(p.lc) == [1.0, -1.0, -1.0, 4.0]  # E +2, E -3, L |-4|, G
    assert list(p.uc) == [3.0, 2.0, 3.0, 9.0]
    assert list(p.lv) == [-INF, -1.0, 0.0]  # negative UP with a default lower bound; only set B1 applies
    assert list(p.uv) == [-2.0, -0.5, 1.0]
    ref = oracle.read_mps(text)
    for k in ("row_ptr", "col_idx", "values", "c", "lc", "uc", "lv", "uv"):
        assert np.array_equal(getattr(p, k), getattr(ref, k)), k


@pytest.mark.parametrize("name", QUICK + SLOW + KNOWN_HARD)
def test_netlib_fixture_reads_as_the_oracle_reads_it(name):
    text = netlib_bytes(name)
    p = sp().read_mps(text)
    ref = oracle.read_mps(text, name)
    assert (p.nrows, p.ncols, p.nnz) == (ref.nrows, ref.ncols, ref.nnz)
    for k in ("row_ptr", "col_idx", "values", "c", "lc", "uc", "lv", "uv"):
        assert np.array_equal(getattr(p, k), getattr(ref, k)), k
    assert p.c0 == ref.c0 and p.maximize == ref.maximize


def test_reads_a_gzipped_file_by_path():
    p = sp().read_mps(f"{NETLIB}/afiro.mps.gz")
    assert (p.nrows, p.ncols, p.name) == (27, 32, "afiro")
