"""MPS / QPS reader (read_mps_file) through the C ABI, on the CPU.

A hand-written file pins every section against values derived by hand
from the format's rules; generated files (LPs and QPs with ranges, every
bound type, QUADOBJ / QMATRIX, OBJSENSE MAX, an objective constant,
markers, gzip) are read by this library and by the reference's own reader
(oracle/_ref, built from the reference's sources) and compared field for
field, exactly."""
import ctypes as C
import gzip
import os

import numpy as np
import pytest

from pdhcg_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")


@pytest.fixture(scope="module")
def mps_lib():
    from pdhcg_b200 import native
    return native.load()


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return capi.bind_api(C.CDLL(REF))


def _read(lib, path):
    prob = lib.read_mps_file(path.encode())
    assert prob, path
    arr = capi.problem_arrays(prob)
    lib.qp_problem_free(prob)
    return arr


HAND = """NAME          HAND
* a comment
ROWS
 N  COST
 L  LIM1
 G  LIM2
 E  MYEQN
 N  FREE2
 E  R4
COLUMNS
    MARKER                 'MARKER'                 'INTORG'
    X1        COST         1.0   LIM1         1.0
    X1        LIM2         1.0
    MARKER                 'MARKER'                 'INTEND'
    X2        COST         2.0   LIM1         1.0
    X2        MYEQN       -1.0   FREE2        5.0
    X3        COST        -1.0   MYEQN        1.0
    X3        R4           2.0
    X4        COST         0.5   R4           1.0
RHS
    RHS       COST        -3.5   LIM1         4.0
    RHS       LIM2         1.0   MYEQN        7.0
    RHS       R4           2.0
RANGES
    RNG       LIM1         2.5   LIM2        -1.5
    RNG       MYEQN       -2.0   R4           3.0
BOUNDS
 UP BND       X1           4.0
 MI BND       X2
 FX BND       X3           1.5
 FR BND       X4
QUADOBJ
    X1        X1           2.0
    X1        X2           0.5
    X4        X4           1.0
ENDATA
"""


def test_mps_reader_known_answer(tmp_path, mps_lib):
    path = tmp_path / "hand.mps"
    path.write_text(HAND)
    a = _read(mps_lib, str(path))
    assert a["n"] == 4 and a["m"] == 4  # COST is the objective, FREE2 is dropped
    np.testing.assert_array_equal(a["c"], [1.0, 2.0, -1.0, 0.5])
    assert a["obj_const"] == 3.5  # RHS on the objective row: constant = -value
    np.testing.assert_array_equal(a["var_lb"], [0.0, -np.inf, 1.5, -np.inf])
    np.testing.assert_array_equal(a["var_ub"], [4.0, np.inf, 1.5, np.inf])
    # L [4 - 2.5, 4], G [1, 1 + 1.5], E with R < 0 [7 - 2, 7], E with R > 0 [2, 2 + 3]
    np.testing.assert_array_equal(a["con_lb"], [1.5, 1.0, 5.0, 2.0])
    np.testing.assert_array_equal(a["con_ub"], [4.0, 2.5, 7.0, 5.0])
    rp, ci, v = a["A"]
    np.testing.assert_array_equal(rp, [0, 2, 3, 5, 7])
    np.testing.assert_array_equal(ci, [0, 1, 0, 1, 2, 2, 3])
    np.testing.assert_array_equal(v, [1.0, 1.0, 1.0, -1.0, 1.0, 2.0, 1.0])
    rp, ci, v = a["Q"]  # QUADOBJ: off-diagonal entries mirrored, file order within rows
    np.testing.assert_array_equal(rp, [0, 2, 3, 3, 4])
    np.testing.assert_array_equal(ci, [0, 1, 0, 3])
    np.testing.assert_array_equal(v, [2.0, 0.5, 0.5, 1.0])
    assert a["qc"] == []


def test_mps_reader_objsense_qmatrix_and_gzip(tmp_path, mps_lib):
    """QMATRIX entries are taken as given (no mirror); a gzip file reads the
    same.  As in the reference reader, a line holding only MAX is read as a
    section header first, so the two-line OBJSENSE form leaves the sense at
    minimize; a sense line whose first token is MAX with more tokens after
    it is what negates c, the constant and Q."""
    text = HAND.replace("QUADOBJ", "QMATRIX").replace("ROWS\n", "OBJSENSE\n    MAX\nROWS\n")
    path = tmp_path / "max.mps.gz"
    with gzip.open(path, "wt") as f:
        f.write(text)
    a = _read(mps_lib, str(path))
    np.testing.assert_array_equal(a["c"], [1.0, 2.0, -1.0, 0.5])
    assert a["obj_const"] == 3.5
    rp, ci, v = a["Q"]
    np.testing.assert_array_equal(rp, [0, 2, 2, 2, 3])
    np.testing.assert_array_equal(ci, [0, 1, 3])
    np.testing.assert_array_equal(v, [2.0, 0.5, 1.0])
    path2 = tmp_path / "max2.mps"
    path2.write_text(HAND.replace("QUADOBJ", "QMATRIX").replace("ROWS\n", "OBJSENSE\n    MAX  SENSE\nROWS\n"))
    b = _read(mps_lib, str(path2))
    np.testing.assert_array_equal(b["c"], [-1.0, -2.0, 1.0, -0.5])
    assert b["obj_const"] == -3.5
    np.testing.assert_array_equal(b["Q"][2], [-2.0, -0.5, -1.0])


def test_mps_reader_rejects_bad_files(tmp_path, mps_lib):
    assert not mps_lib.read_mps_file(str(tmp_path / "missing.mps").encode())
    bad = tmp_path / "bad.mps"
    bad.write_text("ROWS\n N COST\nCOLUMNS\n    COST 1.0\nENDATA\n")  # data before any column name
    assert not mps_lib.read_mps_file(str(bad).encode())


def _write_mps(path, rng, quad, maximize, ranges, qcm):
    """A random LP / QP in MPS with every feature the reader handles."""
    n, m = int(rng.integers(5, 40)), int(rng.integers(3, 25))
    types = rng.choice(["L", "G", "E"], m)
    lines = ["NAME RAND"]
    if maximize:
        lines += ["OBJSENSE", "    MAXIMIZE" if rng.random() < 0.5 else "    MAX  SENSE"]
    lines += ["ROWS", " N  OBJ"] + [f" {t}  R{i}" for i, t in enumerate(types)] + [" N  SPARE"]
    lines.append("COLUMNS")
    for j in range(n):
        if j == n // 2:
            lines.append("    MARKER  'MARKER'  'INTORG'")
        ents = [("OBJ", rng.standard_normal())] if rng.random() < 0.8 else []
        for i in rng.choice(m, int(rng.integers(1, min(m, 5) + 1)), replace=False):
            ents.append((f"R{i}", rng.standard_normal()))
        for k in range(0, len(ents), 2):  # one or two entries per line
            pair = "  ".join(f"{r}  {v:.17g}" for r, v in ents[k:k + 2])
            lines.append(f"    X{j}  {pair}")
        if j == n // 2:
            lines.append("    MARKER  'MARKER'  'INTEND'")
    lines.append("RHS")
    lines.append(f"    RHS  OBJ  {rng.standard_normal():.17g}")
    for i in range(m):
        lines.append(f"    RHS  R{i}  {rng.standard_normal():.17g}")
    if ranges:
        lines.append("RANGES")
        for i in rng.choice(m, m // 2, replace=False):
            lines.append(f"    RNG  R{i}  {rng.standard_normal():.17g}")
    lines.append("BOUNDS")
    for j in range(n):
        t = rng.choice(["UP", "LO", "FX", "FR", "MI", "PL", "BV", "none"])
        if t in ("UP", "LO", "FX"):
            lines.append(f" {t} BND  X{j}  {rng.standard_normal():.17g}")
        elif t != "none":
            lines.append(f" {t} BND  X{j}")
    if quad:
        lines.append("QUADOBJ" if quad == "QUADOBJ" else "QMATRIX")
        for _ in range(2 * n):
            a, b = sorted(rng.integers(0, n, 2))
            lines.append(f"    X{a}  X{b}  {rng.uniform(0.1, 1.0):.17g}")
    if qcm:
        for i in rng.choice(m, 2, replace=False):
            lines.append(f"QCMATRIX  R{i}")
            for _ in range(3):
                a, b = rng.integers(0, n, 2)
                lines.append(f"    X{a}  X{b}  {rng.uniform(0.1, 1.0):.17g}")
    lines.append("ENDATA")
    text = "\n".join(lines) + "\n"
    if str(path).endswith(".gz"):
        with gzip.open(path, "wt") as f:
            f.write(text)
    else:
        path.write_text(text)


def _same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        if k in ("A", "Q"):
            for x, y in zip(a[k], b[k]):
                np.testing.assert_array_equal(x, y, err_msg=k)
        elif k == "qc":
            assert len(a[k]) == len(b[k])
            for (ra, ma), (rb, mb) in zip(a[k], b[k]):
                assert ra == rb
                for x, y in zip(ma, mb):
                    np.testing.assert_array_equal(x, y)
        elif isinstance(a[k], (dict, bytes)):
            assert a[k] == b[k], k
        else:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("case", range(12))
def test_mps_reader_matches_reference_reader(tmp_path, mps_lib, ref_lib, case):
    rng = np.random.default_rng(100 + case)
    quad = [None, "QUADOBJ", "QMATRIX"][case % 3]
    path = tmp_path / (f"r{case}.mps" + (".gz" if case % 4 == 3 else ""))
    _write_mps(path, rng, quad, maximize=case % 2 == 1, ranges=case % 3 != 2, qcm=case >= 9)
    _same(_read(mps_lib, str(path)), _read(ref_lib, str(path)))
