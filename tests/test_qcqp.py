"""QCQP -> SOCP rewrite (qcqp_to_socp_qp) through the C ABI, on the CPU:
QCQPs with <= rows and PSD diagonal Q_i, >= rows with NSD Q_i (flipped),
and rows without a linear part (their s, t slots fixed), in the standard
and the rotated form, rewritten by this library and by the reference's own
build (oracle/_ref), compared field for field, exactly; plus the
transform's refusals and a hand-checked layout."""
import ctypes as C
import os

import numpy as np
import pytest

from pdhcg_b200 import capi

from test_mps import _read, _same

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libpdhcg_ref.so")


@pytest.fixture(scope="module")
def lib():
    from pdhcg_b200 import native
    return native.load()


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return capi.bind_api(C.CDLL(REF))


def qcqp_mps(rng, pinned=False, flips=True):
    """A box-bounded QCQP in MPS: 8-20 variables, 3-8 linear rows, 2-4
    quadratic rows (diagonal Q_i) that x = 0 satisfies strictly."""
    n, m, k = int(rng.integers(8, 21)), int(rng.integers(3, 9)), int(rng.integers(2, 5))
    lines = ["NAME QC", "ROWS", " N  OBJ"]
    sense = []
    for i in range(k):
        s = "G" if (flips and i % 2 == 1) else "L"
        sense.append(s)
        lines.append(f" {s}  Q{i}")
    lines += [f" E  E{i}" for i in range(m)]
    lines.append("COLUMNS")
    x0 = rng.uniform(-0.5, 0.5, n)
    lin = {i: {} for i in range(k)}
    erow = {i: {} for i in range(m)}
    for j in range(n):
        ents = [("OBJ", rng.standard_normal())]
        for i in range(k):
            if not (pinned and i == 0) and rng.random() < 0.5:
                lin[i][j] = rng.standard_normal()
                ents.append((f"Q{i}", lin[i][j]))
        for i in rng.choice(m, 2, replace=False):
            erow[i][j] = rng.standard_normal()
            ents.append((f"E{i}", erow[i][j]))
        for t in range(0, len(ents), 2):
            lines.append(f"    X{j}  " + "  ".join(f"{r}  {v:.17g}" for r, v in ents[t:t + 2]))
    lines.append("RHS")
    for i in range(m):
        lines.append(f"    RHS  E{i}  {sum(v * x0[j] for j, v in erow[i].items()):.17g}")
    for i in range(k):  # slack of 5 at x0 (the quadratic terms are at most 0.5 there)
        val = sum(v * x0[j] for j, v in lin[i].items())
        lines.append(f"    RHS  Q{i}  {(val + 5.0) if sense[i] == 'L' else (-val - 5.0):.17g}")
    lines.append("BOUNDS")
    for j in range(n):
        lines += [f" LO BND  X{j}  -1", f" UP BND  X{j}  1"]
    for i in range(k):
        lines.append(f"QCMATRIX  Q{i}")
        sg = 1.0 if sense[i] == "L" else -1.0
        for j in sorted(rng.choice(n, int(rng.integers(2, 6)), replace=False)):
            lines.append(f"    X{j}  X{j}  {sg * rng.uniform(0.1, 1.0):.17g}")
    lines.append("ENDATA")
    return "\n".join(lines) + "\n"


def _transform(lib, path, form):
    prob = lib.read_mps_file(str(path).encode())
    assert prob
    ext = lib.qcqp_to_socp_qp(prob, form)
    lib.qp_problem_free(prob)
    assert ext
    out = capi.problem_arrays(ext)
    out["num_original_variables"] = ext.contents.num_original_variables
    lib.qp_problem_free(ext)
    return out


@pytest.mark.parametrize("case", range(8))
def test_qcqp_rewrite_matches_reference(tmp_path, lib, ref_lib, case):
    rng = np.random.default_rng(200 + case)
    path = tmp_path / f"qc{case}.mps"
    path.write_text(qcqp_mps(rng, pinned=case >= 6, flips=case % 2 == 0))
    form = capi.CONE_STANDARD_SOC if case % 4 < 2 else capi.CONE_ROTATED_SOC
    _same(_transform(lib, path, form), _transform(ref_lib, path, form))


def test_qcqp_rewrite_layout(tmp_path, lib):
    """One <= row x0 + 2 x0^2 + 0.5 x1^2 <= 3 (rotated form): v = (2 x0, x1),
    block [v0, v1, s, t] after the two variables, rows: x0 + s = 3,
    -2 x0 + v0 = 0, -x1 + v1 = 0, t = 1."""
    text = ("NAME T\nROWS\n N  OBJ\n L  C\nCOLUMNS\n    X0  OBJ  1  C  1\n    X1  OBJ  1\nRHS\n    RHS  C  3\n"
            "QCMATRIX  C\n    X0  X0  2\n    X1  X1  0.5\nENDATA\n")
    path = tmp_path / "t.mps"
    path.write_text(text)
    a = _transform(lib, path, capi.CONE_ROTATED_SOC)
    assert (a["n"], a["m"]) == (6, 4) and a["num_original_variables"] == 2
    assert a["cones"] == {"start": [2], "v_dim": [2], "type": [capi.CONE_ROTATED_SOC]}
    rp, ci, v = a["A"]
    np.testing.assert_array_equal(rp, [0, 2, 4, 6, 7])
    np.testing.assert_array_equal(ci, [0, 4, 0, 2, 1, 3, 5])
    np.testing.assert_allclose(v, [1, 1, -2, 1, -1, 1, 1])
    np.testing.assert_array_equal(a["con_lb"], [3, 0, 0, 1])
    np.testing.assert_array_equal(a["con_ub"], [3, 0, 0, 1])
    assert a["qc"] == [] and a["fixed"] == b""


def test_qcqp_rewrite_refusals(tmp_path, lib):
    base = "NAME T\nROWS\n N  OBJ\n {s}  C\nCOLUMNS\n    X0  OBJ  1  C  1\n    X1  OBJ  1\nRHS\n    RHS  C  3\n"
    for sense, q, why in [("L", "    X0  X1  1\n", "non-diagonal"), ("L", "    X0  X0  1\n    X1  X1  -1\n", "mixed signs"),
                          ("G", "    X0  X0  1\n", "PSD on a >= row"), ("E", "    X0  X0  1\n", "two-sided row")]:
        path = tmp_path / "bad.mps"
        path.write_text(base.format(s=sense) + "QCMATRIX  C\n" + q + "ENDATA\n")
        prob = lib.read_mps_file(str(path).encode())
        assert prob
        assert not lib.qcqp_to_socp_qp(prob, capi.CONE_ROTATED_SOC), why
        lib.qp_problem_free(prob)
    path = tmp_path / "lp.mps"  # nothing to do without quadratic constraints
    path.write_text(base.format(s="L") + "ENDATA\n")
    prob = lib.read_mps_file(str(path).encode())
    assert not lib.qcqp_to_socp_qp(prob, capi.CONE_ROTATED_SOC)
    lib.qp_problem_free(prob)
