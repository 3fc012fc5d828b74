"""Known-answer tests of the reference's lookup tables.

The reference's tables (simkernel.cuh:158-165, markkernel.cuh:36-41) are
the only fixed data of the algorithm.  These tests pin (1) that each 2-input
table is the exact per-vector boolean function, (2) that the oracle holds
those tables, and (3) that the bit-plane forms the kernels use
(pdf_device.cuh) equal them on every entry.
"""
import operator
import subprocess

import numpy as np
import pytest

import helpers
import refmodel as R

OPS = {R.AND: operator.and_, R.NAND: lambda a, b: 1 - (a & b), R.OR: operator.or_,
       R.NOR: lambda a, b: 1 - (a | b), R.XOR: operator.xor, R.XNOR: lambda a, b: 1 - (a ^ b)}


@pytest.mark.parametrize("t", sorted(OPS))
def test_reference_tables_are_per_vector_boolean(t):
    for r in range(4):
        for v in range(4):
            assert R.LUT2[t][r * 4 + v] == R.per_vector(OPS[t], v, r)


def test_stable_and_not_tables():
    # stable[v2 * 2 + v1]: S0 (0,0), T0 (1->0), T1 (0->1), S1 (1,1)
    for v1 in (0, 1):
        for v2 in (0, 1):
            code = R.STABLE[v2 * 2 + v1]
            assert code & 1 == v2 and (code >> 1) == (v1 ^ v2)
    for c in range(4):
        assert R.NOT_LUT[c] == (c ^ 1)


def test_oracle_holds_the_tables():
    o = helpers.oracle().lib()
    for t in list(OPS) + [0, 1, 8, 9, 10, 11]:
        for r in range(4):
            for v in range(4):
                want = R.LUT2[t][r * 4 + v] if t in OPS else 0
                assert o.pdfo_lut2(t, v, r) == want
    for v1 in (0, 1):
        for v2 in (0, 1):
            assert o.pdfo_stable(v1, v2) == R.STABLE[v2 * 2 + v1]
    for c in range(4):
        assert o.pdfo_not(c) == R.NOT_LUT[c]
    for mode in (0, 1):
        for t in range(12):
            for on in range(4):
                for off in range(4):
                    want = (R.SENS[mode][t - 2] >> (on * 4 + off)) & 1 if 2 <= t <= 7 else 0
                    assert o.pdfo_sens(mode, t, on, off) == want


def test_sensitisation_tables_decode():
    # LUT_NR (default): AND/NAND on=T0 & side in {S1,T1}; on=T1 & side=S1.
    nr, r = R.SENS[0], R.SENS[1]
    bits = lambda m: {(i >> 2, i & 3) for i in range(16) if (m >> i) & 1}
    assert bits(nr[0]) == {(R.T0, R.S1), (R.T0, R.T1), (R.T1, R.S1)}
    assert bits(nr[2]) == {(R.T0, R.S0), (R.T1, R.S0), (R.T1, R.T0)}
    assert bits(r[0]) == {(R.T0, R.S1), (R.T1, R.S1)}
    assert bits(r[2]) == {(R.T0, R.S0), (R.T1, R.S0)}
    assert nr[4] == nr[5] == r[4] == r[5] == 0


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("probe") / "lut_probe"
    src = helpers.ROOT / "tests" / "lut_probe.cpp"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{helpers.ROOT / 'include'}",
                    f"-I{helpers.PKG_DIR / 'csrc'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in out.splitlines():
        k, *vals = line.split()
        rows.setdefault(k, []).append(tuple(int(x) for x in vals))
    return rows


def test_device_fold_equals_reference_simlut(probe):
    for t, a, b, code in probe["fold"]:
        # fold step val = simLUT(type, val=a, r=b) of the coalesced overload
        want = R.LUT2[t][b * 4 + a] if t in (R.AND, R.NAND, R.OR, R.NOR) else 0
        assert code == want, (t, a, b)


def test_device_not_equals_reference(probe):
    for a, code in probe["not"]:
        assert code == R.NOT_LUT[a]


def test_device_sens_equals_reference(probe):
    for mode, t, on, off, s in probe["sens"]:
        want = (R.SENS[mode][t - 2] >> (on * 4 + off)) & 1 if 2 <= t <= 7 else 0
        assert s == want, (mode, t, on, off)


def _ref_gate(t, codes):
    """Value of one gate under the reference's kernSimulateP1 (simkernel.cuh:111-149)."""
    if t in (R.BUFF, R.FROM, R.DFF):
        return codes[0]
    v = codes[0]
    if t == R.NOT:
        v = R.NOT_LUT[v]
    for c in codes[1:]:
        v = R.LUT2[t][c * 4 + v] if t in (R.AND, R.NAND, R.OR, R.NOR) else 0
    return v


def test_device_gate_evaluation_equals_reference(probe):
    seen = 0
    for t, nfi, c0, c1, c2, code in probe["gate"]:
        assert code == _ref_gate(t, [c0, c1, c2][:nfi]), (t, nfi, c0, c1, c2)
        seen += 1
    assert seen == 11 * (4 + 16 + 64)


def test_device_mark_flags_equal_reference(probe):
    # markkernel.cuh:233-264: INPT marks on a transition; FROM/BUFF/DFF/NOT and
    # AND..XNOR follow fan-in 0; the side-input test only matters with >= 2 inputs
    for t, nfi, markf0, inpt, sens in probe["flags"]:
        assert inpt == 0
        assert markf0 == int(t in (R.FROM, R.BUFF, R.DFF, R.NOT) or R.AND <= t <= R.XNOR), (t, nfi)
        if sens:
            assert R.AND <= t <= R.NOR and nfi >= 2
        if R.AND <= t <= R.NOR and nfi >= 2:
            assert sens


def test_device_side_input_test_equals_reference(probe):
    """One-pass OR_i AND_{x != i} sens(on=i, off=x) (markkernel.cuh:253-261)
    against the reference's tables, every code combination of 2..4 fan-ins."""
    seen = 0
    for mode, t, nfi, cmb, got in probe["sensall"]:
        codes = [(cmb >> (2 * x)) & 3 for x in range(nfi)]
        tab = R.SENS[mode][t - 2]
        want = int(any(all((tab >> (codes[i] * 4 + codes[x])) & 1 for x in range(nfi) if x != i)
                       for i in range(nfi)))
        assert got == want, (mode, t, nfi, codes)
        seen += 1
    assert seen == 2 * 4 * (16 + 64 + 256)


# ---- FIXED semantics (no reference counterpart; stated from the definitions)


def _fixed_gate(t, codes):
    """True n-input function of AND..XNOR under each vector (refmodel.sim_pair)."""
    out = []
    for vec in (1, 2):
        vs = [(c & 1) if vec == 2 else ((c & 1) ^ (c >> 1)) for c in codes]
        if t in (R.AND, R.NAND):
            o = int(all(vs))
        elif t in (R.OR, R.NOR):
            o = int(any(vs))
        else:
            o = sum(vs) & 1
        out.append(o ^ int(t in (R.NAND, R.NOR, R.XNOR)))
    v1, v2 = out
    return v2 | ((v1 ^ v2) << 1)


def test_device_fixed_gate_evaluation(probe):
    seen = 0
    for t, nfi, cmb, code in probe["fgate"]:
        codes = [(cmb >> (2 * x)) & 3 for x in range(nfi)]
        assert code == _fixed_gate(t, codes), (t, nfi, codes)
        seen += 1
    assert seen == 6 * (4 + 16 + 64 + 256)


def test_device_fixed_flags(probe):
    for t, nfi, markf0, many, sens in probe["fflags"]:
        assert (markf0, many, sens) == ((1, 0, 0) if nfi == 1 else (0, 1, 1)), (t, nfi)


def test_device_fixed_side_test(probe):
    """OR over marked candidates i of AND over x != i of the FIXED side
    condition, every code and mark combination of 2..4 fan-ins."""
    seen = 0
    for nonrobust, t, nfi, cmb, marks, got in probe["fsens"]:
        mode = 3 if nonrobust else 2
        codes = [(cmb >> (2 * x)) & 3 for x in range(nfi)]
        want = int(any((marks >> i) & 1 and all(R.fixed_side_ok(mode, t, codes[i], codes[x])
                                                   for x in range(nfi) if x != i)
                       for i in range(nfi)))
        assert got == want, (mode, t, nfi, codes, marks)
        seen += 1
    assert seen == 2 * 6 * (16 * 4 + 64 * 8 + 256 * 16)


@pytest.mark.parametrize("mode", [2, 3])
def test_oracle_fixed_tables_equal_definitions(mode):
    for t in range(R.AND, R.XNOR + 1):
        for on in range(4):
            for off in range(4):
                assert helpers.oracle().lib().pdfo_sens(mode, t, on, off) == int(R.fixed_side_ok(mode, t, on, off)), \
                    (mode, t, on, off)
