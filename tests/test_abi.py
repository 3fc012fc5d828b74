"""CPU checks of the C ABI: the library loads and exports every function
include/pdf.h declares; netlist validation; the seeded generators; the plane
conversions.  No compute call needs a GPU here."""
import ctypes
import re

import numpy as np
import pytest

import circuits
import helpers

P = helpers.pdf()


def header_functions():
    text = (helpers.ROOT / "include" / "pdf.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pdf_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(P.LIB_PATH)
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    declared = {n for n, _, _ in P.ABI}
    assert set(names) == declared, set(names) ^ declared


def test_abi_version_and_strings():
    L = P.lib()
    assert L.pdf_abi_version() == 2
    assert L.pdf_status_string(0) == b"ok"
    assert L.pdf_status_string(3) == b"path count overflow"


def test_generated_netlists_are_valid():
    for name, nl in circuits.small_suite():
        st, msg = nl.check()
        assert st == 0, (name, msg)


def test_generator_is_deterministic_and_shaped():
    g = P.WORKLOADS["c1"]["gen"]
    a, b = P.gen_netlist(g), P.gen_netlist(g)
    for f in ("level_offsets", "type", "po", "nfi", "nfo", "edge_offset", "edges"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert a.n_gates == 2000 and a.n_pi == 36 and a.n_levels == 41 and int(a.po.sum()) == 7
    assert set(np.unique(a.type[36:])) <= {P.AND, P.NAND, P.OR, P.NOR, P.XOR, P.XNOR, P.NOT, P.BUFF}
    nfi = a.nfi[36:]
    assert nfi.min() >= 1 and nfi.max() <= 4
    assert np.all(nfi[np.isin(a.type[36:], [P.NOT, P.BUFF])] == 1)
    # every level above the inputs takes a fan-in from the level just below
    lvl = np.repeat(np.arange(a.n_levels), np.diff(a.level_offsets))
    for g in range(36, a.n_gates):
        assert lvl[a.fanins(g)].max() == lvl[g] - 1


def test_zipf_fanout_cap():
    nl = circuits.random_small(5, n_gates=3000, n_pi=100, n_po=100, depth=10, zipf=True, fo_max=64)
    assert nl.nfo.max() <= 64


def test_pairs_generator_prefix_stable():
    v1, t1 = P.gen_pairs(42, 5, 100)
    v2, t2 = P.gen_pairs(42, 5, 1000)
    np.testing.assert_array_equal(v1[:, :3], v2[:, :3])
    assert np.all(v1[:, 3] == (v2[:, 3] & 0xF)) and np.all(t1[:, 3] == (t2[:, 3] & 0xF))
    assert v1[:, 3].max() < 16  # tail bits zero


def test_plane_code_roundtrip():
    rng = np.random.default_rng(0)
    codes = helpers.rand_codes(rng, 7, 77)
    v, t = P.planes_from_codes(codes)
    assert v.shape == (7, 3)
    np.testing.assert_array_equal(P.codes_from_planes(v, t, 77), codes)


def _mutated(nl, **kw):
    f = dict(level_offsets=nl.level_offsets, type_=nl.type, po=nl.po, nfi=nl.nfi, nfo=nl.nfo,
             edge_offset=nl.edge_offset, edges=nl.edges)
    f.update(kw)
    return P.Netlist(**{k: np.array(v).copy() for k, v in f.items()})


def test_netlist_check_rejects_malformed():
    nl = circuits.random_small(77)
    assert nl.check()[0] == 0
    bad_type = nl.type.copy(); bad_type[20] = 12
    assert _mutated(nl, type_=bad_type).check()[0] == 1
    inpt_high = nl.type.copy(); inpt_high[30] = P.INPT
    assert _mutated(nl, type_=inpt_high).check()[0] == 1
    bad_po = nl.po.copy(); bad_po[10] = 2
    assert _mutated(nl, po=bad_po).check()[0] == 1
    # a fan-in on the same level (a cycle risk)
    e = nl.edges.copy(); g = int(nl.level_offsets[3]); e[int(nl.edge_offset[g])] = g
    st, msg = _mutated(nl, edges=e).check()
    assert st == 1 and "fan-in" in msg
    # fan-out list that is not the transpose of the fan-ins
    e = nl.edges.copy()
    g = next(x for x in range(nl.n_pi, nl.n_gates) if nl.nfo[x] >= 1 and nl.nfi[x] >= 1)
    o = int(nl.edge_offset[g] + nl.nfi[g])
    others = [x for x in range(int(nl.level_offsets[-2]), nl.n_gates) if x not in nl.fanouts(g)]
    e[o] = others[0]
    assert _mutated(nl, edges=e).check()[0] == 1
    lo = nl.level_offsets.copy(); lo[-1] += 1
    assert _mutated(nl, level_offsets=lo).check()[0] == 1
    nfi0 = nl.nfi.copy(); nfi0[nl.n_pi] = 0
    assert _mutated(nl, nfi=nfi0).check()[0] == 1
    # a fan-in id out of range
    e = nl.edges.copy(); g = int(nl.level_offsets[2]); e[int(nl.edge_offset[g])] = nl.n_gates + 5
    st, msg = _mutated(nl, edges=e).check()
    assert st == 1 and "fan-in" in msg
    # a fan-in on a higher level (a cycle through the level order)
    e = nl.edges.copy(); g = int(nl.level_offsets[2]); e[int(nl.edge_offset[g])] = int(nl.level_offsets[-2])
    st, msg = _mutated(nl, edges=e).check()
    assert st == 1 and "fan-in" in msg
    # level offsets out of order
    lo = nl.level_offsets.copy(); lo[2], lo[3] = lo[3], lo[2]
    assert _mutated(nl, level_offsets=lo).check()[0] == 1


def test_fault_injection_entry_point():
    L = P.lib()
    assert L.pdf_test_inject(0, 1) == 1 and L.pdf_test_inject(3, 1) == 1  # PDF_EINVAL
    assert L.pdf_test_inject(P.INJECT_DEVICE_ALLOC, 0) == 0


def test_generator_library_is_host_only():
    """The workload generator is its own library (no CUDA): a CPU baseline
    can build its inputs without loading the grader."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, 'tests'); import helpers; P = helpers._load('pdf_b200', "
            "helpers.PKG_DIR / '__init__.py'); nl = P.gen_netlist(P.WORKLOADS['c1']['gen']); "
            "v, t = P.gen_pairs(1, nl.n_pi, 100); maps = open('/proc/self/maps').read(); "
            "assert 'libpdf_gen.so' in maps and 'libpdf_b200.so' not in maps and 'libcudart' not in maps, maps; "
            "print(nl.n_gates)")
    out = subprocess.run([sys.executable, "-c", code], cwd=helpers.ROOT, capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "2000", out.stderr


def test_circuit_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(P.PdfError) as e:
        P.Circuit(circuits.random_small(1))
    assert e.value.status == 8  # PDF_ENODEV, never an exit or a trap
