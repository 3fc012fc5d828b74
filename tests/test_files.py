"""Netlist and vector files, the reference's debug-log layouts, and the
fcount command line (main.cu:24-235) end to end.

CPU tests: the .bench reader (levelization, full-scan flip-flop cut, fan-out
branches, errors with line numbers), level-text and .bench round trips, vector
files, and the exact text of the dumps.  GPU tests: the command line's total
equals the oracle on the reference's vector-stream pairs (one pass, many
passes, both tables, both file formats), its logs equal the oracle's planes,
and pdf_mark_forward equals the oracle's unpruned marks."""
import os
import re
import subprocess

import numpy as np
import pytest

import circuits
import helpers

P = helpers.pdf()
O = helpers.oracle()
FCOUNT = str(helpers.PKG_DIR / "fcount")

TINY = """# a tiny circuit
INPUT(a)
INPUT(b)
INPUT(c)
OUTPUT(z)
OUTPUT(y)
n1 = NAND(a, b)
n2 = nor(n1, c)   # lower case type
z = XOR(n2, a)
y = NOT(n1)
"""


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _fanins(nl, g):
    e = int(nl.edge_offset[g])
    return [int(x) for x in nl.edges[e:e + int(nl.nfi[g])]]


def _fanouts(nl, g):
    e = int(nl.edge_offset[g]) + int(nl.nfi[g])
    return [int(x) for x in nl.edges[e:e + int(nl.nfo[g])]]


def test_bench_levelized_in_file_order(tmp_path):
    nl = P.read_bench(_write(tmp_path, "tiny.bench", TINY))
    # a b c | n1 | n2 y | z
    assert list(nl.level_offsets) == [0, 3, 4, 6, 7]
    assert list(nl.type) == [P.INPT] * 3 + [P.NAND, P.NOR, P.NOT, P.XOR]
    assert list(nl.po) == [0, 0, 0, 0, 0, 1, 1]
    assert _fanins(nl, 3) == [0, 1] and _fanins(nl, 4) == [3, 2]
    assert _fanins(nl, 5) == [3] and _fanins(nl, 6) == [4, 0]
    assert _fanouts(nl, 0) == [3, 6] and _fanouts(nl, 3) == [4, 5] and _fanouts(nl, 6) == []


def test_bench_cuts_flip_flops_for_full_scan(tmp_path):
    text = "INPUT(a)\nOUTPUT(q2)\nq = DFF(d)\nd = AND(a, q)\nq2 = OR(q, d)\n"
    nl = P.read_bench(_write(tmp_path, "seq.bench", text))
    # a, q (pseudo input) | d (pseudo output) | q2
    assert list(nl.level_offsets) == [0, 2, 3, 4]
    assert list(nl.type) == [P.INPT, P.INPT, P.AND, P.OR]
    assert list(nl.po) == [0, 0, 1, 1]
    assert _fanins(nl, 2) == [0, 1] and _fanins(nl, 3) == [1, 2]


def test_bench_branches(tmp_path):
    nl = P.read_bench(_write(tmp_path, "tiny.bench", TINY), branches=True)
    G = nl.n_gates
    # stems a (read by n1 and z) and n1 (read by n2 and y) get one FROM per branch
    assert int((nl.type == P.FROM).sum()) == 4 and G == 11
    for g in range(G):
        fo = _fanouts(nl, g)
        if len(fo) > 1:
            assert all(nl.type[u] == P.FROM for u in fo)
        if nl.type[g] == P.FROM:
            assert nl.nfi[g] == 1 and len(fo) == 1


@pytest.mark.parametrize("text, what", [
    ("INPUT(a)\nOUTPUT(z)\nz = AND(a, q)\n", "never defined"),
    ("INPUT(a)\nz = AND(a, a)\nz = OR(a, a)\n", ":3:"),
    ("INPUT(a)\nx = AND(a, y)\ny = OR(a, x)\n", "loop"),
    ("INPUT(a)\nz = MAJ(a, a)\n", ":2:"),
    ("INPUT(a)\nz = NOT(a, a)\n", ":2:"),
    ("INPUT(a)\nz = AND(a,)\n", ":2:"),
    ("INPUT(a\n", ":1:"),
])
def test_bench_errors_name_the_line(tmp_path, text, what):
    with pytest.raises(P.PdfError) as e:
        P.read_bench(_write(tmp_path, "bad.bench", text))
    assert what in str(e.value)


def _same_netlist(a, b, fanout_order=True):
    for f in ("level_offsets", "type", "po", "nfi", "nfo"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)
    for g in range(a.n_gates):
        assert _fanins(a, g) == _fanins(b, g)
        fa, fb = _fanouts(a, g), _fanouts(b, g)
        assert (fa == fb) if fanout_order else (sorted(fa) == sorted(fb))


@pytest.mark.parametrize("k", range(4))
def test_level_text_round_trip(tmp_path, k):
    nl = [circuits.random_small(40 + k, n_gates=400, n_pi=20, n_po=30, depth=9),
          circuits.hub(150), circuits.diamond_chain(12), circuits.small_suite()[k][1]][k]
    path = str(tmp_path / "c.level")
    P.write_level(nl, path)
    _same_netlist(nl, P.read_level(path))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_bench_round_trip(tmp_path, seed):
    nl = P.gen_netlist(P.GenParams(seed=seed, n_gates=3000, n_pi=100, n_po=200, depth=25))
    path = str(tmp_path / "c.bench")
    P.write_bench(nl, path)
    _same_netlist(nl, P.read_bench(path), fanout_order=False)


def test_level_text_errors(tmp_path):
    good = tmp_path / "g.level"
    P.write_level(circuits.diamond_chain(2), str(good))
    lines = good.read_text().splitlines()
    for bad in (["pdf-level 2"] + lines[1:], lines[:-1], lines + [lines[-1]],
                lines[:2] + [lines[3], lines[2]] + lines[4:]):
        p = _write(tmp_path, "b.level", "\n".join(bad) + "\n")
        with pytest.raises(P.PdfError):
            P.read_level(p)


def test_vector_file(tmp_path):
    path = _write(tmp_path, "v.vec", "# vectors\n0101\n1 1 0 0  # spaced\n\n0011\n")
    vec = P.read_vectors(path)
    np.testing.assert_array_equal(vec.T, [[0, 1, 0, 1], [1, 1, 0, 0], [0, 0, 1, 1]])
    for bad in ("0101\n011\n", "01x1\n", ""):
        with pytest.raises(P.PdfError):
            P.read_vectors(_write(tmp_path, "b.vec", bad))


def _planes(bits):
    """[n_gates][n_pairs] 0/1 -> [n_gates][words] uint32."""
    G, n = bits.shape
    out = np.zeros((G, P.words(n)), np.uint32)
    for p in range(n):
        out[:, p // 32] |= bits[:, p].astype(np.uint32) << np.uint32(p % 32)
    return out


def test_dump_layouts(tmp_path):
    rng = np.random.default_rng(5)
    G, n = 7, 40
    codes = rng.integers(0, 4, size=(G, n), dtype=np.uint8)
    marks = rng.integers(0, 2, size=(G, n), dtype=np.uint8)
    head = "Gate:     \t" + "".join(f"{g:>4} " for g in range(G)) + "\n"
    sim_path, mark_path, merge_path = (str(tmp_path / f) for f in ("s.log", "m.log", "g.log"))
    P.dump_sim(sim_path, _planes(codes & 1), _planes(codes >> 1), 30, 0)
    P.dump_sim(sim_path, _planes(codes & 1), _planes(codes >> 1), 10, 30, append=True)
    names = ["S0 ", "S1 ", "T0 ", "T1 "]
    want = head + "".join(f"Vector {p}:\t" + "".join(f"{names[codes[g, p]]:>5}" for g in range(G)) + "\n"
                          for p in range(30))
    want += "".join(f"Vector {30 + p}:\t" + "".join(f"{names[codes[g, p]]:>5}" for g in range(G)) + "\n"
                    for p in range(10))
    assert open(sim_path).read() == want
    P.dump_mark(mark_path, _planes(marks), n, 100)
    want = head + "".join(f"Vector {100 + p}:\t" + "".join(f"{'YN'[1 - marks[g, p]]:>4} " for g in range(G)) + "\n"
                          for p in range(n))
    assert open(mark_path).read() == want
    fx = np.array([0, 5, P.NONE, 7], np.uint32)
    fy = np.array([P.NONE, 1, 2, 3], np.uint32)
    P.dump_merge(merge_path, fx, fy)
    assert open(merge_path).read() == ("Gate 0:\t   0,-1 \nGate 1:\t   5,1 \nGate 2:\t  -1,2 \n"
                                        "Gate 3:\t   7,3 \n")


def test_segment_dump_layout(tmp_path):
    """debugSegmentList (mergekernel.cuh:25-46): Segment s(g0,...): x,y"""
    path = str(tmp_path / "seg.log")
    segs = np.array([[0, 3, 7], [1, 3, 7]], np.uint32)
    P.dump_segments(path, segs, np.array([5, P.NONE], np.uint32), np.array([P.NONE, 2], np.uint32))
    assert open(path).read() == "Segment 0(0,3,7): 5,-1 \nSegment 1(1,3,7): -1,2 \n"


def test_cli_usage_and_errors(tmp_path):
    if not os.path.exists(FCOUNT):
        pytest.skip("fcount not built")
    r = subprocess.run([FCOUNT, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--bench" in r.stdout
    r = subprocess.run([FCOUNT, "x.vec"], capture_output=True, text=True)
    assert r.returncode == 1 and "--bench argument is required" in r.stderr
    r = subprocess.run([FCOUNT, "--bench", _write(tmp_path, "bad.bench", "INPUT(a\n"), "v"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and ":1:" in r.stderr
    r = subprocess.run([FCOUNT, "--segs", "9", "--bench", "x"], capture_output=True, text=True)
    assert r.returncode == 1


# ---------------------------------------------------------------- GPU


def _vectors(tmp_path, n_pi, n_vec, seed):
    rng = np.random.default_rng(seed)
    vec = rng.integers(0, 2, size=(n_pi, n_vec), dtype=np.uint8)
    path = tmp_path / f"v{seed}.vec"
    path.write_text("".join("".join(map(str, vec[:, r])) + "\n" for r in range(n_vec)))
    return vec, str(path)


LINE = re.compile(r"^(.*):(\d+),(\d+),(\d+);([0-9.e+-]+);([0-9.e+-]+);([0-9.e+-]+);([0-9.e+-]+);([0-9.e+-]+);(\d+)$")


def _run(args, cwd=None):
    r = subprocess.run([FCOUNT] + args, capture_output=True, text=True, cwd=cwd, timeout=300)
    assert r.returncode == 0, r.stderr
    return [LINE.match(x) for x in r.stdout.strip().splitlines()]


@pytest.mark.gpu
@pytest.mark.parametrize("robust", [False, True])
def test_cli_total_equals_oracle(tmp_path, robust):
    nl = circuits.random_small(77, n_gates=2000, n_pi=60, n_po=150, depth=30)
    bench = str(tmp_path / "c.bench")
    level = str(tmp_path / "c.level")
    P.write_bench(nl, bench)
    P.write_level(nl, level)
    back = P.read_bench(bench)  # the CLI grades the netlist as read back (fan-out order aside, the same)
    cases = [_vectors(tmp_path, nl.n_pi, n, 10 + n) for n in (1000, 64, 3)]
    flags = ["--robust"] if robust else []
    lines = _run(flags + ["--bench", bench] + [p for _, p in cases])
    lines_chunked = _run(flags + ["--num_patterns", "64", "--bench", bench] + [p for _, p in cases])
    lines_level = _run(flags + ["--bench", level] + [p for _, p in cases])
    for (vec, path), m, mc, ml in zip(cases, lines, lines_chunked, lines_level):
        n = vec.shape[1]
        v, t = P.pairs_from_vectors(vec)
        w = O.grade(back, P.codes_from_planes(v, t, n), n, mark_mode=int(robust))
        for mm in (m, mc, ml):
            assert mm and mm.group(1) == path and int(mm.group(2)) == n
            assert int(mm.group(3)) == nl.n_gates and int(mm.group(4)) == 1
            assert int(mm.group(10)) == w.total


@pytest.mark.gpu
@pytest.mark.parametrize("flags, mode", [(["--fixed"], 3), (["--fixed", "--robust"], 2)])
def test_cli_fixed_modes(tmp_path, flags, mode):
    nl = circuits.random_small(79, n_gates=1500, n_pi=50, n_po=100, depth=20)
    level = str(tmp_path / "c.level")
    P.write_level(nl, level)
    vec, vpath = _vectors(tmp_path, nl.n_pi, 500, 4)
    (m,) = _run(flags + ["--bench", level, vpath])
    v, t = P.pairs_from_vectors(vec)
    assert int(m.group(10)) == O.grade(nl, P.codes_from_planes(v, t, 500), 500, mark_mode=mode).total


@pytest.mark.gpu
def test_cli_logs_equal_oracle_planes(tmp_path):
    nl = circuits.random_small(78, n_gates=300, n_pi=16, n_po=40, depth=12)
    bench = str(tmp_path / "c.bench")
    P.write_bench(nl, bench)
    back = P.read_bench(bench)
    vec, vpath = _vectors(tmp_path, nl.n_pi, 100, 3)
    (m,) = _run(["--verbose", "--sim", "--mark", "--merge", "--cover", "--num_patterns", "64", "--bench", bench,
                 vpath], cwd=str(tmp_path))
    n = vec.shape[1]
    v, t = P.pairs_from_vectors(vec)
    codes = P.codes_from_planes(v, t, n)
    w = O.grade(back, codes, n, chunk=64, want_planes=True)
    assert int(m.group(10)) == w.total
    G = back.n_gates
    names = {"S0": 0, "S1": 1, "T0": 2, "T1": 3}

    def rows(name):
        lines = (tmp_path / name).read_text().splitlines()
        assert lines[0].split() == ["Gate:"] + [str(g) for g in range(G)]
        body = [ln.split("\t", 1) for ln in lines[1:]]
        assert [b[0] for b in body] == [f"Vector {p}:" for p in range(n)]
        return [b[1].split() for b in body]

    sim = np.array([[names[x] for x in r] for r in rows("gpusim-p2.log")], np.uint8).T
    np.testing.assert_array_equal(sim, w.sim)
    mark = np.array([[x == "Y" for x in r] for r in rows("gpumark.log")], np.uint8).T
    np.testing.assert_array_equal(mark, w.mark)
    full = np.array([[x == "Y" for x in r] for r in rows("gpumark-full.log")], np.uint8).T
    np.testing.assert_array_equal(full, O.mark(back, w.sim, n, prune=False))
    merge = [ln.split("\t")[1].split(",") for ln in (tmp_path / "gpumerge.log").read_text().splitlines()]
    np.testing.assert_array_equal([int(x) & 0xFFFFFFFF for x, _ in merge], w.first_x)
    np.testing.assert_array_equal([int(y) & 0xFFFFFFFF for _, y in merge], w.first_y)
    # gpucover.log: per pair, the paths each primary input credits to it,
    # against the oracle's cover of each chunk with the first ids after it
    lines = (tmp_path / "gpucover.log").read_text().splitlines()
    assert lines[0].split() == ["Gate:"] + [str(i) for i in range(back.n_pi)]
    body = [ln.split("\t", 1) for ln in lines[1:]]
    assert [b[0] for b in body] == [f"Vector {p}:" for p in range(n)]
    got = np.array([[int(x) for x in b[1].split()] for b in body], dtype=object).T
    for a in range(0, n, 64):
        b = min(n, a + 64)
        wk = O.grade(back, codes[:, :b], b, chunk=64)
        _, _, want = O.cover(back, w.mark[:, a:b], b - a, a, wk.first_x, wk.first_y, want_counts=True)
        want = want[:, :, 0].astype(object) + (want[:, :, 1].astype(object) << 64)
        np.testing.assert_array_equal(got[:, a:b], want)
    assert int(got.sum()) == w.total


@pytest.mark.gpu
@pytest.mark.parametrize("tile", [0, 32])
def test_cover_counts_equal_oracle(tile):
    """pdf_cover_counts: every primary input's count for every pair, and
    their sum the chunk's count."""
    import torch
    nl = circuits.random_small(79, n_gates=600, n_pi=24, n_po=80, depth=10, mask=circuits.MARKING_TYPES)
    n = 1500
    codes = helpers.rand_codes(np.random.default_rng(2), nl.n_pi, n)
    w = O.grade(nl, codes, n, want_planes=True)
    c = P.Circuit(nl, tile_words=tile)
    s = P.State(c)
    mk = torch.from_numpy(_planes(w.mark).view(np.int32)).cuda()
    sv = torch.from_numpy(_planes(w.sim & 1).view(np.int32)).cuda()
    P.stage_merge(c, s, sv, mk, n, 0)
    tot, raw = P.stage_cover_counts(c, s, mk, n, 0)
    _, _, want = O.cover(nl, w.mark, n, 0, w.first_x, w.first_y, want_counts=True)
    np.testing.assert_array_equal(raw, want)
    assert tot.value == w.total > 0
    assert int(raw[:, :, 0].astype(object).sum()) == w.total


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_mark_forward_equals_oracle_unpruned(mode):
    import torch
    for name, nl in circuits.small_suite()[:6]:
        n = 777
        rng = np.random.default_rng(3)
        codes = helpers.rand_codes(rng, nl.n_pi, n)
        sim = O.sim(nl, codes, n)
        ld = P.words(n) + 3
        sv = torch.from_numpy(_planes(sim & 1).view(np.int32)).cuda()
        st = torch.from_numpy(_planes(sim >> 1).view(np.int32)).cuda()
        pad = torch.zeros((nl.n_gates, ld - sv.shape[1]), dtype=torch.int32, device="cuda")
        sv, st = torch.cat([sv, pad], 1).contiguous(), torch.cat([st, pad], 1).contiguous()
        m = torch.full((nl.n_gates, ld), -1, dtype=torch.int32, device="cuda")
        c = P.Circuit(nl, mark_mode=mode)
        P.stage_mark_forward(c, sv, st, m, n)
        torch.cuda.synchronize()
        got = m.cpu().numpy().view(np.uint32)
        want = _planes(O.mark(nl, sim, n, mark_mode=mode, prune=False))
        np.testing.assert_array_equal(got[:, :want.shape[1]], want, err_msg=name)
