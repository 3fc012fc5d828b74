"""Path segments of N = 2..8 nets (fcount --segs N; main.cu:185-223,
mergekernel.cuh:99-198, coverkernel.cuh:115-230) against the oracle's
restatement: the segment list, the per-segment first pairs and the covered
path count, through the fused grade (one batch and many), the stage calls
and the command line.  The reference's segment generator is not in its
snapshot, so the list follows the oracle's stated definition."""
import re
import subprocess

import numpy as np
import pytest

import circuits
import helpers

P = helpers.pdf()
O = helpers.oracle()
SUITE = circuits.small_suite()


def test_segment_length_is_checked_before_the_device():
    nl = SUITE[0][1]
    with pytest.raises(P.PdfError):
        P.Circuit(nl, seg_len=9)


def _grade(nl, codes, n, N, mode=0, batches=None, **opts):
    c = P.Circuit(nl, mark_mode=mode, seg_len=N, **opts)
    s = P.State(c)
    for b0, b1 in batches or [(0, n)]:
        v, t = P.planes_from_codes(np.ascontiguousarray(codes[:, b0:b1]), P.words(b1 - b0))
        P.grade(c, s, v, t, b1 - b0, pair_base=b0)
    fx, fy, tot = s.snapshot()
    return c, fx, fy, tot


@pytest.mark.gpu
@pytest.mark.parametrize("N", [2, 3, 5, 8])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_grade_segments_equal_oracle(N, mode):
    seen = 0
    # 24 levels of AND/OR/NOT/BUFF with 1-2 fan-ins: marks reach 8 nets deep
    deep = ("deep", circuits.random_small(777, n_gates=900, n_pi=24, n_po=60, depth=24, fmax=2,
                                          mask=(1 << P.AND) | (1 << P.OR) | (1 << P.BUFF) | (1 << P.NOT)))
    for idx, (name, nl) in enumerate(SUITE + [deep]):
        rng = np.random.default_rng(200 + idx)
        n = 700
        codes = helpers.rand_codes(rng, nl.n_pi, n)
        want = O.grade_seg(nl, codes, n, N, mark_mode=mode)
        c, fx, fy, tot = _grade(nl, codes, n, N, mode)
        np.testing.assert_array_equal(c.segments(), want.segs, err_msg=name)
        np.testing.assert_array_equal(fx, want.first_x, err_msg=name)
        np.testing.assert_array_equal(fy, want.first_y, err_msg=name)
        assert tot.value == want.total and tot.flags == want.flags, name
        seen += want.total
    assert seen > 0


@pytest.mark.gpu
@pytest.mark.parametrize("tile_words", [1, 4, 8])
def test_segments_in_batches_and_tiles(tile_words):
    nl = circuits.random_small(4444, n_gates=2500, n_pi=150, n_po=400, depth=12)
    rng = np.random.default_rng(12)
    n = 3000
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    want = O.grade_seg(nl, codes, n, 4, mark_mode=1)
    _, fx, fy, tot = _grade(nl, codes, n, 4, 1, batches=[(0, 1000), (1000, 1037), (1037, 3000)],
                            tile_words=tile_words)
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total and tot.pairs == n


@pytest.mark.gpu
def test_segments_with_planes_requested():
    """store-all planes (host outputs) take the same segment path."""
    nl = SUITE[2][1]
    rng = np.random.default_rng(13)
    n = 333
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    want = O.grade_seg(nl, codes, n, 3)
    c = P.Circuit(nl, seg_len=3)
    s = P.State(c)
    W = P.words(n)
    v, t = P.planes_from_codes(codes, W)
    mark = np.zeros((nl.n_gates, W), np.uint32)
    P.grade(c, s, v, t, n, mark=mark)
    fx, fy, tot = s.snapshot()
    assert tot.value == want.total
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(P.codes_from_planes(mark, mark, n) & 1, O.grade(nl, codes, n, want_planes=True).mark)


@pytest.mark.gpu
def test_segment_stage_calls_equal_oracle():
    import torch
    nl = SUITE[1][1]
    rng = np.random.default_rng(14)
    n = 500
    codes = helpers.rand_codes(rng, nl.n_pi, n)
    want = O.grade_seg(nl, codes, n, 2, mark_mode=0)
    c = P.Circuit(nl, seg_len=2)
    s = P.State(c)
    W = P.words(n)
    v, t = P.planes_from_codes(codes, W)
    dv = torch.from_numpy(v.view(np.int32)).cuda()
    dt = torch.from_numpy(t.view(np.int32)).cuda()
    G = nl.n_gates
    sv = torch.zeros((G, W), dtype=torch.int32, device="cuda")
    st = torch.zeros_like(sv)
    mk = torch.zeros_like(sv)
    P.stage_sim(c, dv, dt, n, sv, st)
    P.stage_mark(c, sv, st, mk, n)
    P.stage_merge(c, s, sv, mk, n, 0)
    tot = P.stage_cover(c, s, mk, n, 0)
    fx, fy, _ = s.snapshot()
    np.testing.assert_array_equal(fx, want.first_x)
    np.testing.assert_array_equal(fy, want.first_y)
    assert tot.value == want.total


@pytest.mark.gpu
def test_segments_refused_where_unsupported():
    import torch
    nl = SUITE[0][1]
    c = P.Circuit(nl, seg_len=2)
    s = P.State(c)
    n = 64
    v = torch.zeros((nl.n_pi, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(P.PdfError) as e:
        P.Batch([(c, s, v, v, n, 0)])
    assert e.value.status == 6  # PDF_ENOTSUP
    fxy = torch.full((c.n_first,), -1, dtype=torch.int32, device="cuda")
    mk = torch.zeros((nl.n_gates, 2), dtype=torch.int32, device="cuda")
    with pytest.raises(P.PdfError):
        P.stage_cover_noalloc(c, mk, n, 0, fxy, fxy)


@pytest.mark.gpu
def test_cli_segments(tmp_path):
    fcount = str(helpers.PKG_DIR / "fcount")
    nl = circuits.random_small(80, n_gates=800, n_pi=40, n_po=80, depth=14)
    level = str(tmp_path / "c.level")
    P.write_level(nl, level)
    rng = np.random.default_rng(6)
    vec = rng.integers(0, 2, size=(nl.n_pi, 300), dtype=np.uint8)
    vpath = tmp_path / "v.vec"
    vpath.write_text("".join("".join(map(str, vec[:, r])) + "\n" for r in range(300)))
    pv, pt = P.pairs_from_vectors(vec)
    codes = P.codes_from_planes(pv, pt, 300)
    for N in (2, 6):
        r = subprocess.run([fcount, "--segs", str(N), "--verbose", "--merge", "--num_patterns", "128",
                            "--bench", level, str(vpath)], capture_output=True, text=True, cwd=str(tmp_path),
                           timeout=300)
        assert r.returncode == 0, r.stderr
        total = int(r.stdout.strip().split(";")[-1])
        want = O.grade_seg(nl, codes, 300, N)
        assert total == want.total
        assert r.stdout.split(":")[1].split(",")[2].startswith(str(N))
        lines = (tmp_path / "gpumerge.log").read_text().splitlines()
        assert len(lines) == len(want.segs)
        for k in (0, len(lines) // 2, len(lines) - 1):
            m = re.match(r"Segment (\d+)\(([\d,]+)\): (-?\d+),(-?\d+) $", lines[k])
            assert m and int(m.group(1)) == k
            assert [int(x) for x in m.group(2).split(",")] == list(want.segs[k])
            assert int(m.group(3)) & 0xFFFFFFFF == want.first_x[k]
            assert int(m.group(4)) & 0xFFFFFFFF == want.first_y[k]
