"""A second, independent restatement of the reference semantics in pure
Python, per pair, for tiny circuits: it checks the C oracle, and its cover
counts paths by explicit enumeration instead of the reference's dynamic
program (coverkernel.cuh:171-230), so it also checks that program.

Tables are the reference's constants (simkernel.cuh:158-165,
markkernel.cuh:36-37).
"""
from __future__ import annotations

INPT, AND, NAND, OR, NOR, XOR, XNOR, BUFF, NOT, FROM, DFF = 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11
S0, S1, T0, T1 = 0, 1, 2, 3

LUT2 = {
    NAND: [S1, S1, S1, S1, S1, S0, T1, T0, S1, T1, T1, S1, S1, T0, S1, T0],
    AND: [S0, S0, S0, S0, S0, S1, T0, T1, S0, T0, T0, S0, S0, T1, S0, T1],
    NOR: [S1, S0, T1, T0, S0, S0, S0, S0, T1, S0, T1, S0, T0, S0, S0, T0],
    OR: [S0, S1, T0, T1, S1, S1, S1, S1, T0, S1, T0, S1, T1, S1, S1, T1],
    XNOR: [S1, S0, T1, T0, S0, S1, T0, T1, T1, T0, S1, S0, T0, T1, S0, S1],
    XOR: [S0, S1, T0, T1, S1, S0, T1, T0, T0, T1, S0, S1, T1, T0, S1, S0],
}
STABLE = [S0, T0, T1, S1]
NOT_LUT = [S1, S0, T1, T0]
SENS = {  # mark_mode -> table indexed by type - 2
    0: [0x2A00, 0x2A00, 0x5100, 0x5100, 0, 0],
    1: [0x2200, 0x2200, 0x1100, 0x1100, 0, 0],
}
FIXED_MODES = (2, 3)  # true n-input gates; no reference counterpart


def fixed_side_ok(mode: int, t: int, on: int, off: int) -> bool:
    """FIXED side-input conditions stated from their definitions (not as tables):
    robust: on c->nc needs side steady nc, on nc->c side final nc, XOR steady;
    non-robust: side final value nc, XOR any.  on must transition."""
    if on < 2:
        return False
    xor = t in (XOR, XNOR)
    nc = 1 if t in (AND, NAND) else 0           # non-controlling value
    off_final, off_steady = off & 1, off < 2
    if mode == 3:
        return True if xor else off_final == nc
    if xor:
        return off_steady
    on_final = on & 1
    if on_final == nc:                          # c -> nc
        return off_steady and off_final == nc
    return off_final == nc                      # nc -> c


def per_vector(op, a: int, b: int) -> int:
    """Code of op applied to each of the two vectors of codes a and b."""
    a2, b2 = a & 1, b & 1
    a1, b1 = a2 ^ (a >> 1), b2 ^ (b >> 1)
    v1, v2 = op(a1, b1) & 1, op(a2, b2) & 1
    return v2 | ((v1 ^ v2) << 1)


def sim_pair(nl, pi_codes, p, mode: int = 0):
    G = nl.n_gates
    val = [0] * G
    for g in range(G):
        t = int(nl.type[g])
        fi = [int(x) for x in nl.fanins(g)]
        if mode in FIXED_MODES and AND <= t <= XNOR:
            bits = [[(val[f] & 1) ^ (val[f] >> 1) for f in fi], [val[f] & 1 for f in fi]]
            out = []
            for vs in bits:  # vector 1, vector 2
                if t in (AND, NAND):
                    o = int(all(vs))
                elif t in (OR, NOR):
                    o = int(any(vs))
                else:
                    o = sum(vs) & 1
                out.append(o ^ (1 if t in (NAND, NOR, XNOR) else 0))
            v1, v2 = out
            val[g] = v2 | ((v1 ^ v2) << 1)
        elif t == INPT:
            val[g] = int(pi_codes[g][p])
        elif t in (BUFF, FROM, DFF):
            val[g] = val[fi[0]]
        else:
            v = val[fi[0]]
            if t == NOT:
                v = NOT_LUT[v]
            for f in fi[1:]:
                # the coalesced simLUT evaluates only AND/NAND/OR/NOR; else 0
                v = LUT2[t][val[f] * 4 + v] if t in (AND, NAND, OR, NOR) else 0
            val[g] = v
    return val


def mark_pair(nl, val, mode: int, prune: bool = True):
    G = nl.n_gates
    m = [0] * G
    for g in range(G):
        t = int(nl.type[g])
        fi = [int(x) for x in nl.fanins(g)]
        trans = 1 if val[g] > 1 else 0
        if t == INPT:
            r = trans
        elif t in (FROM, BUFF, DFF, NOT):
            r = m[fi[0]]
        elif AND <= t <= XNOR and mode in FIXED_MODES:
            r = 0
            for i in range(len(fi)):
                ok = all(fixed_side_ok(mode, t, val[fi[i]], val[fi[j]]) for j in range(len(fi)) if j != i)
                r |= int(ok) & m[fi[i]]
        elif AND <= t <= XNOR:
            r = 0
            for i in range(len(fi)):
                ok = all((SENS[mode][t - 2] >> (val[fi[i]] * 4 + val[fi[j]])) & 1
                         for j in range(len(fi)) if j != i)
                r |= int(ok) & m[fi[0]]
        else:
            r = 0
        m[g] = r & trans
    if prune:
        for g in reversed(range(G)):
            keep = 1 if nl.po[g] else 0
            for fo in nl.fanouts(g):
                keep |= m[int(fo)]
            m[g] &= keep
    return m


def grade(nl, pi_codes, n_pairs: int, mode: int = 0, pair_base: int = 0, first_x=None, first_y=None):
    """Returns (vals[p][g], marks[p][g], first_x, first_y, total) with the cover
    counted by enumerating every marked input-to-output path per pair."""
    G = nl.n_gates
    fx = [0xFFFFFFFF] * G if first_x is None else list(first_x)
    fy = [0xFFFFFFFF] * G if first_y is None else list(first_y)
    vals, marks = [], []
    for p in range(n_pairs):
        v = sim_pair(nl, pi_codes, p, mode)
        m = mark_pair(nl, v, mode)
        vals.append(v)
        marks.append(m)
        for g in range(G):
            if m[g]:
                pid = pair_base + p
                if v[g] & 1:
                    fy[g] = min(fy[g], pid)
                else:
                    fx[g] = min(fx[g], pid)
    total = 0
    lvl0 = int(nl.level_offsets[1])
    for p in range(n_pairs):
        pid = pair_base + p
        m = marks[p]

        def paths(g, credited):
            if not m[g]:
                return 0
            cr = credited or fx[g] == pid or fy[g] == pid
            n = 1 if (nl.po[g] == 1 and cr) else 0
            for fo in nl.fanouts(g):
                n += paths(int(fo), cr)
            return n

        for g in range(lvl0):
            if nl.type[g] == INPT:
                total += paths(g, False)
    return vals, marks, fx, fy, total


def segments(nl, N: int):
    """Directed subpaths of exactly N nets, by first net ascending, then depth
    first along fan-outs in edge order."""
    out = []

    def walk(path):
        if len(path) == N:
            out.append(tuple(path))
            return
        for fo in nl.fanouts(path[-1]):
            walk(path + [int(fo)])

    for g in range(nl.n_gates):
        walk([g])
    return out


def grade_seg(nl, pi_codes, n_pairs: int, N: int, mode: int = 0, pair_base: int = 0):
    """Segments of N nets: a segment's first pair marks all its nets (x/y by
    the first net's value); a pair is credited at a net when it first-detects
    a segment through the net; paths enumerated per pair."""
    segs = segments(nl, N)
    fx = [0xFFFFFFFF] * len(segs)
    fy = [0xFFFFFFFF] * len(segs)
    vals, marks = [], []
    for p in range(n_pairs):
        v = sim_pair(nl, pi_codes, p, mode)
        m = mark_pair(nl, v, mode)
        vals.append(v)
        marks.append(m)
        for k, sg in enumerate(segs):
            if all(m[g] for g in sg):
                if v[sg[0]] & 1:
                    fy[k] = min(fy[k], pair_base + p)
                else:
                    fx[k] = min(fx[k], pair_base + p)
    total = 0
    lvl0 = int(nl.level_offsets[1])
    for p in range(n_pairs):
        pid = pair_base + p
        m = marks[p]
        firsts = set()
        for k, sg in enumerate(segs):
            if fx[k] == pid or fy[k] == pid:
                firsts.update(sg)

        def paths(g, credited):
            if not m[g]:
                return 0
            cr = credited or g in firsts
            n = 1 if (nl.po[g] == 1 and cr) else 0
            for fo in nl.fanouts(g):
                n += paths(int(fo), cr)
            return n

        for g in range(lvl0):
            if nl.type[g] == INPT:
                total += paths(g, False)
    return segs, fx, fy, total
