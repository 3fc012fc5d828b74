"""Test circuits: seeded random netlists of many shapes plus hand-built edge
cases (all built here; the reference ships no circuits)."""
from __future__ import annotations

import numpy as np

import helpers

P = helpers.pdf()

ALL_TYPES = sum(1 << t for t in (P.AND, P.NAND, P.OR, P.NOR, P.XOR, P.XNOR, P.NOT, P.BUFF))
MARKING_TYPES = sum(1 << t for t in (P.AND, P.NAND, P.OR, P.NOR, P.NOT, P.BUFF))
WITH_FROM_DFF = ALL_TYPES | (1 << P.FROM) | (1 << P.DFF)


def random_small(seed: int, n_gates=60, n_pi=8, n_po=20, depth=6, fmin=1, fmax=4, mask=ALL_TYPES,
                 zipf=False, fo_max=0):
    return P.gen_netlist(P.GenParams(seed, n_gates, n_pi, n_po, depth, fmin, fmax,
                                     1 if zipf else 0, 1.5, fo_max, mask))


def small_suite():
    """(name, netlist) pairs: shapes that give nonzero counts and exercise the
    reference's quirks (nfi = 1 on 2-input types, 3/4-input NAND/NOR folds,
    XOR with several inputs, FROM/DFF copies)."""
    out = []
    for i in range(6):
        out.append((f"mix{i}", random_small(1000 + i)))
    for i in range(3):
        out.append((f"marking{i}", random_small(2000 + i, n_gates=80, n_pi=10, n_po=30, depth=8,
                                                mask=MARKING_TYPES)))
    out.append(("wide_fanin", random_small(3000, n_gates=70, n_pi=12, n_po=25, depth=5, fmin=3, fmax=6,
                                           mask=(1 << P.NAND) | (1 << P.NOR) | (1 << P.AND) | (1 << P.OR))))
    out.append(("from_dff", random_small(3001, n_gates=50, n_pi=6, n_po=20, depth=7, mask=WITH_FROM_DFF)))
    out.append(("zipf", random_small(3002, n_gates=90, n_pi=10, n_po=30, depth=6, zipf=True, fo_max=40)))
    out.append(("deep", random_small(3003, n_gates=120, n_pi=6, n_po=60, depth=30)))
    return out


def diamond_chain(k: int):
    """x0 (PI) -> k stages of {a = BUFF(x), b = NOT(x), c = NOT(x),
    y = NAND(a, b, c)}.  Under a falling input every net transitions, the
    3-input NAND folds as NAND(NAND(a, b), c) = T0 and is marked under the
    default table, so the PI reaches the last y along 3^k marked paths."""
    levels = [[0]]
    types = {0: P.INPT}
    fanins = {0: []}
    x, g = 0, 1
    for _ in range(k):
        a, b, c, y = g, g + 1, g + 2, g + 3
        levels.append([a, b, c])
        levels.append([y])
        types.update({a: P.BUFF, b: P.NOT, c: P.NOT, y: P.NAND})
        fanins.update({a: [x], b: [x], c: [x], y: [a, b, c]})
        x, g = y, g + 4
    return P.Netlist.from_fanins(levels, types, [fanins[i] for i in range(g)], [x])


def hub(n_fanout: int = 200, seed: int = 7):
    """A primary input driving n_fanout BUFFs (fan-out >= 128 takes the
    reference's global-memory branch, markkernel.cuh:284-288), half of them
    outputs, plus a second level of 2-input gates."""
    rng = np.random.default_rng(seed)
    levels = [[0, 1, 2], list(range(3, 3 + n_fanout))]
    G1 = 3 + n_fanout
    lvl2 = list(range(G1, G1 + 40))
    levels.append(lvl2)
    types = {0: P.INPT, 1: P.INPT, 2: P.INPT}
    fanins = {}
    for g in levels[1]:
        types[g] = P.BUFF if g % 3 else P.NOT
        fanins[g] = [0]
    for g in lvl2:
        types[g] = int(rng.choice([P.AND, P.OR, P.NAND, P.NOR]))
        fanins[g] = [int(rng.choice(levels[1])), int(rng.choice([1, 2]))]
    G = G1 + 40
    pos = [g for g in levels[1] if g % 2] + lvl2[:20]
    return P.Netlist.from_fanins(levels, [types.get(g, P.INPT) for g in range(G)],
                                 [fanins.get(g, []) for g in range(G)], pos)


def unknown_types():
    """Gate codes outside the reference's switch (UNKN) and single-input
    XOR/XNOR/AND: they pass fan-in 0 through with one input and yield S0 with
    more (simkernel.cuh:131-148, Q1-Q3)."""
    levels = [[0, 1, 2, 3], [4, 5, 6, 7, 8, 9], [10, 11]]
    types = [P.INPT] * 4 + [P.UNKN, P.UNKN, P.XOR, P.XNOR, P.AND, P.NOT, P.XOR, P.OR]
    fanins = [[], [], [], [], [0], [1, 2], [3], [0, 1], [2], [0, 3], [4, 6], [8, 9]]
    return P.Netlist.from_fanins(levels, types, fanins, [4, 5, 6, 7, 8, 9, 10, 11])
