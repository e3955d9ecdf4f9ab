"""Training data for the leaf-value network: turn subgames solved by the GPU
solver.

A sample is one turn subgame of the flop workload: board Ks7s2d plus a turn
card, a pot and effective stack reachable from the flop tree (both players
put the same amount in on the flop: log-uniform pots from 600 to 12000
chips, and all-in pots of 20000 with nothing behind 15% of the time), and
both players' ranges narrowed from the flop ranges by seeded random
per-class factors. The subgame is solved by
libdcfr (fast precision, DCFR alpha 1.5 beta 0 gamma 2) to a target
exploitability; the target of the sample is every hand's expected value
under the average strategies, per player, in units of the pot.

Encoding (input 2 x 1326 + 52 + 2 = 2706 floats):
  [range of player 0 / its max (combo order), range of player 1 / its max,
   one-hot of the 4 board cards, pot / 10000, stack / 10000]
Output (2 x 1326): [EV of player 0's combos / pot, EV of player 1's / pot];
the mask is 1 for combos in the player's range.

The value of a hand comes from one average-strategy traversal
(dcfr_traverse, mode AVERAGE): cfv[h] = norm * sum_j w_o[j] * u(h, j), so
EV(h) = cfv[h] / (norm * sum of the opponent's weights compatible with h),
with norm = 1 / sum over compatible pairs of w_0 * w_1 (hands.rs:95-125).
"""
from __future__ import annotations

import numpy as np

from . import abi, workloads
from .solver import Solver, SolveOptions

IN_DIM = 2 * 1326 + 52 + 2
OUT_DIM = 2 * 1326
FLOP = "Ks7s2d"
SCALE = 10000.0

_COMBO_CARDS = None


def combo_cards() -> np.ndarray:
    global _COMBO_CARDS
    if _COMBO_CARDS is None:
        _COMBO_CARDS = np.array([abi.combo_cards(i) for i in range(1326)], np.int64)
    return _COMBO_CARDS


def encode(r0, r1, board, pot, stack) -> np.ndarray:
    x = np.zeros(IN_DIM, np.float32)
    for p, r in enumerate((r0, r1)):
        m = float(np.max(r))
        if m > 0:
            x[p * 1326:(p + 1) * 1326] = r / m
    for c in board:
        x[2652 + c] = 1.0
    x[2704] = pot / SCALE
    x[2705] = stack / SCALE
    return x


def sample_state(rng, base0, base1):
    """A turn-subgame state reachable from the flop workload's tree."""
    flop = abi.parse_cards(FLOP)
    turn = int(rng.choice([c for c in range(52) if c not in flop]))
    board = flop + [turn]
    # Pots of the flop tree's leaves: both players put the same amount in on
    # the flop, from nothing (600) to all in (20000, nothing behind).
    if rng.random() < 0.15:
        pot = 600 + 2 * 9700
    else:
        pot = int(round(600 * 20.0 ** rng.random()))
    stack = max(0, 9700 - (pot - 600) // 2)
    ranges = []
    classes = workloads.class_combos()
    for base in (base0, base1):
        f = np.zeros(1326, np.float32)
        for g in range(169):
            f[classes[g]] = rng.random() ** 2
        r = (base * f).astype(np.float32)
        for c in board:
            r[(combo_cards() == c).any(axis=1)] = 0.0
        ranges.append(r)
    return board, pot, stack, ranges


def config_of(board, pot, stack, ranges):
    return abi.make_config(board, ranges, pot=pot, stack=stack, menu_=workloads.flop_menu(),
                           storage=abi.STORAGE_F32, **workloads.DCFR)


def hand_evs(g: Solver, cfg) -> tuple[np.ndarray, np.ndarray]:
    """Per-combo EV (chips, relative to the subgame start) of both players
    under the current average strategies, and the mask of valid combos."""
    ev = np.zeros((2, 1326), np.float64)
    mask = np.zeros((2, 1326), np.float32)
    hands = [g.hands(p) for p in range(2)]
    cards = [combo_cards()[h[0].astype(np.int64)] for h in hands]
    w = [h[1].astype(np.float64) for h in hands]
    overlap = ((cards[0][:, None, 0] == cards[1][None, :, 0]) | (cards[0][:, None, 0] == cards[1][None, :, 1]) |
               (cards[0][:, None, 1] == cards[1][None, :, 0]) | (cards[0][:, None, 1] == cards[1][None, :, 1]))
    compat = ~overlap
    total = float(w[0] @ compat @ w[1])
    norm = 1.0 / total
    mass = [compat @ w[1], compat.T @ w[0]]
    for p in range(2):
        cfv = g.traverse(p, abi.MODE_AVERAGE, g.iterations()).astype(np.float64)
        ok = mass[p] > 0
        e = np.zeros_like(cfv)
        e[ok] = cfv[ok] / (norm * mass[p][ok])
        ev[p, hands[p][0]] = e
        mask[p, hands[p][0]] = ok.astype(np.float32)
    return ev, mask


def solve_sample(state, target_pct=0.3, max_iterations=400, check_every=25):
    board, pot, stack, ranges = state
    cfg = config_of(board, pot, stack, ranges)
    g = Solver.new(cfg)
    try:
        prog = g.solve(SolveOptions(max_iterations=max_iterations, target_exploitability_pct=target_pct,
                                    check_every=check_every))
        ev, mask = hand_evs(g, cfg)
        return ev, mask, prog
    finally:
        g.close()


def equity_evs(state):
    """The method without the network: the same state with no chips behind,
    i.e. checked down to showdown (pot split by equity), solved exactly."""
    board, pot, _, ranges = state
    cfg = config_of(board, pot, 0, ranges)
    g = Solver.new(cfg)
    try:
        g.iterate(1)
        return hand_evs(g, cfg)
    finally:
        g.close()


def make_dataset(n: int, seed: int = 4000, target_pct=0.3, max_iterations=400, with_equity=False, base=None,
                 workers: int = 4, part=(0, 1)):
    """n solved samples: inputs [n][2706], targets [n][2652] (EV / pot),
    masks [n][2652] and, optionally, the equity baseline's targets.

    The states are drawn in order from the seed; `workers` host threads then
    solve them concurrently, each with its own solver handle (its own CUDA
    stream and graphs), so one subgame's host-side setup overlaps another's
    GPU iterations. Every solve is deterministic, so the dataset does not
    depend on `workers`. part = (r, R) solves and returns only the samples
    r, r + R, ... (rank r of R data-parallel ranks)."""
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(seed)
    if base is None:
        base = (workloads.dirichlet_range(2000), workloads.dirichlet_range(2001))
    states = [sample_state(rng, *base) for _ in range(n)]
    states = states[part[0]::part[1]]
    n = len(states)
    X = np.zeros((n, IN_DIM), np.float32)
    Y = np.zeros((n, OUT_DIM), np.float32)
    M = np.zeros((n, OUT_DIM), np.float32)
    E = np.zeros((n, OUT_DIM), np.float32) if with_equity else None
    iters = [0] * n

    def one(i):
        st = states[i]
        board, pot, stack, ranges = st
        ev, mask, prog = solve_sample(st, target_pct, max_iterations)
        X[i] = encode(ranges[0], ranges[1], board, pot, stack)
        Y[i] = (ev / pot).reshape(-1)
        M[i] = mask.reshape(-1)
        iters[i] = prog.iteration
        if with_equity:
            eq, _ = equity_evs(st)
            E[i] = (eq / pot).reshape(-1)

    if workers <= 1:
        for i in range(n):
            one(i)
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            list(ex.map(one, range(n)))
    return X, Y, M, E, iters
