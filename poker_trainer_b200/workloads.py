"""Seeded synthetic spots: the river, turn, flop and batched-river solves.

No public benchmark or dataset exists for this path; each spot is generated
from numpy's default_rng with fixed seeds, and the same config object feeds
the GPU solver, the CPU oracle and the benchmark.

River / turn / flop spots use the board, pot, stack, menu and DCFR
parameters of the heads-up solve being benchmarked (alpha 1.5, beta 0,
gamma 2, restarted and unweighted averages as in the reference's
DcfrParams::default, crates/solver/src/cfr.rs:72-80, with gamma passed
explicitly). Ranges are per-class weights expanded to the class's combos
(HandClass::combos, crates/holdem/src/combo.rs:127-149); combos touching
the board are dropped by the solver's HandSet (hands.rs:35-55).
"""
from __future__ import annotations

import numpy as np

from . import abi

DCFR = dict(alpha=1.5, beta=0.0, gamma=2.0, restart_average=True, unweighted_average=True)


def class_combos() -> list[list[int]]:
    """Combo ids of the 169 classes in grid order (combo.rs:98-149)."""
    out = []
    for g in range(169):
        row, col = divmod(g, 13)
        r1, r2 = 12 - row, 12 - col
        hi, lo = max(r1, r2), min(r1, r2)
        pair = hi == lo
        suited = (row < col) and not pair
        combos = []
        for s1 in range(4):
            for s2 in range(4):
                a, b = hi * 4 + s1, lo * 4 + s2
                if a == b:
                    continue
                ok = s1 < s2 if pair else (s1 == s2 if suited else s1 != s2)
                if ok:
                    combos.append(abi.combo_index(a, b))
        out.append(combos)
    return out


_CLASSES = None


def expand_classes(w169: np.ndarray) -> np.ndarray:
    global _CLASSES
    if _CLASSES is None:
        _CLASSES = class_combos()
    out = np.zeros(1326, np.float32)
    for g, combos in enumerate(_CLASSES):
        out[combos] = np.float32(w169[g])
    return out


def uniform_range(seed: int, zero_classes: int = 0) -> np.ndarray:
    """Class weights ~ U[0,1) from default_rng(seed); then `zero_classes`
    classes chosen by rng.choice(169, k, replace=False) are zeroed."""
    rng = np.random.default_rng(seed)
    w = rng.random(169)
    if zero_classes:
        w[rng.choice(169, zero_classes, replace=False)] = 0.0
    return expand_classes(w)


def dirichlet_range(seed: int, keep: int = 68) -> np.ndarray:
    """169-class Dirichlet(0.5), the top `keep` classes kept, d / max(d)."""
    rng = np.random.default_rng(seed)
    d = rng.dirichlet(np.full(169, 0.5))
    order = np.argsort(-d, kind="stable")
    w = np.zeros(169)
    w[order[:keep]] = d[order[:keep]] / d[order[0]]
    return expand_classes(w)


def river_menu() -> abi.Menu:
    return abi.menu(["50%", "100%", "allin"], ["2.5x"], max_raises=3)


def turn_menu() -> abi.Menu:
    return abi.menu(["33%", "75%", "allin"], ["2.5x"], max_raises=3)


def flop_menu() -> abi.Menu:
    return abi.menu(["33%", "75%", "allin"], ["3x"], max_raises=3)


def river_spot(**over) -> abi.Config:
    """River subgame Ks7s2dTh4c, pot 20bb, stacks 90bb, 50%/100%/all-in bets,
    2.5x raise, max 3 bets; uniform class weights, seeds 1000/1001."""
    kw = dict(DCFR, storage=abi.STORAGE_F32)
    kw.update(over)
    return abi.make_config("Ks7s2dTh4c", [uniform_range(1000), uniform_range(1001)], pot=2000, stack=9000,
                           menu_=river_menu(), **kw)


def turn_spot(**over) -> abi.Config:
    """Turn subgame Ks7s2dTh (48 rivers), pot 20bb, stacks 90bb, 33%/75%/all-in
    on turn and river, 2.5x raise; 51 of 169 classes zeroed per player."""
    kw = dict(DCFR, storage=abi.STORAGE_F32)
    kw.update(over)
    return abi.make_config("Ks7s2dTh", [uniform_range(1000, 51), uniform_range(1001, 51)], pot=2000, stack=9000,
                           menu_=turn_menu(), **kw)


def turn_narrow_spot(**over) -> abi.Config:
    """The turn subgame of turn_spot with the flop workload's narrow ranges
    (Dirichlet(0.5) classes thresholded to 68 of 169, seeds 2000/2001): a few
    hundred hands per player, the regime of the warp-per-terminal kernel."""
    kw = dict(DCFR, storage=abi.STORAGE_F32)
    kw.update(over)
    return abi.make_config("Ks7s2dTh", [dirichlet_range(2000), dirichlet_range(2001)], pot=2000, stack=9000,
                           menu_=turn_menu(), **kw)


def flop_spot(**over) -> abi.Config:
    """Flop Ks7s2d, pot 6bb, stacks 97bb, 33%/75%/all-in on every street, 3x
    raise; Dirichlet(0.5) class ranges thresholded to 68 classes; f32,
    isomorphism on (clubs and hearts interchangeable)."""
    kw = dict(DCFR, storage=abi.STORAGE_F32, max_memory_bytes=1 << 40)
    kw.update(over)
    return abi.make_config("Ks7s2d", [dirichlet_range(2000), dirichlet_range(2001)], pot=600, stack=9700,
                           menu_=flop_menu(), **kw)


SIZES = ["33%", "50%", "75%", "100%", "150%"]


def batched_river_spots(count: int = 512, seed: int = 3000, estimate=None, min_nodes=15, max_nodes=400):
    """Independent river spots: 5-card boards from the seed, pot U[400,6000],
    stack U[2000,15000], a menu of 1-3 sizes from {33,50,75,100,150}% plus
    all-in used for bets and raises alike (max 3 bets); redrawn until the
    tree has min_nodes..max_nodes nodes (`estimate(cfg)` gives the node
    count). The sizes serve raises too because a single 2.5x raise caps
    these trees at 63 nodes, short of the 15-400 spread the workload asks
    for. Ranges as the river spot with per-spot seeds."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        board = rng.choice(52, 5, replace=False).tolist()
        pot = int(rng.integers(400, 6001))
        stack = int(rng.integers(2000, 15001))
        k = int(rng.integers(1, 4))
        sizes = sorted(rng.choice(len(SIZES), k, replace=False).tolist())
        bet = [SIZES[i] for i in sizes] + ["allin"]
        i = len(out)
        cfg = abi.make_config(board, [uniform_range(seed + 2 * i + 1), uniform_range(seed + 2 * i + 2)], pot=pot,
                              stack=stack, menu_=abi.menu(bet, bet, max_raises=3),
                              storage=abi.STORAGE_F32, **DCFR)
        if estimate is not None:
            n = estimate(cfg)
            if not (min_nodes <= n <= max_nodes):
                continue
        out.append(cfg)
    return out
