"""Spots of the reference's own tests, restated (ranges in the reference's
notation are parsed by the oracle's restatement of Range::from_str)."""
from __future__ import annotations

import numpy as np

from oracle_api import parse_range
from poker_trainer_b200 import abi

# crates/solver/src/gpu/testutil.rs:61-138 and crates/solver/src/tests.rs.
OOP_T = "AQ, KQ, QJs, JTs, 99, 44, T9s, 87s, A5s, KJs"
IP_T = "AA, KK, AQ, QT, 99, JJ, TT, 98s, KJs, 65s, AJs"


def config(board, oop, ip, pot, stack, menu=None, **kw):
    return abi.make_config(board, [parse_range(oop), parse_range(ip)], pot=pot, stack=stack,
                           menu_=menu if menu is not None else abi.default_menu(), **kw)


def river_config(**kw):
    """testutil.rs:61-71 (default live-game menu)."""
    return config("Qh9d4c2sKs", OOP_T, IP_T, 600, 4000, storage=abi.STORAGE_F32, **kw)


def turn_config(**kw):
    """testutil.rs:79-89: 48 rivers, no suit isomorphism."""
    return config("Qh9d4c2s", OOP_T, IP_T, 600, 4000, storage=abi.STORAGE_F32, **kw)


def iso_turn_config(**kw):
    """testutil.rs:94-104: clubs and hearts interchangeable."""
    return config("Qs9s4d2d", "AQ, KQ, QJs, JTs, 99, 44, T9s, 87s, A5s, KJs, 65s",
                  "AA, KK, AQ, QT, 99, JJ, TT, 98s, KJs, 65s, AJs, 33", 600, 4000, storage=abi.STORAGE_F32, **kw)


def allin_turn_config(**kw):
    """testutil.rs:108-118: pot-sized bet is all-in; runouts to showdowns."""
    return config("Kc8d5h3s", "AA, KK, KQ, 88, 55, A5s, 76s, QJs, JTs, 44, 98s",
                  "AK, KQ, KJ, 99, 33, A4s, T9s, 87s, 66, 76s", 1000, 900, abi.menu(["100%"], []),
                  storage=abi.STORAGE_F32, **kw)


def sampled_flop_config(**kw):
    """tests.rs:151-170: a flop with ChanceMode::Sampled {turn: 8, river: 6,
    seed: 3} and a one-size future menu."""
    return config("Kh7d2c", "AK, KQ, 77, 22, AJs, QJs, T9s, 65s, A5s",
                  "AK, KJ, QQ, JJ, 88, A7s, 98s, JTs, 76s", 600, 9700,
                  future_menu=abi.menu(["66%"], ["3x"]), sampled=(8, 6, 3), **kw)


def sampled_turn_config(seed=3, river=6, **kw):
    """The turn spot of testutil.rs:79-89 with sampled rivers."""
    return turn_config(sampled=(8, river, seed), **kw)


def sampled_allin_turn_config(seed=5, **kw):
    """The all-in turn spot (testutil.rs:108-118) with sampled rivers: the
    pot-sized bet's all-in runouts stay exact, the checked-through rivers
    are sampled."""
    return allin_turn_config(sampled=(8, 5, seed), **kw)


def sampled_iso_flop_config(seed=7, **kw):
    """A flop with clubs and hearts interchangeable (the ranges of
    testutil.rs:94-104 on Qs9s4d) and a short stack, sampled 6 turns and 4
    rivers: all-in runouts stay exact and use isomorphism, so the tree's size
    depends on which turn cards the sample drew."""
    return config("Qs9s4d", "AQ, KQ, QJs, JTs, 99, 44, T9s, 87s, A5s, KJs, 65s",
                  "AA, KK, AQ, QT, 99, JJ, TT, 98s, KJs, 65s, AJs, 33", 600, 1500,
                  abi.menu(["100%"], ["3x"]), storage=abi.STORAGE_F32, sampled=(6, 4, seed), **kw)


def facing_bet(pot, stack, bet):
    """testutil.rs:152-164."""
    return abi.betting_state(abi.RIVER, pot + bet, (0, bet), (stack, stack - bet), bet, bet, 1, 0, (True, False))


def mid_street_config(rake: bool, **kw):
    """testutil.rs:138-150: OOP faces a half-pot bet; ties pay."""
    extra = dict(rake_rate=0.05, rake_cap=300.0) if rake else {}
    extra.update(kw)
    return abi.make_config("Kc8d5h3s2c", [parse_range("AA, KK, KQ, KJ, 88, 55, A5s, 76s, QJs, JTs, 44"),
                                          parse_range("AK, KQ, KJ, KT, 99, 33, A4s, T9s, 87s, 66")],
                           root=facing_bet(1000, 5000, 500), menu_=abi.menu(["50%", "100%"], ["3x"]),
                           storage=abi.STORAGE_F32, **extra)


def random_range(rng, density):
    w = np.where(rng.random(1326) < density, rng.uniform(0.05, 1.0, 1326), 0.0)
    return w.astype(np.float32)


def random_river_config(seed: int):
    """A random river spot in the manner of arb_river_config
    (testutil.rs:199-234): board, sparse-to-dense ranges, pot, stack
    (sometimes none behind), one of three menus, optionally facing a bet and
    raked. numpy's default_rng replaces the proptest generator."""
    rng = np.random.default_rng(seed)
    board = rng.choice(52, 5, replace=False).tolist()
    r0 = random_range(rng, rng.uniform(0.02, 0.5))
    r1 = random_range(rng, rng.uniform(0.02, 0.5))
    pot = int(rng.integers(100, 3000))
    stack = 0 if rng.random() < 0.2 else int(rng.integers(100, 8000))
    m = int(rng.integers(0, 3))
    menu = [abi.menu(["50%", "100%"], ["100%"]), abi.menu(["33%"], []), abi.menu(["75%", "150%"], ["2.5x"])][m]
    kw = {}
    if rng.random() < 0.5:
        kw.update(rake_rate=0.05, rake_cap=300.0)
    cfg = abi.make_config(board, [r0, r1], pot=pot, stack=stack, menu_=menu, storage=abi.STORAGE_F32, **kw)
    if rng.random() < 0.5 and stack > pot // 2:
        cfg.root = facing_bet(pot, stack, pot // 2)
    return cfg


def random_turn_config(seed: int):
    """arb_turn_config (testutil.rs:170-193) with numpy's generator."""
    rng = np.random.default_rng(seed)
    board = rng.choice(52, 4, replace=False).tolist()
    r0 = random_range(rng, rng.uniform(0.02, 0.12))
    r1 = random_range(rng, rng.uniform(0.02, 0.12))
    pot = int(rng.integers(100, 2000))
    stack = int(rng.integers(100, 5000))
    kw = {}
    if rng.random() < 0.5:
        kw.update(rake_rate=0.05, rake_cap=300.0)
    return abi.make_config(board, [r0, r1], pot=pot, stack=stack, menu_=abi.menu(["50%", "100%"], ["100%"]),
                           storage=abi.STORAGE_F32, **kw)
