"""The FP64 best-response oracle on the GPU (dcfr_exploitability_fp64):
exploitability with every reach and value row of the best-response
traversals in double.

- On river spots it equals an independent float64 best response computed
  here with numpy (explicit hand-vs-hand payoff matrices on the oracle's
  tree and the GPU's strategy sums) to 1e-9 relative.
- On every test spot (chance nodes, suit isomorphism, all-in runouts, rake)
  it agrees with the solver's own f32 exploitability within 1e-4 relative,
  the tolerance of the reference's GPU-vs-CPU exploitability check.
"""
import numpy as np
import pytest

import spots
from oracle_api import HandSetOracle, OracleSolver, lib, ptr
from poker_trainer_b200 import abi, workloads
from poker_trainer_b200.solver import Solver

pytestmark = pytest.mark.gpu

SPOTS = {
    "river": spots.river_config,
    "turn": spots.turn_config,
    "iso_turn": spots.iso_turn_config,
    "allin_turn": spots.allin_turn_config,
    "mid_street_raked": lambda: spots.mid_street_config(True),
    "mid_street": lambda: spots.mid_street_config(False),
}


def strengths(board, cards):
    out = np.zeros(len(cards), np.int64)
    for i, (a, b) in enumerate(cards):
        c = np.array(list(board) + [int(a), int(b)], np.int32)
        out[i] = lib().oracle_evaluate(ptr(c), len(c))
    return out


def numpy_best_response(cfg, o, sums):
    """Best-response root values of both players in float64, river trees
    only: cfr.rs:259-479 with Mode::BestResponse, the opponent on the
    average strategy, terminals as eval.rs with explicit payoff matrices."""
    ints, offs, fl, _ = o.nodes()
    board = [cfg.board[i] for i in range(cfg.board_len)]
    hands = [o.hands(q) for q in range(2)]
    cards = [np.array([abi.combo_cards(int(c)) for c in hands[q][0]], np.int64).reshape(-1, 2) for q in range(2)]
    r0 = np.frombuffer(bytes(cfg.ranges[0]), np.float32)
    r1 = np.frombuffer(bytes(cfg.ranges[1]), np.float32)
    norm = 1.0 / HandSetOracle(r0, r1, board).num_combinations()
    half = cfg.root.pot / 2.0
    st = [strengths(board, cards[q]) for q in range(2)]
    res = np.zeros(2)
    for p in range(2):
        q = 1 - p
        cp, co = cards[p], cards[q]
        compat = ~((cp[:, None, 0] == co[None, :, 0]) | (cp[:, None, 0] == co[None, :, 1]) |
                   (cp[:, None, 1] == co[None, :, 0]) | (cp[:, None, 1] == co[None, :, 1]))
        cmp = np.sign(st[p][:, None] - st[q][None, :])

        def rec(v, r):
            kind, player, _, k, first, i0, i1 = ints[v][:7]
            inv = (float(i0), float(i1))
            rake = float(fl[v][0])
            if kind == 0:
                if player == p:
                    return np.max([rec(first + a, r) for a in range(k)], axis=0)
                n = len(hands[player][0])
                off = int(offs[v][0])
                s = sums[off:off + k * n].reshape(k, n).astype(np.float64)
                tot = s.sum(axis=0)
                sig = np.where(tot > 0, s / np.where(tot > 0, tot, 1.0), 1.0 / k)
                return np.sum([rec(first + a, sig[a] * r) for a in range(k)], axis=0)
            if kind == 2:
                val = -(half + inv[p]) if player == p else half + inv[player] - rake
                return val * norm * (compat @ r)
            assert kind == 3, "river trees only"
            win = (half + inv[q] - rake) * norm
            lose = -(half + inv[p]) * norm
            tie = 0.5 * ((inv[q] - inv[p]) - rake) * norm
            pay = np.where(cmp > 0, win, np.where(cmp < 0, lose, tie)) * compat
            return pay @ r

        vals = rec(0, hands[q][1].astype(np.float64))
        res[p] = float(vals @ hands[p][1].astype(np.float64))
    return res


@pytest.mark.parametrize("seed", range(6))
def test_fp64_best_response_matches_numpy_on_rivers(gpu, seed):
    cfg = spots.random_river_config(seed)
    cfg.rake_rate, cfg.rake_cap = 0.0, 0.0
    try:
        o = OracleSolver(cfg)
    except Exception:
        pytest.skip("spot rejected by Solver::new")
    g = Solver.new(cfg)
    g.iterate(25)
    _, sums = g.download_storage()
    e64, br = g.exploitability_fp64()
    ref = numpy_best_response(cfg, o, sums)
    scale = max(abs(ref[0]), abs(ref[1]), 1e-9)
    assert np.all(np.abs(br - ref) <= 1e-9 * scale), (br, ref)
    assert abs(e64 - ref.mean()) <= 1e-9 * scale


def test_fp64_best_response_matches_numpy_on_the_river_workload(gpu):
    cfg = workloads.river_spot()
    o = OracleSolver(cfg)
    g = Solver.new(cfg)
    g.iterate(200)
    _, sums = g.download_storage()
    _, br = g.exploitability_fp64()
    ref = numpy_best_response(cfg, o, sums)
    assert np.all(np.abs(br - ref) <= 1e-9 * np.max(np.abs(ref))), (br, ref)


@pytest.mark.parametrize("precision", ["fast", "exact"])
@pytest.mark.parametrize("name", list(SPOTS))
def test_fp64_tracks_f32_exploitability(gpu, name, precision):
    cfg = SPOTS[name]()
    cfg.precision = abi.PRECISIONS[precision]
    g = Solver.new(cfg)
    g.iterate(30)
    e32 = g.exploitability()
    e64, br = g.exploitability_fp64()
    assert np.isfinite(e64)
    # Relative to the exploitability, floored at 1e-7 of the best-response
    # values it is the difference of (f32 rounding of those values).
    assert abs(e64 - e32) <= 1e-4 * max(abs(e64), 1e-3 * float(np.max(np.abs(br)))), (e64, e32)
