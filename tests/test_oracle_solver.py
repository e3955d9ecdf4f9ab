"""The oracle's solver against the reference's own known-answer tests
(crates/solver/src/tests.rs:45-359, crates/solver/src/iso.rs:149-166),
restated on the oracle (the C++ restatement of the reference's CPU solver).
These pin the oracle before it is trusted as the checker of the GPU path.
CPU only."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import spots
from oracle_api import OracleError, OracleSolver, estimate, lib, parse_range, ptr
from poker_trainer_b200 import abi, workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kats.json")
KATS = json.load(open(GOLDEN))

CHECK = (abi.CHECK, 0)
CALL = (abi.CALL, 0)
FOLD = (abi.FOLD, 0)


def raise_to(x):
    return (abi.RAISE, x)


def config(board, oop, ip, pot, stack, menu, **kw):
    """tests.rs:19-29: street start with equal stacks, big blind 100."""
    return abi.make_config(board, [parse_range(oop), parse_range(ip)], pot=pot, stack=stack, menu_=menu, **kw)


def menu_one(bet, raise_):
    """tests.rs:6-17: the same sizes on every street, no all-in extras."""
    return abi.menu(bet, raise_, max_raises=3, add_allin=0.0, force_allin=0.0, merge=0.0)


def solve(cfg, iters, target, check_every=25):
    s = OracleSolver(cfg)
    p = s.solve(iters, target, check_every)
    return s, p


def combo(s):
    c = abi.parse_cards(s)
    return abi.combo_index(c[0], c[1])


def hand_index(q, combo_id):
    idx = np.nonzero(q["combos"] == combo_id)[0]
    assert len(idx) == 1
    return int(idx[0])


def facing_bet_root(pot, commit, stack, bet):
    return abi.betting_state(abi.RIVER, pot, (0, commit), (stack, stack - commit), bet, bet, 1, 0, (True, False))


def test_polarized_river_toy_game():
    """tests.rs:42-95: AA + half-weighted air vs bluff-catchers; pot-sized
    bet; bluff and call frequencies of one half."""
    cfg = config("Kc8d5h3s2c", "AA, JTs, J9s:0.5", "KQ", 1000, 5000, menu_one(["100%"], []))
    s, p = solve(cfg, 2000, 0.05)
    assert p.exploitability_pct < 0.2
    root = s.query([])
    assert root["actions"] == [CHECK, raise_to(1000)]
    aa = hand_index(root, combo("AsAh"))
    assert root["strategy"][1, aa] > 0.98
    assert abs(root["ev"][1, aa] - 1500.0) < 20.0
    assert abs(root["ev"][0, aa] - 1000.0) < 20.0
    cls = np.zeros(1326, np.uint8)
    lib().oracle_combo_class(ptr(cls))
    bet = tot = 0.0
    for i, c in enumerate(root["combos"]):
        hi, _ = abi.combo_cards(int(c))
        if hi // 4 == 9:  # J-high air
            bet += float(root["reach"][i]) * float(root["strategy"][1, i])
            tot += float(root["reach"][i])
            assert abs(root["ev"][0, i]) < 20.0 and abs(root["ev"][1, i]) < 40.0
    assert abs(bet / tot - 0.5) < 0.05
    facing = s.query([raise_to(1000)])
    assert facing["actions"] == [FOLD, CALL]
    w = facing["reach"].astype(np.float64)
    call = float((facing["strategy"][1] * w).sum() / w.sum())
    assert abs(call - 0.5) < 0.05
    kq = hand_index(facing, combo("KdQd"))
    assert abs(facing["ev"][0, kq]) < 1e-3 and abs(facing["ev"][1, kq]) < 30.0
    ranges = s.ranges_after([raise_to(1000)])
    assert ranges[0][combo("AsAh")] > 0.98
    assert 0.2 < ranges[0][combo("JsTs")] < 0.8


def test_all_in_equity_on_turn():
    """tests.rs:97-113: AA vs KK all-in on the turn; KK has 2 outs of 44."""
    cfg = config("2c7d9hTs", "AhAd", "KhKd", 1000, 1000, menu_one(["allin"], []))
    s, _ = solve(cfg, 50, 0.0)
    facing = s.query([raise_to(1000)])
    assert facing["actions"] == [FOLD, CALL]
    expected = 2.0 / 44.0 * 3000.0 - 1000.0
    assert abs(float(facing["ev"][1, 0]) - expected) < 0.5
    assert abs(facing["ev"][0, 0]) < 1e-3
    assert facing["strategy"][0, 0] > 0.99


def test_mid_street_root_with_ties():
    """tests.rs:115-135: facing a bet on a board where every hand chops."""
    cfg = config("AsKsQsJsTs", "22", "33", 1500, 5000, menu_one(["100%"], ["3x"]))
    cfg.root = facing_bet_root(1500, 500, 5000, 500)
    s, _ = solve(cfg, 200, 0.0)
    root = s.query([])
    assert root["actions"][:2] == [FOLD, CALL]
    assert abs(root["ev"][0, 0]) < 1e-3
    assert abs(root["ev"][1, 0] - 500.0) < 1.0


def test_turn_spot_converges():
    """tests.rs:137-156."""
    s = OracleSolver(spots.config("Qh9d4c2s", spots.OOP_T, spots.IP_T, 600, 4000))
    history = []
    p = s.solve(300, 0.3, 20, history)
    assert p.exploitability_pct < 0.5
    assert history[0][1] > history[-1][1]


def test_too_large_is_rejected():
    """tests.rs:178-185."""
    cfg = config("Kh7d2c", "any", "any", 600, 9700, abi.default_menu(), max_memory_bytes=1 << 20)
    with pytest.raises(OracleError) as e:
        OracleSolver(cfg)
    assert e.value.code == abi.ERR_TOO_LARGE


def test_empty_range_is_rejected():
    """SolverError::EmptyRange (lib.rs:186-192): a range with no hand left
    after board removal."""
    cfg = config("AsAhKd", "AsAh", "KK", 600, 9700, abi.default_menu())
    with pytest.raises(OracleError) as e:
        OracleSolver(cfg)
    assert e.value.code == abi.ERR_EMPTY_RANGE


def max_diff(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)), initial=0.0))


def assert_same_node(a, b, strat_tol, ev_tol):
    assert a["actions"] == b["actions"]
    assert np.array_equal(a["combos"], b["combos"])
    assert max_diff(a["strategy"], b["strategy"]) <= strat_tol
    assert max_diff(a["ev"], b["ev"]) <= ev_tol


def test_batched_river_matches_recursion():
    """tests.rs:197-231: the breadth-first batched river evaluator against
    plain recursion, 5 iterations."""
    a = OracleSolver(spots.turn_config())
    b = OracleSolver(spots.turn_config())
    b.set_batch_river(False)
    pa = a.solve(5, 0.0, 5)
    pb = b.solve(5, 0.0, 5)
    assert abs(pa.exploitability - pb.exploitability) < 1e-4 * (1.0 + abs(pb.exploitability))
    for path in ([], [CHECK], [CHECK, CHECK, "Ks"]):
        assert_same_node(a.query(path), b.query(path), 5e-5, 0.25)


def test_isomorphism_matches_full_tree():
    """tests.rs:233-273: a monotone turn solved with and without suit
    isomorphism, queried through canonical and mirrored rivers."""
    def make(iso):
        return config("Ks9s5s2s", "AA, KQ, QJ, T9, 87, 66, A5", "AK, KJ, JT, 98, 76, 55, Q2", 1000, 3000,
                      menu_one(["66%"], ["3x"]), isomorphism=iso, storage=abi.STORAGE_F32)
    a = OracleSolver(make(True))
    b = OracleSolver(make(False))
    assert a.isomorphic_pairs() >= 3
    sa, sb = a.stats(), b.stats()
    assert sa.player_nodes + sa.chance_nodes + sa.terminal_nodes < sb.player_nodes + sb.chance_nodes + sb.terminal_nodes
    pa = a.solve(60, 0.0, 60)
    pb = b.solve(60, 0.0, 60)
    assert abs(pa.exploitability - pb.exploitability) < 1e-2 * (1.0 + abs(pb.exploitability))
    assert_same_node(a.query([]), b.query([]), 2e-3, 0.5)
    for river in ["7c", "7d", "7h", "As", "Ah"]:
        path = [CHECK, CHECK, river]
        assert_same_node(a.query(path), b.query(path), 2e-3, 0.5)
        ra, rb = a.ranges_after(path), b.ranges_after(path)
        assert max_diff(ra[0], rb[0]) < 1e-3 and max_diff(ra[1], rb[1]) < 1e-3


def test_rake_reduces_chops():
    """tests.rs:305-325: pot 2000 after the call, rake 100, each gets 950."""
    cfg = config("AsKsQsJsTs", "22", "33", 1500, 5000, menu_one(["100%"], ["3x"]), rake_rate=0.05, rake_cap=300.0)
    cfg.root = facing_bet_root(1500, 500, 5000, 500)
    s, _ = solve(cfg, 200, 0.0)
    root = s.query([])
    assert abs(root["ev"][0, 0]) < 1e-3
    assert abs(root["ev"][1, 0] - 450.0) < 1.0


def test_rake_on_folds():
    """tests.rs:327-345: rake on a fold comes from the matched pot only."""
    cfg = config("Kc8d5h3s2c", "AA", "QJs", 1000, 5000, menu_one(["100%"], []), rake_rate=0.05, rake_cap=1e9)
    s, _ = solve(cfg, 300, 0.0)
    root = s.query([])
    aa = hand_index(root, combo("AsAh"))
    assert abs(root["ev"][1, aa] - 950.0) < 2.0
    assert abs(root["ev"][0, aa] - 950.0) < 2.0


@pytest.mark.parametrize("case", KATS["check_schedule"]["cases"])
def test_check_schedule(case):
    prev = case["prev"]
    t, e = case["cur"]
    g = lib().oracle_next_check_gap(prev is not None, prev[0] if prev else 0, prev[1] if prev else 0.0, t, e,
                                    case["target"], case["max_gap"])
    if "gap" in case:
        assert g == case["gap"]
    else:
        lo, hi = case["gap_range"]
        assert lo <= g < hi


@pytest.mark.parametrize("board,expected", KATS["iso"]["symmetric_pairs"])
def test_board_symmetric_pairs(board, expected):
    b = np.array(abi.parse_cards(board), np.int32)
    out = np.zeros(12, np.int32)
    n = lib().oracle_board_symmetric_pairs(ptr(b), len(b), ptr(out))
    if isinstance(expected, int):
        assert n == expected
    else:
        assert [list(out[2 * i:2 * i + 2]) for i in range(n)] == expected


@pytest.mark.parametrize("board,hand,size", KATS["iso"]["orbit"])
def test_iso_orbit(board, hand, size):
    b = np.array(abi.parse_cards(board), np.int32)
    out = np.zeros(8, np.int32)
    assert lib().oracle_iso_orbit(ptr(b), len(b), combo(hand), ptr(out)) == size


def test_discount_schedule():
    """Discount::new (cfr.rs:86-106) at alpha 1.5, beta 0, gamma 2 with
    restarted averages: pos = (t-1)^a / ((t-1)^a + 1), neg = 1/2,
    strat = (s/(s+1))^g with s counted from the last power of 4."""
    p = abi.Params(alpha=1.5, beta=0.0, gamma=2.0, beta_clip=0, restart_average=1, unweighted_average=1)
    out = np.zeros(3, np.float32)
    for t in (1, 2, 3, 4, 5, 17, 100, 1000):
        lib().oracle_discount(t, C.byref(p), ptr(out))
        x = float(t - 1) ** 1.5
        assert out[0] == np.float32(x / (x + 1.0))
        assert out[1] == np.float32(0.5)
        assert 0.0 <= out[2] <= 1.0


def test_handset_normalizer_counts_compatible_pairs():
    """HandSet::new (hands.rs:35-125): the normalizer counts the weighted
    pairs of non-overlapping hands."""
    board = abi.parse_cards("Ks7s2dTh4c")
    r0 = workloads.uniform_range(1000)
    r1 = workloads.uniform_range(1001)
    from oracle_api import HandSetOracle
    hs = HandSetOracle(r0, r1, board)
    assert hs.len(0) == hs.len(1) == 1081
    c0, c1 = hs.cards(0), hs.cards(1)
    w0 = np.array([r0[abi.combo_index(int(a), int(b))] for a, b in c0], np.float64)
    w1 = np.array([r1[abi.combo_index(int(a), int(b))] for a, b in c1], np.float64)
    overlap = (c0[:, None, 0] == c1[None, :, 0]) | (c0[:, None, 0] == c1[None, :, 1]) | \
              (c0[:, None, 1] == c1[None, :, 0]) | (c0[:, None, 1] == c1[None, :, 1])
    expected = float((w0[:, None] * w1[None, :] * ~overlap).sum())
    assert abs(hs.num_combinations() - expected) <= 1e-9 * expected


def test_workload_tree_sizes():
    """The benchmark spots build (sizes from the oracle's estimate)."""
    for cfg, street in ((workloads.river_spot(), abi.RIVER), (workloads.turn_spot(), abi.TURN)):
        st = estimate(cfg)
        assert st.player_nodes > 0 and st.storage_cells > 0
