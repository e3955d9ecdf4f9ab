"""dcfr_showdown_values_noalloc, the entry point for callers that cannot
allocate device memory (their device memory belongs to their own pool
allocator, or they are held to a fixed device-memory budget). Its scratch
is a static device array shared by every call.

It is checked through the C ABI:
- against the solver's own path: on a river spot with no chips behind, both
  players can only check, so the root value of an average-strategy
  traversal (dcfr_traverse) is exactly the showdown value of the opponent's
  root range. Two calls in a row (one per player, so the second runs on the
  first's leftover scratch) must each match within the fast-precision
  traversal tolerance of 1e-5 of the row's scale;
- against the CPU oracle's batched showdown evaluation (showdown_batch with
  its tie pass, crates/solver/src/eval.rs:214-379) with win, lose and tie
  payoffs all non-zero and unequal, within the same tolerance;
- on invalid input: sizes beyond the limit and bad hands are rejected, and
  a negative reach entry gives NaN values.

This file is collected last so that a failing run with -x has already run
every other test; it also passes alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from oracle_api import HandSetOracle
from poker_trainer_b200 import abi, workloads
from poker_trainer_b200 import solver as S
from poker_trainer_b200.solver import Solver

pytestmark = pytest.mark.gpu

TOL = 1e-5  # of the largest magnitude of the reference row
BOARD = "Ks7s2dTh4c"
POT = 2000


def entry():
    f = S.lib().dcfr_showdown_values_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_double, C.c_double,
                  C.c_double, C.c_void_p, C.c_void_p]
    return f


def cards_of(combos):
    out = np.zeros((len(combos), 2), np.uint8)
    for i, c in enumerate(combos):
        out[i] = abi.combo_cards(int(c))
    return np.ascontiguousarray(out)


def test_noalloc_showdown_matches_traversal(gpu):
    import torch

    r0 = workloads.uniform_range(21, 51)
    r1 = workloads.uniform_range(22, 51)
    cfg = abi.make_config(BOARD, [r0, r1], pot=POT, stack=0, menu_=workloads.river_menu(), storage=abi.STORAGE_F32)
    norm = 1.0 / HandSetOracle(r0, r1, abi.parse_cards(BOARD)).num_combinations()
    # showdown_payoffs (crates/solver/src/cfr.rs:239-246) with no invest and
    # no rake: win half the pot, lose half the pot, ties pay nothing.
    win, lose, tie = (POT / 2) * norm, -(POT / 2) * norm, 0.0
    board = (C.c_uint8 * 5)(*abi.parse_cards(BOARD))
    f = entry()
    g = Solver.new(cfg)
    try:
        for p in (0, 1):
            expected = g.traverse(p, abi.MODE_AVERAGE, 1)
            hero, _ = g.hands(p)
            opp, w = g.hands(p ^ 1)
            hc, oc = cards_of(hero), cards_of(opp)
            reach = torch.tensor(w, dtype=torch.float32, device="cuda")
            out = torch.full((len(hero),), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            rc = f(board, hc.ctypes.data, len(hero), oc.ctypes.data, len(opp), reach.data_ptr(), win, lose, tie,
                   out.data_ptr(), None)
            assert rc == abi.OK, S.lib().dcfr_last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            scale = float(np.max(np.abs(expected)))
            diff = float(np.max(np.abs(got.astype(np.float64) - expected.astype(np.float64))))
            assert diff <= TOL * scale, f"player {p}: max diff {diff:e} vs scale {scale:e}"
    finally:
        g.close()


def test_noalloc_rejects_oversized_and_bad_input(gpu):
    f = entry()
    board = (C.c_uint8 * 5)(*abi.parse_cards(BOARD))
    one = np.array([[0, 1]], np.uint8)
    rc = f(board, one.ctypes.data, abi.NUM_COMBOS + 1, one.ctypes.data, 1, None, 1.0, -1.0, 0.0, None, None)
    assert rc == abi.ERR_INVALID_ARG
    assert b"1326" in S.lib().dcfr_last_error()
    on_board = np.array(abi.parse_cards("Ks2c"), np.uint8)
    rc = f(board, on_board.ctypes.data, 1, one.ctypes.data, 1, None, 1.0, -1.0, 0.0, None, None)
    assert rc == abi.ERR_INVALID_ARG


def test_noalloc_matches_oracle_showdown_with_ties(gpu):
    """Win, lose and tie all non-zero and unequal (invests that differ):
    the oracle's batched evaluator with its tie pass is the reference."""
    import torch

    r0 = workloads.uniform_range(31, 40)
    r1 = workloads.uniform_range(32, 40)
    board_cards = abi.parse_cards(BOARD)
    hs = HandSetOracle(r0, r1, board_cards)
    board = (C.c_uint8 * 5)(*board_cards)
    f = entry()
    rng = np.random.default_rng(5)
    for p, (win, lose, tie) in enumerate(((0.7, -0.45, 0.125), (1.3, -0.2, -0.3))):
        hc = np.ascontiguousarray(hs.cards(p))
        oc = np.ascontiguousarray(hs.cards(p ^ 1))
        reach = (rng.random(len(oc)) * (rng.random(len(oc)) < 0.8)).astype(np.float32)
        outs, _ = hs.showdown_batch(p, [reach], [win], [lose], [tie])
        want = np.asarray(outs[0], np.float64)
        d_reach = torch.tensor(reach, device="cuda")
        out = torch.full((len(hc),), float("nan"), dtype=torch.float32, device="cuda")
        rc = f(board, hc.ctypes.data, len(hc), oc.ctypes.data, len(oc), d_reach.data_ptr(), win, lose, tie,
               out.data_ptr(), None)
        assert rc == abi.OK, S.lib().dcfr_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        scale = float(np.max(np.abs(want)))
        diff = float(np.max(np.abs(got - want)))
        assert diff <= TOL * scale, f"player {p}: max diff {diff:e} vs scale {scale:e}"


def test_noalloc_negative_reach_gives_nan(gpu):
    import torch

    hs = HandSetOracle(workloads.uniform_range(41), workloads.uniform_range(42), abi.parse_cards(BOARD))
    hc = np.ascontiguousarray(hs.cards(0))
    oc = np.ascontiguousarray(hs.cards(1))
    reach = np.ones(len(oc), np.float32)
    reach[3] = -0.5
    board = (C.c_uint8 * 5)(*abi.parse_cards(BOARD))
    d_reach = torch.tensor(reach, device="cuda")
    out = torch.zeros(len(hc), dtype=torch.float32, device="cuda")
    rc = entry()(board, hc.ctypes.data, len(hc), oc.ctypes.data, len(oc), d_reach.data_ptr(), 1.0, -1.0, 0.0,
                 out.data_ptr(), None)
    assert rc == abi.OK
    torch.cuda.synchronize()
    assert np.all(np.isnan(out.cpu().numpy()))
    # The scratch is usable again by the next valid call.
    d_reach = torch.ones(len(oc), dtype=torch.float32, device="cuda")
    rc = entry()(board, hc.ctypes.data, len(hc), oc.ctypes.data, len(oc), d_reach.data_ptr(), 1.0, -1.0, 0.0,
                 out.data_ptr(), None)
    assert rc == abi.OK
    torch.cuda.synchronize()
    assert np.all(np.isfinite(out.cpu().numpy()))
