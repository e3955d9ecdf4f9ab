"""The oracle's poker primitives against the reference's own known answers
(tests/golden/reference_kats.json, restated from the reference's unit tests):
card and combo indexing (crates/holdem/src/combo.rs:213-249), the 7-card
evaluator (crates/holdem/src/eval.rs:209-288), bet sizes and the postflop
menu (crates/holdem/src/menu.rs:412-466). CPU only."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle_api import lib, ptr
from poker_trainer_b200 import abi, workloads

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kats.json")
KATS = json.load(open(GOLDEN))


def evaluate(cards: str) -> int:
    c = np.array(abi.parse_cards(cards), np.int32)
    return int(lib().oracle_evaluate(ptr(c), len(c)))


def test_combo_indexing_is_bijective():
    hi_lo = np.zeros(2 * 1326, np.uint8)
    lib().oracle_combos(ptr(hi_lo))
    seen = set()
    for a in range(52):
        for b in range(52):
            if a == b:
                continue
            i = lib().oracle_combo_index(a, b)
            assert i == lib().oracle_combo_index(b, a) == abi.combo_index(a, b)
            x, y = int(hi_lo[2 * i]), int(hi_lo[2 * i + 1])
            assert {x, y} == {a, b}
            assert x // 4 >= y // 4
            seen.add(i)
    assert seen == set(range(1326))


def test_classes_cover_every_combo_once():
    cls = np.zeros(1326, np.uint8)
    lib().oracle_combo_class(ptr(cls))
    out = np.zeros(12, np.int32)
    total = 0
    py = workloads.class_combos()
    for g in range(169):
        n = lib().oracle_class_combos(g, ptr(out))
        total += n
        assert sorted(out[:n].tolist()) == sorted(py[g]), g
        assert all(cls[i] == g for i in out[:n])
    assert total == 1326


@pytest.mark.parametrize("name,grid,count", KATS["class_grid"]["cases"])
def test_class_grid_index(name, grid, count):
    w = np.zeros(1326, np.float32)
    assert lib().oracle_parse_range(name.encode(), ptr(w)) == 0
    combos = np.nonzero(w)[0].tolist()
    assert len(combos) == count
    out = np.zeros(12, np.int32)
    n = lib().oracle_class_combos(grid, ptr(out))
    assert sorted(out[:n].tolist()) == combos


@pytest.mark.parametrize("cards,category", KATS["eval_categories"]["cases"])
def test_eval_categories(cards, category):
    assert evaluate(cards) >> 26 == category


@pytest.mark.parametrize("a,op,b", KATS["eval_ordering"]["cases"])
def test_eval_ordering(a, op, b):
    x, y = evaluate(a), evaluate(b)
    assert {"<": x < y, ">": x > y, "==": x == y}[op]


def test_five_card_category_counts():
    out = np.zeros(9, np.uint32)
    lib().oracle_five_card_counts(ptr(out))
    assert out.tolist() == KATS["five_card_category_counts"]["counts"]


def test_seven_cards_match_best_five():
    """crates/holdem/src/eval.rs:267-287 with numpy's generator in place of
    StdRng: a 7-card evaluation equals the best of its 21 five-card subsets."""
    rng = np.random.default_rng(7)
    idx = [(i, j) for i in range(7) for j in range(i + 1, 7)]
    L = lib()
    for _ in range(3000):
        seven = rng.choice(52, 7, replace=False).astype(np.int32)
        best = 0
        for i, j in idx:
            five = np.ascontiguousarray(np.delete(seven, [i, j]))
            best = max(best, L.oracle_evaluate(ptr(five), 5))
        assert L.oracle_evaluate(ptr(seven), 7) == best, seven


@pytest.mark.parametrize("text,kind,value", KATS["bet_sizes"]["cases"])
def test_parse_bet_sizes(text, kind, value):
    k = C.c_int32()
    v = C.c_double()
    assert lib().oracle_parse_bet_size(text.encode(), C.byref(k), C.byref(v)) == 0
    assert k.value == kind
    if kind != abi.SIZE_ALLIN:
        assert v.value == value
    # The host-side mirror used to build configs parses the same way.
    assert abi.parse_size(text)[0] == kind
    if kind != abi.SIZE_ALLIN:
        assert abi.parse_size(text)[1] == value


@pytest.mark.parametrize("text", KATS["bet_sizes"]["invalid"])
def test_parse_bet_size_rejects(text):
    k = C.c_int32()
    v = C.c_double()
    assert lib().oracle_parse_bet_size(text.encode(), C.byref(k), C.byref(v)) != 0


KIND = {"fold": abi.FOLD, "check": abi.CHECK, "call": abi.CALL, "raise": abi.RAISE}


@pytest.mark.parametrize("case", KATS["menu_actions"]["cases"], ids=lambda c: c["name"])
def test_menu_actions(case):
    menu = abi.Menu()
    lib().oracle_default_menu(C.byref(menu))
    cb = case["current_bet"]
    out = (abi.ActionT * 16)()
    n = lib().oracle_menu_actions(C.byref(menu), case["street"], case["pot"], case["to_call"], cb, case["max_to"],
                                  100 if cb == 0 else 2 * cb, case.get("num_raises", 0 if cb == 0 else 1), 100,
                                  out, 16)
    got = [(out[i].kind, out[i].amount if out[i].kind == abi.RAISE else 0) for i in range(n)]
    assert got == [(KIND[k], a) for k, a in case["actions"]]


def test_default_menu_matches_python_mirror():
    a = abi.Menu()
    lib().oracle_default_menu(C.byref(a))
    b = abi.default_menu()
    assert bytes(a) == bytes(b)
