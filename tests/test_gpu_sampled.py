"""The sampled chance mode on the GPU (ChanceMode::Sampled,
crates/solver/src/tree.rs:128-136, 302-334; sampling.rs:9-54).

The sample is drawn on the host while the tree is built; the kernels run the
resulting tree like any other. In exact precision the GPU must agree with the
oracle bit for bit, which it can only do if both drew the same cards, built
the same chance factors (tree.rs:542, 1 / (k x compatible / available)) and
kept the all-in runouts exact. The reference's own test of the mode
(tests.rs:151-170) is run as written."""
import numpy as np
import pytest

import spots
from oracle_api import OracleError, OracleSolver
from poker_trainer_b200 import abi
from poker_trainer_b200.solver import BadPath, SolveOptions, Solver, SolverError
from test_gpu_parity import assert_bit_equal, exact

pytestmark = pytest.mark.gpu

SPOTS = {
    "sampled_turn": spots.sampled_turn_config,
    "sampled_turn_3_rivers": lambda: spots.sampled_turn_config(seed=11, river=3),
    "sampled_allin_turn": spots.sampled_allin_turn_config,
    "sampled_iso_flop": spots.sampled_iso_flop_config,
}


@pytest.mark.parametrize("name", list(SPOTS))
def test_iterations_bit_identical(gpu, name):
    o = OracleSolver(SPOTS[name]())
    g = Solver.new(exact(SPOTS[name]()))
    assert g.storage_len() == len(o.storage()[0])
    o.iterate(5)
    g.iterate(5)
    ro, so = o.storage()
    rg, sg = g.download_storage()
    assert_bit_equal(rg, ro, f"{name} regrets")
    assert_bit_equal(sg, so, f"{name} sums")
    assert g.exploitability() == o.exploitability()
    assert np.array_equal(g.root_values(), o.root_values())


def test_sampled_cards_are_the_chance_children(gpu):
    """The river dealt after check-check on the turn: the sampled cards are
    reachable in libdcfr's tree with the oracle's queries, the others are
    not (BadPath), and the chance factor is the sampled one."""
    cfg = spots.sampled_turn_config()
    o = OracleSolver(cfg)
    g = Solver.new(exact(spots.sampled_turn_config()))
    o.iterate(4)
    g.iterate(4)
    ints, _, fl, _ = o.nodes()
    chance = [v for v in range(len(ints)) if ints[v, 0] == 1]
    first = chance[0]
    kids = [int(ints[ints[first, 4] + i, 7]) for i in range(ints[first, 3])]
    assert len(kids) == 6
    # 1 / (6 x 44 / 48) in f32 (tree.rs:542).
    assert fl[first, 1] == np.float32(1.0) / (np.float32(6) * np.float32(44) / np.float32(48))
    used = set(abi.parse_cards("Qh9d4c2s"))
    for c in range(52):
        if c in used:
            continue
        path = ["check", "check", abi.card_str(c)]
        if c in kids:
            qo, qg = o.query(path), g.query(path)
            assert qg.actions == qo["actions"]
            assert_bit_equal(qg.strategy.ravel(), qo["strategy"].ravel(), f"{path} strategy")
            assert_bit_equal(qg.ev.ravel(), qo["ev"].ravel(), f"{path} ev")
            assert_bit_equal(g.ranges_after(path).ravel(), o.ranges_after(path).ravel(), f"{path} ranges")
        else:
            with pytest.raises(OracleError):
                o.query(path)
            with pytest.raises(BadPath):
                g.query(path)


def test_reference_sampled_flop_solve(gpu):
    """tests.rs:151-170: estimate has player nodes; 300 iterations to 0.5%
    (checked every 25) end below 1% of the pot; the root's range strategy
    sums to one."""
    cfg = spots.sampled_flop_config()
    est = Solver.estimate(cfg)
    assert est.player_nodes > 0
    s = Solver.new(cfg)
    p = s.solve(SolveOptions(max_iterations=300, target_exploitability_pct=0.5, check_every=25))
    assert p.exploitability_pct < 1.0, p
    total = float(np.sum(s.query().range_strategy()))
    assert abs(total - 1.0) < 1e-4
    e64, _ = s.exploitability_fp64()
    assert abs(e64 - s.exploitability()) <= 1e-4 * max(abs(e64), 1e-3)


@pytest.mark.parametrize("name", ["sampled_turn", "sampled_iso_flop"])
def test_fast_precision_matches_oracle(gpu, name):
    o = OracleSolver(SPOTS[name]())
    g = Solver.new(SPOTS[name]())
    o.iterate(20)
    g.iterate(20)
    eo, eg = o.exploitability(), g.exploitability()
    assert abs(eg - eo) <= 1e-4 * max(abs(eo), 1e-3), (eg, eo)


def test_seed_changes_the_tree(gpu):
    """Two seeds deal different rivers, so the solves differ; the same seed
    repeats bit for bit."""
    a = Solver.new(exact(spots.sampled_turn_config(seed=3)))
    b = Solver.new(exact(spots.sampled_turn_config(seed=3)))
    c = Solver.new(exact(spots.sampled_turn_config(seed=4)))
    for s in (a, b, c):
        s.iterate(6)
    ra, rb, rc = a.download_storage()[0], b.download_storage()[0], c.download_storage()[0]
    assert np.array_equal(ra.view(np.uint32), rb.view(np.uint32))
    assert not np.array_equal(ra, rc)


def test_invalid_sample_sizes_rejected(gpu):
    cfg = spots.sampled_turn_config()
    cfg.chance_river = 0
    with pytest.raises(SolverError):
        Solver.new(cfg)
    cfg = spots.turn_config()
    cfg.chance = 7
    with pytest.raises(SolverError):
        Solver.new(cfg)
