"""Batched river solves (dcfr_batch_*): many independent river spots of
uneven tree size solved by one persistent kernel under a captured CUDA
graph. Each spot's iterations perform the same arithmetic as a single
solve of that spot, so the batch must equal, bit for bit, one
Solver per spot run for the same iterations; it is also checked against the
CPU oracle with the fast-precision tolerances of the reference's own GPU
tests (crates/solver/src/gpu/engine/tests.rs: 1e-4 relative
exploitability)."""
import numpy as np
import pytest

import spots
from oracle_api import OracleSolver, estimate
from poker_trainer_b200 import abi, workloads
from poker_trainer_b200.solver import BatchSolver, Solver, SolverError

pytestmark = pytest.mark.gpu


def random_spots(k):
    out = []
    seed = 0
    while len(out) < k:
        cfg = spots.random_river_config(seed)
        seed += 1
        try:
            OracleSolver(cfg)
        except Exception:
            continue
        out.append(cfg)
    return out


def bits_equal(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return a.shape == b.shape and bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | ((a == 0) & (b == 0))))


def test_batch_equals_single_solves(gpu):
    cfgs = random_spots(10)
    b = BatchSolver.new(cfgs)
    b.iterate(7)
    eb = b.exploitability()
    for i, cfg in enumerate(cfgs):
        g = Solver.new(cfg)
        g.iterate(7)
        rg, sg = g.download_storage()
        rb, sb = b.download_storage(i)
        assert bits_equal(rb, rg), f"spot {i}: regrets differ from the single solve"
        assert bits_equal(sb, sg), f"spot {i}: strategy sums differ from the single solve"
        assert eb[i] == g.exploitability(), f"spot {i}: exploitability"
        g.close()
    b.close()


def test_batch_matches_oracle(gpu):
    cfgs = random_spots(6)
    b = BatchSolver.new(cfgs)
    b.iterate(40)
    eb = b.exploitability()
    for i, cfg in enumerate(cfgs):
        o = OracleSolver(cfg)
        o.iterate(40)
        eo = o.exploitability()
        assert abs(eb[i] - eo) <= 1e-4 * max(abs(eo), 1e-3), (i, eb[i], eo)


def test_batched_workload_spots_converge(gpu):
    """Spots drawn like the batched benchmark (uneven menus and trees of
    15-400 nodes): exploitability falls, and a sample equals single solves."""
    def nodes(cfg):
        st = estimate(cfg)
        return st.player_nodes + st.chance_nodes + st.terminal_nodes
    cfgs = workloads.batched_river_spots(count=48, seed=77, estimate=nodes)
    b = BatchSolver.new(cfgs)
    b.iterate(2)
    e0 = b.exploitability()
    b.iterate(60)
    e1 = b.exploitability()
    assert np.all(np.isfinite(e1))
    assert np.mean(e1 / np.array([c.root.pot for c in cfgs])) < np.mean(e0 / np.array([c.root.pot for c in cfgs]))
    for i in (0, 17, 47):
        g = Solver.new(cfgs[i])
        g.iterate(62)
        rg, sg = g.download_storage()
        rb, sb = b.download_storage(i)
        assert bits_equal(rb, rg) and bits_equal(sb, sg), f"spot {i}"
        g.close()


def test_autotune_keeps_the_solve_state(gpu):
    cfgs = random_spots(12)
    b = BatchSolver.new(cfgs)
    b.iterate(3)
    before = [b.download_storage(i) for i in range(len(cfgs))]
    t = b.autotune(4)
    assert t.candidates > 0 and t.warps >= 1 and t.trial_ms > 0
    assert b.iterations() == 3
    for i in range(len(cfgs)):
        r, s = b.download_storage(i)
        assert bits_equal(r, before[i][0]) and bits_equal(s, before[i][1])
    # Any launch shape gives the same iterates.
    b.iterate(5)
    ref = [b.download_storage(i) for i in range(len(cfgs))]
    c = BatchSolver.new(cfgs)
    alt = c.tuning()
    alt.longest_first = 0
    alt.iterations_per_launch = 3
    c.set_tuning(alt)
    c.iterate(8)
    for i in range(len(cfgs)):
        r, s = c.download_storage(i)
        assert bits_equal(r, ref[i][0]) and bits_equal(s, ref[i][1])


def test_batch_rejects_non_river_spots(gpu):
    with pytest.raises(SolverError) as e:
        BatchSolver.new([spots.turn_config()])
    assert e.value.code == abi.ERR_UNSUPPORTED
