"""Cancellation, progress callbacks and resuming through dcfr_solve, as the
reference's GPU backend tests them (crates/solver/src/gpu/engine/tests.rs):

- cancelled_gpu_solve_returns_and_stays_queryable (tests.rs:299-316): a
  solve whose cancel flag is already set returns finished after no
  iteration, the solver still answers queries, and a progress callback that
  returns false stops the solve at its first check;
- continues_a_cpu_solve (tests.rs:274-285): three CPU (oracle) iterations,
  the storage uploaded with the iteration count, the GPU continuing the
  solve to six; in exact precision the result is bit for bit the oracle's
  six-iteration solve.
"""
import ctypes as C

import numpy as np
import pytest

import spots
from oracle_api import OracleSolver
from poker_trainer_b200 import abi
from poker_trainer_b200.solver import Solver, SolveOptions

pytestmark = pytest.mark.gpu


def opts(iterations):
    return SolveOptions(max_iterations=iterations, target_exploitability_pct=0.0, check_every=iterations)


def exact(cfg):
    cfg.precision = abi.PRECISION_EXACT
    return cfg


@pytest.mark.parametrize("precision", ["exact", "fast"])
def test_cancelled_solve_returns_and_stays_queryable(gpu, precision):
    cfg = spots.river_config()
    cfg.precision = abi.PRECISIONS[precision]
    g = Solver.new(cfg)
    cancel = C.c_int32(1)
    p = g.solve(opts(10), cancel=cancel)
    assert p.finished
    assert g.iterations() == 0
    root = g.query([])
    assert np.all(np.isfinite(root.strategy)) and np.all(np.isfinite(root.ev))
    # Stopping from the progress callback: the first check is at iteration 5.
    seen = []
    p = g.solve(SolveOptions(max_iterations=50, target_exploitability_pct=0.0, check_every=5),
                on_progress=lambda pr: seen.append(pr.iteration) or False)
    assert p.iteration == 5 and g.iterations() == 5
    assert seen == [5]
    # A cleared flag lets the next solve run to its end.
    cancel.value = 0
    p = g.solve(opts(8), cancel=cancel)
    assert p.finished and p.iteration == 8 and g.iterations() == 8
    g.close()


def test_continues_a_cpu_solve(gpu):
    reference = OracleSolver(spots.river_config())
    reference.iterate(6)
    o = OracleSolver(spots.river_config())
    o.iterate(3)
    r, s = o.storage()
    g = Solver.new(exact(spots.river_config()))
    g.upload_storage(r, s)
    g.set_iterations(3)
    p = g.solve(opts(6))
    assert p.iteration == 6 and g.iterations() == 6
    rr, sr = reference.storage()
    rg, sg = g.download_storage()
    for a, b, what in ((rg, rr, "regrets"), (sg, sr, "sums")):
        diff = (a.view(np.uint32) != b.view(np.uint32)) & ~((a == 0) & (b == 0))
        assert not diff.any(), f"{what}: {int(diff.sum())} cells differ"
    assert g.exploitability() == reference.exploitability()
    for path in ([], ["check"]):
        qo = reference.query(path)
        qg = g.query(path)
        assert np.array_equal(np.asarray(qg.strategy, np.float32), qo["strategy"].astype(np.float32)), path
    g.close()


def test_continues_a_cpu_solve_fast(gpu):
    """The same resume in fast precision, within the reference's tolerances
    (5e-5 in strategy, 0.25 chips in EV)."""
    reference = OracleSolver(spots.turn_config())
    reference.iterate(6)
    o = OracleSolver(spots.turn_config())
    o.iterate(3)
    g = Solver.new(spots.turn_config())
    g.upload_storage(*o.storage())
    g.set_iterations(3)
    g.solve(opts(6))
    assert g.iterations() == 6
    for path in ([], ["check"], ["check", "check", "Ks"]):
        qo = reference.query(path)
        qg = g.query(path)
        ds = float(np.max(np.abs(np.asarray(qg.strategy, np.float64) - qo["strategy"].astype(np.float64))))
        de = float(np.max(np.abs(np.asarray(qg.ev, np.float64) - qo["ev"].astype(np.float64))))
        assert ds <= 5e-5 and de <= 0.25, (path, ds, de)
    g.close()
