"""The flop workload (board Ks7s2d, pot 6bb, stacks 97bb, 33%/75%/all-in bets
and a 3x raise on every street, Dirichlet class ranges, f32 storage, suit
isomorphism) against the CPU oracle, by the reference's own GPU-vs-CPU
standards (crates/solver/src/gpu/engine/tests.rs):

- fast precision after the same iteration count: exploitability within 1e-4
  relative, strategies within 5e-5 and EVs within 0.25 chips at the root,
  after a check, and below an isomorphism-canonical and an
  isomorphism-mirrored turn card (fast_short_solves_match_cpu,
  tests.rs:481-490; fast_converged_solves_match_cpu, tests.rs:492-512);
- exact precision bit for bit: two iterations reproduce the oracle's
  committed exploitability, root values and storage digest
  (exact_solves_match_cpu_bit_for_bit, tests.rs:729-754); that storage
  uploaded into a fresh solver downloads with the same digest (the chunked
  transfers in both directions).

The flop tree holds about 2.5 G storage cells (20 GB of regrets and strategy
sums in each solver); the oracle runs its chance children on all host
cores."""
import json
import os

import numpy as np
import pytest

from golden.make_workload_fixtures import storage_digest
from oracle_api import OracleSolver
from poker_trainer_b200 import abi, workloads
from poker_trainer_b200.solver import Solver

pytestmark = pytest.mark.gpu

FIX = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "workload_oracle.json")))

ITERS = 12
STRATEGY_TOL = 5e-5
EV_TOL_CHIPS = 0.25
EXPLOITABILITY_RTOL = 1e-4
# Clubs and hearts are interchangeable on Ks7s2d with these ranges: one of
# each pair of turn cards is solved, the other read through the suit swap.
PATHS = [[], ["check"], ["check", "check", "Ac"], ["check", "check", "Ah"], ["check", "check", "9c"],
         ["check", "check", "9h"]]


def test_flop_exact_matches_fixture(gpu):
    f = FIX["oracle"]["flop"]
    cfg = workloads.flop_spot()
    cfg.precision = abi.PRECISION_EXACT
    g = Solver.new(cfg)
    assert g.isomorphic_pairs() > 0
    g.iterate(f["iterations"])
    assert float(g.exploitability()).hex() == f["exploitability"]
    assert [float(v).hex() for v in g.root_values()] == f["root_values"]
    r, s = g.download_storage()
    g.close()
    assert storage_digest(r, s) == f["storage_sha256"]
    # The same storage up into a fresh solver (all zeros) and down again:
    # both transfers cross in about 40 chunks of at most 64 M values, so a
    # chunk that went astray shows as zeros or misplaced values.
    g = Solver.new(cfg)
    g.upload_storage(r, s)
    r[:] = 0.0
    s[:] = 0.0
    g.download_storage(out=(r, s))
    g.close()
    assert storage_digest(r, s) == f["storage_sha256"]


def test_flop_fast_matches_oracle(gpu):
    cfg = workloads.flop_spot()
    g = Solver.new(cfg)
    g.iterate(ITERS)
    eg = g.exploitability()
    o = OracleSolver(cfg)
    o.iterate(ITERS)
    eo = o.exploitability()
    assert abs(eg - eo) <= EXPLOITABILITY_RTOL * abs(eo), (eg, eo)
    for path in PATHS:
        qo = o.query(path)
        qg = g.query(path)
        assert qg.actions == qo["actions"], path
        assert np.array_equal(qg.combos, qo["combos"]), path
        ds = float(np.max(np.abs(np.asarray(qg.strategy, np.float64) - qo["strategy"].astype(np.float64))))
        de = float(np.max(np.abs(np.asarray(qg.ev, np.float64) - qo["ev"].astype(np.float64))))
        assert ds <= STRATEGY_TOL, f"{path}: strategy differs by {ds:e}"
        assert de <= EV_TOL_CHIPS, f"{path}: EV differs by {de} chips"
