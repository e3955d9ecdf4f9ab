"""The committed workload fixtures (tests/golden/make_workload_fixtures.py).

On the CPU: the seeded workload generators still produce the committed
range weights bit for bit, and the oracle still produces the committed
results. On the GPU: exact precision reproduces the oracle's committed
results bit for bit (exploitability, root values, and the digest of the
regrets and strategy sums); fast precision is within the reference's 1e-4
relative exploitability tolerance."""
import json
import os

import numpy as np
import pytest

from golden.make_workload_fixtures import ORACLE_RUNS, RANGE_WORKLOADS, ranges_of, spot, storage_digest
from poker_trainer_b200 import abi

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIX = json.load(open(os.path.join(HERE, "workload_oracle.json")))
# The flop entry holds 20 GB of storage in each solver: its bit-for-bit GPU
# check lives in test_gpu_flop.py, and the CPU suite does not re-run it.
SMALL_RUNS = [n for n in ORACLE_RUNS if n != "flop"]


def committed_ranges():
    blob = np.fromfile(os.path.join(HERE, "workload_ranges.bin"), dtype="<f4")
    return {n: blob[i * 2652:(i + 1) * 2652].reshape(2, 1326) for i, n in enumerate(FIX["range_workloads"])}


@pytest.mark.parametrize("name", RANGE_WORKLOADS)
def test_workload_ranges_match_fixture(name):
    got = ranges_of(spot(name))
    want = committed_ranges()[name]
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", SMALL_RUNS)
def test_oracle_matches_fixture(name):
    from oracle_api import OracleSolver

    f = FIX["oracle"][name]
    o = OracleSolver(spot(name))
    o.iterate(f["iterations"])
    assert float(o.exploitability()).hex() == f["exploitability"]
    assert [float(v).hex() for v in o.root_values()] == f["root_values"]
    assert storage_digest(*o.storage()) == f["storage_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", SMALL_RUNS)
def test_gpu_exact_matches_fixture(gpu, name):
    from poker_trainer_b200.solver import Solver

    f = FIX["oracle"][name]
    cfg = spot(name)
    cfg.precision = abi.PRECISION_EXACT
    g = Solver.new(cfg)
    g.iterate(f["iterations"])
    assert float(g.exploitability()).hex() == f["exploitability"]
    assert [float(v).hex() for v in g.root_values()] == f["root_values"]
    assert storage_digest(*g.download_storage()) == f["storage_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(ORACLE_RUNS))
def test_gpu_fast_close_to_fixture(gpu, name):
    from poker_trainer_b200.solver import Solver

    f = FIX["oracle"][name]
    g = Solver.new(spot(name))
    g.iterate(f["iterations"])
    want = float.fromhex(f["exploitability"])
    assert abs(g.exploitability() - want) <= 1e-4 * abs(want)
