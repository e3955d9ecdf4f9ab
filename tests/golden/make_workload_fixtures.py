"""Writes the workload fixtures next to this file (run from the repository
root: python tests/golden/make_workload_fixtures.py).

- workload_ranges.bin: the seeded range weights of the river, turn,
  turn-narrow and flop workloads (poker_trainer_b200/workloads.py), float32,
  in that order, [2][1326] each: the inputs every parity test and bench line
  feeds to both the oracle and the GPU.
- workload_oracle.json: the CPU oracle's results on the river, turn and
  flop workloads after a few DCFR iterations (exploitability, root values
  and a checksum of the regrets and strategy sums, each f64 as its exact hex
  form): the outputs the GPU's exact precision must reproduce bit for bit.
  The flop entry holds about 20 GB of storage in the oracle and takes a few
  minutes on 8 host threads.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from poker_trainer_b200 import workloads  # noqa: E402

RANGE_WORKLOADS = ["river", "turn", "turn-narrow", "flop"]
ORACLE_RUNS = {"river": 20, "turn": 3, "flop": 2}


def spot(name):
    return {"river": workloads.river_spot, "turn": workloads.turn_spot, "turn-narrow": workloads.turn_narrow_spot,
            "flop": workloads.flop_spot}[name]()


def ranges_of(cfg) -> np.ndarray:
    return np.array([np.ctypeslib.as_array(cfg.ranges[p]) for p in range(2)], dtype=np.float32)


def storage_digest(regrets: np.ndarray, sums: np.ndarray) -> str:
    """SHA-256 of the f32 regrets then sums, with -0.0 written as +0.0 (the
    same value; the sign of a zero is not part of the solve's result)."""
    h = hashlib.sha256()
    step = 1 << 24  # in pieces: the flop's arrays are 10 GB each
    for a in (regrets, sums):
        for i in range(0, len(a), step):
            c = np.ascontiguousarray(a[i:i + step], np.float32)
            h.update(np.where(c == 0, np.float32(0), c).astype(np.float32).tobytes())
    return h.hexdigest()


def oracle_results() -> dict:
    from oracle_api import OracleSolver

    out = {}
    for name, iters in ORACLE_RUNS.items():
        o = OracleSolver(spot(name))
        o.iterate(iters)
        r, s = o.storage()
        out[name] = {"iterations": iters, "exploitability": float(o.exploitability()).hex(),
                     "root_values": [float(v).hex() for v in o.root_values()],
                     "storage_sha256": storage_digest(r, s)}
    return out


def main():
    blob = np.concatenate([ranges_of(spot(n)).ravel() for n in RANGE_WORKLOADS])
    blob.astype("<f4").tofile(os.path.join(HERE, "workload_ranges.bin"))
    results = oracle_results()
    with open(os.path.join(HERE, "workload_oracle.json"), "w") as f:
        json.dump({"range_workloads": RANGE_WORKLOADS, "oracle": results}, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
