"""The f32 solve's fast-precision terminal kernels against each other.

The panel kernel (terminal_panel.cu: 8 or 4 terminals of one board per
block pass), the warp-per-terminal kernel with static or dynamic
scheduling, the two-warps-per-terminal kernel (terminal_group.cu, the default
where both traversals have at least four terminal tasks per SM) and the
block-scan kernel
(terminal_fast.cu) evaluate the same exact integer prefix sums and
round them with the same f64/f32 operations, so their results must agree
bit for bit: traversal values from random storage in every mode, and the
regrets, strategy sums and exploitability after iterations. The kernel is
chosen per handle by DCFR_TERMINAL_KERNEL when the handle is created.
Agreement with the CPU oracle itself is covered by test_gpu_fast.py and
test_gpu_flop.py, which run the default kernels."""
import numpy as np
import pytest

import spots
from poker_trainer_b200 import abi, workloads
from poker_trainer_b200.solver import Solver

pytestmark = pytest.mark.gpu

KERNELS = ["panel", "panel4", "warp", "warpdyn", "group", "block", "blockdyn"]
SPOTS = {
    "river": workloads.river_spot,
    "turn-narrow": workloads.turn_narrow_spot,
    "iso_turn": spots.iso_turn_config,
    "allin_turn": spots.allin_turn_config,
    "mid_street_raked": lambda: spots.mid_street_config(True),
}


def random_storage(n, seed):
    rng = np.random.default_rng(seed)
    r = (rng.standard_normal(n) * 50).astype(np.float32)
    r[rng.random(n) < 0.3] = 0.0
    s = (rng.random(n) * 10).astype(np.float32)
    s[rng.random(n) < 0.2] = 0.0
    return r, s


def outputs(make, kernel, monkeypatch):
    monkeypatch.setenv("DCFR_TERMINAL_KERNEL", kernel)
    g = Solver.new(make())
    name, per_panel = g.terminal_kernel()
    want = ("panel" if kernel.startswith("panel") else "warp" if kernel.startswith("warp") else "group"
            if kernel == "group" else "block")
    assert name == want, (kernel, name)
    if kernel in ("panel4",):
        assert per_panel == 4
    out = {}
    r, s = random_storage(g.storage_len(), 7)
    for p in (0, 1):
        for mode in (abi.MODE_BEST_RESPONSE, abi.MODE_AVERAGE, abi.MODE_CFR):
            g.upload_storage(r, s)
            out[f"traverse p={p} mode={mode}"] = np.asarray(g.traverse(p, mode, 3), np.float32).copy()
    g.close()
    g = Solver.new(make())
    g.iterate(4)
    rg, sg = g.download_storage()
    out["regrets"], out["sums"] = rg.copy(), sg.copy()
    out["exploitability"] = np.array([g.exploitability()], np.float64)
    g.close()
    return out


def same_bits(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype == np.float32:
        # -0.0 and +0.0 are the same value.
        return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | ((a == 0) & (b == 0))))
    return bool(np.array_equal(a, b))


@pytest.mark.parametrize("name", list(SPOTS))
def test_terminal_kernels_bit_identical(gpu, name, monkeypatch):
    ref = outputs(SPOTS[name], "warp", monkeypatch)
    for kernel in KERNELS:
        if kernel == "warp":
            continue
        got = outputs(SPOTS[name], kernel, monkeypatch)
        for key in ref:
            assert same_bits(got[key], ref[key]), f"{name}: {kernel} differs from warp in {key}"


def test_default_kernel_by_task_count(gpu, monkeypatch):
    """Two warps per terminal where both traversals have at least four
    terminal tasks per SM; a river subgame's few dozen terminals take a whole
    block each (long hand lists)."""
    monkeypatch.delenv("DCFR_TERMINAL_KERNEL", raising=False)
    for make, want in ((workloads.turn_spot, ("group", 0)), (workloads.turn_narrow_spot, ("group", 0)),
                       (workloads.river_spot, ("block", 0))):
        g = Solver.new(make())
        assert g.terminal_kernel() == want
        g.close()
    monkeypatch.setenv("DCFR_TERMINAL_KERNEL", "panel")
    for make, width in ((workloads.turn_spot, 4), (workloads.turn_narrow_spot, 8)):
        g = Solver.new(make())
        assert g.terminal_kernel() == ("panel", width)
        g.close()
