"""The C-ABI boundary without a GPU: libdcfr.so loads, exports every
function include/dcfr.h declares, its structs have the header's layout in
the Python mirror, its host-side tree builder agrees with the oracle's, and
creating a solver where no CUDA device exists fails loudly (no CPU
fallback). CPU only: nothing here launches a kernel."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import spots
from oracle_api import OracleError, estimate as oracle_estimate
from poker_trainer_b200 import abi, workloads
from poker_trainer_b200 import solver as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dcfr.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(dcfr_[a-z_0-9]+)\s*\(", text, flags=re.M)))


def test_header_declares_the_exported_api():
    names = declared_functions()
    assert "dcfr_create" in names and "dcfr_solve" in names and "dcfr_query" in names
    assert sorted(S.EXPORTS) == [n for n in names if n in S.EXPORTS]


def test_library_exports_every_declared_symbol():
    L = S.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


STRUCTS = {
    "dcfr_bet_size": abi.BetSize, "dcfr_street_sizes": abi.StreetSizes, "dcfr_menu": abi.Menu,
    "dcfr_betting_state": abi.BettingState, "dcfr_params": abi.Params, "dcfr_config": abi.Config,
    "dcfr_tree_stats": abi.TreeStats, "dcfr_solve_options": abi.SolveOptions, "dcfr_progress": abi.Progress,
    "dcfr_step": abi.Step, "dcfr_action": abi.ActionT, "dcfr_node_info": abi.NodeInfoHeader,
    "dcfr_kernel_profile": abi.KernelProfile, "dcfr_batch_tuning": abi.BatchTuning,
    "dcfr_setup_profile": abi.SetupProfile,
}


def test_struct_layouts_match_the_header(tmp_path):
    """Compiles a probe against include/dcfr.h with gcc and compares every
    struct's size and field offsets with the ctypes mirror."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dcfr.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            # Python names that are keywords carry a trailing underscore.
            lines.append(f'printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0].rstrip("_") or f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            s, f, v = ln.split()
            got[(s, f)] = int(v)
    for cname, py in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])


def test_config_init_matches_reference_defaults():
    """SolveConfig::new (lib.rs:110-134), PostflopMenu::default
    (menu.rs:119-133), DcfrParams::default (cfr.rs:72-80)."""
    cfg = abi.Config()
    assert S.lib().dcfr_config_init(C.byref(cfg)) == abi.OK
    assert bytes(cfg.menu) == bytes(abi.default_menu())
    assert cfg.big_blind == 100 and cfg.isomorphism == 1 and cfg.storage == abi.STORAGE_AUTO
    assert cfg.max_memory_bytes == 8 << 30
    assert (cfg.dcfr.alpha, cfg.dcfr.beta, cfg.dcfr.gamma) == (1.5, 0.0, 3.0)
    assert cfg.dcfr.restart_average == 1 and cfg.dcfr.unweighted_average == 1 and cfg.dcfr.beta_clip == 0


def estimate(cfg):
    st = abi.TreeStats()
    rc = S.lib().dcfr_estimate(C.byref(cfg), C.byref(st))
    return rc, st


CONFIGS = {
    "river_workload": workloads.river_spot,
    "turn_workload": workloads.turn_spot,
    "flop_workload": workloads.flop_spot,
    "river": spots.river_config,
    "iso_turn": spots.iso_turn_config,
    "allin_turn": spots.allin_turn_config,
    "mid_street_raked": lambda: spots.mid_street_config(True),
    "sampled_flop": spots.sampled_flop_config,
    "sampled_turn": spots.sampled_turn_config,
    "sampled_allin_turn": spots.sampled_allin_turn_config,
    "sampled_iso_flop": spots.sampled_iso_flop_config,
}


@pytest.mark.parametrize("name", list(CONFIGS))
def test_estimate_matches_oracle(name):
    """Tree construction (tree.rs count_tree / Builder) is host code in
    libdcfr; its counts equal the oracle's."""
    cfg = CONFIGS[name]()
    rc, st = estimate(cfg)
    assert rc == abi.OK, S.lib().dcfr_last_error()
    o = oracle_estimate(cfg)
    for f in ("player_nodes", "chance_nodes", "terminal_nodes", "storage_cells", "compressed", "memory_bytes"):
        assert getattr(st, f) == getattr(o, f), f


@pytest.mark.parametrize("seed", range(6))
def test_estimate_matches_oracle_random_rivers(seed):
    cfg = spots.random_river_config(seed)
    rc, st = estimate(cfg)
    try:
        o = oracle_estimate(cfg)
    except RuntimeError:
        assert rc != abi.OK
        return
    assert rc == abi.OK
    assert (st.player_nodes, st.terminal_nodes, st.storage_cells) == (o.player_nodes, o.terminal_nodes,
                                                                       o.storage_cells)


def test_errors_mirror_solver_error():
    cfg = workloads.river_spot()
    cfg.board[1] = cfg.board[0]
    rc, _ = estimate(cfg)
    assert rc == abi.ERR_INVALID_BOARD
    assert S.lib().dcfr_last_error()
    cfg = workloads.river_spot(max_memory_bytes=1 << 10)
    rc, _ = estimate(cfg)
    assert rc in (abi.OK, abi.ERR_TOO_LARGE)
    with pytest.raises(OracleError):
        from oracle_api import OracleSolver
        OracleSolver(abi.make_config("AsAhKd", [np.zeros(1326, np.float32)] * 2, pot=600, stack=9700))


def test_create_without_a_device_fails_loudly():
    """No CPU fallback: with no CUDA device, dcfr_create returns an error
    status and a message instead of solving on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    rc = S.lib().dcfr_create(C.byref(workloads.river_spot()), C.byref(h))
    assert rc != abi.OK
    assert not h.value
    assert S.lib().dcfr_last_error()
