"""Depth-limited flop solves (dcfr_create_depth_limited): the flop tree cut
at the turn deal, its leaves valued by the leaf-value network.

On a flop with no chips behind, the tree is check, check, leaf, so the root
values of an average-strategy traversal are the leaf values themselves; they
must equal the leaf formula evaluated here from the network's own outputs
on inputs built the same way (both ranges in combo order with the dealt
card's hands removed and scaled to a maximum of 1, board and card one-hot,
pot and stack / 10000):
  v[h] = norm * factor * pot * sum_c [c not in h] (EV_c(h) - s_c) * m_c(h),
with m_c(h) the opponent's weight compatible with h and c, factor the
chance node's 1/45, and s_c the zero-sum shift (S_p + S_o) / (2 M) of the
card's network values."""
import numpy as np
import pytest

from oracle_api import HandSetOracle
from poker_trainer_b200 import abi, leafdata, workloads
from poker_trainer_b200.mlp import LeafNet
from poker_trainer_b200.solver import Solver

pytestmark = pytest.mark.gpu


def test_leaf_values_follow_the_network(gpu):
    import torch
    r0, r1 = workloads.dirichlet_range(2000), workloads.dirichlet_range(2001)
    board = abi.parse_cards("Ks7s2d")
    pot = 600
    cfg = abi.make_config(board, [r0, r1], pot=pot, stack=0, menu_=workloads.flop_menu(), storage=abi.STORAGE_F32,
                          **workloads.DCFR)
    net = LeafNet(leafdata.IN_DIM, 256, 2, leafdata.OUT_DIM, max_batch=128, seed=21)
    g = Solver.new_depth_limited(cfg, net)
    cards = [c for c in range(52) if c not in board]
    hs = HandSetOracle(r0, r1, board)
    norm = 1.0 / hs.num_combinations()
    factor = np.float32(1.0) / np.float32(45.0)
    hands = [g.hands(q) for q in range(2)]
    cc = leafdata.combo_cards()
    X = []
    for c in cards:
        w = []
        for q in range(2):
            combos, wt = hands[q]
            r = np.zeros(1326, np.float32)
            keep = ~(cc[combos] == c).any(axis=1)
            r[combos[keep]] = wt[keep]
            w.append(r)
        X.append(leafdata.encode(w[0], w[1], board + [c], pot, 0))
    Y = net.forward(torch.tensor(np.array(X), device="cuda")).cpu().numpy().astype(np.float64)
    cp_all = [cc[hands[q][0]] for q in range(2)]
    w_all = [hands[q][1].astype(np.float64) for q in range(2)]
    compat = ~((cp_all[0][:, None, 0] == cp_all[1][None, :, 0]) | (cp_all[0][:, None, 0] == cp_all[1][None, :, 1]) |
               (cp_all[0][:, None, 1] == cp_all[1][None, :, 0]) | (cp_all[0][:, None, 1] == cp_all[1][None, :, 1]))
    for p in range(2):
        o = 1 - p
        got = g.traverse(p, abi.MODE_AVERAGE, 1).astype(np.float64)
        Cpo = compat if p == 0 else compat.T
        exp = np.zeros(len(hands[p][0]))
        for k, c in enumerate(cards):
            vp = ~(cp_all[p] == c).any(axis=1)
            vo = ~(cp_all[o] == c).any(axis=1)
            mp = (Cpo[:, vo] @ w_all[o][vo]) * vp       # opponent mass of each traverser hand
            mo = (Cpo.T[:, vp] @ w_all[p][vp]) * vo     # traverser mass of each opponent hand
            evp = Y[k, p * 1326 + hands[p][0]]
            evo = Y[k, o * 1326 + hands[o][0]]
            sp = float((w_all[p] * mp * evp).sum())
            so = float((w_all[o] * mo * evo).sum())
            mm = float((w_all[p] * mp).sum())
            shift = 0.5 * (sp + so) / mm if mm > 0 else 0.0
            exp += (evp - shift) * mp
        exp *= norm * float(factor) * pot
        scale = float(np.max(np.abs(exp)))
        assert float(np.max(np.abs(got - exp))) <= 1e-4 * scale, (p, float(np.max(np.abs(got - exp))), scale)
    g.close()


def test_depth_limited_flop_solve_runs(gpu):
    """The flop workload cut at the turn deal builds and iterates with any
    network (convergence with a trained one is checked in
    test_gpu_leafnet.py), and its flop decision nodes carry their blocks in
    the reference storage layout."""
    cfg = workloads.flop_spot()
    net = LeafNet(leafdata.IN_DIM, 256, 2, leafdata.OUT_DIM, max_batch=2048, seed=3)
    g = Solver.new_depth_limited(cfg, net)
    g.iterate(5)
    assert np.isfinite(g.exploitability())
    assert g.node_storage([])[0] == 0
    st = g.stats()
    assert st.chance_nodes == 0 and st.player_nodes > 0
    full = Solver.estimate(cfg)
    assert st.player_nodes < full.player_nodes
