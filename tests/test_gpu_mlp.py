"""The leaf-value network's tensor-core kernels (dcfr_gemm_bf16,
dcfr_mlp_*) against a plain PyTorch fp32 reference of the same ops on the
CPU, computed from the same bf16-rounded operands:

- the GEMM and its four epilogues, at the network's tile shapes;
- the network's loss and every weight and bias gradient, with the bf16
  rounding of activations, pre-activations and output gradients done at the
  same points as the kernels (relative error of each gradient block below
  2e-2);
- the same loss and gradients against the FP64 CPU oracle
  (oracle/mlp_fp64.py, pinned by finite differences), and one Adam step of
  dcfr_mlp_train_step against the oracle's Adam step on the kernels' own
  gradients;
- training: Adam steps reduce the loss on a fixed regression batch.
"""
import numpy as np
import pytest

from poker_trainer_b200.mlp import LeafNet, gemm_bf16, pad128

pytestmark = pytest.mark.gpu


def bf(x):
    import torch
    return x.to(torch.bfloat16).to(torch.float32)


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (256, 384, 192), (384, 256, 2816), (128, 2688, 1024)])
@pytest.mark.parametrize("epi", [0, 1, 2, 3])
def test_gemm_matches_fp32_reference(gpu, m, n, k, epi):
    import torch
    g = torch.Generator().manual_seed(m * 7 + n * 3 + k + epi)
    a = (torch.randn(m, k, generator=g) * 0.5).to(torch.bfloat16)
    b = (torch.randn(n, k, generator=g) * 0.5).to(torch.bfloat16)
    bias = torch.randn(n, generator=g)
    zin = (torch.randn(m, n, generator=g)).to(torch.bfloat16)
    acc = a.float() @ b.float().T
    dev = "cuda"
    c, z = gemm_bf16(a.to(dev), b.to(dev), epi, bias.to(dev) if epi in (1, 2) else None,
                     zin.to(dev) if epi == 3 else None)
    c = c.float().cpu()
    scale = float(acc.abs().max())
    if epi == 0:
        ref = acc
        tol = 1e-5
    elif epi == 1:
        ref = acc + bias
        tol = 1e-5
    elif epi == 2:
        pre = acc + bias
        assert float((z.float().cpu() - bf(pre)).abs().max()) <= 1e-2 * float(pre.abs().max())
        ref = torch.nn.functional.gelu(pre)
        tol = 1e-2
    else:
        x = zin.float()
        gp = 0.5 * (1 + torch.erf(x / np.sqrt(2))) + x * torch.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)
        ref = acc * gp
        tol = 1e-2
    err = float((c - ref).abs().max())
    assert err <= tol * max(float(ref.abs().max()), scale * 1e-3), (err, float(ref.abs().max()))


def reference_gradients(net, flat, x, t, mask):
    """Loss and gradients of the network in fp32 on the CPU with the kernels'
    bf16 rounding points."""
    import torch
    layers = [(torch.tensor(w.copy()), torch.tensor(b.copy())) for w, b in net.split(flat)]
    M = x.shape[0]
    xp = torch.zeros(M, net.kin[0])
    xp[:, :x.shape[1]] = x
    X = [bf(xp)]
    Z = []
    for l in range(net.layers):
        w, b = layers[l]
        pre = X[-1] @ bf(w).T + b
        Z.append(bf(pre))
        X.append(bf(torch.nn.functional.gelu(pre)))
    w, b = layers[-1]
    Y = (X[-1] @ bf(w).T + b)[:, :t.shape[1]]
    cnt = float(mask.sum())
    d = Y - t
    loss = float((mask * d * d).sum() / cnt)
    dY = torch.zeros(M, net.nout[-1])
    dY[:, :t.shape[1]] = 2 * mask * d / cnt
    dY = bf(dY)
    grads = [None] * (net.layers + 1)
    for l in range(net.layers, -1, -1):
        w, _ = layers[l]
        gw = dY.T @ X[l]
        gb = dY.sum(0)
        grads[l] = (gw, gb)
        if l > 0:
            dx = dY @ bf(w)
            z = Z[l - 1]
            gp = 0.5 * (1 + torch.erf(z / np.sqrt(2))) + z * torch.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)
            dY = bf(dx * gp)
    return loss, grads


def test_mlp_gradients_match_fp32_reference(gpu):
    import torch
    net = LeafNet(in_dim=200, hidden=256, layers=3, out_dim=150, max_batch=256, seed=5)
    g = torch.Generator().manual_seed(1)
    x = torch.rand(200, 200, generator=g)
    t = torch.randn(200, 150, generator=g)
    mask = (torch.rand(200, 150, generator=g) < 0.7).float()
    loss, grads = net.gradients(x.cuda(), t.cuda(), mask.cuda())
    flat = net.params()
    rl, rg = reference_gradients(net, flat, x, t, mask)
    assert abs(loss - rl) <= 1e-3 * abs(rl), (loss, rl)
    for l, ((gw, gb), (rw, rb)) in enumerate(zip(net.split(grads), rg)):
        for got, ref, what in ((gw, rw.numpy(), "W"), (gb, rb.numpy(), "b")):
            rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
            assert rel < 2e-2, f"layer {l} {what}: relative error {rel}"


def test_mlp_gradients_match_fp64_oracle(gpu):
    import torch
    from oracle import mlp_fp64
    net = LeafNet(in_dim=130, hidden=256, layers=2, out_dim=200, max_batch=256, seed=7)
    rng = np.random.default_rng(4)
    x = rng.random((160, 130)).astype(np.float32)
    t = rng.normal(size=(160, 200)).astype(np.float32)
    mask = (rng.random((160, 200)) < 0.5).astype(np.float32)
    loss, grads = net.gradients(torch.tensor(x).cuda(), torch.tensor(t).cuda(), torch.tensor(mask).cuda())
    layers = [(w.astype(np.float64), b.astype(np.float64)) for w, b in net.split(net.params())]
    rl, rg = mlp_fp64.loss_and_gradients(layers, x, t, mask, bf16_points=True)
    assert abs(loss - rl) <= 1e-3 * abs(rl), (loss, rl)
    for l, ((gw, gb), (rw, rb)) in enumerate(zip(net.split(grads), rg)):
        for got, ref, what in ((gw, rw, "W"), (gb, rb, "b")):
            rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
            assert rel < 2e-2, f"layer {l} {what}: relative error {rel}"


def test_adam_step_matches_fp64_oracle(gpu):
    import torch
    from oracle import mlp_fp64
    net = LeafNet(in_dim=100, hidden=128, layers=1, out_dim=90, max_batch=128, seed=3)
    rng = np.random.default_rng(8)
    x = torch.tensor(rng.random((128, 100)).astype(np.float32)).cuda()
    t = torch.tensor(rng.normal(size=(128, 90)).astype(np.float32)).cuda()
    p0 = net.params()
    _, g = net.gradients(x, t)
    lr = 1e-3
    net.train_step(x, t, None, lr=lr)
    p1 = net.params()
    ref, _, _ = mlp_fp64.adam_step(p0, g, np.zeros_like(g), np.zeros_like(g), 1, lr)
    real = g != 0  # padded entries have zero gradients and do not move
    assert np.array_equal(p1[~real], p0[~real])
    err = np.abs(p1.astype(np.float64) - ref)[real]
    assert float(err.max()) <= 1e-3 * lr + 1e-6 * float(np.abs(p0).max()), float(err.max())


def test_mlp_training_reduces_loss(gpu):
    import torch
    net = LeafNet(in_dim=300, hidden=256, layers=2, out_dim=128, max_batch=256, seed=9)
    g = torch.Generator().manual_seed(2)
    x = torch.rand(256, 300, generator=g)
    w = torch.randn(300, 128, generator=g) / 17.0
    t = torch.tanh(x @ w)
    xd, td = x.cuda(), t.cuda()
    first = net.train_step(xd, td, None, lr=1e-3)
    for _ in range(300):
        last = net.train_step(xd, td, None, lr=1e-3)
    assert last < 0.1 * first, (first, last)
    y = net.forward(xd).cpu()
    assert float(((y - t) ** 2).mean()) < 0.2 * first


def test_data_parallel_entry_points(gpu):
    """dcfr_mlp_backward + dcfr_mlp_adam_step(lr, 1) is dcfr_mlp_train_step,
    bit for bit; the device gradient buffer (a torch view, as NCCL sees it)
    holds the gradients dcfr_mlp_gradients returns; scaling the buffer by 2
    and stepping with grad_scale 0.5 is the same step again (the
    data-parallel mean over two equal ranks)."""
    import torch
    rng = np.random.default_rng(12)
    x = torch.tensor(rng.random((128, 150)).astype(np.float32)).cuda()
    t = torch.tensor(rng.normal(size=(128, 100)).astype(np.float32)).cuda()
    a = LeafNet(in_dim=150, hidden=128, layers=2, out_dim=100, max_batch=128, seed=4)
    b = LeafNet(in_dim=150, hidden=128, layers=2, out_dim=100, max_batch=128, seed=4)
    c = LeafNet(in_dim=150, hidden=128, layers=2, out_dim=100, max_batch=128, seed=4)
    _, g_host = a.gradients(x, t)
    la = a.train_step(x, t, None, lr=1e-3)
    lb = b.backward(x, t)
    gv = b.grad_tensor()
    assert gv.is_cuda and gv.numel() == b.num_params
    assert np.array_equal(gv.cpu().numpy(), g_host)
    b.adam_step(1e-3, 1.0)
    # The loss scalar is reduced with float atomics (order-dependent in the
    # last bits); the gradients and the weights are not.
    assert abs(la - lb) <= 1e-5 * abs(la)
    assert np.array_equal(a.params(), b.params())
    c.backward(x, t)
    gc = c.grad_tensor()
    gc.mul_(2.0)
    torch.cuda.synchronize()
    c.adam_step(1e-3, 0.5)
    assert np.array_equal(a.params(), c.params())
