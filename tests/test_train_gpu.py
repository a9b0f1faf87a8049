"""Surrogate training on the tensor cores (pb_train_*) against the FP64 oracle.

Tolerances: BF16 operands carry 8 mantissa bits, so each GEMM is compared with
the FP64 product of the *same* BF16-rounded operands at 1e-4 of the output's
scale (FP32 accumulation only); end-to-end gradients (which also round dZ and
the activations to BF16) at 3e-2 of the largest gradient entry, as for the
mma.sync training kernels.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _bf16(a: np.ndarray) -> np.ndarray:
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()


def _dev_bf16(a: np.ndarray) -> torch.Tensor:
    return torch.tensor(a, dtype=torch.float32, device=DEV).to(torch.bfloat16).contiguous()


@pytest.mark.parametrize("M,N,K", [(1, 16, 16), (130, 6, 136), (256, 256, 256), (4096, 64, 200), (300, 136, 48)])
def test_forward_modes_match_fp64(M, N, K):
    from pybasin_b200.train import TRAIN_FWD_GELU, TRAIN_FWD_LINEAR, gemm_tc

    rng = np.random.default_rng(M + 7 * N + K)
    a, w = _bf16(rng.normal(size=(M, K))), _bf16(rng.normal(size=(N, K)))
    bias = rng.normal(size=N).astype(np.float32)
    A, W, b = _dev_bf16(a), _dev_bf16(w), torch.tensor(bias, device=DEV)
    out = torch.full((M, N), float("nan"), dtype=torch.bfloat16, device=DEV)
    zpre = torch.full((M, N), float("nan"), dtype=torch.float32, device=DEV)
    lin = torch.full((M, N), float("nan"), dtype=torch.float32, device=DEV)
    err = torch.zeros((1,), dtype=torch.int32, device=DEV)
    gemm_tc(A, K, 1, W, K, 1, M, N, K, TRAIN_FWD_GELU, bias=b, out_bf16=out, z_pre=zpre, error=err)
    gemm_tc(A, K, 1, W, K, 1, M, N, K, TRAIN_FWD_LINEAR, bias=b, out_f32=lin, error=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    z = a @ w.T + bias
    scale = np.abs(z).max()
    np.testing.assert_allclose(zpre.cpu().numpy(), z, rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(lin.cpu().numpy(), z, rtol=0, atol=1e-4 * scale)
    g = MO.gelu(z)
    np.testing.assert_allclose(out.float().cpu().numpy(), g, rtol=1e-2, atol=1e-4 * scale)


@pytest.mark.parametrize("M,N,K", [(200, 136, 256), (4096, 256, 256), (64, 256, 6)])
def test_input_gradient_mode_matches_fp64(M, N, K):
    """dZ_below = (dZ W) * GELU'(Z_below) with W read transposed (contiguous along N),
    and the per-warp column sums of dZ_below."""
    from pybasin_b200.train import TRAIN_DX, gemm_tc

    rng = np.random.default_rng(M + N + 3 * K)
    dz, w = _bf16(rng.normal(size=(M, K))), _bf16(rng.normal(size=(K, N)))  # W is (K x N): dZ (M x K) @ W
    z_below = rng.normal(size=(M, N)).astype(np.float32)
    out = torch.full((M, N), float("nan"), dtype=torch.bfloat16, device=DEV)
    parts = torch.full((-(-M // 128) * 4, N), float("nan"), dtype=torch.float32, device=DEV)
    # B(n, k) = W[k, n]: sbn = 1, sbk = N
    gemm_tc(_dev_bf16(dz), K, 1, _dev_bf16(w), 1, N, M, N, K, TRAIN_DX, z_in=torch.tensor(z_below, device=DEV),
            ldz=N, out_bf16=out, col_part=parts, ldc=N, ldp=N)
    torch.cuda.synchronize()
    want = (dz @ w) * MO.gelu_grad(z_below.astype(np.float64))
    scale = np.abs(want).max()
    np.testing.assert_allclose(out.float().cpu().numpy(), want, rtol=1e-2, atol=2e-4 * scale)
    np.testing.assert_allclose(parts.sum(0).cpu().numpy(), want.sum(0), rtol=0, atol=1e-4 * np.abs(want).sum(0).max())


@pytest.mark.parametrize("M,N,K", [(256, 136, 4096), (6, 256, 1000), (256, 256, 300)])
def test_weight_gradient_split_k_matches_fp64(M, N, K):
    """dW = dZ^T X over the batch (K rows), both operands read along their rows, in
    chunks of 256 rows whose partials sum to the product."""
    from pybasin_b200.train import TRAIN_DW, gemm_tc

    rng = np.random.default_rng(M * N + K)
    dz, x = _bf16(rng.normal(size=(K, M))), _bf16(rng.normal(size=(K, N)))
    splits = -(-K // 256)
    part = torch.full((splits, M, N), float("nan"), dtype=torch.float32, device=DEV)
    gemm_tc(_dev_bf16(dz), 1, M, _dev_bf16(x), 1, N, M, N, K, TRAIN_DW, out_f32=part, ldc=N)
    # the same with the bias partials from the column of ones
    part2 = torch.full((splits, M, N), float("nan"), dtype=torch.float32, device=DEV)
    bpart = torch.full((splits, M), float("nan"), dtype=torch.float32, device=DEV)
    gemm_tc(_dev_bf16(dz), 1, M, _dev_bf16(x), 1, N, M, N, K, TRAIN_DW, out_f32=part2, ldc=N, col_part=bpart, ldp=M)
    torch.cuda.synchronize()
    want = dz.T @ x
    np.testing.assert_allclose(part.sum(0).cpu().numpy(), want, rtol=0, atol=1e-4 * np.abs(want).max())
    assert torch.equal(part, part2)
    np.testing.assert_allclose(bpart.sum(0).cpu().numpy(), dz.sum(0), rtol=0, atol=1e-4 * np.abs(dz).sum(0).max())


@pytest.mark.parametrize("fused", [True, False])
def test_trainer_gradients_match_oracle(fused):
    from pybasin_b200.surrogate import MLPSurrogate
    from pybasin_b200.train import GraphTrainer

    net = MLPSurrogate(3, 6, hidden=64, depth=3, seed=1, device=DEV, n_freq=7, pad_inputs=True)
    assert net.d_in == 24 and net.d_used == 17
    rng = np.random.default_rng(2)
    n = 700
    x = np.zeros((n, net.d_in))
    x[:, : net.d_used] = _bf16(rng.normal(size=(n, net.d_used)))
    y = rng.integers(0, 6, n)
    tr = GraphTrainer(net, n_rows=n, epochs=1, batch=n, fused=fused)
    gW, gb = tr.gradients(_dev_bf16(x), torch.tensor(y, dtype=torch.int32))
    torch.cuda.synchronize()
    Ws = [w.to(torch.bfloat16).double().cpu().numpy() for w in net.W]
    bs = [b.double().cpu().numpy() for b in net.b]
    z, acts, pres = MO.forward(x, Ws, bs)
    _, d = MO.loss_and_grad(z, y)
    oW, ob = MO.backward(d, acts, pres, Ws)  # d is already the batch mean
    for li in range(len(Ws)):
        np.testing.assert_allclose(gW[li].cpu().numpy(), oW[li], rtol=0, atol=3e-2 * np.abs(oW[li]).max())
        np.testing.assert_allclose(gb[li].cpu().numpy(), ob[li], rtol=0, atol=3e-2 * np.abs(ob[li]).max())
    # the padding columns' weights get no gradient
    assert float(gW[0][:, net.d_used :].abs().max()) == 0.0


@pytest.mark.parametrize("fused", [True, False])
def test_graph_replay_equals_eager_run_and_learns(fused):
    """A captured run replays to bit-identical weights of an eager run (deterministic
    partial sums), twice in a row from the reset weights, and it learns."""
    from pybasin_b200.surrogate import MLPSurrogate
    from pybasin_b200.train import GraphTrainer

    g = torch.Generator().manual_seed(0)
    pts = torch.rand(6000, 2, generator=g) * 2 - 1
    y = ((pts[:, 0] > 0).int() + 2 * (pts[:, 0] ** 2 + pts[:, 1] ** 2 < 0.3).int()).to(torch.int32)
    net = MLPSurrogate(2, 4, hidden=128, depth=3, seed=0, device=DEV, n_freq=16, pad_inputs=True)
    net.fit_normalisation(pts.to(DEV))
    xi = net.inputs(pts.to(DEV), None)
    tr = GraphTrainer(net, n_rows=6000, epochs=12, batch=1024, lr=4e-3, fused=fused)
    tr.train(xi, y.to(DEV), use_graph=False)
    torch.cuda.synchronize()
    eager = [w.clone() for w in net.W]
    st = tr.stats()
    assert st["error"] == 0 and st["accuracy"] > 0.85
    for _ in range(2):
        tr.train(use_graph=True)
        torch.cuda.synchronize()
        for a, b in zip(eager, net.W):
            assert torch.equal(a, b)
    acc = float((net.logits(xi).argmax(1).cpu() == y).float().mean())
    assert acc > 0.97


@pytest.mark.parametrize("fused", [True, False])
def test_data_parallel_trainer_under_a_one_rank_group(fused):
    """The data-parallel path (chunk partials summed, the one all-reduce, AdamW on a
    single partial) under a one-rank NCCL group gives the single-process step: one
    full-batch step from the same weights, equal to summation-order rounding."""
    import os
    import socket

    import torch.distributed as dist

    from pybasin_b200.surrogate import MLPSurrogate
    from pybasin_b200.train import GraphTrainer

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=DEV)
    try:
        g = torch.Generator().manual_seed(3)
        pts = torch.rand(3000, 2, generator=g) * 2 - 1
        y = (pts[:, 0] > 0).to(torch.int32)
        out = []
        for dp in (False, True):
            net = MLPSurrogate(2, 4, hidden=64, depth=2, seed=5, device=DEV, n_freq=8, pad_inputs=True)
            net.fit_normalisation(pts.to(DEV))
            xi = net.inputs(pts.to(DEV), None)
            tr = GraphTrainer(net, n_rows=3000, epochs=1, batch=3000, lr=4e-3, data_parallel=dp, fused=fused)
            tr.train(xi, y.to(DEV), use_graph=False)
            torch.cuda.synchronize()
            out.append([w.clone() for w in net.W])
        for a, b in zip(*out):
            assert (a - b).abs().max().item() <= 1e-6
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [300, 4096])
def test_fused_step_gradients_of_the_surrogate_shape(n):
    """The surrogate's own shape (136 inputs, 4 x 256 GELU, 6 classes) through the
    fused step: several row tiles (the last one ragged for n = 300), every layer's
    chunks and pieces, the weight gradients summed over a cluster.  Gradients of
    the mean loss against the FP64 oracle on the same BF16 inputs and weights."""
    from pybasin_b200.surrogate import MLPSurrogate
    from pybasin_b200.train import GraphTrainer

    net = MLPSurrogate(2, 6, hidden=256, depth=4, seed=3, device=DEV, n_freq=64, pad_inputs=True)
    assert net.d_in == 136
    rng = np.random.default_rng(n)
    x = np.zeros((n, net.d_in))
    x[:, : net.d_used] = _bf16(rng.normal(size=(n, net.d_used)))
    y = rng.integers(0, 6, n)
    tr = GraphTrainer(net, n_rows=n, epochs=1, batch=n, fused=True)
    gW, gb = tr.gradients(_dev_bf16(x), torch.tensor(y, dtype=torch.int32))
    torch.cuda.synchronize()
    assert int(tr.error.item()) == 0
    Ws = [w.to(torch.bfloat16).double().cpu().numpy() for w in net.W]
    bs = [b.double().cpu().numpy() for b in net.b]
    z, acts, pres = MO.forward(x, Ws, bs)
    _, d = MO.loss_and_grad(z, y)
    oW, ob = MO.backward(d, acts, pres, Ws)
    for li in range(len(Ws)):
        np.testing.assert_allclose(gW[li].cpu().numpy(), oW[li], rtol=0, atol=3e-2 * np.abs(oW[li]).max())
        np.testing.assert_allclose(gb[li].cpu().numpy(), ob[li], rtol=0, atol=3e-2 * np.abs(ob[li]).max())


def test_fused_and_per_gemm_training_agree():
    """The same run (shuffles, learning rates, steps) on the two paths: accuracy of the
    trained networks within a point, weights within BF16 training noise."""
    from pybasin_b200.surrogate import MLPSurrogate
    from pybasin_b200.train import GraphTrainer

    g = torch.Generator().manual_seed(5)
    pts = torch.rand(8000, 2, generator=g) * 2 - 1
    y = ((pts[:, 0] > 0).int() + 2 * (pts[:, 0] ** 2 + pts[:, 1] ** 2 < 0.3).int()).to(torch.int32)
    accs = []
    for fused in (True, False):
        net = MLPSurrogate(2, 4, hidden=256, depth=4, seed=0, device=DEV, n_freq=32, pad_inputs=True)
        net.fit_normalisation(pts.to(DEV))
        xi = net.inputs(pts.to(DEV), None)
        tr = GraphTrainer(net, n_rows=8000, epochs=10, batch=2048, lr=4e-3, fused=fused)
        tr.train(xi, y.to(DEV))
        torch.cuda.synchronize()
        assert tr.stats()["error"] == 0
        accs.append(float((net.logits(xi).argmax(1).cpu() == y).float().mean()))
    assert accs[0] > 0.97 and abs(accs[0] - accs[1]) < 0.01
