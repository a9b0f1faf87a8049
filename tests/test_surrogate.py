"""Surrogate MLP: the FP64 NumPy oracle (CPU) and the BF16 tensor-core kernels against it (GPU).

Tolerances: BF16 operands carry 8 mantissa bits, so GEMMs are compared to the
FP64 product of the *same* BF16-rounded operands at 1e-4 relative (FP32
accumulation only), and end-to-end gradients (which also round dZ and the
activations to BF16) at 3e-2 relative to the largest gradient entry.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as MO


def _bf16(a: np.ndarray) -> np.ndarray:
    return torch.tensor(a, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()


def _tiny_net(rng, d_in=3, hidden=32, depth=2, C=4):
    dims = [d_in] + [hidden] * depth + [C]
    Ws = [rng.uniform(-1, 1, (o, i)) / np.sqrt(i) for i, o in zip(dims[:-1], dims[1:])]
    bs = [rng.uniform(-0.1, 0.1, o) for o in dims[1:]]
    return Ws, bs


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    Ws, bs = _tiny_net(rng)
    x = rng.normal(size=(16, 3))
    y = rng.integers(0, 4, 16)

    def loss_of():
        z, _, _ = MO.forward(x, Ws, bs)
        return MO.loss_and_grad(z, y)[0] / len(y)

    z, acts, pres = MO.forward(x, Ws, bs)
    _, d = MO.loss_and_grad(z, y)
    gW, gb = MO.backward(d, acts, pres, Ws)
    eps = 1e-6
    for li in range(len(Ws)):
        for idx in [(0, 0), (1, 2), (Ws[li].shape[0] - 1, Ws[li].shape[1] - 1)]:
            Ws[li][idx] += eps
            lp = loss_of()
            Ws[li][idx] -= 2 * eps
            lm = loss_of()
            Ws[li][idx] += eps
            assert abs((lp - lm) / (2 * eps) - gW[li][idx]) < 1e-6
        bs[li][0] += eps
        lp = loss_of()
        bs[li][0] -= 2 * eps
        lm = loss_of()
        bs[li][0] += eps
        assert abs((lp - lm) / (2 * eps) - gb[li][0]) < 1e-6


# ---------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K", [(1, 5, 3), (64, 64, 32), (130, 257, 70), (1024, 256, 256)])
def test_gemm_matches_fp64_product_of_bf16_operands(M, N, K):
    from pybasin_b200.surrogate import gemm

    rng = np.random.default_rng(M + N + K)
    a = _bf16(rng.normal(size=(M, K)))
    w = _bf16(rng.normal(size=(N, K)))
    bias = rng.normal(size=N).astype(np.float32)
    dev = torch.device("cuda:0")
    A = torch.tensor(a, device=dev).to(torch.bfloat16)
    W = torch.tensor(w, device=dev).to(torch.bfloat16)
    out = torch.empty((M, N), dtype=torch.float32, device=dev)
    zpre = torch.empty((M, N), dtype=torch.float32, device=dev)
    gemm(A, K, 1, W, 1, K, M, N, K, bias=torch.tensor(bias, device=dev), gelu=True, c_f32=out, z_pre=zpre)
    # transposed operand access: C^T = W A^T through strides
    outT = torch.empty((N, M), dtype=torch.float32, device=dev)
    gemm(W, K, 1, A, 1, K, N, M, K, c_f32=outT)
    torch.cuda.synchronize()
    z = a @ w.T + bias
    scale = np.abs(z).max() + 1e-30
    np.testing.assert_allclose(zpre.cpu().numpy(), z, rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(out.cpu().numpy(), MO.gelu(z), rtol=0, atol=1e-4 * scale)
    np.testing.assert_allclose(outT.cpu().numpy(), (a @ w.T).T, rtol=0, atol=1e-4 * scale)


@pytest.mark.gpu
def test_backward_matches_oracle_gradients():
    from pybasin_b200.surrogate import MLPSurrogate

    dev = torch.device("cuda:0")
    net = MLPSurrogate(3, 4, hidden=64, depth=3, seed=1, device=dev)
    rng = np.random.default_rng(2)
    xb = _bf16(rng.normal(size=(256, 3)))
    y = rng.integers(0, 4, 256)
    x_t = torch.tensor(xb, device=dev).to(torch.bfloat16)
    logits, acts, pres = net.forward(x_t, keep=True)
    dzb, dzf, loss, _ = net.loss_grad(logits, torch.tensor(y, dtype=torch.int32, device=dev), 1.0 / 256)
    gW, gb = net.backward(dzb, dzf, acts, pres)
    torch.cuda.synchronize()
    Ws = [w.to(torch.bfloat16).double().cpu().numpy() for w in net.W]
    bs = [b.double().cpu().numpy() for b in net.b]
    z, oacts, opres = MO.forward(xb, Ws, bs)
    oloss, d = MO.loss_and_grad(z, y)
    oW, ob = MO.backward(d, oacts, opres, Ws)
    np.testing.assert_allclose(float(loss.item()), oloss, rtol=2e-2)
    for li in range(len(Ws)):
        sW = np.abs(oW[li]).max()
        np.testing.assert_allclose(gW[li].cpu().numpy(), oW[li], rtol=0, atol=3e-2 * sW)
        sb = np.abs(ob[li]).max()
        np.testing.assert_allclose(gb[li].cpu().numpy(), ob[li], rtol=0, atol=3e-2 * sb)


@pytest.mark.gpu
def test_training_learns_a_separable_problem():
    from pybasin_b200.surrogate import MLPSurrogate

    dev = torch.device("cuda:0")
    g = torch.Generator().manual_seed(0)
    x = torch.rand(8192, 2, generator=g) * 2 - 1
    y = ((x[:, 0] > 0).int() + 2 * (x[:, 0] ** 2 + x[:, 1] ** 2 < 0.3).int()).to(torch.int32)
    net = MLPSurrogate(2, 4, hidden=128, depth=3, seed=0, device=dev)
    net.fit_normalisation(x.to(dev))
    xi = net.inputs(x.to(dev), None)
    hist = net.train(xi, y.to(dev), epochs=15, batch=512, lr=3e-3)
    assert hist.loss[-1] < 0.5 * hist.loss[0]
    assert hist.accuracy[-1] > 0.95


@pytest.mark.gpu
def test_gated_pipeline_matches_integrator_labels_on_duffing():
    from pybasin_b200 import B200Dopri5Solver, DuffingODE, FusedFeatureExtractor
    from pybasin_b200.gated import SurrogateGatedPipeline
    from pybasin_b200.pipeline import BasinStabilityPipeline

    dev = torch.device("cuda:0")
    fx = FusedFeatureExtractor(time_steady=900.0, features=None,
                               features_per_state={0: {"maximum": None, "standard_deviation": None}}, normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=5000, t_eval=(900, 1000), device="cuda:0", precision="mixed",
                              feature_extractor=fx)
    tpl = [[-0.21, 0.02], [1.05, 0.77], [-0.67, 0.02], [-0.46, 0.30], [-0.43, 0.12]]
    pipe = BasinStabilityPipeline(DuffingODE({"delta": 0.08, "k3": 1.0, "A": 0.2}), solver, tpl,
                                  ["y1", "y2", "y3", "y4", "y5"], device=dev)
    gated = SurrogateGatedPipeline(pipe, hidden=128, depth=3, threshold=0.95)

    def ics(n, seed):
        torch.manual_seed(seed)
        return (torch.rand(n, 2) * torch.tensor([2.0, 1.5]) + torch.tensor([-1.0, -0.5])).to(dev)

    hist, _ = gated.train(ics(20000, 1), epochs=20)
    assert hist.accuracy[-1] > 0.6  # Duffing's basins interleave finely; the gate keeps only confident labels
    y0 = ics(20000, 2)
    ref_labels, _ = pipe.run_device(y0)
    ref = ref_labels.clone()
    label, counts, stats = gated.run_device(y0)
    torch.cuda.synchronize()
    assert stats.n_routed < stats.n  # the surrogate labels part of the ICs
    assert stats.n_audited > 0
    # the device summary against host arithmetic: counts of the final labels, and
    # the audit tally (audited rows all routed; confident ones as the gate saw them)
    assert torch.equal(counts.cpu(), torch.bincount(label.long().cpu(), minlength=6))
    audit = gated.audit_mask(20000).bool()
    conf = torch.softmax(gated.net.logits(gated.net.inputs(y0, gated.params)), dim=1).amax(dim=1)
    assert stats.n_audited == int(audit.sum())
    confident_audited = audit & (conf >= 0.95)
    assert abs(stats.audit_confident - int(confident_audited.sum())) <= 2  # FP32 softmax vs the gate's __expf
    assert stats.audit_disagree <= stats.audit_confident
    # host API: class names, or the same labels as indices into the class list
    lab_names, bs, _ = gated.run(y0.cpu())
    lab_idx, bs_idx, _ = gated.run(y0.cpu(), names=False)
    classes = np.array(pipe.classes + ["unbounded"], dtype=object)
    assert lab_idx.dtype == np.int32 and (classes[lab_idx] == lab_names).all()
    assert bs == bs_idx and abs(sum(bs.values()) - 1.0) < 1e-12
    dbs = (torch.bincount(label.long(), minlength=6) - torch.bincount(ref.long(), minlength=6)).abs().max() / 20000
    assert float(dbs) <= 0.005
    assert float((label == ref).double().mean()) >= 0.99


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,d_in", [(300, 256, 256, 256), (129, 80, 48, 40), (7, 16, 16, 5)])
def test_tensor_core_layer_matches_fp64_product_of_bf16_operands(M, N, K, d_in):
    """One layer (no activation) of the tcgen05 inference kernel: x W^T + b."""
    from pybasin_b200.surrogate import infer_tc, pack_tc_weights

    rng = np.random.default_rng(M + N)
    x = _bf16(rng.normal(size=(M, d_in)))
    w = _bf16(rng.normal(size=(N, d_in)))
    bias = rng.normal(size=N).astype(np.float32)
    dev = torch.device("cuda:0")
    X = torch.tensor(x, device=dev).to(torch.bfloat16)
    W = torch.tensor(w, device=dev).to(torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    out = infer_tc(X, [pack_tc_weights(W)], [torch.tensor(bias, device=dev)], [(N, K, N)], N, error=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    z = x @ w.T + bias
    scale = np.abs(z).max()
    np.testing.assert_allclose(out.cpu().numpy(), z, rtol=0, atol=1e-5 * scale)


@pytest.mark.gpu
def test_tensor_core_mlp_matches_layer_by_layer_forward():
    """The fused tcgen05 network (activations kept in shared memory) against the
    training forward (mma.sync GEMMs, activations through HBM): both round the
    activations to BF16 after each layer; the FP32 sums differ in order only."""
    from pybasin_b200.surrogate import MLPSurrogate

    dev = torch.device("cuda:0")
    net = MLPSurrogate(5, 6, hidden=256, depth=4, seed=3, device=dev)
    g = torch.Generator().manual_seed(0)
    x = (torch.randn(1000, 5, generator=g) * 2).to(dev).to(torch.bfloat16)
    ref = net.forward(x)
    packed, shapes = net.packed_tc()
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    from pybasin_b200.surrogate import infer_tc

    tc = infer_tc(x, packed, net.b, shapes, 6, error=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    scale = ref.abs().max().item()
    assert (tc - ref).abs().max().item() <= 2e-2 * scale
    assert (tc.argmax(1) == ref.argmax(1)).float().mean().item() >= 0.995
    assert torch.equal(net.logits(x), tc)  # inference takes the tensor-core path


def test_temperature_calibration_recovers_the_generating_temperature():
    """Labels drawn from softmax(z / 2): the held-out NLL is smallest near T = 2."""
    from pybasin_b200.gated import calibrate_temperature

    rng = np.random.default_rng(5)
    z = rng.normal(0.0, 4.0, (20000, 6))
    p = np.exp(z / 2.0 - (z / 2.0).max(axis=1, keepdims=True))
    p /= p.sum(axis=1, keepdims=True)
    labels = np.array([rng.choice(6, p=row) for row in p])
    assert abs(calibrate_temperature(z, labels) - 2.0) <= 0.1
    # confident logits that are always right: the sharpest temperature of the grid
    assert calibrate_temperature(z, z.argmax(axis=1)) == 0.5


@pytest.mark.gpu
def test_fourier_inputs_match_fp32_reference():
    """pb_surrogate_inputs against the same features in PyTorch FP32, both rounded to
    BF16: z-scored columns, then sin and cos of 2 pi f.z (one BF16 step of 2^-7 at 1
    covers the FP32 differences between the two sine evaluations)."""
    from pybasin_b200.surrogate import MLPSurrogate

    dev = torch.device("cuda:0")
    net = MLPSurrogate(5, 6, hidden=64, depth=2, seed=2, device=dev, n_freq=16, freq_scale=0.7)
    g = torch.Generator().manual_seed(3)
    ic = (torch.rand(3000, 2, generator=g) * 4 - 2).to(dev)
    params = torch.tensor([0.08, 1.0, 0.2], dtype=torch.float64, device=dev)
    raw = torch.cat([ic, params.float().expand(3000, -1)], dim=1)
    net.fit_normalisation(raw)
    x = net.inputs(ic, params).float()
    assert x.shape == (3000, 5 + 32)
    z = (raw - net.shift) * net.scale
    ph = 2 * np.pi * (z.double() @ net.freq.double().T)
    ref = torch.cat([z.double(), torch.sin(ph), torch.cos(ph)], dim=1).float().to(torch.bfloat16).float()
    assert (x - ref).abs().max().item() <= 2.0 ** -7 + 1e-6
    assert (x[:, 2:5] == 0).all()  # constant parameter columns (zero spread) carry nothing


@pytest.mark.gpu
def test_folded_temperature_divides_the_logits():
    from pybasin_b200.surrogate import MLPSurrogate

    dev = torch.device("cuda:0")
    net = MLPSurrogate(5, 6, hidden=128, depth=3, seed=4, device=dev, n_freq=8)
    g = torch.Generator().manual_seed(1)
    ic = torch.randn(2000, 2, generator=g).to(dev)
    params = torch.tensor([0.08, 1.0, 0.2], dtype=torch.float64, device=dev)
    x = net.inputs(ic, params)
    before = net.logits(x)
    net.fold_temperature(2.0)
    after = net.logits(x)
    torch.cuda.synchronize()
    scale = before.abs().max().item()
    assert (after - before / 2.0).abs().max().item() <= 1e-2 * scale


@pytest.mark.gpu
def test_gate_summary_counts_without_routed_rows():
    """pb_gate_summary with no routed rows: class counts of the labels, a zero tally."""
    from pybasin_b200 import _lib as L
    from pybasin_b200.surrogate import _bind, _p

    lib = L.load()
    _bind(lib)
    dev = torch.device("cuda:0")
    g = torch.Generator().manual_seed(4)
    label = torch.randint(0, 6, (50_001,), generator=g, dtype=torch.int32).to(dev)
    counts = torch.full((6,), -1, dtype=torch.int64, device=dev)
    tally = torch.full((3,), -1, dtype=torch.int32, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    assert lib.pb_gate_summary(_p(label), 50_001, 6, None, None, 0, None, None, 0.95, None, None, _p(counts),
                               _p(tally), s) == 0
    torch.cuda.synchronize()
    assert torch.equal(counts.cpu(), torch.bincount(label.long().cpu(), minlength=6))
    assert tally.cpu().tolist() == [0, 0, 0]
    # invalid: more than 64 classes, or a route without its count
    assert lib.pb_gate_summary(_p(label), 10, 65, None, None, 0, None, None, 0.95, None, None, _p(counts),
                               _p(tally), s) != 0
    assert lib.pb_gate_summary(_p(label), 10, 6, _p(label), None, 10, None, None, 0.95, None, None, _p(counts),
                               _p(tally), s) != 0


def test_device_temperature_calibration_equals_the_host_one():
    """The on-device grid search (torch tensors, here on the CPU) picks the same
    temperature as the NumPy one."""
    from pybasin_b200.gated import calibrate_temperature, calibrate_temperature_device

    rng = np.random.default_rng(6)
    z = rng.normal(0.0, 3.0, (5000, 6))
    p = np.exp(z / 1.5 - (z / 1.5).max(axis=1, keepdims=True))
    p /= p.sum(axis=1, keepdims=True)
    labels = np.array([rng.choice(6, p=row) for row in p])
    want = calibrate_temperature(z, labels)
    got = float(calibrate_temperature_device(torch.tensor(z, dtype=torch.float32), torch.tensor(labels)))
    assert abs(got - want) < 1e-6


@pytest.mark.gpu
def test_active_fit_on_the_tensor_cores_gates_duffing_within_delta_bs():
    """fit(): integrator labels of random ICs, a first training run on the tensor
    cores, the least confident ICs of a pool labelled and trained on too, the
    temperature folded in, all queued without a host round trip; then the gated
    pass against the integrator on fresh ICs.  Two fits in a row end in the same
    weights (captured runs replay deterministically)."""
    from pybasin_b200 import B200Dopri5Solver, DuffingODE, FusedFeatureExtractor
    from pybasin_b200.gated import SurrogateGatedPipeline
    from pybasin_b200.pipeline import BasinStabilityPipeline

    dev = torch.device("cuda:0")
    fx = FusedFeatureExtractor(time_steady=900.0, features=None,
                               features_per_state={0: {"maximum": None, "standard_deviation": None}}, normalize=False)
    solver = B200Dopri5Solver(t_span=(0, 1000), t_steps=5000, t_eval=(900, 1000), device="cuda:0", precision="mixed",
                              feature_extractor=fx)
    tpl = [[-0.21, 0.02], [1.05, 0.77], [-0.67, 0.02], [-0.46, 0.30], [-0.43, 0.12]]
    pipe = BasinStabilityPipeline(DuffingODE({"delta": 0.08, "k3": 1.0, "A": 0.2}), solver, tpl,
                                  ["y1", "y2", "y3", "y4", "y5"], device=dev)
    gated = SurrogateGatedPipeline(pipe, hidden=128, depth=3, threshold=0.95, freq_scale=0.6)

    def ics(n, seed):
        torch.manual_seed(seed)
        return (torch.rand(n, 2) * torch.tensor([2.0, 1.5]) + torch.tensor([-1.0, -0.5])).to(dev)

    weights = []
    for _ in range(2):
        info = gated.fit(ics(12000, 1), ics(60000, 3), n_active=6000, epochs=16, batch=2048)
        torch.cuda.synchronize()
        weights.append([w.clone() for w in gated.net.W])
    s = info.summary()
    assert s["train_error_flag"] == 0 and s["n_train"] == 10800 + 6000 and s["n_calibration"] == 1200
    assert 0.5 <= s["temperature"] <= 4.0
    assert all(torch.equal(a, b) for a, b in zip(*weights))
    y0 = ics(20000, 2)
    ref = pipe.run_device(y0)[0].clone()
    label, counts, stats = gated.run_device(y0)
    torch.cuda.synchronize()
    assert stats.n_routed < 0.6 * stats.n
    dbs = (torch.bincount(label.long(), minlength=6) - torch.bincount(ref.long(), minlength=6)).abs().max() / 20000
    assert float(dbs) <= 0.005
    assert float((label == ref).double().mean()) >= 0.99


@pytest.mark.gpu
def test_row_indexed_inputs_and_an_index_out_of_range():
    """pb_surrogate_inputs_rows: each IC takes its own parameter row; a row index
    outside the table gives NaN inputs, and the gate routes such rows."""
    from pybasin_b200.surrogate import MLPSurrogate

    dev = torch.device("cuda:0")
    net = MLPSurrogate(5, 3, hidden=32, depth=2, seed=1, device=dev, n_freq=4, freq_scale=0.5, pad_inputs=True)
    g = torch.Generator().manual_seed(2)
    ic = (torch.rand(500, 2, generator=g) * 2 - 1).to(dev)
    table = torch.tensor([[0.1, t, 1.0] for t in np.linspace(0.1, 1.0, 7)], dtype=torch.float64, device=dev)
    grp = torch.randint(0, 7, (500,), generator=g, dtype=torch.int32).to(dev)
    raw = torch.cat([ic, table.float()[grp.long()]], dim=1)
    net.fit_normalisation(raw)
    x = net.inputs(ic, table, grp).float()
    z = (raw - net.shift) * net.scale
    ph = 2 * np.pi * (z.double() @ net.freq.double().T)
    ref = torch.cat([z.double(), torch.sin(ph), torch.cos(ph)], dim=1).float().to(torch.bfloat16).float()
    assert (x[:, : net.d_used] - ref).abs().max().item() <= 2.0 ** -7 + 1e-6
    bad = grp.clone()
    bad[3] = 7
    xb = net.inputs(ic, table, bad).float()
    assert torch.isnan(xb[3, 2:5]).all() and torch.isfinite(xb[4]).all()


@pytest.mark.gpu
def test_gated_pendulum_torque_sweep_matches_the_integrator_per_point():
    """The surrogate of a parameter study sees each IC's torque: fit on random and
    actively chosen ICs across 16 torque points, then the gated labels of fresh
    ICs against the integrator's, per point.  A 25 % audit (about 1,000 confident
    audited labels per point) lets points whose confident labels disagree with the
    integrator too often fall back to it: at 5,000 ICs per point a basin-stability
    difference of 0.005 is 25 labels, which a smaller audit slice does not resolve."""
    from pybasin_b200 import studies as S
    from pybasin_b200.gated import SurrogateGatedPipeline

    dev = torch.device("cuda:0")
    rows = np.array([[0.1, t, 1.0] for t in np.linspace(0.1, 1.0, 16)])
    pipe = S.pendulum_pipeline("mixed", rows, dev)
    gated = SurrogateGatedPipeline(pipe, hidden=128, depth=3, threshold=0.95, audit_fraction=0.25)

    def sample(n, seed):
        y0 = S.uniform_ics(*S.PENDULUM_BOX, n, seed).to(dev)
        grp = torch.from_numpy(np.random.default_rng(seed).integers(0, 16, n).astype(np.int32)).to(dev)
        return y0, grp

    yr, gr = sample(12000, 1)
    yp, gp = sample(60000, 3)
    info = gated.fit(yr, yp, n_active=6000, epochs=16, batch=2048, group_random=gr, group_pool=gp)
    y0, grp = sample(80000, 2)
    ref_lab, ref_cnt = pipe.run_device(y0, group=grp)
    ref_lab, ref_cnt = ref_lab.clone(), ref_cnt.clone()
    label, counts, stats = gated.run_device(y0, grp)
    torch.cuda.synchronize()
    assert info.summary()["train_error_flag"] == 0
    assert counts.shape == (16, 3) and int(counts.sum()) == 80000
    assert stats.integrated_fraction < 0.9
    n_p = ref_cnt.sum(dim=1).double()
    dbs = ((counts[:, :2] - ref_cnt[:, :2]).abs().max(dim=1).values.double() / n_p).max().item()
    assert dbs <= 0.005
    assert float((label == ref_lab).double().mean()) >= 0.995
    # a fallen-back point carries the integrator's labels exactly
    bad = gated.last_fallback_points.cpu().numpy()
    for q in np.nonzero(bad)[0]:
        sel = (grp == int(q))
        assert torch.equal(label[sel], ref_lab[sel])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 130, 100_003])
def test_two_tile_inference_matches_one_tile_kernel(n):
    """pb_mlp_infer_fused (pairs of row tiles per CTA, the bias as a BF16 column of the
    augmented weights) against pb_mlp_infer_tc (one tile per CTA, FP32 bias added in
    the epilogue) on the surrogate's shape: ragged last tile, an odd tile count, CTAs
    with several pairs; the BF16 rounding of the bias and of the activations bounds
    the difference."""
    from pybasin_b200.surrogate import MLPSurrogate, infer_tc

    dev = torch.device("cuda:0")
    net = MLPSurrogate(2, 6, hidden=256, depth=4, seed=7, device=dev, n_freq=64, pad_inputs=True)
    g = torch.Generator().manual_seed(n)
    ic = (torch.rand(n, 2, generator=g) * 4 - 2).to(dev)
    net.fit_normalisation(ic)
    x = net.inputs(ic, None)
    got = net.logits(x)
    packed, shapes = net.packed_tc()
    ref = infer_tc(x, packed, net.b, shapes, net.n_classes)
    torch.cuda.synchronize()
    assert int(net._fused_error.item()) == 0
    scale = ref.abs().max().item()
    assert (got - ref).abs().max().item() <= 2e-2 * scale
    assert (got.argmax(1) == ref.argmax(1)).float().mean().item() >= 0.99
