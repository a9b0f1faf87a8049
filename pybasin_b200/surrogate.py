"""Learned surrogate: an MLP from (initial condition, parameters) to attractor classes.

The network (inputs -> 4 hidden layers of 256 with GELU, tanh form -> class logits) is
trained on labels produced by the integrator itself, with this library's BF16
tensor-core GEMMs (FP32 accumulation), softmax cross-entropy, GELU backward and
AdamW kernels; FP32 master weights, BF16 copies for the GEMMs.  At inference,
rows whose max softmax probability is below a threshold, plus a seeded random
audit slice, are routed back to the FP32 integrator, so every reported label
is either an integrator label or a confident surrogate label checked by the
audit.  There is no counterpart in the reference.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from pybasin_b200 import _lib as L


def _p(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _bind(lib: ctypes.CDLL) -> None:
    if getattr(lib, "_pb_mlp_bound", False):
        return
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    lib.pb_mlp_gemm.argtypes = [vp, i64, i64, vp, i64, i64, vp, f32, i32, i32, i32, i32, vp, vp, vp, i64, vp]
    lib.pb_mlp_gelu_backward.argtypes = [vp, vp, i64, vp, vp, vp]
    lib.pb_mlp_softmax_xent.argtypes = [vp, vp, i32, i32, f32, vp, vp, vp, vp, vp]
    lib.pb_mlp_bias_grad.argtypes = [vp, i32, i32, f32, vp, vp]
    lib.pb_mlp_adamw.argtypes = [vp, vp, vp, vp, vp, i64, f32, f32, f32, f32, f32, i32, vp]
    lib.pb_mlp_cast_bf16.argtypes = [vp, vp, i64, vp]
    lib.pb_surrogate_inputs.argtypes = [vp, i32, vp, i32, vp, vp, vp, i32, i64, i32, vp, vp]
    lib.pb_surrogate_inputs_rows.argtypes = [vp, i32, vp, i64, i32, vp, vp, vp, vp, i32, i64, i32, vp, vp]
    lib.pb_surrogate_gate.argtypes = [vp, i64, i32, f32, vp, vp, vp, vp, vp, vp]
    lib.pb_gather_rows.argtypes = [vp, i32, vp, vp, i64, vp, vp]
    lib.pb_merge_labels.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    lib.pb_gate_summary.argtypes = [vp, i64, i32, vp, vp, i64, vp, vp, f32, vp, vp, vp, vp, vp]
    lib.pb_mlp_infer_tc.argtypes = [vp, i64, i32, i32, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                    ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32), vp, i32, vp, vp]
    for name in (
        "pb_mlp_infer_tc",
        "pb_mlp_gemm",
        "pb_mlp_gelu_backward",
        "pb_mlp_softmax_xent",
        "pb_mlp_bias_grad",
        "pb_mlp_adamw",
        "pb_mlp_cast_bf16",
        "pb_surrogate_inputs",
        "pb_surrogate_inputs_rows",
        "pb_surrogate_gate",
        "pb_gather_rows",
        "pb_merge_labels",
        "pb_gate_summary",
    ):
        getattr(lib, name).restype = ctypes.c_int
    lib._pb_mlp_bound = True


def pack_tc_weights(W: torch.Tensor) -> torch.Tensor:
    """BF16 weights (N, K) -> the tensor-core operand layout of ``pb_mlp_infer_tc``:
    N and K padded to multiples of 16, 8x8 core matrices, core (n/8, k/8) at
    ((n/8) * (K/8) + k/8) * 64 elements."""
    N, K = W.shape
    Np, Kp = -(-N // 16) * 16, -(-K // 16) * 16
    Wp = torch.zeros((Np, Kp), dtype=torch.bfloat16, device=W.device)
    Wp[:N, :K] = W.to(torch.bfloat16)
    return Wp.view(Np // 8, 8, Kp // 8, 8).permute(0, 2, 1, 3).contiguous().view(-1)


def infer_tc(x: torch.Tensor, packed: list[torch.Tensor], biases: list[torch.Tensor], shapes: list[tuple[int, int, int]],
             n_classes: int, error: torch.Tensor | None = None) -> torch.Tensor:
    """Logits (n, n_classes) of BF16 inputs x through ``pb_mlp_infer_tc``.

    ``shapes[l] = (n_pad, k_pad, n_real)`` of layer l."""
    lib = L.load()
    _bind(lib)
    n, d_in = x.shape
    nl = len(packed)
    out = torch.empty((n, n_classes), dtype=torch.float32, device=x.device)
    vp = ctypes.c_void_p
    w_arr = (vp * nl)(*[p.data_ptr() for p in packed])
    b_arr = (vp * nl)(*[b.data_ptr() for b in biases])
    n_pad = (ctypes.c_int32 * nl)(*[s[0] for s in shapes])
    k_pad = (ctypes.c_int32 * nl)(*[s[1] for s in shapes])
    n_real = (ctypes.c_int32 * nl)(*[s[2] for s in shapes])
    xc = x.contiguous()
    L.check(lib.pb_mlp_infer_tc(_p(xc), n, d_in, nl, w_arr, b_arr, n_pad, k_pad, n_real, _p(out), n_classes,
                                _p(error), torch.cuda.current_stream(x.device).cuda_stream), "pb_mlp_infer_tc")
    return out


def gemm(
    A: torch.Tensor,
    sam: int,
    sak: int,
    B: torch.Tensor,
    sbk: int,
    sbn: int,
    M: int,
    N: int,
    K: int,
    *,
    bias: torch.Tensor | None = None,
    alpha: float = 1.0,
    gelu: bool = False,
    c_f32: torch.Tensor | None = None,
    c_bf16: torch.Tensor | None = None,
    z_pre: torch.Tensor | None = None,
    ldc: int | None = None,
) -> None:
    """C[m,n] = alpha * sum_k A(m,k) B(k,n) (+ bias) with element strides (BF16 in)."""
    lib = L.load()
    _bind(lib)
    s = torch.cuda.current_stream(A.device).cuda_stream
    rc = lib.pb_mlp_gemm(
        _p(A), sam, sak, _p(B), sbk, sbn, _p(bias), alpha, M, N, K, int(gelu), _p(c_f32), _p(c_bf16), _p(z_pre),
        ldc if ldc is not None else N, s,
    )
    L.check(rc, "pb_mlp_gemm")


@dataclass
class TrainHistory:
    loss: list[float] = field(default_factory=list)
    accuracy: list[float] = field(default_factory=list)


class MLPSurrogate:
    """(IC, params) -> class logits; ``depth`` hidden layers of ``hidden`` units with GELU.

    ``d_raw`` columns (IC and parameters) are z-scored; with ``n_freq`` > 0 the
    network also sees sin and cos of 2 pi f.z for ``n_freq`` fixed random
    frequency vectors f ~ N(0, freq_scale^2) per column (random Fourier features:
    a plain MLP on two inputs underfits basins that interleave finely), so
    ``d_in = d_raw + 2 n_freq``."""

    def __init__(self, d_raw: int, n_classes: int, hidden: int = 256, depth: int = 4, seed: int = 0,
                 device: torch.device | str = "cuda", n_freq: int = 0, freq_scale: float = 0.3,
                 pad_inputs: bool = False):
        self.dev = torch.device(device)
        self.d_raw, self.n_freq = d_raw, n_freq
        d_in = d_raw + 2 * n_freq
        # with pad_inputs, input rows are zero padded to a multiple of 8 columns (16-byte
        # rows for the tensor-core training kernels); the padded columns' weights are 0
        self.d_used = d_in
        if pad_inputs:
            d_in = -(-d_in // 8) * 8
        self.d_in, self.n_classes, self.hidden, self.depth = d_in, n_classes, hidden, depth
        rng = np.random.default_rng(seed)
        self.freq = torch.tensor(rng.normal(0.0, freq_scale, (max(n_freq, 1), d_raw)), dtype=torch.float32,
                                 device=self.dev)
        dims = [d_in] + [hidden] * depth + [n_classes]
        self.W: list[torch.Tensor] = []
        self.b: list[torch.Tensor] = []
        for fan_in, fan_out in zip(dims[:-1], dims[1:]):
            # torch.nn.Linear's default uniform bound (over the unpadded inputs)
            bound = 1.0 / np.sqrt(self.d_used if not self.W else fan_in)
            w = rng.uniform(-bound, bound, (fan_out, fan_in))
            if len(self.W) == 0:
                w[:, self.d_used:] = 0.0  # weights of the zero padding columns
            self.W.append(torch.tensor(w, dtype=torch.float32, device=self.dev))
            self.b.append(torch.tensor(rng.uniform(-bound, bound, fan_out), dtype=torch.float32, device=self.dev))
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self.shift = torch.zeros(d_raw, dtype=torch.float32, device=self.dev)
        self.scale = torch.ones(d_raw, dtype=torch.float32, device=self.dev)
        self._adam: list[tuple[torch.Tensor, torch.Tensor]] | None = None
        self._step = 0

    @property
    def n_layers(self) -> int:
        return len(self.W)

    # -- inputs --------------------------------------------------------------
    def fit_normalisation(self, x: torch.Tensor) -> None:
        """Per-column shift/scale from training inputs (zero-variance columns -> scale 0)."""
        mean = x.mean(dim=0)
        std = x.std(dim=0)
        self.shift = mean.to(torch.float32).contiguous()
        self.scale = torch.where(std > 0, 1.0 / std, torch.zeros_like(std)).to(torch.float32).contiguous()

    def inputs(self, ic: torch.Tensor, params: torch.Tensor | None,
               param_index: torch.Tensor | None = None) -> torch.Tensor:
        """BF16 network inputs from FP32 ICs (n, S) and FP64 parameters: one row for
        every IC, or with ``param_index`` (n,) int32 a table ``params`` (P, n_params)
        whose row param_index[r] goes with IC r (a parameter study)."""
        lib = L.load()
        _bind(lib)
        n, S = ic.shape
        prm = None if params is None else params.to(self.dev, torch.float64)
        if prm is not None and prm.dim() == 1:
            prm = prm[None]
        rows, npar = (0, 0) if prm is None else (int(prm.shape[0]), int(prm.shape[1]))
        if S + npar != self.d_raw:
            raise ValueError(f"surrogate expects {self.d_raw} inputs, got {S}+{npar}")
        if param_index is None and rows > 1:
            raise ValueError("a parameter table needs the row of every IC (param_index)")
        out = torch.empty((n, self.d_in), dtype=torch.bfloat16, device=self.dev)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        icc = ic.to(self.dev, torch.float32).contiguous()
        prm = None if prm is None else prm.contiguous()
        pidx = None if param_index is None else param_index.to(self.dev, torch.int32).contiguous()
        freq = self.freq if self.n_freq > 0 else None
        L.check(lib.pb_surrogate_inputs_rows(_p(icc), S, _p(prm), rows, npar, _p(pidx), _p(self.shift),
                                             _p(self.scale), _p(freq), self.n_freq, n, self.d_in, _p(out), s),
                "pb_surrogate_inputs_rows")
        return out

    # -- forward / backward ----------------------------------------------------
    def forward(self, x: torch.Tensor, keep: bool = False):
        """Logits (n, C) FP32 for BF16 inputs x (n, d_in); with keep, the layer inputs
        (BF16) and pre-activations (FP32) for backward."""
        n = x.shape[0]
        acts = [x]
        pres: list[torch.Tensor] = []
        h = x
        for li in range(self.n_layers):
            W = self.Wb[li]
            N, K = W.shape
            last = li == self.n_layers - 1
            if last:
                out = torch.empty((n, N), dtype=torch.float32, device=self.dev)
                gemm(h, K, 1, W, 1, K, n, N, K, bias=self.b[li], c_f32=out)
                return (out, acts, pres) if keep else out
            hb = torch.empty((n, N), dtype=torch.bfloat16, device=self.dev)
            z = torch.empty((n, N), dtype=torch.float32, device=self.dev) if keep else None
            gemm(h, K, 1, W, 1, K, n, N, K, bias=self.b[li], gelu=True, c_bf16=hb, z_pre=z)
            if keep:
                pres.append(z)  # type: ignore[arg-type]
                acts.append(hb)
            h = hb
        raise AssertionError("unreachable")

    def backward(self, dlogits_bf16: torch.Tensor, dlogits_f32: torch.Tensor, acts: list[torch.Tensor],
                 pres: list[torch.Tensor]) -> tuple[list[torch.Tensor], list[torch.Tensor]]:
        """Gradients of the weights and biases given dL/dlogits."""
        lib = L.load()
        _bind(lib)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        n = dlogits_f32.shape[0]
        gW: list[torch.Tensor] = [torch.empty(0)] * self.n_layers
        gb: list[torch.Tensor] = [torch.empty(0)] * self.n_layers
        dz_b, dz_f = dlogits_bf16, dlogits_f32
        for li in reversed(range(self.n_layers)):
            W = self.Wb[li]
            N, K = W.shape
            X = acts[li]
            g = torch.empty((N, K), dtype=torch.float32, device=self.dev)
            gemm(dz_b, 1, N, X, K, 1, N, K, n, c_f32=g)  # dW = dZ^T X
            gW[li] = g
            db = torch.empty((N,), dtype=torch.float32, device=self.dev)
            L.check(lib.pb_mlp_bias_grad(_p(dz_f), n, N, 1.0, _p(db), s), "pb_mlp_bias_grad")
            gb[li] = db
            if li == 0:
                break
            dX = torch.empty((n, K), dtype=torch.float32, device=self.dev)
            gemm(dz_b, N, 1, W, K, 1, n, K, N, c_f32=dX)  # dX = dZ W
            z = pres[li - 1]
            nb = torch.empty((n, K), dtype=torch.bfloat16, device=self.dev)
            nf = torch.empty((n, K), dtype=torch.float32, device=self.dev)
            L.check(lib.pb_mlp_gelu_backward(_p(dX), _p(z), n * K, _p(nb), _p(nf), s), "pb_mlp_gelu_backward")
            dz_b, dz_f = nb, nf
        return gW, gb

    def loss_grad(self, logits: torch.Tensor, labels: torch.Tensor, scale: float):
        lib = L.load()
        _bind(lib)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        n, C = logits.shape
        db = torch.empty((n, C), dtype=torch.bfloat16, device=self.dev)
        df = torch.empty((n, C), dtype=torch.float32, device=self.dev)
        loss = torch.zeros((1,), dtype=torch.float32, device=self.dev)
        corr = torch.zeros((1,), dtype=torch.int32, device=self.dev)
        L.check(lib.pb_mlp_softmax_xent(_p(logits), _p(labels), n, C, scale, _p(db), _p(df), _p(loss), _p(corr), s),
                "pb_mlp_softmax_xent")
        return db, df, loss, corr

    def adamw_step(self, gW: list[torch.Tensor], gb: list[torch.Tensor], lr: float, weight_decay: float) -> None:
        lib = L.load()
        _bind(lib)
        s = torch.cuda.current_stream(self.dev).cuda_stream
        if self._adam is None:
            self._adam = [(torch.zeros_like(p), torch.zeros_like(p)) for p in self.W + self.b]
        self._step += 1
        params = self.W + self.b
        grads = gW + gb
        bf = self.Wb + [None] * len(self.b)
        for p, g, (m1, m2), pb in zip(params, grads, self._adam, bf):
            wd = weight_decay if p.dim() == 2 else 0.0
            L.check(lib.pb_mlp_adamw(_p(p), _p(g), _p(m1), _p(m2), _p(pb), p.numel(), lr, 0.9, 0.999, 1e-8, wd,
                                     self._step, s), "pb_mlp_adamw")

    # -- training ----------------------------------------------------------------
    def train(self, x_in: torch.Tensor, labels: torch.Tensor, epochs: int = 30, batch: int = 1024,
              lr: float = 2e-3, weight_decay: float = 1e-4, seed: int = 0) -> TrainHistory:
        """Minibatch AdamW on BF16 inputs ``x_in`` (n, d_in) and int32 ``labels``."""
        hist = TrainHistory()
        n = x_in.shape[0]
        g = torch.Generator(device="cpu").manual_seed(seed)
        labels = labels.to(self.dev, torch.int32).contiguous()
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.dev)
            tot_loss = torch.zeros((), dtype=torch.float32, device=self.dev)
            tot_corr = torch.zeros((), dtype=torch.int64, device=self.dev)
            lr_ep = lr * 0.5 * (1 + np.cos(np.pi * ep / max(epochs, 1)))  # cosine schedule
            for b0 in range(0, n, batch):
                idx = perm[b0 : b0 + batch]
                xb = x_in.index_select(0, idx).contiguous()
                yb = labels.index_select(0, idx).contiguous()
                m = xb.shape[0]
                logits, acts, pres = self.forward(xb, keep=True)
                dzb, dzf, loss, corr = self.loss_grad(logits, yb, 1.0 / m)
                gW, gb = self.backward(dzb, dzf, acts, pres)
                self.adamw_step(gW, gb, lr_ep, weight_decay)
                tot_loss += loss[0]
                tot_corr += corr[0]
            hist.loss.append(float(tot_loss) / n)
            hist.accuracy.append(float(tot_corr) / n)
        return hist

    # -- inference -----------------------------------------------------------------
    def tc_supported(self) -> bool:
        """The network fits the fused tensor-core kernel (all widths <= 256, <= 8 layers)."""
        dims = [self.d_in] + [w.shape[0] for w in self.Wb]
        return self.n_layers <= 8 and max(dims) <= 256 and os.environ.get("PB_MLP_TC", "1") != "0"

    def packed_tc(self) -> tuple[list[torch.Tensor], list[tuple[int, int, int]]]:
        """Weights in the tensor-core operand layout (rebuilt after every optimiser step)."""
        if getattr(self, "_tc_step", None) != self._step:
            packed, shapes = [], []
            for li, W in enumerate(self.Wb):
                N, K = W.shape
                packed.append(pack_tc_weights(W))
                shapes.append((-(-N // 16) * 16, -(-K // 16) * 16, N))
            self._tc_cache = (packed, shapes)
            self._tc_step = self._step
        return self._tc_cache

    def fused_image(self):
        """(BF16 weight slab images, dims) of the fused training step's layout, with
        the bias as a column of the augmented weights (repacked after every change of
        the weights), or None where the network is outside that step's limits."""
        from pybasin_b200 import train as T

        dims = [self.d_in] + [int(w.shape[0]) for w in self.W]
        if not T.fused_supported(dims) or os.environ.get("PB_MLP_TC", "1") == "0":
            return None
        if getattr(self, "_fused_step", None) != self._step:
            lib = T._lib()
            nl = len(dims) - 1
            dims_c = (ctypes.c_int32 * len(dims))(*dims)
            geo = (ctypes.c_int64 * (3 + 4 * nl))()
            L.check(lib.pb_train_fused_geometry(nl, dims_c, 1, geo, len(geo)), "pb_train_fused_geometry")
            aug = torch.zeros((int(geo[2]),), dtype=torch.float32, device=self.dev)
            for li in range(nl):
                kaug, npad, off = int(geo[3 + 4 * li]), int(geo[4 + 4 * li]), int(geo[5 + 4 * li])
                A = aug[off : off + npad * kaug].view(npad, kaug)
                A[: dims[li + 1], : dims[li]].copy_(self.W[li])
                A[: dims[li + 1], dims[li]].copy_(self.b[li])
            img = torch.empty((int(geo[0]),), dtype=torch.uint8, device=self.dev)
            L.check(lib.pb_train_fused_pack(nl, dims_c, _p(aug), _p(img), torch.cuda.current_stream(self.dev).cuda_stream),
                    "pb_train_fused_pack")
            self._fused_cache = (img, dims_c)
            self._fused_step = self._step
        return self._fused_cache

    def logits(self, x_in: torch.Tensor, chunk: int = 1 << 20) -> torch.Tensor:
        """Inference logits: the two-tile tensor-core kernel on the fused step's
        weight images where the network fits it, else the one-tile tensor-core
        kernel, else the layer-by-layer GEMM path of training."""
        n = x_in.shape[0]
        fused = self.fused_image()
        if fused is not None and n > 0:
            from pybasin_b200 import train as T

            lib = T._lib()
            img, dims_c = fused
            x = x_in.contiguous()
            out = torch.empty((n, self.n_classes), dtype=torch.float32, device=self.dev)
            err = torch.zeros((1,), dtype=torch.int32, device=self.dev)
            L.check(lib.pb_mlp_infer_fused(self.n_layers, dims_c, _p(x), n, _p(img), _p(out), _p(err),
                                           torch.cuda.current_stream(self.dev).cuda_stream), "pb_mlp_infer_fused")
            self._fused_error = err
            return out
        if self.tc_supported():
            packed, shapes = self.packed_tc()
            return infer_tc(x_in, packed, self.b, shapes, self.n_classes)
        out = torch.empty((n, self.n_classes), dtype=torch.float32, device=self.dev)
        for c0 in range(0, n, chunk):
            out[c0 : c0 + chunk] = self.forward(x_in[c0 : c0 + chunk])
        return out

    def state_dict(self) -> dict[str, np.ndarray]:
        d = {f"W{i}": w.cpu().numpy() for i, w in enumerate(self.W)}
        d.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        d["shift"] = self.shift.cpu().numpy()
        d["scale"] = self.scale.cpu().numpy()
        d["freq"] = self.freq.cpu().numpy()
        return d

    def load_state_dict(self, d: dict[str, np.ndarray]) -> None:
        self.W = [torch.tensor(d[f"W{i}"], device=self.dev) for i in range(self.n_layers)]
        self.b = [torch.tensor(d[f"b{i}"], device=self.dev) for i in range(self.n_layers)]
        self.Wb = [w.to(torch.bfloat16) for w in self.W]
        self._tc_step = None  # repack the tensor-core weights
        self.shift = torch.tensor(d["shift"], device=self.dev)
        self.scale = torch.tensor(d["scale"], device=self.dev)
        if "freq" in d:
            self.freq = torch.tensor(d["freq"], device=self.dev)

    def fold_temperature(self, T: float) -> None:
        """Divide the logits by T (folded into the last layer's weights and bias)."""
        # in place: a captured training graph keeps pointing at these tensors
        self.W[-1].div_(T)
        self.b[-1].div_(T)
        self.Wb[-1].copy_(self.W[-1])
        self._adam = None  # the optimiser state no longer matches the weights
        self._step += 1  # repack the tensor-core weights
