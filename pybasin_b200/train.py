"""Surrogate training on the tensor cores, one CUDA graph per training run.

A :class:`GraphTrainer` owns every buffer of a training run of fixed shape
(rows, batch, epochs) on the device: the training set and its shuffled copy,
per-layer activations, pre-activations and gradients, the gradient partials
and the AdamW moments.  The run itself — per epoch a shuffle
(``pb_train_gather``), per minibatch the forward GEMMs, the softmax
cross-entropy, the input- and weight-gradient GEMMs and one multi-tensor AdamW
step (``pb_train_gemm`` / ``pb_train_xent`` / ``pb_train_adamw``, tcgen05
kernels, no allocation) — is captured once as a CUDA graph.  Each later run
copies new rows and labels into the training set, resets the weights to their
initial values and replays the graph: no host work per step, and the same
shuffles, learning rates and Adam step counts as the captured run.

The training matches :meth:`MLPSurrogate.train` (minibatch AdamW, cosine
learning rate per epoch, weight decay on the weights only, softmax
cross-entropy with the 1/M batch mean); the gradients of the weights are sums
of per-chunk partials added in a fixed order, so a run is deterministic.
There is no counterpart in the reference.
"""

from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.surrogate import MLPSurrogate, _p

TRAIN_FWD_GELU, TRAIN_FWD_LINEAR, TRAIN_DX, TRAIN_DW = 0, 1, 2, 3
KC = 256  # K chunk of one CTA (the weight gradient splits the batch into chunks of this)
ROWS = 128  # rows of a CTA tile


def bind(lib: ctypes.CDLL) -> None:
    if getattr(lib, "_pb_train_bound", False):
        return
    vp, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    lib.pb_train_gemm.argtypes = [vp, i64, i64, vp, i64, i64, i32, i32, i32, i32, i32, i32, vp, vp, i64, vp, vp, vp,
                                  vp, vp, i64, i64, i64, vp, vp]
    lib.pb_train_xent.argtypes = [vp, i64, vp, i32, i32, f32, vp, i64, vp, i64, vp, vp, vp, vp]
    lib.pb_train_xent_parts.argtypes = [i32]
    PV = ctypes.POINTER(vp)
    PI64 = ctypes.POINTER(i64)
    lib.pb_train_adamw.argtypes = [i32, PV, PV, PV, PI64, PV, PV, PV, PI64, PI64, ctypes.POINTER(i32),
                                   ctypes.POINTER(f32), f32, f32, f32, f32, i32, vp]
    lib.pb_train_gather.argtypes = [vp, i32, vp, vp, i64, vp, vp, vp, vp]
    PI32 = ctypes.POINTER(i32)
    lib.pb_train_fused_geometry.argtypes = [i32, PI32, i32, PI64, i32]
    lib.pb_train_fused_pack.argtypes = [i32, PI32, vp, vp, vp]
    lib.pb_train_fused_step.argtypes = [i32, PI32, vp, vp, i32, vp, i32, i32, vp, vp, vp, vp, vp, vp, f32, f32, f32,
                                        f32, f32, i32, vp, vp, vp, vp]
    lib.pb_train_fused_adamw.argtypes = [i32, PI32, vp, vp, vp, vp, vp, f32, f32, f32, f32, f32, i32, vp]
    lib.pb_mlp_infer_fused.argtypes = [i32, PI32, vp, i64, vp, vp, vp, vp]
    for name in ("pb_train_gemm", "pb_train_xent", "pb_train_xent_parts", "pb_train_adamw", "pb_train_gather",
                 "pb_train_fused_geometry", "pb_train_fused_pack", "pb_train_fused_step", "pb_train_fused_adamw",
                 "pb_mlp_infer_fused"):
        getattr(lib, name).restype = ctypes.c_int
    lib._pb_train_bound = True


def _lib() -> ctypes.CDLL:
    lib = L.load()
    bind(lib)
    return lib


def gemm_tc(A: torch.Tensor, sam: int, sak: int, B: torch.Tensor, sbn: int, sbk: int, M: int, N: int, K: int,
            mode: int, *, bias: torch.Tensor | None = None, z_in: torch.Tensor | None = None, ldz: int = 0,
            out_f32: torch.Tensor | None = None, out_bf16: torch.Tensor | None = None,
            out_t: torch.Tensor | None = None, z_pre: torch.Tensor | None = None,
            col_part: torch.Tensor | None = None, ldc: int | None = None, ldt: int = 0, ldp: int = 0, kc: int = KC,
            bn: int | None = None, error: torch.Tensor | None = None, stream: int | None = None) -> None:
    """One ``pb_train_gemm`` launch: C (M x N) = A (M x K) B^T with B given as (N x K)
    through element strides (see the C header for the modes)."""
    lib = _lib()
    if bn is None:
        bn = min(64, -(-N // 16) * 16)
    kc = min(kc, -(-K // 16) * 16)
    s = stream if stream is not None else torch.cuda.current_stream(A.device).cuda_stream
    rc = lib.pb_train_gemm(_p(A), sam, sak, _p(B), sbn, sbk, M, N, K, mode, kc, bn, _p(bias), _p(z_in), ldz,
                           _p(out_f32), _p(out_bf16), _p(out_t), _p(z_pre), _p(col_part),
                           ldc if ldc is not None else N, ldt, ldp, _p(error), s)
    L.check(rc, "pb_train_gemm")


def fused_supported(dims: list[int]) -> bool:
    """Whether the fused step (``pb_train_fused_step``) takes a network of these layer
    widths: at most 8 layers, inputs a multiple of 8 up to 256, hidden widths
    multiples of 16 up to 256, 2 to 32 classes."""
    n = len(dims) - 1
    return (1 <= n <= 8 and dims[0] % 8 == 0 and 8 <= dims[0] <= 256
            and all(d % 16 == 0 and 16 <= d <= 256 for d in dims[1:-1]) and 2 <= dims[-1] <= 32)


def dw_tile(n: int) -> int:
    """Columns per CTA of a weight-gradient GEMM with n weight columns plus the bias's
    column of ones: as many tiles as n alone needs at 64 columns, widened to fit."""
    tiles = -(-n // 64)
    return min(256, -(-(-(-(n + 1) // tiles)) // 16) * 16)


class GraphTrainer:
    """A captured training run of ``net`` on ``n_rows`` rows (BF16 inputs of width
    ``net.d_in``, int32 labels): ``epochs`` epochs of minibatches of ``batch`` rows.

    With ``fused`` (the default where :func:`fused_supported` holds) a minibatch step
    is two launches of ``pb_train_fused_step`` (the layer chain of each 128-row tile
    in one kernel, the weight gradients with AdamW in another), on augmented
    parameters ``[W | b]``; otherwise it is the per-GEMM sequence of ``pb_train_gemm``
    launches."""

    def __init__(self, net: MLPSurrogate, n_rows: int, epochs: int, batch: int = 4096, lr: float = 4e-3,
                 weight_decay: float = 1e-4, seed: int = 0, betas: tuple[float, float] = (0.9, 0.999),
                 eps: float = 1e-8, resume: bool = False, data_parallel: bool = False, group=None,
                 fused: bool | None = None):
        """With ``resume``, a run starts from the net's current weights (fresh AdamW
        moments) instead of the weights it had when the trainer was built.  With
        ``data_parallel`` every rank of the process group trains on its own rows
        (the same row count, batch and epochs on every rank): after each backward
        pass the gradients are summed over the rank's rows and averaged over the
        ranks in one collective, so every rank takes the same AdamW step."""
        if net.d_in % 8:
            raise ValueError("GraphTrainer needs input rows of a multiple of 8 columns (MLPSurrogate(pad_inputs=True))")
        self.net = net
        self.resume = resume
        self.data_parallel = data_parallel
        self.group = group
        self.dev = net.dev
        self.n, self.epochs, self.batch = n_rows, epochs, min(batch, n_rows)
        self.lr, self.wd, self.betas, self.eps = lr, weight_decay, betas, eps
        dev = self.dev
        self.dims = [net.d_in] + [int(w.shape[0]) for w in net.W]
        self.fused = fused_supported(self.dims) if fused is None else fused
        if self.fused and not fused_supported(self.dims):
            raise ValueError(f"layer widths {self.dims} are outside the fused training step's limits")
        self.X = torch.zeros((n_rows, net.d_in), dtype=torch.bfloat16, device=dev)
        self.Y = torch.zeros((n_rows,), dtype=torch.int32, device=dev)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.perm = torch.stack([torch.randperm(n_rows, generator=g) for _ in range(epochs)]).to(
            dev, torch.int32).contiguous()
        self.loss = torch.zeros((1,), dtype=torch.float32, device=dev)
        self.correct = torch.zeros((1,), dtype=torch.int32, device=dev)
        self.error = torch.zeros((1,), dtype=torch.int32, device=dev)
        self.graph: torch.cuda.CUDAGraph | None = None
        self.steps = sum(-(-n_rows // self.batch) for _ in range(epochs))
        self.capture_s = 0.0
        self.launches = 0
        self.timing = False
        if self.fused:
            self._init_fused()
        else:
            self._init_gemm()

    def _init_fused(self) -> None:
        lib = _lib()
        net, dev = self.net, self.dev
        L_ = net.n_layers
        self._dims_c = (ctypes.c_int32 * len(self.dims))(*self.dims)
        geo = (ctypes.c_int64 * (3 + 4 * L_))()
        L.check(lib.pb_train_fused_geometry(L_, self._dims_c, self.batch, geo, len(geo)), "pb_train_fused_geometry")
        img_bytes, scratch_bytes, n_aug = int(geo[0]), int(geo[1]), int(geo[2])
        self.kaug = [int(geo[3 + 4 * l]) for l in range(L_)]
        self.npad = [int(geo[4 + 4 * l]) for l in range(L_)]
        self.aug_off = [int(geo[5 + 4 * l]) for l in range(L_)]
        self.w_aug = torch.zeros((n_aug,), dtype=torch.float32, device=dev)
        self.m1 = torch.zeros_like(self.w_aug)
        self.m2 = torch.zeros_like(self.w_aug)
        self.grad = torch.zeros_like(self.w_aug)
        self.w_img = torch.zeros((img_bytes,), dtype=torch.uint8, device=dev)
        self.scratch = torch.zeros((scratch_bytes,), dtype=torch.uint8, device=dev)
        self._views = [self.w_aug[o : o + n * k].view(n, k) for o, n, k in zip(self.aug_off, self.npad, self.kaug)]
        self._gviews = [self.grad[o : o + n * k].view(n, k) for o, n, k in zip(self.aug_off, self.npad, self.kaug)]
        self._aug_from_net()
        self.init_aug = self.w_aug.clone()

    def _init_gemm(self) -> None:
        net, dev = self.net, self.dev
        L_ = net.n_layers
        B = self.batch
        n_rows = self.n
        self.Xs = torch.zeros_like(self.X)
        self.XsT = torch.zeros((net.d_in, n_rows), dtype=torch.bfloat16, device=dev)  # the shuffled inputs transposed
        self.Ys = torch.zeros_like(self.Y)
        self.act = [None] + [torch.zeros((B, self.dims[l + 1]), dtype=torch.bfloat16, device=dev)
                             for l in range(L_ - 1)]
        self.z = [torch.zeros((B, self.dims[l + 1]), dtype=torch.float32, device=dev) for l in range(L_ - 1)]
        self.logits = torch.zeros((B, self.dims[-1]), dtype=torch.float32, device=dev)
        self.dz = [torch.zeros((B, self.dims[l + 1]), dtype=torch.bfloat16, device=dev) for l in range(L_)]
        # transposed copies (units x batch) that the weight-gradient GEMMs read along the batch
        self.actT = [None] + [torch.zeros((self.dims[l + 1], B), dtype=torch.bfloat16, device=dev)
                              for l in range(L_ - 1)]
        self.dzT = [torch.zeros((self.dims[l + 1], B), dtype=torch.bfloat16, device=dev) for l in range(L_)]
        # the transposed BF16 weights live on the net, shared by its trainers (a resumed
        # run reads the ones the previous run's optimiser wrote)
        if getattr(net, "WbT", None) is None or [tuple(w.shape) for w in net.WbT] != \
                [tuple(w.shape[::-1]) for w in net.Wb]:
            net.WbT = [w.t().contiguous() for w in net.Wb]
        self.WbT = net.WbT
        splits = -(-B // KC)
        self.gw_part = [torch.zeros((splits,) + tuple(w.shape), dtype=torch.float32, device=dev) for w in net.W]
        # bias gradients come out of the weight-gradient GEMMs (a column of ones), one
        # partial per batch chunk like the weights
        self.gb_part = [torch.zeros((splits, self.dims[l + 1]), dtype=torch.float32, device=dev) for l in range(L_)]
        self.params = net.W + net.b
        self.m1 = [torch.zeros_like(p) for p in self.params]
        self.m2 = [torch.zeros_like(p) for p in self.params]
        self.init = [p.clone() for p in self.params]
        self.init_bf16 = [w.clone() for w in net.Wb]
        self.init_bf16_t = [w.clone() for w in self.WbT]

    # -- the fused step's augmented parameters -------------------------------------
    def _aug_from_net(self) -> None:
        """[W | b | 0] of every layer from the net's FP32 weights."""
        self.w_aug.zero_()
        for l, A in enumerate(self._views):
            dout, din = self.dims[l + 1], self.dims[l]
            A[:dout, :din].copy_(self.net.W[l])
            A[:dout, din].copy_(self.net.b[l])

    def _net_from_aug(self) -> None:
        """The net's FP32 weights, biases and BF16 copies from the augmented parameters."""
        net = self.net
        for l, A in enumerate(self._views):
            dout, din = self.dims[l + 1], self.dims[l]
            net.W[l].copy_(A[:dout, :din])
            net.b[l].copy_(A[:dout, din])
            net.Wb[l].copy_(net.W[l])
            if getattr(net, "WbT", None) is not None and tuple(net.WbT[l].shape) == (din, dout):
                net.WbT[l].copy_(net.W[l].t())

    def _pack(self, lib, s: int) -> None:
        L.check(lib.pb_train_fused_pack(self.net.n_layers, self._dims_c, _p(self.w_aug), _p(self.w_img), s),
                "pb_train_fused_pack")

    def _fused_step(self, lib, s: int, x: torch.Tensor, y: torch.Tensor, rows: torch.Tensor, M: int, lr: float,
                    step: int, grad: bool) -> None:
        b1, b2 = self.betas
        L.check(lib.pb_train_fused_step(self.net.n_layers, self._dims_c, _p(x), _p(y), x.shape[0], _p(rows), M,
                                        self.batch,
                                        _p(self.w_aug), _p(self.m1), _p(self.m2), _p(self.w_img), _p(self.scratch),
                                        _p(self.grad) if grad else None, lr, b1, b2, self.eps, self.wd, step,
                                        _p(self.loss), _p(self.correct), _p(self.error), s), "pb_train_fused_step")

    def _run_fused(self) -> None:
        lib = _lib()
        s = torch.cuda.current_stream(self.dev).cuda_stream
        if self.resume:
            self._aug_from_net()
        else:
            self.w_aug.copy_(self.init_aug)
        self._pack(lib, s)
        self.m1.zero_()
        self.m2.zero_()
        self.loss.zero_()
        self.correct.zero_()
        b1, b2 = self.betas
        step, launches = 0, 1
        for ep in range(self.epochs):
            lr = self.lr * 0.5 * (1.0 + math.cos(math.pi * ep / max(self.epochs, 1)))
            for b0 in range(0, self.n, self.batch):
                M = min(self.batch, self.n - b0)
                step += 1
                self._fused_step(lib, s, self.X, self.Y, self.perm[ep, b0 : b0 + M], M, lr, step,
                                 grad=self.data_parallel)
                launches += 2
                if self.data_parallel:
                    from pybasin_b200.sharding import allreduce_gradients

                    allreduce_gradients([self.grad], group=self.group)
                    L.check(lib.pb_train_fused_adamw(self.net.n_layers, self._dims_c, _p(self.w_aug), _p(self.m1),
                                                     _p(self.m2), _p(self.grad), _p(self.w_img), lr, b1, b2,
                                                     self.eps, self.wd, step, s), "pb_train_fused_adamw")
                    launches += 1
        self._net_from_aug()
        self.launches = launches

    # -- one run, as launched (captured once) ------------------------------------------
    def _reset(self) -> None:
        if not self.resume:
            for p, p0 in zip(self.params, self.init):
                p.copy_(p0)
            for w, w0 in zip(self.net.Wb, self.init_bf16):
                w.copy_(w0)
            for w, w0 in zip(self.WbT, self.init_bf16_t):
                w.copy_(w0)
        for m in self.m1 + self.m2:
            m.zero_()
        self.loss.zero_()
        self.correct.zero_()

    def _adamw(self, lib, s: int, M: int, lr: float, step: int) -> None:
        net = self.net
        L_ = net.n_layers
        nt = 2 * L_
        vp = ctypes.c_void_p
        w = (vp * nt)(*[p.data_ptr() for p in self.params])
        wb = (vp * nt)(*([x.data_ptr() for x in net.Wb] + [None] * L_))
        wbt = (vp * nt)(*([x.data_ptr() for x in self.WbT] + [None] * L_))
        cols = (ctypes.c_int64 * nt)(*([int(w_.shape[1]) for w_ in net.W] + [1] * L_))
        m1 = (vp * nt)(*[m.data_ptr() for m in self.m1])
        m2 = (vp * nt)(*[m.data_ptr() for m in self.m2])
        parts = (vp * nt)(*([g.data_ptr() for g in self.gw_part] + [g.data_ptr() for g in self.gb_part]))
        n = (ctypes.c_int64 * nt)(*[p.numel() for p in self.params])
        stride = (ctypes.c_int64 * nt)(*([w_.numel() for w_ in net.W] + [b.numel() for b in net.b]))
        splits = 1 if self.data_parallel else -(-M // KC)  # data parallel: reduced into partial 0
        nparts = (ctypes.c_int32 * nt)(*([splits] * (2 * L_)))
        wd = (ctypes.c_float * nt)(*([self.wd] * L_ + [0.0] * L_))
        L.check(lib.pb_train_adamw(nt, w, wb, wbt, cols, m1, m2, parts, n, stride, nparts, wd, lr, self.betas[0],
                                   self.betas[1], self.eps, step, s), "pb_train_adamw")

    def _grads(self, lib, s: int, x: torch.Tensor, xT: torch.Tensor, ldxT: int, y: torch.Tensor, M: int) -> int:
        """Forward, loss and backward of one minibatch (M rows of x, the same rows
        transposed in xT with row stride ldxT, labels y): the gradient partials land
        in gw_part / gb_part.  Returns the launches issued."""
        net = self.net
        L_ = net.n_layers
        dims = self.dims
        d = net.d_in
        C = dims[-1]
        B = self.batch
        h, hw = x, d
        for l in range(L_):
            N, K = dims[l + 1], dims[l]
            if l < L_ - 1:
                gemm_tc(h, hw, 1, net.Wb[l], K, 1, M, N, K, TRAIN_FWD_GELU, bias=net.b[l], out_bf16=self.act[l + 1],
                        out_t=self.actT[l + 1], ldt=B, z_pre=self.z[l], ldc=N, error=self.error, stream=s)
                h, hw = self.act[l + 1], N
            else:
                gemm_tc(h, hw, 1, net.Wb[l], K, 1, M, N, K, TRAIN_FWD_LINEAR, bias=net.b[l], out_f32=self.logits,
                        ldc=N, error=self.error, stream=s)
        L.check(lib.pb_train_xent(_p(self.logits), C, _p(y), M, C, 1.0 / M, _p(self.dz[L_ - 1]), C,
                                  _p(self.dzT[L_ - 1]), B, None, _p(self.loss), _p(self.correct), s), "pb_train_xent")
        launches = L_ + 1
        for l in reversed(range(L_)):
            N, K = dims[l + 1], dims[l]
            XT, ldX = (xT, ldxT) if l == 0 else (self.actT[l], B)
            # dW_l = dZ_l^T X_l and db_l = dZ_l^T 1 over the batch (both read along the
            # batch from the transposed copies), in chunks of KC rows
            gemm_tc(self.dzT[l], B, 1, XT, ldX, 1, N, K, M, TRAIN_DW, out_f32=self.gw_part[l], ldc=K,
                    col_part=self.gb_part[l], ldp=N, bn=dw_tile(K), error=self.error, stream=s)
            launches += 1
            if l > 0:
                # dZ_l-1 = (dZ_l W_l) * GELU'(Z_l-1), W_l read as its transposed copy
                gemm_tc(self.dz[l], N, 1, self.WbT[l], N, 1, M, K, N, TRAIN_DX, z_in=self.z[l - 1], ldz=K,
                        out_bf16=self.dz[l - 1], out_t=self.dzT[l - 1], ldt=B, ldc=K, error=self.error, stream=s)
                launches += 1
        return launches

    def _exchange(self, M: int) -> None:
        """Data parallel: each gradient's chunk partials summed into partial 0, then
        averaged over the ranks (one flat all-reduce)."""
        from pybasin_b200.sharding import allreduce_gradients

        splits = -(-M // KC)
        firsts = []
        for parts in self.gw_part + self.gb_part:
            if splits > 1:
                parts[0].copy_(parts[:splits].sum(0))
            firsts.append(parts[0])
        allreduce_gradients(firsts, group=self.group)

    def gradients(self, x: torch.Tensor, labels: torch.Tensor) -> tuple[list[torch.Tensor], list[torch.Tensor]]:
        """Gradients of the mean loss over one minibatch (at most ``batch`` rows) at the
        current weights, summed from their partials (for checking; no update)."""
        lib = _lib()
        M = x.shape[0]
        if M > self.batch:
            raise ValueError("at most one minibatch")
        y = labels.to(self.dev, torch.int32).contiguous()
        x = x.contiguous()
        if self.fused:
            s = torch.cuda.current_stream(self.dev).cuda_stream
            self._aug_from_net()
            self._pack(lib, s)
            rows = torch.arange(M, dtype=torch.int32, device=self.dev)
            self._fused_step(lib, s, x, y, rows, M, 0.0, 1, grad=True)
            gW = [G[: self.dims[l + 1], : self.dims[l]].clone() for l, G in enumerate(self._gviews)]
            gb = [G[: self.dims[l + 1], self.dims[l]].clone() for l, G in enumerate(self._gviews)]
            return gW, gb
        self._grads(lib, torch.cuda.current_stream(self.dev).cuda_stream, x, x.t().contiguous(), M, y, M)
        splits = -(-M // KC)
        gW = [g[:splits].sum(0) for g in self.gw_part]
        gb = [g[:splits].sum(0) for g in self.gb_part]
        return gW, gb

    def _run(self) -> None:
        if self.fused:
            self._run_fused()
            return
        lib = _lib()
        s = torch.cuda.current_stream(self.dev).cuda_stream
        d = self.net.d_in
        self._reset()
        step = 0
        launches = 0
        for ep in range(self.epochs):
            lr = self.lr * 0.5 * (1.0 + math.cos(math.pi * ep / max(self.epochs, 1)))
            L.check(lib.pb_train_gather(_p(self.X), d, _p(self.Y), _p(self.perm[ep]), self.n, _p(self.Xs),
                                        _p(self.XsT), _p(self.Ys), s), "pb_train_gather")
            launches += 1
            for b0 in range(0, self.n, self.batch):
                M = min(self.batch, self.n - b0)
                launches += self._grads(lib, s, self.Xs[b0 : b0 + M], self.XsT[:, b0:], self.n, self.Ys[b0 : b0 + M],
                                        M)
                if self.data_parallel:
                    self._exchange(M)
                step += 1
                self._adamw(lib, s, M, lr, step)
                launches += 1
        self.launches = launches

    # -- public ------------------------------------------------------------------------
    def capture(self) -> float:
        """Capture the run as a CUDA graph (once); returns the seconds it took."""
        if self.graph is not None:
            return 0.0
        t0 = time.perf_counter()
        # one eager launch first: the kernels' shared-memory limits are raised outside the capture
        if self.fused:
            lib = _lib()
            s = torch.cuda.current_stream(self.dev).cuda_stream
            M = min(self.batch, self.n)
            self._fused_step(lib, s, self.X, self.Y, self.perm[0, :M], M, 0.0, 1, grad=True)
        else:
            gemm_tc(self.X, self.net.d_in, 1, self.net.Wb[0], self.net.d_in, 1, 1, 16, self.net.d_in, TRAIN_FWD_LINEAR,
                    out_f32=self.logits, ldc=self.logits.shape[1], bn=16) if self.logits.shape[1] >= 16 else \
                gemm_tc(self.X, self.net.d_in, 1, self.net.Wb[0], self.net.d_in, 1, 1, self.logits.shape[1],
                        self.net.d_in, TRAIN_FWD_LINEAR, out_f32=self.logits, ldc=self.logits.shape[1])
        torch.cuda.synchronize(self.dev)
        side = torch.cuda.Stream(device=self.dev)
        side.wait_stream(torch.cuda.current_stream(self.dev))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            self._run()
        torch.cuda.current_stream(self.dev).wait_stream(side)
        torch.cuda.synchronize(self.dev)
        self.graph = g
        self.capture_s = time.perf_counter() - t0
        return self.capture_s

    def load(self, x: torch.Tensor, labels: torch.Tensor) -> None:
        """Copy a training set (n_rows x d_in BF16 inputs, int32 labels) in (asynchronous)."""
        if x.shape != self.X.shape or labels.shape != self.Y.shape:
            raise ValueError(f"training set must be {tuple(self.X.shape)} inputs and {tuple(self.Y.shape)} labels")
        self.X.copy_(x, non_blocking=True)
        self.Y.copy_(labels.to(torch.int32), non_blocking=True)

    def train(self, x: torch.Tensor | None = None, labels: torch.Tensor | None = None, use_graph: bool = True) -> None:
        """One training run from the initial weights on the loaded (or given) set;
        asynchronous on the current stream.  The net's weights hold the result."""
        if x is not None:
            self.load(x, labels)
        if use_graph and self.data_parallel:
            import torch.distributed as dist

            # a collective inside the captured run needs NCCL (gloo is host-driven)
            use_graph = dist.is_initialized() and dist.get_backend(self.group) == "nccl"
        if use_graph and self.graph is None:
            self.capture()
        ev = None
        if self.timing:  # CUDA events around the run (read by run_ms)
            ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            ev[0].record()
        if use_graph:
            self.graph.replay()
        else:
            self._run()
        if ev is not None:
            ev[1].record()
        self._events = ev
        self.net._step += 1  # repack the inference weights
        self.net._adam = None

    def run_ms(self) -> float | None:
        """Device time of the last run when ``timing`` was set (waits for it)."""
        if getattr(self, "_events", None) is None:
            return None
        self._events[1].synchronize()
        return self._events[0].elapsed_time(self._events[1])

    def stats(self) -> dict[str, float]:
        """Mean training loss and accuracy over all epochs of the last run, and the error flag."""
        rows = self.n * self.epochs
        return {"loss": float(self.loss.item()) / rows, "accuracy": float(self.correct.item()) / rows,
                "error": int(self.error.item())}

    def flops(self) -> float:
        """Algorithmic FLOPs of one run: 2 K N per layer and row forward, twice that backward
        (input and weight gradients; the first layer has no input gradient)."""
        d = self.dims
        fwd = sum(2 * d[l] * d[l + 1] for l in range(len(d) - 1))
        bwd = 2 * fwd - 2 * d[0] * d[1]
        return float(self.n * self.epochs * (fwd + bwd))
