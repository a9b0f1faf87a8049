"""Device-side driver of ``pb_solve_batch`` / ``pb_label_nearest``.

Owns nothing global: every call allocates its outputs through PyTorch's caching
allocator on the compute device and launches on the given CUDA stream, so
concurrent calls from several host threads (the reference's estimator runs the
main and template integrations in a 2-thread pool,
src/pybasin/basin_stability_estimator.py:499-512) do not interfere.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import torch

from pybasin_b200 import _lib as L


@dataclass(frozen=True)
class FeatureColumn:
    """One output column: feature ``kind`` (a ``pb_feature``) of state ``state``."""

    state: int
    kind: int
    param: float = 0.0
    name: str = ""
    param2: float = 0.0  # second parameter of the two-parameter window kinds


@dataclass
class SolveRequest:
    system: int
    dim: int
    y0: torch.Tensor  # (n_ic, dim) f32/f64 on the compute device
    params: torch.Tensor  # (n_rows, n_params) f64 on the compute device
    save_ts: torch.Tensor  # (n_save,) f64 on the compute device
    t_span: tuple[float, float]
    rtol: float
    atol: float
    layout: int = L.LAYOUT_SINGLE
    param_index: torch.Tensor | None = None  # (n_traj,) int32
    n_traj: int | None = None
    win_begin: int = 0
    columns: list[FeatureColumn] = field(default_factory=list)
    precision: int = L.PREC_FP64
    schedule: int = L.SCHED_QUEUE
    max_steps: int = 16**5
    unbounded_thr: float = 0.0
    keep_final: bool = True
    keep_full: bool = False
    out_dtype: torch.dtype = torch.float32
    keep_steps: bool = False
    block_size: int = 0
    grid_blocks: int = 0
    refill_lanes: int = 0  # QUEUE / PROBED: refill a warp's idle lanes once this many are idle (0: all 32)
    order: torch.Tensor | None = None  # (n_traj,) int32 processing order
    dense_mode: int = L.DENSE_DEFERRED
    window_record_cap: int = 0
    csr_row: torch.Tensor | None = None  # network systems: (n_nodes + 1,) int32
    csr_col: torch.Tensor | None = None  # network systems: (2 * n_edges,) int32
    program: object | None = None  # SYS_USER: the compiled right-hand side (rhs.CompiledRHS)
    peak_cap: int = 0  # orbit data: peak values kept per NUMBER_PEAKS column and trajectory


@dataclass
class SolveResult:
    features: torch.Tensor | None  # (n_traj, F) f64
    status: torch.Tensor  # (n_traj,) int32
    y_final: torch.Tensor | None  # (n_traj, dim)
    y_full: torch.Tensor | None  # (n_save, n_traj, dim)
    steps: torch.Tensor | None  # (n_traj,) int64
    peaks: torch.Tensor | None = None  # (n_traj, n_peak_columns, peak_cap) f64, NaN-padded


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _dtype_code(dt: torch.dtype) -> int:
    if dt == torch.float32:
        return L.DTYPE_F32
    if dt == torch.float64:
        return L.DTYPE_F64
    raise TypeError(f"unsupported dtype {dt}; expected float32 or float64")


def build_args(
    req: SolveRequest, out: SolveResult, queue: torch.Tensor | None, scratch: torch.Tensor | None
) -> L.SolveArgs:
    a = L.SolveArgs()
    n_traj = req.n_traj if req.n_traj is not None else _default_n_traj(req)
    a.system = req.system
    a.dim = req.dim
    a.precision = req.precision
    a.schedule = req.schedule
    a.layout = req.layout
    a.y0_dtype = _dtype_code(req.y0.dtype)
    a.n_params = req.params.shape[1]
    a.block_size = req.block_size
    a.grid_blocks = req.grid_blocks
    a.refill_lanes = req.refill_lanes
    a.n_ic = req.y0.shape[0]
    a.n_param_rows = req.params.shape[0]
    a.n_traj = n_traj
    a.y0 = _ptr(req.y0)
    a.params = _ptr(req.params)
    a.param_index = _ptr(req.param_index)
    a.csr_row = _ptr(req.csr_row)
    a.csr_col = _ptr(req.csr_col)
    a.t0 = float(req.t_span[0])
    a.t1 = float(req.t_span[1])
    a.save_ts = _ptr(req.save_ts)
    a.n_save = req.save_ts.shape[0]
    a.win_begin = req.win_begin
    a.rtol = float(req.rtol)
    a.atol = float(req.atol)
    a.max_steps = int(req.max_steps)
    a.unbounded_thr = float(req.unbounded_thr)
    if len(req.columns) > L.MAX_FEATURES:
        raise ValueError(f"at most {L.MAX_FEATURES} fused feature columns are supported")
    a.n_features = len(req.columns)
    for i, c in enumerate(req.columns):
        a.feat_state[i] = c.state
        a.feat_kind[i] = c.kind
        a.feat_param[i] = float(c.param)
        a.feat_param2[i] = float(c.param2)
    a.features_out = _ptr(out.features)
    a.status_out = _ptr(out.status)
    a.y_final_out = _ptr(out.y_final)
    a.y_full_out = _ptr(out.y_full)
    a.y_out_dtype = _dtype_code(req.out_dtype)
    a.steps_out = _ptr(out.steps)
    a.queue_counter = _ptr(queue)
    a.scratch = _ptr(scratch)
    a.order = _ptr(req.order)
    a.dense_mode = req.dense_mode
    a.window_record_cap = req.window_record_cap
    a.peaks_out = _ptr(out.peaks)
    a.peak_cap = req.peak_cap if out.peaks is not None else 0
    return a


def scratch_bytes(args: L.SolveArgs) -> int:
    """Device scratch ``pb_solve_batch`` needs for ``args`` (median windows, step records)."""
    n = L.load().pb_solve_scratch_bytes(ctypes.byref(args))
    if n < 0:
        raise ValueError("invalid solve arguments")
    return int(n)


def alloc_scratch(args: L.SolveArgs, device: torch.device) -> torch.Tensor | None:
    """Allocate (and attach to ``args``) the scratch buffer, 256-byte aligned."""
    n = scratch_bytes(args)
    if n == 0:
        args.scratch = None
        return None
    buf = torch.empty((n + 256,), dtype=torch.uint8, device=device)
    off = (-buf.data_ptr()) % 256
    view = buf[off : off + n]
    args.scratch = view.data_ptr()
    return view


def _default_n_traj(req: SolveRequest) -> int:
    if req.layout == L.LAYOUT_CROSS:
        return req.y0.shape[0] * req.params.shape[0]
    return req.y0.shape[0]


def launch_solve(lib, args: L.SolveArgs, program, stream_handle: int) -> None:
    """``pb_solve_batch``, or ``pb_solve_batch_rhs`` for a compiled user right-hand side."""
    if args.system == L.SYS_USER:
        if program is None:
            raise ValueError("a user system needs its compiled program (ExpressionODE.program)")
        L.check(lib.pb_solve_batch_rhs(ctypes.c_void_p(program.handle), ctypes.byref(args),
                                       ctypes.c_void_p(stream_handle)), "pb_solve_batch_rhs")
    else:
        L.check(lib.pb_solve_batch(ctypes.byref(args), ctypes.c_void_p(stream_handle)), "pb_solve_batch")


def solve(req: SolveRequest, stream: torch.cuda.Stream | None = None) -> SolveResult:
    """Launch one fused integration on ``stream`` (asynchronous)."""
    lib = L.load()
    dev = req.y0.device
    if dev.type != "cuda":
        raise RuntimeError("pybasin_b200 computes on a CUDA device only; y0 must be on cuda")
    n_traj = req.n_traj if req.n_traj is not None else _default_n_traj(req)
    req.n_traj = n_traj
    F = len(req.columns)
    out = SolveResult(
        features=torch.empty((n_traj, F), dtype=torch.float64, device=dev) if F else None,
        status=torch.empty((n_traj,), dtype=torch.int32, device=dev),
        y_final=torch.empty((n_traj, req.dim), dtype=req.out_dtype, device=dev) if req.keep_final else None,
        y_full=torch.empty((req.save_ts.shape[0], n_traj, req.dim), dtype=req.out_dtype, device=dev)
        if req.keep_full
        else None,
        steps=torch.empty((n_traj,), dtype=torch.int64, device=dev) if req.keep_steps else None,
    )
    n_peak_cols = sum(1 for c in req.columns if c.kind == L.FEAT_NUMBER_PEAKS)
    if req.peak_cap > 0 and n_peak_cols > 0:
        out.peaks = torch.empty((n_traj, n_peak_cols, req.peak_cap), dtype=torch.float64, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    with torch.cuda.stream(s):
        queue = torch.zeros((1,), dtype=torch.int64, device=dev)
        args = build_args(req, out, queue, None)
        scratch = alloc_scratch(args, dev)
    launch_solve(lib, args, req.program, s.cuda_stream)
    # the scratch was allocated on `s`, so the caching allocator keeps it until the
    # kernels queued there before its release have run
    del scratch, queue
    return out


def label_nearest(
    features: torch.Tensor,
    templates: torch.Tensor,
    template_class: torch.Tensor,
    n_classes: int,
    status: torch.Tensor | None = None,
    group_of: torch.Tensor | None = None,
    n_groups: int = 1,
    stream: torch.cuda.Stream | None = None,
) -> tuple[torch.Tensor, torch.Tensor]:
    """1-NN labels (int32, class ``n_classes`` = unbounded) and per-group counts."""
    lib = L.load()
    dev = features.device
    n, nf = features.shape
    labels = torch.empty((n,), dtype=torch.int32, device=dev)
    counts = torch.empty((n_groups, n_classes + 1), dtype=torch.int64, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    rc = lib.pb_label_nearest(
        _ptr(features),
        n,
        nf,
        _ptr(templates),
        templates.shape[0],
        _ptr(template_class),
        n_classes,
        _ptr(status),
        _ptr(group_of),
        n_groups,
        _ptr(labels),
        _ptr(counts),
        ctypes.c_void_p(s.cuda_stream),
    )
    L.check(rc, "pb_label_nearest")
    return labels, counts


def occupancy(system: int, dim: int, precision: int, schedule: int, block: int) -> tuple[int, int]:
    lib = L.load()
    bps = ctypes.c_int32(0)
    sms = ctypes.c_int32(0)
    L.check(
        lib.pb_query_occupancy(system, dim, precision, schedule, block, ctypes.byref(bps), ctypes.byref(sms)),
        "pb_query_occupancy",
    )
    return bps.value, sms.value


def _spread_bits(v: torch.Tensor, dims: int, bits: int) -> torch.Tensor:
    """Place bit b of v at position b*dims (Morton interleave helper)."""
    out = torch.zeros_like(v)
    for b in range(bits):
        out |= ((v >> b) & 1) << (b * dims)
    return out


def morton_keys(y0: torch.Tensor, bits: int | None = None, groups: torch.Tensor | None = None) -> torch.Tensor:
    """Z-order keys of the rows of ``y0`` over their bounding box (PyTorch ops; the
    host-side statement of ``pb_morton_keys``, which is bit-identical on finite input)."""
    n, dims = y0.shape
    d = min(dims, 4)
    bits = bits or max(1, 60 // d if d > 2 else 20)
    bits = min(bits, 62 // d)
    x = y0[:, :d].to(torch.float64)
    lo = x.amin(dim=0, keepdim=True)
    span = (x.amax(dim=0, keepdim=True) - lo).clamp_min(1e-300)
    q = ((x - lo) / span * ((1 << bits) - 1)).nan_to_num(0.0).clamp(0, (1 << bits) - 1).to(torch.int64)
    key = torch.zeros((n,), dtype=torch.int64, device=y0.device)
    for k in range(d):
        key |= _spread_bits(q[:, k], d, bits) << k
    if groups is not None:
        # group-major: 20 bits of group id above 40 bits of (truncated) Morton key
        key = (groups.to(torch.int64) << 40) | (key >> max(0, bits * d - 40))
    return key


def spatial_order(y0: torch.Tensor, bits: int | None = None, groups: torch.Tensor | None = None) -> torch.Tensor:
    """Permutation of the rows of ``y0`` along a Morton (Z-order) curve of its bounding box.

    Neighbouring initial conditions mostly share an attractor and a step count, so
    integrating them in the same warp keeps the warp's lanes busy together.  With
    ``groups`` (e.g. the parameter row of each IC) the order is group-major, so a
    warp does not mix parameter points.  Returns int32 indices on y0's device.
    On CUDA tensors :class:`MortonOrder` computes the same keys in two kernels.
    """
    if y0.shape[0] == 0:
        return torch.zeros((0,), dtype=torch.int32, device=y0.device)
    return torch.argsort(morton_keys(y0, bits, groups)).to(torch.int32)


class MortonOrder:
    """Device Z-order of the ICs (``pb_morton_keys`` + argsort), with its buffers
    kept between calls; keys are bit-identical to :func:`spatial_order`'s."""

    def __init__(self, device: torch.device):
        self.dev = torch.device(device)
        self.box = torch.empty((8,), dtype=torch.int64, device=self.dev)
        self.keys = torch.empty((0,), dtype=torch.int64, device=self.dev)

    def keys_of(self, y0: torch.Tensor, bits: int | None = None, groups: torch.Tensor | None = None) -> torch.Tensor:
        n, dims = y0.shape
        d = min(dims, 4)
        bits = bits or max(1, 60 // d if d > 2 else 20)
        bits = min(bits, 62 // d)
        if self.keys.shape[0] < n:
            self.keys = torch.empty((n,), dtype=torch.int64, device=self.dev)
        if y0.dtype not in (torch.float32, torch.float64) or not y0.is_contiguous():
            y0 = y0.contiguous().to(torch.float64 if y0.dtype == torch.float64 else torch.float32)
        g = None
        if groups is not None:
            g = groups.to(torch.int32).contiguous()
        rc = L.load().pb_morton_keys(
            y0.data_ptr(), L.DTYPE_F64 if y0.dtype == torch.float64 else L.DTYPE_F32, n, dims, bits,
            g.data_ptr() if g is not None else None, self.box.data_ptr(), self.keys.data_ptr(),
            torch.cuda.current_stream(self.dev).cuda_stream,
        )
        L.check(rc, "pb_morton_keys")
        return self.keys[:n]

    def __call__(self, y0: torch.Tensor, bits: int | None = None, groups: torch.Tensor | None = None,
                 out: torch.Tensor | None = None) -> torch.Tensor:
        """int32 processing order: the stable argsort of the keys (``pb_morton_order``,
        a radix sort over the key bits in use), written to ``out`` if given."""
        n, dims = y0.shape
        if out is None:
            out = torch.empty((n,), dtype=torch.int32, device=self.dev)
        if n == 0:
            return out
        d = min(dims, 4)
        bits = min(bits or max(1, 60 // d if d > 2 else 20), 62 // d)
        keys = self.keys_of(y0, bits, groups)
        lib = L.load()
        need = int(lib.pb_morton_order_scratch_bytes(n))
        if need < 0:
            raise RuntimeError("pb_morton_order_scratch_bytes failed")
        if getattr(self, "_sort_scratch", None) is None or self._sort_scratch.numel() < need:
            self._sort_scratch = torch.empty((need,), dtype=torch.uint8, device=self.dev)
        end_bit = 64 if groups is not None else bits * d
        L.check(lib.pb_morton_order(keys.data_ptr(), n, end_bit, self._sort_scratch.data_ptr(), need, out.data_ptr(),
                                    torch.cuda.current_stream(self.dev).cuda_stream), "pb_morton_order")
        return out
