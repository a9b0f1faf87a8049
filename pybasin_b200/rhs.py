"""User right-hand sides compiled at run time (NVRTC) into the fused integrator.

The reference lets users write an ODE symbolically and compiles it to native code
(``SymPyODE``, src/zigode/sympy_ode.py:49-78: SymPy expressions printed as C,
built into a library the native solver loads).  Here the printed expressions
become a device functor inside the same Dopri5 + feature kernels as the built-in
systems (``pb_rhs_compile``), so a user system runs the fused, scheduled,
mixed-precision path too.

* :class:`ExpressionODE` — an ODE system with the reference's interface
  (``params`` mapping in column order, ``ode``, ``get_str``) whose right-hand side
  is a list of expressions (SymPy or strings) over named states, parameters and
  ``t``.  Pass it to :class:`~pybasin_b200.solver.B200Dopri5Solver` like any
  built-in system.
* :func:`compile_rhs` — the C-level entry: C expressions in ``y[i]``, ``p[k]``
  and ``t``.

Compiled modules are cached on disk (``PB_RHS_CACHE``, default
``pybasin_b200/_lib/rhs_cache``) keyed by the generated source, so a system
compiles once per machine (a few seconds for the eight kernel variants).
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path
from typing import Any, Sequence

import numpy as np
import torch

from pybasin_b200 import _lib as L
from pybasin_b200.odes import ODESystem

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
INCLUDE_DIRS = [PKG / "csrc", ROOT / "include"]


def default_cache_dir() -> Path:
    return Path(os.environ.get("PB_RHS_CACHE", PKG / "_lib" / "rhs_cache"))


class CompileError(RuntimeError):
    """NVRTC rejected the generated source; ``log`` holds the compiler output."""

    def __init__(self, code: int, log: str):
        super().__init__(f"pb_rhs_compile failed ({L.error_string(code)}):\n{log}")
        self.code = code
        self.log = log


class CompiledRHS:
    """A loaded program (``pb_rhs_program``) on one device; released on deletion."""

    def __init__(self, handle: int, dim: int, n_params: int, precision: int, device: int):
        self.handle = handle
        self.dim = dim
        self.n_params = n_params
        self.precision = precision
        self.device = device

    def __del__(self):
        h, self.handle = getattr(self, "handle", None), None
        if h:
            try:
                L.load(build_if_missing=False).pb_rhs_release(ctypes.c_void_p(h))
            except Exception:
                pass


def compile_rhs(
    exprs: Sequence[str],
    n_params: int,
    precision: int,
    preamble: str | None = None,
    cache_dir: str | Path | None = None,
    load: bool = True,
) -> CompiledRHS | None:
    """Compile C expressions (``dy[i]/dt = exprs[i]`` in ``y``, ``p``, ``t``) for sm_100a.

    With ``load=False`` only compiles (filling the cache); that needs no GPU.
    Otherwise loads the module on the current CUDA device.
    """
    lib = L.load()
    dim = len(exprs)
    arr = (ctypes.c_char_p * dim)(*[e.encode() for e in exprs])
    inc = (ctypes.c_char_p * len(INCLUDE_DIRS))(*[str(d).encode() for d in INCLUDE_DIRS])
    cache = Path(cache_dir) if cache_dir is not None else default_cache_dir()
    cache.mkdir(parents=True, exist_ok=True)
    log = ctypes.create_string_buffer(1 << 16)
    out = ctypes.c_void_p()
    rc = lib.pb_rhs_compile(
        arr, dim, n_params, preamble.encode() if preamble else None, precision, inc, len(INCLUDE_DIRS),
        str(cache).encode(), ctypes.byref(out) if load else None, log, len(log),
    )
    if rc == L.PB_ECOMPILE:
        raise CompileError(rc, log.value.decode(errors="replace"))
    L.check(rc, "pb_rhs_compile")
    if not load:
        return None
    return CompiledRHS(out.value, dim, n_params, precision, torch.cuda.current_device())


# ---------------------------------------------------------------------------
# SymPy -> C expressions
# ---------------------------------------------------------------------------
def c_expressions(state: Sequence[Any], params: Sequence[Any], rhs: Sequence[Any], time: Any = "t") -> list[str]:
    """Print ``rhs`` as C over ``y[i]`` (state ``i``), ``p[k]`` (parameter ``k``) and ``t``.

    Small integer powers become products (no ``pow`` of a float by an int), and
    ``x**0.5`` becomes ``sqrt(x)``."""
    import sympy as sp
    from sympy.printing.c import C99CodePrinter

    class _Printer(C99CodePrinter):
        def _print_Pow(self, expr):
            b, e = expr.base, expr.exp
            if e.is_Integer and 2 <= int(e) <= 4:
                inner = self.parenthesize(b, 100)
                return "(" + "*".join([inner] * int(e)) + ")"
            if e.is_Integer and int(e) == -1:
                return "(1.0/" + self.parenthesize(b, 100) + ")"
            if e == sp.Rational(1, 2):
                return "sqrt(" + self._print(b) + ")"
            return super()._print_Pow(expr)

    def sym(x):
        return sp.Symbol(x) if isinstance(x, str) else x

    st = [sym(s) for s in state]
    pr = [sym(p) for p in params]
    tt = sym(time)
    repl = {s: sp.Symbol(f"y[{i}]") for i, s in enumerate(st)}
    repl.update({p: sp.Symbol(f"p[{k}]") for k, p in enumerate(pr)})
    repl[tt] = sp.Symbol("t")
    names = {str(s) for s in st} | {str(p) for p in pr} | {str(tt)}
    printer = _Printer()
    out = []
    for r in rhs:
        expr = sp.sympify(r, locals={n: sp.Symbol(n) for n in names}) if isinstance(r, str) else r
        out.append(printer.doprint(sp.sympify(expr).xreplace(repl)))
    return out


class ExpressionODE(ODESystem):
    """ODE system given by expressions; compiled for the GPU on first use.

    :param params: parameter values, in the column order of the parameter array
        (``params_to_array``, src/pybasin/solvers/torch_ode_system.py:57-66).
    :param state: state names (or SymPy symbols), in ``y`` order.
    :param rhs: one expression per state (SymPy or a string over the names and ``t``).
    :param name: used by ``get_str``.
    """

    b200_system = "user"

    def __init__(self, params: dict[str, float], state: Sequence[Any], rhs: Sequence[Any], name: str = "user_ode",
                 time: Any = "t", preamble: str | None = None):
        super().__init__(dict(params))
        if len(rhs) != len(state):
            raise ValueError(f"rhs has {len(rhs)} entries but state has {len(state)}")
        if not 1 <= len(state) <= L.MAX_USER_DIM:
            raise ValueError(f"state dimension must be 1..{L.MAX_USER_DIM}")
        if len(params) > L.MAX_PARAMS:
            raise ValueError(f"at most {L.MAX_PARAMS} parameters are supported")
        self.name = name
        self.state_names = [str(s) for s in state]
        self.param_names = list(params.keys())
        self.b200_rhs = c_expressions(state, self.param_names, rhs, time)
        self.preamble = preamble
        self._sym = (list(state), self.param_names, list(rhs), time)
        self._programs: dict[tuple[int, int], CompiledRHS] = {}
        self._host_fn = None
        self._lock = threading.Lock()

    @classmethod
    def from_sympy(cls, name: str, state, params, rhs, values: dict[str, float]) -> "ExpressionODE":
        """The reference's ``SymPyODE(name, state, params, rhs)`` arguments plus parameter values."""
        names = [str(p) for p in params]
        return cls({n: float(values[n]) for n in names}, state, rhs, name=name)

    def program(self, precision: int, device: int | None = None) -> CompiledRHS:
        """The compiled program for ``precision`` on ``device`` (compiled or loaded once)."""
        dev = torch.cuda.current_device() if device is None else int(device)
        key = (precision, dev)
        with self._lock:
            prog = self._programs.get(key)
            if prog is None:
                with torch.cuda.device(dev):
                    prog = compile_rhs(self.b200_rhs, len(self.param_names), precision, self.preamble)
                self._programs[key] = prog
            return prog

    def ode(self, t, y, p):
        """Host evaluation (NumPy arrays), for checks against CPU integrators."""
        if getattr(self, "_host_fn", None) is None:
            self._host_fn = self._lambdify()
        return np.asarray(self._host_fn(t, list(np.asarray(y)), list(np.asarray(p))), dtype=np.float64)

    def _lambdify(self):
        import sympy as sp

        state, pnames, rhs, time = self._sym
        syms = [sp.Symbol(s) if isinstance(s, str) else s for s in state]
        psyms = [sp.Symbol(n) for n in pnames]
        tsym = sp.Symbol(time) if isinstance(time, str) else time
        names = {str(s) for s in syms} | set(pnames) | {str(tsym)}
        exprs = [sp.sympify(r, locals={n: sp.Symbol(n) for n in names}) if isinstance(r, str) else r for r in rhs]
        return sp.lambdify([tsym, syms, psyms], exprs, "numpy")

    def get_str(self) -> str:
        return f"{self.name}({self.params}): " + "; ".join(
            f"d{s}/dt = {r}" for s, r in zip(self.state_names, self.b200_rhs)
        )
