"""Runtime-compiled right-hand sides: expression printing, NVRTC compile (no GPU needed), errors.

The reference's precedent is SymPyODE (src/zigode/sympy_ode.py:49-78): SymPy
expressions printed as C and compiled to native code.  Here they compile into
the fused integrator kernels; these tests need NVRTC but no GPU.
"""

from __future__ import annotations

import time

import pytest
import sympy as sp

from pybasin_b200 import _lib as L
from pybasin_b200.rhs import CompileError, ExpressionODE, c_expressions, compile_rhs, default_cache_dir


def test_sympy_expressions_print_as_c_over_y_p_t():
    x, v, t = sp.symbols("x v t")
    delta, k3, A = sp.symbols("delta k3 A")
    out = c_expressions([x, v], [delta, k3, A], [v, -delta * v - k3 * x**3 + A * sp.cos(t)], t)
    assert out[0] == "y[1]"
    assert "pow" not in out[1] and "y[0]*y[0]*y[0]" in out[1]
    assert "cos(t)" in out[1] and "p[0]" in out[1] and "p[2]" in out[1]
    # string input, reciprocal and square root
    s = c_expressions(["a", "b"], ["mu"], ["b", "mu*(1 - a**2)*b - a + 1/a + a**0.5"])
    assert "sqrt(y[0])" in s[1] and "(1.0/y[0])" in s[1]


def test_expression_ode_interface_and_checks():
    ode = ExpressionODE({"mu": 1.5}, ["x", "v"], ["v", "mu*(1 - x**2)*v - x"], name="vdp")
    assert ode.params == {"mu": 1.5}
    assert ode.b200_system == "user" and len(ode.b200_rhs) == 2
    assert "vdp" in ode.get_str()
    dy = ode.ode(0.0, [2.0, 0.0], [1.5])
    assert dy.tolist() == [0.0, -2.0]
    with pytest.raises(ValueError):
        ExpressionODE({"mu": 1.0}, ["x", "v"], ["v"])
    from pybasin_b200.odes import resolve_system

    spec = resolve_system(ode, 2)
    assert spec.system == L.SYS_USER and spec.params.tolist() == [1.5]
    with pytest.raises(ValueError):
        resolve_system(ode, 3)


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_nvrtc_compiles_the_fused_kernels_for_sm100a(precision):
    exprs = c_expressions(["x", "v"], ["delta", "k3", "A"], ["v", "-delta*v - k3*x**3 + A*cos(t)"])
    compile_rhs(exprs, 3, precision, load=False)  # compile-ahead: fills the cache, no device
    t0 = time.perf_counter()
    compile_rhs(exprs, 3, precision, load=False)  # now a cache hit
    assert time.perf_counter() - t0 < 1.0
    assert any(default_cache_dir().glob("pbrhs_*.bin"))


def test_compile_error_reports_the_nvrtc_log():
    with pytest.raises(CompileError) as err:
        compile_rhs(["y[1]", "-p[0]*y[1] + not_a_name"], 1, L.PREC_MIXED, load=False)
    assert err.value.code == L.PB_ECOMPILE
    assert "not_a_name" in err.value.log
