// Right-hand sides of the built-in systems as templated device functors.
//
// Each functor exposes S (state dimension), NP (parameter count) and
//   template <class R> static void f(double t, const R* y, R* dy, const R* p)
// where R is the stage arithmetic (double for the plain FP64 kernel, float for
// the mixed kernel).  Time always arrives in FP64; functors that need t reduce
// it in FP64 before handing a small argument to R arithmetic.
#pragma once
#include <cuda_runtime.h>

namespace pb {

__device__ __forceinline__ float r_sin(float x) { return sinf(x); }
__device__ __forceinline__ double r_sin(double x) { return sin(x); }

// cos(t) for t in FP64.  FP64 stages: plain cos.  FP32 stages: reduce t modulo
// 2*pi in FP64 (|t| stays far below 2^40 here, so k*2pi is exact enough) and
// evaluate cosf on the reduced argument in [-pi, pi].
template <class R>
__device__ __forceinline__ R cos_of_time(double t);
template <>
__device__ __forceinline__ double cos_of_time<double>(double t) { return cos(t); }
template <>
__device__ __forceinline__ float cos_of_time<float>(double t)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double inv_two_pi = 0.15915494309189533576888376337251;
    double k = rint(t * inv_two_pi);
    double r = fma(-k, two_pi, t);
    return cosf(static_cast<float>(r));
}

// dy/dt = p0 * y  (tests/unit/solvers/test_solver.py:16-21 of the reference)
template <int DIM>
struct SysLinear {
    static constexpr int S = DIM;
    static constexpr int NP = 1;
    template <class R>
    __device__ __forceinline__ static void f(double, const R* y, R* dy, const R* p)
    {
#pragma unroll
        for (int i = 0; i < S; ++i) dy[i] = p[0] * y[i];
    }
};

// Damped driven pendulum, p = [alpha, T, K]
// (case_studies/pendulum/pendulum_ode.py:23-40)
struct SysPendulum {
    static constexpr int S = 2;
    static constexpr int NP = 3;
    template <class R>
    __device__ __forceinline__ static void f(double, const R* y, R* dy, const R* p)
    {
        dy[0] = y[1];
        dy[1] = -p[0] * y[1] + p[1] - p[2] * r_sin(y[0]);
    }
};

// Forced Duffing oscillator, p = [delta, k3, A]
// (case_studies/duffing_oscillator/duffing_ode.py:26-42)
struct SysDuffing {
    static constexpr int S = 2;
    static constexpr int NP = 3;
    template <class R>
    __device__ __forceinline__ static void f(double t, const R* y, R* dy, const R* p)
    {
        const R x = y[0];
        dy[0] = y[1];
        dy[1] = -p[0] * y[1] - p[1] * x * x * x + p[2] * cos_of_time<R>(t);
    }
};

// Lorenz system, p = [sigma, r, b].  MASKED freezes the flow once max|y| >= 200
// (case_studies/lorenz/lorenz_ode.py:28-64); the plain variant is the JAX one
// used with a stop event (case_studies/lorenz/lorenz_jax_ode.py).
template <bool MASKED>
struct SysLorenz {
    static constexpr int S = 3;
    static constexpr int NP = 3;
    template <class R>
    __device__ __forceinline__ static void f(double, const R* y, R* dy, const R* p)
    {
        R f0 = p[0] * (y[1] - y[0]);
        R f1 = p[1] * y[0] - y[0] * y[2] - y[1];
        R f2 = y[0] * y[1] - p[2] * y[2];
        if (MASKED) {
            R m = fmax(fabs(y[0]), fmax(fabs(y[1]), fabs(y[2])));
            if (!(m < R(200))) f0 = f1 = f2 = R(0);
        }
        dy[0] = f0;
        dy[1] = f1;
        dy[2] = f2;
    }
};

}  // namespace pb
