// Right-hand sides of the built-in systems as templated device functors.
//
// Each functor exposes S (state dimension), NP (parameter count) and
//   template <class R, class Clock> static void f(const Clock& c, const R* y, R* dy, const R* p)
// where R is the stage arithmetic (double for the plain FP64 kernel, float for
// the mixed kernel) and `c` is the time of the stage.  Time is kept in FP64 by
// the integrator; the FP32 clock carries it already reduced modulo 2*pi (one
// FP64 reduction per step, stage offsets added in FP32), which is all a
// periodically forced system needs.
#pragma once
#include "pb_compat.cuh"

namespace pb {

// time of one stage, FP64 kernel: the stage instant itself
struct ClockF64 {
    double t;
};
// time of one stage, FP32 kernel: the stage instant modulo 2*pi, in [-pi, pi + h]
struct ClockF32 {
    float phase;
};

__device__ __forceinline__ double clock_cos(const ClockF64& c) { return cos(c.t); }
// stage instant of an FP64 clock (right-hand sides that use t itself, kExactTime)
__device__ __forceinline__ double clock_time(const ClockF64& c) { return c.t; }

// Sys::kExactTime if the system declares it, else false (the built-in systems use
// cos(t) only, through the FP32 phase clock in the mixed kernel)
template <class Sys, class = void>
struct exact_time {
    static constexpr bool value = false;
};
template <class Sys>
struct exact_time<Sys, decltype(void(Sys::kExactTime))> {
    static constexpr bool value = Sys::kExactTime;
};
__device__ __forceinline__ float clock_cos(const ClockF32& c)
{
#ifndef PB_ACCURATE_COS
    // the step's phases lie in [-pi, pi + h] (base reduced into [-pi, pi] in FP64);
    // measured max |__cosf(x) - cos(x)| on B200 is 4.0e-7 for |x| <= pi, 4.2e-7 for
    // |x| <= pi + 1 and 7.1e-7 for |x| <= 2 pi, at or below the FP32 stage
    // resolution of a unit-scale state
    return __cosf(c.phase);
#else
    return cosf(c.phase);
#endif
}

// Explicit fused multiply-add.  Every multiply-add with two product operands in
// the integrator and the built-in right-hand sides is written with it, so the
// rounding does not depend on which product the compiler contracts in a given
// kernel: the queue, probed, plain and redo kernels produce bit-identical
// trajectories.
__device__ __forceinline__ float fmad(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmad(double a, double b, double c) { return fma(a, b, c); }

__device__ __forceinline__ float r_sin(float x) { return sinf(x); }
__device__ __forceinline__ double r_sin(double x) { return sin(x); }
__device__ __forceinline__ float r_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double r_abs(double x) { return fabs(x); }

// Per-step time base: t and dt in FP64; stage clocks derived from it.
struct TimeBaseF64 {
    double t, dt;
    __device__ __forceinline__ ClockF64 at(double c) const { return ClockF64{t + c * dt}; }
};
struct TimeBaseF32 {
    float r0, h;  // t mod 2*pi (FP64-reduced, then rounded), FP32 step
    __device__ __forceinline__ ClockF32 at(double c) const { return ClockF32{r0 + static_cast<float>(c) * h}; }
};
// t - 2*pi*k with k the nearest integer to t / (2*pi), in [-pi, pi]
__device__ __forceinline__ float reduce_two_pi(double t)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double inv_two_pi = 0.15915494309189533576888376337251;
    const double k = rint(t * inv_two_pi);
    return static_cast<float>(fma(-k, two_pi, t));
}

// dy/dt = p0 * y  (tests/unit/solvers/test_solver.py:16-21 of the reference)
template <int DIM>
struct SysLinear {
    static constexpr int S = DIM;
    static constexpr int NP = 1;
    static constexpr bool kTime = false;
    template <class R, class C>
    __device__ __forceinline__ static void f(const C&, const R* y, R* dy, const R* p)
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
    static constexpr bool kTime = false;
    template <class R, class C>
    __device__ __forceinline__ static void f(const C&, const R* y, R* dy, const R* p)
    {
        dy[0] = y[1];
        dy[1] = fmad(-p[2], r_sin(y[0]), fmad(-p[0], y[1], p[1]));
    }
};

// Forced Duffing oscillator, p = [delta, k3, A]
// (case_studies/duffing_oscillator/duffing_ode.py:26-42)
struct SysDuffing {
    static constexpr int S = 2;
    static constexpr int NP = 3;
    static constexpr bool kTime = true;
    template <class R, class C>
    __device__ __forceinline__ static void f(const C& c, const R* y, R* dy, const R* p)
    {
        // -delta*v - k3*x^3 + A*cos(t), grouped for a two-level dependency chain
        const R x = y[0];
        dy[0] = y[1];
        const R forcing = p[2] * static_cast<R>(clock_cos(c));
        dy[1] = fmad(-p[1] * x, x * x, fmad(-p[0], y[1], forcing));
    }
};

// Friction oscillator with a smoothed stick-slip law, p = [v_d, xi, musd, mud,
// muv, v0] (case_studies/friction/friction_ode.py:32-75): slip when
// |v - v_d| > 1e-4, else a transition when |x + 2 xi v| > mud musd, else stick.
__device__ __forceinline__ float r_exp(float x) { return expf(x); }
__device__ __forceinline__ double r_exp(double x) { return exp(x); }
__device__ __forceinline__ float r_tanh(float x) { return tanhf(x); }
__device__ __forceinline__ double r_tanh(double x) { return tanh(x); }

struct SysFriction {
    static constexpr int S = 2;
    static constexpr int NP = 6;
    static constexpr bool kTime = false;
    template <class R, class C>
    __device__ __forceinline__ static void f(const C&, const R* y, R* dy, const R* p)
    {
        const R vd = p[0], xi = p[1], musd = p[2], mud = p[3], muv = p[4], v0 = p[5];
        const R disp = y[0], vel = y[1];
        const R vrel = vel - vd;
        const R avr = r_abs(vrel) / v0;
        const R f_fric = fmad(muv, avr, fmad(mud * (musd - R(1)), r_exp(-avr), mud));
        const R base = fmad(R(-2) * xi, vel, -disp);  // -disp - 2 xi vel
        const bool slip = r_abs(vrel) > R(1e-4);
        const bool trans = r_abs(base) > mud * musd;
        const R slip_vel = fmad(-r_tanh(R(50) * vrel), f_fric, base);
        const R trans_vel = fmad(mud * musd, r_tanh(R(50) * f_fric), base);
        const R stick_vel = vd - vel;
        dy[0] = (slip || trans) ? vel : vd;
        dy[1] = slip ? slip_vel : (trans ? trans_vel : stick_vel);
    }
};

// Lorenz system, p = [sigma, r, b].  MASKED freezes the flow once max|y| >= 200
// (case_studies/lorenz/lorenz_ode.py:28-64); the plain variant is the JAX one
// used with a stop event (case_studies/lorenz/lorenz_jax_ode.py).
template <bool MASKED>
struct SysLorenz {
    static constexpr int S = 3;
    static constexpr int NP = 3;
    static constexpr bool kTime = false;
    template <class R, class C>
    __device__ __forceinline__ static void f(const C&, const R* y, R* dy, const R* p)
    {
        R f0 = p[0] * (y[1] - y[0]);
        R f1 = fmad(p[1], y[0], fmad(-y[0], y[2], -y[1]));
        R f2 = fmad(y[0], y[1], -p[2] * y[2]);
        if (MASKED) {
            const R m = fmax(r_abs(y[0]), fmax(r_abs(y[1]), r_abs(y[2])));
            if (!(m < R(200))) f0 = f1 = f2 = R(0);
        }
        dy[0] = f0;
        dy[1] = f1;
        dy[2] = f2;
    }
};

}  // namespace pb
