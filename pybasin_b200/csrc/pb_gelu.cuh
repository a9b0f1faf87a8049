// GELU activation of the surrogate MLP, tanh form: 0.5 x (1 + tanh(u)),
// u = sqrt(2/pi) (x + 0.044715 x^3), with the hardware tanh (tanh.approx.f32,
// relative error about 2^-11, far below the BF16 rounding of the activations).
// Shared by the training kernels and the tensor-core inference kernel so that
// both evaluate the same function.
#pragma once

namespace pb {

__device__ __forceinline__ float tanh_approx(float x)
{
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// sqrt(2/pi), sqrt(2/pi) * 0.044715 and three times the latter
constexpr float kGeluA = 0.7978845608028654f;
constexpr float kGeluB = 0.0356774081363001f;
constexpr float kGeluB3 = 0.1070322244089003f;

__device__ __forceinline__ float gelu(float x)
{
    const float t = tanh_approx(x * fmaf(kGeluB, x * x, kGeluA));
    const float hx = 0.5f * x;
    return fmaf(hx, t, hx);
}

// Two FP32 lanes in one 64-bit register for the packed FP32 instructions of sm_100
// (fma/mul .f32x2, round to nearest, no flush): each lane rounds exactly as the
// scalar instruction does, so a packed form of a formula is bit-identical to it.
struct f32x2 {
    unsigned long long v;
};
__device__ __forceinline__ f32x2 f2(float a, float b)
{
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2_split(f32x2 x, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v));
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b)
{
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}

// gelu of two values, the operations of gelu() lane by lane
__device__ __forceinline__ void gelu2(float x0, float x1, float& g0, float& g1)
{
    const f32x2 x = f2(x0, x1);
    float u0, u1;
    f2_split(mul2(x, fma2(f2(kGeluB, kGeluB), mul2(x, x), f2(kGeluA, kGeluA))), u0, u1);
    const f32x2 t = f2(tanh_approx(u0), tanh_approx(u1));
    const f32x2 hx = mul2(f2(0.5f, 0.5f), x);
    f2_split(fma2(hx, t, hx), g0, g1);
}

// d gelu / dx = 0.5 (1 + t) + 0.5 x (1 - t^2) du/dx, du/dx = sqrt(2/pi) (1 + 3 * 0.044715 x^2)
__device__ __forceinline__ float gelu_grad(float x)
{
    const float x2 = x * x;
    const float t = tanh_approx(x * fmaf(kGeluB, x2, kGeluA));
    const float du = fmaf(kGeluB3, x2, kGeluA);
    return fmaf(0.5f * x * du, fmaf(-t, t, 1.f), 0.5f * (1.f + t));
}

}  // namespace pb
