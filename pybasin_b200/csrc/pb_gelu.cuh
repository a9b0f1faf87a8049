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

// d gelu / dx = 0.5 (1 + t) + 0.5 x (1 - t^2) du/dx, du/dx = sqrt(2/pi) (1 + 3 * 0.044715 x^2)
__device__ __forceinline__ float gelu_grad(float x)
{
    const float x2 = x * x;
    const float t = tanh_approx(x * fmaf(kGeluB, x2, kGeluA));
    const float du = fmaf(kGeluB3, x2, kGeluA);
    return fmaf(0.5f * x * du, fmaf(-t, t, 1.f), 0.5f * (1.f + t));
}

}  // namespace pb
