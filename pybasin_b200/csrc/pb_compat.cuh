// Lets the kernel headers compile both under nvcc and under NVRTC (the runtime
// compilation of user right-hand sides, pb_rtc.cu), where no host headers exist:
// the fixed-width integer types, the two CUDART constants the kernels use, and
// two type traits.
#pragma once
#ifdef __CUDACC_RTC__
typedef signed char int8_t;
typedef short int16_t;
typedef int int32_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
#define CUDART_INF __longlong_as_double(0x7ff0000000000000LL)
#define CUDART_NAN __longlong_as_double(0xfff8000000000000LL)
#else
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>
#endif

namespace pb {
template <class A, class B>
struct same_type {
    static constexpr bool value = false;
};
template <class A>
struct same_type<A, A> {
    static constexpr bool value = true;
};
template <bool B, class T, class F>
struct pick_type {
    using type = T;
};
template <class T, class F>
struct pick_type<false, T, F> {
    using type = F;
};
}  // namespace pb
