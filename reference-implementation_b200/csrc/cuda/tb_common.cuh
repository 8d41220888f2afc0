// Device helpers shared by the kernels: element loads and stores for every
// TAPP storage type, rounding to the 16-bit operand formats, fast integer
// division for index decoding, and launch bookkeeping.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "../tb_plan.h"

// TAPP storage types (api/include/tapp/datatype.h:15-42 of the reference)
enum { T_F32 = 0, T_F64 = 1, T_C32 = 2, T_C64 = 3, T_F16 = 4, T_BF16 = 5 };

namespace tb {

void count_launch(int n = 1);
// counts one device or page-locked host allocation the library asks CUDA for
void count_allocation();
// stream-ordered allocation from the library's own device pool (runtime.cu)
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s);

// ---------------------------------------------------------------------------
// Division by an invariant 32-bit divisor with a multiply-high
// (T. Granlund, P. Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994): q = (umulhi(n, m) + n) >> s for n < 2^32.
struct FastDiv {
    uint32_t d, m, s;
};

inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d ? d : 1;
    uint32_t s = 0;
    while ((1ull << s) < f.d) s++;
    f.s = s;
    f.m = (uint32_t)((((1ull << s) - f.d) << 32) / f.d + 1);
    if (f.d == 1) f.m = 0;
    return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f)
{
    uint64_t t = (uint64_t)__umulhi(n, f.m) + n;
    return (uint32_t)(t >> f.s);
}

// ---------------------------------------------------------------------------
// Two fused multiply-adds d_i = a_i * b_i + d_i in one instruction for
// binary32 (fma.rn.f32x2 of sm_100: the same two round-to-nearest results as
// two fmaf calls, half the issue slots); binary64 runs two fma calls.
__device__ __forceinline__ void fma2(float& d0, float& d1, float a0, float a1, float b0, float b1)
{
    asm("{\n\t.reg .b64 ra, rb, rc;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%0, %1};\n\t"
        "fma.rn.f32x2 rc, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rc;\n\t}"
        : "+f"(d0), "+f"(d1)
        : "f"(a0), "f"(a1), "f"(b0), "f"(b1));
}

__device__ __forceinline__ void fma2(double& d0, double& d1, double a0, double a1, double b0, double b1)
{
    d0 = fma(a0, b0, d0);
    d1 = fma(a1, b1, d1);
}

// ---------------------------------------------------------------------------
// rounding of operands to the precision's input format
template <typename R>
__device__ __forceinline__ R round_in(R x, int mode)
{
    if (mode == TB_ROUND_F16) return (R)__half2float(__float2half_rn((float)x));
    if (mode == TB_ROUND_BF16) return (R)__bfloat162float(__float2bfloat16_rn((float)x));
    if (mode == TB_ROUND_F32) return (R)(float)x;
    return x;
}

__device__ __forceinline__ float round_in_from_double(double x, int mode)
{
    if (mode == TB_ROUND_F16) return __half2float(__double2half(x));
    if (mode == TB_ROUND_BF16) return __bfloat162float(__double2bfloat16(x));
    return (float)x;
}

// Loads element `off` of a tensor of storage type t as (re, im) in the
// compute real type R. Conversion to R rounds to nearest, as the reference's
// C conversions do (get_val, product.c:10830).
template <typename R>
__device__ __forceinline__ void load_elem(const void* base, int64_t off, int t, R& re, R& im)
{
    switch (t) {
    case T_F32: re = (R)__ldg((const float*)base + off); im = 0; break;
    case T_F64: re = (R)__ldg((const double*)base + off); im = 0; break;
    case T_C32: re = (R)__ldg((const float*)base + 2 * off); im = (R)__ldg((const float*)base + 2 * off + 1); break;
    case T_C64: re = (R)__ldg((const double*)base + 2 * off); im = (R)__ldg((const double*)base + 2 * off + 1); break;
    case T_F16: re = (R)__half2float(((const __half*)base)[off]); im = 0; break;
    case T_BF16: re = (R)__bfloat162float(((const __nv_bfloat16*)base)[off]); im = 0; break;
    default: re = 0; im = 0; break;
    }
}

// Load with rounding to the 16-bit operand format of the precision; from
// binary64 storage the rounding is done in one step.
template <typename R>
__device__ __forceinline__ void load_rounded(const void* base, int64_t off, int t, int mode, R& re, R& im)
{
    if (mode == TB_ROUND_NONE) { load_elem<R>(base, off, t, re, im); return; }
    if (t == T_F64 || t == T_C64) {
        double a, b;
        load_elem<double>(base, off, t, a, b);
        re = (R)round_in_from_double(a, mode);
        im = (R)round_in_from_double(b, mode);
        return;
    }
    load_elem<R>(base, off, t, re, im);
    re = round_in<R>(re, mode);
    im = round_in<R>(im, mode);
}

// Stores (re, im) into element `off` of storage type t (real types keep the
// real part, as C's complex-to-real conversion does).
template <typename R>
__device__ __forceinline__ void store_elem(void* base, int64_t off, int t, R re, R im)
{
    switch (t) {
    case T_F32: ((float*)base)[off] = (float)re; break;
    case T_F64: ((double*)base)[off] = (double)re; break;
    case T_C32: ((float*)base)[2 * off] = (float)re; ((float*)base)[2 * off + 1] = (float)im; break;
    case T_C64: ((double*)base)[2 * off] = (double)re; ((double*)base)[2 * off + 1] = (double)im; break;
    case T_F16: ((__half*)base)[off] = __float2half_rn((float)re); break;
    case T_BF16: ((__nv_bfloat16*)base)[off] = __float2bfloat16_rn((float)re); break;
    default: break;
    }
}

__host__ __device__ inline bool is_complex_type(int t) { return t == T_C32 || t == T_C64; }

}  // namespace tb
