// Tensor-core path for real- and complex-valued products on sm_100a.
//
//   1. k_pack (twice): gathers op_A(A) and op_B(B) from their strided layouts
//      into K-major 16-bit operand panels A''[l][m][k'] and B''[l][n'][k'],
//      summing unary modes, conjugating, and rounding to the precision's
//      operand format on the way (the reference's get_val /
//      sum_unary_contractions, product.c:1863, :10830). Complex operands
//      become real panels (4M form): A'' holds (re, im) pairs along k',
//      B'' holds two rows per n, (re, -im) and (im, re), so one real GEMM
//      yields the real and imaginary parts in adjacent columns. The split
//      mode for binary32 stores three segments along k' — A: hi, hi, lo and
//      B: hi, lo, hi with hi = bf16(x), lo = bf16(x - hi) — so the GEMM sums
//      hi*hi + hi*lo + lo*hi.
//   2. k_gemm: persistent warp-specialised GEMM, one 128x256 output tile per
//      step: warp 0 issues TMA loads (128B-swizzled, 4-stage mbarrier ring),
//      warp 1 issues tcgen05.mma (kind::f16, fp32 accumulators in TMEM,
//      two accumulator buffers), warp 2 owns the TMEM allocation, warps 4-7
//      drain TMEM with tcgen05.ld and apply the fused epilogue
//      D = op_D(alpha * acc + beta * op_C(C)) with D's and C's own strides.
// Every wait on an mbarrier is bounded in time; on expiry the kernel records
// an error word the host reads back, and returns.
#include <cuda.h>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../tb_cuda.h"
#include "tb_common.cuh"
#include "tc_device.cuh"

namespace tb {
int* device_error_word();
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s);
cudaError_t stage_copy(void* dev_dst, const void* src, size_t bytes, cudaStream_t s);

namespace tc {

// ---------------------------------------------------------------------------
// pack
struct PackParams {
    const void* src;
    const void* const* srcs;  // batched product: source of batch b (grid.z = b * Lsz + l), else NULL
    void* dst;
    int32_t type, conj, round_mode, cplx, is_B, split, fmt, rows_fast;
    int64_t R, K, Lsz, Kseg, Kld, Rout;
    ModeList rows, ks, ls, us;  // s0 = stride in the source tensor
    int64_t usize;
};

constexpr int PR = 64, PK = 32;

__device__ __forceinline__ void put16(void* dst, int64_t idx, float v, int fmt)
{
    if (fmt == 1) ((__half*)dst)[idx] = __float2half_rn(v);
    else ((__nv_bfloat16*)dst)[idx] = __float2bfloat16_rn(v);
}

__device__ __forceinline__ float q16(float v, int fmt)
{
    return fmt == 1 ? __half2float(__float2half_rn(v)) : __bfloat162float(__float2bfloat16_rn(v));
}

__global__ void __launch_bounds__(256) k_pack(PackParams p)
{
    // a GEMM launched after this pack as a programmatic dependent may start
    // its set-up once every block of this grid has begun; it reads nothing
    // of the panels before this grid has finished (griddepcontrol.wait)
    asm volatile("griddepcontrol.launch_dependents;");
    __shared__ float vr[PR][PK + 1];
    __shared__ float vi[PR][PK + 1];
    __shared__ int64_t rowOff[PR];
    __shared__ int64_t kOff[PK];
    __shared__ int64_t lOff;
    const int64_t r0 = (int64_t)blockIdx.x * PR, k0 = (int64_t)blockIdx.y * PK, l = blockIdx.z;
    const int64_t lsrc = p.srcs ? l % p.Lsz : l;  // batch mode of the source; l also counts batches
    const void* src = p.srcs ? p.srcs[l / p.Lsz] : p.src;
    const int t = threadIdx.x;
    if (t < PR) {
        int64_t o = 0, dummy;
        if (r0 + t < p.R) decode2(p.rows, r0 + t, o, dummy);
        rowOff[t] = o;
    } else if (t < PR + PK) {
        int64_t o = 0, dummy;
        if (k0 + t - PR < p.K) decode2(p.ks, k0 + t - PR, o, dummy);
        kOff[t - PR] = o;
    } else if (t == PR + PK) {
        int64_t o, dummy;
        decode2(p.ls, lsrc, o, dummy);
        lOff = o;
    }
    __syncthreads();
    // phase 1: gather source values (coalesced along the source's fastest mode)
    for (int e = t; e < PR * PK; e += blockDim.x) {
        int r, kk;
        if (p.rows_fast) { r = e % PR; kk = e / PR; }
        else { kk = e % PK; r = e / PK; }
        float re = 0.f, im = 0.f;
        if (r0 + r < p.R && k0 + kk < p.K) {
            const int64_t off = lOff + rowOff[r] + kOff[kk];
            if (p.us.n == 0) {
                load_rounded<float>(src, off, p.type, p.round_mode, re, im);
                if (p.conj) im = -im;
            } else {
                int64_t c[TB_MAXMODES];
                for (int j = 0; j < p.us.n; j++) c[j] = 0;
                int64_t o = off;
                for (int64_t u = 0; u < p.usize; u++) {
                    float xr, xi;
                    load_elem<float>(src, o, p.type, xr, xi);
                    if (p.conj) xi = -xi;
                    re += xr;
                    im += xi;
                    if (p.round_mode != TB_ROUND_NONE) {
                        re = round_in<float>(re, p.round_mode);
                        im = round_in<float>(im, p.round_mode);
                    }
                    for (int j = 0; j < p.us.n; j++) {
                        o += p.us.s0[j];
                        if (++c[j] < p.us.ext[j]) break;
                        o -= p.us.s0[j] * p.us.ext[j];
                        c[j] = 0;
                    }
                }
            }
        }
        vr[r][kk] = re;
        vi[r][kk] = im;
    }
    __syncthreads();
    // phase 2: write K-major 16-bit panels, two elements per store
    const int rmul = (p.cplx && p.is_B) ? 2 : 1;
    const int cmul = p.cplx ? 2 : 1;
    const int ocols = PK * cmul;           // output columns of this tile per segment
    const int orows = PR * rmul;
    for (int e = t; e < orows * (ocols / 2) * p.split; e += blockDim.x) {
        const int cp = e % (ocols / 2);
        const int rest = e / (ocols / 2);
        const int ro = rest % orows;
        const int seg = rest / orows;
        const int r = ro / rmul, variant = ro % rmul;
        const int64_t rg = r0 + r;
        if (rg >= p.R) continue;
        const int64_t col = k0 * cmul + 2 * cp;  // output column of the first element
        if (col >= p.Kseg) continue;
        float v[2];
        for (int h = 0; h < 2; h++) {
            const int oc = 2 * cp + h;                // column inside the tile
            float x;
            if (!p.cplx) {
                x = vr[r][oc];
            } else {
                const int kk = oc >> 1, part = oc & 1;
                const float a = vr[r][kk], b = vi[r][kk];
                if (!p.is_B) x = part ? b : a;                 // (re, im)
                else if (variant == 0) x = part ? -b : a;      // row for the real output
                else x = part ? a : b;                         // row for the imaginary output
            }
            if (p.split == 3) {
                const float hi = q16(x, 0);
                const float lo = x - hi;
                // A: hi, hi, lo   B: hi, lo, hi
                const bool use_lo = p.is_B ? (seg == 1) : (seg == 2);
                x = use_lo ? lo : hi;
            }
            v[h] = x;
        }
        const int64_t base = ((int64_t)l * p.Rout + rg * rmul + variant) * p.Kld + seg * p.Kseg + col;
        if (col + 1 < p.Kseg) {
            if (p.fmt == 1) *(__half2*)((__half*)p.dst + base) = __floats2half2_rn(v[0], v[1]);
            else *(__nv_bfloat162*)((__nv_bfloat16*)p.dst + base) = __floats2bfloat162_rn(v[0], v[1]);
        } else {
            put16(p.dst, base, v[0], p.fmt);
        }
    }
}

// Fast pack for the common case: real operands, no unary modes. A 64x64
// (rows x k) tile per block; 16 independent loads per thread in flight, then
// 16-byte stores of eight 16-bit values along k.
constexpr int FR = 64, FK = 64;

template <typename T>
__device__ __forceinline__ float load_as_float(const void* base, int64_t off)
{
    return (float)__ldg((const T*)base + off);
}
template <>
__device__ __forceinline__ float load_as_float<__half>(const void* base, int64_t off)
{
    return __half2float(((const __half*)base)[off]);
}
template <>
__device__ __forceinline__ float load_as_float<__nv_bfloat16>(const void* base, int64_t off)
{
    return __bfloat162float(((const __nv_bfloat16*)base)[off]);
}

// ROWS_FAST: the source is contiguous along the first row (M or N) mode, else
// along the first contracted mode. VEC = 4: that mode has stride 1, an extent
// divisible by 4 and every other stride (and the base) keeps 16-byte
// alignment, so four neighbours come in one 16-byte load.
template <typename T, int SPLIT, int FMT, bool ROWS_FAST, int VEC>
__global__ void __launch_bounds__(256, 4) k_pack_real(PackParams p)
{
    // a GEMM launched after this pack as a programmatic dependent may start
    // its set-up once every block of this grid has begun; it reads nothing
    // of the panels before this grid has finished (griddepcontrol.wait)
    asm volatile("griddepcontrol.launch_dependents;");
    __shared__ float v[FR][FK + 1];
    __shared__ int64_t rowOff[FR];
    __shared__ int64_t kOff[FK];
    __shared__ int64_t lOff;
    const int64_t r0 = (int64_t)blockIdx.x * FR, k0 = (int64_t)blockIdx.y * FK, l = blockIdx.z;
    const int64_t lsrc = p.srcs ? l % p.Lsz : l;  // batch mode of the source; l also counts batches
    const void* src = p.srcs ? p.srcs[l / p.Lsz] : p.src;
    const int t = threadIdx.x;
    if (t < FR) {
        int64_t o = 0, dummy;
        if (r0 + t < p.R) decode2(p.rows, r0 + t, o, dummy);
        rowOff[t] = o;
    } else if (t < FR + FK) {
        int64_t o = 0, dummy;
        if (k0 + t - FR < p.K) decode2(p.ks, k0 + t - FR, o, dummy);
        kOff[t - FR] = o;
    } else if (t == FR + FK) {
        int64_t o, dummy;
        decode2(p.ls, lsrc, o, dummy);
        lOff = o;
    }
    __syncthreads();
    constexpr int NV = FR * FK / 256 / VEC;  // vector loads per thread
    constexpr int G = (ROWS_FAST ? FR : FK) / VEC;  // vectors along the fast direction
    float x[NV][VEC];
#pragma unroll
    for (int u = 0; u < NV; u++) {
        const int e = t + 256 * u;
        const int fg = e % G, sl = e / G;              // fast-direction group, slow index
        const int r = ROWS_FAST ? fg * VEC : sl;
        const int kk = ROWS_FAST ? sl : fg * VEC;
        const bool in = (r0 + r < p.R) && (k0 + kk < p.K);
        const int64_t off = lOff + rowOff[r] + kOff[kk];
        if (VEC == 4) {
            float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in) q = __ldg((const float4*)((const float*)src + off));
            x[u][0] = q.x; x[u][VEC > 1 ? 1 : 0] = q.y; x[u][VEC > 2 ? 2 : 0] = q.z; x[u][VEC > 3 ? 3 : 0] = q.w;
        } else {
            x[u][0] = in ? load_as_float<T>(src, off) : 0.f;
        }
    }
#pragma unroll
    for (int u = 0; u < NV; u++) {
        const int e = t + 256 * u;
        const int fg = e % G, sl = e / G;
#pragma unroll
        for (int h = 0; h < VEC; h++) {
            const int r = ROWS_FAST ? fg * VEC + h : sl;
            const int kk = ROWS_FAST ? sl : fg * VEC + h;
            float y = x[u][h];
            if (SPLIT == 1 && p.round_mode != TB_ROUND_NONE) y = round_in<float>(y, p.round_mode);
            v[r][kk] = y;
        }
    }
    __syncthreads();
    // FR rows x FK/8 groups of eight per segment
    for (int item = t; item < FR * (FK / 8) * SPLIT; item += 256) {
        const int g = item % (FK / 8);
        const int r = (item / (FK / 8)) % FR;
        const int seg = item / (FR * (FK / 8));
        const int64_t rg = r0 + r;
        const int64_t col = k0 + g * 8;
        if (rg >= p.R || col >= p.Kseg) continue;
        uint32_t w[4];
#pragma unroll
        for (int h = 0; h < 4; h++) {
            float a = v[r][g * 8 + 2 * h], b = v[r][g * 8 + 2 * h + 1];
            if (SPLIT >= 2) {
                const float ah = __bfloat162float(__float2bfloat16_rn(a));
                const float bh = __bfloat162float(__float2bfloat16_rn(b));
                // three segments: A hi, hi, lo and B hi, lo, hi; two: [hi | lo] for both
                const bool use_lo = SPLIT == 2 ? seg == 1 : p.is_B ? (seg == 1) : (seg == 2);
                if (use_lo) { a -= ah; b -= bh; } else { a = ah; b = bh; }
            }
            if (FMT == 1) {
                __half2 q = __floats2half2_rn(a, b);
                w[h] = *(uint32_t*)&q;
            } else {
                __nv_bfloat162 q = __floats2bfloat162_rn(a, b);
                w[h] = *(uint32_t*)&q;
            }
        }
        const int64_t idx = ((int64_t)l * p.Rout + rg) * p.Kld + seg * p.Kseg + col;
        *(uint4*)((uint16_t*)p.dst + idx) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    // launched as a programmatic dependent of the pack before it (the first
    // operand's), this grid ends only after that one has: whoever waits for
    // this grid's completion then has both operands' panels
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Pipelined pack for binary32 sources contiguous along the contraction and
// read 16 bytes at a time (the VEC = 4, K-fast case above: the first
// contracted mode has stride 1 and an extent divisible by 4, every other
// stride keeps 16-byte alignment). Persistent blocks of 128 threads walk the
// 64 x 64 tiles (block b: tiles b, b + grid, ...) and copy each tile into a
// ring of PP_STAGES shared-memory slots with cp.async, PP_STAGES - 1 tiles
// ahead of the one being written out, so a block keeps ~48 KiB of loads in
// flight without holding them in registers (the one-tile kernel above has one
// load phase and one store phase per block). Slot layout [r][k], 68 floats
// per row, read without bank conflicts: thread (r, g) reads k = 8g..8g+7 as
// two 16-byte reads, lanes 4-7 of each quarter-warp reading their second half
// first. Output words and their order are those of k_pack_real (same
// rounding, same [hi | lo] or three-segment split), so the two kernels write
// identical panels. On the 64^4 contraction's B operand: 23.2 us against
// 26.9 us for k_pack_real; for sources contiguous along the rows the
// transposed reads made it slower than k_pack_real (41.8 against 28.0 us),
// so those keep k_pack_real.
constexpr int PP_THREADS = 128, PP_STAGES = 4, PP_PITCH = 68;
constexpr int PP_SLOT = 64 * PP_PITCH;  // floats per slot
struct PackTab {
    int64_t row[64];
    int64_t k[64];
    const float* src;  // the tile's batch base
    int64_t pad;
};
constexpr int PP_SMEM = PP_STAGES * PP_SLOT * 4 + 2 * (int)sizeof(PackTab);

// multiply-high divisors of the pipelined pack's index arithmetic (every
// extent, row count, contraction length and tile count below 2^31)
struct PackDivs {
    FastDiv rows[TB_MAXMODES], ks[TB_MAXMODES], ls[TB_MAXMODES];
    FastDiv tiles_k, tiles_r, lsz;
};

__device__ __forceinline__ int64_t pp_decode(const ModeList& m, const FastDiv* f, uint32_t idx)
{
    int64_t o = 0;
    for (int j = 0; j < m.n; j++) {
        const uint32_t q = fdiv(idx, f[j]);
        o += (int64_t)(idx - q * f[j].d) * m.s0[j];
        idx = q;
    }
    return o;
}

__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void* src, bool in)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void pp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void pp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// eight values of row rg at columns col..col+7, every segment, as k_pack_real writes them
template <int SPLIT, int FMT>
__device__ __forceinline__ void pp_put8(const PackParams& p, int64_t l, int64_t rg, int64_t col, const float (&x)[8])
{
#pragma unroll
    for (int seg = 0; seg < SPLIT; seg++) {
        uint32_t w[4];
#pragma unroll
        for (int h = 0; h < 4; h++) {
            float a = x[2 * h], b = x[2 * h + 1];
            if (SPLIT == 1 && p.round_mode != TB_ROUND_NONE) {
                a = round_in<float>(a, p.round_mode);
                b = round_in<float>(b, p.round_mode);
            }
            if (SPLIT >= 2) {
                const float ah = __bfloat162float(__float2bfloat16_rn(a));
                const float bh = __bfloat162float(__float2bfloat16_rn(b));
                const bool use_lo = SPLIT == 2 ? seg == 1 : p.is_B ? (seg == 1) : (seg == 2);
                if (use_lo) { a -= ah; b -= bh; } else { a = ah; b = bh; }
            }
            if (FMT == 1) {
                __half2 q = __floats2half2_rn(a, b);
                w[h] = *(uint32_t*)&q;
            } else {
                __nv_bfloat162 q = __floats2bfloat162_rn(a, b);
                w[h] = *(uint32_t*)&q;
            }
        }
        const int64_t idx = ((int64_t)l * p.Rout + rg) * p.Kld + seg * p.Kseg + col;
        *(uint4*)((uint16_t*)p.dst + idx) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

template <int SPLIT, int FMT>
__global__ void __launch_bounds__(PP_THREADS) k_pack_pipe(PackParams p, PackDivs dv, int32_t ntiles)
{
    // a GEMM launched after this pack as a programmatic dependent may start
    // its set-up once every block of this grid has begun; it reads nothing
    // of the panels before this grid has finished (griddepcontrol.wait)
    asm volatile("griddepcontrol.launch_dependents;");
    extern __shared__ __align__(16) float pp_sm[];
    float* slots = pp_sm;
    PackTab* tab = (PackTab*)(pp_sm + PP_STAGES * PP_SLOT);
    const int t = threadIdx.x;
    const int32_t first = blockIdx.x, step = gridDim.x;
    const int32_t nloc = first < ntiles ? (ntiles - 1 - first) / step + 1 : 0;
    auto tile_of = [&](int32_t i, int64_t& r0, int64_t& k0, int64_t& l) {
        const uint32_t j = (uint32_t)(first + i * step);
        const uint32_t jk = fdiv(j, dv.tiles_k), jr = fdiv(jk, dv.tiles_r);
        k0 = (int64_t)(j - jk * dv.tiles_k.d) * 64;
        r0 = (int64_t)(jk - jr * dv.tiles_r.d) * 64;
        l = jr;
    };
    // source offsets of tile i's 64 rows (threads 0-63) and 64 columns (64-127)
    auto make_tab = [&](int32_t i, PackTab& tb) {
        if (i >= nloc) return;
        int64_t r0, k0, l, o = 0;
        tile_of(i, r0, k0, l);
        if (t < 64) {
            if (r0 + t < p.R) o = pp_decode(p.rows, dv.rows, (uint32_t)(r0 + t));
            tb.row[t] = o;
        } else {
            const int kk = t - 64;
            if (k0 + kk < p.K) o = pp_decode(p.ks, dv.ks, (uint32_t)(k0 + kk));
            tb.k[kk] = o;
        }
        if (t == 0) {
            const uint32_t b = p.srcs ? fdiv((uint32_t)l, dv.lsz) : 0u;
            const uint32_t lsrc = (uint32_t)l - b * dv.lsz.d;
            o = pp_decode(p.ls, dv.ls, p.srcs ? lsrc : (uint32_t)l);
            tb.src = (const float*)(p.srcs ? p.srcs[b] : p.src) + o;
        }
    };
    // 1024 chunks of 16 bytes per tile, 8 per thread; outside the tensor: zeros
    auto issue = [&](int32_t i, const PackTab& tb) {
        if (i < nloc) {
            int64_t r0, k0, l;
            tile_of(i, r0, k0, l);
            const uint32_t sb = smem_u32(slots + (i % PP_STAGES) * PP_SLOT);
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int c = t + PP_THREADS * u;
                const int r = c / 16, kk = (c % 16) * 4;
                const uint32_t dst = sb + (uint32_t)(r * PP_PITCH + kk) * 4u;
                const bool in = r0 + r < p.R && k0 + kk < p.K;
                cp_async16_zfill(dst, in ? (const void*)(tb.src + tb.row[r] + tb.k[kk]) : (const void*)tb.src, in);
            }
        }
        pp_commit();  // empty groups keep the count uniform
    };
    auto store = [&](int32_t i) {
        int64_t r0, k0, l;
        tile_of(i, r0, k0, l);
        const float* v = slots + (i % PP_STAGES) * PP_SLOT;
#pragma unroll
        for (int it = 0; it < 4; it++) {
            const int e = t + PP_THREADS * it;
            const int g = e % 8, r = e / 8;
            const int64_t rg = r0 + r, col = k0 + g * 8;
            if (rg >= p.R || col >= p.Kseg) continue;
            const int h0 = (g >> 2) & 1;
            const float4 a = *(const float4*)(v + r * PP_PITCH + g * 8 + 4 * h0);
            const float4 b = *(const float4*)(v + r * PP_PITCH + g * 8 + 4 * (1 - h0));
            const float4 lo4 = h0 ? b : a, hi4 = h0 ? a : b;
            const float x[8] = {lo4.x, lo4.y, lo4.z, lo4.w, hi4.x, hi4.y, hi4.z, hi4.w};
            pp_put8<SPLIT, FMT>(p, l, rg, col, x);
        }
    };
    for (int i = 0; i < PP_STAGES - 1; i++) {
        make_tab(i, tab[i & 1]);
        __syncthreads();
        issue(i, tab[i & 1]);
    }
    make_tab(PP_STAGES - 1, tab[(PP_STAGES - 1) & 1]);
    for (int32_t i = 0; i < nloc; i++) {
        pp_wait<PP_STAGES - 2>();  // this thread's copies of tile i have landed
        __syncthreads();           // everyone's have; slot (i - 1) and table (i + S) are free
        issue(i + PP_STAGES - 1, tab[(i + PP_STAGES - 1) & 1]);
        make_tab(i + PP_STAGES, tab[(i + PP_STAGES) & 1]);
        store(i);
    }
    pp_wait<0>();
    // launched as a programmatic dependent of the pack before it (the first
    // operand's), this grid ends only after that one has: whoever waits for
    // this grid's completion then has both operands' panels
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

static int num_sms();

// Launches a pack kernel; pdl: as a programmatic dependent of the pack just
// before it in the stream (the other operand's, same product), so that its
// blocks start while that pack's last blocks drain. The packs read only the
// product's operands, which the stream work before the first pack produced.
template <typename K, typename... Args>
static void launch_pack_kernel(K kern, dim3 grid, unsigned threads, size_t smem, cudaStream_t s, bool pdl,
                               Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    (void)cudaLaunchKernelEx(&cfg, kern, args...);
}

// false: the kernel could not be given its shared memory (the caller runs k_pack_real)
template <int SPLIT, int FMT>
static bool launch_pack_pipe(const PackParams& pp, int64_t lz, cudaStream_t s, bool pdl)
{
    auto kern = k_pack_pipe<SPLIT, FMT>;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev]) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, PP_SMEM) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        if (dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    const int64_t tiles_r = (pp.R + 63) / 64, tiles_k = (pp.Kseg + 63) / 64;
    const int64_t ntiles = tiles_r * tiles_k * lz;
    const int64_t grid = std::min<int64_t>(ntiles, (int64_t)num_sms() * 3);
    PackDivs dv;
    memset(&dv, 0, sizeof(dv));
    for (int j = 0; j < pp.rows.n; j++) dv.rows[j] = make_fastdiv((uint32_t)pp.rows.ext[j]);
    for (int j = 0; j < pp.ks.n; j++) dv.ks[j] = make_fastdiv((uint32_t)pp.ks.ext[j]);
    for (int j = 0; j < pp.ls.n; j++) dv.ls[j] = make_fastdiv((uint32_t)pp.ls.ext[j]);
    dv.tiles_k = make_fastdiv((uint32_t)tiles_k);
    dv.tiles_r = make_fastdiv((uint32_t)tiles_r);
    dv.lsz = make_fastdiv((uint32_t)std::max<int64_t>(pp.Lsz, 1));
    if (grid > 0) launch_pack_kernel(kern, dim3((unsigned)grid), PP_THREADS, PP_SMEM, s, pdl, pp, dv, (int32_t)ntiles);
    return true;
}

// the pipelined pack's 32-bit index arithmetic covers the operand
static bool pack_pipe_fits(const PackParams& pp, int64_t lz)
{
    const int64_t lim = (int64_t)1 << 31;
    const int64_t ntiles = ((pp.R + 63) / 64) * ((pp.Kseg + 63) / 64) * lz;
    if (pp.R >= lim || pp.Kseg >= lim || pp.K >= lim || lz >= lim || ntiles >= lim) return false;
    const ModeList* ms[3] = {&pp.rows, &pp.ks, &pp.ls};
    for (const ModeList* m : ms)
        for (int j = 0; j < m->n; j++)
            if (m->ext[j] < 1 || m->ext[j] >= lim) return false;
    return !pp.srcs || pp.Lsz >= 1;
}

static bool launch_pack_pipe3(const PackParams& pp, int split, int fmt, int64_t lz, cudaStream_t s, bool pdl)
{
    if (split == 3) return launch_pack_pipe<3, 0>(pp, lz, s, pdl);
    if (split == 2) return launch_pack_pipe<2, 0>(pp, lz, s, pdl);
    if (fmt == 1) return launch_pack_pipe<1, 1>(pp, lz, s, pdl);
    return launch_pack_pipe<1, 0>(pp, lz, s, pdl);
}

template <typename T, bool RF, int VEC>
static void launch_pack_real3(const PackParams& pp, int split, int fmt, dim3 grid, cudaStream_t s, bool pdl)
{
    if (split == 3) launch_pack_kernel(k_pack_real<T, 3, 0, RF, VEC>, grid, 256, 0, s, pdl, pp);
    else if (split == 2) launch_pack_kernel(k_pack_real<T, 2, 0, RF, VEC>, grid, 256, 0, s, pdl, pp);
    else if (fmt == 1) launch_pack_kernel(k_pack_real<T, 1, 1, RF, VEC>, grid, 256, 0, s, pdl, pp);
    else launch_pack_kernel(k_pack_real<T, 1, 0, RF, VEC>, grid, 256, 0, s, pdl, pp);
}

// whether a mode list's first mode has stride 1 and extent % 4 == 0 and all
// other strides of `others` keep 4-element alignment
static bool vec4_ok(const ModeList& fast, const ModeList* others[], int nothers, const void* base)
{
    if (fast.n < 1 || fast.s0[0] != 1 || fast.ext[0] % 4 != 0 || ((uintptr_t)base & 15) != 0) return false;
    for (int j = 1; j < fast.n; j++)
        if (fast.s0[j] % 4 != 0) return false;
    for (int i = 0; i < nothers; i++)
        for (int j = 0; j < others[i]->n; j++)
            if (others[i]->s0[j] % 4 != 0) return false;
    return true;
}

// grid.z = lz panel batches (the batch modes, times the batches of a batched
// product); aligned: every source base of a batched product is 16-byte aligned
template <typename T>
static void launch_pack_real(const PackParams& pp, int split, int fmt, int64_t lz, bool aligned, cudaStream_t s,
                             bool pdl = false)
{
    dim3 grid((unsigned)((pp.R + FR - 1) / FR), (unsigned)((pp.Kseg + FK - 1) / FK), (unsigned)lz);
    const bool rf = pp.rows_fast != 0;
    bool v4 = false;
    if (sizeof(T) == 4 && aligned) {
        const ModeList* others[3] = {rf ? &pp.ks : &pp.rows, &pp.ls, &pp.us};
        v4 = vec4_ok(rf ? pp.rows : pp.ks, others, 2, pp.src);
    }
    if (v4 && !rf && pack_pipe_fits(pp, lz) && launch_pack_pipe3(pp, split, fmt, lz, s, pdl)) return;
    if (rf) {
        if (v4) launch_pack_real3<T, true, 4>(pp, split, fmt, grid, s, pdl);
        else launch_pack_real3<T, true, 1>(pp, split, fmt, grid, s, pdl);
    } else {
        if (v4) launch_pack_real3<T, false, 4>(pp, split, fmt, grid, s, pdl);
        else launch_pack_real3<T, false, 1>(pp, split, fmt, grid, s, pdl);
    }
}

// Self-test of the bounded waits: one thread waits, with the kernels' own
// flag_wait and mbar_wait, on a flag that nothing raises and on the first
// phase of an mbarrier that nothing completes, limit_ns each. Both must give
// up and raise the abort word; out = {flag wait returned, abort word after
// it, barrier wait returned, abort word after it}.
__global__ void k_wait_selftest(const int* flag, int* out, unsigned long long limit_ns)
{
    __shared__ uint64_t bar;
    __shared__ int abort_word;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_word = 0;
    out[0] = flag_wait(flag, &abort_word, limit_ns) ? 1 : 0;
    out[1] = abort_word;
    abort_word = 0;
    out[2] = mbar_wait(&bar, 0, &abort_word, limit_ns) ? 1 : 0;
    out[3] = abort_word;
}

// CVT: the split-bfloat16 product of binary32 operands read in place by
// eight converter warps (warps 8-15, 512 threads) instead of TMA loads of
// packed panels; stages of 64 KiB (A hi, A lo, B hi, B lo), three MMAs per
// 16-deep step (hi*hi, hi*lo, lo*hi), four epilogue warps (4-7).
// LOAD = 2: the split-bfloat16 product from packed panels that hold each
// operand's hi and lo parts side by side ([hi | lo] along k): TMA brings A hi,
// A lo, B hi, B lo of one 64-deep block into a 64 KiB stage and the same
// three MMAs run on it (4 bytes of panel per element instead of the 6 of
// three-segment panels).
template <int EPI, bool CTA2, int LOAD = 0>
__global__ void __launch_bounds__(LOAD == 1 ? 512 : NTHREADS, 1)
    k_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmParams p,
           uint32_t idesc, const __grid_constant__ CUtensorMap tmC, const __grid_constant__ CUtensorMap tmD)
{
    using G = Geo<CTA2>;
    constexpr bool CVT = LOAD == 1, SPL = LOAD == 2, TRI = LOAD != 0;  // TRI: three MMAs per step
    constexpr int NS = TRI ? 3 : G::stages;
    constexpr int SB = TRI ? 4 * BM * BK * 2 : G::stage_bytes;  // bytes per stage
    constexpr int EW = CVT ? 4 : EPI_WARPS;                      // epilogue warps
    constexpr int ET = EW * 32;
    constexpr int CS = EW / 4;  // a warp's chunk step: the warps of a lane quarter interleave
    static_assert(!TRI || (CTA2 && NS * SB <= STAGES * STAGE_BYTES), "split stages fit the ring");
    auto epi_bar = [] { epi_bar_n<ET>(); };
    constexpr int KSTEP = EPI == EPI_I32 ? 2 * BK : BK;  // elements per 128-byte stage row
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // 1024-byte alignment by pointer arithmetic on the shared array (an
    // integer round trip would turn every access below into a generic one)
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* tiles = smem;
    uint8_t* bars = smem + STAGES * STAGE_BYTES;  // 256 bytes of barriers and flags
    uint64_t* full = (uint64_t*)bars;             // up to 6
    uint64_t* empty = (uint64_t*)(bars + 48);     // up to 6
    uint64_t* tfull = (uint64_t*)(bars + 96);
    uint64_t* tempty = (uint64_t*)(bars + 112);
    uint64_t* cbar = (uint64_t*)(bars + 128);     // one per epilogue warp
    uint32_t* tmem_slot = (uint32_t*)(bars + 192);
    volatile int* abort_flag = (volatile int*)(bars + 196);
    volatile int* epi_ok = (volatile int*)(bars + 200);
    volatile int* epi_first = (volatile int*)(bars + 204);
    uint8_t* staging = smem + STAGES * STAGE_BYTES + 256;
    int64_t* colC = (int64_t*)staging;
    int64_t* colD = colC + BN;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = CTA2 ? cluster_rank() : 0;  // 0 = the pair's leader, which issues the MMAs
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; s++) {
            // CVT: one arrival per converter warp (of both CTAs of a pair)
            mbar_init(&full[s], CVT ? (CTA2 ? 16 : 8) : 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&tfull[a], 1);
            // one CTA: every epilogue thread arrives; pair: one arrival per
            // epilogue warp of either CTA, on the leader's barrier
            mbar_init(&tempty[a], CTA2 ? 2 * EW : ET);
        }
        for (int w = 0; w < EW; w++) mbar_init(&cbar[w], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        if (CTA2) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                         "r"(TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
    }
    fence_before();
    if (CTA2) cluster_sync();  // barriers of both CTAs initialised before any remote signal
    else __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_slot;
    // launched as a programmatic dependent of the operand pack: everything
    // above touched only shared and tensor memory; wait for the pack's grid
    // (and its writes) before any global access (a no-op otherwise)
    asm volatile("griddepcontrol.wait;" ::: "memory");

    // tiles: one CTA walks 128x256 tiles; a pair walks 256x256 tiles together
    const int unit = CTA2 ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int units = CTA2 ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    const int num_items = p.num_tiles + p.split_tiles;
    const int my_tiles = num_items > unit ? (num_items - 1 - unit) / units + 1 : 0;

    // in-place operands take up to six 8 KB boxes a stage: warp 0 issues A's
    // (and the stage's expected bytes), warp 3 B's, so the two issue streams
    // overlap; a box that lands before the expectation only drives the
    // barrier's transaction count below zero for a moment
    const bool two_producers = p.a_direct || p.b_direct;
    if (!CVT && (warp == 0 || (warp == 3 && two_producers))) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            const bool do_a = warp == 0, do_b = warp == 3 || !two_producers;
            uint32_t g = 0;
            int64_t last_issued[NS];
            for (int s = 0; s < NS; s++) last_issued[s] = -1;
            bool ok = true;
            for (int i = 0; i < my_tiles && ok; i++) {
                const Item it = item_of(p, unit + i * units);
                const int tile = it.tile;
                const int tm = tile % p.tiles_m;
                const int rest = tile / p.tiles_m;
                const int tn = rest % p.tiles_n;
                const int l = rest / p.tiles_n;
                // in-place operands: row coordinates of this tile's 64-row
                // chunks (fixed for the tile) and the contraction coordinate
                // stepped by 64 per block (no divisions in the loop below)
                const int arow = tm * G::tile_m + (int)rank * BM, brow = tn * BN + (int)rank * G::b_rows;
                int ar0[2] = {0, 0}, ar1[2] = {0, 0}, br0[4] = {0, 0, 0, 0}, br1[4] = {0, 0, 0, 0};
                int akc0 = 0, akc1 = 0, bkc0 = 0, bkc1 = 0;
                if (p.a_direct && do_a) {
#pragma unroll
                    for (int c = 0; c < 2; c++) {
                        ar0[c] = (arow + 64 * c) % p.a_e0;
                        ar1[c] = (arow + 64 * c) / p.a_e0;
                    }
                    akc0 = (it.kb0 * BK) % p.a_k0;
                    akc1 = (it.kb0 * BK) / p.a_k0;
                }
                if (p.b_direct && do_b) {
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        br0[c] = (brow + 64 * c) % p.b_e0;
                        br1[c] = (brow + 64 * c) / p.b_e0;
                    }
                    bkc0 = (it.kb0 * BK) % p.b_k0;
                    bkc1 = (it.kb0 * BK) / p.b_k0;
                }
                for (int kb = it.kb0; kb < it.kb1; kb++, g++) {
                    const int s = g % NS;
                    const uint32_t ph = (g / NS) & 1;
                    if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                    uint8_t* a = tiles + s * SB;
                    // one chunk of an in-place operand: logical coordinates
                    // (row0, k0, row1, k1, batch) or (k0, row0, k1, row1,
                    // batch), then those of the dims the map keeps
                    auto chunk = [&](uint8_t* dst, const CUtensorMap* tm_, int rc0, int rc1, int kc0, int kc1, int mn,
                                     int dims, uint32_t fb) {
                        const int c0 = mn ? rc0 : kc0, c1 = mn ? kc0 : rc0, c2 = mn ? rc1 : kc1, c3 = mn ? kc1 : rc1;
                        int q[5] = {c0, c1, 0, 0, 0};
                        int n = 2;
                        if (dims & 4) { q[2] = c2; n = 3; }
                        if (dims & 8) {
                            if (n == 2) q[2] = c3; else q[3] = c3;
                            n++;
                        }
                        if (dims & 16) {
                            if (n == 2) q[2] = l; else if (n == 3) q[3] = l; else q[4] = l;
                            n++;
                        }
                        if (n <= 3) {
                            if (CTA2) tma_load_3d_pair(dst, tm_, fb, q[0], q[1], q[2]);
                            else tma_load_3d(dst, tm_, &full[s], q[0], q[1], q[2]);
                        } else if (n == 4) {
                            if (CTA2) tma_load_4d_pair(dst, tm_, fb, q);
                            else tma_load_4d(dst, tm_, &full[s], q);
                        } else {
                            if (CTA2) tma_load_5d_pair(dst, tm_, fb, q);
                            else tma_load_5d(dst, tm_, &full[s], q);
                        }
                    };
                    const uint32_t fb = CTA2 ? cluster_addr(&full[s], 0) : 0;
                    if (!do_a) {
                    } else if (CTA2) {
                        // both halves land on the leader's barrier, which expects the pair's bytes
                        if (rank == 0) mbar_expect_tx(&full[s], 2 * SB);
                    } else {
                        mbar_expect_tx(&full[s], G::stage_bytes);
                    }
                    if (SPL) {
                        // A hi, A lo, B hi, B lo of block kb (lo at k offset lo_off)
                        tma_load_3d_pair(a, &tmA, fb, kb * BK, arow, l);
                        tma_load_3d_pair(a + 16384, &tmA, fb, p.lo_off + kb * BK, arow, l);
                        tma_load_3d_pair(a + 32768, &tmB, fb, kb * BK, brow, l);
                        tma_load_3d_pair(a + 49152, &tmB, fb, p.lo_off + kb * BK, brow, l);
                    } else if (!do_a) {
                    } else if (p.a_direct) {
                        const int nc = p.a_box ? 1 : BM / 64;
#pragma unroll
                        for (int c = 0; c < 2; c++)
                            if (c < nc) chunk(a + c * 8192, &tmA, ar0[c], ar1[c], akc0, akc1, p.a_mn, p.a_dims, fb);
                        if ((akc0 += BK) == p.a_k0) { akc0 = 0; akc1++; }
                    } else if (CTA2) {
                        tma_load_3d_pair(a, &tmA, fb, kb * KSTEP, arow, l);
                    } else {
                        tma_load_3d(a, &tmA, &full[s], kb * KSTEP, tm * BM, l);
                    }
                    if (SPL || !do_b) {
                    } else if (p.b_direct) {
                        const int nc = p.b_box ? 1 : G::b_rows / 64;
#pragma unroll
                        for (int c = 0; c < 4; c++)
                            if (c < nc)
                                chunk(a + G::a_bytes + c * 8192, &tmB, br0[c], br1[c], bkc0, bkc1, p.b_mn, p.b_dims, fb);
                        if ((bkc0 += BK) == p.b_k0) { bkc0 = 0; bkc1++; }
                    } else if (CTA2) {
                        tma_load_3d_pair(a + G::a_bytes, &tmB, fb, kb * KSTEP, brow, l);
                    } else {
                        tma_load_3d(a + G::a_bytes, &tmB, &full[s], kb * KSTEP, tn * BN, l);
                    }
                    last_issued[s] = g;
                }
            }
            if (!do_a) {
                // warp 0 drains the stages: a phase completes only when the
                // boxes of both producers have landed
                if (CTA2 && rank != 0 && !ok) {
                    const unsigned long long t0 = now_ns();
                    while (now_ns() - t0 < 200000ull) {
                    }
                }
            } else if (!CTA2 || rank == 0) {
                // every issued load must land before the block exits: the phase of
                // the last load issued on a stage stays complete once reached
                int never = 0;
                for (int s = 0; s < NS; s++)
                    if (last_issued[s] >= 0)
                        mbar_wait(&full[s], (uint32_t)(last_issued[s] / NS) & 1, (volatile int*)&never);
            } else if (!ok) {
                // the second CTA's loads signal the leader: after an expired wait,
                // give loads in flight time to land before this CTA exits
                const unsigned long long t0 = now_ns();
                while (now_ns() - t0 < 200000ull) {
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer (the leader of a pair) ----------------
        if (lane == 0 && (!CTA2 || rank == 0)) {
            uint32_t g = 0;
            bool ok = true;
            for (int i = 0; i < my_tiles && ok; i++) {
                const int acc = i & 1;
                const uint32_t aph = (i >> 1) & 1;
                if (!mbar_wait(&tempty[acc], aph ^ 1, abort_flag)) break;
                fence_after();
                const uint32_t d_tmem = tmem_base + acc * BN;
                const Item it = item_of(p, unit + i * units);
                for (int kb = it.kb0; kb < it.kb1; kb++, g++) {
                    const int kr = kb - it.kb0;  // accumulate from the item's second block on
                    const int s = g % NS;
                    const uint32_t ph = (g / NS) & 1;
                    if (!mbar_wait<CVT && CTA2>(&full[s], ph, abort_flag)) { ok = false; break; }
                    fence_after();
                    const uint32_t a = smem_u32(tiles + s * SB);
                    const uint32_t b = a + G::a_bytes;
#pragma unroll
                    for (int k = 0; k < BK / 16; k++) {  // 32 bytes of K per instruction
                        if (TRI) {
                            // A hi, A lo, B hi, B lo tiles of 16 KiB: hi*hi + hi*lo + lo*hi
                            auto desc = [&](uint32_t t, int mn) {
                                return mn ? smem_desc_mn(t + k * 2048) : smem_desc(t + k * 32);
                            };
                            const uint64_t ah = desc(a, p.a_mn), al = desc(a + 16384, p.a_mn);
                            const uint64_t bh = desc(a + 32768, p.b_mn), bl = desc(a + 49152, p.b_mn);
                            mma_f16_pair(d_tmem, ah, bh, idesc, (kr | k) != 0);
                            mma_f16_pair(d_tmem, ah, bl, idesc, 1);
                            mma_f16_pair(d_tmem, al, bh, idesc, 1);
                        } else if (EPI != EPI_I32 && (p.a_mn | p.b_mn)) {
                            // an MN-major operand advances 16 k-rows (2048 bytes) per instruction
                            const uint64_t da = p.a_mn ? smem_desc_mn(a + k * 2048) : smem_desc(a + k * 32);
                            const uint64_t db = p.b_mn ? smem_desc_mn(b + k * 2048) : smem_desc(b + k * 32);
                            if (CTA2) mma_f16_pair(d_tmem, da, db, idesc, (kr | k) != 0);
                            else mma_f16(d_tmem, da, db, idesc, (kr | k) != 0);
                        } else if (EPI == EPI_I32) {
                            if (CTA2) mma_i8_pair(d_tmem, smem_desc(a + k * 32), smem_desc(b + k * 32), idesc, (kr | k) != 0);
                            else mma_i8(d_tmem, smem_desc(a + k * 32), smem_desc(b + k * 32), idesc, (kr | k) != 0);
                        } else {
                            if (CTA2) mma_f16_pair(d_tmem, smem_desc(a + k * 32), smem_desc(b + k * 32), idesc, (kr | k) != 0);
                            else mma_f16(d_tmem, smem_desc(a + k * 32), smem_desc(b + k * 32), idesc, (kr | k) != 0);
                        }
                    }
                    if (CTA2) mma_commit_pair(&empty[s]);
                    else mma_commit(&empty[s]);
                }
                if (ok) {
                    if (CTA2) mma_commit_pair(&tfull[acc]);
                    else mma_commit(&tfull[acc]);
                }
            }
            // wait for the last MMAs before TMEM can be released
            volatile int never = 0;
            if (g > 0) {
                const uint32_t last = g - 1;
                mbar_wait(&empty[last % NS], (last / NS) & 1, &never);
            }
        }
    } else if (warp >= 4 && warp < 4 + EW) {
        // ---------------- epilogue ----------------
        // Warp w drains TMEM lanes 32*(w%4)..+31 (its lane quarter); the two
        // warps of a quarter take alternate 32-column chunks. For each chunk
        // the beta*C values are fetched first (independent loads in flight
        // together), then the accumulators, then D is written.
        const EpiParams& e = p.e;
        const int q = warp & 3;
        const int half = (warp - 4) >> 2;        // 0 or 1: which chunks
        const int et = threadIdx.x - 128;        // 0 .. ET-1
        const int cols_out = e.cplx ? BN / 2 : BN;
        uint32_t epi_cphase = 0;  // completed phases of this warp's C-box barrier
        // the accumulator buffer is free again once every epilogue thread has
        // read it (pair: once per warp, on the leader's barrier)
        auto release_acc = [&](int acc) {
            if (CTA2) {
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(cluster_addr(&tempty[acc], 0));
            } else {
                mbar_arrive(&tempty[acc]);
            }
        };
        for (int i = 0; i < my_tiles; i++) {
            const Item it = item_of(p, unit + i * units);
            const int tile = it.tile;
            const int tm = tile % p.tiles_m;
            const int rest = tile / p.tiles_m;
            const int tn = rest % p.tiles_n;
            const int l = rest / p.tiles_n;
            const int64_t row0 = (int64_t)tm * G::tile_m + (int64_t)rank * BM;  // this CTA's first row
            // column offsets of this tile (the TMA epilogue needs none: its
            // staging boxes share this memory)
            for (int c = et; EPI != EPI_TMA && EPI != EPI_I32 && c < cols_out; c += ET) {
                const int64_t n = (int64_t)tn * cols_out + c;
                int64_t oc = 0, od = 0;
                if (n < e.N) decode2(e.nn, n, oc, od);
                colC[c] = oc;
                colD[c] = od;
            }
            int64_t lC, lD;
            const void* Cbase = e.C;
            void* Dbase = e.D;
            int64_t lt = l;
            if (e.Ds) {  // batched product: this tile's batch and batch mode
                lt = l % e.Lper;
                Cbase = e.Cs[l / e.Lper];
                Dbase = e.Ds[l / e.Lper];
            }
            decode2(e.ll, lt, lC, lD);
            const int64_t m = row0 + q * 32 + lane;
            const bool mok = m < e.M;
            int64_t rC = 0, rD = 0;
            if (mok) decode2(e.mm, m, rC, rD);
            rC += lC;
            rD += lD;
            const int acc = i & 1;
            const uint32_t aph = (i >> 1) & 1;
            // split tiles: this CTA's slice of the partial sums and its flag
            const int slot = it.role ? (it.tile - (p.num_tiles - p.split_tiles)) * 2 + (int)rank : 0;
            float* part = it.role ? p.partial + (size_t)slot * BN * BM : nullptr;
            bool pre = false, pre_ok = true, add_part = false;
            if ((EPI == EPI_TMA || EPI == EPI_F32) && it.role) {
                // a half of a split tile: the first half to finish hands its
                // raw sums over, the second adds them and writes D
                if (et == 0) {
                    const int w = mbar_wait(&tfull[acc], aph, abort_flag) ? 1 : 0;
                    *epi_first = w ? (atomicAdd(&p.pcount[slot], 1) == 0) : 0;
                    *epi_ok = w;
                }
                epi_bar();
                const bool ok0 = *epi_ok != 0, first = *epi_first != 0;
                fence_after();
                if (ok0 && first) {
#pragma unroll 1
                    for (int t = 0; t < BN / 32 / CS; t++) {
                        const int ch = half + CS * t;
                        uint32_t r[32];
                        tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + acc * BN + ch * 32, r);
#pragma unroll
                        for (int j = 0; j < 32; j++) part[(ch * 32 + j) * BM + q * 32 + lane] = __uint_as_float(r[j]);
                    }
                    __threadfence();
                }
                if (!ok0 || first) {
                    fence_before();
                    release_acc(acc);
                    epi_bar();
                    if (et == 0 && ok0) atomicExch(&p.pready[slot], 1);
                    continue;
                }
                epi_bar();  // every thread has read the outcome above
                if (et == 0) *epi_ok = flag_wait(&p.pready[slot], abort_flag) ? 1 : 0;
                epi_bar();
                pre = true;
                pre_ok = *epi_ok != 0;
                add_part = true;
            }
            if (EPI == EPI_TMA) {
                // Per chunk: TMA-load the 32x32 box of C into this warp's
                // staging box, combine with the accumulators, write D into the
                // same box and TMA-store it. The first box of C is requested
                // before the accumulators are ready.
                const int ew = warp - 4;
                float* box = (float*)(staging + ew * STAGE_EPI_BYTES);
                int mc[5];  // tensor-map coordinates of this warp's rows
                {
                    // the last mode keeps the whole quotient: rows past M give a
                    // coordinate past the tensor map, where TMA clips the box
                    int64_t r = row0 + q * 32;
                    for (int j = 0; j < e.mm.n; j++) {
                        const int64_t c = j + 1 < e.mm.n ? r % e.mm.ext[j] : r;
                        r /= e.mm.ext[j];
                        mc[j] = (int)c;
                    }
                }
                // the tensor maps of this tile's batch (written to global memory
                // before the launch: acquire them for the tensor-map proxy)
                const CUtensorMap* mapC = &tmC;
                const CUtensorMap* mapD = &tmD;
                if (e.tmDs) {
                    mapD = e.tmDs + l / e.Lper;
                    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mapD) : "memory");
                    if (e.tmCs) {
                        mapC = e.tmCs + l / e.Lper;
                        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mapC) : "memory");
                    }
                }
                int lc[5];
                {
                    int64_t r = lt;
                    for (int j = 0; j < e.ll.n; j++) {
                        lc[j] = (int)(r % e.ll.ext[j]);
                        r /= e.ll.ext[j];
                    }
                }
                auto coords = [&](int ch, int (&cc)[5]) {
                    int nc[5];
                    int64_t r = (int64_t)tn * BN + ch * 32;
                    for (int j = 0; j < e.nn.n; j++) {
                        nc[j] = (int)(j + 1 < e.nn.n ? r % e.nn.ext[j] : r);
                        r /= e.nn.ext[j];
                    }
                    int k = 0;
                    cc[k++] = mc[0];
                    cc[k++] = nc[0];
                    for (int j = 1; j < e.mm.n; j++) cc[k++] = mc[j];
                    for (int j = 1; j < e.nn.n; j++) cc[k++] = nc[j];
                    for (int j = 0; j < e.ll.n; j++) cc[k++] = lc[j];
                    while (k < 5) cc[k++] = 0;
                };
                const int nch = BN / 32 / CS;  // chunks per warp
                const float alpha = e.alpha_re, beta = e.beta_re;
                const int rmode = e.round_C;
                const bool bzero = e.beta_zero != 0;
                bool ok = true;
                auto issue_c = [&](int t) {
                    if (lane == 0 && !bzero) {
                        int cc[5];
                        coords(half + CS * t, cc);
                        mbar_expect_tx(&cbar[ew], STAGE_EPI_BYTES);
                        tma_load_5d(box, mapC, &cbar[ew], cc);
                    }
                };
                issue_c(0);
                if (!pre) {
                    if (et == 0) *epi_ok = mbar_wait(&tfull[acc], aph, abort_flag) ? 1 : 0;
                    epi_bar();
                    ok = *epi_ok != 0;
                } else {
                    ok = pre_ok;
                }
                fence_after();
#pragma unroll 1
                for (int t = 0; t < nch; t++) {
                    const int ch = half + CS * t;
                    uint32_t r[32];
                    if (ok) tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + acc * BN + ch * 32, r);
                    if (ok && add_part) {
#pragma unroll
                        for (int j = 0; j < 32; j++)
                            r[j] = __float_as_uint(__uint_as_float(r[j]) + __ldcg(&part[(ch * 32 + j) * BM + q * 32 + lane]));
                    }
                    bool cok = true;
                    if (!bzero) {
                        cok = mbar_wait(&cbar[ew], epi_cphase & 1, abort_flag);
                        cok = __all_sync(0xffffffffu, cok);
                        epi_cphase++;
                    }
                    if (ok && cok) {
                        float cv[32];
#pragma unroll
                        for (int j = 0; j < 32; j++) cv[j] = bzero ? 0.f : box[j * 32 + lane];
#pragma unroll
                        for (int j = 0; j < 32; j++)
                            box[j * 32 + lane] = fmaf(alpha, __uint_as_float(r[j]), beta * round_in<float>(cv[j], rmode));
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    }
                    __syncwarp();
                    if (lane == 0 && ok && cok) {
                        int cc[5];
                        coords(ch, cc);
                        tma_store_5d(mapD, box, cc);
                        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                        // the box is reused by the next load: wait until the store has read it
                        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                    }
                    __syncwarp();
                    if (!cok) ok = false;
                    if (t + 1 < nch && ok) issue_c(t + 1);
                }
                fence_before();
                release_acc(acc);
                epi_bar();
                continue;
            }
            if (EPI == EPI_I32) {
                // integer products of one level of slices: scaled exactly by a
                // power of two and added into the binary64 workspace W, laid
                // out [l][n][m] so that the 32 lanes (32 consecutive rows m)
                // read and write 256 contiguous bytes per column
                if (et == 0) *epi_ok = mbar_wait(&tfull[acc], aph, abort_flag) ? 1 : 0;
                epi_bar();
                const bool ok = *epi_ok != 0;
                fence_after();
                if (ok) {
                    const double sc = e.level_scale;
                    const bool first = e.w_first != 0;
                    double* wl = e.W + (int64_t)l * e.N * e.M + m;
#pragma unroll 1
                    for (int t = 0; t < BN / 32 / CS; t++) {
                        const int ch = half + CS * t;
                        uint32_t r[32];
                        __syncwarp();
                        tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + acc * BN + ch * 32, r);
                        const int64_t c0 = (int64_t)tn * BN + ch * 32;
                        if (!mok || c0 >= e.N) continue;
                        const int nj = e.N - c0 < 32 ? (int)(e.N - c0) : 32;
#pragma unroll
                        for (int h = 0; h < 2; h++) {
                            // 16 columns: their old values loaded together, then added in column order
                            double old[16];
#pragma unroll
                            for (int j = 0; j < 16; j++)
                                old[j] = (!first && 16 * h + j < nj) ? wl[(c0 + 16 * h + j) * e.M] : 0.0;
#pragma unroll
                            for (int j = 0; j < 16; j++) {
                                if (16 * h + j < nj) {
                                    double v = (double)(int)r[16 * h + j] * sc;
                                    if (!first) v += old[j];
                                    wl[(c0 + 16 * h + j) * e.M] = v;
                                }
                            }
                        }
                    }
                }
                fence_before();
                release_acc(acc);
                epi_bar();
                continue;
            }
            if (EPI == EPI_F32) {
                // C does not depend on the accumulators: fetch the first chunk
                // while the MMAs of this tile may still run
                epi_bar();  // column offsets of this tile are visible
                float buf[2][32];  // ping-pong: chunk t uses buf[t & 1], chunk t+1 loads into the other
                const float* Cb = (const float*)Cbase + rC;
                auto fetch = [&](int ch, float (&dst)[32]) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const int c = ch * 32 + j;
                        dst[j] = (!e.beta_zero && mok && (int64_t)tn * BN + c < e.N) ? ld_nc_f32(Cb + colC[c]) : 0.f;
                    }
                };
                fetch(half, buf[0]);
                constexpr int NCH = BN / 32 / CS;
                bool ok = pre_ok;
                if (!pre) {
                    if (et == 0) *epi_ok = mbar_wait(&tfull[acc], aph, abort_flag) ? 1 : 0;
                    epi_bar();
                    ok = *epi_ok != 0;
                }
                fence_after();
                if (ok) {
#pragma unroll
                    for (int t = 0; t < NCH; t++) {
                        const int ch = half + CS * t;
                        if (t + 1 < NCH) fetch(ch + CS, buf[(t + 1) & 1]);
                        uint32_t r[32];
                        tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + acc * BN + ch * 32, r);
                        if (add_part) {
#pragma unroll
                            for (int j = 0; j < 32; j++)
                                r[j] = __float_as_uint(__uint_as_float(r[j]) +
                                                       __ldcg(&part[(ch * 32 + j) * BM + q * 32 + lane]));
                        }
#pragma unroll
                        for (int j = 0; j < 32; j++) {
                            const int c = ch * 32 + j;
                            if (mok && (int64_t)tn * BN + c < e.N)
                                ((float*)Dbase)[rD + colD[c]] = fmaf(e.alpha_re, __uint_as_float(r[j]),
                                                                   e.beta_re * round_in<float>(buf[t & 1][j], e.round_C));
                        }
                    }
                }
                fence_before();
                release_acc(acc);
                epi_bar();  // offsets and *epi_ok may be rewritten after this point
                continue;
            }
            if (et == 0) *epi_ok = mbar_wait(&tfull[acc], aph, abort_flag) ? 1 : 0;
            epi_bar();  // column offsets and the wait's outcome are visible to every epilogue thread
            const bool ok = *epi_ok != 0;
            fence_after();
            if (ok) {
                for (int ch = half; ch < BN / 32; ch += CS) {
                    const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + acc * BN + ch * 32;
                    if (!e.cplx) {
                        float br[32], bi[32];
#pragma unroll
                        for (int j = 0; j < 32; j++) {
                            const int c = ch * 32 + j;
                            br[j] = bi[j] = 0.f;
                            if (mok && (int64_t)tn * BN + c < e.N) load_beta_c(e, Cbase, rC + colC[c], br[j], bi[j]);
                        }
                        uint32_t r[32];
                        tmem_ld32(taddr, r);
#pragma unroll
                        for (int j = 0; j < 32; j++) {
                            const int c = ch * 32 + j;
                            if (mok && (int64_t)tn * BN + c < e.N)
                                finish_out(e, Dbase, rD + colD[c], __uint_as_float(r[j]), 0.f, br[j], bi[j]);
                        }
                    } else {
                        float br[16], bi[16];
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const int c = ch * 16 + j;
                            br[j] = bi[j] = 0.f;
                            if (mok && (int64_t)tn * cols_out + c < e.N) load_beta_c(e, Cbase, rC + colC[c], br[j], bi[j]);
                        }
                        uint32_t r[32];
                        tmem_ld32(taddr, r);
#pragma unroll
                        for (int j = 0; j < 16; j++) {
                            const int c = ch * 16 + j;
                            if (mok && (int64_t)tn * cols_out + c < e.N)
                                finish_out(e, Dbase, rD + colD[c], __uint_as_float(r[2 * j]), __uint_as_float(r[2 * j + 1]),
                                           br[j], bi[j]);
                        }
                    }
                }
            }
            fence_before();
            release_acc(acc);
            epi_bar();  // offsets and *epi_ok may be rewritten after this point
        }
        // no early exit above: every epilogue thread takes every tile's barriers,
        // and after an expired wait the remaining waits give up at once
        if (EPI == EPI_TMA && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    } else if (CVT && warp >= 8) {
        // ---------------- converters: binary32 tiles -> bfloat16 hi / lo ----------------
        // Every wait is bounded; a converter that gives up stops converting,
        // and the MMA issuer's next wait on the stage it would have filled
        // gives up too.
        const int cw = warp - 8, lo3 = lane & 7, hi2 = lane >> 3;
        uint32_t g = 0;
        bool ok = true;
        for (int i = 0; i < my_tiles && ok; i++) {
            const Item it = item_of(p, unit + i * units);
            const int tile = it.tile;
            const int tm = tile % p.tiles_m;
            const int rest = tile / p.tiles_m;
            const int tn = rest % p.tiles_n;
            const int l = rest / p.tiles_n;
            int64_t ra_off[4], rb_off[4];
            const float* abase = cvt_rows(p.ca, (int64_t)tm * G::tile_m + (int64_t)rank * BM, l, cw, lo3, hi2, ra_off);
            const float* bbase = cvt_rows(p.cb, (int64_t)tn * BN + (int64_t)rank * G::b_rows, l, cw, lo3, hi2, rb_off);
            float xa[32], xb[32];
            cvt_load(p.ca, abase, ra_off, it.kb0, cw, lo3, hi2, xa);
            cvt_load(p.cb, bbase, rb_off, it.kb0, cw, lo3, hi2, xb);
            for (int kb = it.kb0; kb < it.kb1; kb++, g++) {
                const int s = g % NS;
                const uint32_t ph = (g / NS) & 1;
                if (!mbar_wait(&empty[s], ph ^ 1, abort_flag)) { ok = false; break; }
                const uint32_t st = smem_u32(tiles + s * SB);
                // each operand's next block is requested as soon as its
                // registers are free, so the loads run under the other's stores
                cvt_store(p.ca, xa, st, st + 16384, cw, lo3, hi2);
                if (kb + 1 < it.kb1) cvt_load(p.ca, abase, ra_off, kb + 1, cw, lo3, hi2, xa);
                cvt_store(p.cb, xb, st + 32768, st + 49152, cw, lo3, hi2);
                if (kb + 1 < it.kb1) cvt_load(p.cb, bbase, rb_off, kb + 1, cw, lo3, hi2, xb);
                // generic-proxy stores -> the MMAs' async-proxy reads
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    if (CTA2) mbar_arrive_cluster(cluster_addr(&full[s], 0));
                    else mbar_arrive(&full[s]);
                }
            }
        }
    }
    fence_before();
    if (CTA2) cluster_sync();  // the leader's MMAs into this CTA's TMEM, and remote signals, are done
    else __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(p.error, 1);
    if (warp == 2) {
        fence_after();
        if (CTA2) asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
        else asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS));
    }
}

// ---------------------------------------------------------------------------
// host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

static bool make_map(CUtensorMap* tm, void* base, int fmt, uint64_t kld, uint64_t rows, uint64_t L, uint32_t box_rows)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[3] = {kld, rows, L};
    cuuint64_t strides[2] = {kld * 2, kld * rows * 2};
    cuuint32_t box[3] = {(cuuint32_t)BK, box_rows, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(tm, fmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims,
                     strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}


// Tensor map of C (which = 2) or D (which = 3) for the TMA epilogue, or false
// when the layout does not allow it: binary32, the first M mode contiguous
// (stride 1) with an extent that is a multiple of 32, the first N mode with an
// extent that is a multiple of 32, every other stride positive and a multiple
// of 16 bytes, at most 5 dimensions. Box: 32 x 32 x 1 x 1 x 1.
static bool make_epi_map(CUtensorMap* tm, void* base, const tb_plan* P, int which)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc || !base) return false;
    const tb_modes& M = P->M;
    const tb_modes& N = P->N;
    const tb_modes& L = P->L;
    if (M.n < 1 || N.n < 1) return false;
    const int rank = 2 + (M.n - 1) + (N.n - 1) + L.n;
    if (rank > 5) return false;
    auto st = [&](const tb_modes& m, int j) { return which == 2 ? m.sC[j] : m.sD[j]; };
    if (st(M, 0) != 1 || M.ext[0] % 32 != 0 || N.ext[0] % 32 != 0) return false;
    if (((uintptr_t)base & 15) != 0) return false;
    cuuint64_t dims[5], strides[4];
    int k = 0;
    int64_t sd[5];
    dims[k] = (cuuint64_t)M.ext[0]; sd[k++] = 1;
    dims[k] = (cuuint64_t)N.ext[0]; sd[k++] = st(N, 0);
    for (int j = 1; j < M.n; j++) { dims[k] = (cuuint64_t)M.ext[j]; sd[k++] = st(M, j); }
    for (int j = 1; j < N.n; j++) { dims[k] = (cuuint64_t)N.ext[j]; sd[k++] = st(N, j); }
    for (int j = 0; j < L.n; j++) { dims[k] = (cuuint64_t)L.ext[j]; sd[k++] = st(L, j); }
    for (int j = 1; j < k; j++) {
        if (sd[j] <= 0 || (sd[j] * 4) % 16 != 0 || sd[j] * 4 >= (1ll << 40)) return false;
        strides[j - 1] = (cuuint64_t)(sd[j] * 4);
    }
    while (k < 5) {  // unit dimensions up to rank 5
        dims[k] = 1;
        strides[k - 1] = strides[k - 2];
        k++;
    }
    cuuint32_t box[5] = {32, 32, 1, 1, 1};
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static void fill_modes(ModeList& m, const tb_modes& src, int which0, int which1)
{
    memset(&m, 0, sizeof(m));
    m.n = src.n;
    for (int j = 0; j < src.n; j++) {
        m.ext[j] = src.ext[j];
        const int64_t* s[4] = {src.sA, src.sB, src.sC, src.sD};
        m.s0[j] = which0 >= 0 ? s[which0][j] : 0;
        m.s1[j] = which1 >= 0 ? s[which1][j] : 0;
    }
}

static int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

static int num_sms()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

// smallest |stride| among a mode list's modes (for the load order of the pack)
static int64_t min_stride(const tb_modes& m, int which)
{
    const int64_t* s = which == 0 ? m.sA : m.sB;
    int64_t best = INT64_MAX;
    for (int j = 0; j < m.n; j++) {
        int64_t v = s[j] < 0 ? -s[j] : s[j];
        if (v != 0 && v < best) best = v;
    }
    return best;
}

struct Workspace {
    void* buf = nullptr;
    size_t bytes = 0;
};


// Launches the GEMM: 1-CTA (128x256 tiles) or CTA pairs (256x256 tiles,
// cluster of 2, cta_group::2) when M spans at least two 128-row halves.
// load 1: the split-bfloat16 GEMM converting binary32 operands in place;
// load 2: the split-bfloat16 GEMM from [hi | lo] panels (both pairs only).
static cudaError_t launch_gemm(int kind, bool cta2, int grid, const CUtensorMap& tmA, const CUtensorMap& tmB,
                               const GemmParams& gp, uint32_t idesc, const CUtensorMap& tmC, const CUtensorMap& tmD,
                               cudaStream_t s, int load = 0, bool pdl = false)
{
    void (*kern)(CUtensorMap, CUtensorMap, GemmParams, uint32_t, CUtensorMap, CUtensorMap);
    if (load == 1)
        kern = kind == EPI_TMA ? k_gemm<EPI_TMA, true, 1> : kind == EPI_F32 ? k_gemm<EPI_F32, true, 1>
               : k_gemm<EPI_ANY, true, 1>;
    else if (load == 2)
        kern = kind == EPI_TMA ? k_gemm<EPI_TMA, true, 2> : kind == EPI_F32 ? k_gemm<EPI_F32, true, 2>
               : k_gemm<EPI_ANY, true, 2>;
    else if (cta2)
        kern = kind == EPI_TMA ? k_gemm<EPI_TMA, true> : kind == EPI_F32 ? k_gemm<EPI_F32, true>
               : kind == EPI_I32 ? k_gemm<EPI_I32, true> : k_gemm<EPI_ANY, true>;
    else
        kern = kind == EPI_TMA ? k_gemm<EPI_TMA, false> : kind == EPI_F32 ? k_gemm<EPI_F32, false>
               : kind == EPI_I32 ? k_gemm<EPI_I32, false> : k_gemm<EPI_ANY, false>;
    static int attr_done[64][4][2][3];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev][kind][cta2][load]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev][kind][cta2][load] = 1;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(load == 1 ? 512 : NTHREADS, 1, 1);
    cfg.dynamicSmemBytes = SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cta2 ? 2 : 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 2 : 1;
    return cudaLaunchKernelEx(&cfg, kern, tmA, tmB, gp, idesc, tmC, tmD);
}

// Tensor map of an 8-bit panel view: rows of `kext` bytes (the K range one
// GEMM reads) `row_bytes` apart, `rows` rows per batch, L batches.
static bool make_map_i8(CUtensorMap* tm, const void* base, uint64_t kext, uint64_t row_bytes, uint64_t rows,
                        uint64_t L, uint32_t box_rows)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc || ((uintptr_t)base & 15) || (row_bytes & 15) || (kext & 15)) return false;
    cuuint64_t dims[3] = {kext, rows, L};
    cuuint64_t strides[2] = {row_bytes, row_bytes * rows};
    cuuint32_t box[3] = {(cuuint32_t)(2 * BK), box_rows, 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tc

// One integer GEMM over 8-bit slice panels: A8 [L][M][row_bytes] and B8
// [L][Nout][row_bytes] bytes, each GEMM reading `klen` bytes per row from
// byte a_off (A) and b_off (B) on; W[l][m][n] (+)= scale * sum. |sum| must
// stay below 2^31 (the caller bounds the number of terms).
cudaError_t launch_gemm_i8(const void* A8, const void* B8, int64_t row_bytes, int64_t M, int64_t Nout, int64_t L,
                           int64_t a_off, int64_t b_off, int64_t klen, double* W, double scale, int first,
                           cudaStream_t s)
{
    using namespace tc;
    int* flag = device_error_word();
    if (!flag) return cudaErrorMemoryAllocation;
    const bool cta2 = M >= 2 * BM && num_sms() % 2 == 0;
    CUtensorMap tmA, tmB;
    if (!make_map_i8(&tmA, (const char*)A8 + a_off, (uint64_t)klen, (uint64_t)row_bytes, (uint64_t)M, (uint64_t)L, BM) ||
        !make_map_i8(&tmB, (const char*)B8 + b_off, (uint64_t)klen, (uint64_t)row_bytes, (uint64_t)Nout, (uint64_t)L,
                     cta2 ? Geo<true>::b_rows : BN))
        return cudaErrorInvalidValue;
    GemmParams gp;
    memset(&gp, 0, sizeof(gp));
    gp.tiles_m = (int)((M + (cta2 ? 2 * BM : BM) - 1) / (cta2 ? 2 * BM : BM));
    gp.tiles_n = (int)((Nout + BN - 1) / BN);
    gp.num_tiles = gp.tiles_m * gp.tiles_n * (int)L;
    gp.num_kb = (int)((klen + 2 * BK - 1) / (2 * BK));
    gp.error = flag;
    gp.e.M = M;
    gp.e.N = Nout;
    gp.e.L = L;
    gp.e.W = W;
    gp.e.level_scale = scale;
    gp.e.w_first = first;
    const uint32_t mma_m = cta2 ? 2 * BM : BM;
    // D: signed 32-bit (2), A and B: signed 8-bit (1)
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((mma_m >> 4) << 24);
    const int units = cta2 ? num_sms() / 2 : num_sms();
    const int grid = (gp.num_tiles < units ? gp.num_tiles : units) * (cta2 ? 2 : 1);
    cudaError_t e = launch_gemm(EPI_I32, cta2, grid, tmA, tmB, gp, idesc, tmA, tmA, s);
    count_launch();
    return e;
}

// Tensor map reading an operand in place (16-bit storage of the product's
// 16-bit precision, real, no unary modes): dims (row0, k0, row1, k1, batch)
// when the first row mode is contiguous (MN-major tiles) or (k0, row0, k1,
// row1, batch) when the first contracted mode is (K-major tiles); box 64 x 64.
// False when the layout does not allow it (more than two row or contracted
// modes or one batch mode, extents of the leading modes not multiples of 64,
// strides not positive multiples of 16 bytes, base not 16-byte aligned).
static bool make_direct_map(CUtensorMap* tm, const void* base, const tb_plan* P, int side, int rows, int* mn, int* e0,
                            int* k0, int* boxmode, int* dmask)
{
    using namespace tc;
    EncodeTiledFn enc = encode_fn();
    const tb_modes& R = side == 0 ? P->M : P->N;
    const tb_modes& K = P->K;
    const tb_modes& L = P->L;
    auto st = [&](const tb_modes& m, int j) { return side == 0 ? m.sA[j] : m.sB[j]; };
    if (!enc || !base || ((uintptr_t)base & 15) || R.n < 1 || R.n > 2 || K.n < 1 || K.n > 2 || L.n > 1) return false;
    int major;
    if (st(R, 0) == 1 && R.ext[0] % 64 == 0 && K.ext[0] % 64 == 0) major = 1;
    else if (st(K, 0) == 1 && K.ext[0] % 64 == 0 && R.ext[0] % 64 == 0) major = 0;
    else return false;
    cuuint64_t dims[5];
    int64_t str[5];
    const tb_modes* first = major ? &R : &K;
    const tb_modes* second = major ? &K : &R;
    dims[0] = (cuuint64_t)first->ext[0];
    str[0] = 1;
    dims[1] = (cuuint64_t)second->ext[0];
    str[1] = st(*second, 0);
    dims[2] = first->n > 1 ? (cuuint64_t)first->ext[1] : 1;
    str[2] = first->n > 1 ? st(*first, 1) : str[1];
    dims[3] = second->n > 1 ? (cuuint64_t)second->ext[1] : 1;
    str[3] = second->n > 1 ? st(*second, 1) : str[2];
    dims[4] = L.n ? (cuuint64_t)L.ext[0] : 1;
    str[4] = L.n ? st(L, 0) : str[3];
    cuuint64_t strides[4];
    for (int j = 1; j < 5; j++) {
        if (str[j] <= 0 || (str[j] * 2) % 16 != 0 || str[j] * 2 >= (1ll << 40)) return false;
        strides[j - 1] = (cuuint64_t)(str[j] * 2);
    }
    // one box per tile when the rows allow it (fewer, larger copies)
    cuuint32_t box[5] = {64, 64, 1, 1, 1};
    int bm = 0;
    if (R.ext[0] == 64 && R.n == 2 && R.ext[1] >= rows / 64) {
        bm = 1;
        box[major ? 2 : 3] = (cuuint32_t)(rows / 64);
    } else if (!major && R.ext[0] % rows == 0) {
        bm = 2;
        box[1] = (cuuint32_t)rows;
    }
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    const int fmt = P->tc_mode == TB_TC_F16 ? 1 : 0;
    // keep dims 0 and 1 and every dim of extent > 1; a 3-d map at least
    cuuint64_t cd[5];
    cuuint64_t cs[4];
    cuuint32_t cb[5];
    int rank = 0, mask = 0;
    int64_t cstr[5];
    for (int j = 0; j < 5; j++) {
        if (j >= 2 && dims[j] == 1) continue;
        cd[rank] = dims[j];
        cstr[rank] = j == 0 ? 1 : str[j];
        cb[rank] = box[j];
        mask |= 1 << j;
        rank++;
    }
    for (int j = 2; rank < 3 && j < 5; j++)
        if (!(mask >> j & 1)) {  // pad with a unit dim, in logical order
            mask |= 1 << j;
            rank = 0;
            for (int i = 0; i < 5; i++)
                if (mask >> i & 1) {
                    cd[rank] = dims[i];
                    cstr[rank] = i == 0 ? 1 : str[i];
                    cb[rank] = box[i];
                    rank++;
                }
        }
    for (int j = 1; j < rank; j++) cs[j - 1] = (cuuint64_t)(cstr[j] * 2);
    if (enc(tm, fmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, rank, const_cast<void*>(base),
            cd, cs, cb, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    *mn = major;
    *e0 = (int)R.ext[0];
    *k0 = (int)K.ext[0];
    *boxmode = bm;
    *dmask = mask;
    return true;
}

// whether an operand can be read in place (besides its layout, checked by
// make_direct_map): its storage is the product's 16-bit operand type
static bool direct_type_ok(const tb_plan* P, int side)
{
    const int t = side == 0 ? P->tA : P->tB;
    const int need = P->tc_mode == TB_TC_BF16 ? T_BF16 : P->tc_mode == TB_TC_F16 ? T_F16 : -1;
    const tb_modes& U = side == 0 ? P->UA : P->UB;
    return t == need && U.n == 0 && P->compute == TB_R32 && (int64_t)P->K.size < (1ll << 31) &&
           (side == 0 ? P->M.size : P->N.size) < (1ll << 31);
}

// Batches per launch group of a batched product: the panels of one group at
// most 2 GiB (one batch always), grid.z = batches x batch modes <= 65535.
static int64_t group_batches(int64_t num, size_t per_batch, int64_t Lsz, int64_t tiles_per_batch)
{
    int64_t G = per_batch ? (int64_t)(((size_t)2 << 30) / per_batch) : num;
    if (G > 65535 / Lsz) G = 65535 / Lsz;
    if (G * tiles_per_batch > (1ll << 30)) G = (1ll << 30) / tiles_per_batch;
    if (G > num) G = num;
    return G < 1 ? 1 : G;
}

// Index map of a mode list for the in-place converters (at most 4 modes,
// every index below 2^31).
static bool make_cvt_dim(tc::CvtDim* o, const tb_modes& m, int side)
{
    if (m.n > 4 || m.size >= (1ll << 31)) return false;
    memset(o, 0, sizeof(*o));
    o->n = m.n;
    o->size = (uint32_t)m.size;
    for (int j = 0; j < m.n; j++) {
        o->div[j] = make_fastdiv((uint32_t)m.ext[j]);
        o->st[j] = side == 0 ? m.sA[j] : m.sB[j];
    }
    return true;
}

// Whether operand `side` (0 A, 1 B) of a tensor-core product can be read in
// place by converter warps, and its description if so: binary32 storage, no
// unary modes, at most 4 row, contracted and batch modes. vec = 1 (two
// 16-byte loads per run of 8 elements) when its contiguous mode comes first
// in its row or contracted list with stride 1 and an extent divisible by 8,
// every other stride is divisible by 4 and the base is 16-byte aligned;
// otherwise, with `scalar_ok` (the grouped kernel), vec = 0: element-wise
// loads through offset tables, any strides.
static bool make_cvt_operand(tc::CvtOperand* o, const tb_plan* P, int side, const void* base, bool scalar_ok = false)
{
    using namespace tc;
    const tb_modes& R = side == 0 ? P->M : P->N;
    const tb_modes& U = side == 0 ? P->UA : P->UB;
    if ((side == 0 ? P->tA : P->tB) != T_F32 || U.n != 0 || !base || ((uintptr_t)base & 3) || R.n < 1 ||
        P->K.n < 1)
        return false;
    memset(o, 0, sizeof(*o));
    if (!make_cvt_dim(&o->rows, R, side) || !make_cvt_dim(&o->ks, P->K, side) || !make_cvt_dim(&o->ls, P->L, side))
        return false;
    o->base = (const float*)base;
    o->mn = min_stride(R, side) < min_stride(P->K, side);
    const CvtDim& fast = o->mn ? o->rows : o->ks;
    bool vec = ((uintptr_t)base & 15) == 0 && fast.st[0] == 1 && fast.div[0].d % 8 == 0;
    const CvtDim* all[3] = {&o->rows, &o->ks, &o->ls};
    for (int i = 0; i < 3 && vec; i++)
        for (int j = 0; j < all[i]->n; j++)
            if (!(all[i] == &fast && j == 0) && all[i]->st[j] % 4 != 0) vec = false;
    o->vec = vec;
    return vec || scalar_ok;
}

// Whether a split-bfloat16 product can run on the converter warps with A
// and B read in place (CTA pairs: at least 256 rows of A), and their
// descriptions.
static bool split_in_place(const tb_plan* P, const void* A, const void* B, tc::CvtOperand* ca, tc::CvtOperand* cb)
{
    return P->path == TB_PATH_TC && P->tc_mode == TB_TC_SPLIT_BF16 && P->compute == TB_R32 &&
           P->M.size >= 2 * tc::BM && tc::num_sms() % 2 == 0 && make_cvt_operand(ca, P, 0, A) &&
           make_cvt_operand(cb, P, 1, B);
}

// Whether a split-bfloat16 product can run from [hi | lo] panels: a real
// product on CTA pairs whose operands both go through the real pack (no
// unary modes, real storage).
static bool split_panels_ok(const tb_plan* P)
{
    auto real = [](int t) { return t == T_F32 || t == T_F64 || t == T_F16 || t == T_BF16; };
    return P->path == TB_PATH_TC && P->tc_mode == TB_TC_SPLIT_BF16 && P->compute == TB_R32 &&
           P->M.size >= 2 * tc::BM && tc::num_sms() % 2 == 0 && P->UA.n == 0 && P->UB.n == 0 && real(P->tA) &&
           real(P->tB);
}

// Route of a split-bfloat16 product's operands: 1 read in place by the
// converter warps, 2 [hi | lo] panels, 0 three-segment panels. The
// automatic choice (split_route 1) prefers the panels where both are
// possible: the converters are slower on the measured workloads.
static int split_route(const tb_plan* P, bool in_place_ok)
{
    const bool panels = split_panels_ok(P);
    if (in_place_ok && (P->split_route == 3 || !panels)) return 1;
    return panels ? 2 : 0;
}

// Epilogue parameters of one product (or one group of a batched product,
// Lg = batches x batch modes) for C and D with their own strides.
static void fill_epilogue(tc::EpiParams& ep, const tb_plan* P, const void* C, void* D, int64_t Lg)
{
    using namespace tc;
    ep.C = C;
    ep.D = D;
    ep.tC = P->tC;
    ep.tD = P->tD;
    ep.cplx = P->compute == TB_C32;
    ep.beta_zero = P->beta_zero;
    ep.conjC = P->conjC;
    ep.conjD = P->conjD;
    ep.conjD_f32 = P->conjD_round_f32;
    ep.round_C = P->round_in;
    ep.alpha_re = (float)P->alpha_re;
    ep.alpha_im = (float)P->alpha_im;
    ep.beta_re = (float)P->beta_re;
    ep.beta_im = (float)P->beta_im;
    ep.M = P->M.size;
    ep.N = P->N.size;
    ep.L = Lg;
    fill_modes(ep.mm, P->M, 2, 3);
    fill_modes(ep.nn, P->N, 2, 3);
    fill_modes(ep.ll, P->L, 2, 3);
}

// Descriptor of one product for the grouped kernel (group.cu): a real
// binary32 product of the tensor-core path (16-bit precisions or split
// bfloat16) whose operands the converter warps read in place. cta2: 256 x
// 256 tiles on CTA pairs, else 128 x 128. False when it does not qualify.
bool group_item(const tb_plan* P, const tb_ptrs* d, bool cta2, tc::GroupItem* g)
{
    using namespace tc;
    if (P->path != TB_PATH_TC || P->compute != TB_R32 ||
        (P->tc_mode != TB_TC_BF16 && P->tc_mode != TB_TC_F16 && P->tc_mode != TB_TC_SPLIT_BF16))
        return false;
    memset(g, 0, sizeof(*g));
    if (!make_cvt_operand(&g->a, P, 0, d->A, true) || !make_cvt_operand(&g->b, P, 1, d->B, true)) return false;
    fill_epilogue(g->e, P, d->C, d->D, P->L.size);
    const int64_t tm = cta2 ? 2 * BM : BM, tn = cta2 ? BN : 128;
    const int64_t tiles_m = (P->M.size + tm - 1) / tm, tiles_n = (P->N.size + tn - 1) / tn;
    if (tiles_m * tiles_n * P->L.size >= (1ll << 30)) return false;
    g->tiles_m = (int32_t)tiles_m;
    g->tiles_n = (int32_t)tiles_n;
    g->num_kb = (int32_t)((P->K.size + BK - 1) / BK);
    g->mode = P->tc_mode;
    const uint32_t ab = P->tc_mode == TB_TC_F16 ? 0u : 1u;  // operand format: 0 f16, 1 bf16
    g->idesc = (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)g->a.mn << 15) | ((uint32_t)g->b.mn << 16) |
               ((uint32_t)(tn >> 3) << 17) | ((uint32_t)(tm >> 4) << 24);
    g->f32_epi = P->tD == T_F32 && (P->beta_zero || P->tC == T_F32) && !P->conjD;
    return true;
}

int tc_sm_count() { return tc::num_sms(); }

// A last round that fills at most half the units runs its tiles as two
// half-contraction items each (partial sums handed over in memory). Only the
// binary32 epilogues (EPI_TMA, EPI_F32) hand over partial sums. The hand-over
// counters are zeroed here, before the operand packs are launched, so that
// nothing stands between the last pack and the GEMM in the stream.
struct SplitRound {
    int r = 0;
    void* ws = nullptr;
};

static SplitRound plan_split_round(bool f32_epi, int num_tiles, int num_kb, int units, cudaStream_t s)
{
    using namespace tc;
    SplitRound sr;
    if (!(f32_epi && num_tiles > units && num_kb >= 2)) return sr;
    const int r = num_tiles % units;
    if (r == 0 || 2 * r > units) return sr;
    const size_t pbytes = (size_t)r * 2 * BN * BM * sizeof(float);
    const size_t fbytes = (size_t)r * 2 * 2 * sizeof(int);
    if (pool_alloc(&sr.ws, pbytes + fbytes, s) == cudaSuccess &&
        cudaMemsetAsync((char*)sr.ws + pbytes, 0, fbytes, s) == cudaSuccess) {
        sr.r = r;
    } else if (sr.ws) {
        cudaFreeAsync(sr.ws, s);
        sr.ws = nullptr;
    }
    (void)cudaGetLastError();
    return sr;
}

static void use_split_round(tc::GemmParams& gp, const SplitRound& sr)
{
    using namespace tc;
    if (!sr.r) return;
    const size_t pbytes = (size_t)sr.r * 2 * BN * BM * sizeof(float);
    gp.split_tiles = sr.r;
    gp.partial = (float*)sr.ws;
    gp.pcount = (int*)((char*)sr.ws + pbytes);
    gp.pready = gp.pcount + sr.r * 2;
}

cudaError_t launch_tc(const tb_plan* P, const tb_ptrs* d, int num, cudaStream_t s, int* kernels, void** main_timer)
{
    // split-bfloat16 products whose binary32 operands the converter warps
    // read in place (every batch's A and B 16-byte aligned): no pack
    // launches, no panels
    tc::CvtOperand cva, cvb;
    bool in_place = split_in_place(P, d[0].A, d[0].B, &cva, &cvb);
    for (int b = 1; b < num && in_place; b++)
        if (((uintptr_t)d[b].A & 15) || ((uintptr_t)d[b].B & 15)) in_place = false;
    const int route = P->tc_mode == TB_TC_SPLIT_BF16 ? split_route(P, in_place) : 0;
    const bool cvt = route == 1, spl = route == 2;
    using namespace tc;
    *kernels = 0;
    const int cplx = P->compute == TB_C32;
    const int split = P->tc_mode == TB_TC_SPLIT_BF16 ? (spl ? 2 : 3) : 1;
    const int fmt = P->tc_mode == TB_TC_F16 ? 1 : 0;
    const int64_t M = P->M.size, N = P->N.size, Lsz = P->L.size, K = P->K.size;
    const int64_t Kreal = K * (cplx ? 2 : 1);
    // [hi | lo] panels: each part a whole number of 64-deep blocks (zeros past K)
    const int64_t Kseg = round_up(Kreal, spl ? 64 : 8);
    const int64_t Kld = Kseg * split;
    const int64_t Nout = N * (cplx ? 2 : 1);
    const size_t bytesA = cvt ? 0 : (size_t)Lsz * M * Kld * 2, bytesB = cvt ? 0 : (size_t)Lsz * Nout * Kld * 2;
    const bool cta2 = M >= 2 * BM && num_sms() % 2 == 0;
    const int64_t tiles_per_batch = ((M + (cta2 ? 2 * BM : BM) - 1) / (cta2 ? 2 * BM : BM)) * ((Nout + BN - 1) / BN) * Lsz;
    // A batched product runs in groups of G batches: one pack launch per
    // operand and one GEMM launch per group, the batches' panels side by side
    // (batch b, mode l at panel batch index b * Lsz + l) and the epilogue
    // finding each tile's C and D through pointer arrays.
    const int64_t G = num > 1 ? group_batches(num, bytesA + bytesB, Lsz, tiles_per_batch) : 1;
    const size_t scratch = round_up((int64_t)(bytesA * G), 256) + round_up((int64_t)(bytesB * G), 256);

    void* ws = nullptr;
    cudaError_t e = cudaSuccess;
    if (scratch) e = pool_alloc(&ws, scratch, s);  // reused by every group: same stream, in order
    if (e != cudaSuccess) return e;
    int* flag = device_error_word();
    if (!flag) {
        if (ws) cudaFreeAsync(ws, s);
        return cudaErrorMemoryAllocation;
    }
    const void** dptr = nullptr;  // device copy of [A...][B...][C...][D...]
    CUtensorMap* maps = nullptr;    // host staging of one group's epilogue tensor maps
    CUtensorMap* dmaps = nullptr;   // their device copy
    bool a_vec_ok = true, b_vec_ok = true;
    if (G > 1) {
        const size_t pbytes = sizeof(void*) * 4 * (size_t)num;
        const void** host = (const void**)malloc(pbytes);
        if (!host) {
            if (ws) cudaFreeAsync(ws, s);
            return cudaErrorMemoryAllocation;
        }
        for (int b = 0; b < num; b++) {
            host[b] = d[b].A;
            host[num + b] = d[b].B;
            host[2 * num + b] = d[b].C;
            host[3 * num + b] = d[b].D;
            if (((uintptr_t)d[b].A & 15) != 0) a_vec_ok = false;
            if (((uintptr_t)d[b].B & 15) != 0) b_vec_ok = false;
        }
        e = pool_alloc((void**)&dptr, pbytes, s);
        if (e == cudaSuccess) e = stage_copy(dptr, host, pbytes, s);
        free(host);
        if (e == cudaSuccess) {
            maps = (CUtensorMap*)aligned_alloc(64, sizeof(CUtensorMap) * 2 * (size_t)G);
            if (maps && pool_alloc((void**)&dmaps, sizeof(CUtensorMap) * 2 * (size_t)G, s) != cudaSuccess) {
                free(maps);
                maps = nullptr;
                dmaps = nullptr;
            }
        }
        if (e != cudaSuccess) {
            if (dptr) cudaFreeAsync(dptr, s);
            if (ws) cudaFreeAsync(ws, s);
            return e;
        }
    }
    for (int64_t b0 = 0; b0 < num; b0 += G) {
        const int64_t g = num - b0 < G ? num - b0 : G;  // batches in this group
        const int64_t Lg = g * Lsz;
        char* base = (char*)ws;
        void* pA = base;
        void* pB = base + round_up((int64_t)(bytesA * G), 256);

        // operands read in place need no pack (single products only: the maps
        // describe one batch's tensors)
        CUtensorMap dmap[2];
        int dir[2] = {0, 0}, dmn[2] = {0, 0}, de0[2] = {0, 0}, dk0[2] = {0, 0}, dbox[2] = {0, 0}, dmask[2] = {0, 0};
        if (cvt) dir[0] = dir[1] = 1;  // no pack; the converters read A and B
        else if (G == 1 && split == 1)
            for (int side = 0; side < 2; side++)
                dir[side] = direct_type_ok(P, side) &&
                            make_direct_map(&dmap[side], side == 0 ? d[b0].A : d[b0].B, P, side,
                                            side == 0 ? BM : (cta2 ? Geo<true>::b_rows : BN), &dmn[side], &de0[side],
                                            &dk0[side], &dbox[side], &dmask[side]);

        // the split last round's counters, zeroed before the packs
        const bool f32_epi = !cplx && P->tD == T_F32 && (P->beta_zero || P->tC == T_F32) && !P->conjD;
        const int units = cta2 ? num_sms() / 2 : num_sms();
        const int64_t g_tiles = ((M + (cta2 ? 2 * BM : BM) - 1) / (cta2 ? 2 * BM : BM)) * ((Nout + BN - 1) / BN) * Lg;
        const int64_t g_kb = ((cvt ? K : spl ? Kseg : Kld) + BK - 1) / BK;
        const SplitRound sr = plan_split_round(f32_epi, (int)g_tiles, (int)g_kb, units, s);
        int packs = 0;

        // pack A and B
        for (int side = 0; side < 2; side++) {
            if (dir[side]) continue;
            PackParams pp;
            memset(&pp, 0, sizeof(pp));
            pp.src = side == 0 ? d[b0].A : d[b0].B;
            if (G > 1) pp.srcs = dptr + (side == 0 ? 0 : num) + b0;
            pp.dst = side == 0 ? pA : pB;
            pp.type = side == 0 ? P->tA : P->tB;
            pp.conj = side == 0 ? P->conjA : P->conjB;
            pp.round_mode = split == 3 ? TB_ROUND_NONE : P->round_in;
            pp.cplx = cplx;
            pp.is_B = side;
            pp.split = split;
            pp.fmt = fmt;
            pp.R = side == 0 ? M : N;
            pp.K = K;
            pp.Lsz = Lsz;
            pp.Kseg = Kseg;
            pp.Kld = Kld;
            pp.Rout = side == 0 ? M : Nout;
            const int which = side;  // stride of A or of B
            fill_modes(pp.rows, side == 0 ? P->M : P->N, which, -1);
            fill_modes(pp.ks, P->K, which, -1);
            fill_modes(pp.ls, P->L, which, -1);
            fill_modes(pp.us, side == 0 ? P->UA : P->UB, which, -1);
            pp.usize = side == 0 ? P->UA.size : P->UB.size;
            pp.rows_fast = min_stride(side == 0 ? P->M : P->N, which) < min_stride(P->K, which);
            if (!cplx && pp.us.n == 0 && (pp.type == T_F32 || pp.type == T_F64 || pp.type == T_F16 ||
                                           pp.type == T_BF16)) {
                // the vector loads need every batch's base 16-byte aligned
                const bool al = side == 0 ? a_vec_ok : b_vec_ok;
                // B's pack right after A's (a single product) overlaps its tail
                const bool pdl = G == 1 && packs == 1;
                switch (pp.type) {
                case T_F32: launch_pack_real<float>(pp, split, fmt, Lg, al, s, pdl); break;
                case T_F64: launch_pack_real<double>(pp, split, fmt, Lg, al, s, pdl); break;
                case T_F16: launch_pack_real<__half>(pp, split, fmt, Lg, al, s, pdl); break;
                default: launch_pack_real<__nv_bfloat16>(pp, split, fmt, Lg, al, s, pdl); break;
                }
            } else {
                dim3 grid((unsigned)((pp.R + PR - 1) / PR), (unsigned)((Kseg / (cplx ? 2 : 1) + PK - 1) / PK),
                          (unsigned)Lg);
                k_pack<<<grid, 256, 0, s>>>(pp);
            }
            count_launch();
            (*kernels)++;
            packs++;
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) {
            if (sr.ws) cudaFreeAsync(sr.ws, s);
            break;
        }

        CUtensorMap tmA, tmB;
        if (cvt) {
            memset(&tmA, 0, sizeof(tmA));  // unused: no TMA operand loads
            tmB = tmA;
        } else {
            if (dir[0]) tmA = dmap[0];
            if (dir[1]) tmB = dmap[1];
        }
        if (cvt) {
        } else if ((!dir[0] && !make_map(&tmA, pA, fmt, Kld, M, Lg, BM)) ||
            (!dir[1] && !make_map(&tmB, pB, fmt, Kld, Nout, Lg, cta2 ? Geo<true>::b_rows : BN))) {
            e = cudaErrorInvalidValue;
            if (sr.ws) cudaFreeAsync(sr.ws, s);
            break;
        }
        GemmParams gp;
        memset(&gp, 0, sizeof(gp));
        gp.tiles_m = (int)((M + (cta2 ? 2 * BM : BM) - 1) / (cta2 ? 2 * BM : BM));
        gp.tiles_n = (int)((Nout + BN - 1) / BN);
        gp.num_tiles = gp.tiles_m * gp.tiles_n * (int)Lg;
        gp.num_kb = (int)(((cvt ? K : spl ? Kseg : Kld) + BK - 1) / BK);
        gp.lo_off = spl ? (int32_t)Kseg : 0;
        gp.error = flag;
        if (cvt) {
            gp.ca = cva;
            gp.cb = cvb;
            gp.ca.base = (const float*)d[b0].A;
            gp.cb.base = (const float*)d[b0].B;
            if (G > 1) {
                gp.ca.bases = (const void* const*)(dptr + b0);
                gp.cb.bases = (const void* const*)(dptr + num + b0);
                gp.ca.lper = gp.cb.lper = Lsz;
            }
            gp.a_mn = cva.mn;
            gp.b_mn = cvb.mn;
        }
        gp.a_direct = cvt ? 0 : dir[0];
        gp.b_direct = cvt ? 0 : dir[1];
        if (!cvt) {
            gp.a_mn = dir[0] && dmn[0];
            gp.b_mn = dir[1] && dmn[1];
        }
        gp.a_e0 = de0[0];
        gp.a_k0 = dk0[0];
        gp.b_e0 = de0[1];
        gp.b_k0 = dk0[1];
        gp.a_box = dbox[0];
        gp.b_box = dbox[1];
        gp.a_dims = dmask[0];
        gp.b_dims = dmask[1];
        EpiParams& ep = gp.e;
        fill_epilogue(ep, P, d[b0].C, d[b0].D, Lg);
        if (G > 1) {
            ep.Cs = dptr + 2 * num + b0;
            ep.Ds = (void* const*)(dptr + 3 * num + b0);
            ep.Lper = Lsz;
        }
        const uint32_t ab = fmt == 1 ? 0u : 1u;  // operand format: 0 f16, 1 bf16
        const uint32_t mma_m = cta2 ? 2 * BM : BM;
        const uint32_t idesc = (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)gp.a_mn << 15) |
                               ((uint32_t)gp.b_mn << 16) | ((uint32_t)(BN >> 3) << 17) | ((mma_m >> 4) << 24);
        CUtensorMap tmC = tmA, tmD = tmA;  // placeholders when the TMA epilogue is not used
        bool tma_epi = false;
        if (G == 1) {
            tma_epi = f32_epi && make_epi_map(&tmD, d[b0].D, P, 3) &&
                      (P->beta_zero || make_epi_map(&tmC, const_cast<void*>(d[b0].C), P, 2));
        } else if (f32_epi && maps) {
            // one C and one D tensor map per batch of the group, in global memory
            bool ok = true;
            const int nm = P->beta_zero ? 1 : 2;
            for (int64_t b = 0; b < g && ok; b++) {
                ok = make_epi_map(&maps[b], d[b0 + b].D, P, 3) &&
                     (P->beta_zero || make_epi_map(&maps[g + b], const_cast<void*>(d[b0 + b].C), P, 2));
            }
            if (ok && stage_copy(dmaps, maps, sizeof(CUtensorMap) * (size_t)(nm * g), s) == cudaSuccess) {
                ep.tmDs = dmaps;
                ep.tmCs = P->beta_zero ? nullptr : dmaps + g;
                tma_epi = true;
            }
        }
        const int kind = tma_epi ? EPI_TMA : (f32_epi ? EPI_F32 : EPI_ANY);
        use_split_round(gp, sr);
        const int items = gp.num_tiles + gp.split_tiles;
        const int grid = (items < units ? items : units) * (cta2 ? 2 : 1);
        const bool timed = main_timer && b0 == 0;
        // the GEMM follows its last pack directly (a single product: no
        // staging copy between them; no timer event) as a programmatic
        // dependent launch: its CTAs start, set up their barriers and tensor
        // memory while the pack drains, and wait for the pack's grid
        // (griddepcontrol.wait) before their first global memory access
        const bool pdl = packs > 0 && G == 1 && !timed;
        if (timed) tbk_timer_begin(s, main_timer);
        e = launch_gemm(kind, cta2, grid, tmA, tmB, gp, idesc, tmC, tmD, s, cvt ? 1 : spl ? 2 : 0, pdl);
        if (timed) tbk_timer_end(s, *main_timer);
        if (sr.ws) cudaFreeAsync(sr.ws, s);
        count_launch();
        (*kernels)++;
        if (e != cudaSuccess) break;
    }
    if (dptr) cudaFreeAsync(dptr, s);
    if (dmaps) cudaFreeAsync(dmaps, s);
    free(maps);
    if (ws) cudaFreeAsync(ws, s);
    return e;
}

}  // namespace tb

// ---------------------------------------------------------------------------
// Allocation-free variant of the tensor-core product.
//
// Some callers cannot allocate device memory while they run a product: code
// that runs inside a host-side allocator callback or a memory manager, code
// that has reserved the whole device for its own pool, or code that must not
// touch the allocator at all once its setup is done. For them the packed
// operand panels and the kernel's error word live in the fixed array below
// instead of stream-ordered allocations.
//
//   - Every GPU that loads this library holds the array (TB_NOALLOC_SCRATCH
//     bytes) until the process exits.
//   - The array's device address is looked up once per device, with that
//     device current, on the first call there (cudaGetSymbolAddress; the name
//     of a __device__ array is only a host-side stand-in, not an address the
//     GPU can use), and again on the first call after a cudaDeviceReset gave
//     the device a new context. Make that first call before any stream
//     capture.
//   - All calls share the array and it keeps the last call's contents; calls
//     whose work overlaps on the GPU (other streams, or several host threads)
//     race on it. The pack kernels write every panel element the GEMM reads,
//     padding included; only the error word has to start at zero and is
//     cleared at set-up and after each reported error.
//   - A synchronous call reads the error word after its kernels; an
//     asynchronous call cannot, so a wait that expired in it is reported by
//     the next synchronous call on the same device.
namespace tb {
namespace tc {

constexpr size_t NOALLOC_SCRATCH = (size_t)32 << 20;  // 32 MiB
constexpr size_t NOALLOC_RESERVED = 256;              // error word + padding at the front

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH];

static void* g_noalloc_ptr[64];
static unsigned long long g_noalloc_ctx[64];  // id of the context the address belongs to
static std::mutex g_noalloc_mutex;

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// Unique id of the current context (0 when the driver cannot tell). A
// cudaDeviceReset ends the context and the next one gets a new id, so an
// address looked up in the old one is not reused.
static unsigned long long current_ctx_id()
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)p;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)p;
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// device address of the array on the current device (set-up on first use in
// each context of the device)
static cudaError_t noalloc_base(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    // 0 when the driver cannot name the context: the address is then kept
    // for the life of the process
    const unsigned long long ctx = g_noalloc_ptr[dev] ? current_ctx_id() : 0;
    if (!g_noalloc_ptr[dev] || (ctx != 0 && g_noalloc_ctx[dev] != ctx)) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the device's context current
        if (e != cudaSuccess) return e;
        e = cudaMemset(p, 0, NOALLOC_RESERVED);  // error word starts at zero
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
        g_noalloc_ctx[dev] = current_ctx_id();
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

}  // namespace tc
}  // namespace tb

extern "C" {

size_t tbk_noalloc_capacity(void) { return tb::tc::NOALLOC_SCRATCH - tb::tc::NOALLOC_RESERVED; }

// Scratch bytes the tensor-core path needs for this plan.
size_t tbk_tc_scratch_bytes(const tb_plan* P)
{
    using namespace tb::tc;
    const int cplx = P->compute == TB_C32;
    const int split = P->tc_mode == TB_TC_SPLIT_BF16 ? 3 : 1;
    const int64_t Kseg = round_up(P->K.size * (cplx ? 2 : 1), 8);
    const int64_t Kld = Kseg * split;
    const int64_t Nout = P->N.size * (cplx ? 2 : 1);
    return (size_t)round_up((int64_t)P->L.size * P->M.size * Kld * 2, 256) +
           (size_t)round_up((int64_t)P->L.size * Nout * Kld * 2, 256);
}

// The tensor-core product of tb::launch_tc with its scratch taken from the
// fixed array. Returns cudaErrorMemoryAllocation, without launching, when the
// plan needs more than tbk_noalloc_capacity() bytes.
int tbk_run_plan_tc_noalloc(const tb_plan* P, const tb_ptrs* d, void* stream, int* kernels)
{
    using namespace tb;
    using namespace tb::tc;
    cudaStream_t s = (cudaStream_t)stream;
    *kernels = 0;
    if (P->path != TB_PATH_TC) return (int)cudaErrorInvalidValue;
    if (tbk_tc_scratch_bytes(P) > tbk_noalloc_capacity()) return (int)cudaErrorMemoryAllocation;
    void* base = nullptr;
    cudaError_t e = noalloc_base(&base);
    if (e != cudaSuccess) return (int)e;
    int* flag = (int*)base;
    char* ws = (char*)base + NOALLOC_RESERVED;

    const int cplx = P->compute == TB_C32;
    const int split = P->tc_mode == TB_TC_SPLIT_BF16 ? 3 : 1;
    const int fmt = P->tc_mode == TB_TC_F16 ? 1 : 0;
    const int64_t M = P->M.size, N = P->N.size, Lsz = P->L.size, K = P->K.size;
    const int64_t Kseg = round_up(K * (cplx ? 2 : 1), 8);
    const int64_t Kld = Kseg * split;
    const int64_t Nout = N * (cplx ? 2 : 1);
    void* pA = ws;
    void* pB = ws + round_up(Lsz * M * Kld * 2, 256);

    for (int side = 0; side < 2; side++) {
        PackParams pp;
        memset(&pp, 0, sizeof(pp));
        pp.src = side == 0 ? d->A : d->B;
        pp.dst = side == 0 ? pA : pB;
        pp.type = side == 0 ? P->tA : P->tB;
        pp.conj = side == 0 ? P->conjA : P->conjB;
        pp.round_mode = split == 3 ? TB_ROUND_NONE : P->round_in;
        pp.cplx = cplx;
        pp.is_B = side;
        pp.split = split;
        pp.fmt = fmt;
        pp.R = side == 0 ? M : N;
        pp.K = K;
        pp.Lsz = Lsz;
        pp.Kseg = Kseg;
        pp.Kld = Kld;
        pp.Rout = side == 0 ? M : Nout;
        fill_modes(pp.rows, side == 0 ? P->M : P->N, side, -1);
        fill_modes(pp.ks, P->K, side, -1);
        fill_modes(pp.ls, P->L, side, -1);
        fill_modes(pp.us, side == 0 ? P->UA : P->UB, side, -1);
        pp.usize = side == 0 ? P->UA.size : P->UB.size;
        pp.rows_fast = min_stride(side == 0 ? P->M : P->N, side) < min_stride(P->K, side);
        if (!cplx && pp.us.n == 0 && (pp.type == T_F32 || pp.type == T_F64 || pp.type == T_F16 || pp.type == T_BF16)) {
            switch (pp.type) {
            case T_F32: launch_pack_real<float>(pp, split, fmt, pp.Lsz, true, s); break;
            case T_F64: launch_pack_real<double>(pp, split, fmt, pp.Lsz, true, s); break;
            case T_F16: launch_pack_real<__half>(pp, split, fmt, pp.Lsz, true, s); break;
            default: launch_pack_real<__nv_bfloat16>(pp, split, fmt, pp.Lsz, true, s); break;
            }
        } else {
            dim3 grid((unsigned)((pp.R + PR - 1) / PR), (unsigned)((Kseg / (cplx ? 2 : 1) + PK - 1) / PK),
                      (unsigned)Lsz);
            k_pack<<<grid, 256, 0, s>>>(pp);
        }
        count_launch();
        (*kernels)++;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return (int)e;

    CUtensorMap tmA, tmB;
    if (!make_map(&tmA, pA, fmt, Kld, M, Lsz, BM) || !make_map(&tmB, pB, fmt, Kld, Nout, Lsz, BN))
        return (int)cudaErrorInvalidValue;
    GemmParams gp;
    memset(&gp, 0, sizeof(gp));
    gp.tiles_m = (int)((M + BM - 1) / BM);
    gp.tiles_n = (int)((Nout + BN - 1) / BN);
    gp.num_tiles = gp.tiles_m * gp.tiles_n * (int)Lsz;
    gp.num_kb = (int)((Kld + BK - 1) / BK);
    gp.error = flag;
    EpiParams& ep = gp.e;
    ep.C = d->C;
    ep.D = d->D;
    ep.tC = P->tC;
    ep.tD = P->tD;
    ep.cplx = cplx;
    ep.beta_zero = P->beta_zero;
    ep.conjC = P->conjC;
    ep.conjD = P->conjD;
    ep.conjD_f32 = P->conjD_round_f32;
    ep.round_C = P->round_in;
    ep.alpha_re = (float)P->alpha_re;
    ep.alpha_im = (float)P->alpha_im;
    ep.beta_re = (float)P->beta_re;
    ep.beta_im = (float)P->beta_im;
    ep.M = M;
    ep.N = N;
    ep.L = Lsz;
    fill_modes(ep.mm, P->M, 2, 3);
    fill_modes(ep.nn, P->N, 2, 3);
    fill_modes(ep.ll, P->L, 2, 3);
    const uint32_t ab = fmt == 1 ? 0u : 1u;
    const uint32_t idesc = (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
    const bool f32_epi = !cplx && P->tD == T_F32 && (P->beta_zero || P->tC == T_F32) && !P->conjD;
    CUtensorMap tmC = tmA, tmD = tmA;
    const bool tma_epi = f32_epi && make_epi_map(&tmD, d->D, P, 3) &&
                         (P->beta_zero || make_epi_map(&tmC, const_cast<void*>(d->C), P, 2));
    const int kind = tma_epi ? EPI_TMA : (f32_epi ? EPI_F32 : EPI_ANY);
    const int grid = gp.num_tiles < num_sms() ? gp.num_tiles : num_sms();
    e = launch_gemm(kind, false, grid, tmA, tmB, gp, idesc, tmC, tmD, s);
    count_launch();
    (*kernels)++;
    return (int)e;
}

// Runs k_wait_selftest with waits of limit_ns and copies its four words to
// out (synchronises; the flag and the words are allocated for the call).
int tbk_wait_selftest(unsigned long long limit_ns, int* out)
{
    int* d = nullptr;
    tb::count_allocation();
    cudaError_t e = cudaMalloc((void**)&d, 8 * sizeof(int));
    if (e != cudaSuccess) return (int)e;
    e = cudaMemset(d, 0, 8 * sizeof(int));
    if (e == cudaSuccess) {
        tb::tc::k_wait_selftest<<<1, 32>>>(d, d + 4, limit_ns);
        tb::count_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(out, d + 4, 4 * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return (int)e;
}

// How the tensor-core path loads a plan's operands when A and B start on
// 16-byte boundaries: 1 split-bfloat16 read in place by the converter warps
// (one launch), 0 otherwise (packed panels). No kernel launch or copy.
int tbk_tc_split_in_place(const tb_plan* P)
{
    tb::tc::CvtOperand ca, cb;
    const void* aligned = (const void*)(uintptr_t)256;
    if (P->path != TB_PATH_TC || P->tc_mode != TB_TC_SPLIT_BF16) return 0;
    return tb::split_route(P, tb::split_in_place(P, aligned, aligned, &ca, &cb)) == 1;
}

// Whether a plan can join a grouped tensor-core launch with operands A and B
// (group.cu). No device call.
int tbk_tc_groupable(const tb_plan* P, const void* A, const void* B)
{
    tb::tc::GroupItem g;
    tb_ptrs d = {A, B, nullptr, nullptr};
    return tb::group_item(P, &d, true, &g) ? 1 : 0;
}

// Whether the grouped kernel computes the same bits for a plan as the
// single-product path (TAPP_execute_product) does: the same operand values,
// the same order of MMAs along the contraction and the same epilogue. That
// holds unless the single product would run its split bfloat16 from
// three-segment panels (fewer than 256 rows) or hand a last round of tiles
// over as half contractions (more tiles than SM units). No device call.
int tbk_tc_group_same_as_solo(const tb_plan* P)
{
    using namespace tb;
    using namespace tb::tc;
    if (P->tc_mode == TB_TC_SPLIT_BF16 && !split_panels_ok(P)) return 0;
    const bool cta2 = P->M.size >= 2 * BM && num_sms() % 2 == 0;
    const int64_t tiles = ((P->M.size + (cta2 ? 2 * BM : BM) - 1) / (cta2 ? 2 * BM : BM)) *
                          ((P->N.size + BN - 1) / BN) * P->L.size;
    return tiles <= (cta2 ? num_sms() / 2 : num_sms());
}

// Reads and clears the error word of the allocation-free path (synchronises).
int tbk_noalloc_check_error(void)
{
    void* base = nullptr;
    cudaError_t e = tb::tc::noalloc_base(&base);
    if (e != cudaSuccess) return (int)e;
    int v = 0;
    e = cudaMemcpy(&v, base, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return (int)e;
    if (v) {
        cudaMemset(base, 0, sizeof(int));
        return (int)cudaErrorLaunchTimeout;
    }
    return 0;
}

}  // extern "C"
