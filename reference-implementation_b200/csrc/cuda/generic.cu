// CUDA-core product kernels for every shape, storage type and precision.
//
//   k_elementwise  one thread per element of D: decodes the free coordinates,
//                  then walks the contracted coordinates and, inside, the
//                  unary coordinates of A and of B. This is the reference's
//                  loop nest (reference_implementation/src/product.c:338-399)
//                  with the outer loop spread over threads.
//   k_reduce       one block per element of D for few outputs with a long
//                  contraction: the contracted range is split over the
//                  block's threads and combined with warp shuffles.
//
// Both evaluate D = op_D(alpha * sum op_A(A) op_B(B) + beta * op_C(C)) in the
// plan's compute domain (real/complex, binary32/binary64) and honour the
// plan's operand rounding for the 16-bit precisions.
#include <cstdio>

#include "tb_common.cuh"

namespace tb {

struct GenParams {
    int32_t nF, nK, nUA, nUB;
    int32_t tA, tB, tC, tD;
    int32_t round_in, conjA, conjB, conjC, conjD, conjD_f32, beta_zero, small_F;
    int32_t warp, pad_;  // warp: one warp per output (warp_element), else one thread (element)
    int64_t sizeF, sizeK, sizeUA, sizeUB;
    double alpha_re, alpha_im, beta_re, beta_im;
    FastDiv fF[TB_MAXMODES];
    int64_t F_ext[TB_MAXMODES], F_sA[TB_MAXMODES], F_sB[TB_MAXMODES], F_sC[TB_MAXMODES], F_sD[TB_MAXMODES];
    int64_t K_ext[TB_MAXMODES], K_sA[TB_MAXMODES], K_sB[TB_MAXMODES];
    FastDiv fK[TB_MAXMODES];
    int64_t UA_ext[TB_MAXMODES], UA_s[TB_MAXMODES];
    int64_t UB_ext[TB_MAXMODES], UB_s[TB_MAXMODES];
};

// complex helpers on (re, im) pairs; CPLX=false keeps only the real part
template <typename R, bool CPLX>
__device__ __forceinline__ void cmac(R& sr, R& si, R ar, R ai, R br, R bi)
{
    if (CPLX) {
        sr = fma(ar, br, sr);
        sr = fma(-ai, bi, sr);
        si = fma(ar, bi, si);
        si = fma(ai, br, si);
    } else {
        sr = fma(ar, br, sr);
    }
}

// sum over the unary coordinates of one operand at base offset `off`
template <typename R, bool CPLX>
__device__ __forceinline__ void unary_sum(const void* base, int64_t off, int t, int conj, int rmode, int n,
                                          int64_t size, const int64_t* ext, const int64_t* str, R& re, R& im)
{
    if (n == 0) {
        load_rounded<R>(base, off, t, rmode, re, im);
        if (conj) im = -im;
        return;
    }
    re = 0;
    im = 0;
    int64_t c[TB_MAXMODES];
    for (int j = 0; j < n; j++) c[j] = 0;
    int64_t o = off;
    for (int64_t u = 0; u < size; u++) {
        R xr, xi;
        load_elem<R>(base, o, t, xr, xi);
        if (conj) xi = -xi;
        re += xr;
        im += xi;
        if (rmode != TB_ROUND_NONE) {  // the 16-bit precisions keep the running sum in 16 bits
            re = round_in<R>(re, rmode);
            im = round_in<R>(im, rmode);
        }
        for (int j = 0; j < n; j++) {
            o += str[j];
            if (++c[j] < ext[j]) break;
            o -= str[j] * ext[j];
            c[j] = 0;
        }
    }
}

template <typename R, bool CPLX>
__device__ __forceinline__ void finish(const GenParams& p, R sr, R si, const void* C, int64_t oC, void* D, int64_t oD)
{
    // alpha * sum
    R ar = (R)p.alpha_re, ai = (R)p.alpha_im;
    R accr, acci;
    if (CPLX) {
        accr = ar * sr - ai * si;
        acci = ar * si + ai * sr;
    } else {
        accr = ar * sr;
        acci = 0;
    }
    if (!p.beta_zero) {
        R cr, ci;
        load_rounded<R>(C, oC, p.tC, p.round_in, cr, ci);
        if (p.conjC) ci = -ci;
        R br = (R)p.beta_re, bi = (R)p.beta_im;
        if (CPLX) {
            accr += br * cr - bi * ci;
            acci += br * ci + bi * cr;
        } else {
            accr += br * cr;
        }
    }
    if (p.conjD) {
        if (p.conjD_f32) {
            accr = (R)(float)accr;
            acci = (R)(float)acci;
        }
        acci = -acci;
    }
    store_elem<R>(D, oD, p.tD, accr, acci);
}

// offsets in A, B, C and D of the free coordinates of output index i
__device__ __forceinline__ void free_offsets(const GenParams& p, int64_t i, int64_t& oA, int64_t& oB, int64_t& oC,
                                             int64_t& oD)
{
    oA = oB = oC = oD = 0;
    if (p.small_F) {
        uint32_t r = (uint32_t)i;
        for (int j = 0; j < p.nF; j++) {
            uint32_t q = fdiv(r, p.fF[j]);
            int64_t c = r - q * p.fF[j].d;
            r = q;
            oA += c * p.F_sA[j];
            oB += c * p.F_sB[j];
            oC += c * p.F_sC[j];
            oD += c * p.F_sD[j];
        }
    } else {
        int64_t r = i;
        for (int j = 0; j < p.nF; j++) {
            int64_t c = r % p.F_ext[j];
            r /= p.F_ext[j];
            oA += c * p.F_sA[j];
            oB += c * p.F_sB[j];
            oC += c * p.F_sC[j];
            oD += c * p.F_sD[j];
        }
    }
}

// one element of D: the reference's loop nest for output index i
template <typename R, bool CPLX>
__device__ __forceinline__ void element(const GenParams& p, const void* A, const void* B, const void* C, void* D,
                                        int64_t i)
{
    int64_t oA, oB, oC, oD;
    free_offsets(p, i, oA, oB, oC, oD);
    R sr = 0, si = 0;
    int64_t kc[TB_MAXMODES];
    for (int j = 0; j < p.nK; j++) kc[j] = 0;
    int64_t kA = oA, kB = oB;
    int64_t k0 = 0;
    if (p.nUA == 0 && p.nUB == 0) {
        // no unary modes: UNR terms' loads issued together, then their
        // multiply-adds in order (the same values and order as below)
        constexpr int UNR = (CPLX || sizeof(R) == 8) ? 4 : 8;
        for (; k0 + UNR <= p.sizeK; k0 += UNR) {
            R ar[UNR], ai[UNR], br[UNR], bi[UNR];
#pragma unroll
            for (int u = 0; u < UNR; u++) {
                load_rounded<R>(A, kA, p.tA, p.round_in, ar[u], ai[u]);
                load_rounded<R>(B, kB, p.tB, p.round_in, br[u], bi[u]);
                for (int j = 0; j < p.nK; j++) {
                    kA += p.K_sA[j];
                    kB += p.K_sB[j];
                    if (++kc[j] < p.K_ext[j]) break;
                    kA -= p.K_sA[j] * p.K_ext[j];
                    kB -= p.K_sB[j] * p.K_ext[j];
                    kc[j] = 0;
                }
            }
#pragma unroll
            for (int u = 0; u < UNR; u++) {
                if (p.conjA) ai[u] = -ai[u];
                if (p.conjB) bi[u] = -bi[u];
                cmac<R, CPLX>(sr, si, ar[u], ai[u], br[u], bi[u]);
            }
        }
    }
    for (int64_t k = k0; k < p.sizeK; k++) {
        R ar, ai, br, bi;
        unary_sum<R, CPLX>(A, kA, p.tA, p.conjA, p.round_in, p.nUA, p.sizeUA, p.UA_ext, p.UA_s, ar, ai);
        unary_sum<R, CPLX>(B, kB, p.tB, p.conjB, p.round_in, p.nUB, p.sizeUB, p.UB_ext, p.UB_s, br, bi);
        cmac<R, CPLX>(sr, si, ar, ai, br, bi);
        for (int j = 0; j < p.nK; j++) {
            kA += p.K_sA[j];
            kB += p.K_sB[j];
            if (++kc[j] < p.K_ext[j]) break;
            kA -= p.K_sA[j] * p.K_ext[j];
            kB -= p.K_sB[j] * p.K_ext[j];
            kc[j] = 0;
        }
    }
    finish<R, CPLX>(p, sr, si, C, oC, D, oD);
}

template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) k_elementwise(GenParams p, const void* A, const void* B, const void* C, void* D)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.sizeF; i += stride)
        element<R, CPLX>(p, A, B, C, D, i);
}

// One warp per element of D for products whose contraction runs along an
// operand's contiguous mode while consecutive outputs do not (batched
// matrix-vector and Hadamard products with A stored contraction-fastest):
// the lanes take every 32nd term (lane j the terms j, j + 32, ...), so each
// load of the warp reads 32 neighbouring elements instead of 32 elements a
// whole row apart, and a shuffle tree adds the 32 partial sums (a fixed
// order: the same bits in every run).
template <typename R, bool CPLX>
__device__ __forceinline__ void warp_element(const GenParams& p, const void* A, const void* B, const void* C, void* D,
                                             int64_t i, int lane)
{
    {
        int64_t oA, oB, oC, oD;
        free_offsets(p, i, oA, oB, oC, oD);
        R sr = 0, si = 0;
        auto term_offsets = [&](int64_t k, int64_t& kA, int64_t& kB) {
            kA = oA;
            kB = oB;
            uint32_t r = (uint32_t)k;
            for (int j = 0; j < p.nK; j++) {
                const uint32_t q = j + 1 < p.nK ? fdiv(r, p.fK[j]) : 0;
                const int64_t c = j + 1 < p.nK ? (int64_t)(r - q * p.fK[j].d) : (int64_t)r;
                r = q;
                kA += c * p.K_sA[j];
                kB += c * p.K_sB[j];
            }
        };
        int64_t k0 = lane;
        if (p.nUA == 0 && p.nUB == 0) {
            // the lane's next 4 terms loaded together, then added in order
            for (; k0 + 3 * 32 < p.sizeK; k0 += 4 * 32) {
                R ar[4], ai[4], br[4], bi[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    int64_t kA, kB;
                    term_offsets(k0 + 32 * u, kA, kB);
                    load_rounded<R>(A, kA, p.tA, p.round_in, ar[u], ai[u]);
                    load_rounded<R>(B, kB, p.tB, p.round_in, br[u], bi[u]);
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (p.conjA) ai[u] = -ai[u];
                    if (p.conjB) bi[u] = -bi[u];
                    cmac<R, CPLX>(sr, si, ar[u], ai[u], br[u], bi[u]);
                }
            }
        }
        for (int64_t k = k0; k < p.sizeK; k += 32) {
            int64_t kA, kB;
            term_offsets(k, kA, kB);
            R ar, ai, br, bi;
            unary_sum<R, CPLX>(A, kA, p.tA, p.conjA, p.round_in, p.nUA, p.sizeUA, p.UA_ext, p.UA_s, ar, ai);
            unary_sum<R, CPLX>(B, kB, p.tB, p.conjB, p.round_in, p.nUB, p.sizeUB, p.UB_ext, p.UB_s, br, bi);
            cmac<R, CPLX>(sr, si, ar, ai, br, bi);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            if (CPLX) si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (lane == 0) finish<R, CPLX>(p, sr, si, C, oC, D, oD);
    }
}

template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) k_warpdot(GenParams p, const void* A, const void* B, const void* C, void* D)
{
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < p.sizeF; i += warps)
        warp_element<R, CPLX>(p, A, B, C, D, i, threadIdx.x & 31);
}

// Many independent products of the same compute domain in one launch:
// product j owns blocks [first[j], first[j+1]) and walks its elements with
// them. Descriptors and operand pointers live in device memory.
template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) k_elementwise_group(const GenParams* __restrict__ params,
                                                           const tb_ptrs* __restrict__ ptrs,
                                                           const int64_t* __restrict__ first, int n)
{
    int lo = 0, hi = n - 1;  // last j with first[j] <= blockIdx.x
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= (int64_t)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const GenParams& p = params[lo];
    const tb_ptrs q = ptrs[lo];
    const int64_t nb = first[lo + 1] - first[lo];
    if (p.warp) {
        const int64_t warps = nb * (blockDim.x >> 5);
        for (int64_t i = ((int64_t)blockIdx.x - first[lo]) * (blockDim.x >> 5) + (threadIdx.x >> 5); i < p.sizeF;
             i += warps)
            warp_element<R, CPLX>(p, q.A, q.B, q.C, q.D, i, threadIdx.x & 31);
        return;
    }
    const int64_t stride = nb * blockDim.x;
    for (int64_t i = ((int64_t)blockIdx.x - first[lo]) * blockDim.x + threadIdx.x; i < p.sizeF; i += stride)
        element<R, CPLX>(p, q.A, q.B, q.C, q.D, i);
}

template <typename R>
__device__ __forceinline__ R warp_sum(R v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Few outputs, long contraction: block (x, y) sums the y-th chunk of the
// contracted range of output x with all its threads (combined by warp
// shuffles). With one chunk the block finishes the output itself; with
// several, each chunk's sum goes to a workspace and k_reduce_final adds the
// chunks in order and finishes, so the result does not depend on scheduling.
template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) k_reduce(GenParams p, const void* A, const void* B, const void* C, void* D,
                                                int64_t chunk, R* ws)
{
    __shared__ R red[2][8];
    const int64_t kbeg = (int64_t)blockIdx.y * chunk;
    const int64_t kend = kbeg + chunk < p.sizeK ? kbeg + chunk : p.sizeK;
    for (int64_t i = blockIdx.x; i < p.sizeF; i += gridDim.x) {
        int64_t oA = 0, oB = 0, oC = 0, oD = 0;
        int64_t r = i;
        for (int j = 0; j < p.nF; j++) {
            int64_t c = r % p.F_ext[j];
            r /= p.F_ext[j];
            oA += c * p.F_sA[j];
            oB += c * p.F_sB[j];
            oC += c * p.F_sC[j];
            oD += c * p.F_sD[j];
        }
        R sr = 0, si = 0;
        for (int64_t k = kbeg + threadIdx.x; k < kend; k += blockDim.x) {
            uint32_t rk = (uint32_t)k;
            int64_t kA = oA, kB = oB;
            for (int j = 0; j < p.nK; j++) {
                uint32_t q = fdiv(rk, p.fK[j]);
                int64_t c = rk - q * p.fK[j].d;
                rk = q;
                kA += c * p.K_sA[j];
                kB += c * p.K_sB[j];
            }
            R ar, ai, br, bi;
            unary_sum<R, CPLX>(A, kA, p.tA, p.conjA, p.round_in, p.nUA, p.sizeUA, p.UA_ext, p.UA_s, ar, ai);
            unary_sum<R, CPLX>(B, kB, p.tB, p.conjB, p.round_in, p.nUB, p.sizeUB, p.UB_ext, p.UB_s, br, bi);
            cmac<R, CPLX>(sr, si, ar, ai, br, bi);
        }
        sr = warp_sum(sr);
        if (CPLX) si = warp_sum(si);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        if (l == 0) { red[0][w] = sr; red[1][w] = si; }
        __syncthreads();
        if (threadIdx.x == 0) {
            R tr = 0, ti = 0;
            for (int j = 0; j < (int)(blockDim.x >> 5); j++) { tr += red[0][j]; ti += red[1][j]; }
            if (ws) {
                ws[(blockIdx.y * p.sizeF + i) * 2] = tr;
                ws[(blockIdx.y * p.sizeF + i) * 2 + 1] = ti;
            } else {
                finish<R, CPLX>(p, tr, ti, C, oC, D, oD);
            }
        }
        __syncthreads();
    }
}

template <typename R, bool CPLX>
__global__ void __launch_bounds__(256) k_reduce_final(GenParams p, const void* C, void* D, int chunks, const R* ws)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.sizeF; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t oC = 0, oD = 0, r = i;
        for (int j = 0; j < p.nF; j++) {
            int64_t c = r % p.F_ext[j];
            r /= p.F_ext[j];
            oC += c * p.F_sC[j];
            oD += c * p.F_sD[j];
        }
        R tr = 0, ti = 0;
        for (int z = 0; z < chunks; z++) {
            tr += ws[(z * p.sizeF + i) * 2];
            ti += ws[(z * p.sizeF + i) * 2 + 1];
        }
        finish<R, CPLX>(p, tr, ti, C, oC, D, oD);
    }
}

// chunks of the contraction for the reduction path: about 8 blocks per SM in
// all, every chunk at least 2048 terms long
static int reduce_chunks(int64_t outs, int64_t K)
{
    if (outs <= 0) return 1;
    int64_t S = (148 * 8 + outs - 1) / outs;
    const int64_t by_len = K / 2048;
    if (S > by_len) S = by_len;
    if (S > 4096) S = 4096;
    return S < 1 ? 1 : (int)S;
}

size_t reduce_scratch_bytes(const tb_plan* P, size_t real_bytes)
{
    const int S = reduce_chunks(P->F.size, P->K.size);
    return S > 1 ? (size_t)S * (size_t)P->F.size * 2 * real_bytes : 0;
}

static bool warpdot_ok(const GenParams& g);

static void fill_params(const tb_plan* P, GenParams& g)
{
    memset(&g, 0, sizeof(g));
    g.nF = P->F.n; g.nK = P->K.n; g.nUA = P->UA.n; g.nUB = P->UB.n;
    g.tA = P->tA; g.tB = P->tB; g.tC = P->tC; g.tD = P->tD;
    g.round_in = P->round_in;
    g.conjA = P->conjA; g.conjB = P->conjB; g.conjC = P->conjC; g.conjD = P->conjD;
    g.conjD_f32 = P->conjD_round_f32;
    g.beta_zero = P->beta_zero;
    g.sizeF = P->F.size; g.sizeK = P->K.size; g.sizeUA = P->UA.size; g.sizeUB = P->UB.size;
    g.alpha_re = P->alpha_re; g.alpha_im = P->alpha_im;
    g.beta_re = P->beta_re; g.beta_im = P->beta_im;
    g.small_F = P->F.size < (1ll << 31);
    for (int j = 0; j < P->F.n; j++) {
        g.F_ext[j] = P->F.ext[j];
        g.fF[j] = make_fastdiv(g.small_F ? (uint32_t)P->F.ext[j] : 1u);
        g.F_sA[j] = P->F.sA[j]; g.F_sB[j] = P->F.sB[j]; g.F_sC[j] = P->F.sC[j]; g.F_sD[j] = P->F.sD[j];
    }
    for (int j = 0; j < P->K.n; j++) {
        g.K_ext[j] = P->K.ext[j];
        g.fK[j] = make_fastdiv(P->K.size < (1ll << 31) ? (uint32_t)P->K.ext[j] : 1u);
        g.K_sA[j] = P->K.sA[j]; g.K_sB[j] = P->K.sB[j];
    }
    for (int j = 0; j < P->UA.n; j++) { g.UA_ext[j] = P->UA.ext[j]; g.UA_s[j] = P->UA.sA[j]; }
    for (int j = 0; j < P->UB.n; j++) { g.UB_ext[j] = P->UB.ext[j]; g.UB_s[j] = P->UB.sB[j]; }
    g.warp = warpdot_ok(g) ? 1 : 0;
}

// Element path kernel: the warp per output (k_warpdot)
//   - when an operand is contiguous along the contraction while consecutive
//     outputs step it by a stride other than 0 or 1 (one thread per output
//     would read it a row apart from lane to lane), for contractions of at
//     least 64 terms;
//   - when one thread per output makes less than a wave (fewer than 148 x 256
//     outputs) and each output sums at least 8 terms with at least 64 loads
//     in all (unary sums included): the lanes share the terms.
static bool warpdot_ok(const GenParams& g)
{
    if (g.sizeK >= (1ll << 31) || g.nK < 1 || g.nF < 1) return false;
    if (g.sizeF < 148 * 256 && g.sizeK >= 8 && (double)g.sizeK * (double)(g.sizeUA + g.sizeUB) >= 64.0) return true;
    if (g.sizeK < 64) return false;
    auto a = [](int64_t x) { return x < 0 ? -x : x; };
    // not when consecutive outputs already walk the other operand along its
    // contiguous mode (threads per output read that one in whole lines)
    const bool by_A = a(g.K_sA[0]) == 1 && a(g.F_sA[0]) > 1 && a(g.F_sB[0]) != 1;
    const bool by_B = a(g.K_sB[0]) == 1 && a(g.F_sB[0]) > 1 && a(g.F_sA[0]) != 1;
    return by_A || by_B;
}

template <typename R, bool CPLX>
static cudaError_t launch_typed(const GenParams& g, int path, const tb_ptrs* d, cudaStream_t s)
{
    if (path == TB_PATH_REDUCE && g.sizeK < (1ll << 31)) {
        const int S = reduce_chunks(g.sizeF, g.sizeK);
        int64_t bx = g.sizeF < 148 * 16 ? g.sizeF : 148 * 16;
        if (bx < 1) bx = 1;
        if (S == 1) {
            k_reduce<R, CPLX><<<(unsigned)bx, 256, 0, s>>>(g, d->A, d->B, d->C, d->D, g.sizeK, (R*)nullptr);
            count_launch();
            return cudaGetLastError();
        }
        const int64_t chunk = (g.sizeK + S - 1) / S;
        const int chunks = (int)((g.sizeK + chunk - 1) / chunk);
        void* ws = nullptr;
        cudaError_t e = pool_alloc(&ws, (size_t)chunks * (size_t)g.sizeF * 2 * sizeof(R), s);
        if (e != cudaSuccess) return e;
        k_reduce<R, CPLX><<<dim3((unsigned)bx, (unsigned)chunks), 256, 0, s>>>(g, d->A, d->B, d->C, d->D, chunk,
                                                                            (R*)ws);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            int64_t b2 = (g.sizeF + 255) / 256;
            if (b2 > 148 * 8) b2 = 148 * 8;
            k_reduce_final<R, CPLX><<<(unsigned)b2, 256, 0, s>>>(g, d->C, d->D, chunks, (const R*)ws);
            e = cudaGetLastError();
        }
        count_launch(2);
        cudaFreeAsync(ws, s);
        return e;
    } else if (g.warp) {
        int64_t blocks = (g.sizeF + 7) / 8;  // 8 warps, one output each
        if (blocks > 148 * 32) blocks = 148 * 32;
        if (blocks < 1) blocks = 1;
        k_warpdot<R, CPLX><<<(unsigned)blocks, 256, 0, s>>>(g, d->A, d->B, d->C, d->D);
    } else {
        int64_t blocks = (g.sizeF + 255) / 256;
        if (blocks > 148 * 64) blocks = 148 * 64;
        if (blocks < 1) blocks = 1;
        k_elementwise<R, CPLX><<<(unsigned)blocks, 256, 0, s>>>(g, d->A, d->B, d->C, d->D);
    }
    count_launch();
    return cudaGetLastError();
}

size_t group_descriptor_bytes(int n)
{
    return (size_t)n * sizeof(GenParams) + (size_t)n * sizeof(tb_ptrs) + (size_t)(n + 1) * sizeof(int64_t) + 64;
}

// Fills `host` (pinned, group_descriptor_bytes(n)) with the descriptors of n
// products of one compute domain, copies it to `dev` and launches one grouped
// kernel. The host buffer must stay untouched until the copy has run.
cudaError_t launch_generic_group(const tb_plan* const* P, const tb_ptrs* d, int n, void* host, void* dev,
                                 cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    char* h = (char*)host;
    GenParams* hp = (GenParams*)h;
    tb_ptrs* hq = (tb_ptrs*)(h + (size_t)n * sizeof(GenParams));
    int64_t* hf = (int64_t*)(h + (size_t)n * (sizeof(GenParams) + sizeof(tb_ptrs)));
    int64_t blocks = 0;
    for (int j = 0; j < n; j++) {
        fill_params(P[j], hp[j]);
        hq[j] = d[j];
        hf[j] = blocks;
        // warp-per-output products: 8 outputs per block
        int64_t b = hp[j].warp ? (P[j]->F.size + 7) / 8 : (P[j]->F.size + 255) / 256;
        if (b > 148 * 8) b = 148 * 8;
        if (b < 1) b = 1;
        blocks += b;
    }
    hf[n] = blocks;
    const size_t bytes = group_descriptor_bytes(n);
    cudaError_t e = cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    char* dv = (char*)dev;
    const GenParams* dp = (const GenParams*)dv;
    const tb_ptrs* dq = (const tb_ptrs*)(dv + (size_t)n * sizeof(GenParams));
    const int64_t* df = (const int64_t*)(dv + (size_t)n * (sizeof(GenParams) + sizeof(tb_ptrs)));
    if (blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
    switch (P[0]->compute) {
    case TB_R32: k_elementwise_group<float, false><<<(unsigned)blocks, 256, 0, s>>>(dp, dq, df, n); break;
    case TB_R64: k_elementwise_group<double, false><<<(unsigned)blocks, 256, 0, s>>>(dp, dq, df, n); break;
    case TB_C32: k_elementwise_group<float, true><<<(unsigned)blocks, 256, 0, s>>>(dp, dq, df, n); break;
    default: k_elementwise_group<double, true><<<(unsigned)blocks, 256, 0, s>>>(dp, dq, df, n); break;
    }
    count_launch();
    return cudaGetLastError();
}

// Copy of one operand (its free, contracted and unary modes) into a dense
// buffer whose first mode is the first output mode and whose other modes
// follow in free, contracted, unary order, so that the element kernel reads
// it along its walk of the outputs instead of one line per lane. Element
// values are copied as stored (2-byte elements, or 4-byte words).
struct StageParams {
    const unsigned char* src;
    unsigned char* dst;
    int32_t n, words;  // modes; 4-byte words per element (0: one 2-byte element)
    int64_t size;
    int64_t s[3 * TB_MAXMODES];  // source strides, in elements
    FastDiv f[3 * TB_MAXMODES];
};

__global__ void __launch_bounds__(256) k_stage(StageParams p)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.size; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t r = (uint32_t)i;
        int64_t o = 0;
        for (int j = 0; j < p.n; j++) {
            const uint32_t q = fdiv(r, p.f[j]);
            o += (int64_t)(r - q * p.f[j].d) * p.s[j];
            r = q;
        }
        if (p.words == 0) {
            ((uint16_t*)p.dst)[i] = __ldg((const uint16_t*)p.src + o);
        } else {
            for (int w = 0; w < p.words; w++)
                ((uint32_t*)p.dst)[i * p.words + w] = __ldg((const uint32_t*)p.src + o * p.words + w);
        }
    }
}

static int stored_bytes(int t)
{
    switch (t) {
    case T_F32: return 4;
    case T_F64: return 8;
    case T_C32: return 8;
    case T_C64: return 16;
    default: return 2;
    }
}

// The operand `side` (0 A, 1 B) of the element path copied into scratch in
// the order of the output walk; g's strides and d's pointer then refer to
// the copy. *ws: the scratch, to be freed after the element kernel.
static cudaError_t stage_operand(const tb_plan* P, int side, GenParams& g, tb_ptrs& d, void** ws, cudaStream_t s)
{
    StageParams sp;
    memset(&sp, 0, sizeof(sp));
    int64_t* F_s = side ? g.F_sB : g.F_sA;
    int64_t* K_s = side ? g.K_sB : g.K_sA;
    int64_t* U_s = side ? g.UB_s : g.UA_s;
    const tb_modes& U = side ? P->UB : P->UA;
    int n = 0;
    int64_t acc = 1;
    auto add = [&](int64_t ext, int64_t& stride) {
        sp.s[n] = stride;
        sp.f[n] = make_fastdiv((uint32_t)ext);
        n++;
        stride = acc;
        acc *= ext;
    };
    for (int j = 0; j < P->F.n; j++)
        if (F_s[j] != 0) add(P->F.ext[j], F_s[j]);
    for (int j = 0; j < P->K.n; j++) add(P->K.ext[j], K_s[j]);
    for (int j = 0; j < U.n; j++) add(U.ext[j], U_s[j]);
    if (acc >= (1ll << 31)) return cudaErrorInvalidValue;
    const int tY = side ? P->tB : P->tA;
    const int eb = stored_bytes(tY);
    sp.n = n;
    sp.words = eb / 4;
    sp.size = acc;
    sp.src = (const unsigned char*)(side ? d.B : d.A);
    cudaError_t e = pool_alloc(ws, (size_t)acc * (size_t)eb, s);
    if (e != cudaSuccess) return e;
    sp.dst = (unsigned char*)*ws;
    int64_t blocks = (acc + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_stage<<<(unsigned)blocks, 256, 0, s>>>(sp);
    count_launch();
    if (side) d.B = *ws;
    else d.A = *ws;
    return cudaGetLastError();
}

cudaError_t launch_generic(const tb_plan* P, const tb_ptrs* d, cudaStream_t s, int* kernels)
{
    GenParams g;
    fill_params(P, g);
    *kernels = 1;
    tb_ptrs dd = *d;
    void* ws = nullptr;
    if (P->path == TB_PATH_GENERIC && P->elem_stage && !g.warp) {
        cudaError_t e = stage_operand(P, P->elem_stage - 1, g, dd, &ws, s);
        if (e != cudaSuccess) {
            if (ws) cudaFreeAsync(ws, s);
            return e;
        }
        *kernels = 2;
    }
    cudaError_t e = cudaErrorInvalidValue;
    switch (P->compute) {
    case TB_R32: e = launch_typed<float, false>(g, P->path, &dd, s); break;
    case TB_R64: e = launch_typed<double, false>(g, P->path, &dd, s); break;
    case TB_C32: e = launch_typed<float, true>(g, P->path, &dd, s); break;
    case TB_C64: e = launch_typed<double, true>(g, P->path, &dd, s); break;
    }
    if (ws) cudaFreeAsync(ws, s);
    return e;
}

}  // namespace tb

// ---------------------------------------------------------------------------
// Device-resident request loop (host side: host/loop.c). A persistent kernel
// of G blocks serves small products as they arrive, without a launch per
// product. The host writes product t's descriptor into slot t % R of a ring
// in page-locked host memory mapped into the device, then the slot's
// sequence word (t + 1) last. Block 0 polls that word (system-scope acquire
// loads, a short sleep between polls), copies the descriptor into the same
// slot of a ring in device memory and raises its device sequence word; the
// other blocks poll the device word (an L2 read instead of a PCIe read).
// Every block then computes its share of D's elements (element i on block
// i / 256 mod G) with the element kernel's own per-output function, so the
// bits equal TAPP_execute_product's on the element path; the last block to
// finish (an arrival counter per slot) publishes t + 1 in the host slot's
// completion word after a system fence. A block that sees no new product for
// idle_ns stores the ticket it waits for in device memory and returns, so
// the loop never spins without a bound; the host relaunches it when
// products arrive again and the last launch has ended.
namespace tb {

struct LoopSlot {
    GenParams p;
    tb_ptrs q;
    int32_t compute;
    int32_t warp;    // 1: one warp per output (the kernel TAPP_execute_product would run)
    int64_t seq;     // t + 1 once the descriptor of ticket t is complete (written last)
    int64_t done;    // t + 1 once ticket t's D is written
    int64_t pad2[6];
};

struct LoopParams {
    LoopSlot* slots;      // device pointer of the mapped ring
    LoopSlot* dslots;     // ring in device memory: block 0's copies
    int64_t* dseq;        // device memory: t + 1 once dslots[t % R] holds ticket t
    int* arrive;          // device memory: blocks done with the slot's current ticket
    int64_t* next;        // device memory: per block, the ticket it serves next
    int32_t nslots;
    int32_t pad;
    unsigned long long idle_ns;
};

__device__ __forceinline__ unsigned long long loop_now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int64_t ld_acquire_sys(const int64_t* p)
{
    int64_t v;
    asm volatile("ld.acquire.sys.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int64_t ld_acquire_gpu(const int64_t* p)
{
    int64_t v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_sys(int64_t* p, int64_t v)
{
    asm volatile("st.release.sys.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release_gpu(int64_t* p, int64_t v)
{
    asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

template <typename R, bool CPLX>
__device__ __forceinline__ void loop_product(const GenParams& p, const tb_ptrs& q, int warp)
{
    if (warp) {
        const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
        for (int64_t i = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < p.sizeF; i += warps)
            warp_element<R, CPLX>(p, q.A, q.B, q.C, q.D, i, threadIdx.x & 31);
        return;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.sizeF; i += stride)
        element<R, CPLX>(p, q.A, q.B, q.C, q.D, i);
}

__global__ void __launch_bounds__(256) k_request_loop(LoopParams lp)
{
    __shared__ GenParams sp;
    __shared__ tb_ptrs sq;
    __shared__ int scomp, swarp, go;
    const int b = blockIdx.x;
    int64_t t = lp.next[b];
    unsigned long long last = loop_now_ns();
    for (;;) {
        const int64_t s = t % lp.nslots;
        LoopSlot* hs = &lp.slots[s];
        LoopSlot* ds = &lp.dslots[s];
        if (threadIdx.x == 0) {
            // block 0 watches the host ring, the others the device copy
            const int64_t* word = b == 0 ? &hs->seq : &lp.dseq[s];
            int posted = 0;
            for (;;) {
                if ((b == 0 ? ld_acquire_sys(word) : ld_acquire_gpu(word)) == t + 1) {
                    posted = 1;
                    break;
                }
                if (loop_now_ns() - last > lp.idle_ns) break;
                __nanosleep(b == 0 ? 256 : 128);
            }
            go = posted;
        }
        __syncthreads();
        if (!go) break;
        {
            // the descriptor into shared memory: from host memory on block 0
            // (which also fills the device copy), from the device copy elsewhere
            const volatile int64_t* src = (const volatile int64_t*)(b == 0 ? &hs->p : &ds->p);
            int64_t* dst = (int64_t*)&sp;
            int64_t* dcopy = (int64_t*)&ds->p;
            for (int w = threadIdx.x; w < (int)(sizeof(GenParams) / 8); w += blockDim.x) {
                const int64_t v = src[w];
                dst[w] = v;
                if (b == 0) dcopy[w] = v;
            }
            if (threadIdx.x == 0) {
                const volatile tb_ptrs* vq = b == 0 ? &hs->q : &ds->q;
                sq.A = vq->A;
                sq.B = vq->B;
                sq.C = vq->C;
                sq.D = vq->D;
                scomp = *(const volatile int32_t*)(b == 0 ? &hs->compute : &ds->compute);
                swarp = *(const volatile int32_t*)(b == 0 ? &hs->warp : &ds->warp);
                if (b == 0) {
                    ds->q = sq;
                    ds->compute = scomp;
                    ds->warp = swarp;
                }
            }
        }
        __syncthreads();
        if (b == 0 && threadIdx.x == 0) {
            __threadfence();
            st_release_gpu(&lp.dseq[s], t + 1);  // the device copy is complete
        }
        switch (scomp) {
        case TB_R32: loop_product<float, false>(sp, sq, swarp); break;
        case TB_R64: loop_product<double, false>(sp, sq, swarp); break;
        case TB_C32: loop_product<float, true>(sp, sq, swarp); break;
        default: loop_product<double, true>(sp, sq, swarp); break;
        }
        __syncthreads();  // this block's outputs of the product written
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(&lp.arrive[s], 1) == (int)gridDim.x - 1) {
                // the last block: every output is written
                lp.arrive[s] = 0;
                __threadfence_system();
                st_release_sys(&hs->done, t + 1);
            }
        }
        t++;
        last = loop_now_ns();
    }
    if (threadIdx.x == 0) lp.next[b] = t;
}

size_t loop_slot_bytes() { return sizeof(LoopSlot); }

// Fills ring slot `slot` (host memory) with a product's descriptor, all
// but the sequence word.
void loop_fill(void* slot, const tb_plan* P, const tb_ptrs* d)
{
    LoopSlot* s = (LoopSlot*)slot;
    fill_params(P, s->p);
    if (P->path == TB_PATH_NOOP) s->p.sizeF = 0;  // nothing to write (empty D, or a precision left as is)
    s->q = *d;
    s->compute = P->compute;
    s->warp = s->p.warp;
}

// device state of a loop: the ring copy, its sequence words, the arrival
// counters and the per-block tickets (zeroed; every block starts at ticket 0)
size_t loop_state_bytes(int nslots, int blocks)
{
    return (size_t)nslots * (sizeof(LoopSlot) + sizeof(int64_t) + sizeof(int)) + (size_t)blocks * sizeof(int64_t) + 64;
}

cudaError_t loop_launch(void* slots_dev, void* state, int nslots, int blocks, unsigned long long idle_ns,
                        cudaStream_t s)
{
    LoopParams lp;
    char* st = (char*)state;
    lp.slots = (LoopSlot*)slots_dev;
    lp.dslots = (LoopSlot*)st;
    lp.dseq = (int64_t*)(st + (size_t)nslots * sizeof(LoopSlot));
    lp.next = lp.dseq + nslots;
    lp.arrive = (int*)(lp.next + blocks);
    lp.nslots = nslots;
    lp.pad = 0;
    lp.idle_ns = idle_ns;
    k_request_loop<<<blocks, 256, 0, s>>>(lp);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tb

// Kernel of the element path for a plan: 0 one thread per output, 1 one warp
// per output (k_warpdot). No device call.
extern "C" int tbk_generic_kernel(const tb_plan* P)
{
    tb::GenParams g;
    tb::fill_params(P, g);
    return g.warp;
}
