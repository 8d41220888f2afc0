// Sliced binary64 products on the integer tensor cores (an Ozaki-style
// scheme): TB_PATH_SLICED, chosen for binary64 / complex-double products when
// the executor asks for S slices (TAPP_B200_ATTR_F64_MODE = S).
//
// Every row r of A (over the contracted index k) gets the exponent E_r with
// |A[r,k]| < 2^E_r for all k; every column of B gets F_c the same way. Then
//     A[r,k] = 2^E_r (sum_{s<S} a_s[r,k] 2^(-7(s+1)) + e),  |e| < 2^(-7S),
// with signed 7-bit digits a_s in [-127, 127] taken by truncation
// (y <- 128 y, digit = trunc(y), y <- y - digit; every step is exact in
// binary64), and likewise for B. The product keeps the digit pairs with
// s + t < S:
//     D = alpha 2^(E_r + F_c) sum_{L<S} 2^(-7(L+2)) sum_{s+t=L} a_s . b_t
//         + beta C
// Each inner sum over k is an exact 32-bit integer product on tcgen05
// (kind::i8). The digits of one row are stored slice after slice,
// A8[l][r][s][k'], and those of B in reverse slice order, B8[l][c][S-1-t][k'],
// so that all pairs of one level L are ONE contiguous K range of both panels:
// the level is a single GEMM of (L+1) K-segments. Levels whose sum could
// reach 2^31 (pairs x K x 127^2) are cut into several GEMMs, and a contraction
// longer than 133,120 is cut into chunks. Each GEMM adds 2^(-7(L+2)) x its
// integer result into a binary64 workspace W (exact scaling, one rounding per
// addition); the finish kernel applies 2^(E+F), alpha, beta.C and op_D.
//
// Complex operands use the 4M real form of the tensor-core path: A rows hold
// (re, im) pairs along k, B contributes two rows per column, (re, -im) and
// (im, re); conjugation is folded in as a sign. A row or column holding a
// non-finite value gives NaN outputs (the scheme needs finite inputs).
#include <cstdio>
#include <cstring>

#include "../tb_cuda.h"
#include "tb_common.cuh"

namespace tb {

cudaError_t launch_gemm_i8(const void* A8, const void* B8, int64_t row_bytes, int64_t M, int64_t Nout, int64_t L,
                           int64_t a_off, int64_t b_off, int64_t klen, double* W, double scale, int first,
                           cudaStream_t s);

namespace sl {

constexpr int TR = 32;                  // source rows per slicing tile
constexpr int TK = 64;                  // digit bytes per slice row per tile
// Row exponents are kept as code = e + EXP_BIAS (0 for a zero row, EXP_BAD
// when the row holds a non-finite value), so that a zeroed array and
// atomicMax over blocks that each see part of a row give the row's code.
constexpr int EXP_BIAS = 2048;
constexpr int EXP_BAD = 1 << 20;
constexpr int64_t MAX_TERMS = 2147483647ll / (127 * 127);  // products per int32 sum
constexpr int64_t K_CHUNK = MAX_TERMS / 128 * 128;         // 133,120

struct Modes {
    int32_t n, pad;
    int64_t ext[TB_MAXMODES];
    int64_t s[TB_MAXMODES];
};

__host__ __device__ inline int64_t mode_offset(const Modes& m, int64_t idx)
{
    int64_t o = 0;
    for (int j = 0; j < m.n; j++) {
        o += (idx % m.ext[j]) * m.s[j];
        idx /= m.ext[j];
    }
    return o;
}

// offset tables: job j fills t_j[i] = offset of index i in modes m_j
struct OffsetJobs {
    int32_t n;
    int32_t pad;
    Modes m[8];
    int64_t len[8];
    int64_t* out[8];
};

__global__ void __launch_bounds__(256) k_offsets(OffsetJobs jobs)
{
    const int j = blockIdx.y;
    if (j >= jobs.n) return;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < jobs.len[j]; i += (int64_t)gridDim.x * blockDim.x)
        jobs.out[j][i] = mode_offset(jobs.m[j], i);
}

struct SliceParams {
    const void* src;
    int32_t type, conj, cplx, is_B, S, pad;
    int64_t R, K, Lsz;    // source rows, contracted length (complex elements), batch
    int64_t Kp;           // digit bytes per slice row (multiple of 16)
    int64_t Rout;         // panel rows: R, or 2R for complex B
    Modes ls;             // batch modes, source strides
    const int64_t* roff;  // [R] source offset of each row
    const int64_t* koff;  // [K] source offset of each contracted index
    int32_t* expo;        // [L][R]
    int8_t* dst;          // [L][Rout][S][Kp]
};

// code of x: 0 for zero, e + EXP_BIAS with |x| < 2^e (IEEE binary64
// fields), EXP_BAD for a non-finite value
__device__ __forceinline__ int exp_code(double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    const int be = (int)((b >> 52) & 0x7ff);
    if (be == 0x7ff) return EXP_BAD;
    if ((b << 1) == 0) return 0;
    return (be == 0 ? -1022 : be - 1022) + EXP_BIAS;
}

// 2^-e for a row code (0 for zero and non-finite rows: their digits are 0)
__device__ __forceinline__ double row_inverse(int code)
{
    return (code == 0 || code >= EXP_BAD) ? 0.0 : scalbn(1.0, EXP_BIAS - code);
}

// Row exponent codes, the contracted range split over grid.y; partial maxima
// meet in p.expo (zeroed first) by atomicMax. RF: rows contiguous in the
// source (threads along rows), otherwise one warp per row along k.
template <bool RF>
__global__ void __launch_bounds__(256, 4) k_exponents(SliceParams p, int64_t kchunk)
{
    __shared__ int part[8][TR];
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * TR;
    const int64_t l = blockIdx.z;
    const int64_t lo = mode_offset(p.ls, l);
    const int64_t kb = (int64_t)blockIdx.y * kchunk;
    const int64_t ke = kb + kchunk < p.K ? kb + kchunk : p.K;
    if (RF) {
        const int r = t % TR, kq = t / TR;
        int c = 0;
        if (r0 + r < p.R) {
            const int64_t ro = p.roff[r0 + r] + lo;
            int64_t k = kb + kq;
            // four loads in flight before their exponents are taken
            for (; k + 24 < ke; k += 32) {
                double re[4], im[4];
#pragma unroll
                for (int u = 0; u < 4; u++) load_elem<double>(p.src, ro + p.koff[k + 8 * u], p.type, re[u], im[u]);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    c = max(c, exp_code(re[u]));
                    if (p.cplx) c = max(c, exp_code(im[u]));
                }
            }
            for (; k < ke; k += 8) {
                double re, im;
                load_elem<double>(p.src, ro + p.koff[k], p.type, re, im);
                c = max(c, exp_code(re));
                if (p.cplx) c = max(c, exp_code(im));
            }
        }
        part[kq][r] = c;
        __syncthreads();
        if (t < TR && r0 + t < p.R) {
            int m = 0;
            for (int j = 0; j < 8; j++) m = max(m, part[j][t]);
            if (m) atomicMax(&p.expo[l * p.R + r0 + t], m);
        }
    } else {
        const int w = t >> 5, lane = t & 31;
        for (int i = 0; i < TR / 8; i++) {
            const int r = w * (TR / 8) + i;
            int c = 0;
            if (r0 + r < p.R) {
                const int64_t ro = p.roff[r0 + r] + lo;
                int64_t k = kb + lane;
                for (; k + 96 < ke; k += 128) {
                    double re[4], im[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) load_elem<double>(p.src, ro + p.koff[k + 32 * u], p.type, re[u], im[u]);
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        c = max(c, exp_code(re[u]));
                        if (p.cplx) c = max(c, exp_code(im[u]));
                    }
                }
                for (; k < ke; k += 32) {
                    double re, im;
                    load_elem<double>(p.src, ro + p.koff[k], p.type, re, im);
                    c = max(c, exp_code(re));
                    if (p.cplx) c = max(c, exp_code(im));
                }
            }
            for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
            if (lane == 0 && c && r0 + r < p.R) atomicMax(&p.expo[l * p.R + r0 + r], c);
        }
    }
}

// the S digits of 8 values, written as 8-byte groups of one slice row each
// (B's slices in reverse order)
__device__ __forceinline__ void put_digits(const SliceParams& p, int64_t out_row, int64_t kbyte, double (&y)[8])
{
    int8_t* base = p.dst + out_row * p.S * p.Kp + kbyte;
    for (int s = 0; s < p.S; s++) {
        const int pos = p.is_B ? p.S - 1 - s : s;
        uint32_t w[2] = {0u, 0u};
#pragma unroll
        for (int j = 0; j < 8; j++) {
            y[j] *= 128.0;
            const int d = (int)y[j];  // truncation toward zero, |d| <= 127
            y[j] -= (double)d;
            w[j >> 2] |= (uint32_t)(uint8_t)(int8_t)d << (8 * (j & 3));
        }
        *(uint2*)(base + (int64_t)pos * p.Kp) = make_uint2(w[0], w[1]);
    }
}

// digits of a TR x TK tile of the panel (TR source rows; TK digit bytes per
// slice row, i.e. TK source elements, or TK/2 complex ones)
template <bool RF, bool CPLX>
__global__ void __launch_bounds__(256) k_slice(SliceParams p)
{
    constexpr int TKS = CPLX ? TK / 2 : TK;
    __shared__ double tre[TR][TKS + 1];
    __shared__ double tim[CPLX ? TR : 1][CPLX ? TKS + 1 : 1];
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * TR;
    const int64_t kt = blockIdx.y;
    const int64_t l = blockIdx.z;
    const int64_t ks0 = kt * TKS;
    const int64_t lo = mode_offset(p.ls, l);
    // all of this thread's loads in flight before the shared-memory stores
    constexpr int PER = TR * TKS / 256;
    double lre[PER], lim[PER];
#pragma unroll
    for (int u = 0; u < PER; u++) {
        const int e = t + 256 * u;
        const int r = RF ? e % TR : e / TKS;
        const int kk = RF ? e / TR : e % TKS;
        lre[u] = 0.0;
        lim[u] = 0.0;
        if (r0 + r < p.R && ks0 + kk < p.K)
            load_elem<double>(p.src, p.roff[r0 + r] + lo + p.koff[ks0 + kk], p.type, lre[u], lim[u]);
    }
#pragma unroll
    for (int u = 0; u < PER; u++) {
        const int e = t + 256 * u;
        const int r = RF ? e % TR : e / TKS;
        const int kk = RF ? e / TR : e % TKS;
        tre[r][kk] = lre[u];
        if (CPLX) tim[r][kk] = p.conj ? -lim[u] : lim[u];
    }
    __syncthreads();
    const int r = t >> 3, kc = (t & 7) * 8;
    const int64_t kbyte = kt * TK + kc;
    if (r0 + r >= p.R || kbyte >= p.Kp) return;
    const double inv = row_inverse(p.expo[l * p.R + r0 + r]);
    if (!CPLX) {
        double y[8];
#pragma unroll
        for (int j = 0; j < 8; j++) y[j] = tre[r][kc + j] * inv;
        put_digits(p, l * p.Rout + r0 + r, kbyte, y);
    } else if (!p.is_B) {
        double y[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int kk = (kc + j) >> 1;
            y[j] = ((kc + j) & 1 ? tim[r][kk] : tre[r][kk]) * inv;
        }
        put_digits(p, l * p.Rout + r0 + r, kbyte, y);
    } else {
        // rows 2c: (re, -im), 2c + 1: (im, re)
        double y0[8], y1[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int kk = (kc + j) >> 1;
            const bool odd = (kc + j) & 1;
            y0[j] = (odd ? -tim[r][kk] : tre[r][kk]) * inv;
            y1[j] = (odd ? tre[r][kk] : tim[r][kk]) * inv;
        }
        put_digits(p, l * p.Rout + 2 * (r0 + r), kbyte, y0);
        put_digits(p, l * p.Rout + 2 * (r0 + r) + 1, kbyte, y1);
    }
}

struct FinishParams {
    const void* C;
    void* D;
    int32_t tC, tD, cplx, beta_zero, conjC, conjD, conjD_f32, round_C, m_fast, pad;
    double alpha_re, alpha_im, beta_re, beta_im;
    int64_t M, N, L, Nout;
    const double* W;
    const int32_t* expA;
    const int32_t* expB;
    const int64_t* mC;
    const int64_t* mD;
    const int64_t* nC;
    const int64_t* nD;
    Modes lC, lD;
};

// D = op_D(alpha 2^(E+F) W + beta op_C(C)) in binary64
template <bool CPLX>
__global__ void __launch_bounds__(256) k_sliced_finish(FinishParams p)
{
    const int64_t total = p.L * p.M * p.N;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t m, n, l;
        if (p.m_fast) {
            m = e % p.M;
            n = (e / p.M) % p.N;
        } else {
            n = e % p.N;
            m = (e / p.N) % p.M;
        }
        l = e / (p.M * p.N);
        // W is laid out [l][n][m] (n over the Nout real columns)
        const double* w = p.W + (l * p.Nout + (CPLX ? 2 * n : n)) * p.M + m;
        const int Ea = p.expA[l * p.M + m], Fb = p.expB[l * p.N + n];
        double xr, xi = 0.0;
        if (Ea >= EXP_BAD || Fb >= EXP_BAD) {
            xr = __longlong_as_double(0x7ff8000000000000ll);
            xi = CPLX ? xr : 0.0;
        } else if (Ea == 0 || Fb == 0) {
            xr = 0.0;
        } else {
            const int sh = Ea + Fb - 2 * EXP_BIAS;
            xr = scalbn(w[0], sh);
            if (CPLX) xi = scalbn(w[p.M], sh);
        }
        double vr = p.alpha_re * xr - (CPLX ? p.alpha_im * xi : 0.0);
        double vi = CPLX ? p.alpha_re * xi + p.alpha_im * xr : 0.0;
        const int64_t oc = p.mC[m] + p.nC[n] + mode_offset(p.lC, l);
        const int64_t od = p.mD[m] + p.nD[n] + mode_offset(p.lD, l);
        if (!p.beta_zero) {
            double cr, ci;
            load_rounded<double>(p.C, oc, p.tC, p.round_C, cr, ci);
            if (p.conjC) ci = -ci;
            vr = fma(p.beta_re, cr, vr);
            if (CPLX) {
                vr = fma(-p.beta_im, ci, vr);
                vi = fma(p.beta_re, ci, fma(p.beta_im, cr, vi));
            }
        }
        if (p.conjD) {
            if (p.conjD_f32) {
                vr = (double)(float)vr;
                vi = (double)(float)vi;
            }
            vi = -vi;
        }
        store_elem<double>(p.D, od, p.tD, vr, vi);
    }
}

static void fill(Modes& m, const tb_modes& src, int which)
{
    memset(&m, 0, sizeof(m));
    m.n = src.n;
    const int64_t* st[4] = {src.sA, src.sB, src.sC, src.sD};
    for (int j = 0; j < src.n; j++) {
        m.ext[j] = src.ext[j];
        m.s[j] = st[which][j];
    }
}

static int64_t min_abs(const tb_modes& m, int which)
{
    const int64_t* st[4] = {m.sA, m.sB, m.sC, m.sD};
    int64_t best = INT64_MAX;
    for (int j = 0; j < m.n; j++) {
        const int64_t v = st[which][j] < 0 ? -st[which][j] : st[which][j];
        if (v && v < best) best = v;
    }
    return best;
}

static int64_t up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// scratch layout of one sliced product
struct Layout {
    int64_t Kreal, Kp, row_bytes, Nout;
    size_t oA8, oB8, oW, oEA, oEB, oT, total;
};

static Layout layout(const tb_plan* P)
{
    Layout y;
    const int cplx = P->compute == TB_C64;
    const int64_t M = P->M.size, N = P->N.size, L = P->L.size, K = P->K.size;
    y.Kreal = K * (cplx ? 2 : 1);
    y.Kp = up(y.Kreal, 16);
    y.row_bytes = (int64_t)P->slices * y.Kp;
    y.Nout = N * (cplx ? 2 : 1);
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t o = at;
        at += (size_t)up((int64_t)bytes, 256);
        return o;
    };
    y.oA8 = take((size_t)(L * M * y.row_bytes));
    y.oB8 = take((size_t)(L * y.Nout * y.row_bytes));
    y.oW = take((size_t)(L * M * y.Nout) * 8);
    y.oEA = take((size_t)(L * M) * 4);
    y.oEB = take((size_t)(L * N) * 4);
    y.oT = take((size_t)(2 * M + 2 * K + 2 * N + 2 * M + 2 * N) * 8);  // roffA koffA roffB koffB mC mD nC nD
    y.total = at;
    return y;
}

}  // namespace sl

size_t sliced_scratch_bytes(const tb_plan* P) { return sl::layout(P).total; }

cudaError_t launch_sliced(const tb_plan* P, const tb_ptrs* d, cudaStream_t s, int* kernels, void** main_timer)
{
    using namespace sl;
    *kernels = 0;
    const int S = P->slices;
    const int cplx = P->compute == TB_C64;
    const int64_t M = P->M.size, N = P->N.size, L = P->L.size, K = P->K.size;
    if (S < 2 || S > 16 || K <= 0) return cudaErrorInvalidValue;
    const Layout y = layout(P);
    void* ws = nullptr;
    cudaError_t e = pool_alloc(&ws, y.total, s);
    if (e != cudaSuccess) return e;
    char* base = (char*)ws;
    int8_t* A8 = (int8_t*)(base + y.oA8);
    int8_t* B8 = (int8_t*)(base + y.oB8);
    double* W = (double*)(base + y.oW);
    int32_t* EA = (int32_t*)(base + y.oEA);
    int32_t* EB = (int32_t*)(base + y.oEB);
    int64_t* T = (int64_t*)(base + y.oT);
    int64_t* roffA = T;
    int64_t* koffA = roffA + M;
    int64_t* roffB = koffA + K;
    int64_t* koffB = roffB + N;
    int64_t* mC = koffB + K;
    int64_t* mD = mC + M;
    int64_t* nC = mD + M;
    int64_t* nD = nC + N;

    // offset tables
    OffsetJobs jobs;
    memset(&jobs, 0, sizeof(jobs));
    const tb_modes* src[8] = {&P->M, &P->K, &P->N, &P->K, &P->M, &P->M, &P->N, &P->N};
    const int which[8] = {0, 0, 1, 1, 2, 3, 2, 3};
    int64_t* outs[8] = {roffA, koffA, roffB, koffB, mC, mD, nC, nD};
    jobs.n = 8;
    int64_t longest = 0;
    for (int j = 0; j < 8; j++) {
        fill(jobs.m[j], *src[j], which[j]);
        jobs.len[j] = src[j]->size;
        jobs.out[j] = outs[j];
        if (jobs.len[j] > longest) longest = jobs.len[j];
    }
    int64_t gx = (longest + 255) / 256;
    if (gx > 148 * 8) gx = 148 * 8;
    k_offsets<<<dim3((unsigned)gx, 8), 256, 0, s>>>(jobs);
    count_launch();
    (*kernels)++;

    // exponents and digit panels of A (rows M) and B (rows N)
    for (int side = 0; side < 2 && e == cudaSuccess; side++) {
        SliceParams sp;
        memset(&sp, 0, sizeof(sp));
        sp.src = side == 0 ? d->A : d->B;
        sp.type = side == 0 ? P->tA : P->tB;
        sp.conj = side == 0 ? P->conjA : P->conjB;
        sp.cplx = cplx;
        sp.is_B = side;
        sp.S = S;
        sp.R = side == 0 ? M : N;
        sp.K = K;
        sp.Lsz = L;
        sp.Kp = y.Kp;
        sp.Rout = side == 0 ? M : y.Nout;
        fill(sp.ls, P->L, side);
        sp.roff = side == 0 ? roffA : roffB;
        sp.koff = side == 0 ? koffA : koffB;
        sp.expo = side == 0 ? EA : EB;
        sp.dst = side == 0 ? A8 : B8;
        const bool rf = min_abs(side == 0 ? P->M : P->N, side) < min_abs(P->K, side);
        // about 8 blocks per SM, each over at least 256 contracted terms
        const int64_t row_tiles = (sp.R + TR - 1) / TR * L;
        int64_t ky = (148 * 8 + row_tiles - 1) / row_tiles;
        if (ky > (K + 255) / 256) ky = (K + 255) / 256;
        if (ky > 65535) ky = 65535;
        if (ky < 1) ky = 1;
        const int64_t kchunk = (K + ky - 1) / ky;
        ky = (K + kchunk - 1) / kchunk;
        e = cudaMemsetAsync(sp.expo, 0, (size_t)(L * sp.R) * sizeof(int32_t), s);
        if (e != cudaSuccess) break;
        const dim3 ge((unsigned)((sp.R + TR - 1) / TR), (unsigned)ky, (unsigned)L);
        if (rf) k_exponents<true><<<ge, 256, 0, s>>>(sp, kchunk);
        else k_exponents<false><<<ge, 256, 0, s>>>(sp, kchunk);
        const dim3 gs((unsigned)((sp.R + TR - 1) / TR), (unsigned)((y.Kp + TK - 1) / TK), (unsigned)L);
        if (cplx) {
            if (rf) k_slice<true, true><<<gs, 256, 0, s>>>(sp);
            else k_slice<false, true><<<gs, 256, 0, s>>>(sp);
        } else {
            if (rf) k_slice<true, false><<<gs, 256, 0, s>>>(sp);
            else k_slice<false, false><<<gs, 256, 0, s>>>(sp);
        }
        count_launch(2);
        (*kernels) += 2;
        e = cudaGetLastError();
    }

    // levels of digit pairs, each one or more integer GEMMs
    if (e == cudaSuccess && main_timer) tbk_timer_begin(s, main_timer);
    const int64_t pmax = MAX_TERMS / y.Kreal;
    bool first = true;
    for (int lv = 0; lv < S && e == cudaSuccess; lv++) {
        const double scale = ldexp(1.0, -7 * (lv + 2));
        if (pmax >= 1) {
            for (int64_t s0 = 0; s0 <= lv && e == cudaSuccess; s0 += pmax) {
                const int64_t s1 = s0 + pmax - 1 < lv ? s0 + pmax - 1 : lv;
                e = launch_gemm_i8(A8, B8, y.row_bytes, M, y.Nout, L, s0 * y.Kp, (S - 1 - lv + s0) * y.Kp,
                                   (s1 - s0 + 1) * y.Kp, W, scale, first ? 1 : 0, s);
                first = false;
                (*kernels)++;
            }
        } else {
            for (int64_t sa = 0; sa <= lv && e == cudaSuccess; sa++)
                for (int64_t k0 = 0; k0 < y.Kp && e == cudaSuccess; k0 += K_CHUNK) {
                    const int64_t len = y.Kp - k0 < K_CHUNK ? y.Kp - k0 : K_CHUNK;
                    e = launch_gemm_i8(A8, B8, y.row_bytes, M, y.Nout, L, sa * y.Kp + k0, (S - 1 - lv + sa) * y.Kp + k0,
                                       len, W, scale, first ? 1 : 0, s);
                    first = false;
                    (*kernels)++;
                }
        }
    }
    if (main_timer && *main_timer) tbk_timer_end(s, *main_timer);

    if (e == cudaSuccess) {
        FinishParams fp;
        memset(&fp, 0, sizeof(fp));
        fp.C = d->C;
        fp.D = d->D;
        fp.tC = P->tC;
        fp.tD = P->tD;
        fp.cplx = cplx;
        fp.beta_zero = P->beta_zero;
        fp.conjC = P->conjC;
        fp.conjD = P->conjD;
        fp.conjD_f32 = P->conjD_round_f32;
        fp.round_C = P->round_in;
        fp.m_fast = min_abs(P->M, 3) <= min_abs(P->N, 3);
        fp.alpha_re = P->alpha_re;
        fp.alpha_im = P->alpha_im;
        fp.beta_re = P->beta_re;
        fp.beta_im = P->beta_im;
        fp.M = M;
        fp.N = N;
        fp.L = L;
        fp.Nout = y.Nout;
        fp.W = W;
        fp.expA = EA;
        fp.expB = EB;
        fp.mC = mC;
        fp.mD = mD;
        fp.nC = nC;
        fp.nD = nD;
        fill(fp.lC, P->L, 2);
        fill(fp.lD, P->L, 3);
        int64_t g = (L * M * N + 255) / 256;
        if (g > 148 * 16) g = 148 * 16;
        if (cplx) k_sliced_finish<true><<<(unsigned)g, 256, 0, s>>>(fp);
        else k_sliced_finish<false><<<(unsigned)g, 256, 0, s>>>(fp);
        count_launch();
        (*kernels)++;
        e = cudaGetLastError();
    }
    cudaFreeAsync(ws, s);
    return e;
}

}  // namespace tb
