// Tiled CUDA-core GEMM (binary32 / binary64, real or complex): the plain GPU
// path for large contractions that the tensor cores do not take (F32F32
// without split mode, F64F64, DEFAULT on float/double/complex data).
// Complex operands keep real and imaginary planes in shared memory and
// accumulate with four FMAs per product; op_A/op_B conjugation is applied at
// load, op_C and op_D in the epilogue.
//
// One launch per product, operands gathered in place from their strided
// layouts: each block owns a BM x BN tile of the L/M/N view
// (D[l,m,n] = alpha * sum_k A[l,m,k] B[l,k,n] + beta * C[l,m,n]); per BK slice
// of the contraction it resolves the slice's offsets once (a table of BK
// entries per operand), loads the A and B slices into shared memory (threads
// walk the operand's contiguous direction), and every thread accumulates a
// TM x TN register tile with FMAs. The epilogue writes D through row/column
// offset tables with D's and C's own strides.
#include <cstdio>
#include <cstring>

#include "tb_common.cuh"

namespace tb {
namespace simt {

struct Modes {
    int32_t n, pad;
    int64_t ext[TB_MAXMODES];
    int64_t s0[TB_MAXMODES];
    int64_t s1[TB_MAXMODES];
};

__device__ __forceinline__ void decode(const Modes& m, int64_t idx, int64_t& o0, int64_t& o1)
{
    o0 = 0;
    o1 = 0;
    for (int j = 0; j < m.n; j++) {
        const int64_t c = idx % m.ext[j];
        idx /= m.ext[j];
        o0 += c * m.s0[j];
        o1 += c * m.s1[j];
    }
}

struct Params {
    const void* A;
    const void* B;
    const void* C;
    void* D;
    int32_t tA, tB, tC, tD, round_in, beta_zero, a_rows_fast, b_rows_fast;
    int64_t M, N, K, L;
    double alpha, beta, alpha_im, beta_im;
    int32_t conjA, conjB, conjC, conjD, conjD_f32, pad2;
    Modes am, ak, al;  // A: rows (M), contraction, batch (s0 = stride in A)
    Modes bn, bk, bl;  // B: rows (N), contraction, batch (s0 = stride in B)
    Modes cm, cn, cl;  // C (s0) and D (s1) strides of M, N, L modes
    int32_t tiles_m, tiles_n;
};

template <typename T, bool CPLX, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN)) k_simt(Params p)
{
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int NP = CPLX ? 2 : 1;  // real and imaginary planes
    __shared__ T As[2][NP][BK][BM + 1];
    __shared__ T Bs[2][NP][BK][BN + 1];
    __shared__ int64_t aRow[BM], bRow[BN];
    __shared__ int64_t aK[2][BK], bK[2][BK];
    __shared__ int64_t dRow[BM], cRow[BM], dCol[BN], cCol[BN];

    const int t = threadIdx.x;
    const int64_t tile = blockIdx.x;
    const int tm = (int)(tile % p.tiles_m);
    const int64_t rest = tile / p.tiles_m;
    const int tn = (int)(rest % p.tiles_n);
    const int64_t l = rest / p.tiles_n;
    const int64_t m0 = (int64_t)tm * BM, n0 = (int64_t)tn * BN;

    int64_t aL, bL, cL, dL, dummy;
    decode(p.al, l, aL, dummy);
    decode(p.bl, l, bL, dummy);
    decode(p.cl, l, cL, dL);
    for (int i = t; i < BM; i += NT) {
        int64_t o = 0, oc = 0, od = 0;
        if (m0 + i < p.M) {
            decode(p.am, m0 + i, o, dummy);
            decode(p.cm, m0 + i, oc, od);
        }
        aRow[i] = o + aL;
        cRow[i] = oc + cL;
        dRow[i] = od + dL;
    }
    for (int i = t; i < BN; i += NT) {
        int64_t o = 0, oc = 0, od = 0;
        if (n0 + i < p.N) {
            decode(p.bn, n0 + i, o, dummy);
            decode(p.cn, n0 + i, oc, od);
        }
        bRow[i] = o + bL;
        cCol[i] = oc;
        dCol[i] = od;
    }
    // offsets of one contraction slice
    auto slice_offsets = [&](int64_t k0, int buf) {
        if (t < BK) {
            int64_t o = 0;
            if (k0 + t < p.K) decode(p.ak, k0 + t, o, dummy);
            aK[buf][t] = o;
        } else if (t < 2 * BK) {
            int64_t o = 0;
            if (k0 + t - BK < p.K) decode(p.bk, k0 + t - BK, o, dummy);
            bK[buf][t - BK] = o;
        }
    };
    constexpr int A_PER = BM * BK / NT, B_PER = BN * BK / NT;
    T ra[A_PER][NP], rb[B_PER][NP];
    auto load_slice = [&](int64_t k0, int buf) {
#pragma unroll
        for (int u = 0; u < A_PER; u++) {
            const int e = t + NT * u;
            const int r = p.a_rows_fast ? e % BM : e / BK;
            const int kk = p.a_rows_fast ? e / BM : e % BK;
            T x = 0, xi = 0;
            if (m0 + r < p.M && k0 + kk < p.K)
                load_rounded<T>(p.A, aRow[r] + aK[buf][kk], p.tA, p.round_in, x, xi);
            ra[u][0] = x;
            if (CPLX) ra[u][NP - 1] = p.conjA ? -xi : xi;
        }
#pragma unroll
        for (int u = 0; u < B_PER; u++) {
            const int e = t + NT * u;
            const int r = p.b_rows_fast ? e % BN : e / BK;
            const int kk = p.b_rows_fast ? e / BN : e % BK;
            T x = 0, xi = 0;
            if (n0 + r < p.N && k0 + kk < p.K)
                load_rounded<T>(p.B, bRow[r] + bK[buf][kk], p.tB, p.round_in, x, xi);
            rb[u][0] = x;
            if (CPLX) rb[u][NP - 1] = p.conjB ? -xi : xi;
        }
    };
    auto store_slice = [&](int buf) {
#pragma unroll
        for (int u = 0; u < A_PER; u++) {
            const int e = t + NT * u;
            const int r = p.a_rows_fast ? e % BM : e / BK;
            const int kk = p.a_rows_fast ? e / BM : e % BK;
#pragma unroll
            for (int c = 0; c < NP; c++) As[buf][c][kk][r] = ra[u][c];
        }
#pragma unroll
        for (int u = 0; u < B_PER; u++) {
            const int e = t + NT * u;
            const int r = p.b_rows_fast ? e % BN : e / BK;
            const int kk = p.b_rows_fast ? e / BN : e % BK;
#pragma unroll
            for (int c = 0; c < NP; c++) Bs[buf][c][kk][r] = rb[u][c];
        }
    };

    T acc[TM][TN][NP];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
            for (int c = 0; c < NP; c++) acc[i][j][c] = 0;
    const int tr = t / (BN / TN), tc = t % (BN / TN);  // thread's rows tr*TM.., columns tc + j*(BN/TN)

    slice_offsets(0, 0);
    __syncthreads();
    load_slice(0, 0);
    store_slice(0);
    const int64_t nslices = (p.K + BK - 1) / BK;
    if (nslices > 1) slice_offsets(BK, 1);
    __syncthreads();
    for (int64_t s = 0; s < nslices; s++) {
        const int buf = (int)(s & 1);
        if (s + 1 < nslices) load_slice((s + 1) * BK, buf ^ 1);  // global loads in flight during the FMAs
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T a[TM][NP], b[TN][NP];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int c = 0; c < NP; c++) a[i][c] = As[buf][c][kk][tr * TM + i];
#pragma unroll
            for (int j = 0; j < TN; j++)
#pragma unroll
                for (int c = 0; c < NP; c++) b[j][c] = Bs[buf][c][kk][tc + j * (BN / TN)];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) {
                    acc[i][j][0] = fma(a[i][0], b[j][0], acc[i][j][0]);
                    if (CPLX) {
                        acc[i][j][0] = fma(-a[i][NP - 1], b[j][NP - 1], acc[i][j][0]);
                        acc[i][j][NP - 1] = fma(a[i][0], b[j][NP - 1], acc[i][j][NP - 1]);
                        acc[i][j][NP - 1] = fma(a[i][NP - 1], b[j][0], acc[i][j][NP - 1]);
                    }
                }
        }
        if (s + 1 < nslices) {
            store_slice(buf ^ 1);
            __syncthreads();
            if (s + 2 < nslices) slice_offsets((s + 2) * BK, buf);
            __syncthreads();
        }
    }
    // epilogue: D = op_D(alpha * acc + beta * op_C(C))
    const T ar = (T)p.alpha, ai = (T)p.alpha_im, br = (T)p.beta, bi = (T)p.beta_im;
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int r = tr * TM + i;
        if (m0 + r >= p.M) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int c = tc + j * (BN / TN);
            if (n0 + c >= p.N) continue;
            const T xr = acc[i][j][0], xi = CPLX ? acc[i][j][NP - 1] : (T)0;
            T vr = ar * xr - (CPLX ? ai * xi : (T)0);
            T vi = CPLX ? ar * xi + ai * xr : (T)0;
            if (!p.beta_zero) {
                T cr, ci;
                load_rounded<T>(p.C, cRow[r] + cCol[c], p.tC, p.round_in, cr, ci);
                if (p.conjC) ci = -ci;
                vr = fma(br, cr, vr);
                if (CPLX) {
                    vr = fma(-bi, ci, vr);
                    vi = fma(br, ci, fma(bi, cr, vi));
                }
            }
            if (p.conjD) {
                if (p.conjD_f32) {
                    vr = (T)(float)vr;
                    vi = (T)(float)vi;
                }
                vi = -vi;
            }
            store_elem<T>(p.D, dRow[r] + dCol[c], p.tD, vr, vi);
        }
    }
}

static void fill(Modes& m, const tb_modes& src, int w0, int w1)
{
    memset(&m, 0, sizeof(m));
    m.n = src.n;
    const int64_t* s[4] = {src.sA, src.sB, src.sC, src.sD};
    for (int j = 0; j < src.n; j++) {
        m.ext[j] = src.ext[j];
        m.s0[j] = w0 >= 0 ? s[w0][j] : 0;
        m.s1[j] = w1 >= 0 ? s[w1][j] : 0;
    }
}

static int64_t min_abs(const tb_modes& m, int w)
{
    const int64_t* s = w == 0 ? m.sA : m.sB;
    int64_t best = INT64_MAX;
    for (int j = 0; j < m.n; j++) {
        const int64_t v = s[j] < 0 ? -s[j] : s[j];
        if (v && v < best) best = v;
    }
    return best;
}

template <typename T, bool CPLX, int BM, int BN, int BK, int TM, int TN>
static cudaError_t launch(Params& p, cudaStream_t s)
{
    p.tiles_m = (int)((p.M + BM - 1) / BM);
    p.tiles_n = (int)((p.N + BN - 1) / BN);
    const int64_t blocks = (int64_t)p.tiles_m * p.tiles_n * p.L;
    if (blocks <= 0 || blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
    k_simt<T, CPLX, BM, BN, BK, TM, TN><<<(unsigned)blocks, (BM / TM) * (BN / TN), 0, s>>>(p);
    count_launch();
    return cudaGetLastError();
}

}  // namespace simt

cudaError_t launch_simt(const tb_plan* P, const tb_ptrs* d, cudaStream_t s)
{
    using namespace simt;
    Params p;
    memset(&p, 0, sizeof(p));
    p.A = d->A;
    p.B = d->B;
    p.C = d->C;
    p.D = d->D;
    p.tA = P->tA;
    p.tB = P->tB;
    p.tC = P->tC;
    p.tD = P->tD;
    p.round_in = P->round_in;
    p.beta_zero = P->beta_zero;
    p.M = P->M.size;
    p.N = P->N.size;
    p.K = P->K.size;
    p.L = P->L.size;
    p.alpha = P->alpha_re;
    p.beta = P->beta_re;
    p.alpha_im = P->alpha_im;
    p.beta_im = P->beta_im;
    p.conjA = P->conjA;
    p.conjB = P->conjB;
    p.conjC = P->conjC;
    p.conjD = P->conjD;
    p.conjD_f32 = P->conjD_round_f32;
    fill(p.am, P->M, 0, -1);
    fill(p.ak, P->K, 0, -1);
    fill(p.al, P->L, 0, -1);
    fill(p.bn, P->N, 1, -1);
    fill(p.bk, P->K, 1, -1);
    fill(p.bl, P->L, 1, -1);
    fill(p.cm, P->M, 2, 3);
    fill(p.cn, P->N, 2, 3);
    fill(p.cl, P->L, 2, 3);
    p.a_rows_fast = min_abs(P->M, 0) < min_abs(P->K, 0);
    p.b_rows_fast = min_abs(P->N, 1) < min_abs(P->K, 1);
    switch (P->compute) {
    case TB_R64: return launch<double, false, 64, 64, 16, 4, 4>(p, s);
    case TB_C32: return launch<float, true, 64, 64, 8, 4, 4>(p, s);
    case TB_C64: return launch<double, true, 64, 64, 8, 4, 4>(p, s);
    default: return launch<float, false, 128, 128, 16, 8, 8>(p, s);
    }
}

}  // namespace tb
