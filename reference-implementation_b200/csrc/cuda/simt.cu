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
//
// Shapes: the view is turned so that M >= N (D^T = B^T A^T; the roles of A
// and B, and of C's/D's row and column strides, swap), and the tile is chosen
// by N: 128x128 (binary32) or 64x64 for wide products, 128x32 and 128x16 for
// narrow ones (mode-n products with a small rank). When the tiles cannot
// fill the GPU and the contraction is long, the contraction is split over
// grid.y: each split writes its raw sums to a workspace and k_simt_final adds
// the splits in a fixed order and applies the epilogue, so results do not
// depend on scheduling.
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
    int32_t conjA, conjB, conjC, conjD, conjD_f32, d_rows_fast;
    Modes am, ak, al;  // A: rows (M), contraction, batch (s0 = stride in A)
    Modes bn, bk, bl;  // B: rows (N), contraction, batch (s0 = stride in B)
    Modes cm, cn, cl;  // C (s0) and D (s1) strides of M, N, L modes
    int32_t tiles_m, tiles_n;
    int64_t k_chunk;   // contraction length of one split (multiple of BK)
    void* ws;          // split sums [split][l][m][n][plane], or NULL: epilogue in place
};

// D = op_D(alpha * acc + beta * op_C(C)) for one element
template <typename T, bool CPLX>
__device__ __forceinline__ void epilogue_store(const Params& p, T xr, T xi, int64_t oc, int64_t od)
{
    const T ar = (T)p.alpha, ai = (T)p.alpha_im, br = (T)p.beta, bi = (T)p.beta_im;
    T vr = ar * xr - (CPLX ? ai * xi : (T)0);
    T vi = CPLX ? ar * xi + ai * xr : (T)0;
    if (!p.beta_zero) {
        T cr, ci;
        load_rounded<T>(p.C, oc, p.tC, p.round_in, cr, ci);
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
    store_elem<T>(p.D, od, p.tD, vr, vi);
}

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
    const int64_t kbeg = (int64_t)blockIdx.y * p.k_chunk;
    const int64_t kend = kbeg + p.k_chunk < p.K ? kbeg + p.k_chunk : p.K;

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
            if (k0 + t < kend) decode(p.ak, k0 + t, o, dummy);
            aK[buf][t] = o;
        } else if (t < 2 * BK) {
            int64_t o = 0;
            if (k0 + t - BK < kend) decode(p.bk, k0 + t - BK, o, dummy);
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
            if (m0 + r < p.M && k0 + kk < kend)
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
            if (n0 + r < p.N && k0 + kk < kend)
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
    // thread (tr, tc) owns rows tr + i*RT and columns tc + j*CT of the tile; a
    // warp runs along D's contiguous side (rows when d_rows_fast), so that the
    // epilogue's loads of C and stores of D coalesce
    constexpr int RT = BM / TM, CT = BN / TN;
    const int tr = p.d_rows_fast ? t % RT : t / CT;
    const int tc = p.d_rows_fast ? t / RT : t % CT;

    slice_offsets(kbeg, 0);
    __syncthreads();
    load_slice(kbeg, 0);
    store_slice(0);
    const int64_t nslices = (kend - kbeg + BK - 1) / BK;
    if (nslices > 1) slice_offsets(kbeg + BK, 1);
    __syncthreads();
    for (int64_t s = 0; s < nslices; s++) {
        const int buf = (int)(s & 1);
        if (s + 1 < nslices) load_slice(kbeg + (s + 1) * BK, buf ^ 1);  // global loads in flight during the FMAs
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T a[TM][NP], b[TN][NP];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int c = 0; c < NP; c++) a[i][c] = As[buf][c][kk][tr + i * RT];
#pragma unroll
            for (int j = 0; j < TN; j++)
#pragma unroll
                for (int c = 0; c < NP; c++) b[j][c] = Bs[buf][c][kk][tc + j * CT];
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
            if (s + 2 < nslices) slice_offsets(kbeg + (s + 2) * BK, buf);
            __syncthreads();
        }
    }
    if (p.ws) {
        // raw split sums; the final kernel adds the splits and finishes
        T* w = (T*)p.ws;
        const int64_t base = ((int64_t)blockIdx.y * p.L + l) * p.M;
#pragma unroll
        for (int i = 0; i < TM; i++) {
            const int r = tr + i * RT;
            if (m0 + r >= p.M) continue;
#pragma unroll
            for (int j = 0; j < TN; j++) {
                const int c = tc + j * CT;
                if (n0 + c >= p.N) continue;
                const int64_t at = ((base + m0 + r) * p.N + n0 + c) * NP;
#pragma unroll
                for (int q = 0; q < NP; q++) w[at + q] = acc[i][j][q];
            }
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int r = tr + i * RT;
        if (m0 + r >= p.M) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int c = tc + j * CT;
            if (n0 + c >= p.N) continue;
            epilogue_store<T, CPLX>(p, acc[i][j][0], CPLX ? acc[i][j][NP - 1] : (T)0, cRow[r] + cCol[c],
                                    dRow[r] + dCol[c]);
        }
    }
}

// adds the splits of every element of D in split order, then the epilogue
template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_simt_final(Params p, int splits)
{
    constexpr int NP = CPLX ? 2 : 1;
    const T* w = (const T*)p.ws;
    const int64_t total = p.L * p.M * p.N;
    const int64_t plane = total * NP;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = e % p.N;
        const int64_t m = (e / p.N) % p.M;
        const int64_t l = e / (p.N * p.M);
        T xr = 0, xi = 0;
        for (int z = 0; z < splits; z++) {
            xr += w[z * plane + e * NP];
            if (CPLX) xi += w[z * plane + e * NP + NP - 1];
        }
        int64_t cm, dm, cn, dn, cl, dl;
        decode(p.cm, m, cm, dm);
        decode(p.cn, n, cn, dn);
        decode(p.cl, l, cl, dl);
        epilogue_store<T, CPLX>(p, xr, xi, cm + cn + cl, dm + dn + dl);
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
    const int64_t* s = w == 0 ? m.sA : w == 1 ? m.sB : w == 2 ? m.sC : m.sD;
    int64_t best = INT64_MAX;
    for (int j = 0; j < m.n; j++) {
        const int64_t v = s[j] < 0 ? -s[j] : s[j];
        if (v && v < best) best = v;
    }
    return best;
}

// Split of the contraction: enough CTAs to fill the GPU when the tiles do
// not, each split at least 4 slices long, the workspace at most 256 MiB.
struct Split {
    int splits;
    int64_t chunk;
    size_t ws_bytes;
};

static Split choose_split(int64_t tiles, int64_t K, int64_t outs, int bk, size_t elem)
{
    Split r = {1, K, 0};
    const int64_t slices = (K + bk - 1) / bk;
    const int64_t target = 148 * 4;
    if (tiles >= target / 2 || slices < 8) return r;
    int64_t S = (target + tiles - 1) / tiles;
    if (S > slices / 4) S = slices / 4;
    if (S > 1024) S = 1024;
    while (S > 1 && (double)S * (double)outs * (double)elem > 256.0 * 1024 * 1024) S /= 2;
    if (S <= 1) return r;
    const int64_t per = (slices + S - 1) / S;
    r.chunk = per * bk;
    r.splits = (int)((K + r.chunk - 1) / r.chunk);
    r.ws_bytes = (size_t)r.splits * (size_t)outs * elem;
    return r;
}

template <typename T, bool CPLX, int BM, int BN, int BK, int TM, int TN>
struct Cfg {
    static Split split(const Params& p)
    {
        const int64_t tiles = ((p.M + BM - 1) / BM) * ((p.N + BN - 1) / BN) * p.L;
        return choose_split(tiles, p.K, p.L * p.M * p.N, BK, sizeof(T) * (CPLX ? 2 : 1));
    }

    static cudaError_t launch(Params& p, cudaStream_t s)
    {
        p.tiles_m = (int)((p.M + BM - 1) / BM);
        p.tiles_n = (int)((p.N + BN - 1) / BN);
        const int64_t blocks = (int64_t)p.tiles_m * p.tiles_n * p.L;
        if (blocks <= 0 || blocks > 0x7fffffff) return cudaErrorInvalidConfiguration;
        const Split sp = split(p);
        p.k_chunk = sp.chunk;
        p.ws = nullptr;
        if (sp.splits > 1) {
            cudaError_t e = pool_alloc(&p.ws, sp.ws_bytes, s);
            if (e != cudaSuccess) return e;
        }
        k_simt<T, CPLX, BM, BN, BK, TM, TN><<<dim3((unsigned)blocks, (unsigned)sp.splits), (BM / TM) * (BN / TN), 0, s>>>(p);
        count_launch();
        cudaError_t e = cudaGetLastError();
        if (sp.splits > 1) {
            if (e == cudaSuccess) {
                const int64_t total = p.L * p.M * p.N;
                int64_t g = (total + 255) / 256;
                if (g > 148 * 16) g = 148 * 16;
                k_simt_final<T, CPLX><<<(unsigned)g, 256, 0, s>>>(p, sp.splits);
                count_launch();
                e = cudaGetLastError();
            }
            cudaFreeAsync(p.ws, s);
        }
        return e;
    }
};

// tile shapes: wide (binary32), square, narrow N
enum { TILE_WIDE, TILE_SQUARE, TILE_N32, TILE_N16 };

static int tile_for(int compute, int64_t M, int64_t N)
{
    if (N <= 16 && (compute == TB_R32 || compute == TB_R64)) return TILE_N16;
    if (N <= 32) return TILE_N32;
    if (compute == TB_R32 && M > 64 && N > 64) return TILE_WIDE;
    return TILE_SQUARE;
}

template <typename F>
static auto with_cfg(int compute, int tile, F&& f)
{
    switch (compute) {
    case TB_R64:
        if (tile == TILE_N16) return f(Cfg<double, false, 128, 16, 16, 4, 2>());
        if (tile == TILE_N32) return f(Cfg<double, false, 128, 32, 16, 4, 4>());
        return f(Cfg<double, false, 64, 64, 16, 4, 4>());
    case TB_C32:
        if (tile == TILE_N32) return f(Cfg<float, true, 128, 32, 8, 4, 4>());
        return f(Cfg<float, true, 64, 64, 8, 4, 4>());
    case TB_C64:
        if (tile == TILE_N32) return f(Cfg<double, true, 128, 32, 8, 4, 4>());
        return f(Cfg<double, true, 64, 64, 8, 4, 4>());
    default:
        if (tile == TILE_N16) return f(Cfg<float, false, 128, 16, 16, 4, 2>());
        if (tile == TILE_N32) return f(Cfg<float, false, 128, 32, 16, 4, 4>());
        if (tile == TILE_WIDE) return f(Cfg<float, false, 128, 128, 16, 8, 8>());
        return f(Cfg<float, false, 64, 64, 16, 4, 4>());
    }
}

}  // namespace simt

// the launch parameters of a plan, turned so that M >= N
static void simt_params(const tb_plan* P, const tb_ptrs* d, simt::Params& p)
{
    using namespace simt;
    memset(&p, 0, sizeof(p));
    const int swap = P->N.size > P->M.size;
    const tb_modes& Mm = swap ? P->N : P->M;
    const tb_modes& Nm = swap ? P->M : P->N;
    const int wa = swap ? 1 : 0, wb = swap ? 0 : 1;  // which operand plays A and B
    p.A = swap ? d->B : d->A;
    p.B = swap ? d->A : d->B;
    p.C = d->C;
    p.D = d->D;
    p.tA = swap ? P->tB : P->tA;
    p.tB = swap ? P->tA : P->tB;
    p.tC = P->tC;
    p.tD = P->tD;
    p.round_in = P->round_in;
    p.beta_zero = P->beta_zero;
    p.M = Mm.size;
    p.N = Nm.size;
    p.K = P->K.size;
    p.L = P->L.size;
    p.alpha = P->alpha_re;
    p.beta = P->beta_re;
    p.alpha_im = P->alpha_im;
    p.beta_im = P->beta_im;
    p.conjA = swap ? P->conjB : P->conjA;
    p.conjB = swap ? P->conjA : P->conjB;
    p.conjC = P->conjC;
    p.conjD = P->conjD;
    p.conjD_f32 = P->conjD_round_f32;
    fill(p.am, Mm, wa, -1);
    fill(p.ak, P->K, wa, -1);
    fill(p.al, P->L, wa, -1);
    fill(p.bn, Nm, wb, -1);
    fill(p.bk, P->K, wb, -1);
    fill(p.bl, P->L, wb, -1);
    fill(p.cm, Mm, 2, 3);
    fill(p.cn, Nm, 2, 3);
    fill(p.cl, P->L, 2, 3);
    p.a_rows_fast = min_abs(Mm, wa) < min_abs(P->K, wa);
    p.b_rows_fast = min_abs(Nm, wb) < min_abs(P->K, wb);
    p.d_rows_fast = min_abs(Mm, 3) <= min_abs(Nm, 3);
}

size_t simt_scratch_bytes(const tb_plan* P)
{
    using namespace simt;
    Params p;
    tb_ptrs d = {nullptr, nullptr, nullptr, nullptr};
    simt_params(P, &d, p);
    return with_cfg(P->compute, tile_for(P->compute, p.M, p.N), [&](auto cfg) { return decltype(cfg)::split(p).ws_bytes; });
}

cudaError_t launch_simt(const tb_plan* P, const tb_ptrs* d, cudaStream_t s)
{
    using namespace simt;
    Params p;
    simt_params(P, d, p);
    return with_cfg(P->compute, tile_for(P->compute, p.M, p.N), [&](auto cfg) { return decltype(cfg)::launch(p, s); });
}

}  // namespace tb
