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
    int32_t a_vec, b_vec;  // operand read 16 bytes at a time (see vec_side)
};

// D = op_D(alpha * acc + beta * op_C(C)) for one element whose C value
// (cr, ci) is already loaded (rounded, not yet conjugated)
template <typename T, bool CPLX>
__device__ __forceinline__ void epilogue_value(const Params& p, T xr, T xi, T cr, T ci, T& out_r, T& out_i)
{
    const T ar = (T)p.alpha, ai = (T)p.alpha_im, br = (T)p.beta, bi = (T)p.beta_im;
    T vr = ar * xr - (CPLX ? ai * xi : (T)0);
    T vi = CPLX ? ar * xi + ai * xr : (T)0;
    if (!p.beta_zero) {
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
    out_r = vr;
    out_i = vi;
}

template <typename T, bool CPLX>
__device__ __forceinline__ void epilogue_store_c(const Params& p, T xr, T xi, T cr, T ci, int64_t od)
{
    T vr, vi;
    epilogue_value<T, CPLX>(p, xr, xi, cr, ci, vr, vi);
    store_elem<T>(p.D, od, p.tD, vr, vi);
}

// the same, loading C first
template <typename T, bool CPLX>
__device__ __forceinline__ void epilogue_store(const Params& p, T xr, T xi, int64_t oc, int64_t od)
{
    T cr = 0, ci = 0;
    if (!p.beta_zero) load_rounded<T>(p.C, oc, p.tC, p.round_in, cr, ci);
    epilogue_store_c<T, CPLX>(p, xr, xi, cr, ci, od);
}

template <typename T, bool CPLX, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), (CPLX && sizeof(T) == 8) ? 1 : 2)
k_simt(Params p)
{
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int NP = CPLX ? 2 : 1;  // real and imaginary planes
    // V4: real binary32 with register tiles in groups of four rows and four
    // columns, read from shared memory as 16-byte vectors (rows padded by 4
    // to keep them aligned); else scalar reads (rows padded by 1)
    constexpr bool V4 = !CPLX && sizeof(T) == 4 && TM % 4 == 0 && TN % 4 == 0;
    constexpr int PAD = V4 ? 4 : 1;
    __shared__ __align__(16) T As[2][NP][BK][BM + PAD];
    __shared__ __align__(16) T Bs[2][NP][BK][BN + PAD];
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
    // VA / VB: with a_vec / b_vec set, VW neighbours along the operand's
    // contiguous mode (4 binary32 or 2 binary64) come in one 16-byte load
    constexpr int VW = 16 / sizeof(T);
    constexpr bool VA = !CPLX && A_PER % VW == 0, VB = !CPLX && B_PER % VW == 0;
    T ra[A_PER][NP], rb[B_PER][NP];
    // element (r, kk) of group u of VW: along rows or along the contraction
    auto vec_rk = [&](int u, bool rows_fast, int rows, int& r, int& kk) {
        const int e = t + NT * u;
        if (rows_fast) {
            r = (e % (rows / VW)) * VW;
            kk = e / (rows / VW);
        } else {
            kk = (e % (BK / VW)) * VW;
            r = e / (BK / VW);
        }
    };
    auto loadv = [&](const void* base, int64_t off, bool in, T* dst) {
        if constexpr (sizeof(T) == 4) {
            float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
            if (in) q = __ldg((const float4*)((const float*)base + off));
            dst[0] = q.x; dst[1] = q.y; dst[2] = q.z; dst[3] = q.w;
        } else {
            double2 q = make_double2(0.0, 0.0);
            if (in) q = __ldg((const double2*)((const double*)base + off));
            dst[0] = q.x; dst[1] = q.y;
        }
        if (p.round_in != TB_ROUND_NONE)
            for (int h = 0; h < VW; h++) dst[h] = round_in<T>(dst[h], p.round_in);
    };
    auto load_slice = [&](int64_t k0, int buf) {
        if constexpr (VA) {
            if (p.a_vec) {
#pragma unroll
                for (int u = 0; u < A_PER / VW; u++) {
                    int r, kk;
                    vec_rk(u, p.a_rows_fast, BM, r, kk);
                    T v[VW];
                    loadv(p.A, aRow[r] + aK[buf][kk], m0 + r < p.M && k0 + kk < kend, v);
#pragma unroll
                    for (int h = 0; h < VW; h++) ra[VW * u + h][0] = v[h];
                }
                goto b_side;
            }
        }
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
    b_side:
        if constexpr (VB) {
            if (p.b_vec) {
#pragma unroll
                for (int u = 0; u < B_PER / VW; u++) {
                    int r, kk;
                    vec_rk(u, p.b_rows_fast, BN, r, kk);
                    T v[VW];
                    loadv(p.B, bRow[r] + bK[buf][kk], n0 + r < p.N && k0 + kk < kend, v);
#pragma unroll
                    for (int h = 0; h < VW; h++) rb[VW * u + h][0] = v[h];
                }
                return;
            }
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
        if constexpr (VA) {
            if (p.a_vec) {
#pragma unroll
                for (int u = 0; u < A_PER / VW; u++) {
                    int r, kk;
                    vec_rk(u, p.a_rows_fast, BM, r, kk);
                    if (V4 && p.a_rows_fast) {
                        *(float4*)&As[buf][0][kk][r] =
                            make_float4(ra[VW * u][0], ra[VW * u + 1][0], ra[VW * u + 2][0], ra[VW * u + 3][0]);
                    } else if (p.a_rows_fast) {
#pragma unroll
                        for (int h = 0; h < VW; h++) As[buf][0][kk][r + h] = ra[VW * u + h][0];
                    } else {
#pragma unroll
                        for (int h = 0; h < VW; h++) As[buf][0][kk + h][r] = ra[VW * u + h][0];
                    }
                }
                goto b_store;
            }
        }
#pragma unroll
        for (int u = 0; u < A_PER; u++) {
            const int e = t + NT * u;
            const int r = p.a_rows_fast ? e % BM : e / BK;
            const int kk = p.a_rows_fast ? e / BM : e % BK;
#pragma unroll
            for (int c = 0; c < NP; c++) As[buf][c][kk][r] = ra[u][c];
        }
    b_store:
        if constexpr (VB) {
            if (p.b_vec) {
#pragma unroll
                for (int u = 0; u < B_PER / VW; u++) {
                    int r, kk;
                    vec_rk(u, p.b_rows_fast, BN, r, kk);
                    if (V4 && p.b_rows_fast) {
                        *(float4*)&Bs[buf][0][kk][r] =
                            make_float4(rb[VW * u][0], rb[VW * u + 1][0], rb[VW * u + 2][0], rb[VW * u + 3][0]);
                    } else if (p.b_rows_fast) {
#pragma unroll
                        for (int h = 0; h < VW; h++) Bs[buf][0][kk][r + h] = rb[VW * u + h][0];
                    } else {
#pragma unroll
                        for (int h = 0; h < VW; h++) Bs[buf][0][kk + h][r] = rb[VW * u + h][0];
                    }
                }
                return;
            }
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
    // row of register row i and column of register column j: strided by RT
    // (CT), or, with V4, groups of four consecutive rows (columns) RT*4
    // (CT*4) apart
    auto row_of = [&](int i) { return V4 ? (i / 4) * (RT * 4) + tr * 4 + (i % 4) : tr + i * RT; };
    auto col_of = [&](int j) { return V4 ? (j / 4) * (CT * 4) + tc * 4 + (j % 4) : tc + j * CT; };

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
            if constexpr (V4) {
#pragma unroll
                for (int i = 0; i < TM; i += 4) {
                    const float4 q = *(const float4*)&As[buf][0][kk][row_of(i)];
                    a[i][0] = q.x; a[i + 1][0] = q.y; a[i + 2][0] = q.z; a[i + 3][0] = q.w;
                }
#pragma unroll
                for (int j = 0; j < TN; j += 4) {
                    const float4 q = *(const float4*)&Bs[buf][0][kk][col_of(j)];
                    b[j][0] = q.x; b[j + 1][0] = q.y; b[j + 2][0] = q.z; b[j + 3][0] = q.w;
                }
            } else {
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int c = 0; c < NP; c++) a[i][c] = As[buf][c][kk][row_of(i)];
#pragma unroll
                for (int j = 0; j < TN; j++)
#pragma unroll
                    for (int c = 0; c < NP; c++) b[j][c] = Bs[buf][c][kk][col_of(j)];
            }
            // pairs of fused multiply-adds per instruction (fma2), each
            // accumulator updated in the same order as one fma at a time
#pragma unroll
            for (int i = 0; i < TM; i++) {
                if (CPLX) {
#pragma unroll
                    for (int j = 0; j < TN; j++) {
                        // re += ar br, im += ar bi; then re += -ai bi, im += ai br
                        fma2(acc[i][j][0], acc[i][j][NP - 1], a[i][0], a[i][0], b[j][0], b[j][NP - 1]);
                        fma2(acc[i][j][0], acc[i][j][NP - 1], -a[i][NP - 1], a[i][NP - 1], b[j][NP - 1], b[j][0]);
                    }
                } else {
                    static_assert(CPLX || TN % 2 == 0, "register tiles of an even width");
#pragma unroll
                    for (int j = 0; j < TN; j += 2)
                        fma2(acc[i][j][0], acc[i][j + 1][0], a[i][0], a[i][0], b[j][0], b[j + 1][0]);
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
            const int r = row_of(i);
            if (m0 + r >= p.M) continue;
#pragma unroll
            for (int j = 0; j < TN; j++) {
                const int c = col_of(j);
                if (n0 + c >= p.N) continue;
                const int64_t at = ((base + m0 + r) * p.N + n0 + c) * NP;
#pragma unroll
                for (int q = 0; q < NP; q++) w[at + q] = acc[i][j][q];
            }
        }
        return;
    }
    // a row's C values are loaded together (C may alias D, so loads cannot
    // move past the stores on their own), then its D values stored
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int r = row_of(i);
        if (m0 + r >= p.M) continue;
        T cr[TN], ci[TN];
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int c = col_of(j);
            cr[j] = 0;
            ci[j] = 0;
            if (!p.beta_zero && n0 + c < p.N) load_rounded<T>(p.C, cRow[r] + cCol[c], p.tC, p.round_in, cr[j], ci[j]);
        }
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int c = col_of(j);
            if (n0 + c >= p.N) continue;
            epilogue_store_c<T, CPLX>(p, acc[i][j][0], CPLX ? acc[i][j][NP - 1] : (T)0, cr[j], ci[j], dRow[r] + dCol[c]);
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

// ---------------------------------------------------------------------------
// Narrow products (N <= 64 after turning, short contraction, real): the
// mode-n products of Tucker decompositions and their kin. A 64-wide tile
// wastes most of its FMAs on them and its set-up dominates, so instead every
// block stages B[l] (K x NB, padded with zeros) in shared memory once and
// streams 256 rows of A per step, one row per thread: K loads and K x NB
// FMAs per row, accumulators in registers, then the epilogue of its N
// outputs. A loads coalesce when A's rows are contiguous (the common case);
// row offsets decode with 32-bit multiply-high division.
constexpr int NARROW_MAX_SMEM = 100 * 1024;
constexpr int NARROW_COOP_SMEM = 227 * 1024;  // the cooperative variant's limit

struct NarrowParams {
    Params p;
    FastDiv fm[TB_MAXMODES];  // M extents
    int32_t nb;               // padded N
    int32_t stage_c;          // streaming kernel: C (stored as T) staged in shared memory
};

// DIRECT: A is stored as T and not rounded (plain loads, no type dispatch)
template <typename T, int NB, bool DIRECT>
__global__ void __launch_bounds__(256) k_narrow(NarrowParams np)
{
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    T* Bs = (T*)nsm;                                     // [K][NB]
    int64_t* kA = (int64_t*)(nsm + sizeof(T) * NB * p.K);  // [K] contracted offsets in A
    int64_t* nC = kA + p.K;                              // [NB] column offsets in C
    int64_t* nD = nC + NB;                               // [NB] column offsets in D
    const int t = threadIdx.x;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += 256) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    // B panel: element (k, n) = op_B(B)[l, k, n], rounded as the precision asks
    for (int64_t e = t; e < p.K * NB; e += 256) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        T x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<T>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
        }
        Bs[k * NB + n] = x;
    }
    __syncthreads();
    const int64_t tiles = (p.M + 255) / 256;
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t m = tile * 256 + t;
        if (m >= p.M) continue;
        // row offsets in A, C and D
        int64_t oA = 0, oC = 0, oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
        T acc[NB];
#pragma unroll
        for (int n = 0; n < NB; n++) acc[n] = 0;
        // contraction in chunks of U, the next chunk's loads in flight while
        // the current one is multiplied
        constexpr int U = 8;
        T cur[U], nxt[U];
        auto load_chunk = [&](int64_t k0, T (&dst)[U]) {
#pragma unroll
            for (int u = 0; u < U; u++) {
                T im;
                dst[u] = 0;
                if (k0 + u < p.K) {
                    if (DIRECT) dst[u] = __ldg((const T*)p.A + oA + kA[k0 + u]);
                    else load_rounded<T>(p.A, oA + kA[k0 + u], p.tA, p.round_in, dst[u], im);
                }
            }
        };
        load_chunk(0, cur);
        for (int64_t k0 = 0; k0 < p.K; k0 += U) {
            if (k0 + U < p.K) load_chunk(k0 + U, nxt);
#pragma unroll
            for (int u = 0; u < U; u++) {
                if (k0 + u < p.K) {
                    const T* b = Bs + (k0 + u) * NB;
#pragma unroll
                    for (int n = 0; n < NB; n += 2) fma2(acc[n], acc[n + 1], cur[u], cur[u], b[n], b[n + 1]);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) cur[u] = nxt[u];
        }
        // epilogue in groups of 8 outputs: the group's C values first (loads
        // in flight together), then D = op_D(alpha acc + beta C)
        const T al = (T)p.alpha, be = (T)p.beta;
#pragma unroll
        for (int g = 0; g < NB; g += 8) {
            T cv[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                T im;
                cv[j] = 0;
                if (!p.beta_zero && g + j < p.N) load_rounded<T>(p.C, oC + nC[g + j], p.tC, p.round_in, cv[j], im);
            }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (g + j < p.N) {
                    T v = p.beta_zero ? al * acc[g + j] : fma(be, cv[j], al * acc[g + j]);
                    if (p.conjD && p.conjD_f32) v = (T)(float)v;  // op_D under the F64 precision rounds as conjf
                    store_elem<T>(p.D, oD + nD[g + j], p.tD, v, (T)0);
                }
            }
        }
    }
}

// Streaming variant of k_narrow for A stored as T: every thread copies its
// own row of A into its own column of a shared-memory ring with cp.async (S
// chunks of KC contracted values, S - 1 of them in flight while one is
// multiplied, across tile boundaries; 48 KiB a block, so that two blocks
// share an SM), so the latency of HBM is covered by the copies in flight
// instead of by registers. Its row of C is copied the same way at the start
// of each tile. A thread only reads what it copied itself: cp.async.wait_group
// orders the two, and no block barrier is needed after the B panel is staged.
template <typename T>
struct StreamRing {
    static constexpr int KC = sizeof(T) == 4 ? 16 : 8;  // contracted values per chunk
    static constexpr int S = 3;                         // chunks in the ring
    static constexpr size_t bytes = sizeof(T) * (size_t)KC * S * 256;
};

__device__ __forceinline__ void cp_async_elem4(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem8(uint32_t dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// RND: A and C are rounded to the precision's 16-bit operand format after
// their shared-memory reads (binary32 storage only: the same rounding as a
// rounding load)
template <typename T, int NB, bool RND>
__global__ void __launch_bounds__(256) k_narrow_stream(NarrowParams np)
{
    using RING = StreamRing<T>;
    constexpr int KC = RING::KC, S = RING::S;
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    T* ring = (T*)nsm;                                       // [S][KC][256]
    const size_t cbytes = np.stage_c ? sizeof(T) * NB * 256 : 0;
    T* Cs = (T*)(nsm + RING::bytes);                         // [NB][256] when staged
    T* Bs = (T*)(nsm + RING::bytes + cbytes);                // [K][NB]
    int64_t* kA = (int64_t*)(nsm + RING::bytes + cbytes + sizeof(T) * NB * p.K);  // [K]
    int64_t* nC = kA + p.K;                                  // [NB]
    int64_t* nD = nC + NB;                                   // [NB]
    const int t = threadIdx.x;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += 256) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    for (int64_t e = t; e < p.K * NB; e += 256) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        T x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<T>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
        }
        Bs[k * NB + n] = x;
    }
    __syncthreads();

    const int64_t tiles = (p.M + 255) / 256;
    if ((int64_t)blockIdx.x >= tiles) return;
    const int64_t my_tiles = (tiles - 1 - blockIdx.x) / gridDim.x + 1;
    const int nchunks = (int)((p.K + KC - 1) / KC);
    const int64_t total = my_tiles * nchunks;
    const T* A = (const T*)p.A;
    const uint32_t ring_base = (uint32_t)__cvta_generic_to_shared(ring) + (uint32_t)t * sizeof(T);

    // offsets of this thread's row in tile i (A; C and D), -1: no row
    auto row_offsets = [&](int64_t i, int64_t& oA, int64_t& oC, int64_t& oD) {
        const int64_t m = ((int64_t)blockIdx.x + i * gridDim.x) * 256 + t;
        oA = oC = oD = -1;
        if (m >= p.M) return;
        oA = oC = oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
    };
    // producer: the copies of chunk g (tile g / nchunks, chunk g % nchunks)
    int64_t p_tile = -1, p_oA = -1;
    int p_chunk = 0;
    auto issue = [&](int64_t g) {
        if (g < total) {
            if (p_chunk == 0) {
                p_tile++;
                int64_t c_, d_;
                row_offsets(p_tile, p_oA, c_, d_);
            }
            if (p_oA >= 0) {
                const int k0 = p_chunk * KC;
                const uint32_t dst = ring_base + (uint32_t)((g % S) * KC * 256) * sizeof(T);
#pragma unroll
                for (int kk = 0; kk < KC; kk++) {
                    if (k0 + kk < p.K) {
                        const T* src = A + p_oA + kA[k0 + kk];
                        if (sizeof(T) == 4) cp_async_elem4(dst + kk * 256 * sizeof(T), src);
                        else cp_async_elem8(dst + kk * 256 * sizeof(T), src);
                    }
                }
            }
            if (++p_chunk == nchunks) p_chunk = 0;
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
#pragma unroll
    for (int g = 0; g < S - 1; g++) issue(g);

    T acc[NB];
    int64_t oA = -1, oC = -1, oD = -1;
    int c = 0;
    int64_t ti = 0;
    const T al = (T)p.alpha, be = (T)p.beta;
    const uint32_t cs_base = (uint32_t)__cvta_generic_to_shared(Cs) + (uint32_t)t * sizeof(T);
    // the copies of C join the group committed next, so at the tile's last
    // chunk at most min(S - 1, nchunks - 1) younger groups may be pending
    const int c_pending = nchunks - 1 < S - 1 ? nchunks - 1 : S - 1;
    for (int64_t g = 0; g < total; g++) {
        if (c == 0) {
            row_offsets(ti, oA, oC, oD);
#pragma unroll
            for (int n = 0; n < NB; n++) acc[n] = 0;
            if (np.stage_c && oA >= 0) {
                for (int n = 0; n < p.N; n++) {
                    const T* src = (const T*)p.C + oC + nC[n];
                    if (sizeof(T) == 4) cp_async_elem4(cs_base + n * 256 * sizeof(T), src);
                    else cp_async_elem8(cs_base + n * 256 * sizeof(T), src);
                }
            }
        }
        issue(g + S - 1);
        cp_async_wait<S - 1>();  // this thread's copies of chunk g have landed
        if (oA >= 0) {
            const T* a = ring + (size_t)(g % S) * KC * 256 + t;
            const int k0 = c * KC;
            const int kn = p.K - k0 < KC ? (int)(p.K - k0) : KC;
            // B rows as 16-byte vectors (NB is a multiple of 8, the panel
            // 16-byte aligned); a short unroll keeps the loop in the
            // instruction cache
#pragma unroll 2
            for (int kk = 0; kk < kn; kk++) {
                T x = a[kk * 256];
                if (RND) x = round_in<T>(x, p.round_in);
                const T* b = Bs + (k0 + kk) * NB;
                if (sizeof(T) == 4) {
#pragma unroll
                    for (int n = 0; n < NB; n += 4) {
                        const float4 q = *(const float4*)((const float*)b + n);
                        fma2(acc[n], acc[n + 1], x, x, (T)q.x, (T)q.y);
                        fma2(acc[n + 2], acc[n + 3], x, x, (T)q.z, (T)q.w);
                    }
                } else {
#pragma unroll
                    for (int n = 0; n < NB; n += 2) {
                        const double2 q = *(const double2*)((const double*)b + n);
                        fma2(acc[n], acc[n + 1], x, x, (T)q.x, (T)q.y);
                    }
                }
            }
        }
        if (++c == nchunks) {
            c = 0;
            ti++;
            if (oA >= 0 && np.stage_c) {
                static_assert(S == 3, "the waits below cover c_pending = 0 .. S - 1");
                if (c_pending == 0) cp_async_wait<0>();
                else if (c_pending == 1) cp_async_wait<1>();
                const bool d_as_t = p.tD == (sizeof(T) == 4 ? T_F32 : T_F64);
#pragma unroll
                for (int n = 0; n < NB; n++) {
                    if (n < p.N) {
                        T cv = Cs[n * 256 + t];
                        if (RND) cv = round_in<T>(cv, p.round_in);
                        T v = fma(be, cv, al * acc[n]);
                        if (p.conjD && p.conjD_f32) v = (T)(float)v;  // op_D under the F64 precision rounds as conjf
                        if (d_as_t) ((T*)p.D)[oD + nD[n]] = v;
                        else store_elem<T>(p.D, oD + nD[n], p.tD, v, (T)0);
                    }
                }
            } else if (oA >= 0) {
#pragma unroll
                for (int gq = 0; gq < NB; gq += 8) {
                    T cv[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        T im;
                        cv[j] = 0;
                        if (!p.beta_zero && gq + j < p.N) load_rounded<T>(p.C, oC + nC[gq + j], p.tC, p.round_in, cv[j], im);
                    }
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        if (gq + j < p.N) {
                            T v = p.beta_zero ? al * acc[gq + j] : fma(be, cv[j], al * acc[gq + j]);
                            if (p.conjD && p.conjD_f32) v = (T)(float)v;  // op_D under the F64 precision rounds as conjf
                            store_elem<T>(p.D, oD + nD[gq + j], p.tD, v, (T)0);
                        }
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
}

// Variant of k_narrow_stream for products whose A is contiguous along the
// contraction and whose D (and C) along the columns, such as mode-n products
// on the first mode: a thread's own row would be read and written 4 bytes at
// a time with every lane of a warp on a different line. Here each warp
// copies its 32 rows cooperatively, consecutive lanes on consecutive
// addresses: the A chunks into a ring laid out [slot][row][KC + 1] and the
// rows of C into a staging buffer [row][NB + 1]; the thread of a row
// multiplies as before, writes its results into its row of the staging
// buffer, and the warp stores them to D the same cooperative way. Row offsets
// of other lanes come by shuffles; __syncwarp orders the lanes' copies, reads
// and writes (rows never leave their warp, so no block barrier is needed).
constexpr int COOP_KC = 8;

template <typename T, int NB, bool RND>
__global__ void __launch_bounds__(256) k_narrow_coop(NarrowParams np)
{
    // chunks of 8 contracted values keep ring + staging buffer small enough
    // for two blocks per SM
    constexpr int KC = COOP_KC, S = StreamRing<T>::S, KP = KC + 1, NP1 = NB + 1;
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    T* ring = (T*)nsm;                                                  // [S][256][KP]
    T* Ts = ring + (size_t)S * 256 * KP;                                // [256][NP1]
    T* Bs = Ts + (size_t)256 * NP1;                                     // [K][NB]
    int64_t* kA = (int64_t*)(((uintptr_t)(Bs + (size_t)NB * p.K) + 15) & ~(uintptr_t)15);  // [K]
    int64_t* nC = kA + p.K;                                             // [NB]
    int64_t* nD = nC + NB;                                              // [NB]
    const int t = threadIdx.x, lane = t & 31, wbase = t & ~31;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += 256) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    for (int64_t e = t; e < p.K * NB; e += 256) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        T x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<T>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
        }
        Bs[k * NB + n] = x;
    }
    __syncthreads();

    const int64_t tiles = (p.M + 255) / 256;
    if ((int64_t)blockIdx.x >= tiles) return;
    const int64_t my_tiles = (tiles - 1 - blockIdx.x) / gridDim.x + 1;
    const int nchunks = (int)((p.K + KC - 1) / KC);
    const int64_t total = my_tiles * nchunks;
    const T* A = (const T*)p.A;
    const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring);
    const uint32_t ts_s = (uint32_t)__cvta_generic_to_shared(Ts);

    auto row_offsets = [&](int64_t i, int64_t& oA, int64_t& oC, int64_t& oD) {
        const int64_t m = ((int64_t)blockIdx.x + i * gridDim.x) * 256 + t;
        oA = oC = oD = -1;
        if (m >= p.M) return;
        oA = oC = oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
    };
    auto shfl64 = [](int64_t v, int src) { return (int64_t)__shfl_sync(0xffffffffu, (long long)v, src); };
    // producer: the warp's copies of chunk g; every lane calls it with the same g
    int64_t p_tile = -1, p_oA = -1;
    int p_chunk = 0;
    auto issue = [&](int64_t g) {
        if (g < total) {
            if (p_chunk == 0) {
                p_tile++;
                int64_t c_, d_;
                row_offsets(p_tile, p_oA, c_, d_);
            }
            const int k0 = p_chunk * KC;
            const uint32_t slot = ring_s + (uint32_t)(((g % S) * 256 + wbase) * KP) * sizeof(T);
#pragma unroll 4
            for (int f = lane; f < 32 * KC; f += 32) {
                const int r = f / KC, kk = f % KC;
                const int64_t oa = shfl64(p_oA, r);
                if (oa >= 0 && k0 + kk < p.K) {
                    const T* src = A + oa + kA[k0 + kk];
                    const uint32_t dst = slot + (uint32_t)(r * KP + kk) * sizeof(T);
                    if (sizeof(T) == 4) cp_async_elem4(dst, src);
                    else cp_async_elem8(dst, src);
                }
            }
            if (++p_chunk == nchunks) p_chunk = 0;
        }
        cp_async_commit();
    };
#pragma unroll
    for (int g = 0; g < S - 1; g++) issue(g);

    T acc[NB];
    int64_t oA = -1, oC = -1, oD = -1;
    int c = 0;
    int64_t ti = 0;
    const T al = (T)p.alpha, be = (T)p.beta;
    const int c_pending = nchunks - 1 < S - 1 ? nchunks - 1 : S - 1;
    T* trow = Ts + (size_t)t * NP1;
    for (int64_t g = 0; g < total; g++) {
        __syncwarp();  // the slot refilled below was read by every lane in the last round
        if (c == 0) {
            row_offsets(ti, oA, oC, oD);
#pragma unroll
            for (int n = 0; n < NB; n++) acc[n] = 0;
            if (np.stage_c) {
#pragma unroll 4
                for (int f = lane; f < 32 * NB; f += 32) {
                    const int r = f / NB, n = f % NB;
                    const int64_t oc = shfl64(oC, r);
                    if (oc >= 0 && n < p.N) {
                        const T* src = (const T*)p.C + oc + nC[n];
                        const uint32_t dst = ts_s + (uint32_t)((wbase + r) * NP1 + n) * sizeof(T);
                        if (sizeof(T) == 4) cp_async_elem4(dst, src);
                        else cp_async_elem8(dst, src);
                    }
                }
            }
        }
        issue(g + S - 1);
        cp_async_wait<S - 1>();
        __syncwarp();  // the warp's copies of chunk g have landed
        if (oA >= 0) {
            const T* a = ring + (size_t)((g % S) * 256 + t) * KP;
            const int k0 = c * KC;
            const int kn = p.K - k0 < KC ? (int)(p.K - k0) : KC;
#pragma unroll 2
            for (int kk = 0; kk < kn; kk++) {
                T x = a[kk];
                if (RND) x = round_in<T>(x, p.round_in);
                const T* b = Bs + (k0 + kk) * NB;
                if (sizeof(T) == 4) {
#pragma unroll
                    for (int n = 0; n < NB; n += 4) {
                        const float4 q = *(const float4*)((const float*)b + n);
                        fma2(acc[n], acc[n + 1], x, x, (T)q.x, (T)q.y);
                        fma2(acc[n + 2], acc[n + 3], x, x, (T)q.z, (T)q.w);
                    }
                } else {
#pragma unroll
                    for (int n = 0; n < NB; n += 2) {
                        const double2 q = *(const double2*)((const double*)b + n);
                        fma2(acc[n], acc[n + 1], x, x, (T)q.x, (T)q.y);
                    }
                }
            }
        }
        if (++c == nchunks) {
            c = 0;
            ti++;
            static_assert(S == 3, "the waits below cover c_pending = 0 .. S - 1");
            if (np.stage_c) {
                if (c_pending == 0) cp_async_wait<0>();
                else if (c_pending == 1) cp_async_wait<1>();
            }
            __syncwarp();  // the warp's copies of C have landed
            if (oA >= 0) {
#pragma unroll
                for (int n = 0; n < NB; n++) {
                    T cv = np.stage_c ? trow[n] : (T)0;
                    if (RND) cv = round_in<T>(cv, p.round_in);
                    T v = p.beta_zero ? al * acc[n] : fma(be, cv, al * acc[n]);
                    if (p.conjD && p.conjD_f32) v = (T)(float)v;  // op_D under the F64 precision rounds as conjf
                    trow[n] = v;
                }
            }
            __syncwarp();  // the warp's results are in the staging buffer
            const bool d_as_t = p.tD == (sizeof(T) == 4 ? T_F32 : T_F64);
#pragma unroll 4
            for (int f = lane; f < 32 * NB; f += 32) {
                const int r = f / NB, n = f % NB;
                const int64_t od = shfl64(oD, r);
                if (od >= 0 && n < p.N) {
                    const T v = Ts[(size_t)(wbase + r) * NP1 + n];
                    if (d_as_t) ((T*)p.D)[od + nD[n]] = v;
                    else store_elem<T>(p.D, od + nD[n], p.tD, v, (T)0);
                }
            }
        }
    }
    cp_async_wait<0>();
}

// Complex-float variant of k_narrow_stream (A stored as complex float, rows
// contiguous in A and D, at most 32 columns): a ring of complex values per
// thread, B as complex pairs in shared memory, four FMAs per product in the
// order of the tiled kernel, op_A/op_B conjugation at load, and the tiled
// kernel's epilogue (alpha, beta, op_C, op_D) with C loaded eight at a time.
template <int NB>
__global__ void __launch_bounds__(256) k_narrow_cstream(NarrowParams np)
{
    constexpr int KC = 8, S = 3;
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    float2* ring = (float2*)nsm;                 // [S][KC][256]
    float2* Bs = ring + S * KC * 256;            // [K][NB]
    int64_t* kA = (int64_t*)(Bs + (size_t)NB * p.K);  // [K]
    int64_t* nC = kA + p.K;                      // [NB]
    int64_t* nD = nC + NB;                       // [NB]
    const int t = threadIdx.x;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += 256) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    for (int64_t e = t; e < p.K * NB; e += 256) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        float x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<float>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
            if (p.conjB) xi = -xi;
        }
        Bs[k * NB + n] = make_float2(x, xi);
    }
    __syncthreads();

    const int64_t tiles = (p.M + 255) / 256;
    if ((int64_t)blockIdx.x >= tiles) return;
    const int64_t my_tiles = (tiles - 1 - blockIdx.x) / gridDim.x + 1;
    const int nchunks = (int)((p.K + KC - 1) / KC);
    const int64_t total = my_tiles * nchunks;
    const float* A = (const float*)p.A;
    const uint32_t ring_base = (uint32_t)__cvta_generic_to_shared(ring) + (uint32_t)t * sizeof(float2);
    auto row_offsets = [&](int64_t i, int64_t& oA, int64_t& oC, int64_t& oD) {
        const int64_t m = ((int64_t)blockIdx.x + i * gridDim.x) * 256 + t;
        oA = oC = oD = -1;
        if (m >= p.M) return;
        oA = oC = oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
    };
    int64_t p_tile = -1, p_oA = -1;
    int p_chunk = 0;
    auto issue = [&](int64_t g) {
        if (g < total) {
            if (p_chunk == 0) {
                p_tile++;
                int64_t c_, d_;
                row_offsets(p_tile, p_oA, c_, d_);
            }
            if (p_oA >= 0) {
                const int k0 = p_chunk * KC;
                const uint32_t dst = ring_base + (uint32_t)((g % S) * KC * 256) * sizeof(float2);
#pragma unroll
                for (int kk = 0; kk < KC; kk++)
                    if (k0 + kk < p.K) cp_async_elem8(dst + kk * 256 * sizeof(float2), A + 2 * (p_oA + kA[k0 + kk]));
            }
            if (++p_chunk == nchunks) p_chunk = 0;
        }
        cp_async_commit();
    };
#pragma unroll
    for (int g = 0; g < S - 1; g++) issue(g);

    float ar_[NB], ai_[NB];
    int64_t oA = -1, oC = -1, oD = -1;
    int c = 0;
    int64_t ti = 0;
    for (int64_t g = 0; g < total; g++) {
        if (c == 0) {
            row_offsets(ti, oA, oC, oD);
#pragma unroll
            for (int n = 0; n < NB; n++) ar_[n] = ai_[n] = 0.f;
        }
        issue(g + S - 1);
        cp_async_wait<S - 1>();
        if (oA >= 0) {
            const float2* a = ring + (size_t)(g % S) * KC * 256 + t;
            const int k0 = c * KC;
            const int kn = p.K - k0 < KC ? (int)(p.K - k0) : KC;
#pragma unroll 2
            for (int kk = 0; kk < kn; kk++) {
                const float2 x = a[kk * 256];
                const float xr = x.x, xi = p.conjA ? -x.y : x.y;
                const float4* b = (const float4*)(Bs + (k0 + kk) * NB);
#pragma unroll
                for (int n = 0; n < NB; n += 2) {
                    const float4 q = b[n / 2];
                    ar_[n] = fmaf(xr, q.x, ar_[n]);
                    ar_[n] = fmaf(-xi, q.y, ar_[n]);
                    ai_[n] = fmaf(xr, q.y, ai_[n]);
                    ai_[n] = fmaf(xi, q.x, ai_[n]);
                    ar_[n + 1] = fmaf(xr, q.z, ar_[n + 1]);
                    ar_[n + 1] = fmaf(-xi, q.w, ar_[n + 1]);
                    ai_[n + 1] = fmaf(xr, q.w, ai_[n + 1]);
                    ai_[n + 1] = fmaf(xi, q.z, ai_[n + 1]);
                }
            }
        }
        if (++c == nchunks) {
            c = 0;
            ti++;
            if (oA >= 0) {
#pragma unroll
                for (int gq = 0; gq < NB; gq += 8) {
                    float cr[8], ci[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        cr[j] = ci[j] = 0.f;
                        if (!p.beta_zero && gq + j < p.N) load_rounded<float>(p.C, oC + nC[gq + j], p.tC, p.round_in, cr[j], ci[j]);
                    }
#pragma unroll
                    for (int j = 0; j < 8; j++)
                        if (gq + j < p.N) epilogue_store_c<float, true>(p, ar_[gq + j], ai_[gq + j], cr[j], ci[j], oD + nD[gq + j]);
                }
            }
        }
    }
    cp_async_wait<0>();
}

// Register-tiled narrow kernel for A, C and D contiguous along their first
// row mode, VR rows to one vector (binary32: VR = 4, 16 bytes, or 2 when the
// row extents only allow pairs; binary64: VR = 2). A block of NB / 8 x H
// warps (H = 2 for binary32, 4 for binary64, whose tiles hold half as many
// rows per byte) takes tiles of TR = 32 H VR rows. Per chunk of KC
// contracted values (16 KiB of A) the whole block copies the tile's chunk
// with cp.async as VR-row vectors into a ring of S chunks (4; 3 for
// binary64, so that two blocks fit an SM) laid out [k][row]; thread t always
// copies row group t % 32H, so it decodes one row offset per tile. After a
// block barrier, thread (column group c, warp h of c, lane) multiplies row
// group 32 h + lane by columns 8c..8c+7: per contracted value one vector of A and
// two (binary64: four) 16-byte broadcast reads of the B panel feed 8 VR
// independent multiply-adds. At the start of each tile a thread copies the C
// vectors of its own outputs into its own part of a shared-memory buffer
// with cp.async (read back in the epilogue, ordered by cp.async.wait_group);
// D is stored as VR-row vectors.
// Every output sees the same fused multiply-adds in the same order as in
// k_narrow_stream (acc = fma(a_k, b_k, acc) for k = 0, 1, ...; then
// fma(beta, c, alpha acc)), so the two kernels give the same bits.
template <typename T, int VR>
struct NarrowVec;
template <>
struct NarrowVec<float, 4> {
    using V = float4;
    __device__ static void get(const V& v, float (&x)[4]) { x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w; }
    __device__ static V put(const float (&x)[4]) { return make_float4(x[0], x[1], x[2], x[3]); }
};
template <>
struct NarrowVec<float, 2> {
    using V = float2;
    __device__ static void get(const V& v, float (&x)[2]) { x[0] = v.x; x[1] = v.y; }
    __device__ static V put(const float (&x)[2]) { return make_float2(x[0], x[1]); }
};
template <>
struct NarrowVec<double, 2> {
    using V = double2;
    __device__ static void get(const V& v, double (&x)[2]) { x[0] = v.x; x[1] = v.y; }
    __device__ static V put(const double (&x)[2]) { return make_double2(x[0], x[1]); }
};

template <int BYTES>
__device__ __forceinline__ void cp_async_vec(uint32_t dst, const void* src)
{
    if (BYTES == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

constexpr int NVEC_CHUNK_BYTES = 16384, NVEC_MAX_SMEM = 200 * 1024;

// H: warps per column group (TR = 32 H VR rows per tile); S: chunks in the
// ring. Binary64 up to width 32 takes 4 warps per column group (at most 512
// threads of about 80 registers) and 3 chunks, so that two blocks fit an SM.
template <typename T, int NB>
struct NarrowVecShape {
    static constexpr bool WIDE = sizeof(T) == 8 && NB <= 32;
    static constexpr int H = WIDE ? 4 : 2;
    static constexpr int S = WIDE ? 3 : 4;
};

// The multiply-adds of one chunk for the first NP column pairs of a thread's
// 8 columns (kn contracted values; a: the thread's rows in the ring, b: the
// B panel at the chunk's first value and the group's first column).
template <typename T, int NB, int VR, int NP>
__device__ __forceinline__ void nvec_chunk(T (&acc)[VR][8], const T* a, const T* b, int kn)
{
    using NV = NarrowVec<T, VR>;
    using V = typename NV::V;
    constexpr int TR = 32 * NarrowVecShape<T, NB>::H * VR;
#pragma unroll 2
    for (int kk = 0; kk < kn; kk++) {
        T x[VR];
        NV::get(*(const V*)(a + kk * TR), x);
        const T* bk = b + (size_t)kk * NB;
        T bv[8];
        if (sizeof(T) == 4) {
            const float4 q0 = *(const float4*)bk;
            bv[0] = (T)q0.x; bv[1] = (T)q0.y; bv[2] = (T)q0.z; bv[3] = (T)q0.w;
            if (NP > 2) {
                const float4 q1 = *(const float4*)(bk + 4);
                bv[4] = (T)q1.x; bv[5] = (T)q1.y; bv[6] = (T)q1.z; bv[7] = (T)q1.w;
            }
        } else {
#pragma unroll
            for (int n = 0; n < 2 * NP; n += 2) {
                const double2 q = *(const double2*)((const double*)bk + n);
                bv[n] = (T)q.x;
                bv[n + 1] = (T)q.y;
            }
        }
#pragma unroll
        for (int r = 0; r < VR; r++)
#pragma unroll
            for (int n = 0; n < 2 * NP; n += 2) fma2(acc[r][n], acc[r][n + 1], x[r], x[r], bv[n], bv[n + 1]);
    }
}

template <typename T, int NB, int VR, bool RND>
__global__ void __launch_bounds__(NB * 4 * NarrowVecShape<T, NB>::H) k_narrow_vec(NarrowParams np)
{
    constexpr int H = NarrowVecShape<T, NB>::H, S = NarrowVecShape<T, NB>::S;
    constexpr int RG = 32 * H, NT = NB / 8 * RG, TR = RG * VR, KC = NVEC_CHUNK_BYTES / (TR * (int)sizeof(T));
    using NV = NarrowVec<T, VR>;
    using V = typename NV::V;
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    T* ring = (T*)nsm;                                    // [S][KC][TR]
    T* Cs = ring + (size_t)S * KC * TR;                   // [NB][TR] when C is read
    T* Bs = Cs + (p.beta_zero ? 0 : (size_t)NB * TR);     // [K][NB]
    int64_t* kA = (int64_t*)(Bs + (size_t)NB * p.K);      // [K] (NB is a multiple of 8: 8-byte aligned)
    int64_t* nC = kA + p.K;                               // [NB]
    int64_t* nD = nC + NB;                                // [NB]
    const int t = threadIdx.x;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += NT) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    for (int64_t e = t; e < p.K * NB; e += NT) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        T x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<T>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
        }
        Bs[k * NB + n] = x;
    }
    __syncthreads();

    const int64_t tiles = (p.M + TR - 1) / TR;
    if ((int64_t)blockIdx.x >= tiles) return;
    const int64_t my_tiles = (tiles - 1 - blockIdx.x) / gridDim.x + 1;
    const int nchunks = (int)((p.K + KC - 1) / KC);
    const int64_t total = my_tiles * nchunks;
    const T* A = (const T*)p.A;
    // offsets in A, C and D of the first row of row group rg of tile i (-1: past M;
    // the VR rows of a group are consecutive in all three)
    auto group_offsets = [&](int64_t i, int rg, int64_t& oA, int64_t& oC, int64_t& oD) {
        const int64_t m = ((int64_t)blockIdx.x + i * gridDim.x) * TR + (int64_t)rg * VR;
        oA = oC = oD = -1;
        if (m >= p.M) return;
        oA = oC = oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
    };
    // producer: thread t copies row group t % RG at contracted values t / RG, t / RG + NT / RG, ...
    const int prg = t % RG, pk0 = t / RG;
    constexpr int PKS = NT / RG;
    const uint32_t ring_base = (uint32_t)__cvta_generic_to_shared(ring) + (uint32_t)(prg * VR * sizeof(T));
    int64_t p_tile = -1, p_oA = -1;
    int p_chunk = 0;
    auto issue = [&](int64_t g) {
        if (g < total) {
            if (p_chunk == 0) {
                p_tile++;
                int64_t c_, d_;
                group_offsets(p_tile, prg, p_oA, c_, d_);
            }
            if (p_oA >= 0) {
                const int k0 = p_chunk * KC;
                const uint32_t dst = ring_base + (uint32_t)((g % S) * KC * TR * sizeof(T));
                for (int kk = pk0; kk < KC; kk += PKS)
                    if (k0 + kk < p.K) cp_async_vec<VR * (int)sizeof(T)>(dst + kk * TR * sizeof(T), A + p_oA + kA[k0 + kk]);
            }
            if (++p_chunk == nchunks) p_chunk = 0;
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
#pragma unroll
    for (int g = 0; g < S - 1; g++) issue(g);

    const int lane = t & 31, w = t >> 5;
    const int cg = w / H, crg = (w % H) * 32 + lane;
    const T al = (T)p.alpha, be = (T)p.beta;
    T acc[VR][8];
    const uint32_t cs_base = (uint32_t)__cvta_generic_to_shared(Cs) + (uint32_t)((cg * 8 * TR + crg * VR) * sizeof(T));
    int64_t oA = -1, oC = -1, oD = -1;
    int c = 0;
    int64_t ti = 0;
    for (int64_t g = 0; g < total; g++) {
        if (c == 0) {
            group_offsets(ti, crg, oA, oC, oD);
#pragma unroll
            for (int r = 0; r < VR; r++)
#pragma unroll
                for (int n = 0; n < 8; n++) acc[r][n] = 0;
        }
        cp_async_wait<S - 2>();  // this thread's copies of chunk g have landed
        __syncthreads();         // everyone's have; the slot of chunk g - 1 is free
        if (c == 0 && oA >= 0 && !p.beta_zero) {
            // this thread's C vectors join the group committed next
#pragma unroll
            for (int n = 0; n < 8; n++)
                if (cg * 8 + n < p.N)
                    cp_async_vec<VR * (int)sizeof(T)>(cs_base + (uint32_t)(n * TR * sizeof(T)),
                                                       (const T*)p.C + oC + nC[cg * 8 + n]);
        }
        issue(g + S - 1);
        if (RND) {
            // the chunk rounded once in place, each value by one thread
            float4* ch = (float4*)(ring + (size_t)(g % S) * KC * TR);
            for (int e = t; e < KC * TR * (int)sizeof(T) / 16; e += NT) {
                float4 v = ch[e];
                v.x = round_in<float>(v.x, p.round_in);
                v.y = round_in<float>(v.y, p.round_in);
                v.z = round_in<float>(v.z, p.round_in);
                v.w = round_in<float>(v.w, p.round_in);
                ch[e] = v;
            }
            __syncthreads();
        }
        const bool last = c == nchunks - 1;
        if (oA >= 0) {
            const T* a = ring + (size_t)(g % S) * KC * TR + crg * VR;
            const int k0 = c * KC;
            const int kn = p.K - k0 < KC ? (int)(p.K - k0) : KC;
            // column pairs of this warp's group that hold outputs (the last
            // group of a padded width has fewer): warp-uniform choice
            // (4-row binary32 tiles only: the other forms ran slower with the
            // extra code paths)
            const int pairs = (int)((p.N - cg * 8 + 1) / 2);
            const T* b = Bs + (size_t)k0 * NB + cg * 8;
            if constexpr (sizeof(T) == 4 && VR == 4) {
                if (pairs >= 4) nvec_chunk<T, NB, VR, 4>(acc, a, b, kn);
                else if (pairs == 3) nvec_chunk<T, NB, VR, 3>(acc, a, b, kn);
                else if (pairs == 2) nvec_chunk<T, NB, VR, 2>(acc, a, b, kn);
                else nvec_chunk<T, NB, VR, 1>(acc, a, b, kn);
            } else {
                (void)pairs;
                nvec_chunk<T, NB, VR, 4>(acc, a, b, kn);
            }
        }
        if (last) {
            if (oA >= 0) {
                // the tile's C copies went with the group of its first chunk:
                // at most nchunks - 1 younger groups may still be pending
                if (!p.beta_zero && nchunks < S) {
                    static_assert(S <= 4, "the waits below cover nchunks = 1 .. 3");
                    if (nchunks == 1) cp_async_wait<0>();
                    else if (nchunks == 2) cp_async_wait<1>();
                    else cp_async_wait<2>();
                }
#pragma unroll
                for (int n = 0; n < 8; n++) {
                    if (cg * 8 + n < p.N) {
                        T cv[VR] = {};
                        if (!p.beta_zero) NV::get(*(const V*)(Cs + (size_t)(cg * 8 + n) * TR + crg * VR), cv);
                        T y[VR];
#pragma unroll
                        for (int r = 0; r < VR; r++) {
                            if (RND && !p.beta_zero) cv[r] = round_in<T>(cv[r], p.round_in);
                            T v = p.beta_zero ? al * acc[r][n] : fma(be, cv[r], al * acc[r][n]);
                            if (p.conjD && p.conjD_f32) v = (T)(float)v;  // op_D under the F64 precision rounds as conjf
                            y[r] = v;
                        }
                        *(V*)((T*)p.D + oD + nD[cg * 8 + n]) = NV::put(y);
                    }
                }
            }
            c = 0;
            ti++;
        } else {
            c++;
        }
    }
    cp_async_wait<0>();
}

// Complex-float form of k_narrow_vec: A, C and D stored as complex float and
// contiguous along the first row mode (2 rows per 16-byte vector, other
// strides even, bases 16-byte aligned). Tiles of 128 rows, chunks of 16
// contracted values (16 KiB) copied by cp.async into a ring [k][row]; a
// thread owns 2 rows x 8 columns: per contracted value one vector of A and
// four broadcast vectors of B (op_B applied when the panel is built) feed
// 16 complex multiply-adds as paired (re, im) fused multiply-adds in the
// order of k_narrow_cstream (re: a_r b_r then -a_i b_i; im: a_r b_i then
// a_i b_r), so the two kernels give the same bits. C is copied per thread at
// the tile's start; the epilogue is k_narrow_cstream's (epilogue_value) and
// D is stored as 2-row vectors.
template <int NB>
__global__ void __launch_bounds__(NB * 8) k_narrow_cvec(NarrowParams np)
{
    constexpr int H = 2, VR = 2, RG = 32 * H, NT = NB / 8 * RG, TR = RG * VR, S = 4;
    constexpr int KC = NVEC_CHUNK_BYTES / (TR * 8);
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    float2* ring = (float2*)nsm;                            // [S][KC][TR]
    float2* Cs = ring + (size_t)S * KC * TR;                // [NB][TR] when C is read
    float2* Bs = Cs + (p.beta_zero ? 0 : (size_t)NB * TR);  // [K][NB]
    int64_t* kA = (int64_t*)(Bs + (size_t)NB * p.K);        // [K]
    int64_t* nC = kA + p.K;                                 // [NB]
    int64_t* nD = nC + NB;                                  // [NB]
    const int t = threadIdx.x;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += NT) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    for (int64_t e = t; e < p.K * NB; e += NT) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        float x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<float>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
            if (p.conjB) xi = -xi;
        }
        Bs[k * NB + n] = make_float2(x, xi);
    }
    __syncthreads();

    const int64_t tiles = (p.M + TR - 1) / TR;
    if ((int64_t)blockIdx.x >= tiles) return;
    const int64_t my_tiles = (tiles - 1 - blockIdx.x) / gridDim.x + 1;
    const int nchunks = (int)((p.K + KC - 1) / KC);
    const int64_t total = my_tiles * nchunks;
    const float* A = (const float*)p.A;
    auto group_offsets = [&](int64_t i, int rg, int64_t& oA, int64_t& oC, int64_t& oD) {
        const int64_t m = ((int64_t)blockIdx.x + i * gridDim.x) * TR + (int64_t)rg * VR;
        oA = oC = oD = -1;
        if (m >= p.M) return;
        oA = oC = oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
    };
    const int prg = t % RG, pk0 = t / RG;
    constexpr int PKS = NT / RG;
    const uint32_t ring_base = (uint32_t)__cvta_generic_to_shared(ring) + (uint32_t)(prg * VR * 8);
    int64_t p_tile = -1, p_oA = -1;
    int p_chunk = 0;
    auto issue = [&](int64_t g) {
        if (g < total) {
            if (p_chunk == 0) {
                p_tile++;
                int64_t c_, d_;
                group_offsets(p_tile, prg, p_oA, c_, d_);
            }
            if (p_oA >= 0) {
                const int k0 = p_chunk * KC;
                const uint32_t dst = ring_base + (uint32_t)((g % S) * KC * TR * 8);
                for (int kk = pk0; kk < KC; kk += PKS)
                    if (k0 + kk < p.K) cp_async_vec<16>(dst + kk * TR * 8, A + 2 * (p_oA + kA[k0 + kk]));
            }
            if (++p_chunk == nchunks) p_chunk = 0;
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
#pragma unroll
    for (int g = 0; g < S - 1; g++) issue(g);

    const int lane = t & 31, w = t >> 5;
    const int cg = w / H, crg = (w % H) * 32 + lane;
    float ar_[VR][8], ai_[VR][8];
    const uint32_t cs_base = (uint32_t)__cvta_generic_to_shared(Cs) + (uint32_t)((cg * 8 * TR + crg * VR) * 8);
    int64_t oA = -1, oC = -1, oD = -1;
    int c = 0;
    int64_t ti = 0;
    for (int64_t g = 0; g < total; g++) {
        if (c == 0) {
            group_offsets(ti, crg, oA, oC, oD);
#pragma unroll
            for (int r = 0; r < VR; r++)
#pragma unroll
                for (int n = 0; n < 8; n++) ar_[r][n] = ai_[r][n] = 0.f;
        }
        cp_async_wait<S - 2>();  // this thread's copies of chunk g have landed
        __syncthreads();         // everyone's have; the slot of chunk g - 1 is free
        if (c == 0 && oA >= 0 && !p.beta_zero) {
#pragma unroll
            for (int n = 0; n < 8; n++)
                if (cg * 8 + n < p.N)
                    cp_async_vec<16>(cs_base + (uint32_t)(n * TR * 8), (const float*)p.C + 2 * (oC + nC[cg * 8 + n]));
        }
        issue(g + S - 1);
        const bool last = c == nchunks - 1;
        if (oA >= 0) {
            const float2* a = ring + (size_t)(g % S) * KC * TR + crg * VR;
            const int k0 = c * KC;
            const int kn = p.K - k0 < KC ? (int)(p.K - k0) : KC;
#pragma unroll 2
            for (int kk = 0; kk < kn; kk++) {
                const float4 av = *(const float4*)(a + kk * TR);
                const float xr[2] = {av.x, av.z};
                const float xi[2] = {p.conjA ? -av.y : av.y, p.conjA ? -av.w : av.w};
                const float4* b = (const float4*)(Bs + (size_t)(k0 + kk) * NB + cg * 8);
                float br[8], bi[8];
#pragma unroll
                for (int h = 0; h < 4; h++) {
                    const float4 q = b[h];
                    br[2 * h] = q.x;
                    bi[2 * h] = q.y;
                    br[2 * h + 1] = q.z;
                    bi[2 * h + 1] = q.w;
                }
#pragma unroll
                for (int r = 0; r < VR; r++)
#pragma unroll
                    for (int n = 0; n < 8; n++) {
                        fma2(ar_[r][n], ai_[r][n], xr[r], xr[r], br[n], bi[n]);
                        fma2(ar_[r][n], ai_[r][n], -xi[r], xi[r], bi[n], br[n]);
                    }
            }
        }
        if (last) {
            if (oA >= 0) {
                if (!p.beta_zero && nchunks < S) {
                    if (nchunks == 1) cp_async_wait<0>();
                    else if (nchunks == 2) cp_async_wait<1>();
                    else cp_async_wait<2>();
                }
#pragma unroll
                for (int n = 0; n < 8; n++) {
                    if (cg * 8 + n < p.N) {
                        float4 cv = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (!p.beta_zero) cv = *(const float4*)(Cs + (size_t)(cg * 8 + n) * TR + crg * VR);
                        float v0r, v0i, v1r, v1i;
                        epilogue_value<float, true>(p, ar_[0][n], ai_[0][n], cv.x, cv.y, v0r, v0i);
                        epilogue_value<float, true>(p, ar_[1][n], ai_[1][n], cv.z, cv.w, v1r, v1i);
                        *(float4*)((float*)p.D + 2 * (oD + nD[cg * 8 + n])) = make_float4(v0r, v0i, v1r, v1i);
                    }
                }
            }
            c = 0;
            ti++;
        } else {
            c++;
        }
    }
    cp_async_wait<0>();
}

// Register-tiled narrow kernel for binary32 A contiguous along the
// contraction (mode-n products on the first mode: each row of A is a run of
// K values; D's rows run along the columns). Tiles of 128 rows; per chunk of
// 32 contracted values the block copies the tile's chunk with cp.async in
// 16-byte units (8 consecutive threads on one row's 128 bytes) into a ring
// of 2 chunks laid out [row][unit], unit u of row r stored at u ^ ((r / 4) %
// 8), so that the 8 row groups a quarter-warp reads at one unit fall on 8
// different bank groups. Thread (column group c, lane) takes rows
// 4 lane..4 lane + 3 and columns 8c..8c+7: per 4 contracted values four
// 16-byte reads of A and eight broadcast reads of the B panel feed 128
// multiply-adds. C is read and D written directly from the registers (each
// thread 8 consecutive columns of its rows), so a block needs about 55 KiB
// of shared memory and four blocks (20 warps at width 40) share an SM. Every
// output sees the fused multiply-adds of k_narrow_stream in the same order,
// so the kernels give the same bits.
constexpr int NKT_TR = 128, NKT_KC = 32, NKT_S = 2;

template <int NB>
struct NktShape {
    static constexpr int MIN_BLOCKS = NB <= 40 ? 4 : NB <= 48 ? 3 : 2;
};

template <int NB, bool RND>
__global__ void __launch_bounds__(NB * 4, NktShape<NB>::MIN_BLOCKS) k_narrow_kt(NarrowParams np)
{
    constexpr int NT = NB * 4, TR = NKT_TR, KC = NKT_KC, S = NKT_S, UNITS = KC / 4;
    const Params& p = np.p;
    extern __shared__ __align__(16) unsigned char nsm[];
    float* ring = (float*)nsm;                            // [S][TR][KC]
    float* Bs = ring + (size_t)S * TR * KC;               // [K][NB]
    int64_t* kA = (int64_t*)(Bs + (size_t)NB * p.K);      // [K]
    int64_t* nC = kA + p.K;                               // [NB]
    int64_t* nD = nC + NB;                                // [NB]
    const int t = threadIdx.x;
    const int64_t l = blockIdx.y;
    int64_t lA, lB, lC, lD, dummy;
    decode(p.al, l, lA, dummy);
    decode(p.bl, l, lB, dummy);
    decode(p.cl, l, lC, lD);
    for (int64_t k = t; k < p.K; k += NT) {
        int64_t o;
        decode(p.ak, k, o, dummy);
        kA[k] = o + lA;
    }
    if (t < NB) {
        int64_t oc = 0, od = 0;
        if (t < p.N) decode(p.cn, t, oc, od);
        nC[t] = oc + lC;
        nD[t] = od + lD;
    }
    for (int64_t e = t; e < p.K * NB; e += NT) {
        const int64_t k = e / NB;
        const int n = (int)(e % NB);
        float x = 0, xi = 0;
        if (n < p.N) {
            int64_t ob, ok;
            decode(p.bn, n, ob, dummy);
            decode(p.bk, k, ok, dummy);
            load_rounded<float>(p.B, lB + ob + ok, p.tB, p.round_in, x, xi);
        }
        Bs[k * NB + n] = x;
    }
    __syncthreads();

    const int64_t tiles = (p.M + TR - 1) / TR;
    if ((int64_t)blockIdx.x >= tiles) return;
    const int64_t my_tiles = (tiles - 1 - blockIdx.x) / gridDim.x + 1;
    const int nchunks = (int)((p.K + KC - 1) / KC);
    const int64_t total = my_tiles * nchunks;
    const float* A = (const float*)p.A;
    // offsets of row m in A, C and D (-1: past M)
    auto row_offsets = [&](int64_t m, int64_t& oA, int64_t& oC, int64_t& oD) {
        oA = oC = oD = -1;
        if (m >= p.M) return;
        oA = oC = oD = 0;
        uint32_t r = (uint32_t)m;
        for (int j = 0; j < p.am.n; j++) {
            const uint32_t q = fdiv(r, np.fm[j]);
            const int64_t c = (int64_t)(r - q * np.fm[j].d);
            r = q;
            oA += c * p.am.s0[j];
            oC += c * p.cm.s0[j];
            oD += c * p.cm.s1[j];
        }
    };
    auto tile_row0 = [&](int64_t i) { return ((int64_t)blockIdx.x + i * gridDim.x) * TR; };
    // producer: unit c = t + NT u of the chunk is row c / UNITS, unit c % UNITS;
    // NT is a multiple of UNITS, so a thread keeps its unit and walks rows
    const int pu = t % UNITS, pr0 = t / UNITS;
    constexpr int PRS = NT / UNITS;
    const uint32_t ring_base = (uint32_t)__cvta_generic_to_shared(ring);
    int64_t p_tile = -1;
    int p_chunk = 0;
    auto issue = [&](int64_t g) {
        if (g < total) {
            if (p_chunk == 0) p_tile++;
            const int k0 = p_chunk * KC;
            const int k = k0 + 4 * pu;
            if (k < p.K) {
                const uint32_t slot = ring_base + (uint32_t)((g % S) * TR * KC * 4);
                for (int r = pr0; r < TR; r += PRS) {
                    int64_t oA, oC_, oD_;
                    row_offsets(tile_row0(p_tile) + r, oA, oC_, oD_);
                    if (oA < 0) break;
                    const uint32_t dst = slot + (uint32_t)((r * UNITS + (pu ^ ((r >> 2) & 7))) * 16);
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(A + oA + kA[k]) : "memory");
                }
            }
            if (++p_chunk == nchunks) p_chunk = 0;
        }
        cp_async_commit();  // empty groups keep the count uniform
    };
    issue(0);

    const int lane = t & 31, cg = t >> 5;
    const float al = (float)p.alpha, be = (float)p.beta;
    float acc[4][8];
    int c = 0;
    int64_t ti = 0;
    for (int64_t g = 0; g < total; g++) {
        cp_async_wait<0>();  // this thread's copies of chunk g have landed
        __syncthreads();     // everyone's have; the other slot (chunk g - 1) is free
        issue(g + 1);
        if (RND) {
            // the chunk rounded once in place, each value by one thread
            float4* ch = (float4*)(ring + (size_t)(g % S) * TR * KC);
            for (int e = t; e < TR * KC / 4; e += NT) {
                float4 v = ch[e];
                v.x = round_in<float>(v.x, p.round_in);
                v.y = round_in<float>(v.y, p.round_in);
                v.z = round_in<float>(v.z, p.round_in);
                v.w = round_in<float>(v.w, p.round_in);
                ch[e] = v;
            }
            __syncthreads();
        }
        if (c == 0) {
#pragma unroll
            for (int j = 0; j < 4; j++)
#pragma unroll
                for (int n = 0; n < 8; n++) acc[j][n] = 0.f;
        }
        {
            const float* slot = ring + (size_t)(g % S) * TR * KC;
            const int k0 = c * KC;
            const int kn = p.K - k0 < KC ? (int)(p.K - k0) : KC;
            for (int u = 0; u < kn / 4; u++) {
                float a[4][4];
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int r = 4 * lane + j;
                    const float4 q = *(const float4*)(slot + (size_t)(r * UNITS + (u ^ (lane & 7))) * 4);
                    a[j][0] = q.x; a[j][1] = q.y; a[j][2] = q.z; a[j][3] = q.w;
                }
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const float* b = Bs + (size_t)(k0 + 4 * u + kk) * NB + cg * 8;
                    const float4 q0 = *(const float4*)b, q1 = *(const float4*)(b + 4);
                    const float bv[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float x = a[j][kk];
#pragma unroll
                        for (int n = 0; n < 8; n += 2) fma2(acc[j][n], acc[j][n + 1], x, x, bv[n], bv[n + 1]);
                    }
                }
            }
        }
        if (++c == nchunks) {
            // D = alpha acc + beta C for this thread's 4 rows x 8 columns,
            // straight from and to global memory
            const int64_t m0 = tile_row0(ti);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                int64_t oA_, oC, oD;
                row_offsets(m0 + 4 * lane + j, oA_, oC, oD);
                if (oA_ < 0) break;
                float cv[8];
#pragma unroll
                for (int n = 0; n < 8; n++) {
                    cv[n] = 0.f;
                    if (!p.beta_zero && cg * 8 + n < p.N) cv[n] = ((const float*)p.C)[oC + nC[cg * 8 + n]];
                }
#pragma unroll
                for (int n = 0; n < 8; n++) {
                    if (cg * 8 + n < p.N) {
                        float c1 = cv[n];
                        if (RND && !p.beta_zero) c1 = round_in<float>(c1, p.round_in);
                        float v = p.beta_zero ? al * acc[j][n] : fmaf(be, c1, al * acc[j][n]);
                        if (p.conjD && p.conjD_f32) v = (float)v;
                        ((float*)p.D)[oD + nD[cg * 8 + n]] = v;
                    }
                }
            }
            c = 0;
            ti++;
        }
    }
    cp_async_wait<0>();
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

// Whether a real operand stored as the compute type can be read w elements
// at a time (w = 4 binary32, 2 binary64): its contiguous mode (the first row
// mode when rows_fast, else the first contracted mode) has stride 1 and an
// extent divisible by w, every other stride keeps w-element alignment and the
// base is 16-byte aligned, so the w neighbours of an aligned group lie in one
// 16-byte word (the extents then make M or K a multiple of w, and a group is
// wholly in range or not).
static bool vec_side(const simt::Modes& rows, const simt::Modes& ks, const simt::Modes& ls, int rows_fast,
                     const void* base, int t, int want_t, int w)
{
    if (t != want_t || ((uintptr_t)base & 15) != 0) return false;
    const simt::Modes& f = rows_fast ? rows : ks;
    const simt::Modes& o = rows_fast ? ks : rows;
    if (f.n < 1 || f.s0[0] != 1 || f.ext[0] % w != 0) return false;
    for (int j = 1; j < f.n; j++)
        if (f.s0[j] % w != 0) return false;
    for (int j = 0; j < o.n; j++)
        if (o.s0[j] % w != 0) return false;
    for (int j = 0; j < ls.n; j++)
        if (ls.s0[j] % w != 0) return false;
    return true;
}

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
    if (P->compute == TB_R32 || P->compute == TB_R64) {
        const int want = P->compute == TB_R32 ? T_F32 : T_F64, w = P->compute == TB_R32 ? 4 : 2;
        p.a_vec = vec_side(p.am, p.ak, p.al, p.a_rows_fast, p.A, p.tA, want, w);
        p.b_vec = vec_side(p.bn, p.bk, p.bl, p.b_rows_fast, p.B, p.tB, want, w);
    }
}

static int narrow_width(const tb_plan* P, const simt::Params& p);

size_t simt_scratch_bytes(const tb_plan* P)
{
    using namespace simt;
    Params p;
    tb_ptrs d = {nullptr, nullptr, nullptr, nullptr};
    simt_params(P, &d, p);
    if (narrow_width(P, p)) return 0;
    return with_cfg(P->compute, tile_for(P->compute, p.M, p.N), [&](auto cfg) { return decltype(cfg)::split(p).ws_bytes; });
}

// padded width of the narrow kernel for a turned view, or 0 when it does not apply
static bool vec_choice_ok(const simt::Params& p, int nb, size_t es);
static bool cvec_ok(const simt::Params& p, int nb);

static int narrow_width(const tb_plan* P, const simt::Params& p)
{
    // complex float: the streaming kernels (A read as stored, rows contiguous
    // in A and D); more than 32 columns only in 2-row vectors (k_narrow_cvec)
    const bool cplx = P->compute == TB_C32;
    if (cplx && (p.N > 64 || p.tA != T_C32 || p.round_in != TB_ROUND_NONE || !p.a_rows_fast || !p.d_rows_fast ||
                 (uintptr_t)p.A % 8 != 0))
        return 0;
    if (P->compute != TB_R32 && P->compute != TB_R64 && !cplx) return 0;
    if (p.N > 64 || p.M < 1024 || p.M >= (1ll << 31) || p.L > 65535 || p.K < 1) return 0;
    const int nb = (int)((p.N + 7) / 8 * 8);  // widths in steps of 8: at most 7 padded columns
    const size_t es = P->compute == TB_R32 ? 4 : 8;
    const size_t smem = es * (size_t)nb * (size_t)p.K + 8 * ((size_t)p.K + 2 * (size_t)nb);
    if (smem > (size_t)simt::NARROW_MAX_SMEM) return 0;
    if (cplx) return p.N <= 32 || cvec_ok(p, nb) ? nb : 0;
    // the one-row-per-thread kernels pay only where a 64-wide tile wastes
    // work or the contraction is short; the register tiles also beyond
    if (p.N > 48 && p.K > 64 && !vec_choice_ok(p, nb, es)) return 0;
    return nb;
}

// Which narrow kernel a turned view runs, and what it stages: one decision
// for the launcher and for tapp_b200_describe_plan.
//   NK_REG     k_narrow: register prefetch, conversion and rounding at load
//   NK_STREAM  k_narrow_stream: A read as stored (binary32, also under the
//              16-bit precisions, which round after the copy; binary64 up to
//              width 48 with D contiguous along its rows)
//   NK_COOP    k_narrow_coop: binary32 streaming with A contiguous along the
//              contraction and D along the columns (C staged whenever read)
//   NK_VEC     k_narrow_vec: A, C and D contiguous along the first row mode,
//              read and written as VR-row vectors (register tiles)
//   NK_KT      k_narrow_kt: binary32 A contiguous along the contraction in
//              16-byte runs (register tiles, swizzled shared-memory ring)
enum { NK_REG = 1, NK_STREAM = 2, NK_COOP = 3, NK_VEC = 5, NK_KT = 7 };
struct NarrowChoice {
    int kind;
    bool rnd, stage_c;
    size_t smem;
    int vr;  // NK_VEC: rows per vector
};

// whether k_narrow_vec can read A and C and write D as vr-row vectors: the
// first row mode has stride 1 in all three and an extent divisible by vr,
// every other stride and every base keeps the vector's alignment
static bool nvec_layout(const simt::Params& p, int vr, size_t es)
{
    auto strides_ok = [&](const simt::Modes& m, bool d_side, int from) {
        for (int j = from; j < m.n; j++)
            if ((d_side ? m.s1[j] : m.s0[j]) % vr != 0) return false;
        return true;
    };
    const uintptr_t vb = (uintptr_t)vr * es;
    if (p.am.n < 1 || p.am.s0[0] != 1 || p.am.ext[0] % vr != 0 || p.cm.s1[0] != 1) return false;
    if (!strides_ok(p.am, false, 1) || !strides_ok(p.ak, false, 0) || !strides_ok(p.al, false, 0)) return false;
    if (!strides_ok(p.cm, true, 1) || !strides_ok(p.cn, true, 0) || !strides_ok(p.cl, true, 0)) return false;
    if ((uintptr_t)p.A % vb != 0 || (uintptr_t)p.D % vb != 0) return false;
    if (!p.beta_zero && (p.cm.s0[0] != 1 || !strides_ok(p.cm, false, 1) || !strides_ok(p.cn, false, 0) ||
                         !strides_ok(p.cl, false, 0) || (uintptr_t)p.C % vb != 0))
        return false;
    return true;
}

// whether k_narrow_kt can copy A's rows in 16-byte runs along the
// contraction: the first contracted mode has stride 1 and an extent
// divisible by 4, every other stride of A and its base keep 16-byte alignment
static bool nkt_layout(const simt::Params& p)
{
    auto strides_ok = [&](const simt::Modes& m, int from) {
        for (int j = from; j < m.n; j++)
            if (m.s0[j] % 4 != 0) return false;
        return true;
    };
    return p.ak.n >= 1 && p.ak.s0[0] == 1 && p.ak.ext[0] % 4 == 0 && strides_ok(p.ak, 1) && strides_ok(p.am, 0) &&
           strides_ok(p.al, 0) && (uintptr_t)p.A % 16 == 0;
}

static size_t nkt_smem(const simt::Params& p, int nb)
{
    using namespace simt;
    return (size_t)NKT_S * NKT_TR * NKT_KC * 4 + 4 * (size_t)nb * (size_t)p.K + 8 * ((size_t)p.K + 2 * (size_t)nb);
}

static NarrowChoice narrow_choice(const simt::Params& p, int nb, size_t es)
{
    using namespace simt;
    NarrowChoice c;
    const bool f32 = es == 4;
    const size_t ring = f32 ? StreamRing<float>::bytes : StreamRing<double>::bytes;
    size_t smem = es * (size_t)nb * (size_t)p.K + 8 * ((size_t)p.K + 2 * (size_t)nb);
    // binary64 wider than 48 leaves no registers for the ring's bookkeeping;
    // binary64 with D contiguous along the columns: each thread would write a
    // row of its own, and the ring only costs occupancy
    const bool stream_ok = f32 || nb <= 48;
    const int t_own = f32 ? T_F32 : T_F64;
    c.rnd = p.round_in != TB_ROUND_NONE;  // rounding after the copy is the rounding load's for binary32 only
    c.vr = 0;
    if (p.tA == t_own && p.tD == t_own && (p.beta_zero || p.tC == t_own) && (f32 || !c.rnd)) {
        const int vr = f32 ? (nvec_layout(p, 4, es) ? 4 : nvec_layout(p, 2, es) ? 2 : 0) : (nvec_layout(p, 2, es) ? 2 : 0);
        const bool wide = !f32 && nb <= 32;  // NarrowVecShape
        const int H = wide ? 4 : 2, S = wide ? 3 : 4;
        const size_t vsmem = (size_t)S * NVEC_CHUNK_BYTES + (p.beta_zero ? 0 : es * (size_t)nb * 32 * H * vr) +
                             es * (size_t)nb * (size_t)p.K + 8 * ((size_t)p.K + 2 * (size_t)nb);
        if (vr && vsmem <= (size_t)NVEC_MAX_SMEM) {
            c.kind = NK_VEC;
            c.vr = vr;
            c.stage_c = false;
            c.smem = vsmem;
            return c;
        }
        // widths of 24 and more: at least 3 warps a block
        if (f32 && nb >= 24 && nkt_layout(p) && nkt_smem(p, nb) <= (size_t)NVEC_MAX_SMEM) {
            c.kind = NK_KT;
            c.stage_c = false;
            c.smem = nkt_smem(p, nb);
            return c;
        }
    }
    const bool stream = stream_ok && p.tA == t_own && (!c.rnd || f32) && (uintptr_t)p.A % es == 0 &&
                        (f32 || p.d_rows_fast);
    c.kind = stream ? NK_STREAM : NK_REG;
    c.stage_c = false;
    if (stream) {
        smem += ring;
        const size_t cb = es * (size_t)nb * 256;
        if (!p.beta_zero && p.tC == t_own && (uintptr_t)p.C % es == 0 && smem + cb <= (size_t)NARROW_MAX_SMEM + ring) {
            c.stage_c = true;
            smem += cb;
        }
    }
    if (f32 && stream && !p.a_rows_fast && !p.d_rows_fast) {
        const size_t coop_smem = es * (size_t)StreamRing<float>::S * 256 * (COOP_KC + 1) + es * 256 * (nb + 1) +
                                 es * (size_t)nb * (size_t)p.K + 16 + 8 * ((size_t)p.K + 2 * (size_t)nb);
        const bool c_ok = p.beta_zero || (p.tC == t_own && (uintptr_t)p.C % es == 0);
        if (c_ok && coop_smem <= NARROW_COOP_SMEM) {
            c.kind = NK_COOP;
            c.stage_c = !p.beta_zero;
            smem = coop_smem;
        }
    }
    c.smem = smem;
    return c;
}

// whether a register-tiled kernel takes a product of this width
static bool vec_choice_ok(const simt::Params& p, int nb, size_t es)
{
    const int k = narrow_choice(p, nb, es).kind;
    return k == NK_VEC || k == NK_KT;
}

template <typename T, int NB>
static cudaError_t launch_narrow_vec(simt::NarrowParams& np, const NarrowChoice& ch, cudaStream_t s)
{
    using namespace simt;
    const Params& p = np.p;
    void (*kern)(NarrowParams);
    int variant = 0;
    if constexpr (sizeof(T) == 4) {
        if (ch.vr == 4) kern = ch.rnd ? k_narrow_vec<float, NB, 4, true> : k_narrow_vec<float, NB, 4, false>;
        else kern = ch.rnd ? k_narrow_vec<float, NB, 2, true> : k_narrow_vec<float, NB, 2, false>;
        variant = (ch.vr == 4 ? 0 : 2) + (int)ch.rnd;
    } else {
        kern = k_narrow_vec<double, NB, 2, false>;
    }
    static int attr_done[64][4];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev][variant]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, NVEC_MAX_SMEM);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev][variant] = 1;
    }
    constexpr int H = NarrowVecShape<T, NB>::H;
    const int threads = NB * 4 * H;
    const int64_t tiles = (p.M + 32 * H * ch.vr - 1) / (32 * H * ch.vr);
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, ch.smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    int64_t gx = ((int64_t)148 * per_sm + p.L - 1) / p.L;
    if (gx > tiles) gx = tiles;
    if (gx < 1) gx = 1;
    kern<<<dim3((unsigned)gx, (unsigned)p.L), threads, ch.smem, s>>>(np);
    count_launch();
    return cudaGetLastError();
}

template <int NB>
static cudaError_t launch_narrow_kt(simt::NarrowParams& np, const NarrowChoice& ch, cudaStream_t s)
{
    using namespace simt;
    const Params& p = np.p;
    void (*kern)(NarrowParams) = ch.rnd ? k_narrow_kt<NB, true> : k_narrow_kt<NB, false>;
    static int attr_done[64][2];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev][ch.rnd]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, NVEC_MAX_SMEM);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev][ch.rnd] = 1;
    }
    const int threads = NB * 4;
    const int64_t tiles = (p.M + NKT_TR - 1) / NKT_TR;
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, ch.smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    int64_t gx = ((int64_t)148 * per_sm + p.L - 1) / p.L;
    if (gx > tiles) gx = tiles;
    if (gx < 1) gx = 1;
    kern<<<dim3((unsigned)gx, (unsigned)p.L), threads, ch.smem, s>>>(np);
    count_launch();
    return cudaGetLastError();
}

template <typename T, int NB>
static cudaError_t launch_narrow_t(simt::NarrowParams& np, cudaStream_t s)
{
    using namespace simt;
    const Params& p = np.p;
    const NarrowChoice ch = narrow_choice(p, NB, sizeof(T));
    if (ch.kind == NK_VEC) return launch_narrow_vec<T, NB>(np, ch, s);
    if constexpr (sizeof(T) == 4 && NB >= 24) {
        if (ch.kind == NK_KT) return launch_narrow_kt<NB>(np, ch, s);
    }
    const bool plain_a = p.tA == (sizeof(T) == 4 ? T_F32 : T_F64) && p.round_in == TB_ROUND_NONE;
    void (*kern)(NarrowParams) = plain_a ? k_narrow<T, NB, true> : k_narrow<T, NB, false>;
    if constexpr (sizeof(T) == 4) {
        if (ch.kind == NK_STREAM) kern = ch.rnd ? k_narrow_stream<T, NB, true> : k_narrow_stream<T, NB, false>;
        if (ch.kind == NK_COOP) kern = ch.rnd ? k_narrow_coop<T, NB, true> : k_narrow_coop<T, NB, false>;
    } else if constexpr (NB <= 48) {
        if (ch.kind == NK_STREAM) kern = k_narrow_stream<T, NB, false>;
    }
    np.stage_c = ch.stage_c ? 1 : 0;
    const size_t smem = ch.smem;
    const bool stream = ch.kind != NK_REG;
    const int variant = ch.kind == NK_COOP ? 4 + (int)ch.rnd : ch.kind == NK_STREAM ? 2 + (int)ch.rnd : plain_a ? 1 : 0;
    static int attr_done[64][6];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev][variant]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             variant >= 4 ? NARROW_COOP_SMEM : NARROW_MAX_SMEM + (int)StreamRing<T>::bytes);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev][variant] = 1;
    }
    const int64_t tiles = (p.M + 255) / 256;
    // the streaming kernel: one wave of resident blocks; the others: 8 per SM
    int per_sm = 8;
    if (stream && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem) != cudaSuccess || per_sm < 1))
        per_sm = 1;
    int64_t gx = ((int64_t)148 * per_sm + p.L - 1) / p.L;
    if (gx > tiles) gx = tiles;
    if (gx < 1) gx = 1;
    kern<<<dim3((unsigned)gx, (unsigned)p.L), 256, smem, s>>>(np);
    count_launch();
    return cudaGetLastError();
}

// complex float in 2-row vectors (k_narrow_cvec): complex-float A, C and D,
// rows contiguous and 16-byte aligned, no operand rounding
static size_t cvec_smem(const simt::Params& p, int nb)
{
    return (size_t)4 * simt::NVEC_CHUNK_BYTES + (p.beta_zero ? 0 : (size_t)8 * nb * 128) + (size_t)8 * nb * (size_t)p.K +
           8 * ((size_t)p.K + 2 * (size_t)nb);
}

static bool cvec_ok(const simt::Params& p, int nb)
{
    return p.tA == T_C32 && p.tD == T_C32 && (p.beta_zero || p.tC == T_C32) && p.round_in == TB_ROUND_NONE &&
           nvec_layout(p, 2, 8) && cvec_smem(p, nb) <= (size_t)simt::NVEC_MAX_SMEM;
}

template <int NB>
static cudaError_t launch_narrow_cvec(simt::NarrowParams& np, cudaStream_t s)
{
    using namespace simt;
    const Params& p = np.p;
    const size_t smem = cvec_smem(p, NB);
    auto kern = k_narrow_cvec<NB>;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, NVEC_MAX_SMEM);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    const int threads = NB * 8;
    const int64_t tiles = (p.M + 127) / 128;
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    int64_t gx = ((int64_t)148 * per_sm + p.L - 1) / p.L;
    if (gx > tiles) gx = tiles;
    if (gx < 1) gx = 1;
    kern<<<dim3((unsigned)gx, (unsigned)p.L), threads, smem, s>>>(np);
    count_launch();
    return cudaGetLastError();
}

template <int NB>
static cudaError_t launch_narrow_c(simt::NarrowParams& np, cudaStream_t s)
{
    using namespace simt;
    const Params& p = np.p;
    if (cvec_ok(p, NB)) return launch_narrow_cvec<NB>(np, s);
    const size_t smem = sizeof(float2) * (size_t)(3 * 8 * 256) + sizeof(float2) * NB * (size_t)p.K +
                        8 * ((size_t)p.K + 2 * NB);
    auto kern = k_narrow_cstream<NB>;
    static int attr_done[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             NARROW_MAX_SMEM + (int)(sizeof(float2) * 3 * 8 * 256));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_done[dev] = 1;
    }
    const int64_t tiles = (p.M + 255) / 256;
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
    int64_t gx = ((int64_t)148 * per_sm + p.L - 1) / p.L;
    if (gx > tiles) gx = tiles;
    if (gx < 1) gx = 1;
    kern<<<dim3((unsigned)gx, (unsigned)p.L), 256, smem, s>>>(np);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_simt(const tb_plan* P, const tb_ptrs* d, cudaStream_t s)
{
    using namespace simt;
    Params p;
    simt_params(P, d, p);
    const int nb = narrow_width(P, p);
    if (nb) {
        NarrowParams np;
        memset(&np, 0, sizeof(np));
        np.p = p;
        np.nb = nb;
        for (int j = 0; j < p.am.n; j++) np.fm[j] = make_fastdiv((uint32_t)p.am.ext[j]);
        if (P->compute == TB_C32) {
            switch (nb) {
            case 8: return launch_narrow_c<8>(np, s);
            case 16: return launch_narrow_c<16>(np, s);
            case 24: return launch_narrow_c<24>(np, s);
            case 32: return launch_narrow_c<32>(np, s);
            // wider: 2-row vectors only (narrow_width checked cvec_ok)
            case 40: return launch_narrow_cvec<40>(np, s);
            case 48: return launch_narrow_cvec<48>(np, s);
            case 56: return launch_narrow_cvec<56>(np, s);
            default: return launch_narrow_cvec<64>(np, s);
            }
        }
        if (P->compute == TB_R32) {
            switch (nb) {
            case 8: return launch_narrow_t<float, 8>(np, s);
            case 16: return launch_narrow_t<float, 16>(np, s);
            case 24: return launch_narrow_t<float, 24>(np, s);
            case 32: return launch_narrow_t<float, 32>(np, s);
            case 40: return launch_narrow_t<float, 40>(np, s);
            case 48: return launch_narrow_t<float, 48>(np, s);
            case 56: return launch_narrow_t<float, 56>(np, s);
            default: return launch_narrow_t<float, 64>(np, s);
            }
        }
        switch (nb) {
        case 8: return launch_narrow_t<double, 8>(np, s);
        case 16: return launch_narrow_t<double, 16>(np, s);
        case 24: return launch_narrow_t<double, 24>(np, s);
        case 32: return launch_narrow_t<double, 32>(np, s);
        case 40: return launch_narrow_t<double, 40>(np, s);
        case 48: return launch_narrow_t<double, 48>(np, s);
        case 56: return launch_narrow_t<double, 56>(np, s);
        default: return launch_narrow_t<double, 64>(np, s);
        }
    }
    return with_cfg(P->compute, tile_for(P->compute, p.M, p.N), [&](auto cfg) { return decltype(cfg)::launch(p, s); });
}

}  // namespace tb

// The CUDA-core kernel a plan of the simt path runs, for operands aligned to
// their element size and, for 5, to the row vector (the launcher falls back
// to another narrow or the tiled kernel for others): 0 tiled, 1 narrow with
// register prefetch, 2 narrow streaming, 3 narrow cooperative, 4 complex
// narrow streaming, 5 narrow with row vectors, 6 complex narrow with row
// vectors, 7 narrow with contraction runs. No device call.
extern "C" int tbk_simt_kernel(const tb_plan* P)
{
    using namespace tb;
    simt::Params p;
    tb_ptrs d = {nullptr, nullptr, nullptr, nullptr};
    simt_params(P, &d, p);
    const int nb = narrow_width(P, p);
    if (!nb) return 0;
    if (P->compute == TB_C32) return cvec_ok(p, nb) ? 6 : 4;
    return narrow_choice(p, nb, P->compute == TB_R32 ? 4 : 8).kind;
}
