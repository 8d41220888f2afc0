// Device-side building blocks of the tensor-core kernels (tc.cu, group.cu):
// tile geometry, the launch parameter structs, mbarrier waits with time
// limits, TMA and tcgen05 instruction wrappers, shared-memory descriptors,
// the epilogue's element helpers and the in-place binary32 converters.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "../tb_plan.h"
#include "tb_common.cuh"

namespace tb {
namespace tc {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;
constexpr int B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;

// Stage geometry per CTA. One CTA: A 128x64 and B 256x64 per stage, 4
// stages. CTA pair (cta_group::2, 256x256 tiles): each CTA holds its 128
// rows of A and 128 of the 256 columns of B, 6 stages. Same 192 KiB.
template <bool CTA2>
struct Geo {
    static constexpr int stages = CTA2 ? 6 : 4;
    static constexpr int b_rows = CTA2 ? 128 : 256;   // rows of B per CTA per stage
    static constexpr int a_bytes = BM * BK * 2;
    static constexpr int b_bytes = b_rows * BK * 2;
    static constexpr int stage_bytes = a_bytes + b_bytes;
    static constexpr int tile_m = CTA2 ? 2 * BM : BM;  // output rows per tile
};
static_assert(Geo<true>::stages * Geo<true>::stage_bytes == STAGES * STAGE_BYTES, "same ring size");
constexpr int TMEM_COLS = 512;
constexpr int EPI_WARPS = 8;                    // two warps per TMEM lane quarter
constexpr int EPI_THREADS = EPI_WARPS * 32;
constexpr int NTHREADS = 128 + EPI_THREADS;
constexpr int STAGE_EPI_BYTES = 32 * 32 * 4;  // one 32x32 fp32 box per epilogue warp
// tiles | barriers | epilogue staging (the per-thread epilogue keeps its
// column-offset tables in the staging area instead)
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/ + 8 * STAGE_EPI_BYTES;
static_assert(2 * BN * 8 <= 8 * STAGE_EPI_BYTES, "column tables fit in the staging area");
static_assert(SMEM_BYTES <= 232448, "dynamic shared memory limit of sm_100");
constexpr unsigned long long WAIT_NS = 4000000000ull;  // 4 s per wait

struct ModeList {
    int32_t n;
    int32_t pad;
    int64_t ext[TB_MAXMODES];
    int64_t s0[TB_MAXMODES];  // stride in the first tensor (C, or the packed source)
    int64_t s1[TB_MAXMODES];  // stride in the second tensor (D)
};

__host__ __device__ inline void decode2(const ModeList& m, int64_t idx, int64_t& o0, int64_t& o1)
{
    o0 = 0;
    o1 = 0;
    for (int j = 0; j < m.n; j++) {
        int64_t c = idx % m.ext[j];
        idx /= m.ext[j];
        o0 += c * m.s0[j];
        o1 += c * m.s1[j];
    }
}


// ---------------------------------------------------------------------------
// GEMM
struct EpiParams {
    const void* C;
    void* D;
    int32_t tC, tD, cplx, beta_zero, conjC, conjD, conjD_f32, round_C;
    float alpha_re, alpha_im, beta_re, beta_im;
    int64_t M, N, L;   // output sizes (N counts complex elements when cplx)
    ModeList mm, nn, ll;  // s0 = stride in C, s1 = stride in D
    // EPI_I32 (integer slice products): W[l][m][n] = (first ? 0 : W) + level_scale * acc,
    // W dense binary64 with N columns
    double* W;
    double level_scale;
    int32_t w_first, w_pad;
    // batched product: C and D of batch b = l / Lper (device arrays), else NULL;
    // with the TMA epilogue, also their tensor maps (tmCs NULL when beta = 0)
    const void* const* Cs;
    void* const* Ds;
    const CUtensorMap* tmCs;
    const CUtensorMap* tmDs;
    int64_t Lper;
};

// An operand the tensor-core kernels read in place from binary32 storage:
// index -> element offset maps of its row (M or N), contracted and batch
// modes (at most 4 each, indices below 2^31), and its major side: mn = 1
// when it is closer to contiguous along a row mode than along a contracted
// mode (MN-major tiles), else K-major tiles. With vec = 1 the contiguous
// mode has stride 1 and an extent divisible by 8, every other stride is a
// multiple of 4 and the base is 16-byte aligned, so each run of 8 elements
// along it is two 16-byte loads (the single-product kernel needs this);
// with vec = 0 (grouped kernel only) elements are loaded one by one through
// offset tables.
struct CvtDim {
    int32_t n;
    uint32_t size;
    FastDiv div[4];
    int64_t st[4];
};
struct CvtOperand {
    const float* base;
    const void* const* bases;  // batched product: base of batch b = l / lper, else NULL
    int64_t lper;              // batch modes per batch
    int32_t mn;                // contiguous along a row mode (MN-major tiles), else along k
    int32_t vec;               // runs of 8 elements are two aligned 16-byte loads, else element loads
    CvtDim rows, ks, ls;
};

struct GemmParams {
    int32_t tiles_m, tiles_n, num_tiles, num_kb;
    EpiParams e;
    int* error;       // set to 1 when a wait times out
    // The last split_tiles tiles (the last, partial round of the persistent
    // schedule) run as two work items each, the two halves of the
    // contraction. Whichever half finishes first (pcount, per tile and CTA
    // rank) writes its raw sums to partial ([col][row]) and raises pready; the
    // other adds them and runs the epilogue. The first is running when the
    // second waits for it, so the wait cannot depend on scheduling. pcount and
    // pready start at zero.
    int32_t split_tiles, pad_s;
    float* partial;
    int* pcount;
    int* pready;
    // Operands read in place (16-bit storage, no pack): the tensor map has
    // the dims (row mode 0, k mode 0, row mode 1, k mode 1, batch) in the
    // MN-major case and (k mode 0, row mode 0, k mode 1, row mode 1, batch)
    // in the K-major case; every stage loads 64-row x 64-k boxes. e0/k0 are
    // the extents of row mode 0 and k mode 0 (multiples of 64).
    int32_t a_direct, b_direct, a_mn, b_mn;
    int32_t a_e0, a_k0, b_e0, b_k0;
    // box shape of each direct operand: 0 one 64-row box per 64 rows, 1 all
    // rows in one box along row mode 1 (row mode 0 has extent 64), 2 all rows
    // in one box along row mode 0 (K-major, extent a multiple of the rows)
    int32_t a_box, b_box;
    // logical dims present in each direct operand's map (bit j: dim j; dims
    // of extent 1 are left out, fewer dims copy faster)
    int32_t a_dims, b_dims;
    // split-bfloat16 GEMM reading binary32 operands in place (k_gemm<.., CVT>)
    CvtOperand ca, cb;
    // split-bfloat16 GEMM from [hi | lo] panels (k_gemm<.., 2>): k offset of the lo parts
    int32_t lo_off, pad_lo;
};

// work item it of the persistent schedule: tile, contraction-block range and
// role (0 whole tile, 1 and 2 the two halves of a split tile)
struct Item {
    int tile, kb0, kb1, role;
};

__device__ __forceinline__ Item item_of(const GemmParams& p, int it)
{
    const int nfull = p.num_tiles - p.split_tiles;
    if (it < nfull) return Item{it, 0, p.num_kb, 0};
    const int j = it - nfull, kh = p.num_kb / 2;
    return (j & 1) ? Item{nfull + j / 2, kh, p.num_kb, 2} : Item{nfull + j / 2, 0, kh, 1};
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// try_wait with cluster-scope acquire: for a barrier that threads of the
// other CTA of a pair arrive on (release, cluster scope) after writing
// shared memory that this thread's MMAs then read
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `parity` to complete; gives up after limit_ns (4 s
// in the kernels; or at once when another role already gave up), raises
// *abort_flag and returns false.
template <bool CLUSTER = false>
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned long long limit_ns = WAIT_NS)
{
    auto try_ = [&] { return CLUSTER ? mbar_try_cluster(bar, parity) : mbar_try(bar, parity); };
    if (try_()) return true;
    const unsigned long long t0 = now_ns();
    for (uint32_t i = 1;; i++) {
        if (try_()) return true;
        if ((i & 255) == 0) {
            if (*abort_flag) return false;
            if (now_ns() - t0 > limit_ns) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}

// Waits until another CTA raised *flag (acquire, GPU scope); gives up like
// mbar_wait.
__device__ __forceinline__ bool flag_wait(const int* flag, volatile int* abort_flag,
                                          unsigned long long limit_ns = WAIT_NS)
{
    const unsigned long long t0 = now_ns();
    for (uint32_t i = 0;; i++) {
        int v;
        asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v) return true;
        if ((i & 63) == 63) {
            if (*abort_flag) return false;
            if (now_ns() - t0 > limit_ns) {
                *abort_flag = 1;
                return false;
            }
        }
    }
}


__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, uint64_t* bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"(tm), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* tm, uint64_t* bar, const int (&c)[5])
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6, %7}], [%2];"
        ::"r"(smem_u32(dst)), "l"(tm), "r"(smem_u32(bar)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4])
        : "memory");
}

__device__ __forceinline__ void tma_store_5d(const CUtensorMap* tm, const void* src, const int (&c)[5])
{
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5, %6}], [%1];"
                 ::"l"(tm), "r"(smem_u32(src)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4])
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d_pair(void* dst, const CUtensorMap* tm, uint32_t bar_cluster, int c0, int c1,
                                                 int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"(tm), "r"(bar_cluster), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* tm, uint64_t* bar, const int (&c)[5])
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
        ::"r"(smem_u32(dst)), "l"(tm), "r"(smem_u32(bar)), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3])
        : "memory");
}

__device__ __forceinline__ void tma_load_4d_pair(void* dst, const CUtensorMap* tm, uint32_t bar_cluster, const int (&c)[5])
{
    asm volatile(
        "cp.async.bulk.tensor.4d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
        ::"r"(smem_u32(dst)), "l"(tm), "r"(bar_cluster), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3])
        : "memory");
}

__device__ __forceinline__ void tma_load_3d_c(void* dst, const CUtensorMap* tm, uint64_t* bar, const int (&c)[5])
{
    tma_load_3d(dst, tm, bar, c[0], c[1], c[2]);
}

__device__ __forceinline__ void tma_load_5d_pair(void* dst, const CUtensorMap* tm, uint32_t bar_cluster, const int (&c)[5])
{
    asm volatile(
        "cp.async.bulk.tensor.5d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6, %7}], [%2];"
        ::"r"(smem_u32(dst)), "l"(tm), "r"(bar_cluster), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4])
        : "memory");
}

// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar_cluster)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}

__device__ __forceinline__ void mma_f16_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

// commit to the barrier at this offset in both CTAs of the pair
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar)
{
    const uint16_t mask = 3;
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
                 ::"r"(smem_u32(bar)), "h"(mask)
                 : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// K-major operand tile with 128-byte swizzle: rows of 64 16-bit elements,
// 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)1 << 16;             // leading byte offset 16 B (unused with 128B swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset between 8-row groups
    d |= (uint64_t)1 << 46;             // descriptor version (sm100)
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

// signed 8-bit operands, 32-bit integer accumulators (exact)
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

// MN-major operand tile with 128-byte swizzle: 64-element (128-byte) rows
// along M/N holding one k each, 8 k-rows per 1024-byte group (SBO), the
// second 64-row half of the tile 8 KiB further (LBO)
__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)(8192 >> 4) << 16;   // leading byte offset: between 64-row halves
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset: between 8-k groups
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// read-only global load kept as its own instruction, so a run of them stays
// in flight together before any result is used
__device__ __forceinline__ float ld_nc_f32(const float* p)
{
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}

template <int N>
__device__ __forceinline__ void epi_bar_n() { asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory"); }

// beta * op_C(C) for one output (0 when beta == 0)
__device__ __forceinline__ void load_beta_c(const EpiParams& e, const void* Cbase, int64_t offC, float& br, float& bi)
{
    br = 0.f;
    bi = 0.f;
    if (e.beta_zero) return;
    float cr, ci;
    load_rounded<float>(Cbase, offC, e.tC, e.round_C, cr, ci);
    if (e.conjC) ci = -ci;
    if (e.cplx) {
        br = e.beta_re * cr - e.beta_im * ci;
        bi = e.beta_re * ci + e.beta_im * cr;
    } else {
        br = e.beta_re * cr;
    }
}

__device__ __forceinline__ void finish_out(const EpiParams& e, void* Dbase, int64_t offD, float ar, float ai, float br,
                                           float bi)
{
    float accr, acci;
    if (e.cplx) {
        accr = e.alpha_re * ar - e.alpha_im * ai + br;
        acci = e.alpha_re * ai + e.alpha_im * ar + bi;
    } else {
        accr = e.alpha_re * ar + br;
        acci = 0.f;
    }
    if (e.conjD) acci = -acci;
    store_elem<float>(Dbase, offD, e.tD, accr, acci);
}

// ---------------------------------------------------------------------------
// In-place split-bfloat16 operands (k_gemm<.., CVT = true>): eight converter
// warps per CTA load the binary32 tiles of A and B with 16-byte loads,
// split every value into hi = bf16(x) and lo = bf16(x - hi), and store both
// in the swizzled layouts the MMAs read (K-major or MN-major, 128-byte
// swizzle). Per CTA and 64-deep contraction block a converter thread owns 4
// units of 8 consecutive elements of each operand:
//   K-major (contiguous along k): rows hi2 + 4 cw + 32 j (j < 4), the k run
//     8 lo3 .. 8 lo3 + 7; the 8 lanes of a row store one whole 128-byte row
//   MN-major (contiguous along rows): rows 64 h + 8 lo3 .. + 7 (h < 2) at
//     k = hi2 + 4 cw + 32 jk (jk < 2); 8 lanes store one 128-byte k-line
// (cw the converter warp, lo3 = lane % 8, hi2 = lane / 8), so every store
// of a warp covers whole 128-byte lines (no bank conflicts) and every 8
// lanes read 256 contiguous bytes.
__device__ __forceinline__ int64_t cvt_decode(const CvtDim& d, uint32_t idx)
{
    int64_t off = 0;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        if (j + 1 >= d.n) break;
        const uint32_t q = fdiv(idx, d.div[j]);
        off += (int64_t)(idx - q * d.div[j].d) * d.st[j];
        idx = q;
    }
    return d.n ? off + (int64_t)idx * d.st[d.n - 1] : 0;
}

// element offsets of this thread's unit rows for one tile (-1: past the
// end); returns the tile's operand base (its batch's, in a batched product)
__device__ __forceinline__ const float* cvt_rows(const CvtOperand& o, int64_t row0, int64_t l, int cw, int lo3,
                                                 int hi2, int64_t (&roff)[4])
{
    const float* base = o.base;
    if (o.bases) {
        base = (const float*)o.bases[l / o.lper];
        l %= o.lper;
    }
    const int64_t loff = cvt_decode(o.ls, (uint32_t)l);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int64_t r;
        if (o.mn) r = j < 2 ? row0 + 64 * j + 8 * lo3 : -1;
        else r = row0 + hi2 + 4 * cw + 32 * j;
        roff[j] = (r >= 0 && r < (int64_t)o.rows.size) ? loff + cvt_decode(o.rows, (uint32_t)r) : -1;
    }
    return base;
}

__device__ __forceinline__ float4 ld_nc_v4(const float* p)
{
    float4 v;
    asm volatile("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}

// the 4 units of contraction block kb into x (zeros past the tensor's end)
__device__ __forceinline__ void cvt_load(const CvtOperand& o, const float* base, const int64_t (&roff)[4], int kb,
                                         int cw, int lo3, int hi2, float (&x)[32])
{
#pragma unroll
    for (int u = 0; u < 4; u++) {
        int64_t ro;
        uint32_t k;
        if (o.mn) {
            ro = roff[u & 1];
            k = (uint32_t)kb * 64 + hi2 + 4 * cw + 32 * (u >> 1);
        } else {
            ro = roff[u];
            k = (uint32_t)kb * 64 + 8 * lo3;
        }
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
        if (ro >= 0 && k < o.ks.size) {
            const float* q = base + ro + cvt_decode(o.ks, k);
            a = ld_nc_v4(q);
            b = ld_nc_v4(q + 4);
        }
        x[8 * u + 0] = a.x; x[8 * u + 1] = a.y; x[8 * u + 2] = a.z; x[8 * u + 3] = a.w;
        x[8 * u + 4] = b.x; x[8 * u + 5] = b.y; x[8 * u + 6] = b.z; x[8 * u + 7] = b.w;
    }
}

// hi = bf16(x), lo = bf16(x - hi) of 8 values as two 16-byte vectors
__device__ __forceinline__ void split8(const float* x, uint4& hi, uint4& lo)
{
    uint32_t h[4], w[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        __nv_bfloat162 q = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
        h[i] = *(uint32_t*)&q;
        const float a = __uint_as_float(h[i] << 16), b = __uint_as_float(h[i] & 0xffff0000u);
        __nv_bfloat162 r = __floats2bfloat162_rn(x[2 * i] - a, x[2 * i + 1] - b);
        w[i] = *(uint32_t*)&r;
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, const uint4& v)
{
    asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

// stores the split units into the hi and lo tiles (128 x 64 each, 16 KiB)
__device__ __forceinline__ void cvt_store(const CvtOperand& o, const float (&x)[32], uint32_t hi_tile,
                                          uint32_t lo_tile, int cw, int lo3, int hi2)
{
#pragma unroll
    for (int u = 0; u < 4; u++) {
        uint32_t off;
        if (o.mn) {
            const int k = hi2 + 4 * cw + 32 * (u >> 1), h = u & 1;
            off = h * 8192 + (k >> 3) * 1024 + (k & 7) * 128 + ((lo3 ^ (k & 7)) << 4);
        } else {
            const int r = hi2 + 4 * cw + 32 * u;
            off = r * 128 + ((lo3 ^ (r & 7)) << 4);
        }
        uint4 hi, lo;
        split8(&x[8 * u], hi, lo);
        st_shared_v4(hi_tile + off, hi);
        st_shared_v4(lo_tile + off, lo);
    }
}

// the units rounded to the 16-bit operand format (fmt 1 f16, else bfloat16)
// into one tile: the precisions BF16BF16_ACCUM_F32 and F16F16_ACCUM_F32 on
// binary32 storage
__device__ __forceinline__ void cvt_store_round(const CvtOperand& o, const float (&x)[32], uint32_t tile, int fmt,
                                                int cw, int lo3, int hi2)
{
#pragma unroll
    for (int u = 0; u < 4; u++) {
        uint32_t off;
        if (o.mn) {
            const int k = hi2 + 4 * cw + 32 * (u >> 1), h = u & 1;
            off = h * 8192 + (k >> 3) * 1024 + (k & 7) * 128 + ((lo3 ^ (k & 7)) << 4);
        } else {
            const int r = hi2 + 4 * cw + 32 * u;
            off = r * 128 + ((lo3 ^ (r & 7)) << 4);
        }
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if (fmt == 1) {
                __half2 q = __floats2half2_rn(x[8 * u + 2 * i], x[8 * u + 2 * i + 1]);
                w[i] = *(uint32_t*)&q;
            } else {
                __nv_bfloat162 q = __floats2bfloat162_rn(x[8 * u + 2 * i], x[8 * u + 2 * i + 1]);
                w[i] = *(uint32_t*)&q;
            }
        }
        st_shared_v4(tile + off, make_uint4(w[0], w[1], w[2], w[3]));
    }
}

// ---------------------------------------------------------------------------
// Grouped products (group.cu): one persistent launch over the tiles of many
// products of different shapes. Product j's work items (tiles) are numbered
// from first on; every role finds an item's product by binary search.
struct GroupItem {
    CvtOperand a, b;
    EpiParams e;
    int32_t tiles_m, tiles_n, num_kb;
    int32_t mode;      // TB_TC_BF16, TB_TC_F16 (operands rounded) or TB_TC_SPLIT_BF16
    uint32_t idesc;    // MMA instruction descriptor (formats, majors, tile shape)
    int32_t f32_epi;   // C and D binary32, real, no op_D: D = fma(alpha, acc, beta * C)
    int32_t first;     // number of work items of products 0 .. j-1
    int32_t pad;
};

struct GroupParams {
    const GroupItem* items;
    int32_t n, total;  // products, work items
    int* error;        // set to 1 when a wait times out
};

// EPI_F32: real product, C and D binary32 (the common case, specialised);
// EPI_ANY: every storage type, complex outputs, op_C / op_D.
// EPI_TMA: like EPI_F32, with C and D moved by TMA tensor copies through a
// per-warp shared-memory box (C and D expressible as tensor maps).
// EPI_I32: signed 8-bit operands (kind::i8, rows of 128 elements per stage),
// 32-bit integer accumulators added into a binary64 workspace.
enum { EPI_ANY = 0, EPI_F32 = 1, EPI_TMA = 2, EPI_I32 = 3 };

}  // namespace tc
}  // namespace tb
