// Grouped tensor-core products: one persistent launch runs the tiles of many
// products of different shapes (M, N, K, strides, precision mode, epilogue)
// together, so that a served mix of small and mid-size contractions fills
// the GPU with one launch instead of one launch sequence per product. The
// batched product of the reference's API (api/include/tapp/product.h:66-75,
// declared but not implemented there) covers many products of ONE plan; a
// group covers products of different plans.
//
// Every product is a binary32-storage product of the tensor-core path whose
// operands the converter warps read in place (tc_device.cuh: cvt_*): no pack
// launches and no operand panels. Per product, the converters either round
// the operands to the precision's 16-bit format (BF16BF16_ACCUM_F32,
// F16F16_ACCUM_F32: one MMA per 16-deep step) or split them into bfloat16
// hi and lo parts (float32 in split mode: hi*hi + hi*lo + lo*hi); each tile
// has the fused epilogue of its own product. Operands whose layout allows it
// come in 16-byte runs; any other layout element by element through offset
// tables in shared memory.
//
// Two tile shapes, chosen per launch: 256 x 256 tiles on CTA pairs
// (cta_group::2, as the single-product kernel) or 128 x 128 tiles on single
// CTAs (more tiles for small products). Threads: warp 1 issues the MMAs,
// warp 2 owns TMEM (two accumulators), warps 4-7 run the epilogue, warps
// 8-15 convert. Every wait is bounded (4 s); on expiry the kernel raises the
// error word, stops and frees TMEM.
#include <cuda.h>
#include <cstring>

#include "../tb_cuda.h"
#include "tb_common.cuh"
#include "tc_device.cuh"

namespace tb {
int* device_error_word();
// descriptor of one product for the grouped kernel (tc.cu); false when the
// product does not qualify
bool group_item(const tb_plan* P, const tb_ptrs* d, bool cta2, tc::GroupItem* g);
int tc_sm_count();

namespace tc {

constexpr int GROUP_THREADS = 512;
constexpr int GROUP_NS = 3;                      // stages of 64 KiB: A hi, A lo, B hi, B lo
constexpr int GROUP_SB = 4 * BM * BK * 2;
// tiles | alignment | barriers | epilogue column tables | converter offset tables
constexpr int GROUP_SMEM = GROUP_NS * GROUP_SB + 1024 + 256 + 2 * 256 * 8 + (2 * 128 + 2 * 64) * 8;

// barrier among the converter warps (8-15)
__device__ __forceinline__ void conv_bar() { asm volatile("bar.sync 2, 256;" ::: "memory"); }

// The 4 units of this thread (tc_device.cuh: cvt_load) element by element:
// offsets from this tile's row table and this block's k table (-1: past the
// end, read as zero).
__device__ __forceinline__ void tab_load(const CvtOperand& o, const int64_t* rows, const int64_t* ks, int cw, int lo3,
                                         int hi2, float (&x)[32])
{
#pragma unroll
    for (int u = 0; u < 4; u++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            int64_t ro, ko;
            if (o.mn) {
                ro = rows[(u & 1) * 64 + 8 * lo3 + i];
                ko = ks[hi2 + 4 * cw + 32 * (u >> 1)];
            } else {
                ro = rows[hi2 + 4 * cw + 32 * u];
                ko = ks[8 * lo3 + i];
            }
            x[8 * u + i] = (ro >= 0 && ko >= 0) ? __ldg(o.base + ro + ko) : 0.f;
        }
    }
}

__device__ __forceinline__ int group_find(const GroupItem* items, int n, int it)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&items[mid].first) <= it) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <bool CTA2>
__global__ void __launch_bounds__(GROUP_THREADS, 1) k_group(const GroupParams gp)
{
    constexpr int TN = CTA2 ? 256 : 128;      // tile columns
    constexpr int TM = CTA2 ? 256 : 128;      // tile rows (each CTA holds 128)
    constexpr int TCOLS = CTA2 ? 512 : 256;   // TMEM columns: two accumulators
    constexpr int NS = GROUP_NS, SB = GROUP_SB;
    constexpr int EW = 4, ET = EW * 32;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    uint8_t* tiles = smem;
    uint8_t* bars = smem + NS * SB;
    uint64_t* full = (uint64_t*)bars;
    uint64_t* empty = (uint64_t*)(bars + 32);
    uint64_t* tfull = (uint64_t*)(bars + 64);
    uint64_t* tempty = (uint64_t*)(bars + 80);
    uint32_t* tmem_slot = (uint32_t*)(bars + 96);
    volatile int* abort_flag = (volatile int*)(bars + 100);
    volatile int* epi_ok = (volatile int*)(bars + 104);
    int64_t* colC = (int64_t*)(bars + 256);
    int64_t* colD = colC + 256;
    int64_t* rowTab = colD + 256;   // [A rows 128][B rows 128] of the converters' tile
    int64_t* kTab = rowTab + 256;   // [A 64][B 64] offsets of the current contraction block

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = CTA2 ? cluster_rank() : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&full[s], CTA2 ? 16 : 8);  // one arrival per converter warp (both CTAs of a pair)
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], CTA2 ? 2 * EW : ET);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        if (CTA2) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                         "r"(TCOLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                         "r"(TCOLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
    }
    fence_before();
    if (CTA2) cluster_sync();
    else __syncthreads();
    fence_after();
    const uint32_t tmem_base = *tmem_slot;

    const int unit = CTA2 ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
    const int units = CTA2 ? (int)(gridDim.x >> 1) : (int)gridDim.x;
    const int my_items = gp.total > unit ? (gp.total - 1 - unit) / units + 1 : 0;

    // the work item's product and tile coordinates
    auto locate = [&](int i, int& j, int& tm, int& tn, int& l) {
        const int it = unit + i * units;
        j = group_find(gp.items, gp.n, it);
        const GroupItem& P = gp.items[j];
        const int tile = it - P.first;
        tm = tile % P.tiles_m;
        const int rest = tile / P.tiles_m;
        tn = rest % P.tiles_n;
        l = rest / P.tiles_n;
    };

    if (warp == 1) {
        // ---------------- MMA issuer (the leader of a pair) ----------------
        if (lane == 0 && (!CTA2 || rank == 0)) {
            uint32_t g = 0;
            bool ok = true;
            for (int i = 0; i < my_items && ok; i++) {
                int j, tm, tn, l;
                locate(i, j, tm, tn, l);
                const GroupItem& P = gp.items[j];
                const int nkb = P.num_kb, split = P.mode == TB_TC_SPLIT_BF16;
                const uint32_t idesc = P.idesc;
                const int amn = P.a.mn, bmn = P.b.mn;
                const int acc = i & 1;
                const uint32_t aph = (i >> 1) & 1;
                if (!mbar_wait(&tempty[acc], aph ^ 1, abort_flag)) break;
                fence_after();
                const uint32_t d_tmem = tmem_base + acc * TN;
                for (int kb = 0; kb < nkb; kb++, g++) {
                    const int s = g % NS;
                    const uint32_t ph = (g / NS) & 1;
                    if (!mbar_wait<CTA2>(&full[s], ph, abort_flag)) { ok = false; break; }
                    fence_after();
                    const uint32_t a = smem_u32(tiles + s * SB);
#pragma unroll
                    for (int k = 0; k < BK / 16; k++) {
                        auto desc = [&](uint32_t t, int mn) {
                            return mn ? smem_desc_mn(t + k * 2048) : smem_desc(t + k * 32);
                        };
                        const uint64_t ah = desc(a, amn), bh = desc(a + 32768, bmn);
                        const uint32_t accumulate = (kb | k) != 0;
                        if (CTA2) mma_f16_pair(d_tmem, ah, bh, idesc, accumulate);
                        else mma_f16(d_tmem, ah, bh, idesc, accumulate);
                        if (split) {
                            const uint64_t al = desc(a + 16384, amn), bl = desc(a + 49152, bmn);
                            if (CTA2) {
                                mma_f16_pair(d_tmem, ah, bl, idesc, 1);
                                mma_f16_pair(d_tmem, al, bh, idesc, 1);
                            } else {
                                mma_f16(d_tmem, ah, bl, idesc, 1);
                                mma_f16(d_tmem, al, bh, idesc, 1);
                            }
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
            volatile int never = 0;
            if (g > 0) {
                const uint32_t last = g - 1;
                mbar_wait(&empty[last % NS], (last / NS) & 1, &never);
            }
        }
    } else if (warp >= 4 && warp < 8) {
        // ---------------- epilogue ----------------
        const int q = warp & 3;
        const int et = threadIdx.x - 128;
        auto release_acc = [&](int acc) {
            if (CTA2) {
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(cluster_addr(&tempty[acc], 0));
            } else {
                mbar_arrive(&tempty[acc]);
            }
        };
        for (int i = 0; i < my_items; i++) {
            int j, tm, tn, l;
            locate(i, j, tm, tn, l);
            const EpiParams& e = gp.items[j].e;
            const bool f32e = gp.items[j].f32_epi != 0;
            for (int c = et; c < TN; c += ET) {
                const int64_t n = (int64_t)tn * TN + c;
                int64_t oc = 0, od = 0;
                if (n < e.N) decode2(e.nn, n, oc, od);
                colC[c] = oc;
                colD[c] = od;
            }
            int64_t lC, lD;
            decode2(e.ll, l, lC, lD);
            const int64_t m = (int64_t)tm * TM + (int64_t)rank * BM + q * 32 + lane;
            const bool mok = m < e.M;
            int64_t rC = 0, rD = 0;
            if (mok) decode2(e.mm, m, rC, rD);
            rC += lC;
            rD += lD;
            const int acc = i & 1;
            const uint32_t aph = (i >> 1) & 1;
            if (et == 0) *epi_ok = mbar_wait(&tfull[acc], aph, abort_flag) ? 1 : 0;
            epi_bar_n<ET>();  // column tables and the wait's outcome visible
            const bool ok = *epi_ok != 0;
            fence_after();
            if (ok) {
#pragma unroll 1
                for (int ch = 0; ch < TN / 32; ch++) {
                    // f32e: raw C (the formula of the single-product kernel's
                    // binary32 epilogue); else beta * op_C(C)
                    float br[32];
#pragma unroll
                    for (int jj = 0; jj < 32; jj++) {
                        const int c = ch * 32 + jj;
                        const bool in = mok && (int64_t)tn * TN + c < e.N;
                        br[jj] = 0.f;
                        if (f32e) {
                            if (in && !e.beta_zero) br[jj] = ld_nc_f32((const float*)e.C + rC + colC[c]);
                        } else if (in) {
                            float bi;
                            load_beta_c(e, e.C, rC + colC[c], br[jj], bi);
                        }
                    }
                    uint32_t r[32];
                    tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + acc * TN + ch * 32, r);
#pragma unroll
                    for (int jj = 0; jj < 32; jj++) {
                        const int c = ch * 32 + jj;
                        if (!mok || (int64_t)tn * TN + c >= e.N) continue;
                        if (f32e)
                            ((float*)e.D)[rD + colD[c]] =
                                fmaf(e.alpha_re, __uint_as_float(r[jj]), e.beta_re * round_in<float>(br[jj], e.round_C));
                        else
                            finish_out(e, e.D, rD + colD[c], __uint_as_float(r[jj]), 0.f, br[jj], 0.f);
                    }
                }
            }
            fence_before();
            release_acc(acc);
            epi_bar_n<ET>();  // tables and *epi_ok may be rewritten after this point
        }
    } else if (warp >= 8) {
        // ---------------- converters ----------------
        const int cw = warp - 8, lo3 = lane & 7, hi2 = lane >> 3;
        uint32_t g = 0;
        bool ok = true;
        for (int i = 0; i < my_items && ok; i++) {
            int j, tm, tn, l;
            locate(i, j, tm, tn, l);
            const GroupItem& P = gp.items[j];
            const int mode = P.mode, nkb = P.num_kb;
            const int fmt = mode == TB_TC_F16 ? 1 : 0;
            // stores one operand's units of a block into stage s (side 0 A, 1 B)
            auto store1 = [&](int s, int side, const float (&x)[32]) {
                const uint32_t st = smem_u32(tiles + s * SB) + side * 32768;
                const CvtOperand& o = side ? P.b : P.a;
                if (mode == TB_TC_SPLIT_BF16) cvt_store(o, x, st, st + 16384, cw, lo3, hi2);
                else cvt_store_round(o, x, st, fmt, cw, lo3, hi2);
            };
            // the stage is complete: hand it to the MMA issuer
            auto signal = [&](int s) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    if (CTA2) mbar_arrive_cluster(cluster_addr(&full[s], 0));
                    else mbar_arrive(&full[s]);
                }
            };
            if (P.a.vec && P.b.vec) {
                // 16-byte runs; the next block's loads in flight under this block's stores
                int64_t ra[4], rb[4];
                const float* abase = cvt_rows(P.a, (int64_t)tm * TM + (int64_t)rank * BM, l, cw, lo3, hi2, ra);
                const float* bbase = cvt_rows(P.b, (int64_t)tn * TN + (int64_t)rank * BM, l, cw, lo3, hi2, rb);
                float xa[32], xb[32];
                cvt_load(P.a, abase, ra, 0, cw, lo3, hi2, xa);
                cvt_load(P.b, bbase, rb, 0, cw, lo3, hi2, xb);
                for (int kb = 0; kb < nkb; kb++, g++) {
                    const int s = g % NS;
                    if (!mbar_wait(&empty[s], ((g / NS) & 1) ^ 1, abort_flag)) { ok = false; break; }
                    store1(s, 0, xa);
                    if (kb + 1 < nkb) cvt_load(P.a, abase, ra, kb + 1, cw, lo3, hi2, xa);
                    store1(s, 1, xb);
                    if (kb + 1 < nkb) cvt_load(P.b, bbase, rb, kb + 1, cw, lo3, hi2, xb);
                    signal(s);
                }
            } else {
                // element loads through offset tables: this tile's rows once,
                // each block's contraction offsets as it comes
                const int ct = threadIdx.x - 256;
                {
                    const int side = ct >> 7, r = ct & 127;
                    const CvtOperand& o = side ? P.b : P.a;
                    const int64_t row = (side ? (int64_t)tn * TN : (int64_t)tm * TM) + (int64_t)rank * BM + r;
                    rowTab[ct] = row < (int64_t)o.rows.size
                                     ? cvt_decode(o.ls, (uint32_t)l) + cvt_decode(o.rows, (uint32_t)row)
                                     : -1;
                }
                for (int kb = 0; kb < nkb; kb++, g++) {
                    if (ct < 128) {
                        const int side = ct >> 6;
                        const CvtOperand& o = side ? P.b : P.a;
                        const uint32_t k = (uint32_t)kb * 64 + (ct & 63);
                        kTab[ct] = k < o.ks.size ? cvt_decode(o.ks, k) : -1;
                    }
                    conv_bar();  // tables written
                    float xa[32], xb[32];
                    tab_load(P.a, rowTab, kTab, cw, lo3, hi2, xa);
                    tab_load(P.b, rowTab + 128, kTab + 64, cw, lo3, hi2, xb);
                    conv_bar();  // tables read: the next block (or tile) may rewrite them
                    const int s = g % NS;
                    if (!mbar_wait(&empty[s], ((g / NS) & 1) ^ 1, abort_flag)) { ok = false; break; }
                    store1(s, 0, xa);
                    store1(s, 1, xb);
                    signal(s);
                }
            }
        }
    }
    fence_before();
    if (CTA2) cluster_sync();
    else __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(gp.error, 1);
    if (warp == 2) {
        fence_after();
        if (CTA2) asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TCOLS));
        else asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TCOLS));
    }
}

}  // namespace tc

size_t group_tc_bytes(int n) { return (size_t)n * sizeof(tc::GroupItem) + 64; }

// Fills `host` (group_tc_bytes(n)) with the descriptors of n grouped
// products, copies them to `dev` and launches one grouped kernel with tile
// shape `tile` (1: 256 x 256 on CTA pairs, 2: 128 x 128). Returns
// cudaErrorInvalidValue, launching nothing, when a product does not qualify.
cudaError_t launch_group_tc(const tb_plan* const* P, const tb_ptrs* d, int n, void* host, void* dev, int tile,
                            cudaStream_t s, int64_t* tiles_out)
{
    using namespace tc;
    if (n <= 0) return cudaSuccess;
    const bool cta2 = tile != 2;
    GroupItem* h = (GroupItem*)host;
    int64_t total = 0;
    for (int j = 0; j < n; j++) {
        if (!group_item(P[j], &d[j], cta2, &h[j])) return cudaErrorInvalidValue;
        h[j].first = (int32_t)total;
        total += (int64_t)h[j].tiles_m * h[j].tiles_n * P[j]->L.size;
        if (total >= (1ll << 30)) return cudaErrorInvalidValue;
    }
    if (tiles_out) *tiles_out = total;
    if (total == 0) return cudaSuccess;
    int* flag = device_error_word();
    if (!flag) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMemcpyAsync(dev, host, sizeof(GroupItem) * (size_t)n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    GroupParams gp;
    gp.items = (const GroupItem*)dev;
    gp.n = n;
    gp.total = (int32_t)total;
    gp.error = flag;
    void (*kern)(const GroupParams) = cta2 ? k_group<true> : k_group<false>;
    static int attr_done[64][2];
    int devno = 0;
    cudaGetDevice(&devno);
    if (devno < 0 || devno >= 64 || !attr_done[devno][cta2]) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, GROUP_SMEM);
        if (e != cudaSuccess) return e;
        if (devno >= 0 && devno < 64) attr_done[devno][cta2] = 1;
    }
    const int units = cta2 ? tc_sm_count() / 2 : tc_sm_count();
    const int grid = (int)(total < units ? total : units) * (cta2 ? 2 : 1);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(GROUP_THREADS, 1, 1);
    cfg.dynamicSmemBytes = GROUP_SMEM;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cta2 ? 2 : 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, kern, gp);
    count_launch();
    return e;
}

}  // namespace tb
