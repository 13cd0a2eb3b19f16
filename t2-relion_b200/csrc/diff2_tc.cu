// Coarse diff2 on the 5th-generation tensor cores (tcgen05, sm_100a) with a
// three-product split-BF16 contraction and FP32 accumulation in TMEM.
//
// The cross term of diff2 (src/ml_optimiser.cpp:7251-7272; the reference's
// coarse_splitImg_BCF_PMO.cuh:139-693 runs it as 3xTF32 mma.sync) is a real
// GEMM over K = 2P interleaved (re, im) values:
//     C[oc][b*T+t] = sum_k Proj[oc][k] * Img[b*T+t][k]
// Every FP32 operand x is split as hi = bf16(x), lo = bf16(x - hi), and
//     C ~= Ph.Ih + Ph.Il + Pl.Ih      (the lo.lo term is below FP32 resolution)
// The three products accumulate into one FP32 TMEM accumulator.
//
// Kernel: persistent, one CTA per SM, 192 threads.
//   warp 0      TMA producer: per 64-wide K block loads Ph, Pl (128 x 64) and
//               Ih, Il (256 x 64) with 128-byte swizzle into a 2-stage ring
//   warp 1      MMA issuer: 12 x tcgen05.mma (M128 N256 K16) per K block (4 per
//               product; the network GEMMs use one product, BF16 x BF16) into a
//               double-buffered 2 x 256-column TMEM accumulator
//   warps 2-5   epilogue: tcgen05.ld 32x32b, transpose through shared memory,
//               diff2 = c0 + norm - C written coalesced along t, per-particle
//               minimum by shared + global atomics
// Every mbarrier wait is bounded (2 s); on expiry the CTA records
// T2B_ERR_TIMEOUT in a device flag, waits (bounded) for its own copies and
// MMAs, frees TMEM and returns.
#include "t2b_internal.cuh"
#include "project_pixel.cuh"
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cstring>

namespace t2b {
namespace {

constexpr int TM = 128, TN = 256, TK = 64;
constexpr int STAGES = 2;       // pipeline stages of 128 x 256 tiles (96 KB each)
constexpr int MAXSTAGES = 8;
#ifndef T2B_L2_AHEAD
#define T2B_L2_AHEAD 4
#endif
constexpr int L2_AHEAD = T2B_L2_AHEAD;  // k-blocks between an A tile's L2 prefetch and its load    // narrower tiles and fewer products: more, smaller stages in the same space
constexpr uint32_t A_BYTES = TM * TK * 2;              // 16 KB
constexpr uint32_t B_BYTES = TN * TK * 2;              // 32 KB
constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // 96 KB
constexpr int NTHREADS = 192;
constexpr uint32_t TMEM_COLS = 512;
constexpr int EPI_LD = 33;
constexpr size_t SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 4 * 32 * EPI_LD * 4 + 4 * (TN + 2) * 4;
constexpr unsigned long long WAIT_NS = 2000000000ull;

// instruction descriptor: D f32, A/B bf16, both K-major, M = 128; N (bits 17-22, N/8)
// is set per launch (256, or 96 for one particle's translations)
constexpr uint32_t IDESC_BASE = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TM >> 4) << 24);
__host__ __device__ constexpr uint32_t idesc_for(int n) { return IDESC_BASE | ((uint32_t)(n >> 3) << 17); }

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of parity `parity`; false on timeout / abort.
__device__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag)
{
    const unsigned long long t0 = gtimer();
    for (uint32_t i = 1;; i++) {
        if (mbar_try(b, parity)) return true;
        if ((i & 255u) == 0) {
            if (*abort_flag) return false;
            if (gtimer() - t0 > WAIT_NS) return false;
        }
    }
}

__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            su32(dst)),
        "l"(map), "r"(su32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Bring one box of a tensor map into L2 ahead of its load (no shared memory, no barrier).
__device__ __forceinline__ void tma_prefetch_l2(const CUtensorMap* map, int x, int y)
{
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(map), "r"(x), "r"(y)
                 : "memory");
}

// One contiguous block global -> shared (untiled bulk copy): the operand is stored
// pre-swizzled, so the block lands in the layout the UMMA descriptor reads
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     su32(dst)),
                 "l"(src), "r"(bytes), "r"(su32(bar))
                 : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1 << 16;             // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;   // stride byte offset
    d |= (uint64_t)1 << 46;             // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;             // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void umma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            dtmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r)
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ unsigned f2key(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Tile order: groups of `group` orientation tiles, the batch columns inside a
// group, so the 148 tiles that run together share few operand strips (the group
// size is chosen by t2b_autotune; 16 by default).
__device__ __forceinline__ void tile_coords(int tile, int m_tiles, int n_tiles, int group, int& mt, int& nt)
{
    const int per_group = group * n_tiles;
    const int g = tile / per_group;
    const int first = g * group;
    const int gm = min(group, m_tiles - first);
    const int r = tile - g * per_group;
    mt = first + r % gm;
    nt = r / gm;
}

struct TcParams {
    int m_tiles, n_tiles, kblocks;
    int group;                // dense tiles: orientation tiles per raster group (0: 16)
    int ksplit;               // raw GEMMs: K split into this many slices (0/1: none); slice s writes
                              // its partial product at out + s * ncols * KO
    int raw;                  // 1: store the contraction itself (norm and network GEMMs), 0: diff2 epilogue
    int KO, T, ncols;
    const float* c0;
    const float* norms;
    const unsigned char* skip;
    float* d2c;
    unsigned* minkey;
    int* err;
    int products;             // 1: hi.hi, 2: + hi(A).lo(B), 3: + lo(A).hi(B) (split-BF16)
    // proposal tiles (mode 1): tile i holds particles [i*ppt, i*ppt + ppt) (ppt * kslot
    // = 128); A rows [i*128, i*128+128) are their proposals premultiplied by the
    // conjugate particle image (kslot rows each, the first KO of them used), B the T
    // phase rows of the translations, the same for every tile; norms and d2c are per
    // (particle, proposal); ncols = particles of the batch.
    // mode 2 tiles hold one particle (ppt = 1): B rows from tile*T (its own images).
    int mode, ppt, kslot;
    // mode 1: A and B are stored pre-swizzled and K-blocked (swz_offset): the tile of rows
    // [y, y + n) of k-block kb is one contiguous block, fetched by one bulk copy
    const void* a_hi;
    const void* a_lo;
    const void* b_hi;
    const void* b_lo;
    int a_rows, b_rows;       // rows of each k-block layer
    const int* prop;          // mode 1: global orientation of every (particle, proposal)
    const int* gate;          // run only when (*gate != 0) == gate_run (null: always)
    int gate_run;
    const int* cnt;           // run only when cnt_lo <= *cnt <= cnt_hi (null: always)
    int cnt_lo, cnt_hi;
    int tn;                   // N of the tile (multiple of 32, <= 256; 0 = 256); B maps with a tn-row box
    int mtp;                  // mode 2: consecutive tiles per particle (0 = 1); A rows of tile i are
                              // rows [i*128, i*128+128), candidate j = (i % mtp)*128 + row
    // mode 2 (low-resolution rescoring, tiles as mode 1 with ppt = 1): no diff2 is stored;
    // each epilogue thread reduces its own row (candidate j) over the translations,
    // d2c[b*KO + j] = log sum_t pdf_t exp(C_t) - norm_j + log pdf_o(j)  (c0 omitted)
    const double* pdf_t;      // n x T
    const double* pdf_oc;     // K*O
    // mode 1 with ksplit = 2: the two K slices of an m-tile run on two CTAs; each epilogue
    // warp stores its slice's accumulator rows in part (per m-tile, slice, warp: nchunk x
    // 32 x 32 floats, column-major in the lane), and the warp that arrives second on
    // fix[m-tile * 4 + warp] (zero before the launch) adds the other slice's and emits
    float* part;
    int* fix;
    // dense and raw-row tiles over one chunk of the orientations (mode 0): the tile's row oc
    // (< KO, the chunk's rows) is global orientation row0 + oc of a batch layout whose rows
    // are ko_stride long (0: KO); skip, norms and the output are indexed globally
    int row0, ko_stride;
};

// maps: device array of tensor-map descriptors (encoded once per configuration);
// the A (orientation) operand uses maps[ia], maps[ia+1] (hi, lo), the B operand
// maps[ib], maps[ib+1].
__global__ void __launch_bounds__(NTHREADS, 1)
k_diff2_tc(const CUtensorMap* __restrict__ maps, int ia, int ib, TcParams p)
{
    if (p.gate && ((*p.gate != 0) != (p.gate_run != 0))) return;  // uniform: the whole CTA leaves
    if (p.cnt && (*p.cnt < p.cnt_lo || *p.cnt > p.cnt_hi)) return;
    const CUtensorMap* mPh = maps + ia;
    const CUtensorMap* mPl = maps + ia + 1;
    const CUtensorMap* mIh = maps + ib;
    const CUtensorMap* mIl = maps + ib + 1;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[MAXSTAGES], empty_bar[MAXSTAGES], tfull_bar[2], tempty_bar[2], drain_bar;
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // stage geometry of this launch: B box of tn rows; narrow tiles get a third stage
    const int tn_l = p.tn ? p.tn : TN;
    const uint32_t bbytes = (uint32_t)tn_l * TK * 2;                 // multiple of 1024
    // stage layout [A hi | A lo (3 products) | B hi | B lo (2+ products)]; as many stages as
    // fit in the stage area, so narrow or single-product tiles keep more copies in flight
    const uint32_t a_st = A_BYTES * (p.products == 3 ? 2u : 1u);
    const uint32_t sbytes = a_st + bbytes * (p.products >= 2 ? 2u : 1u);
    const int nst = min(MAXSTAGES, (int)((uint32_t)(STAGES * STAGE_BYTES) / sbytes));
    const uint32_t base = (su32(smem_raw) + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - su32(smem_raw));
    float* epi = reinterpret_cast<float*>(gbase + STAGES * STAGE_BYTES);          // 4 x 32 x 33
    unsigned* smin = reinterpret_cast<unsigned*>(epi + 4 * 32 * EPI_LD);          // 4 x (TN+2)

    if (threadIdx.x == 0) {
        for (int s = 0; s < MAXSTAGES; s++) { mbar_init(&full_bar[s], 1); mbar_init(&empty_bar[s], 1); }
        for (int s = 0; s < 2; s++) { mbar_init(&tfull_bar[s], 1); mbar_init(&tempty_bar[s], 4); }
        mbar_init(&drain_bar, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_slot;
    const int ksp = p.ksplit > 1 ? p.ksplit : 1;
    const int ntiles = p.m_tiles * p.n_tiles * ksp;
    const int kper = (p.kblocks + ksp - 1) / ksp;   // k-blocks per slice

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer
        // only the descriptors this launch reads (the lo slots may not exist)
        const CUtensorMap* ms[4] = {mPh, mIh, mIl, mPl};
        // (proposal tiles read no tensor map: their operands come by bulk copies)
        const int nmaps = p.mode == 1 ? 0 : 2 + (p.products >= 2 ? 1 : 0) + (p.products == 3 ? 1 : 0);
        for (int j = 0; j < nmaps; j++) {
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(ms[j]) : "memory");
            asm volatile("prefetch.tensormap [%0];" ::"l"(ms[j]) : "memory");
        }
        int it = 0;
        int issued[MAXSTAGES] = {};
        uint32_t last_par[MAXSTAGES] = {};
        const uint32_t tx_bytes = A_BYTES * (p.products == 3 ? 2u : 1u) + bbytes * (p.products >= 2 ? 2u : 1u);
        // A tiles read by one column tile only (the audit contractions) come from DRAM once, and
        // wide stages leave room for two in shared memory: fetch them into L2 L2_AHEAD k-blocks
        // before their loads, so the loads find them there (with more stages the loads in
        // flight already cover the latency, and the prefetches only add requests)
        const bool pf = L2_AHEAD > 0 && p.mode == 0 && p.n_tiles == 1 && nst <= 2;
        auto prefetch_a = [&](int kb, int ya) {
            tma_prefetch_l2(mPh, kb * TK, ya);
            if (p.products == 3) tma_prefetch_l2(mPl, kb * TK, ya);
        };
        for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x) {
            int ya, yb;
            const int kb0 = (tile % ksp) * kper, kb1 = min(p.kblocks, kb0 + kper);
            if (p.mode == 0) {
                int mt, nt;
                tile_coords(tile / ksp, p.m_tiles, p.n_tiles, p.group ? p.group : 16, mt, nt);
                ya = mt * TM;
                yb = nt * tn_l;
            } else if (p.mode == 1) {
                ya = (tile / ksp) * TM;
                yb = 0;
            } else {
                ya = tile * TM;
                yb = (tile / (p.mtp ? p.mtp : 1)) * p.T;
            }
            if (pf)
                for (int kb = kb0 + 1; kb < min(kb1, kb0 + L2_AHEAD); kb++) prefetch_a(kb, ya);
            for (int kb = kb0; kb < kb1; kb++, it++) {
                const int s = it % nst;
                const uint32_t ph = (uint32_t)(it / nst) & 1u;
                if (pf && kb + L2_AHEAD < kb1) prefetch_a(kb + L2_AHEAD, ya);
                if (!mbar_wait(&empty_bar[s], ph ^ 1u, &abort_flag)) { abort_flag = 1; break; }
                uint8_t* st = gbase + s * sbytes;
                mbar_expect_tx(&full_bar[s], tx_bytes);
                if (p.mode == 1) {
                    const size_t ao = ((size_t)kb * p.a_rows + ya) * (TK * 2), bo = ((size_t)kb * p.b_rows + yb) * (TK * 2);
                    bulk_load(st, static_cast<const uint8_t*>(p.a_hi) + ao, A_BYTES, &full_bar[s]);
                    bulk_load(st + A_BYTES, static_cast<const uint8_t*>(p.a_lo) + ao, A_BYTES, &full_bar[s]);
                    bulk_load(st + a_st, static_cast<const uint8_t*>(p.b_hi) + bo, bbytes, &full_bar[s]);
                    bulk_load(st + a_st + bbytes, static_cast<const uint8_t*>(p.b_lo) + bo, bbytes, &full_bar[s]);
                } else {
                    tma_load(st, mPh, &full_bar[s], kb * TK, ya);
                    if (p.products == 3) tma_load(st + A_BYTES, mPl, &full_bar[s], kb * TK, ya);
                    tma_load(st + a_st, mIh, &full_bar[s], kb * TK, yb);
                    if (p.products >= 2) tma_load(st + a_st + bbytes, mIl, &full_bar[s], kb * TK, yb);
                }
                issued[s] = 1;
                last_par[s] = ph;
            }
        }
        if (abort_flag) {
            // let the copies already in flight land before the CTA exits
            volatile int never = 0;
            for (int s = 0; s < nst; s++)
                if (issued[s]) mbar_wait(&full_bar[s], last_par[s], &never);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        const uint32_t idesc = idesc_for(p.tn ? p.tn : TN);
        int it = 0, tl = 0;
        for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x, tl++) {
            const int abuf = tl & 1;
            const uint32_t aph = (uint32_t)(tl >> 1) & 1u;
            if (!mbar_wait(&tempty_bar[abuf], aph ^ 1u, &abort_flag)) { abort_flag = 1; break; }
            tc_fence_after();
            const uint32_t dt = tmem + (uint32_t)(abuf * TN);
            bool ok = true;
            const int kb0 = (tile % ksp) * kper, kb1 = min(p.kblocks, kb0 + kper);
            for (int kb = kb0; kb < kb1; kb++, it++) {
                const int s = it % nst;
                const uint32_t ph = (uint32_t)(it / nst) & 1u;
                if (!mbar_wait(&full_bar[s], ph, &abort_flag)) { ok = false; break; }
                tc_fence_after();
                const uint32_t sa = base + s * sbytes;
                const uint64_t dPh = sdesc(sa), dPl = sdesc(sa + A_BYTES);
                const uint64_t dIh = sdesc(sa + a_st), dIl = sdesc(sa + a_st + bbytes);
#pragma unroll
                for (int k = 0; k < TK / 16; k++) {
                    const uint64_t ko = (uint64_t)(k * 32) >> 4;  // 32 bytes per K=16 step
                    umma(dt, dPh + ko, dIh + ko, idesc, (kb != kb0 || k != 0));
                    if (p.products >= 2) umma(dt, dPh + ko, dIl + ko, idesc, 1);
                    if (p.products == 3) umma(dt, dPl + ko, dIh + ko, idesc, 1);
                }
                umma_commit(&empty_bar[s]);  // stage free once these MMAs retire
            }
            if (!ok) { abort_flag = 1; break; }
            umma_commit(&tfull_bar[abuf]);   // accumulator ready
        }
        // drain: every MMA issued by this thread has retired before TMEM is freed
        umma_commit(&drain_bar);
        volatile int never = 0;
        mbar_wait(&drain_bar, 0, &never);
    } else if (warp >= 2) {
        // ---------------- epilogue (warps 2..5 -> TMEM lane quarters 2,3,0,1)
        const int q = warp & 3;
        const int ew = warp - 2;
        float* sbuf = epi + ew * 32 * EPI_LD;
        unsigned* wmin = smin + ew * (TN + 2);
        int tl = 0;
        for (int tile = blockIdx.x; tile < ntiles && !abort_flag; tile += gridDim.x, tl++) {
            int mt = 0, nt = 0;
            if (p.mode == 0) tile_coords(tile / ksp, p.m_tiles, p.n_tiles, p.group ? p.group : 16, mt, nt);
            float* const outp = p.d2c + (size_t)(tile % ksp) * p.ncols * p.KO * p.T;   // raw: the slice's partial
            const int abuf = tl & 1;
            const uint32_t aph = (uint32_t)(tl >> 1) & 1u;
            if (!mbar_wait(&tfull_bar[abuf], aph, &abort_flag)) { abort_flag = 1; break; }
            tc_fence_after();
            const int n0 = nt * tn_l;
            const int mtp = p.mtp ? p.mtp : 1;
            const int tt = tile / ksp;   // the m-tile (modes 1, 2)
            const int bfirst = p.mode == 0 ? n0 / p.T : (tt / mtp) * p.ppt;
            const int jbase = p.mode == 0 ? 0 : (tt % mtp) * TM;
            for (int i = lane; i < TN + 2; i += 32) wmin[i] = 0xffffffffu;
            // proposal tiles: the per-row data of the warp's 32 rows (orientation skip flag
            // and norm), one row per lane, broadcast by shuffles in the chunk loop below
            int my_skip = 1;
            float my_norm = 0.f;
            if (p.mode != 0) {
                const int row = q * 32 + lane;
                const int bp = row / p.kslot, j = jbase + row - bp * p.kslot;
                const int bb = bfirst + bp;
                if (bp < p.ppt && bb < p.ncols && j < p.KO) {
                    const size_t pj = (size_t)bb * p.KO + j;
                    my_skip = p.skip[p.prop[pj]] ? 1 : 0;
                    my_norm = p.norms[pj];
                    if (p.mode == 1) my_norm = p.c0[bb] + my_norm;   // diff2 = (c0 + norm) - C
                }
            }
            __syncwarp();
            const int nchunk = (p.tn ? p.tn : TN) / 32;
            // split-K proposal tiles: exchange the slices' partial sums through global memory;
            // the sum own + other is the same whichever slice finishes second
            const float* other = nullptr;
            bool emit = true;
            if (p.mode == 1 && ksp == 2) {
                const int slice = tile % ksp;
                const size_t wsz = (size_t)nchunk * 1024;
                float* mine = p.part + (((size_t)tt * 2 + slice) * 4 + q) * wsz;
                for (int c = 0; c < nchunk; c++) {
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(abuf * TN + c * 32), v);
#pragma unroll
                    for (int e = 0; e < 32; e++) mine[(size_t)c * 1024 + e * 32 + lane] = __uint_as_float(v[e]);
                }
                __threadfence();
                __syncwarp();
                int first = 0;
                if (lane == 0) first = atomicAdd(&p.fix[tt * 4 + q], 1) == 0;
                first = __shfl_sync(0xffffffffu, first, 0);
                if (first) {
                    emit = false;
                } else {
                    __threadfence();
                    other = p.part + (((size_t)tt * 2 + (1 - slice)) * 4 + q) * wsz;
                }
            }
            if (p.mode == 2) {
                // the thread's row straight from TMEM (32x32b: lane = row, 32 columns per load):
                // score = M + log sum_t pdf_t exp(C_t - M), M = max_t C_t, in two passes over
                // TMEM (the max, then the sum) with no data-dependent branch; pdf_t of column
                // c*32 + e is held by lane e (as FP32) and broadcast by a shuffle
                const double* pt = p.pdf_t + (size_t)bfirst * p.T;
                float wv[TN / 32];
#pragma unroll
                for (int c = 0; c < TN / 32; c++) {
                    const int t = c * 32 + lane;
                    wv[c] = (c < nchunk && t < p.T && bfirst < p.ncols) ? (float)pt[t] : 0.f;
                }
                float m = -INFINITY;
#pragma unroll
                for (int c = 0; c < TN / 32; c++) {
                    if (c >= nchunk) break;
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(abuf * TN + c * 32), v);
#pragma unroll
                    for (int e = 0; e < 32; e++)
                        if (c * 32 + e < p.T) m = fmaxf(m, __uint_as_float(v[e]));
                }
                float sacc = 0.f;
#pragma unroll
                for (int c = 0; c < TN / 32; c++) {
                    if (c >= nchunk) break;
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(abuf * TN + c * 32), v);
#pragma unroll
                    for (int e = 0; e < 32; e++) {
                        const float w = __shfl_sync(0xffffffffu, wv[c], e);
                        if (c * 32 + e < p.T) sacc += w * __expf(__uint_as_float(v[e]) - m);
                    }
                }
                const int j = jbase + q * 32 + lane;
                if (j < p.KO && bfirst < p.ncols) {
                    const size_t pj = (size_t)bfirst * p.KO + j;
                    p.d2c[pj] = (my_skip || !(sacc > 0.f)) ? -INFINITY
                                                           : m - my_norm + __logf(sacc) + (float)log(p.pdf_oc[p.prop[pj]]);
                }
            }
            // raw products with one column per batch entry (norms, network layers: out[col][row]):
            // the TMEM lane is the row, which is the contiguous axis of the output, so each of
            // the 32 columns of a load is one coalesced 128-byte store, no transpose
            const bool raw_rows = p.mode == 0 && p.raw && p.T == 1;
            const size_t ks = p.ko_stride ? (size_t)p.ko_stride : (size_t)p.KO;
            if (raw_rows) {
                const int oc = mt * TM + q * 32 + lane;
                for (int c = 0; c < nchunk; c++) {
                    uint32_t v[32];
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(abuf * TN + c * 32), v);
                    if (oc < p.KO) {
#pragma unroll
                        for (int e = 0; e < 32; e++) {
                            const int col = n0 + c * 32 + e;
                            if (col < p.ncols) outp[(size_t)col * ks + p.row0 + oc] = __uint_as_float(v[e]);
                        }
                    }
                }
            }
            for (int c = 0; c < (p.mode == 2 || !emit || raw_rows ? 0 : nchunk); c++) {
                uint32_t v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(abuf * TN + c * 32), v);
                if (other) {
#pragma unroll
                    for (int e = 0; e < 32; e++)
                        v[e] = __float_as_uint(__uint_as_float(v[e]) + __ldcg(other + (size_t)c * 1024 + e * 32 + lane));
                }
#pragma unroll
                for (int j = 0; j < 32; j++) sbuf[lane * EPI_LD + j] = __uint_as_float(v[j]);
                __syncwarp();
                unsigned lmin = 0xffffffffu;
                int b;
                if (p.mode == 0) {
                    // lane = column within the chunk; rows walk the warp's 32 TMEM lanes
                    const int col = n0 + c * 32 + lane;
                    const bool cok = col < p.ncols;
                    b = cok ? col / p.T : 0;
                    const int t = cok ? col - b * p.T : 0;
                    const float c0 = (cok && !p.raw) ? p.c0[b] : 0.f;  // raw mode has no c0 array
                    for (int r = 0; r < 32; r++) {
                        const int oc = mt * TM + q * 32 + r;
                        if (!cok || oc >= p.KO) continue;
                        const size_t og = (size_t)p.row0 + oc;
                        float d;
                        if (p.raw) {
                            d = sbuf[r * EPI_LD + lane];
                        } else if (p.skip[og]) {
                            d = -999.f;
                        } else {
                            d = c0 + p.norms[(size_t)b * ks + og] - sbuf[r * EPI_LD + lane];
                            lmin = min(lmin, f2key(d));
                        }
                        outp[((size_t)b * ks + og) * p.T + t] = d;
                    }
                } else {
                    // proposal tile: column = translation; the warp's 32 rows are proposals of
                    // one particle (kslot a multiple of 32)
                    const int t = c * 32 + lane;
                    const int bp = (q * 32) / p.kslot;
                    b = bfirst + bp;
                    const bool cok = t < p.T && bp < p.ppt && b < p.ncols;
                    for (int r = 0; r < 32; r++) {
                        const int j = q * 32 + r - bp * p.kslot;
                        const int skip_r = __shfl_sync(0xffffffffu, my_skip, r);
                        const float cn_r = __shfl_sync(0xffffffffu, my_norm, r);
                        if (!cok || j >= p.KO) continue;
                        const size_t pj = (size_t)b * p.KO + j;
                        float d;
                        if (skip_r) {
                            d = -999.f;
                        } else {
                            d = cn_r - sbuf[r * EPI_LD + lane];
                            lmin = min(lmin, f2key(d));
                        }
                        p.d2c[pj * p.T + t] = d;
                    }
                }
                if (lmin != 0xffffffffu) atomicMin(&wmin[b - bfirst], lmin);
                __syncwarp();
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty_bar[abuf]);
            for (int i = lane; i < TN + 2; i += 32) {
                const int b = bfirst + i;
                if (wmin[i] != 0xffffffffu && (p.mode == 0 ? b * p.T < p.ncols : b < p.ncols))
                    atomicMin(&p.minkey[b], wmin[i]);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    if (abort_flag && threadIdx.x == 0) atomicExch(p.err, T2B_ERR_TIMEOUT);
    tc_fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// ------------------------------------------------------------------ operands
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo)
{
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Chunked coarse pass: the projections of `rows` orientations (Euler matrices eul) interpolated
// straight into the split-BF16 operands, element (row, kk) = window pixel kpix[kk]: Ph/Pl
// (re, im pairs, kdim / 2 per row) and the |projection|^2 operand Nh/Nl (kn per row), rows up
// to rpad and elements beyond nk zero.  The same values as k_project followed by k_split_proj
// and k_split_norm_proj (one project_window_pixel each), without the FP32 table in between.
__global__ void __launch_bounds__(256) k_project_split(cudaTextureObject_t mdl, Volume v,
                                                       const double* __restrict__ eul, int rows, int rpad, int s,
                                                       const int* __restrict__ kpix, int nk, int kh, int kn,
                                                       __nv_bfloat162* __restrict__ ph, __nv_bfloat162* __restrict__ pl,
                                                       __nv_bfloat16* __restrict__ nh, __nv_bfloat16* __restrict__ nl)
{
    const int r = blockIdx.y;
    const int kk = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rpad || kk >= kn) return;
    float2 z = make_float2(0.f, 0.f);
    if (r < rows && kk < nk) z = project_window_pixel(mdl, v, eul + 9 * (size_t)r, kpix[kk], s);
    if (kk < kh) {
        __nv_bfloat16 h0, l0, h1, l1;
        split_bf16(z.x, h0, l0);
        split_bf16(z.y, h1, l1);
        ph[(size_t)r * kh + kk] = __halves2bfloat162(h0, h1);
        pl[(size_t)r * kh + kk] = __halves2bfloat162(l0, l1);
    }
    split_bf16(z.x * z.x + z.y * z.y, nh[(size_t)r * kn + kk], nl[(size_t)r * kn + kk]);
}

// projections (K*O x P complex) -> Ph/Pl (m_pad x kdim bf16), zero padded
__global__ void k_split_proj(const float2* __restrict__ proj, int rows, int P, const int* __restrict__ kpix, int nk,
                             int kdim, __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, long long total)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / (kdim / 2);
        const int kk = (int)(i - r * (kdim / 2));
        float2 v = make_float2(0.f, 0.f);
        if (r < rows && kk < nk) v = proj[r * P + kpix[kk]];
        __nv_bfloat16 h0, l0, h1, l1;
        split_bf16(v.x, h0, l0);
        split_bf16(v.y, h1, l1);
        reinterpret_cast<__nv_bfloat162*>(hi)[i] = __halves2bfloat162(h0, h1);
        reinterpret_cast<__nv_bfloat162*>(lo)[i] = __halves2bfloat162(l0, l1);
    }
}

// shifted, CTF- and sigma-weighted images: column b*T+t, value cvec_b[p] * ab_t[p];
// one operand row per CTA iteration, 4 complex values (16-byte stores) per thread.
// cvec = null: the phase rows ab_t themselves.  Returns at once while *gate != 0
// (learned proposals in use: only the full coarse pass reads these rows).
__global__ void __launch_bounds__(128) k_split_img(const float2* __restrict__ cvec, const float2* __restrict__ ab,
                                                   int ncols, int nrows, int T, int P, const int* __restrict__ kpix,
                                                   int nk, int kdim, __nv_bfloat16* __restrict__ hi,
                                                   __nv_bfloat16* __restrict__ lo, const int* gate, int swz)
{
    if (gate && *gate != 0) return;
    const int nv = kdim / 8;  // groups of 4 complex values
    for (int col = blockIdx.x; col < nrows; col += gridDim.x) {
        const bool ok = col < ncols;
        const int b = ok ? col / T : 0, t = ok ? col - b * T : 0;
        const float2* cb = cvec ? cvec + (size_t)b * P : nullptr;
        const float2* at = ab + (size_t)t * P;
        // row-major rows, or (swz) the pre-swizzled K-blocked layout of swz_offset
        uint4* dh = reinterpret_cast<uint4*>(hi);
        uint4* dl = reinterpret_cast<uint4*>(lo);
        for (int g = threadIdx.x; g < nv; g += blockDim.x) {
            __nv_bfloat162 h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int kk = 4 * g + e;
                float2 v = make_float2(0.f, 0.f);
                if (ok && kk < nk) {
                    const int pp = kpix[kk];
                    const float2 a = at[pp];
                    if (cb) {
                        const float2 c = cb[pp];
                        v = make_float2(c.x * a.x - c.y * a.y, c.x * a.y + c.y * a.x);
                    } else {
                        v = a;
                    }
                }
                __nv_bfloat16 h0, l0, h1, l1;
                split_bf16(v.x, h0, l0);
                split_bf16(v.y, h1, l1);
                h[e] = __halves2bfloat162(h0, h1);
                l[e] = __halves2bfloat162(l0, l1);
            }
            const size_t o = swz ? swz_offset(col, 8 * g, nrows) / 8 : (size_t)col * (kdim / 8) + g;
            dh[o] = *reinterpret_cast<const uint4*>(h);
            dl[o] = *reinterpret_cast<const uint4*>(l);
        }
    }
}

// |projection|^2 (K*O x P) -> hi/lo (m_pad x kn), zero padded
__global__ void k_split_norm_proj(const float2* __restrict__ proj, int rows, int P, const int* __restrict__ kpix,
                                  int nk, int kn, __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                  long long total)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / kn;
        const int kk = (int)(i - r * kn);
        float v = 0.f;
        if (r < rows && kk < nk) {
            const float2 z = proj[r * P + kpix[kk]];
            v = z.x * z.x + z.y * z.y;
        }
        split_bf16(v, hi[i], lo[i]);
    }
}

// 0.5 M (scale CTF)^2 (n x P) -> hi/lo (b_pad x kn)
__global__ void k_split_w2(const float* __restrict__ w2, int n, int P, const int* __restrict__ kpix, int nk, int kn,
                           __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, long long total)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / kn;
        const int kk = (int)(i - r * kn);
        const float v = (r < n && kk < nk) ? w2[r * P + kpix[kk]] : 0.f;
        split_bf16(v, hi[i], lo[i]);
    }
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encoder()
{
    static EncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
            throw Error{T2B_ERR_CUDA, "cuTensorMapEncodeTiled unavailable"};
        fn = reinterpret_cast<EncodeFn>(p);
    }
    return fn;
}

CUtensorMap make_map(void* ptr, int rows, int kdim, int box_rows)
{
    CUtensorMap m;
    const cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kdim * 2};
    const cuuint32_t box[2] = {(cuuint32_t)TK, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims, strides, box, estr,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error{T2B_ERR_CUDA, "cuTensorMapEncodeTiled failed"};
    return m;
}

int sms()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

}  // namespace

bool tc_supported() { return true; }

size_t tc_kdim(int nk) { return (size_t)((2 * nk + TK - 1) / TK) * TK; }
size_t tc_kn(int nk) { return (size_t)((nk + TK - 1) / TK) * TK; }

// descriptor slots in op.maps (TC_MAP_SLOTS of 128 bytes)
enum { MAP_PH = 0, MAP_PL, MAP_IH, MAP_IL, MAP_NH, MAP_NL, MAP_WH, MAP_WL,
       MAP_IAH, MAP_IAL, MAP_RAH, MAP_RAL, MAP_RBH, MAP_RBL,
       MAP_IH128, MAP_IL128, MAP_WAH, MAP_WAL, MAP_IAH_N, MAP_IAL_N, MAP_COUNT };
static_assert(MAP_COUNT <= TC_MAP_SLOTS, "tensor-map slots");
static_assert(sizeof(CUtensorMap) == 128, "tensor-map size");

void tc_encode(void* ptr, int rows, int kdim, bool a_side, void* out128, int box_rows)
{
    const CUtensorMap m = make_map(ptr, rows, kdim, box_rows > 0 ? box_rows : (a_side ? TM : TN));
    std::memcpy(out128, &m, sizeof(m));
}

void tc_prepare_projections(const Tables& tb, TcOperands& op, cudaStream_t st)
{
    T2B_REQUIRE(op.maps, T2B_ERR_STATE, "tensor-map buffer not allocated");
    CUtensorMap h[MAP_WL + 1];
    h[MAP_PH] = make_map(op.bh, op.m_pad, op.kdim, TM);
    h[MAP_PL] = make_map(op.bl, op.m_pad, op.kdim, TM);
    h[MAP_IH] = make_map(op.ah, op.n_pad, op.kdim, TN);
    h[MAP_IL] = make_map(op.al, op.n_pad, op.kdim, TN);
    h[MAP_NH] = make_map(op.nh, op.m_pad, op.kn, TM);
    h[MAP_NL] = make_map(op.nl, op.m_pad, op.kn, TM);
    h[MAP_WH] = make_map(op.wh, op.b_pad, op.kn, TN);
    h[MAP_WL] = make_map(op.wl, op.b_pad, op.kn, TN);
    T2B_CUDA(cudaStreamSynchronize(st));
    T2B_CUDA(cudaMemcpy(op.maps, h, sizeof(h), cudaMemcpyHostToDevice));  // slots MAP_PH..MAP_WL
    // and with a 128-row box: dense coarse tiles of 128 columns (t2b_autotune)
    CUtensorMap h128[2] = {make_map(op.ah, op.n_pad, op.kdim, 128), make_map(op.al, op.n_pad, op.kdim, 128)};
    T2B_CUDA(cudaMemcpy(static_cast<unsigned char*>(op.maps) + 128 * MAP_IH128, h128, sizeof(h128),
                        cudaMemcpyHostToDevice));
    const int rows = op.chunk > 0 ? op.chunk : tb.K * tb.O;
    // sizes were fixed when the operand buffers were allocated
    T2B_REQUIRE(op.m_pad == (rows + TM - 1) / TM * TM && op.kdim == (int)tc_kdim(tb.nk), T2B_ERR_STATE,
                "tensor-core operand sizes do not match their allocation");
    if (op.chunk == 0) tc_split_chunk(tb, op, rows, st);   // chunked: split per chunk in each batch
}

void tc_project_split(const Tables& tb, TcOperands& op, cudaTextureObject_t mtex, const Volume& v, const double* eul,
                      int rows, cudaStream_t st)
{
    T2B_REQUIRE(op.bh && op.nh && rows >= 1 && rows <= op.m_pad && op.kn >= op.kdim / 2, T2B_ERR_STATE,
                "tensor-core operands not allocated");
    const int rpad = (rows + TM - 1) / TM * TM;
    dim3 grid((op.kn + 255) / 256, rpad);
    k_project_split<<<grid, 256, 0, st>>>(mtex, v, eul, rows, rpad, tb.s, tb.kpix, tb.nk,
                                          op.kdim / 2, op.kn,
                                          (__nv_bfloat162*)op.bh, (__nv_bfloat162*)op.bl, (__nv_bfloat16*)op.nh,
                                          (__nv_bfloat16*)op.nl);
    T2B_CUDA(cudaGetLastError());
}

// Rows [0, rows) of the resident table tb.proj_c into the split-BF16 projection and |projection|^2 operands; the
// rows up to the operands' next multiple of 128 are zeroed.
void tc_split_chunk(const Tables& tb, TcOperands& op, int rows, cudaStream_t st)
{
    T2B_REQUIRE(op.bh && op.bl && rows >= 1 && rows <= op.m_pad, T2B_ERR_STATE, "tensor-core operands not allocated");
    const long long rpad = (rows + TM - 1) / TM * TM;
    k_split_proj<<<4 * sms(), 256, 0, st>>>(tb.proj_c, rows, tb.P, tb.kpix, tb.nk, op.kdim, (__nv_bfloat16*)op.bh,
                                            (__nv_bfloat16*)op.bl, rpad * op.kdim / 2);
    T2B_REQUIRE(op.nh && op.nl && op.kn == (int)tc_kn(tb.nk), T2B_ERR_STATE, "norm operands not allocated");
    k_split_norm_proj<<<4 * sms(), 256, 0, st>>>(tb.proj_c, rows, tb.P, tb.kpix, tb.nk, op.kn, (__nv_bfloat16*)op.nh,
                                                 (__nv_bfloat16*)op.nl, rpad * op.kn);
    T2B_CUDA(cudaGetLastError());
}

void tc_init_attributes()
{
    T2B_CUDA(cudaFuncSetAttribute(k_diff2_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES));
    (void)encoder();
    (void)sms();
}

static void launch_gemm(const TcOperands& op, int ia, int ib, TcParams& p, cudaStream_t st)
{
    const int grid = std::min(sms(), p.m_tiles * p.n_tiles * std::max(1, p.ksplit));
    k_diff2_tc<<<grid, NTHREADS, SMEM_BYTES, st>>>(static_cast<const CUtensorMap*>(op.maps), ia, ib, p);
    T2B_CUDA(cudaGetLastError());
}

// N[b][oc] = sum_p w2[b][p] |P_oc[p]|^2 with the same split-BF16 tensor-core kernel
void tc_launch_norms(const Tables& tb, const Work& w, TcOperands& op, cudaStream_t st, const int* gate, int gate_run,
                     RowChunk ch, bool split_w2)
{
    const int b_pad = (w.n + TN - 1) / TN * TN;
    T2B_REQUIRE(b_pad <= op.b_pad, T2B_ERR_ARG, "batch larger than the tensor-core workspace");
    if (split_w2) {
        k_split_w2<<<4 * sms(), 256, 0, st>>>(w.w2, w.n, tb.P, tb.kpix, tb.nk, op.kn, (__nv_bfloat16*)op.wh,
                                              (__nv_bfloat16*)op.wl, (long long)b_pad * op.kn);
        T2B_CUDA(cudaGetLastError());
    }
    TcParams p{};
    p.m_tiles = ch.rows ? (ch.rows + TM - 1) / TM : op.m_pad / TM;
    p.n_tiles = b_pad / TN;
    p.kblocks = op.kn / TK;
    p.raw = 1;
    p.KO = ch.rows ? ch.rows : tb.K * tb.O;
    p.row0 = ch.row0;
    p.ko_stride = ch.rows ? tb.K * tb.O : 0;
    p.T = 1;
    p.ncols = w.n;
    p.skip = tb.skip;
    p.d2c = w.norms;
    p.minkey = w.minkey_c;
    p.err = w.err;
    p.products = 3;
    p.gate = gate;
    p.gate_run = gate_run;
    launch_gemm(op, MAP_NH, MAP_WH, p, st);
}

void tc_split_images(const Tables& tb, const Work& w, TcOperands& op, cudaStream_t st, const int* gate)
{
    const int ncols = w.n * tb.T;
    const int n_pad = (ncols + TN - 1) / TN * TN;
    T2B_REQUIRE(n_pad <= op.n_pad, T2B_ERR_ARG, "batch larger than the tensor-core workspace");
    k_split_img<<<std::min(n_pad, 16 * sms()), 128, 0, st>>>(w.cvec, tb.ab_c, ncols, n_pad, tb.T, tb.P, tb.kpix, tb.nk,
                                                            op.kdim, (__nv_bfloat16*)op.ah, (__nv_bfloat16*)op.al,
                                                            gate, 0);
    T2B_CUDA(cudaGetLastError());
}

void tc_split_phases(const Tables& tb, const TcOperands& op, int rows, void* hi, void* lo, cudaStream_t st)
{
    T2B_REQUIRE(rows >= tb.T, T2B_ERR_ARG, "phase operand rows");
    T2B_REQUIRE(rows % 8 == 0, T2B_ERR_ARG, "phase operand rows");
    k_split_img<<<std::min(rows, 16 * sms()), 128, 0, st>>>(nullptr, tb.ab_c, tb.T, rows, tb.T, tb.P, tb.kpix, tb.nk,
                                                           op.kdim, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, nullptr, 1);
    T2B_CUDA(cudaGetLastError());
}

void tc_launch_diff2(const Tables& tb, const Work& w, TcOperands& op, cudaStream_t st, const int* gate, int gate_run,
                     RowChunk ch)
{
    const int ncols = w.n * tb.T;
    const int n_pad = (ncols + TN - 1) / TN * TN;
    T2B_REQUIRE(n_pad <= op.n_pad, T2B_ERR_ARG, "batch larger than the tensor-core workspace");
    T2B_REQUIRE(op.dense_tn == 256 || op.dense_tn == 128, T2B_ERR_ARG, "dense tile width");
    TcParams p{};
    p.raw = 0;
    p.m_tiles = ch.rows ? (ch.rows + TM - 1) / TM : op.m_pad / TM;
    p.n_tiles = (ncols + op.dense_tn - 1) / op.dense_tn;
    p.tn = op.dense_tn == TN ? 0 : op.dense_tn;
    p.group = op.group_m;
    p.kblocks = op.kdim / TK;
    p.KO = ch.rows ? ch.rows : tb.K * tb.O;
    p.row0 = ch.row0;
    p.ko_stride = ch.rows ? tb.K * tb.O : 0;
    p.T = tb.T;
    p.ncols = ncols;
    p.c0 = w.c0;
    p.norms = w.norms;
    p.skip = tb.skip;
    p.d2c = w.d2c;
    p.minkey = w.minkey_c;
    p.err = w.err;
    p.products = 3;
    p.gate = gate;
    p.gate_run = gate_run;
    launch_gemm(op, MAP_PH, op.dense_tn == TN ? MAP_IH : MAP_IH128, p, st);
}

void tc_set_map(TcOperands& op, int slot, void* ptr, int rows, int kdim, bool a_side)
{
    T2B_REQUIRE(slot >= MAP_IAH && slot < MAP_COUNT && op.maps, T2B_ERR_STATE, "bad tensor-map slot");
    unsigned char blob[128];
    tc_encode(ptr, rows, kdim, a_side, blob);
    T2B_CUDA(cudaMemcpy(static_cast<unsigned char*>(op.maps) + 128 * slot, blob, 128, cudaMemcpyHostToDevice));
}

int tc_slot_audit() { return MAP_IAH; }
int tc_slot_rescore() { return MAP_RAH; }
int tc_slot_audit_w2() { return MAP_WAH; }
int tc_slot_audit_narrow() { return MAP_IAH_N; }

void tc_set_map_box(TcOperands& op, int slot, void* ptr, int rows, int kdim, int box_rows)
{
    T2B_REQUIRE(slot >= MAP_IAH && slot < MAP_COUNT && op.maps, T2B_ERR_STATE, "bad tensor-map slot");
    const CUtensorMap m = make_map(ptr, rows, kdim, box_rows);
    T2B_CUDA(cudaMemcpy(static_cast<unsigned char*>(op.maps) + 128 * slot, &m, 128, cudaMemcpyHostToDevice));
}

// Low-resolution rescoring contraction: particle b's K1 candidates (gathered ring
// projections, slots MAP_RAH/RAL, rows b*K1 + j) against its T shifted ring
// images (MAP_RBH/RBL, 96-row box from row b*T); the epilogue reduces every
// candidate's row to its score (mode 2) into score[b*K1 + j].  K1 a multiple of 128.
void tc_launch_rescore(int n, int k1, int T, int kr, TcOperands& op, const float* norms, const unsigned char* skip,
                       const int* cand, const double* pdf_t, const double* pdf_oc, float* score, int* err,
                       cudaStream_t st)
{
    T2B_REQUIRE(k1 % TM == 0 && T <= 96 && kr % TK == 0, T2B_ERR_STATE, "rescoring tile shape");
    TcParams p{};
    p.mode = 2;
    p.ppt = 1;
    p.kslot = TM;
    p.mtp = k1 / TM;
    p.tn = 96;
    p.m_tiles = n * p.mtp;
    p.n_tiles = 1;
    p.kblocks = kr / TK;
    p.KO = k1;
    p.T = T;
    p.ncols = n;
    p.norms = norms;
    p.skip = skip;
    p.prop = cand;
    p.pdf_t = pdf_t;
    p.pdf_oc = pdf_oc;
    p.d2c = score;
    p.err = err;
    p.products = 3;
    launch_gemm(op, MAP_RAH, MAP_RBH, p, st);
}

// Restricted coarse pass: every particle against its own proposals only.
// Cross term C[b, j][t] = Re sum_p P_oc(j)[p] conj(cvec_b[p] ab_t[p])
//                       = Re sum_p (P_oc(j)[p] conj(cvec_b[p])) conj(ab_t[p]),
// so the A rows (a_hi/a_lo, a_rows rows, row b*kslot + j) hold the proposal times the
// conjugate particle image (k_prop_gather) and B is the T phase rows ab_t padded to tn
// rows (b_hi/b_lo), shared by every tile and resident in L2; both are stored
// pre-swizzled and K-blocked (swz_offset) and fetched by one bulk copy per tile and
// k-block.  Tiles of 128 / kslot particles.  Runs while *w.gate != 0.
void tc_launch_prop(const Tables& tb, const Work& w, TcOperands& op, int kslot, int tn, const float* nprop,
                    const void* a_hi, const void* a_lo, int a_rows, const void* b_hi, const void* b_lo,
                    float* part, int* fix, int part_tiles, cudaStream_t st)
{
    T2B_REQUIRE((kslot == 64 || kslot == TM) && w.kprop <= kslot && tb.T <= tn && tn % 32 == 0 && tn <= TN,
                T2B_ERR_STATE, "proposal tile shape");
    TcParams p{};
    p.mode = 1;
    p.a_hi = a_hi;
    p.a_lo = a_lo;
    p.b_hi = b_hi;
    p.b_lo = b_lo;
    p.a_rows = a_rows;
    p.b_rows = tn;
    p.ppt = TM / kslot;
    p.kslot = kslot;
    p.m_tiles = (w.n + p.ppt - 1) / p.ppt;
    // fewer m-tiles than half the SMs: two K slices per m-tile (the sum of the two partial
    // accumulators is order-independent, so the result does not depend on the split)
    if (part && fix && 2 * p.m_tiles <= sms() && p.m_tiles <= part_tiles && op.kdim / TK >= 2) {
        p.ksplit = 2;
        p.part = part;
        p.fix = fix;
        T2B_CUDA(cudaMemsetAsync(fix, 0, (size_t)p.m_tiles * 4 * sizeof(int), st));
    }
    p.n_tiles = 1;
    p.kblocks = op.kdim / TK;
    p.KO = w.kprop;
    p.T = tb.T;
    p.ncols = w.n;
    p.c0 = w.c0;
    p.norms = nprop;
    p.skip = tb.skip;
    p.prop = w.prop;
    p.d2c = w.d2c;
    p.minkey = w.minkey_c;
    p.err = w.err;
    p.products = 3;
    p.gate = w.gate;
    p.gate_run = 1;
    p.tn = tn;
    T2B_REQUIRE(a_rows % 8 == 0 && (w.n + p.ppt - 1) / p.ppt * TM <= a_rows, T2B_ERR_STATE, "proposal operand rows");
    launch_gemm(op, MAP_PH, MAP_IH, p, st);   // (the maps are not read: bulk copies)
}

// Norms of the audited particles N[a][oc] = sum_k w2_a[k] |P_oc|^2_k: the full
// pass's norm contraction (|P|^2 operand MAP_NH/NL) against the audit slots' w2
// rows (MAP_WAH/WAL, split-BF16, 32-row box): 128 x 32 tiles, one pass over the
// |P|^2 operand at the memory rate, the same sums as the full pass's norms.
void tc_launch_audit_norms(const Tables& tb, TcOperands& op, int na_max, float* norma, int* err, cudaStream_t st)
{
    TcParams p{};
    p.m_tiles = op.m_pad / TM;
    p.n_tiles = (na_max + 31) / 32;
    p.kblocks = op.kn / TK;
    p.raw = 1;
    p.KO = tb.K * tb.O;
    p.T = 1;
    p.ncols = na_max;
    p.skip = tb.skip;
    p.d2c = norma;
    p.err = err;
    p.products = 3;
    p.group = op.group_m;
    p.tn = 32;
    launch_gemm(op, MAP_NH, MAP_WAH, p, st);
}

// Full coarse pass of the audited particles: dense tiles over every
// orientation against the audit image operand (MAP_IAH/IAL, na_max*T rows).
// Column tiles: the fewest 256-wide ones for the audited columns, each narrowed to a
// multiple of 32 (11 audited particles x 81 shifts: 4 x 224 columns, not 4 x 256).
// The audited count na of a batch is known on the device only: with na_max slots, a
// batch of fewer audited particles runs the narrower variant (na_max - 1 slots,
// MAP_IAH_N/IAL_N) when its tiles cover fewer columns, a batch of na_max the full one;
// each launch returns at once unless the count is its own.
static void audit_shape(int cols, int& n_tiles, int& tn)
{
    n_tiles = (cols + TN - 1) / TN;
    tn = ((cols + n_tiles - 1) / n_tiles + 31) / 32 * 32;
}

int tc_audit_tn(int na, int T)
{
    int nt, tn;
    audit_shape(na * T, nt, tn);
    return tn;
}

int tc_audit_narrow_tn(int na_max, int T)
{
    if (na_max < 2) return 0;
    int nf, tf, nn, tnn;
    audit_shape(na_max * T, nf, tf);
    audit_shape((na_max - 1) * T, nn, tnn);
    return nn * tnn < nf * tf ? tnn : 0;
}

void tc_launch_audit(const Tables& tb, TcOperands& op, int na_max, const int* na, const float* c0a,
                     const float* norma, float* d2a, unsigned* minkeya, int* err, cudaStream_t st)
{
    TcParams p{};
    int tf = TN;
    p.m_tiles = op.m_pad / TM;
    audit_shape(na_max * tb.T, p.n_tiles, tf);
    p.tn = tf == TN ? 0 : tf;
    p.kblocks = op.kdim / TK;
    p.KO = tb.K * tb.O;
    p.T = tb.T;
    p.ncols = na_max * tb.T;
    p.c0 = c0a;
    p.norms = norma;
    p.skip = tb.skip;
    p.d2c = d2a;
    p.minkey = minkeya;
    p.err = err;
    p.products = 3;
    p.group = op.group_m;
    const int tn_n = tc_audit_narrow_tn(na_max, tb.T);
    if (tn_n > 0 && na) {
        TcParams q = p;
        int tq = TN;
        audit_shape((na_max - 1) * tb.T, q.n_tiles, tq);
        q.ncols = (na_max - 1) * tb.T;
        q.tn = tq == TN ? 0 : tq;
        q.cnt = na;
        q.cnt_lo = 1;
        q.cnt_hi = na_max - 1;
        launch_gemm(op, MAP_PH, MAP_IAH_N, q, st);
        p.cnt = na;
        p.cnt_lo = na_max;
        p.cnt_hi = na_max;
    }
    launch_gemm(op, MAP_PH, MAP_IAH, p, st);
}

// out[n][m] = sum_k A[m][k] B[n][k]: both operands K-major BF16 behind the
// tensor maps maps[ia] (A, 128-row box) and maps[ib] (B, a tn-row box: 256 or
// 128); K a multiple of 64; products = 1 is one BF16 product (the lo halves are
// not read).  ksplit > 1 splits K into slices (more tiles for a small M x N):
// slice s writes its partial product at out + s * N * M, to be summed in a fixed
// order by the caller; returns the number of slices written.
int tc_gemm_raw(const void* maps, int ia, int ib, int M, int N, int K, float* out, int products, int* err,
                cudaStream_t st, int ksplit, int tn)
{
    T2B_REQUIRE(K % TK == 0 && M > 0 && N > 0 && products >= 1 && products <= 3, T2B_ERR_ARG, "tensor-core GEMM shape");
    T2B_REQUIRE(tn == 256 || tn == 128, T2B_ERR_ARG, "tensor-core GEMM tile width");
    TcParams p{};
    p.m_tiles = (M + TM - 1) / TM;
    p.n_tiles = (N + tn - 1) / tn;
    p.kblocks = K / TK;
    // no empty slice: ceil(kblocks / kper) slices of kper = ceil(kblocks / ksplit) k-blocks
    const int kper = (p.kblocks + std::max(1, ksplit) - 1) / std::max(1, ksplit);
    p.ksplit = (p.kblocks + kper - 1) / kper;
    p.tn = tn == TN ? 0 : tn;
    p.raw = 1;
    p.KO = M;
    p.T = 1;
    p.ncols = N;
    p.d2c = out;
    p.err = err;
    p.products = products;
    const int grid = std::min(sms(), p.m_tiles * p.n_tiles * p.ksplit);
    k_diff2_tc<<<grid, NTHREADS, SMEM_BYTES, st>>>(static_cast<const CUtensorMap*>(maps), ia, ib, p);
    T2B_CUDA(cudaGetLastError());
    return p.ksplit;
}

}  // namespace t2b
