// Batched ensembles: many frictional-parameter instances that share a fault
// geometry march together, so that the traction product of every Runge-Kutta
// stage becomes one dense contraction T = K V per geometry (K: 3N x 2N receiver
// x source DOFs, V: 2N x instances) on the tcgen05 tensor cores, or, for a
// geometry held as a hierarchical matrix, the two-pass contraction described
// before k_hm_contract.
//
// Precision.  A dense geometry's K and V are both held as fp16 hi/lo pairs,
// the lo image the residual times 2^11, with power-of-two scales per K row, per
// 128-row x 64-source K-block and per 64-source V-block (the scales keep every
// value inside fp16's range).  Each 16-source step forms Khi Vhi + 2^-11 (Khi
// Vlo + Klo Vhi) in FP32 in tensor memory (the V hi and lo images are
// consecutive rows of one operand, so one MMA of N = 2 NI takes both Khi
// products into two accumulator halves that the drain adds); every 64-source
// k-block goes into a fresh accumulator that the drain scales and adds into
// FP32, then FP64, register sums.  The dropped Klo Vlo term and the residuals
// are of relative size 2^-21.  A hierarchical geometry holds its images as two
// or three bf16 planes (k_hm_contract).  State,
// stage combinations, error norm and step control stay FP64 and follow the
// single-instance integrator (rk.cu) per instance: every instance has its own
// step size, time, accept/reject decision and counters, and the reference
// RKQSm controller (fortran/3d/src/ode45.f90:51-108) accepts or rejects each attempt.
//
// Anchored stages.  The contraction's rounding (about 1e-5 of |K| |v|) would
// otherwise enter the embedded error estimate h sum_i dc_i k_i directly: for
// components whose state and rate are near zero (dip and normal traction and
// dip slip of a strike-slip fault) the ratio |yerr/yscal| is then set by the
// rounding and not by h, and at rtol 1e-8 nearly every attempt is rejected.
// Stage 1 of a step therefore contracts v1 = v(y) once (the anchor t1 = K v1,
// kept with v1), and stages 2-6 contract only the increment: t_s = t1 +
// K (v_s - v1).  Since sum_i dc_i = 0 the anchor's rounding cancels from the
// error estimate, and the increments' rounding scales with |v_s - v1|, which
// vanishes with h like the truncation error it competes with.
//
// Memory layout.  K is stored once per geometry, already in the byte image of
// the shared-memory tiles that the MMA reads: for every 128-row tile and
// 64-source k-block, a 16 KB fp16 hi image then a 16 KB lo image (scaled by
// 2^11), rows of 128 bytes in the 128-byte swizzle (16-byte chunk c of row r at
// chunk c ^ (r mod 8)), with a power-of-two scale per row and per 128 x 64
// block.  One 32 KB cp.async.bulk moves a whole k-block of a tile.  V is written
// by the stage prologue directly in the same image form (instances are the rows
// of the B operand), with a power-of-two scale per instance and k-block.  No
// tensor map is needed and nothing is re-laid out per stage.
//
// Contraction kernel.  Persistent, one CTA per SM, 320 threads: warp 0 issues
// the bulk copies (4 stages in flight), one lane of warp 1 issues tcgen05.mma
// and tcgen05.commit, warps 2-9 drain.  Every k-block accumulates into its own
// tensor-memory accumulator (four in turn), which the drain scales and adds
// into register sums (FP32 over 8 k-blocks, then FP64), so the tensor core's
// truncating accumulation spans 64 products.  (Accumulating a pair of k-blocks
// with 128-source scale blocks saves about 9 % of the kernel's cycles but took
// the ensemble's slip-rate histories from 2.3e-7 to 1.3e-6 of the FP64 oracle.)
// Work is a list of segments (tile, k-range) per CTA, produced on the host by a
// scheduler that the autotuner picks (stream-K, or split-K with longest-first
// packing), so geometries of uneven sizes balance across the SMs; every segment
// is then cut to at most 256 k-blocks.
// The partial sums of a tile are added in k order, in FP64, by the stage
// epilogue kernel: results are deterministic for a given schedule and an
// instance's column never depends on the other instances.
//
// Every mbarrier wait is bounded (about 4 s of %globaltimer); one that runs out
// records UCG_E_TIMEOUT, the CTA stops issuing, waits (bounded) for its copies
// and MMAs in flight, frees its tensor memory and returns.
//
// One attempt of all instances is 6 x (prologue, contraction, epilogue) plus a
// finish and a control kernel; the attempt is the body of a CUDA-graph while
// loop whose condition the control kernel sets, so a whole run of many
// attempts is ONE graph launch.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <queue>
#include <string>
#include <map>
#include <numeric>
#include <array>
#include <vector>
#include <cuda_bf16.h>
#include "ucg_internal.cuh"
#include "mlp.cuh"

namespace ucg {
namespace ens {

constexpr int BM = 128;                 // K rows per tile (MMA M)
constexpr int BK = 64;                  // sources per k-block (one 128-byte row of 16-bit values)
constexpr int A_HALF = BM * BK * 2;     // one 16-bit image of a tile k-block: 16 KB
constexpr int A_IMG = 2 * A_HALF;       // hi + lo
constexpr float LO_SCALE = 2048.0f, LO_UNSCALE = 1.0f / 2048.0f;   // dense images: lo = 2^11 residual
constexpr int MAX_GEOM = 16;
constexpr int EW_THREADS = 128;         // element-wise kernels: elements per block
constexpr int ST_THREADS = 256;         // finish / commit kernels: threads per block
constexpr int ST_PER = 4;               // state entries per thread (independent loads in flight)
constexpr int ST_SPAN = ST_THREADS * ST_PER;
constexpr unsigned long long TIMEOUT_NS = 4000000000ull;

// KLO: the stage also reads the K lo image (three MMAs per k-step); without it
// (stage increments) only the hi image is read and two MMAs run, Khi Vhi + Khi Vlo.
// MT: M-tiles per work unit sharing each V stage (2 halves the V bytes per K byte).
template <int NI, bool KLO, int MT>
struct Tile {
    static constexpr int B_HALF = NI * BK * 2;
    static constexpr int B_IMG = 2 * B_HALF;
    static constexpr int A_BYTES = KLO ? A_IMG : A_HALF;   // per M-tile
    static constexpr int STAGE = MT * A_BYTES + B_IMG;
    static constexpr int STAGES = (6 * 32768) / STAGE < 8 ? (6 * 32768) / STAGE : 8;   // ~192 KB in flight
    static constexpr int SMEM = STAGES * STAGE + 1024;   // + slack for 1024-byte alignment
    // MERGE: the V hi and lo images lie back to back in the stage, so one MMA
    // of N = 2 NI computes Khi Vhi and Khi Vlo into the two halves of a
    // 2 NI-column accumulator (the drain adds them); when two sets of MT such
    // accumulators do not fit the 512 tensor-memory columns, two MMAs of N = NI
    // accumulate into one NI-column accumulator instead
    static constexpr bool MERGE = 2 * MT * 2 * NI <= 512;
    static constexpr int ACC_N = MERGE ? 2 * NI : NI;
    // sets of MT FP32 accumulators in flight between the MMA issuer and the
    // drain: four where the 512 tensor-memory columns hold them, else two
    static constexpr int NACC = 4 * MT * ACC_N <= 512 ? 4 : 2;
    static constexpr uint32_t TMEM_COLS = NACC * MT * ACC_N;
    // instruction descriptor: F32 accumulator, A and B fp16 (format 0; the
    // dense images) or bf16 (format 1; the hierarchical images), both K-major,
    // N (bits 17-22, N/8), M = 128 (bits 24-28, M/16)
    static constexpr uint32_t idesc(int n, bool bf16)
    {
        return (1u << 4) | (bf16 ? (1u << 7) | (1u << 10) : 0u) | ((uint32_t)(n >> 3) << 17) |
               ((uint32_t)(BM >> 4) << 24);
    }
    static constexpr uint32_t IDESC = idesc(NI, false);
    static constexpr uint32_t IDESC2 = idesc(2 * NI, false);
    static constexpr uint32_t IDESC_BF = idesc(NI, true);
    static constexpr uint32_t IDESC2_BF = idesc(2 * NI, true);
    // KDRAIN: every k-block's products go into a fresh accumulator that the
    // drain warps add, in FP32 with round-to-nearest, into per-thread register
    // sums (MT NI of them).  The tensor core's own FP32 accumulation truncates
    // at every addition; over a whole segment (hundreds of k-blocks) that bias
    // grows with the segment length and sits in every stage rate, where the
    // embedded error estimate cannot tell it from truncation error and shrinks
    // the step.  Drained per k-block it covers 4 MMAs only.  Off where the
    // register sums would not fit (128 instances x 2 M-tiles).
    static constexpr bool KDRAIN = true;
    static constexpr int NCOL = MT == 2 ? NI : NI / 2;   // register sums per drain thread
    static constexpr bool TWO_LEVEL = NCOL <= 32;          // FP32 over FOLD k-blocks, then FP64
    static constexpr int FOLD = 8;
    static_assert(MERGE, "the drain adds the hi and 2^-11 halves of a merged accumulator");
};

// byte offset of element (r, k) in a 128-byte-swizzled tile image with 128-byte rows
__host__ __device__ __forceinline__ uint32_t sw128(int r, int k)
{
    return (uint32_t)r * 128u + ((((uint32_t)(k >> 3) ^ (uint32_t)(r & 7)) << 4) | ((uint32_t)(k & 7) << 1));
}

// per-instance integrator control (the single-instance Ctl, one per instance)
struct InstCtl {
    double h, time, dt_next, hdid, vmax;
    unsigned long long errbits;
    long long accepted, rejected;
    int need_stage1, pending, status, active, nonfinite, in_event;
    double t_event;             // start time of the first step with max V >= the event threshold
    long long n_events;         // threshold up-crossings
    // step-size model inputs (mlp.cuh)
    double hist[8];             // last accepted steps, most recent first
    unsigned long long thmin_key;   // min log10 theta at the start of the step (ordered key)
    int nhist, first_attempt, has_feat, pad2;
    float feat[mlp::NIN];       // inputs at the last acceptance (for the trace of the next first attempt)
};

struct EnsGlobal {
    double t_end, epsilon, hmax;
    long long attempts;         // attempts of the current launch
    long long budget;           // attempt limit of the current launch
    long long total_attempts;
    double ev_on, ev_off;       // event thresholds on max V (m/s)
    int active_count;
    int err;                    // UCG_E_TIMEOUT from the contraction
    // step-size model and trace recording
    const __half *mlp_P;
    const mlp::Norm *mlp_N;
    float *trace;               // records of TRACE_LEN floats
    unsigned long long trace_cap, trace_n;
    // fault injection for tests of the bounded waits (ucg_ens_test_wait_timeout):
    // wait_ns != 0 replaces the 4 s limit of the dense contraction's data waits;
    // test_hold makes the CTA owning the first segment issue no copies
    unsigned long long wait_ns;
    int test_hold;
    int inc_full;               // stages 2-6 contracted in the anchor's three-term form
};

// one trace record: the 11 model inputs at an acceptance, then log10 of the
// next step's first attempt and log10 max(errmax, 1e-12) of that attempt, and
// 1 if it was accepted
constexpr int TRACE_LEN = mlp::NIN + 3;

struct GeomDev {
    int np, ninst, mtiles, kblocks;
    int tile0;                  // unit id of tile (nt = 0, mt = 0) in the single-tile plan
    int pair0, mpairs;          // unit id of pair (nt = 0, 0) in the paired plan; pairs per instance tile
    int blk_e0, epb_e;          // element-wise grid: first block, blocks per instance
    int blk_s0, epb_s;          // state-wise grid
    uint8_t *B;                 // V images [ntile][kblock][hi | lo]
    float *vscale;              // dense: V image scale per [ntile][kblock][instance of the tile]
    const float *rscale;        // per K row (mtiles * 128)
    double *y, *ys, *k[6], *ycand, *yerr, *yscal;           // [ninst][7 np]
    double *v1, *t1;            // stage-1 anchor: [ninst][2 np] velocities, [ninst][3 np] tractions
    const double *vpl_c, *vpl_s, *a, *b, *sig, *L, *damping; // [ninst][np]
    InstCtl *ctl;               // [ninst]
    // hierarchical K (hier != 0): B is the B space of the hierarchical contraction
    int hier, hleaves, hunit0, hpl;    // hpl: bf16 planes of the hierarchical images (2 or 3)
    size_t hbtile;              // bytes of one instance tile's B space
    const int *hperm;           // permuted position -> element
    const int *hinv;            // element -> permuted position
    const int2 *hrow;           // permuted position -> (row leaf, local row of its first component)
    const int *hxpos;           // element -> B-space slot of its first source column
};

struct EnsArgs {
    int ngeom, ni, blocks_e, blocks_s;
    GeomDev g[MAX_GEOM];
    const float *ws1, *ws2;     // partial sums: [slot][ni][128] (single tiles), [slot][2][ni][128] (pairs)
    const int *piece0_1, *npieces_1, *piece0_2, *npieces_2;
    EnsGlobal *glob;
    // hierarchical pass 2: per unit its first piece, pieces and partial-sum rows;
    // per piece the float offset of its partial sums
    const float *hws2;
    const int *hp0, *hnp, *hrows;
    const long *hpws;
};

// a work unit: one M-tile, or two consecutive M-tiles of a geometry (a1 null when
// the geometry's last tile has no partner)
struct GemmTile {
    const uint8_t *a;           // K images of k-block 0 of the (first) M-tile
    const uint8_t *a1;          // the second M-tile's, or null
    const uint8_t *b;           // V images of k-block 0 of this instance tile
    const float *ks, *ks1;      // K image scale per k-block of the (first, second) M-tile
    const float *vs;            // V image scales of k-block 0 of this instance tile ([kblock][ni])
};
struct GemmSeg {
    int tile, kb0, kb1, slot;
};

// ---- PTX helpers ------------------------------------------------------------------

__device__ __forceinline__ uint32_t s_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint64_t *b, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_addr(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(s_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bar_arrive(uint64_t *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s_addr(b)) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(s_addr(b)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// bounded wait; abort == nullptr waits out the deadline regardless of other threads
__device__ __forceinline__ bool bar_wait(uint64_t *b, uint32_t parity, volatile int *abort,
                                         unsigned long long limit = TIMEOUT_NS)
{
    if (bar_try(b, parity)) return true;
    const unsigned long long t0 = now_ns();
    for (unsigned it = 1;; it++) {
        if (bar_try(b, parity)) return true;
        if ((it & 127u) == 0u) {
            if (abort && *abort) return false;
            if (now_ns() - t0 > limit) return false;
        }
    }
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *b)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(s_addr(dst)), "l"(src), "r"(bytes), "r"(s_addr(b)) : "memory");
}
// the same with an L2 eviction priority: operand images stream through once
// (evict first); the instances' values are read by many tiles (evict last)
__device__ __forceinline__ uint64_t l2_policy(bool keep)
{
    uint64_t p;
    if (keep)
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    else
        asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void bulk_load_hint(void *dst, const void *src, uint32_t bytes, uint64_t *b, uint64_t pol)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
                 ::"r"(s_addr(dst)), "l"(src), "r"(bytes), "r"(s_addr(b)), "l"(pol) : "memory");
}
// shared-memory matrix descriptor: K-major operand, 128-byte swizzle, 8-row
// groups 1024 bytes apart (SBO), descriptor version 1
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
           ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                 " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t *b)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(s_addr(b))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t r[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t r[16])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld8_async(uint32_t taddr, uint32_t r[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- the contraction ---------------------------------------------------------------

template <int NI, bool KLO, int MT>
__global__ void __launch_bounds__(320, 1) k_bf16x3_contract(const GemmTile *__restrict__ tiles,
        const GemmSeg *__restrict__ segs, const int *__restrict__ cta_seg, float *__restrict__ ws, EnsGlobal *gl)
{
    int *err = &gl->err;
    const unsigned long long lim = gl->wait_ns ? gl->wait_ns : TIMEOUT_NS;
    // (test_hold: the CTA that owns the first segment issues no copies, its MMA
    // issuer's wait runs out; a small plan leaves some CTAs without segments)
    const bool hold = gl->test_hold && cta_seg[blockIdx.x] == 0 && cta_seg[blockIdx.x + 1] > 0;
    using T = Tile<NI, KLO, MT>;
    extern __shared__ unsigned char dyn_smem[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dyn_smem) + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full[T::STAGES], empty[T::STAGES], acc_full[T::NACC], acc_empty[T::NACC],
        drain;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = cta_seg[blockIdx.x], q1 = cta_seg[blockIdx.x + 1];

    if (threadIdx.x == 0) {
        for (int s = 0; s < T::STAGES; s++) {
            bar_init(&full[s], 1);
            bar_init(&empty[s], 1);
        }
        for (int b = 0; b < T::NACC; b++) {
            bar_init(&acc_full[b], 1);
            bar_init(&acc_empty[b], 8);   // both drain warpgroups
        }
        bar_init(&drain, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_addr(&tmem_slot)),
                     "r"(T::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    auto fail = [&]() {
        abort_flag = 1;
        atomicExch(err, (int)UCG_E_TIMEOUT);
    };

    if (warp == 0) {
        if (lane == 0) {
            // producer: per k-block one copy of K per M-tile of the unit and one copy of V
            const uint64_t pol_a = l2_policy(false), pol_b = l2_policy(true);
            long issued = 0;
            // the next segments' descriptors are loaded ahead (segment two
            // ahead, its tile one ahead), off the copy issue's critical path
            GemmSeg s1 = q0 < q1 ? segs[q0] : GemmSeg{0, 0, 0, 0};
            GemmSeg s2 = q0 + 1 < q1 ? segs[q0 + 1] : s1;
            GemmTile t1 = q0 < q1 ? tiles[s1.tile] : GemmTile{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
            for (int q = q0; q < q1 && !abort_flag && !hold; q++) {
                const GemmSeg sg = s1;
                const GemmTile tl = t1;
                s1 = s2;
                if (q + 1 < q1) t1 = tiles[s1.tile];
                if (q + 2 < q1) s2 = segs[q + 2];
                const bool two = MT == 2 && tl.a1 != nullptr;
                const uint32_t bytes = (uint32_t)((two ? 2 : 1) * T::A_BYTES + T::B_IMG);
                for (int kb = sg.kb0; kb < sg.kb1; kb++) {
                    const int s = (int)(issued % T::STAGES);
                    const uint32_t ph = (uint32_t)((issued / T::STAGES) & 1);
                    if (!bar_wait(&empty[s], ph ^ 1u, &abort_flag, lim)) {
                        if (!abort_flag) fail();
                        break;
                    }
                    uint8_t *st = smem + (size_t)s * T::STAGE;
                    bar_expect_tx(&full[s], bytes);
                    bulk_load_hint(st, tl.a + (size_t)kb * A_IMG, T::A_BYTES, &full[s], pol_a);
                    if (two) bulk_load_hint(st + T::A_BYTES, tl.a1 + (size_t)kb * A_IMG, T::A_BYTES, &full[s], pol_a);
                    bulk_load_hint(st + MT * T::A_BYTES, tl.b + (size_t)kb * T::B_IMG, T::B_IMG, &full[s], pol_b);
                    issued++;
                }
            }
            // the last copy into each stage has landed before the CTA may exit
            for (long i = issued - T::STAGES > 0 ? issued - T::STAGES : 0; i < issued; i++)
                bar_wait(&full[i % T::STAGES], (uint32_t)((i / T::STAGES) & 1), nullptr);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            long it = 0;
            int tc = 0;
            bool issued_any = false;
            for (int q = q0; q < q1 && !abort_flag; q++, tc++) {
                const GemmSeg sg = segs[q];
                const int nt = (MT == 2 && tiles[sg.tile].a1 != nullptr) ? 2 : 1;
                int buf = tc % T::NACC;
                uint32_t use = (uint32_t)(tc / T::NACC);
                if (!T::KDRAIN) {
                    if (!bar_wait(&acc_empty[buf], (use & 1u) ^ 1u, &abort_flag, lim)) {
                        if (!abort_flag) fail();
                        break;
                    }
                    tc_fence_after();
                }
                bool ok = true;
                for (int kb = sg.kb0; kb < sg.kb1; kb++, it++) {
                    if (T::KDRAIN) {
                        // one accumulator per k-block, taking the NACC sets in turn
                        buf = (int)(it % T::NACC);
                        use = (uint32_t)(it / T::NACC);
                        if (!bar_wait(&acc_empty[buf], (use & 1u) ^ 1u, &abort_flag, lim)) {
                            if (!abort_flag) fail();
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                    }
                    const int s = (int)(it % T::STAGES);
                    const uint32_t ph = (uint32_t)((it / T::STAGES) & 1);
                    if (!bar_wait(&full[s], ph, &abort_flag, lim)) {
                        if (!abort_flag) fail();
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a = s_addr(smem + (size_t)s * T::STAGE);
                    const uint32_t b = a + MT * T::A_BYTES;
#pragma unroll
                    for (int j = 0; j < BK / 16; j++) {
                        const uint64_t bhi = sw128_desc(b + 32u * j), blo = sw128_desc(b + T::B_HALF + 32u * j);
                        const uint32_t acc = ((!T::KDRAIN && kb > sg.kb0) || j > 0) ? 1u : 0u;
#pragma unroll
                        for (int u = 0; u < MT; u++) {
                            if (u < nt) {
                                const uint32_t d = tmem + (uint32_t)((buf * MT + u) * T::ACC_N);
                                const uint32_t au = a + (uint32_t)(u * T::A_BYTES);
                                const uint64_t ahi = sw128_desc(au + 32u * j);
                                if (T::MERGE) {
                                    // rows 0..NI-1 of the B operand are Vhi, NI..2NI-1 Vlo:
                                    // columns 0..NI-1 take Khi Vhi, NI..2NI-1 the products
                                    // that carry 2^-11 (Khi Vlo, and in the anchor Klo Vhi)
                                    mma_bf16(d, ahi, bhi, T::IDESC2, acc);
                                    if (KLO)
                                        mma_bf16(d + (uint32_t)NI, sw128_desc(au + A_HALF + 32u * j), bhi, T::IDESC,
                                                 1u);
                                } else {
                                    mma_bf16(d, ahi, bhi, T::IDESC, acc);
                                    mma_bf16(d, ahi, blo, T::IDESC, 1u);
                                    if (KLO) mma_bf16(d, sw128_desc(au + A_HALF + 32u * j), bhi, T::IDESC, 1u);
                                }
                            }
                        }
                    }
                    issued_any = true;
                    mma_commit(&empty[s]);   // frees the stage once these MMAs have read it
                    if (T::KDRAIN) mma_commit(&acc_full[buf]);
                }
                if (!ok) break;
                if (!T::KDRAIN) mma_commit(&acc_full[buf]);
            }
            // no MMA may be in flight when the tensor memory is released
            if (issued_any) {
                mma_commit(&drain);
                bar_wait(&drain, 0u, nullptr);
            }
        }
        __syncwarp();
    } else {
        // drain per k-block, two warpgroups (warps 2-5 and 6-9): warp w reads
        // tensor-memory lanes 32 (w mod 4) .. +31 (tile rows); with two M-tiles a
        // group takes one tile, with one M-tile half of its instance columns.
        // Every k-block's partial sums (hi products + 2^-11 lo products, times
        // the K block and V block scales) are added in FP64 registers; a
        // segment's sums go to the workspace when its last k-block is in
        const int quarter = warp & 3;
        const int grp = (warp - 2) >> 2;
        const int row = quarter * 32 + lane;
        constexpr int NC = T::NCOL;                   // columns per thread
        const int u = (MT == 2) ? grp : 0;            // the M-tile this group drains
        const int cbase = (MT == 2) ? 0 : grp * NC;   // its first instance column
        long it = 0;
        bool ok = true;
        for (int q = q0; q < q1 && ok; q++) {
            const GemmSeg sg = segs[q];
            const int nt = (MT == 2 && tiles[sg.tile].a1 != nullptr) ? 2 : 1;
            const bool mine = u < nt;                 // a pair's missing second tile: wait and release only
            // FP32 sums over up to FOLD k-blocks, folded into FP64 sums (with one
            // M-tile per group; the two-tile increments keep FP32 sums, their K
            // hi truncation dominates)
            float part[NC];
            double sum[T::TWO_LEVEL ? NC : 1];
#pragma unroll
            for (int c = 0; c < NC; c++) part[c] = 0.0f;
#pragma unroll
            for (int c = 0; c < (T::TWO_LEVEL ? NC : 1); c++) sum[c] = 0.0;
            const GemmTile tl = tiles[sg.tile];
            // the k-block's scales: the tile's K block scale and, per lane, the V
            // block scale of its instance columns cbase + lane + 32 j, loaded one
            // k-block ahead and multiplied only when used (a product formed at
            // the load would wait out the L2 latency in every k-block once the
            // drain is the busy side), the lane's product broadcast to the warp
            // by shuffles
            constexpr int NL = (NC + 31) / 32;       // instance columns per lane
            const float *ksu = u == 0 ? tl.ks : tl.ks1;
            float nk = 0.0f, nv[NL];
            auto load_scales = [&](int k) {
                nk = ksu[k];
#pragma unroll
                for (int j = 0; j < NL; j++)
                    nv[j] = (32 * j + lane < NC) ? __ldg(tl.vs + (size_t)k * NI + cbase + 32 * j + lane) : 0.0f;
            };
#pragma unroll
            for (int j = 0; j < NL; j++) nv[j] = 0.0f;
            if (mine && sg.kb0 < sg.kb1) load_scales(sg.kb0);
            for (int kb = sg.kb0; kb < sg.kb1; kb++, it++) {
                const int buf = (int)(it % T::NACC);
                const uint32_t use = (uint32_t)(it / T::NACC);
                float skv[NL];
#pragma unroll
                for (int j = 0; j < NL; j++) skv[j] = nk * nv[j];
                if (mine && kb + 1 < sg.kb1) load_scales(kb + 1);
                int got = 0;
                if (lane == 0) got = bar_wait(&acc_full[buf], use & 1u, &abort_flag, lim) ? 1 : 0;
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    if (lane == 0 && !abort_flag) fail();
                    ok = false;
                    break;
                }
                tc_fence_after();
                // the accumulator goes back to the MMA issuer as soon as the last
                // batch of its columns is in registers, before that batch is added
                auto release = [&]() {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) bar_arrive(&acc_empty[buf]);
                };
                if (mine) {
                    const uint32_t tbase = tmem + (uint32_t)((buf * MT + u) * T::ACC_N + cbase) +
                                           ((uint32_t)(quarter * 32) << 16);
                    constexpr int LB = NC < 32 ? NC : 32;     // columns per batch of loads
#pragma unroll
                    for (int c0 = 0; c0 < NC; c0 += LB) {
                        uint32_t r[LB], r2[LB];
#pragma unroll
                        for (int c = 0; c < LB; c += 8) {
                            tmem_ld8_async(tbase + (uint32_t)(c0 + c), r + c);
                            tmem_ld8_async(tbase + (uint32_t)(c0 + c + NI), r2 + c);
                        }
                        tmem_wait_ld();
                        if (c0 + LB >= NC) release();
#pragma unroll
                        for (int i = 0; i < LB; i++) {
                            // hi products + 2^-11 lo products, times the block scales (powers of
                            // two: exact)
                            const int c = c0 + i;
                            const float sc = __shfl_sync(0xffffffffu, skv[c >> 5], c & 31);
                            const float x = __fmaf_rn(__uint_as_float(r2[i]), LO_UNSCALE, __uint_as_float(r[i]));
                            part[c] = __fmaf_rn(x, sc, part[c]);
                        }
                    }
                    if (T::TWO_LEVEL && ((kb - sg.kb0) % T::FOLD == T::FOLD - 1 || kb == sg.kb1 - 1)) {
#pragma unroll
                        for (int c = 0; c < NC; c++) {
                            sum[T::TWO_LEVEL ? c : 0] += (double)part[c];
                            part[c] = 0.0f;
                        }
                    }
                } else {
                    release();
                }
            }
            if (!ok) break;
            if (mine) {
                float *dst = ws + ((size_t)sg.slot * MT + u) * NI * BM + (size_t)cbase * BM + row;
#pragma unroll
                for (int c = 0; c < NC; c++)
                    dst[(size_t)c * BM] = T::TWO_LEVEL ? (float)sum[T::TWO_LEVEL ? c : 0] : part[c];
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::TMEM_COLS)
                     : "memory");
    }
}

// ---- the hierarchical contraction -------------------------------------------------------
//
// T = H V for a hierarchical K (hmatrix.cu) in two passes of one kernel:
//   pass 1: Z = Vs X for every stack Vs of the low-rank blocks that share a source
//           cluster (their V factors stacked, each block's rank rounded up to 8
//           with zero rows), over the cluster's source columns;
//   pass 2: T_leaf = [dense | U] [X ; Z] for every row leaf, over the leaf's
//           dense blocks' source columns and its low-rank blocks' rank entries.
// Operands are stored in the K-major core-matrix layout without swizzle: a
// K-group is 8 consecutive K entries (16 bytes of bf16), an 8-row group of one
// K-group is one 128-byte core matrix, and an image is [K-group][row group] per
// plane (hi, then lo, or hi, mid, lo).  Granularity 8 along K lets a row leaf's K range
// concatenate pieces of any length multiple of 8 (leaf columns, ranks) and the
// B operand of every K-group be fetched from wherever its instances' values
// live (X: the permuted sources; Z: pass 1's output), merged into one bulk copy
// per run of consecutive K-groups.  Rows of a unit beyond its 8-row groups are
// read by the 128-row MMA from the stage's own buffer and land in accumulator
// lanes that are never drained.
constexpr int HSUB_KG3 = 8;                  // three planes: K-groups per fresh accumulator (64 entries)
constexpr int HKG_STAGE = 8;                  // K-groups per stage (four K-steps of 16); see HTile::KG

// tensor-memory columns of a hierarchical CTA: two accumulators of two NI-column
// parts (every plane count), a power of two as tcgen05.alloc takes
constexpr int hm_cols(int ni, int) { return 4 * ni; }
// CTAs per SM: two when their tensor memory fits the SM's 512 columns; two
// independent pipelines per SM hide the per-stage issue latency that bounds
// one (measured: 20 % less time per launch)
constexpr int hm_ctas(int ni, int pl) { return 2 * hm_cols(ni, pl) <= 512 ? 2 : 1; }

// PL planes of bf16 per operand value: 2 (hi, lo: 16 significant bits) or 3
// (hi, mid, lo: 24 bits, an FP32 value exactly)
template <int NI, bool KLO, int PL>
struct HTile {
    static_assert(PL == 2 || (PL == 3 && KLO && NI <= 64), "planes");
    static constexpr int B_KG = PL * NI * 16;             // every plane of one K-group for NI instances
    static constexpr int CTAS = hm_ctas(NI, PL);
    static constexpr int BUDGET = CTAS == 2 ? 104 * 1024 : 208 * 1024;
    // two rings: the operand images stream from HBM and need many bytes in
    // flight; the B K-groups come from L2 and need few
    // K-groups per stage: 8, or 16 for the increments (hi planes) of a lone
    // CTA: fewer, larger stages where the stage is cheap and room allows; 4
    // for three planes in two CTAs
    static constexpr int KG = (PL == 3 && CTAS == 2) ? HKG_STAGE / 2 : (KLO || CTAS == 2) ? HKG_STAGE : 2 * HKG_STAGE;
    static constexpr int A_PLANE = KG * 16 * 128;          // one plane of a stage for 16 row groups
    static constexpr int A_STAGE = KLO ? PL * A_PLANE : A_PLANE;
    static constexpr int B_STAGE = KG * B_KG;
    static constexpr int SB_FIT = (BUDGET - A_STAGE) / B_STAGE;
    static constexpr int SB_CAP = (KLO && (CTAS == 2 || PL == 3)) ? 2 : 3;
    static constexpr int SB = SB_FIT < SB_CAP ? SB_FIT : SB_CAP;
    static constexpr int SA_FIT = (BUDGET - SB * B_STAGE) / A_STAGE;
    static constexpr int SA = SA_FIT < 12 ? SA_FIT : 12;
    static constexpr int SMEM = SA * A_STAGE + SB * B_STAGE + 1024;   // + 1024 for the alignment
    static_assert(SA >= 2 && SB >= 1 && SMEM * CTAS <= 227 * 1024, "hierarchical contraction rings");
    // an accumulator has two NI-column parts, which the drain adds.  Two
    // planes: one MMA of N = 2 NI per K-step reads the hi and lo planes of the
    // B K-groups together (consecutive 8-row groups): Ahi [Bhi; Blo], then Alo
    // Bhi into part 0.  Three planes: the six products of weight 2^-16 and above
    // (the three left out are below 2^-24 of the value), Ahi [Bhi; Bmid] with
    // N = 2 NI, then Ahi Blo, Amid Bhi, Amid Bmid and Alo Bhi into part 1, so
    // that part 0 takes one tensor-core addition per K-step and part 1, 2^-8 of
    // it, keeps the small products to 2^-31 of the value
    static constexpr int ACC = 2 * NI;                     // columns of one accumulator
    // three planes: a fresh accumulator every SUB_KG K-groups (64 entries),
    // which the drain adds into FP32 register sums with round-to-nearest; the
    // tensor core's own accumulation truncates at each K-step, a bias that
    // grows with the run (two planes: one accumulator per segment, their
    // 16-bit images outweigh it)
    static constexpr int SUB_KG = PL == 3 ? HSUB_KG3 : 0;
    static_assert(SUB_KG == 0 || (SUB_KG % KG == 0 && SUB_KG % 2 == 0), "sub-segments of whole stages");
    static constexpr uint32_t TMEM_COLS = hm_cols(NI, PL);
    static constexpr uint32_t IDESC = Tile<NI, false, 1>::idesc(NI, true);
    static constexpr uint32_t IDESC2 = Tile<NI, false, 1>::idesc(2 * NI, true);
};

struct HUnit {                  // one M-tile of one pass for one instance tile
    const uint8_t *a;           // hi planes [K-group][g][128 B]; the lo planes follow at a + lo_off
    long lo_off;
    const int *bidx;            // per K-group: its K-group in the instance tile's B space
    const uint8_t *b;           // the instance tile's B space: [K-group][hi | lo][NI / 8][128 B]
    const int *zdst;            // pass 1: per 8-row group, its Z K-group in the B space
    int g, nkg;                 // 8-row groups (1..16), K-groups (even)
    int rows;                   // rows of its partial sums (8 g)
    int pad;
};
struct HSeg {
    int unit, kg0, kg1;         // K-groups [kg0, kg1), both even
    int direct;                 // pass 1, the unit's only segment: Z straight into the B space
    long ws;                    // float offset of its partial sums [NI][rows] (not direct)
};

// shared-memory descriptor of a K-major operand without swizzle: K-groups `lbo`
// bytes apart, 8-row groups `sbo` bytes apart, descriptor version 1
__device__ __forceinline__ uint64_t cm_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1u << 46);
}

template <int NI, bool KLO, int PL>
__global__ void __launch_bounds__(224, hm_ctas(NI, PL)) k_hm_contract(const HUnit *__restrict__ units,
        const HSeg *__restrict__ segs, const int *__restrict__ cta_seg, float *__restrict__ ws, int *err)
{
    // warp 0: operand-image producer; warp 1: MMA issue; warps 2-5: drain
    // (tensor-memory lane quarter = warp mod 4); warp 6: B producer.  Both
    // producers walk the same sequence of stages (segments in order, KG
    // K-groups at a time), each into its own ring.
    using T = HTile<NI, KLO, PL>;
    extern __shared__ unsigned char dyn_smem[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(dyn_smem) + 1023) & ~(uintptr_t)1023);
    uint8_t *bring = smem + (size_t)T::SA * T::A_STAGE;
    __shared__ __align__(8) uint64_t fullA[T::SA], emptyA[T::SA], fullB[T::SB], emptyB[T::SB], acc_full[2],
        acc_empty[2], drain;
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q0 = cta_seg[blockIdx.x], q1 = cta_seg[blockIdx.x + 1];

    if (threadIdx.x == 0) {
        for (int s = 0; s < T::SA; s++) {
            bar_init(&fullA[s], 1);
            bar_init(&emptyA[s], 1);
        }
        for (int s = 0; s < T::SB; s++) {
            bar_init(&fullB[s], 1);
            bar_init(&emptyB[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            bar_init(&acc_full[b], 1);
            bar_init(&acc_empty[b], 4);
        }
        bar_init(&drain, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_addr(&tmem_slot)),
                     "r"(T::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    auto fail = [&]() {
        abort_flag = 1;
        atomicExch(err, (int)UCG_E_TIMEOUT);
    };

    if (warp == 0) {
        if (lane == 0) {
            // operand images: the unit's hi (and lo) planes of the stage's K-groups
            const uint64_t pol_a = l2_policy(false);
            long issued = 0;
            // descriptors loaded ahead: the segment two ahead, its unit one ahead
            HSeg s1 = q0 < q1 ? segs[q0] : HSeg{0, 0, 0, 0, 0};
            HSeg s2 = q0 + 1 < q1 ? segs[q0 + 1] : s1;
            const uint8_t *a1 = nullptr;
            long lo1 = 0;
            int g1 = 1;
            if (q0 < q1) {
                a1 = units[s1.unit].a;
                lo1 = units[s1.unit].lo_off;
                g1 = units[s1.unit].g;
            }
            for (int q = q0; q < q1 && !abort_flag; q++) {
                const HSeg sg = s1;
                const uint8_t *ua = a1;
                const long ulo = lo1;
                const uint32_t plane = (uint32_t)g1 * 128u;
                s1 = s2;
                if (q + 1 < q1) {
                    a1 = units[s1.unit].a;
                    lo1 = units[s1.unit].lo_off;
                    g1 = units[s1.unit].g;
                }
                if (q + 2 < q1) s2 = segs[q + 2];
                bool ok = true;
                for (int kg = sg.kg0; kg < sg.kg1; kg += T::KG) {
                    const int nk = min(T::KG, sg.kg1 - kg);
                    const int s = (int)(issued % T::SA);
                    const uint32_t ph = (uint32_t)((issued / T::SA) & 1);
                    if (!bar_wait(&emptyA[s], ph ^ 1u, &abort_flag)) {
                        if (!abort_flag) fail();
                        ok = false;
                        break;
                    }
                    uint8_t *st = smem + (size_t)s * T::A_STAGE;
                    const uint32_t abytes = (uint32_t)nk * plane;
                    bar_expect_tx(&fullA[s], (KLO ? (uint32_t)PL : 1u) * abytes);
                    bulk_load_hint(st, ua + (size_t)kg * plane, abytes, &fullA[s], pol_a);
                    if (KLO)
#pragma unroll
                        for (int p = 1; p < PL; p++)
                            bulk_load_hint(st + p * T::A_PLANE, ua + p * ulo + (size_t)kg * plane, abytes, &fullA[s],
                                           pol_a);
                    issued++;
                }
                if (!ok) break;
            }
            for (long i = issued - T::SA > 0 ? issued - T::SA : 0; i < issued; i++)
                bar_wait(&fullA[i % T::SA], (uint32_t)((i / T::SA) & 1), nullptr);
        }
    } else if (warp == 6) {
        // B: the whole warp loads the B K-groups of 32 stages at once (lane l:
        // stage l); lane 0 takes each stage's from its lane by shuffle and
        // issues one copy per run of consecutive B K-groups
        const uint64_t pol_b = l2_policy(true);
        long issued = 0;
        bool stop = false;
        // descriptors loaded ahead: the segment two ahead, its unit one ahead
        HSeg s1 = q0 < q1 ? segs[q0] : HSeg{0, 0, 0, 0, 0};
        HSeg s2 = q0 + 1 < q1 ? segs[q0 + 1] : s1;
        const int *x1 = nullptr;
        const uint8_t *b1 = nullptr;
        if (q0 < q1) {
            x1 = units[s1.unit].bidx;
            b1 = units[s1.unit].b;
        }
        for (int q = q0; q < q1 && !stop; q++) {
            const HSeg sg = s1;
            const int *ubidx = x1;
            const uint8_t *ub = b1;
            s1 = s2;
            if (q + 1 < q1) {
                x1 = units[s1.unit].bidx;
                b1 = units[s1.unit].b;
            }
            if (q + 2 < q1) s2 = segs[q + 2];
            for (int kgb = sg.kg0; kgb < sg.kg1 && !stop; kgb += 32 * T::KG) {
                int my[T::KG];
                const int kgl = kgb + lane * T::KG;
#pragma unroll
                for (int j = 0; j < T::KG; j++) my[j] = kgl + j < sg.kg1 ? __ldg(ubidx + kgl + j) : 0;
                const int nst = min(32, (sg.kg1 - kgb + T::KG - 1) / T::KG);
                for (int t = 0; t < nst; t++) {
                    const int kg = kgb + t * T::KG;
                    const int nk = min(T::KG, sg.kg1 - kg);
                    int bi[T::KG];
#pragma unroll
                    for (int j = 0; j < T::KG; j++) bi[j] = __shfl_sync(0xffffffffu, my[j], t);
                    const int s = (int)(issued % T::SB);
                    const uint32_t ph = (uint32_t)((issued / T::SB) & 1);
                    int ok = 1;
                    if (lane == 0) ok = bar_wait(&emptyB[s], ph ^ 1u, &abort_flag) ? 1 : 0;
                    ok = __shfl_sync(0xffffffffu, ok, 0);
                    if (!ok) {
                        if (lane == 0 && !abort_flag) fail();
                        stop = true;
                        break;
                    }
                    if (lane == 0) {
                        uint8_t *bst = bring + (size_t)s * T::B_STAGE;
                        bar_expect_tx(&fullB[s], (uint32_t)nk * T::B_KG);
                        int rs = 0, bs = bi[0];
#pragma unroll
                        for (int j = 1; j <= T::KG; j++) {
                            if (j > nk) break;
                            const bool cont = j < T::KG && j < nk && bi[j] == bi[j - 1] + 1;
                            if (!cont) {
                                bulk_load_hint(bst + (size_t)rs * T::B_KG, ub + (size_t)bs * T::B_KG,
                                               (uint32_t)(j - rs) * T::B_KG, &fullB[s], pol_b);
                                if (j < T::KG && j < nk) {
                                    rs = j;
                                    bs = bi[j];
                                }
                            }
                        }
                    }
                    __syncwarp();
                    issued++;
                }
            }
        }
        if (lane == 0)
            for (long i = issued - T::SB > 0 ? issued - T::SB : 0; i < issued; i++)
                bar_wait(&fullB[i % T::SB], (uint32_t)((i / T::SB) & 1), nullptr);
    } else if (warp == 1) {
        if (lane == 0) {
            long it = 0;
            int tc = 0;
            bool issued_any = false;
            for (int q = q0; q < q1 && !abort_flag; q++) {
                const HSeg sg = segs[q];
                const uint32_t plane = (uint32_t)units[sg.unit].g * 128u;
                bool ok = true;
                const int span = T::SUB_KG ? T::SUB_KG : sg.kg1 - sg.kg0;
                for (int k0 = sg.kg0; k0 < sg.kg1 && ok; k0 += span, tc++) {
                    const int k1 = min(sg.kg1, k0 + span);
                    const int buf = tc & 1;
                    const uint32_t use = (uint32_t)(tc >> 1);
                    if (!bar_wait(&acc_empty[buf], (use & 1u) ^ 1u, &abort_flag)) {
                        if (!abort_flag) fail();
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)(buf * T::ACC);
                    for (int kg = k0; kg < k1; kg += T::KG, it++) {
                        const int nk = min(T::KG, sg.kg1 - kg);
                        const int sa = (int)(it % T::SA), sb = (int)(it % T::SB);
                        if (!bar_wait(&fullA[sa], (uint32_t)((it / T::SA) & 1), &abort_flag) ||
                            !bar_wait(&fullB[sb], (uint32_t)((it / T::SB) & 1), &abort_flag)) {
                            if (!abort_flag) fail();
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t a = s_addr(smem + (size_t)sa * T::A_STAGE);
                        const uint32_t b = s_addr(bring + (size_t)sb * T::B_STAGE);
                        for (int j = 0; j < nk / 2; j++) {
                            const uint32_t ao = (uint32_t)(2 * j) * plane, bo = (uint32_t)(2 * j) * T::B_KG;
                            const uint64_t ahi = cm_desc(a + ao, plane, 128u);
                            const uint64_t bhl = cm_desc(b + bo, T::B_KG, 128u);   // hi rows, then the other planes'
                            const uint32_t acc = (kg > k0 || j > 0) ? 1u : 0u;
                            mma_bf16(d, ahi, bhl, T::IDESC2, acc);
                            if (PL == 3) {
                                const uint32_t d1 = d + (uint32_t)NI;
                                const uint64_t amid = cm_desc(a + T::A_PLANE + ao, plane, 128u);
                                const uint64_t bmid = cm_desc(b + bo + NI * 16, T::B_KG, 128u);
                                mma_bf16(d1, ahi, cm_desc(b + bo + 2 * NI * 16, T::B_KG, 128u), T::IDESC, 1u);
                                mma_bf16(d1, amid, bhl, T::IDESC, 1u);
                                mma_bf16(d1, amid, bmid, T::IDESC, 1u);
                                mma_bf16(d1, cm_desc(a + 2 * T::A_PLANE + ao, plane, 128u), bhl, T::IDESC, 1u);
                            } else if (KLO) {
                                mma_bf16(d, cm_desc(a + T::A_PLANE + ao, plane, 128u), bhl, T::IDESC, 1u);
                            }
                        }
                        issued_any = true;
                        mma_commit(&emptyA[sa]);   // each frees its slot once these MMAs have read it
                        mma_commit(&emptyB[sb]);
                    }
                    if (!ok) break;
                    mma_commit(&acc_full[buf]);
                }
            }
            if (issued_any) {
                mma_commit(&drain);
                bar_wait(&drain, 0u, nullptr);
            }
        }
        __syncwarp();
    } else {
        // drain: warp w reads tensor-memory lanes 32 (w mod 4) .. +31 = unit rows;
        // rows past the unit's 8-row groups are not written
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        int tc = 0;
        if constexpr (T::SUB_KG == 0) {
            // two planes: one accumulator per segment
            for (int q = q0; q < q1; q++, tc++) {
                const HSeg sg = segs[q];
                const int rows = units[sg.unit].rows;
                const int buf = tc & 1;
                const uint32_t use = (uint32_t)(tc >> 1);
                int ok = 0;
                if (lane == 0) ok = bar_wait(&acc_full[buf], use & 1u, &abort_flag) ? 1 : 0;
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) {
                    if (lane == 0 && !abort_flag) fail();
                    break;
                }
                tc_fence_after();
                const uint32_t tbase = tmem + (uint32_t)(buf * T::ACC) + ((uint32_t)(quarter * 32) << 16);
                if (sg.direct) {
                    // the whole K range of a pass-1 unit: Z = the sum, split into
                    // bf16 hi and lo at its B-space slot (rank entry row, instance)
                    uint8_t *zb = nullptr;
                    if (row < rows) {
                        const HUnit &U = units[sg.unit];
                        zb = const_cast<uint8_t *>(U.b) + (size_t)U.zdst[row >> 3] * T::B_KG + (size_t)(row & 7) * 2;
                    }
#pragma unroll
                    for (int c0 = 0; c0 < NI; c0 += 16) {
                        uint32_t r[16], r2[16];
                        tmem_ld16(tbase + (uint32_t)c0, r);
                        tmem_ld16(tbase + (uint32_t)(c0 + NI), r2);
                        if (row < rows) {
#pragma unroll
                            for (int i = 0; i < 16; i++) {
                                const float z = __uint_as_float(r[i]) + __uint_as_float(r2[i]);
                                const __nv_bfloat16 h = __float2bfloat16_rn(z);
                                const __nv_bfloat16 l = __float2bfloat16_rn(z - __bfloat162float(h));
                                const int inst = c0 + i;
                                uint8_t *pz = zb + (size_t)(inst >> 3) * 128 + (size_t)(inst & 7) * 16;
                                *reinterpret_cast<__nv_bfloat16 *>(pz) = h;
                                *reinterpret_cast<__nv_bfloat16 *>(pz + NI * 16) = l;
                            }
                        }
                    }
                } else {
                    float *dst = ws + sg.ws + row;
#pragma unroll
                    for (int c0 = 0; c0 < NI; c0 += 16) {
                        uint32_t r[16], r2[16];
                        tmem_ld16(tbase + (uint32_t)c0, r);
                        tmem_ld16(tbase + (uint32_t)(c0 + NI), r2);
                        if (row < rows) {
#pragma unroll
                            for (int i = 0; i < 16; i++)
                                dst[(size_t)(c0 + i) * rows] = __uint_as_float(r[i]) + __uint_as_float(r2[i]);
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) bar_arrive(&acc_empty[buf]);
            }
        } else {
            // three planes: a fresh accumulator every SUB_KG K-groups, added
            // into FP32 register sums that the segment's end writes out
            for (int q = q0; q < q1; q++) {
                const HSeg sg = segs[q];
                const int rows = units[sg.unit].rows;
                // 16 instances' values of this row out: a pass-1 unit with its
                // whole K range writes Z, split into PL bf16 planes, at its B-space
                // slot (rank entry row, instance); the others their partial sums
                auto put16 = [&](int c0, const float *z) {
                    if (row >= rows) return;
                    if (sg.direct) {
                        const HUnit &U = units[sg.unit];
                        uint8_t *zb = const_cast<uint8_t *>(U.b) + (size_t)U.zdst[row >> 3] * T::B_KG + (size_t)(row & 7) * 2;
#pragma unroll
                        for (int i = 0; i < 16; i++) {
                            const int inst = c0 + i;
                            uint8_t *pz = zb + (size_t)(inst >> 3) * 128 + (size_t)(inst & 7) * 16;
                            float x = z[i];
#pragma unroll
                            for (int p = 0; p < PL; p++) {
                                // each plane the rest rounded to bf16 (the differences are exact)
                                const __nv_bfloat16 h = __float2bfloat16_rn(x);
                                *reinterpret_cast<__nv_bfloat16 *>(pz + (size_t)p * NI * 16) = h;
                                x = x - __bfloat162float(h);
                            }
                        }
                    } else {
                        float *dst = ws + sg.ws + row;
#pragma unroll
                        for (int i = 0; i < 16; i++) dst[(size_t)(c0 + i) * rows] = z[i];
                    }
                };
                const int span = T::SUB_KG ? T::SUB_KG : sg.kg1 - sg.kg0;
                const int nsub = span > 0 ? (sg.kg1 - sg.kg0 + span - 1) / span : 0;
                float sum[T::SUB_KG ? NI : 1];
#pragma unroll
                for (int c = 0; c < (T::SUB_KG ? NI : 1); c++) sum[c] = 0.0f;
                bool ok = true;
#pragma unroll 1
                for (int sub = 0; sub < nsub; sub++, tc++) {
                    const int buf = tc & 1;
                    const uint32_t use = (uint32_t)(tc >> 1);
                    int got = 0;
                    if (lane == 0) got = bar_wait(&acc_full[buf], use & 1u, &abort_flag) ? 1 : 0;
                    got = __shfl_sync(0xffffffffu, got, 0);
                    if (!got) {
                        if (lane == 0 && !abort_flag) fail();
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t tbase = tmem + (uint32_t)(buf * T::ACC) + ((uint32_t)(quarter * 32) << 16);
                    // the sum of the accumulator's PL parts for 16 instances, the
                    // small parts first
                    auto load16 = [&](int c0, float *z) {
                        uint32_t r[16], r2[16];
                        tmem_ld16(tbase + (uint32_t)c0, r);
                        tmem_ld16(tbase + (uint32_t)(c0 + NI), r2);
#pragma unroll
                        for (int i = 0; i < 16; i++) z[i] = __uint_as_float(r[i]) + __uint_as_float(r2[i]);
                    };
                    if constexpr (T::SUB_KG > 0) {
#pragma unroll
                        for (int c0 = 0; c0 < NI; c0 += 16) {
                            float z[16];
                            load16(c0, z);
#pragma unroll
                            for (int i = 0; i < 16; i++) sum[c0 + i] += z[i];
                        }
                    } else if (sg.direct) {
#pragma unroll
                        for (int c0 = 0; c0 < NI; c0 += 16) {
                            float z[16];
                            load16(c0, z);
                            put16(c0, z);
                        }
                    } else {
#pragma unroll
                        for (int c0 = 0; c0 < NI; c0 += 16) {
                            float z[16];
                            load16(c0, z);
                            put16(c0, z);
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) bar_arrive(&acc_empty[buf]);
                }
                if (!ok) break;
                if constexpr (T::SUB_KG > 0) {
#pragma unroll
                    for (int c0 = 0; c0 < NI; c0 += 16) put16(c0, sum + c0);
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::TMEM_COLS)
                     : "memory");
    }
}

// the bf16 planes of an FP64 value: each plane the rest rounded to nearest
// (the differences are exact in FP64)
template <int PL>
__device__ __forceinline__ void split_planes(double x, __nv_bfloat16 (&p)[PL])
{
#pragma unroll
    for (int j = 0; j < PL; j++) {
        p[j] = __double2bfloat16(x);
        x = x - (double)__bfloat162float(p[j]);
    }
}

// one K-group of an operand image from FP64 values: value(row r, slot k) =
// src[k][(r - row0) stride] for rows row0 .. row0 + nrows - 1, zero where src[k]
// is null; one thread per row writes its 16 bytes of every plane
struct HPackJob {
    uint8_t *dst;               // the K-group's hi plane; the next planes lo_off bytes apart
    long lo_off;
    long stride;
    int row0, nrows;
    const double *src[8];
};

template <int PL>
__global__ void k_hm_pack(const HPackJob *__restrict__ jobs)
{
    const HPackJob J = jobs[blockIdx.x];
    const int t = threadIdx.x;
    if (t >= J.nrows) return;
    const int r = J.row0 + t;
    uint32_t w[PL][4];
#pragma unroll
    for (int k = 0; k < 8; k += 2) {
        __nv_bfloat16 a[PL], b[PL];
        split_planes<PL>(J.src[k] ? J.src[k][(long)t * J.stride] : 0.0, a);
        split_planes<PL>(J.src[k + 1] ? J.src[k + 1][(long)t * J.stride] : 0.0, b);
#pragma unroll
        for (int p = 0; p < PL; p++)
            w[p][k / 2] = (uint32_t)__bfloat16_as_ushort(a[p]) | ((uint32_t)__bfloat16_as_ushort(b[p]) << 16);
    }
    uint8_t *q = J.dst + (size_t)(r >> 3) * 128 + (size_t)(r & 7) * 16;
#pragma unroll
    for (int p = 0; p < PL; p++)
        *reinterpret_cast<uint4 *>(q + p * J.lo_off) = make_uint4(w[p][0], w[p][1], w[p][2], w[p][3]);
}

// a B-space entry (instance rr of a tile, slot `pos` = 8 K-group + k, k even) and
// the next slot from two FP64 values, split into pl planes (2 or 3)
__device__ __forceinline__ void put_x(uint8_t *Bt, int ni, int pl, int rr, int pos, double v0, double v1)
{
    uint8_t *base = Bt + (size_t)(pos >> 3) * (pl * ni * 16) + (size_t)(rr >> 3) * 128 + (size_t)(rr & 7) * 16 +
                    (size_t)(pos & 7) * 2;
    __nv_bfloat16 a[3], b[3];
    if (pl == 3) {
        split_planes<3>(v0, a);
        split_planes<3>(v1, b);
    } else {
        __nv_bfloat16 a2[2], b2[2];
        split_planes<2>(v0, a2);
        split_planes<2>(v1, b2);
        a[0] = a2[0], a[1] = a2[1], b[0] = b2[0], b[1] = b2[1];
    }
    for (int p = 0; p < pl; p++)
        *reinterpret_cast<__nv_bfloat162 *>(base + (size_t)p * ni * 16) = __halves2bfloat162(a[p], b[p]);
}

// pass 1's output into the B space for the units cut into several pieces (the
// drain writes the others directly): one thread per (unit, 8-row group,
// instance) adds the unit's partial sums in k order (FP64) and writes 8 rank
// entries of Z as hi and lo
struct HZUnit {
    uint8_t *b;                 // the instance tile's B space
    const int *zdst;            // per 8-row group of the unit: its K-group in the B space
    int g, rows, p0, np, pad;
};

template <int PL>
__global__ void k_hm_zconv(const HZUnit *__restrict__ zu, const long *__restrict__ pws,
                           const float *__restrict__ ws, int ni)
{
    const HZUnit U = zu[blockIdx.x];
    for (int w = threadIdx.x; w < U.g * ni; w += blockDim.x) {
        const int grp = w / ni, i = w % ni;
        double z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int p = 0; p < U.np; p++) {
            const float4 *src = reinterpret_cast<const float4 *>(ws + pws[U.p0 + p] + (long)i * U.rows + grp * 8);
            const float4 a = src[0], b = src[1];
            z[0] += a.x; z[1] += a.y; z[2] += a.z; z[3] += a.w;
            z[4] += b.x; z[5] += b.y; z[6] += b.z; z[7] += b.w;
        }
        uint32_t wd[PL][4];
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
            __nv_bfloat16 a[PL], b[PL];
            split_planes<PL>(z[k], a);
            split_planes<PL>(z[k + 1], b);
#pragma unroll
            for (int p = 0; p < PL; p++)
                wd[p][k / 2] = (uint32_t)__bfloat16_as_ushort(a[p]) | ((uint32_t)__bfloat16_as_ushort(b[p]) << 16);
        }
        uint8_t *q = U.b + (size_t)U.zdst[grp] * (PL * ni * 16) + (size_t)(i >> 3) * 128 + (size_t)(i & 7) * 16;
#pragma unroll
        for (int p = 0; p < PL; p++)
            *reinterpret_cast<uint4 *>(q + (size_t)p * ni * 16) = make_uint4(wd[p][0], wd[p][1], wd[p][2], wd[p][3]);
    }
}

// ---- K images ----------------------------------------------------------------------

// power-of-two row scale >= max |K(r,:)| (1 for an all-zero row)
__global__ void k_row_scale(const double *__restrict__ K, long m, long n, long rows_pad, float *__restrict__ scale)
{
    const long r = blockIdx.x * (long)(blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows_pad) return;
    double mx = 0.0;
    if (r < m)
        for (long c = lane; c < n; c += 32) mx = fmax(mx, fabs(K[r * n + c]));
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (lane == 0) {
        float s = 1.0f;
        if (mx > 0.0) {
            int e;
            frexp(mx, &e);               // mx = f 2^e, 0.5 <= f < 1
            s = ldexpf(1.0f, e);         // s >= mx, |K/s| <= 1
        }
        scale[r] = s;
    }
}

// Dense operand images are fp16 pairs with one power-of-two scale per image
// block (a 128-row x 64-source K block, or the 64 sources of one instance's V
// k-block): x = s (hi + 2^-11 lo) with hi = fp16(x / s) and lo the rounded
// residual scaled by 2^11, so that it stays a normal fp16 number: 22
// significant bits for every entry above 2^-14 of its block's largest (an
// absolute 2^-25 of that below).  The MMAs run on the hi and lo images as
// they are; the drain applies 2^-11 to the lo products and the two block
// scales to every k-block's partial sums before adding them up.
__device__ __forceinline__ float pow2_at_least(double m)
{
    if (!(m > 0.0)) return 1.0f;
    int e;
    frexp(m, &e);                 // m = f 2^e, 0.5 <= f < 1
    return ldexpf(1.0f, e);       // >= m
}

__device__ __forceinline__ void split16(double x, __half &hi, __half &lo)
{
    hi = __double2half(x);
    lo = __double2half((x - (double)__half2float(hi)) * (double)LO_SCALE);
}

// the scale of one 128 x 64 block of K with its rows divided by their row
// scales (one CTA per block): rows far smaller than others of the same tile
// (a traction component that vanishes by symmetry) keep their own precision
__global__ void k_block_scale(const double *__restrict__ K, long m, long n, int kblocks,
                              const float *__restrict__ rscale, float *__restrict__ ks)
{
    const int mt = blockIdx.x / kblocks, kb = blockIdx.x % kblocks;
    double mx = 0.0;
    for (int t = threadIdx.x; t < BM * BK; t += blockDim.x) {
        const long r = (long)mt * BM + t / BK, c = (long)kb * BK + t % BK;
        if (r < m && c < n) mx = fmax(mx, fabs(K[r * n + c]) / (double)rscale[r]);
    }
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmax(t, wm[w]);
        ks[blockIdx.x] = pow2_at_least(t);
    }
}

// one thread per (row, 8 sources): 8 doubles in, 16 bytes of hi and of lo out
__global__ void k_pack_k(const double *__restrict__ K, long m, long n, int kblocks, long rows_pad,
                         const float *__restrict__ rscale, const float *__restrict__ ks, uint8_t *__restrict__ img)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long per_row = (long)kblocks * (BK / 8);
    if (t >= rows_pad * per_row) return;
    const long r = t / per_row;
    const int c8 = (int)(t % per_row);
    const int kb = c8 / (BK / 8), kk = (c8 % (BK / 8)) * 8;
    const long c0 = (long)kb * BK + kk;
    const long mt = r / BM;
    const double inv = 1.0 / ((double)rscale[r] * (double)ks[mt * kblocks + kb]);
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
        const double x0 = (r < m && c0 + j < n) ? K[r * n + c0 + j] * inv : 0.0;
        const double x1 = (r < m && c0 + j + 1 < n) ? K[r * n + c0 + j + 1] * inv : 0.0;
        __half h0, h1, l0, l1;
        split16(x0, h0, l0);
        split16(x1, h1, l1);
        hi[j / 2] = (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
        lo[j / 2] = (uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
    }
    const int rr = (int)(r % BM);
    uint8_t *base = img + ((size_t)mt * kblocks + kb) * A_IMG + sw128(rr, kk);
    *reinterpret_cast<uint4 *>(base) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    *reinterpret_cast<uint4 *>(base + A_HALF) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

// write the source pair (c, c+1), c even, of instance i into the V images with
// the scale s of its k-block
__device__ __forceinline__ void put_v(uint8_t *B, int ni, int kblocks, int i, long c, double v0, double v1, float s)
{
    const int nt = i / ni, rr = i % ni;
    const int kb = (int)(c / BK), kk = (int)(c % BK);
    const size_t bimg = (size_t)2 * ni * BK * 2;
    uint8_t *base = B + ((size_t)nt * kblocks + kb) * bimg + sw128(rr, kk);
    const double inv = 1.0 / (double)s;
    __half h0, h1, l0, l1;
    split16(v0 * inv, h0, l0);
    split16(v1 * inv, h1, l1);
    *reinterpret_cast<__half2 *>(base) = __halves2half2(h0, h1);
    *reinterpret_cast<__half2 *>(base + (size_t)ni * BK * 2) = __halves2half2(l0, l1);
}

// the k-block scale of 32 consecutive source pairs held by the lanes of a
// warp (lanes without a pair pass 0): the largest magnitude rounded up to a
// power of two, the same on every lane
__device__ __forceinline__ float warp_block_scale(double v0, double v1)
{
    double m = fmax(fabs(v0), fabs(v1));
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    return pow2_at_least(m);
}

// dense V (instance-major, ninst x n) into the images of one geometry: one warp
// per (instance, k-block), lane j the source pair j of the k-block
__global__ void k_pack_v_dense(uint8_t *B, float *vscale, int ni, int kblocks, int ninst, long n,
                               const double *__restrict__ V)
{
    const long w = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (long)ninst * kblocks) return;     // uniform over the warp
    const int i = (int)(w / kblocks), kb = (int)(w % kblocks);
    const long c = (long)kb * BK + 2 * lane;
    const double v0 = (c < n) ? V[(long)i * n + c] : 0.0;
    const double v1 = (c + 1 < n) ? V[(long)i * n + c + 1] : 0.0;
    const float s = warp_block_scale(v0, v1);
    if (lane == 0) vscale[((size_t)(i / ni) * kblocks + kb) * ni + i % ni] = s;
    put_v(B, ni, kblocks, i, c, v0, v1, s);
}

// row r of instance i from the partial sums, added in k order: `paired`
// selects the paired plan's workspace (stage increments) over the single-tile
// plan's (anchor)
__device__ __forceinline__ double traction_row(const EnsArgs *A, const GeomDev &G, int i, long r, bool paired)
{
    const int ni = A->ni;
    const int mt = (int)(r / BM), rr = (int)(r % BM);
    const float *w;
    int np_;
    size_t stride;
    if (paired) {
        const int unit = G.pair0 + (i / ni) * G.mpairs + mt / 2;
        const int p0 = A->piece0_2[unit];
        np_ = A->npieces_2[unit];
        w = A->ws2 + (((size_t)p0 * 2 + (mt & 1)) * ni + (i % ni)) * BM + rr;
        stride = (size_t)2 * ni * BM;
    } else {
        const int unit = G.tile0 + (i / ni) * G.mtiles + mt;
        const int p0 = A->piece0_1[unit];
        np_ = A->npieces_1[unit];
        w = A->ws1 + ((size_t)p0 * ni + (i % ni)) * BM + rr;
        stride = (size_t)ni * BM;
    }
    double s = 0.0;
    for (int p = 0; p < np_; p++) s += (double)w[(size_t)p * stride];
    return s * (double)G.rscale[r];
}

// row 3 p + q (permuted position p) of instance i for a hierarchical geometry:
// the pass-2 partial sums of its row leaf, added in k order
__device__ __forceinline__ double traction_row_h(const EnsArgs *A, const GeomDev &G, int i, int p, int q)
{
    const int2 rl = G.hrow[p];
    const int unit = G.hunit0 + (i / A->ni) * G.hleaves + rl.x;
    const int p0 = A->hp0[unit], np_ = A->hnp[unit];
    const long off = (long)(i % A->ni) * A->hrows[unit] + rl.y + q;
    double s = 0.0;
    for (int j = 0; j < np_; j++) s += (double)A->hws2[A->hpws[p0 + j] + off];
    return s;
}

// the three rows of a hierarchical geometry's element at permuted position p
// (local rows 3p' .. 3p' + 2 of its row leaf) for instance i: one lookup of the
// unit and its pieces for the three, each row's partial sums added in k order
// as traction_row_h does (measured: 20 % less time per right-hand side than a
// lookup per row; for the dense plan's rows it was 4 % slower)
__device__ __forceinline__ void traction_rows_h(const EnsArgs *A, const GeomDev &G, int i, int p, double inc[3])
{
    const int2 rl = G.hrow[p];
    const int unit = G.hunit0 + (i / A->ni) * G.hleaves + rl.x;
    const int p0 = A->hp0[unit], np_ = A->hnp[unit];
    const float *w = A->hws2 + (long)(i % A->ni) * A->hrows[unit] + rl.y;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < np_; j++) {
        const float *x = w + A->hpws[p0 + j];
        s0 += (double)x[0];
        s1 += (double)x[1];
        s2 += (double)x[2];
    }
    inc[0] = s0;
    inc[1] = s1;
    inc[2] = s2;
}

// T (instance-major, ninst x m, K's row order) of a hierarchical geometry
__global__ void k_reduce_h(const EnsArgs *A, int gi, double *T)
{
    const GeomDev &G = A->g[gi];
    const long m = 3L * G.np;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)G.ninst * m) return;
    const int i = (int)(t / m);
    const long r = t % m;
    T[t] = traction_row_h(A, G, i, G.hinv[r / 3], (int)(r % 3));
}

// dense V (instance-major, ninst x n) into a hierarchical geometry's X slots
__global__ void k_pack_x_dense(const EnsArgs *A, int gi, const double *__restrict__ V)
{
    const GeomDev &G = A->g[gi];
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)G.ninst * G.np) return;
    const int i = (int)(t / G.np), e = (int)(t % G.np);
    const double *v = V + (long)i * 2 * G.np + 2L * e;
    put_x(G.B + (size_t)(i / A->ni) * G.hbtile, A->ni, G.hpl, i % A->ni, G.hxpos[e], v[0], v[1]);
}

// T (instance-major, ninst x m) of geometry gi from the workspace
__global__ void k_reduce_dense(const EnsArgs *A, int gi, double *T, int paired)
{
    const GeomDev &G = A->g[gi];
    const long m = 3L * G.np;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)G.ninst * m) return;
    const int i = (int)(t / m);
    const long r = t % m;
    T[t] = traction_row(A, G, i, r, paired != 0);
}

// ---- Runge-Kutta stages for all instances --------------------------------------------

__device__ __constant__ double e_B[6][5] = {
    {0, 0, 0, 0, 0},
    {0.2, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
    {0.3, -0.9, 1.2, 0, 0},
    {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0},
    {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};

static const double E_LG10 = 2.302585092994045684017991454684364208;

__device__ __forceinline__ bool inst_live(const InstCtl *c, const EnsGlobal *g)
{
    return c->active && c->status == 0 && g->err == 0;
}

__device__ __forceinline__ int geom_of(const EnsArgs *A, int blk, bool state_grid)
{
    int gi = 0;
    while (gi + 1 < A->ngeom && blk >= (state_grid ? A->g[gi + 1].blk_s0 : A->g[gi + 1].blk_e0)) gi++;
    return gi;
}

template <int S>
__device__ __forceinline__ double ens_comb(const GeomDev &G, long i, double h)
{
    const double y = G.y[i];
    if (S == 1) return y;
    if (S == 2) return __dadd_rn(y, __dmul_rn(__dmul_rn(h, e_B[1][0]), G.k[0][i]));
    double r = __dmul_rn(e_B[S - 1][0], G.k[0][i]);
#pragma unroll
    for (int j = 1; j < S - 1; j++) r = __dadd_rn(r, __dmul_rn(e_B[S - 1][j], G.k[j][i]));
    return __dadd_rn(y, __dmul_rn(h, r));
}

// stage state, velocities and the V images (ratestate.f90:667-707 per instance).
// A block holds EW_THREADS consecutive elements of one instance, whose 7-double
// state tuples are one contiguous range: the stage state is formed over that
// range flat (coalesced), kept in shared memory, and each thread then takes its
// element's velocity from there.  The velocity components of the stage rate
// are written by k_ens_rhs with the rest of the tuple.
template <int S>
__global__ void __launch_bounds__(EW_THREADS) k_ens_prologue(const EnsArgs *__restrict__ A)
{
    __shared__ double sh[7 * EW_THREADS];
    const int gi = geom_of(A, blockIdx.x, false);
    const GeomDev &G = A->g[gi];
    const int local = blockIdx.x - G.blk_e0;
    const int i = local / G.epb_e;
    const int e0 = (local % G.epb_e) * EW_THREADS;
    if (i >= G.ninst) return;                        // uniform over the block
    const int ne = min(EW_THREADS, G.np - e0);
    const int e = e0 + threadIdx.x;
    const bool valid = threadIdx.x < ne;
    InstCtl *c = G.ctl + i;
    const bool pend = S == 1 && c->pending;
    const bool work = inst_live(c, A->glob) && !(S == 1 && !c->need_stage1);
    const double h = c->h;
    const long base = (long)i * 7 * G.np + 7L * e0;
#pragma unroll
    for (int u = 0; u < 7; u++) {
        const int f = threadIdx.x + u * EW_THREADS;
        if (f >= 7 * ne) break;
        const long x = base + f;
        double v = 0.0;
        if (S == 1) {
            v = pend ? G.ycand[x] : G.y[x];
            if (pend) G.y[x] = v;
        } else if (work) {
            v = ens_comb<S>(G, x, h);
            G.ys[x] = v;
            if (S == 2 && c->need_stage1) G.yscal[x] = fabs(G.y[x]) + fabs(h * G.k[0][x]) + 1.0e-30;
        }
        sh[f] = v;
    }
    __syncthreads();
    unsigned long long vkey = 0ull, tkey = ~0ull;   // max V and min log10 theta of this element (stage 1)
    double v0 = 0.0, v1 = 0.0;
    if (valid) {
        const double *yy = sh + 7 * threadIdx.x;
        if (work) {
            const double rake = atan2(yy[3], yy[2]);
            const double vel = exp(yy[6] * E_LG10);
            const double vs = vel * cos(rake), vd = vel * sin(rake);
            const long pe = (long)i * G.np + e;
            v0 = vs - G.vpl_c[pe];
            v1 = vd - G.vpl_s[pe];
            if (!isfinite(vel) || !isfinite(rake)) {
                c->nonfinite = 1;
                v0 = v1 = 0.0;
            }
            if (S == 1) {
                vkey = (unsigned long long)__double_as_longlong(vel);
                tkey = mlp::ord_key(yy[5]);
                G.v1[2 * pe] = v0;
                G.v1[2 * pe + 1] = v1;
            } else {
                // increment over the stage-1 anchor
                v0 = v0 - G.v1[2 * pe];
                v1 = v1 - G.v1[2 * pe + 1];
            }
        }
        if (G.hier) put_x(G.B + (size_t)(i / A->ni) * G.hbtile, A->ni, G.hpl, i % A->ni, G.hxpos[e], v0, v1);
    }
    if (!G.hier) {
        // a warp holds the 32 elements (64 sources) of one k-block: its scale,
        // then every element's pair of sources
        const float sv = warp_block_scale(v0, v1);
        const int ew = e0 + (threadIdx.x & ~31);          // the warp's first element
        if ((threadIdx.x & 31) == 0 && ew < G.np)
            G.vscale[((size_t)(i / A->ni) * G.kblocks + ew / 32) * A->ni + i % A->ni] = sv;
        if (valid) put_v(G.B, A->ni, G.kblocks, i, 2L * e, v0, v1, sv);
    }
    if (S == 1) {
        // the block's elements belong to one instance: reduce over the warp,
        // one atomic per warp (identity values on lanes past the last element)
        for (int off = 16; off > 0; off >>= 1) {
            vkey = max(vkey, __shfl_xor_sync(0xffffffffu, vkey, off));
            tkey = min(tkey, __shfl_xor_sync(0xffffffffu, tkey, off));
        }
        if ((threadIdx.x & 31) == 0) {
            if (vkey) atomicMax((unsigned long long *)&c->vmax, vkey);
            if (tkey != ~0ull) atomicMin(&c->thmin_key, tkey);
        }
    }
}

// the stage rate of one element (ratestate.f90:731-776) from its stage state
// yy (7 doubles) and traction t: all 7 components into k
__device__ __forceinline__ void ens_rate(const double *yy, const double t[3], double L, double bb, double sg,
                                         double aa, double eta, double *k)
{
    const double rake = atan2(yy[3], yy[2]);
    const double vel = exp(yy[6] * E_LG10);
    const double cr = cos(rake), sr = sin(rake);
    const double dth = (exp(-yy[5] * E_LG10) - vel / L) / E_LG10;
    const double dtau = t[0] * cr + t[1] * sr;
    const double dv = (dtau - bb * sg * dth * E_LG10) / (aa * sg + eta * vel) / E_LG10;
    const double corr = eta * vel * dv * E_LG10;
    k[0] = vel * cr;
    k[1] = vel * sr;
    k[2] = t[0] - corr * cr;
    k[3] = t[1] - corr * sr;
    k[4] = t[2];
    k[5] = dth;
    k[6] = dv;
}

// traction rates from the contraction and the rate-state right-hand side
// (ratestate.f90:731-776 per instance).  The block's contiguous state range and
// rate range go through shared memory (coalesced); a hierarchical geometry
// gathers each element's partial sums from the cluster order.
// 12 blocks per SM (40 registers, a few spilled): the kernel waits on memory,
// and more resident warps hide it better than fewer that spill nothing
// (measured at N = 20k x 64: 5.96 ms per attempt against 6.08 at 80 registers)
template <int S>
__global__ void __launch_bounds__(EW_THREADS, 12) k_ens_rhs(const EnsArgs *__restrict__ A)
{
    __shared__ double sh[7 * EW_THREADS];
    const int gi = geom_of(A, blockIdx.x, false);
    const GeomDev &G = A->g[gi];
    const int local = blockIdx.x - G.blk_e0;
    const int i = local / G.epb_e;
    const int e0 = (local % G.epb_e) * EW_THREADS;
    if (i >= G.ninst) return;                        // uniform over the block
    const InstCtl *c = G.ctl + i;
    if (!inst_live(c, A->glob) || (S == 1 && !c->need_stage1)) return;
    const int ne = min(EW_THREADS, G.np - e0);
    const int el = e0 + threadIdx.x;
    const bool valid = threadIdx.x < ne;
    const double *ysrc = (S == 1) ? G.y : G.ys;
    double *ks = G.k[S - 1];
    const long base = (long)i * 7 * G.np + 7L * e0;
#pragma unroll
    for (int u = 0; u < 7; u++) {
        const int f = threadIdx.x + u * EW_THREADS;
        if (f < 7 * ne) sh[f] = ysrc[base + f];
    }
    __syncthreads();
    if (valid) {
        const int e = el;
        double t[3];
        double *t1 = G.t1 + (long)i * 3 * G.np + 3L * e;
        // a hierarchical geometry's partial sums lie in the cluster order: the
        // element's permuted position finds them (a gather of a few floats per
        // row, while the state and the rate stay coalesced)
        double inc[3];
        if (G.hier) {
            traction_rows_h(A, G, i, G.hinv[e], inc);
        } else {
#pragma unroll
            for (int q = 0; q < 3; q++) inc[q] = traction_row(A, G, i, 3L * e + q, S > 1 && !A->glob->inc_full);
        }
#pragma unroll
        for (int q = 0; q < 3; q++) {
            if (S == 1) {
                t1[q] = inc[q];
                t[q] = inc[q];
            } else {
                t[q] = t1[q] + inc[q];
            }
        }
        const long pe = (long)i * G.np + e;
        double k[7];
        ens_rate(sh + 7 * threadIdx.x, t, G.L[pe], G.b[pe], G.sig[pe], G.a[pe], G.damping[pe], k);
        for (int q = 0; q < 7; q++) sh[7 * threadIdx.x + q] = k[q];   // each thread its own slots
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 7; u++) {
        const int f = threadIdx.x + u * EW_THREADS;
        if (f < 7 * ne) ks[base + f] = sh[f];
    }
}

#define E_C1 (37.0 / 378.0)
#define E_C3 (250.0 / 621.0)
#define E_C4 (125.0 / 594.0)
#define E_C6 (512.0 / 1771.0)
#define E_DC1 (E_C1 - 2825.0 / 27648.0)
#define E_DC3 (E_C3 - 18575.0 / 48384.0)
#define E_DC4 (E_C4 - 13525.0 / 55296.0)
#define E_DC5 (-277.0 / 14336.0)
#define E_DC6 (E_C6 - 0.25)

// candidate, error estimate and max |yerr/yscal| per instance (ode45.f90:184-200, 68-76)
__global__ void k_ens_finish(const EnsArgs *__restrict__ A)
{
    const int gi = geom_of(A, blockIdx.x, true);
    const GeomDev &G = A->g[gi];
    const int local = blockIdx.x - G.blk_s0;
    const int i = local / G.epb_s;
    if (i >= G.ninst) return;
    InstCtl *c = G.ctl + i;
    if (!inst_live(c, A->glob)) return;        // uniform over the block
    const long len = 7L * G.np;
    const long j0 = (long)(local % G.epb_s) * ST_SPAN + threadIdx.x;
    const double h = c->h;
    double mx = 0.0;
    bool bad = false;
#pragma unroll
    for (int u = 0; u < ST_PER; u++) {
        const long j = j0 + (long)u * ST_THREADS;
        if (j < len) {
            const long x = (long)i * len + j;
            const double k1 = G.k[0][x], k3 = G.k[2][x], k4 = G.k[3][x], k5 = G.k[4][x], k6 = G.k[5][x];
            double r = __dmul_rn(E_C1, k1);
            r = __dadd_rn(r, __dmul_rn(E_C3, k3));
            r = __dadd_rn(r, __dmul_rn(E_C4, k4));
            r = __dadd_rn(r, __dmul_rn(E_C6, k6));
            const double yc = __dadd_rn(G.y[x], __dmul_rn(h, r));
            double er = __dmul_rn(E_DC1, k1);
            er = __dadd_rn(er, __dmul_rn(E_DC3, k3));
            er = __dadd_rn(er, __dmul_rn(E_DC4, k4));
            er = __dadd_rn(er, __dmul_rn(E_DC5, k5));
            er = __dadd_rn(er, __dmul_rn(E_DC6, k6));
            er = __dmul_rn(h, er);
            G.ycand[x] = yc;
            G.yerr[x] = er;
            mx = fmax(mx, fabs(er / G.yscal[x]));
            bad = bad || !isfinite(yc);
        }
    }
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    bad = __any_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        if (mx > 0.0) atomicMax(&c->errbits, (unsigned long long)__double_as_longlong(mx));
        if (bad) c->nonfinite = 1;
    }
}

// RKQSm decision per instance (ode45.f90:77-106) and the loop condition.  With a
// step-size model, the instances that accepted in this attempt are collected per
// chunk of blockDim.x instances and each warp evaluates the model for one of
// them (weights read from global memory).
constexpr int CTL_THREADS = 512;    // 16 warps: up to 16 model evaluations in one round

__global__ void __launch_bounds__(CTL_THREADS) k_ens_control(const EnsArgs *__restrict__ A,
                                                               cudaGraphConditionalHandle cond, int in_graph)
{
    EnsGlobal *gl = A->glob;
    const double SAFETY = 0.7, PGROW = -0.2, PSHRNK = -0.15, ERRCON = 1.89e-4;
    __shared__ mlp::Norm norm;
    __shared__ float feat[CTL_THREADS][mlp::NIN];
    __shared__ InstCtl *who[CTL_THREADS];
    __shared__ int nwho;
    __shared__ int wsum[CTL_THREADS / 32];
    // the model's weights are read where they are (global memory, cached): a copy
    // into shared memory at every launch costs more than the few evaluations
    // of one attempt read
    const bool model = gl->mlp_P != nullptr;
    const __half *wt = gl->mlp_P;
    if (model && threadIdx.x == 0) norm = *gl->mlp_N;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int live = 0;
    for (int gi = 0; gi < A->ngeom; gi++) {
        const GeomDev &G = A->g[gi];
        for (int base = 0; base < G.ninst; base += blockDim.x) {
            if (threadIdx.x == 0) nwho = 0;
            __syncthreads();
            const int i = base + threadIdx.x;
            InstCtl *c = i < G.ninst ? G.ctl + i : nullptr;
            if (c && inst_live(c, gl)) {
                double errmax = __longlong_as_double((long long)c->errbits);
                c->errbits = 0ull;
                if (c->nonfinite) {
                    c->status = UCG_E_NONFINITE;
                    c->active = 0;
                } else {
                    errmax = errmax / gl->epsilon;
                    double h = c->h;
                    if (gl->trace && c->first_attempt && c->has_feat) {
                        const unsigned long long k = atomicAdd(&gl->trace_n, 1ull);
                        if (k < gl->trace_cap) {
                            float *rec = gl->trace + k * TRACE_LEN;
                            for (int q = 0; q < mlp::NIN; q++) rec[q] = c->feat[q];
                            rec[mlp::NIN] = (float)log10(h);
                            rec[mlp::NIN + 1] = (float)log10(fmax(errmax, 1e-12));
                            rec[mlp::NIN + 2] = errmax > 1.0 ? 0.0f : 1.0f;
                        }
                    }
                    c->first_attempt = 0;
                    if (errmax > 1.0) {
                        h = h * SAFETY * pow(errmax, PSHRNK);
                        if (h < 0.5 * h) h = 0.5 * h;
                        c->h = h;
                        c->rejected += 1;
                        c->need_stage1 = 0;
                        c->pending = 0;
                        if (0.0 + h == 0.0) {
                            c->status = UCG_E_STEP_UNDERFLOW;
                            c->active = 0;
                        } else {
                            live++;
                        }
                    } else {
                        double hnext;
                        if (errmax > ERRCON) hnext = SAFETY * h * pow(errmax, PGROW);
                        else hnext = 10.0 * h;
                        if (hnext > gl->hmax) hnext = gl->hmax;
                        // inputs of the step-size model at this acceptance
                        for (int q = 7; q > 0; q--) c->hist[q] = c->hist[q - 1];
                        c->hist[0] = h;
                        c->nhist = c->nhist < 8 ? c->nhist + 1 : 8;
                        c->has_feat = c->nhist >= 8;
                        if (c->has_feat) {
                            mlp::features(c->vmax, mlp::ord_val(c->thmin_key), c->hist, errmax, c->feat);
                            if (model) {
                                const int k = atomicAdd(&nwho, 1);
                                who[k] = c;
                                for (int q = 0; q < mlp::NIN; q++) feat[k][q] = c->feat[q];
                            }
                        }
                        c->first_attempt = 1;
                        c->thmin_key = ~0ull;
                        // event catalogue: max V at the start of this step against the thresholds
                        if (!c->in_event && c->vmax >= gl->ev_on) {
                            c->in_event = 1;
                            if (c->n_events == 0) c->t_event = c->time;
                            c->n_events += 1;
                        } else if (c->in_event && c->vmax < gl->ev_off) {
                            c->in_event = 0;
                        }
                        c->hdid = h;
                        c->time = c->time + h;
                        c->dt_next = hnext;
                        c->h = hnext;
                        c->accepted += 1;
                        c->pending = 1;
                        c->vmax = 0.0;
                        c->need_stage1 = 1;
                        if (c->time >= gl->t_end) c->active = 0;
                        else live++;
                    }
                }
            }
            __syncthreads();
            // the model's proposals for this chunk's acceptances: one warp each
            for (int k = warp; k < nwho; k += nwarps) {
                float x[mlp::NIN];
                for (int q = 0; q < mlp::NIN; q++) x[q] = feat[k][q];
                const float lp = mlp::eval_warp(wt, norm, x);
                if ((threadIdx.x & 31) == 0) {
                    InstCtl *c = who[k];
                    const double h = c->hdid;
                    double hn = fmin(fmax(pow(10.0, (double)lp), 0.2 * h), 10.0 * h);
                    if (hn > gl->hmax) hn = gl->hmax;
                    c->h = hn;
                    c->dt_next = hn;
                }
            }
            __syncthreads();
        }
    }
    for (int off = 16; off > 0; off >>= 1) live += __shfl_xor_sync(0xffffffffu, live, off);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = live;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += wsum[w];
        gl->active_count = tot;
        gl->attempts += 1;
        gl->total_attempts += 1;
        const bool more = tot > 0 && gl->attempts < gl->budget && gl->err == 0;
        if (in_graph) cudaGraphSetConditional(cond, more ? 1u : 0u);
    }
}

// start of a launch: activate every healthy instance short of t_end
__global__ void k_ens_begin(const EnsArgs *__restrict__ A)
{
    EnsGlobal *gl = A->glob;
    for (int gi = 0; gi < A->ngeom; gi++) {
        const GeomDev &G = A->g[gi];
        for (int i = threadIdx.x; i < G.ninst; i += blockDim.x) {
            InstCtl *c = G.ctl + i;
            c->active = (c->status == 0 && c->time < gl->t_end) ? 1 : 0;
        }
    }
    if (threadIdx.x == 0) gl->attempts = 0;
}

// end of a launch: copy accepted candidates that no later attempt committed
__global__ void k_ens_commit(const EnsArgs *__restrict__ A)
{
    const int gi = geom_of(A, blockIdx.x, true);
    const GeomDev &G = A->g[gi];
    const int local = blockIdx.x - G.blk_s0;
    const int i = local / G.epb_s;
    if (i >= G.ninst || !G.ctl[i].pending) return;
    const long len = 7L * G.np;
    const long j0 = (long)(local % G.epb_s) * ST_SPAN + threadIdx.x;
#pragma unroll
    for (int u = 0; u < ST_PER; u++) {
        const long j = j0 + (long)u * ST_THREADS;
        if (j < len) G.y[(long)i * len + j] = G.ycand[(long)i * len + j];
    }
}

// ucg_ens_put_states: the staged states (in the candidate vector, unused
// between launches) replace the instances' states; an instance whose state
// changed in any bit re-evaluates f(y) and yscal at its next attempt, one
// handed back the state it had keeps its stage-1 rate, as the device-resident
// loop would
__global__ void k_ens_put(double *__restrict__ y, const double *__restrict__ staged, InstCtl *__restrict__ ctl,
                          long len, long total)
{
    for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < total; j += (long)gridDim.x * blockDim.x) {
        const double v = staged[j];
        if (__double_as_longlong(v) != __double_as_longlong(y[j])) {
            y[j] = v;
            ctl[j / len].need_stage1 = 1;
        }
    }
}

__global__ void k_ens_clear_pending(const EnsArgs *__restrict__ A)
{
    for (int gi = 0; gi < A->ngeom; gi++) {
        const GeomDev &G = A->g[gi];
        for (int i = threadIdx.x; i < G.ninst; i += blockDim.x) G.ctl[i].pending = 0;
    }
}

}  // namespace ens
}  // namespace ucg

// ======================================================================================
// host side
// ======================================================================================

using namespace ucg;
using namespace ucg::ens;

struct EnsGeomHost {
    int np = 0, ninst = 0, mtiles = 0, kblocks = 0;
    long m = 0, n = 0;
    uint8_t *A = nullptr;      // K images
    float *rscale = nullptr;
    float *kscale = nullptr;   // dense: K image scale per [mtile][kblock]
    float *vscale = nullptr;   // dense: V image scale per [ntile][kblock][ni]
    double *state = nullptr;   // 12 vectors of ninst * 7 np
    double *anchor = nullptr;  // v1 (ninst * 2 np) then t1 (ninst * 3 np)
    double *par = nullptr;     // 7 vectors of ninst * np
    InstCtl *ctl = nullptr;
    uint8_t *B = nullptr;      // V images (B space of a hierarchical geometry) for the current ni
    int b_ni = 0;
    // hierarchical K: operand images of both passes and the maps of the B space
    bool hier = false;
    int hpl = 2;               // bf16 planes of its images and B space
    struct HU {                // a unit of one pass, without its instance tile
        long a_off, lo_off, bidx_off;
        long zdst_off;         // pass 1: offset of its 8-row groups' Z destinations
        int g, nkg;
    };
    std::vector<HU> hu1, hu2;  // pass 1 (tiles of the rank stacks), pass 2 (row leaves)
    uint8_t *hA = nullptr;
    int *hbidx = nullptr, *hperm = nullptr, *hinv = nullptr, *hxpos = nullptr, *hzdst = nullptr;
    int2 *hrow = nullptr;
    int nbkg = 0, hleaves = 0;
    size_t h_img_bytes = 0, h_fp64_bytes = 0;
    long h_kg1 = 0, h_kg2 = 0;  // K-groups of the two passes (one instance tile)
};

struct HPlanBufs {
    HUnit *units = nullptr;
    HSeg *segs = nullptr;
    int *cta = nullptr;
    float *ws = nullptr;
    long *pws = nullptr;       // per piece: float offset of its partial sums
    int *p0 = nullptr, *np = nullptr, *rows = nullptr;   // per unit
    HZUnit *zu = nullptr;      // pass 1: the units cut into several pieces, their Z destinations
    int nunits = 0, nsegs = 0, nzu = 0;
    size_t ws_floats = 0;
};

struct PlanBufs {
    GemmTile *tiles = nullptr;
    GemmSeg *segs = nullptr;
    int *cta = nullptr;
    int *piece0 = nullptr, *npieces = nullptr;
    float *ws = nullptr;
    int nunits = 0, nsegs = 0, nslots = 0;
    std::string name;
};

struct ucg_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sms = 148;
    std::string err;
    std::vector<EnsGeomHost> geoms;
    double epsilon = 1.0e-6, hmax = 1.7976931348623158e308;

    // plan: instance tile width and two schedules with their workspaces: single
    // M-tiles for the anchor's contraction, pairs of M-tiles for the increments'
    int ni = 0;
    bool planned = false;
    std::string plan_name;
    PlanBufs p1, p2;
    HPlanBufs h1, h2;          // hierarchical geometries: pass 1 and pass 2
    std::string tune_report;

    EnsArgs *d_args = nullptr;
    EnsGlobal *d_glob = nullptr;
    EnsGlobal *h_glob = nullptr;   // pinned
    cudaGraphExec_t graph = nullptr;
    bool use_graph = true;     // false: attempts launched one by one from the host
    bool inc_full = true;      // stage increments: three-term form (Khi Vhi + Khi Vlo + Klo Vhi)
    int hplanes = 3;           // bf16 planes of the hierarchical geometries' images (2 or 3)
    long launches = 0;
};

namespace {

int efail(ucg_ensemble *E, cudaError_t e, const char *what)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    E->err = buf;
    return e == cudaErrorMemoryAllocation ? UCG_E_OOM : UCG_E_CUDA;
}
#define ECUDA(call)                                             \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return efail(E, e_, #call);      \
    } while (0)

int ebad(ucg_ensemble *E, int st, const char *msg)
{
    E->err = msg;
    return st;
}

// ---- hierarchical geometries --------------------------------------------------------------
//
// The B space of one instance tile holds, K-group after K-group: X (every row
// leaf's source columns in the permuted order, each leaf's columns rounded up
// to 8), Z (every low-rank block's rank entries rounded up to 8, the blocks
// ordered by their receiver cluster, so that the blocks over one row leaf form
// one run per level of the cluster tree) and one K-group of zeros that pads a
// unit's K range to an even number of K-groups.  A row leaf's K-groups are
// ordered by their place in the B space, which merges its B copies into few
// long runs.

// operand images, B-space maps and unit templates of a hierarchical geometry
int build_hgeom(ucg_ensemble *E, const ucg::HLayout &L, EnsGeomHost &g)
{
    const int np = L.np, NL = L.n_leaves;
    std::vector<int> xkg0(NL + 1, 0), leaf_of_pos(np), kg_leaf;
    for (int l = 0; l < NL; l++) {
        const int sz = L.leaf_e0[l + 1] - L.leaf_e0[l];
        if (3 * sz > BM)
            return ebad(E, UCG_E_UNSUPPORTED,
                        "hierarchical ensemble: row leaves of at most 42 patches (build the matrix with leaf <= 42)");
        xkg0[l + 1] = xkg0[l] + (2 * sz + 7) / 8;
        for (int p = L.leaf_e0[l]; p < L.leaf_e0[l + 1]; p++) leaf_of_pos[p] = l;
        for (int q = xkg0[l]; q < xkg0[l + 1]; q++) kg_leaf.push_back(l);
    }
    const int nx = xkg0[NL];
    // rank stacks: the low-rank blocks of one source cluster, in block order
    std::map<std::pair<int, int>, std::vector<int>> stacks;
    for (int b = 0; b < (int)L.lr.size(); b++)
        if (L.lr[b].k > 0) stacks[{L.lr[b].s0, L.lr[b].n}].push_back(b);
    std::vector<int> zkg_b(L.lr.size(), -1);
    auto pad8 = [](int k) { return (k + 7) & ~7; };
    int zk = nx;
    {
        std::vector<int> order;
        for (int b = 0; b < (int)L.lr.size(); b++)
            if (L.lr[b].k > 0) order.push_back(b);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return L.lr[x].r0 != L.lr[y].r0 ? L.lr[x].r0 < L.lr[y].r0 : L.lr[x].m > L.lr[y].m;
        });
        for (int b : order) {
            zkg_b[b] = zk;
            zk += pad8(L.lr[b].k) / 8;
        }
    }
    std::vector<int> zdst;
    std::vector<HPackJob> jobs;
    std::vector<long> dst_off;   // per job: byte offset of its K-group in the images
    std::vector<int> bidx;
    long a_off = 0;
    // pass 1
    for (const auto &st : stacks) {
        const int s0 = st.first.first, n = st.first.second;
        const int ne = n / 2;
        const int l0 = leaf_of_pos[s0], l1 = leaf_of_pos[s0 + ne - 1];
        if (L.leaf_e0[l0] != s0 || L.leaf_e0[l1 + 1] != s0 + ne)
            return ebad(E, UCG_E_STATE, "hierarchical matrix: a source cluster is not a union of leaves");
        const int kx0 = xkg0[l0], nk = xkg0[l1 + 1] - kx0, nke = nk + (nk & 1);
        std::vector<int> rowoff;
        int R = 0;
        std::vector<int> grp_dst;   // per 8-row group of the stack: its Z K-group
        for (int b : st.second) {
            rowoff.push_back(R);
            for (int r = 0; r < pad8(L.lr[b].k); r += 8) grp_dst.push_back(zkg_b[b] + r / 8);
            R += pad8(L.lr[b].k);
        }
        for (int t0 = 0; t0 < R; t0 += 128) {
            const int rows_t = std::min(128, R - t0), gg = rows_t / 8;
            EnsGeomHost::HU u;
            u.a_off = a_off;
            u.lo_off = (long)nke * gg * 128;
            u.bidx_off = (long)bidx.size();
            u.g = gg;
            u.nkg = nke;
            u.zdst_off = (long)zdst.size();
            for (int q = 0; q < gg; q++) zdst.push_back(grp_dst[t0 / 8 + q]);
            for (int j = 0; j < nk; j++) bidx.push_back(kx0 + j);
            if (nk & 1) bidx.push_back(-1);   // the zero K-group, resolved below
            for (size_t bi = 0; bi < st.second.size(); bi++) {
                const int b = st.second[bi];
                const ucg::HLayout::LowRank &B = L.lr[b];
                const int rb = std::max(rowoff[bi], t0), re = std::min(rowoff[bi] + B.k, t0 + rows_t);
                if (re <= rb) continue;
                const int lbeg = rb - rowoff[bi];
                for (int j = 0; j < nk; j++) {
                    HPackJob J;
                    J.dst = nullptr;
                    dst_off.push_back(a_off + (long)j * gg * 128);
                    J.lo_off = u.lo_off;
                    J.stride = B.n;
                    J.row0 = rb - t0;
                    J.nrows = re - rb;
                    const int lf = kg_leaf[kx0 + j];
                    for (int k = 0; k < 8; k++) {
                        const int lc = 8 * (kx0 + j - xkg0[lf]) + k;
                        const int sz = L.leaf_e0[lf + 1] - L.leaf_e0[lf];
                        J.src[k] = nullptr;
                        if (lc < 2 * sz) {
                            const int c = 2 * L.leaf_e0[lf] + lc - 2 * s0;
                            J.src[k] = B.V + (long)lbeg * B.n + c;
                        }
                    }
                    jobs.push_back(J);
                }
            }
            a_off += g.hpl * u.lo_off;
            g.hu1.push_back(u);
            g.h_kg1 += nke;
        }
    }
    const int zero_kg = zk;
    g.nbkg = zk + 1;
    // pass 2
    std::vector<int> seen(g.nbkg, -1);
    for (int l = 0; l < NL; l++) {
        const int rows = 3 * (L.leaf_e0[l + 1] - L.leaf_e0[l]), gg = (rows + 7) / 8;
        std::vector<int> kgs;                       // B K-groups in order of first use
        std::vector<std::array<const double *, 8>> src;
        for (int q = L.leaf_term0[l]; q < L.leaf_term0[l + 1]; q++) {
            const ucg::HLayout::Term &T = L.terms[q];
            for (int j = 0; j < T.cols; j++) {
                int bkg, slot;
                if (T.xsel == 0) {
                    const long col = T.xoff + j;
                    const int p = (int)(col / 2), lf = leaf_of_pos[p];
                    const int lc = (int)(col - 2L * L.leaf_e0[lf]);
                    bkg = xkg0[lf] + lc / 8;
                    slot = lc % 8;
                } else {
                    const long zi = T.xoff + j;
                    int lo = 0, hi = (int)L.lr.size() - 1;   // the block with zoff <= zi < zoff + k
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) / 2;
                        if (L.lr[mid].zoff <= zi) lo = mid; else hi = mid - 1;
                    }
                    const int r = (int)(zi - L.lr[lo].zoff);
                    if (zkg_b[lo] < 0 || r >= L.lr[lo].k)
                        return ebad(E, UCG_E_STATE, "hierarchical matrix: a rank entry has no block");
                    bkg = zkg_b[lo] + r / 8;
                    slot = r % 8;
                }
                if (seen[bkg] != l) {
                    seen[bkg] = l;
                    kgs.push_back(bkg);
                    src.emplace_back();
                    src.back().fill(nullptr);
                }
                // the K-group was appended when first met; later columns of a
                // term continue the same or the next K-group
                int a = (int)kgs.size() - 1;
                if (kgs[a] != bkg) {
                    a = -1;
                    for (int x = (int)kgs.size() - 1; x >= 0; x--)
                        if (kgs[x] == bkg) { a = x; break; }
                }
                src[a][slot] = L.panel + T.poff + (long)j * rows;
            }
        }
        const int nk = (int)kgs.size(), nke = nk + (nk & 1);
        // the leaf's K-groups in B-space order: consecutive B K-groups become
        // one copy (the sum's order is fixed by this, so results stay deterministic)
        std::vector<int> ord(nk);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](int x, int y) { return kgs[x] < kgs[y]; });
        EnsGeomHost::HU u;
        u.a_off = a_off;
        u.lo_off = (long)nke * gg * 128;
        u.bidx_off = (long)bidx.size();
        u.g = gg;
        u.nkg = nke;
        u.zdst_off = -1;
        for (int j = 0; j < nk; j++) {
            bidx.push_back(kgs[ord[j]]);
            HPackJob J;
            J.dst = nullptr;
            dst_off.push_back(a_off + (long)j * gg * 128);
            J.lo_off = u.lo_off;
            J.stride = 1;
            J.row0 = 0;
            J.nrows = rows;
            for (int k = 0; k < 8; k++) J.src[k] = src[ord[j]][k];
            jobs.push_back(J);
        }
        if (nk & 1) bidx.push_back(zero_kg);
        a_off += g.hpl * u.lo_off;
        g.hu2.push_back(u);
        g.h_kg2 += nke;
    }
    for (int &b : bidx)
        if (b < 0) b = zero_kg;
    g.hleaves = NL;
    g.h_img_bytes = (size_t)a_off;
    // device images and maps
    std::vector<int> inv(np), xpos(np);
    std::vector<int2> hrow(np);
    for (int p = 0; p < np; p++) {
        const int e = L.perm[p], lf = leaf_of_pos[p];
        inv[e] = p;
        hrow[p] = make_int2(lf, 3 * (p - L.leaf_e0[lf]));
        xpos[e] = 8 * xkg0[lf] + 2 * (p - L.leaf_e0[lf]);
    }
    ECUDA(cudaMalloc(&g.hA, std::max<size_t>(g.h_img_bytes, 256)));
    ECUDA(cudaMemsetAsync(g.hA, 0, std::max<size_t>(g.h_img_bytes, 256), E->stream));
    ECUDA(cudaMalloc(&g.hbidx, sizeof(int) * std::max<size_t>(bidx.size(), 1)));
    ECUDA(cudaMalloc(&g.hzdst, sizeof(int) * std::max<size_t>(zdst.size(), 1)));
    if (!zdst.empty())
        ECUDA(cudaMemcpyAsync(g.hzdst, zdst.data(), sizeof(int) * zdst.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMalloc(&g.hperm, sizeof(int) * np));
    ECUDA(cudaMalloc(&g.hinv, sizeof(int) * np));
    ECUDA(cudaMalloc(&g.hxpos, sizeof(int) * np));
    ECUDA(cudaMalloc(&g.hrow, sizeof(int2) * np));
    if (!bidx.empty())
        ECUDA(cudaMemcpyAsync(g.hbidx, bidx.data(), sizeof(int) * bidx.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(g.hperm, L.perm.data(), sizeof(int) * np, cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(g.hinv, inv.data(), sizeof(int) * np, cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(g.hxpos, xpos.data(), sizeof(int) * np, cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(g.hrow, hrow.data(), sizeof(int2) * np, cudaMemcpyHostToDevice, E->stream));
    // the pack jobs, in batches
    const size_t BATCH = 1 << 18;
    HPackJob *jd = nullptr;
    ECUDA(cudaMalloc(&jd, sizeof(HPackJob) * std::min(BATCH, std::max<size_t>(jobs.size(), 1))));
    for (size_t j0 = 0; j0 < jobs.size(); j0 += BATCH) {
        const size_t nb = std::min(BATCH, jobs.size() - j0);
        for (size_t j = j0; j < j0 + nb; j++) jobs[j].dst = g.hA + dst_off[j];
        cudaError_t e = cudaMemcpyAsync(jd, jobs.data() + j0, sizeof(HPackJob) * nb, cudaMemcpyHostToDevice, E->stream);
        if (e == cudaSuccess) {
            if (g.hpl == 3)
                k_hm_pack<3><<<(unsigned)nb, 128, 0, E->stream>>>(jd);
            else
                k_hm_pack<2><<<(unsigned)nb, 128, 0, E->stream>>>(jd);
            E->launches++;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);   // the job buffer is reused
        if (e != cudaSuccess) {
            cudaFree(jd);
            return efail(E, e, "hierarchical operand images");
        }
    }
    cudaFree(jd);
    g.hier = true;
    return UCG_OK;
}

// ---- schedules ------------------------------------------------------------------------

struct Sched {
    std::vector<GemmSeg> segs;
    std::vector<int> cta;        // P + 1 offsets into segs
    std::vector<int> piece0, npieces;
    int nslots = 0;
    std::string name;
};

// number the partial sums of each tile in k order
void number_pieces(Sched &s, int ntiles)
{
    std::vector<std::vector<int>> per(ntiles);
    for (int q = 0; q < (int)s.segs.size(); q++) per[s.segs[q].tile].push_back(q);
    s.piece0.assign(ntiles, 0);
    s.npieces.assign(ntiles, 0);
    int slot = 0;
    for (int t = 0; t < ntiles; t++) {
        std::sort(per[t].begin(), per[t].end(), [&](int x, int y) { return s.segs[x].kb0 < s.segs[y].kb0; });
        s.piece0[t] = slot;
        s.npieces[t] = (int)per[t].size();
        for (int q : per[t]) s.segs[q].slot = slot++;
    }
    s.nslots = slot;
}

// stream-K: the (tile, k-block) sequence cut into P equal contiguous ranges
Sched sched_stream_k(const std::vector<int> &tkb, int P)
{
    Sched s;
    s.name = "stream-k";
    const int nt = (int)tkb.size();
    std::vector<long> pre(nt + 1, 0);
    for (int t = 0; t < nt; t++) pre[t + 1] = pre[t] + tkb[t];
    const long W = pre[nt];
    s.cta.assign(P + 1, 0);
    int t = 0;
    for (int c = 0; c < P; c++) {
        const long lo = W * c / P, hi = W * (c + 1) / P;
        s.cta[c] = (int)s.segs.size();
        while (t < nt && pre[t + 1] <= lo) t++;
        for (int u = t; u < nt && pre[u] < hi; u++) {
            const long a = std::max(lo, pre[u]) - pre[u], b = std::min(hi, pre[u + 1]) - pre[u];
            if (b > a) s.segs.push_back(GemmSeg{u, (int)a, (int)b, 0});
        }
    }
    s.cta[P] = (int)s.segs.size();
    number_pieces(s, nt);
    return s;
}

// split-K with chunks of about `chunk` k-blocks, longest-first onto the least
// loaded CTA (each segment also costs `ovh` k-blocks of drain and pipeline fill)
Sched sched_split_lpt(const std::vector<int> &tkb, int P, int chunk, int ovh)
{
    Sched s;
    s.name = chunk > 0 ? "split-k" + std::to_string(chunk) + "+lpt" : "tiles+lpt";
    struct Unit { int tile, kb0, kb1; };
    std::vector<Unit> units;
    for (int t = 0; t < (int)tkb.size(); t++) {
        const int parts = chunk > 0 ? std::max(1, (tkb[t] + chunk - 1) / chunk) : 1;
        for (int j = 0; j < parts; j++) {
            const int a = (int)((long)tkb[t] * j / parts), b = (int)((long)tkb[t] * (j + 1) / parts);
            if (b > a) units.push_back(Unit{t, a, b});
        }
    }
    std::stable_sort(units.begin(), units.end(),
                     [](const Unit &x, const Unit &y) { return (x.kb1 - x.kb0) > (y.kb1 - y.kb0); });
    using Load = std::pair<long, int>;
    std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
    for (int c = 0; c < P; c++) heap.push(Load(0, c));
    std::vector<std::vector<Unit>> per(P);
    for (const Unit &u : units) {
        Load l = heap.top();
        heap.pop();
        per[l.second].push_back(u);
        l.first += (u.kb1 - u.kb0) + ovh;
        heap.push(l);
    }
    s.cta.assign(P + 1, 0);
    for (int c = 0; c < P; c++) {
        std::sort(per[c].begin(), per[c].end(),
                  [](const Unit &x, const Unit &y) { return x.tile != y.tile ? x.tile < y.tile : x.kb0 < y.kb0; });
        s.cta[c] = (int)s.segs.size();
        for (const Unit &u : per[c]) s.segs.push_back(GemmSeg{u.tile, u.kb0, u.kb1, 0});
    }
    s.cta[P] = (int)s.segs.size();
    number_pieces(s, (int)tkb.size());
    return s;
}

// predicted makespan in k-blocks (the largest per-CTA load)
long sched_cost(const Sched &s, int ovh)
{
    long worst = 0;
    for (size_t c = 0; c + 1 < s.cta.size(); c++) {
        long l = 0;
        for (int q = s.cta[c]; q < s.cta[c + 1]; q++) l += s.segs[q].kb1 - s.segs[q].kb0 + ovh;
        worst = std::max(worst, l);
    }
    return worst;
}

// stream-K over units of unequal cost per step: the summed cost cut into P equal
// ranges; a step belongs to the CTA whose range holds the cost at its start
Sched sched_weighted(const std::vector<int> &steps, const std::vector<int> &w, int P)
{
    Sched s;
    s.name = "weighted stream-k";
    const int nu = (int)steps.size();
    std::vector<long> pre(nu + 1, 0);
    for (int u = 0; u < nu; u++) pre[u + 1] = pre[u] + (long)steps[u] * w[u];
    const long W = pre[nu];
    auto first_step = [&](int u, long x) -> int {   // first step of u starting at cost >= x
        if (x <= pre[u]) return 0;
        const long k = (x - pre[u] + w[u] - 1) / w[u];
        return (int)std::min<long>(k, steps[u]);
    };
    s.cta.assign(P + 1, 0);
    int u0 = 0;
    for (int c = 0; c < P; c++) {
        const long lo = W * c / P, hi = W * (c + 1) / P;
        s.cta[c] = (int)s.segs.size();
        while (u0 < nu && pre[u0 + 1] <= lo) u0++;
        for (int u = u0; u < nu && pre[u] < hi; u++) {
            const int a = first_step(u, lo), b = first_step(u, hi);
            if (b > a) s.segs.push_back(GemmSeg{u, a, b, 0});
        }
    }
    s.cta[P] = (int)s.segs.size();
    number_pieces(s, nu);
    return s;
}

// every segment cut, within its CTA, into pieces of at most SEG_MAX_KB k-blocks:
// one FP32 tensor-memory accumulator then sums at most 64 SEG_MAX_KB products
// (16,384 sources), whatever N, and the pieces are added in FP64 by the stage
// epilogue, which bounds the accumulation error of the contraction.  Measured
// at N = 20k x 64 (max |T - K V| / (|K| |V|) on 768 rows, ms per attempt): no
// cap 8.9e-5 / 5.95, 256 k-blocks 4.8e-5 / 6.07, 128 k-blocks 3.1e-5 / 6.21
constexpr int SEG_MAX_KB = 256;

void cap_segments(Sched &s, int ntiles, int cap = SEG_MAX_KB)
{
    std::vector<GemmSeg> segs;
    std::vector<int> cta(s.cta.size(), 0);
    for (size_t c = 0; c + 1 < s.cta.size(); c++) {
        cta[c] = (int)segs.size();
        for (int q = s.cta[c]; q < s.cta[c + 1]; q++) {
            const GemmSeg g = s.segs[q];
            for (int k = g.kb0; k < g.kb1; k += cap)
                segs.push_back(GemmSeg{g.tile, k, std::min(g.kb1, k + cap), 0});
        }
    }
    cta.back() = (int)segs.size();
    s.segs.swap(segs);
    s.cta.swap(cta);
    number_pieces(s, ntiles);
}

size_t b_bytes(const EnsGeomHost &g, int ni)
{
    const int ntl = (g.ninst + ni - 1) / ni;
    if (g.hier) return (size_t)ntl * g.nbkg * (size_t)(g.hpl * ni * 16);
    return (size_t)ntl * g.kblocks * (size_t)(2 * ni * BK * 2);
}

void free_hbufs(HPlanBufs &P)
{
    void *ptrs[] = {P.units, P.segs, P.cta, P.ws, P.pws, P.p0, P.np, P.rows, P.zu};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    P = HPlanBufs();
}

// one pass of the hierarchical geometries for instance tiles of width ni: units
// (pass 1 or 2 of every geometry and instance tile), weighted stream-K segments,
// partial-sum offsets, and for pass 1 the Z destination of every unit
int upload_hplan(ucg_ensemble *E, HPlanBufs &P, int ni, int pass)
{
    std::vector<HUnit> units;
    std::vector<HZUnit> zu;
    for (const EnsGeomHost &g : E->geoms) {
        if (!g.hier) continue;
        const int ntl = (g.ninst + ni - 1) / ni;
        const size_t bt = (size_t)g.nbkg * g.hpl * ni * 16;
        for (int nt = 0; nt < ntl; nt++)
            for (const EnsGeomHost::HU &h : (pass == 1 ? g.hu1 : g.hu2)) {
                HUnit u;
                u.a = g.hA + h.a_off;
                u.lo_off = h.lo_off;
                u.bidx = g.hbidx + h.bidx_off;
                u.b = g.B + nt * bt;
                u.zdst = pass == 1 ? g.hzdst + h.zdst_off : nullptr;
                u.g = h.g;
                u.nkg = h.nkg;
                u.rows = 8 * h.g;
                u.pad = 0;
                units.push_back(u);
                if (pass == 1) zu.push_back(HZUnit{g.B + nt * bt, g.hzdst + h.zdst_off, h.g, 8 * h.g, 0, 0, 0});
            }
    }
    P.nunits = (int)units.size();
    if (units.empty()) return UCG_OK;
    std::vector<int> steps, w;
    for (const HUnit &u : units) {
        steps.push_back(u.nkg / 2);
        w.push_back(u.g + 4);      // a K-step's bytes grow with the row groups; its MMAs do not
    }
    Sched s = sched_weighted(steps, w, hm_ctas(ni, E->hplanes) * E->sms);   // HTile<ni, *, planes>::CTAS per SM
    // 512 K-steps (8,192 K entries) per FP32 partial sum (three planes: of
    // register sums over fresh 64-entry accumulators; measured as accurate
    // as runs of 1,024 entries, and 7 % faster per attempt)
    cap_segments(s, P.nunits, 512);
    // partial sums for every piece, except a pass-1 unit's only one, whose
    // drain writes Z directly
    std::vector<long> pws(std::max(1, s.nslots), 0);
    long off = 0;
    for (int u = 0; u < P.nunits; u++) {
        if (pass == 1 && s.npieces[u] == 1) continue;
        for (int j = 0; j < s.npieces[u]; j++) {
            pws[s.piece0[u] + j] = off;
            off += (long)units[u].rows * ni;
        }
    }
    std::vector<HSeg> segs;
    for (const GemmSeg &q : s.segs)
        segs.push_back(HSeg{q.tile, 2 * q.kb0, 2 * q.kb1, pass == 1 && s.npieces[q.tile] == 1 ? 1 : 0, pws[q.slot]});
    std::vector<int> rows;
    for (const HUnit &u : units) rows.push_back(u.rows);
    {
        std::vector<HZUnit> split;   // k_hm_zconv: the units cut into several pieces
        for (size_t u = 0; u < zu.size(); u++)
            if (s.npieces[u] > 1) {
                zu[u].p0 = s.piece0[u];
                zu[u].np = s.npieces[u];
                split.push_back(zu[u]);
            }
        zu.swap(split);
        P.nzu = (int)zu.size();
    }
    P.nsegs = (int)segs.size();
    P.ws_floats = (size_t)std::max<long>(off, 4);
    ECUDA(cudaMalloc(&P.units, sizeof(HUnit) * units.size()));
    ECUDA(cudaMalloc(&P.segs, sizeof(HSeg) * std::max<size_t>(segs.size(), 1)));
    ECUDA(cudaMalloc(&P.cta, sizeof(int) * s.cta.size()));
    ECUDA(cudaMalloc(&P.ws, sizeof(float) * P.ws_floats));
    ECUDA(cudaMalloc(&P.pws, sizeof(long) * pws.size()));
    ECUDA(cudaMalloc(&P.p0, sizeof(int) * units.size()));
    ECUDA(cudaMalloc(&P.np, sizeof(int) * units.size()));
    ECUDA(cudaMalloc(&P.rows, sizeof(int) * units.size()));
    ECUDA(cudaMemsetAsync(P.ws, 0, sizeof(float) * P.ws_floats, E->stream));
    ECUDA(cudaMemcpyAsync(P.units, units.data(), sizeof(HUnit) * units.size(), cudaMemcpyHostToDevice, E->stream));
    if (!segs.empty())
        ECUDA(cudaMemcpyAsync(P.segs, segs.data(), sizeof(HSeg) * segs.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.cta, s.cta.data(), sizeof(int) * s.cta.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.pws, pws.data(), sizeof(long) * pws.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.p0, s.piece0.data(), sizeof(int) * units.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.np, s.npieces.data(), sizeof(int) * units.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.rows, rows.data(), sizeof(int) * units.size(), cudaMemcpyHostToDevice, E->stream));
    if (pass == 1 && !zu.empty()) {
        ECUDA(cudaMalloc(&P.zu, sizeof(HZUnit) * zu.size()));
        ECUDA(cudaMemcpyAsync(P.zu, zu.data(), sizeof(HZUnit) * zu.size(), cudaMemcpyHostToDevice, E->stream));
    }
    // the host vectors are released on return: the copies must have been made
    ECUDA(cudaStreamSynchronize(E->stream));
    return UCG_OK;
}

template <int NI, bool KLO, int PL>
cudaError_t prepare_hcontract_one()
{
    return cudaFuncSetAttribute(k_hm_contract<NI, KLO, PL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                HTile<NI, KLO, PL>::SMEM);
}

template <int NI>
cudaError_t prepare_hcontract_t(int planes)
{
    if constexpr (NI <= 64)
        if (planes == 3) return prepare_hcontract_one<NI, true, 3>();
    cudaError_t e = prepare_hcontract_one<NI, true, 2>();
    if (e != cudaSuccess) return e;
    return prepare_hcontract_one<NI, false, 2>();
}

template <int NI, bool KLO, int PL>
cudaError_t launch_hpass_t(ucg_ensemble *E, const HPlanBufs &P)
{
    using T = HTile<NI, KLO, PL>;
    k_hm_contract<NI, KLO, PL><<<T::CTAS * E->sms, 224, T::SMEM, E->stream>>>(P.units, P.segs, P.cta, P.ws,
                                                                           &E->d_glob->err);
    E->launches++;
    return cudaGetLastError();
}

// three planes: every stage in the one form (the increments' two-term option
// is a form of the dense contraction and of the two-plane images)
cudaError_t launch_hpass(ucg_ensemble *E, const HPlanBufs &P, bool klo)
{
    if (E->hplanes == 3) {
        switch (E->ni) {
        case 32: return launch_hpass_t<32, true, 3>(E, P);
        case 64: return launch_hpass_t<64, true, 3>(E, P);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (E->ni) {
    case 32: return klo ? launch_hpass_t<32, true, 2>(E, P) : launch_hpass_t<32, false, 2>(E, P);
    case 64: return klo ? launch_hpass_t<64, true, 2>(E, P) : launch_hpass_t<64, false, 2>(E, P);
    case 128: return klo ? launch_hpass_t<128, true, 2>(E, P) : launch_hpass_t<128, false, 2>(E, P);
    default: return cudaErrorInvalidValue;
    }
}

// T = H V of every hierarchical geometry: pass 1, Z into the B space, pass 2
cudaError_t launch_hier(ucg_ensemble *E, bool klo)
{
    cudaError_t e = cudaSuccess;
    if (E->h1.nunits > 0) {
        e = launch_hpass(E, E->h1, klo);
        if (e != cudaSuccess) return e;
        if (E->h1.nzu > 0) {
            if (E->hplanes == 3)
                k_hm_zconv<3><<<E->h1.nzu, 256, 0, E->stream>>>(E->h1.zu, E->h1.pws, E->h1.ws, E->ni);
            else
                k_hm_zconv<2><<<E->h1.nzu, 256, 0, E->stream>>>(E->h1.zu, E->h1.pws, E->h1.ws, E->ni);
            E->launches++;
            e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    if (E->h2.nunits > 0) e = launch_hpass(E, E->h2, klo);
    return e;
}

// the dynamic shared-memory limit is raised once per plan, outside any capture
template <int NI>
cudaError_t prepare_contract_t()
{
    cudaError_t e = cudaFuncSetAttribute(k_bf16x3_contract<NI, true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         Tile<NI, true, 1>::SMEM);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_bf16x3_contract<NI, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Tile<NI, false, 2>::SMEM);
}

cudaError_t prepare_contract(int ni, int planes)
{
    cudaError_t e;
    switch (ni) {
    case 32: e = prepare_contract_t<32>(); break;
    case 64: e = prepare_contract_t<64>(); break;
    case 128: e = cudaSuccess; break;   // hierarchical geometries only: no dense contraction
    default: return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    switch (ni) {
    case 32: return prepare_hcontract_t<32>(planes);
    case 64: return prepare_hcontract_t<64>(planes);
    default: return prepare_hcontract_t<128>(planes);
    }
}

template <int NI, bool KLO, int MT>
cudaError_t launch_contract_t(ucg_ensemble *E, const PlanBufs &P)
{
    k_bf16x3_contract<NI, KLO, MT><<<E->sms, 320, Tile<NI, KLO, MT>::SMEM, E->stream>>>(P.tiles, P.segs, P.cta,
                                                                                        P.ws, E->d_glob);
    E->launches++;
    return cudaGetLastError();
}

// klo: the anchor's contraction (K hi and lo, single M-tiles); otherwise the
// stage increments' Khi (Vhi + Vlo) over pairs of M-tiles
cudaError_t launch_contract(ucg_ensemble *E, bool klo = true)
{
    if (E->p1.nunits == 0) return cudaSuccess;   // no dense geometry
    switch (E->ni) {
    case 32: return klo ? launch_contract_t<32, true, 1>(E, E->p1) : launch_contract_t<32, false, 2>(E, E->p2);
    case 64: return klo ? launch_contract_t<64, true, 1>(E, E->p1) : launch_contract_t<64, false, 2>(E, E->p2);
    default: return cudaErrorInvalidValue;   // 128-instance tiles: hierarchical geometries only
    }
}

// the contraction of every geometry, dense and hierarchical
cudaError_t launch_all(ucg_ensemble *E, bool klo)
{
    cudaError_t e = launch_contract(E, klo);
    if (e == cudaSuccess) e = launch_hier(E, klo);
    return e;
}

void free_bufs(PlanBufs &P)
{
    void *ptrs[] = {P.tiles, P.segs, P.cta, P.piece0, P.npieces, P.ws};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    P = PlanBufs();
}

void free_plan(ucg_ensemble *E)
{
    free_bufs(E->p1);
    free_bufs(E->p2);
    free_hbufs(E->h1);
    free_hbufs(E->h2);
    if (E->graph) cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
    E->planned = false;
}

// work units (single M-tiles, mt = 1, or pairs, mt = 2) and their k-blocks, in
// unit-id order: geometry, instance tile, M-tile (pair)
std::vector<int> unit_kblocks(ucg_ensemble *E, int ni, int mt)
{
    std::vector<int> tkb;
    for (const EnsGeomHost &g : E->geoms) {
        if (g.hier) continue;
        const int ntl = (g.ninst + ni - 1) / ni;
        const int nu = (g.mtiles + mt - 1) / mt;
        for (int nt = 0; nt < ntl; nt++)
            for (int u = 0; u < nu; u++) tkb.push_back(g.kblocks);
    }
    return tkb;
}

// (re)allocate the V images for instance tiles of width ni
int ensure_b(ucg_ensemble *E, int ni)
{
    for (EnsGeomHost &g : E->geoms) {
        if (g.B && g.b_ni == ni) continue;
        if (g.B) cudaFree(g.B);
        if (g.vscale) cudaFree(g.vscale);
        g.B = nullptr;
        g.vscale = nullptr;
        const size_t bytes = b_bytes(g, ni);
        ECUDA(cudaMalloc(&g.B, bytes));
        ECUDA(cudaMemsetAsync(g.B, 0, bytes, E->stream));
        if (!g.hier) {
            // padding instances of the last tile keep zero images and zero scales
            const size_t vb = sizeof(float) * (size_t)((g.ninst + ni - 1) / ni) * g.kblocks * ni;
            ECUDA(cudaMalloc(&g.vscale, vb));
            ECUDA(cudaMemsetAsync(g.vscale, 0, vb, E->stream));
        }
        g.b_ni = ni;
    }
    return UCG_OK;
}

int upload_plan(ucg_ensemble *E, PlanBufs &P, int ni, int mt, const Sched &s)
{
    std::vector<GemmTile> units;
    for (const EnsGeomHost &g : E->geoms) {
        if (g.hier) continue;
        const int ntl = (g.ninst + ni - 1) / ni;
        for (int nt = 0; nt < ntl; nt++)
            for (int t = 0; t < g.mtiles; t += mt)
                units.push_back(GemmTile{g.A + (size_t)t * g.kblocks * A_IMG,
                                         (mt == 2 && t + 1 < g.mtiles) ? g.A + (size_t)(t + 1) * g.kblocks * A_IMG
                                                                       : nullptr,
                                         g.B + (size_t)nt * g.kblocks * (size_t)(2 * ni * BK * 2),
                                         g.kscale + (size_t)t * g.kblocks,
                                         (mt == 2 && t + 1 < g.mtiles) ? g.kscale + (size_t)(t + 1) * g.kblocks
                                                                       : nullptr,
                                         g.vscale + (size_t)nt * g.kblocks * ni});
    }
    P.nunits = (int)units.size();
    P.nsegs = (int)s.segs.size();
    P.nslots = s.nslots;
    P.name = s.name;
    if (units.empty()) return UCG_OK;   // no dense geometry
    ECUDA(cudaMalloc(&P.tiles, sizeof(GemmTile) * units.size()));
    ECUDA(cudaMalloc(&P.segs, sizeof(GemmSeg) * std::max<size_t>(1, s.segs.size())));
    ECUDA(cudaMalloc(&P.cta, sizeof(int) * s.cta.size()));
    ECUDA(cudaMalloc(&P.piece0, sizeof(int) * units.size()));
    ECUDA(cudaMalloc(&P.npieces, sizeof(int) * units.size()));
    const size_t ws_bytes = (size_t)std::max(1, s.nslots) * mt * ni * BM * sizeof(float);
    ECUDA(cudaMalloc(&P.ws, ws_bytes));
    ECUDA(cudaMemsetAsync(P.ws, 0, ws_bytes, E->stream));
    ECUDA(cudaMemcpyAsync(P.tiles, units.data(), sizeof(GemmTile) * units.size(), cudaMemcpyHostToDevice, E->stream));
    if (!s.segs.empty())
        ECUDA(cudaMemcpyAsync(P.segs, s.segs.data(), sizeof(GemmSeg) * s.segs.size(), cudaMemcpyHostToDevice,
                              E->stream));
    ECUDA(cudaMemcpyAsync(P.cta, s.cta.data(), sizeof(int) * s.cta.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.piece0, s.piece0.data(), sizeof(int) * units.size(), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(P.npieces, s.npieces.data(), sizeof(int) * units.size(), cudaMemcpyHostToDevice,
                          E->stream));
    return UCG_OK;
}

// upload both schedules and the kernel argument block for instance tiles of width ni
int install_plan(ucg_ensemble *E, int ni, const Sched &s1, const Sched &s2)
{
    free_plan(E);
    int st = ensure_b(E, ni);
    if (st) return st;
    ECUDA(prepare_contract(ni, E->hplanes));
    E->ni = ni;
    if ((st = upload_plan(E, E->p1, ni, 1, s1)) || (st = upload_plan(E, E->p2, ni, 2, s2))) return st;
    if ((st = upload_hplan(E, E->h1, ni, 1)) || (st = upload_hplan(E, E->h2, ni, 2))) return st;

    // kernel argument block
    EnsArgs a;
    memset(&a, 0, sizeof a);
    a.ngeom = (int)E->geoms.size();
    a.ni = ni;
    int tile0 = 0, pair0 = 0, be = 0, bs = 0, hunit0 = 0;
    for (int gi = 0; gi < a.ngeom; gi++) {
        const EnsGeomHost &g = E->geoms[gi];
        GeomDev &d = a.g[gi];
        d.np = g.np;
        d.ninst = g.ninst;
        d.mtiles = g.mtiles;
        d.kblocks = g.kblocks;
        const int ntl = (g.ninst + ni - 1) / ni;
        if (g.hier) {
            d.hier = 1;
            d.hleaves = g.hleaves;
            d.hunit0 = hunit0;
            hunit0 += ntl * g.hleaves;
            d.hbtile = (size_t)g.nbkg * g.hpl * ni * 16;
            d.hpl = g.hpl;
            d.hperm = g.hperm;
            d.hinv = g.hinv;
            d.hrow = g.hrow;
            d.hxpos = g.hxpos;
        } else {
            d.tile0 = tile0;
            tile0 += ntl * g.mtiles;
            d.mpairs = (g.mtiles + 1) / 2;
            d.pair0 = pair0;
            pair0 += ntl * d.mpairs;
        }
        d.epb_e = (g.np + EW_THREADS - 1) / EW_THREADS;
        d.blk_e0 = be;
        be += d.epb_e * g.ninst;
        d.epb_s = (int)((7L * g.np + ST_SPAN - 1) / ST_SPAN);
        d.blk_s0 = bs;
        bs += d.epb_s * g.ninst;
        d.B = g.B;
        d.vscale = g.vscale;
        d.rscale = g.rscale;
        const long len = (long)g.ninst * 7 * g.np;
        double *v = g.state;
        d.y = v; v += len;
        d.ys = v; v += len;
        for (int j = 0; j < 6; j++) { d.k[j] = v; v += len; }
        d.ycand = v; v += len;
        d.yerr = v; v += len;
        d.yscal = v; v += len;
        d.v1 = g.anchor;
        d.t1 = g.anchor + 2L * g.ninst * g.np;
        const long pl = (long)g.ninst * g.np;
        d.vpl_c = g.par; d.vpl_s = g.par + pl; d.a = g.par + 2 * pl; d.b = g.par + 3 * pl;
        d.sig = g.par + 4 * pl; d.L = g.par + 5 * pl; d.damping = g.par + 6 * pl;
        d.ctl = g.ctl;
    }
    a.blocks_e = be;
    a.blocks_s = bs;
    a.ws1 = E->p1.ws;
    a.piece0_1 = E->p1.piece0;
    a.npieces_1 = E->p1.npieces;
    a.ws2 = E->p2.ws;
    a.piece0_2 = E->p2.piece0;
    a.npieces_2 = E->p2.npieces;
    a.hws2 = E->h2.ws;
    a.hp0 = E->h2.p0;
    a.hnp = E->h2.np;
    a.hrows = E->h2.rows;
    a.hpws = E->h2.pws;
    a.glob = E->d_glob;
    ECUDA(cudaMemcpyAsync(E->d_args, &a, sizeof a, cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaStreamSynchronize(E->stream));
    E->plan_name = "ni=" + std::to_string(ni) + " anchor " + s1.name + ", increments " + s2.name + " (pairs)";
    if (E->h1.nunits + E->h2.nunits > 0) {
        size_t img = 0;
        for (const EnsGeomHost &g : E->geoms)
            if (g.hier) img += g.h_img_bytes;
        char buf[256];
        snprintf(buf, sizeof buf,
                 "; hierarchical: pass 1 %d units / %d segments, pass 2 %d units / %d segments, images %.4f GB",
                 E->h1.nunits, E->h1.nsegs, E->h2.nunits, E->h2.nsegs, img * 1e-9);
        E->plan_name += buf;
    }
    E->planned = true;
    return UCG_OK;
}

bool has_dense(const ucg_ensemble *E)
{
    for (const EnsGeomHost &g : E->geoms)
        if (!g.hier) return true;
    return false;
}

// instance tile width: 128 only for hierarchical-only ensembles of two-plane
// images (the dense contraction's per-k-block drain, and the three-plane
// hierarchical one, keep a register sum per instance of the tile and thread)
int default_ni(ucg_ensemble *E)
{
    int mx = 1;
    for (const EnsGeomHost &g : E->geoms) mx = std::max(mx, g.ninst);
    const int ni = mx <= 32 ? 32 : (mx <= 64 ? 64 : 128);
    return (ni == 128 && (has_dense(E) || E->hplanes == 3)) ? 64 : ni;
}

// the schedule of a kind for the single-tile (mt 1) or paired (mt 2) units

Sched make_sched(ucg_ensemble *E, int ni, int mt, int kind, int chunk)
{
    const std::vector<int> tkb = unit_kblocks(E, ni, mt);
    Sched s = kind == UCG_ENS_STREAM_K ? sched_stream_k(tkb, E->sms) : sched_split_lpt(tkb, E->sms, chunk, 2);
    // the anchor form only: the increments read K hi alone, whose 2^-9
    // truncation outweighs their FP32 accumulation at any length (their error
    // against FP64 measured the same with and without the cap)
    if (mt == 1) cap_segments(s, (int)tkb.size());
    return s;
}

int ensure_plan(ucg_ensemble *E)
{
    if (E->planned) return UCG_OK;
    if (E->geoms.empty()) return ebad(E, UCG_E_STATE, "ensemble has no geometry");
    const int ni = default_ni(E);
    return install_plan(E, ni, make_sched(E, ni, 1, UCG_ENS_STREAM_K, 0), make_sched(E, ni, 2, UCG_ENS_STREAM_K, 0));
}

// mean device time per launch: the best of three trials of `reps` launches, so
// that a host-side stall between launches does not decide a plan
int time_contract(ucg_ensemble *E, int reps, double *ms, bool klo = true)
{
    cudaEvent_t a, b;
    ECUDA(cudaEventCreate(&a));
    ECUDA(cudaEventCreate(&b));
    for (int w = 0; w < 2; w++) ECUDA(launch_all(E, klo));
    double best = 1e300;
    for (int trial = 0; trial < 3; trial++) {
        ECUDA(cudaEventRecord(a, E->stream));
        for (int r = 0; r < reps; r++) ECUDA(launch_all(E, klo));
        ECUDA(cudaEventRecord(b, E->stream));
        ECUDA(cudaEventSynchronize(b));
        float t = 0.0f;
        cudaEventElapsedTime(&t, a, b);
        best = std::min(best, (double)t / reps);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = best;
    int e = 0;
    ECUDA(cudaMemcpy(&e, &E->d_glob->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return ebad(E, e, "contraction: a bounded device wait gave up");
    return UCG_OK;
}

// one Runge-Kutta stage for every instance
template <int S>
cudaError_t enqueue_stage(ucg_ensemble *E, int be)
{
    k_ens_prologue<S><<<be, EW_THREADS, 0, E->stream>>>(E->d_args);
    cudaError_t e = launch_all(E, S == 1 || E->inc_full);
    if (e != cudaSuccess) return e;
    k_ens_rhs<S><<<be, EW_THREADS, 0, E->stream>>>(E->d_args);
    E->launches += 2;
    return cudaGetLastError();
}

int build_graph(ucg_ensemble *E)
{
    if (E->graph) return UCG_OK;
    int be = 0, bs = 0;
    for (const EnsGeomHost &g : E->geoms) {
        be += g.ninst * ((g.np + EW_THREADS - 1) / EW_THREADS);
        bs += g.ninst * (int)((7L * g.np + ST_SPAN - 1) / ST_SPAN);
    }
    cudaGraph_t g;
    ECUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1u, cudaGraphCondAssignDefault);
    // head: activate
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(E->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        k_ens_begin<<<1, 256, 0, E->stream>>>(E->d_args);
        cudaGraph_t tmp;
        e = cudaStreamEndCapture(E->stream, &tmp);
    }
    cudaGraphNode_t head = nullptr, loop = nullptr;
    if (e == cudaSuccess) {
        size_t nn = 1;
        e = cudaGraphGetNodes(g, &head, &nn);
        if (e == cudaSuccess && nn != 1) e = cudaErrorInvalidValue;
    }
    // while (cond) { one attempt }
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&loop, g, &head, 1, &cp);
    if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(E->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = enqueue_stage<1>(E, be);
            if (le == cudaSuccess) le = enqueue_stage<2>(E, be);
            if (le == cudaSuccess) le = enqueue_stage<3>(E, be);
            if (le == cudaSuccess) le = enqueue_stage<4>(E, be);
            if (le == cudaSuccess) le = enqueue_stage<5>(E, be);
            if (le == cudaSuccess) le = enqueue_stage<6>(E, be);
            k_ens_finish<<<bs, ST_THREADS, 0, E->stream>>>(E->d_args);
            k_ens_control<<<1, CTL_THREADS, 0, E->stream>>>(E->d_args, cond, 1);
            E->launches += 2;
            cudaGraph_t tmp;
            e = cudaStreamEndCapture(E->stream, &tmp);
            if (e == cudaSuccess && le != cudaSuccess) e = le;
        }
    }
    // tail: commit what the last attempts accepted
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(E->stream, g, &loop, nullptr, 1, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        k_ens_commit<<<bs, ST_THREADS, 0, E->stream>>>(E->d_args);
        k_ens_clear_pending<<<1, 256, 0, E->stream>>>(E->d_args);
        cudaGraph_t tmp;
        e = cudaStreamEndCapture(E->stream, &tmp);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&E->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        E->graph = nullptr;
        return efail(E, e, "ensemble graph");
    }
    return UCG_OK;
}

bool geom_ok(ucg_ensemble *E, int gi, int i)
{
    return E && gi >= 0 && gi < (int)E->geoms.size() && i >= 0 && i < E->geoms[gi].ninst;
}

}  // namespace

extern "C" {

int ucg_ens_create(ucg_ensemble **out, int device)
{
    if (!out) return UCG_E_BADARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return UCG_E_NODEVICE;
    if (device < 0 || device >= count) return UCG_E_BADARG;
    ucg_ensemble *E = new (std::nothrow) ucg_ensemble();
    if (!E) return UCG_E_OOM;
    E->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&E->d_args, sizeof(EnsArgs));
    if (e == cudaSuccess) e = cudaMalloc(&E->d_glob, sizeof(EnsGlobal));
    if (e == cudaSuccess) e = cudaMallocHost(&E->h_glob, sizeof(EnsGlobal));
    if (e != cudaSuccess) {
        delete E;
        return e == cudaErrorMemoryAllocation ? UCG_E_OOM : UCG_E_CUDA;
    }
    cudaDeviceGetAttribute(&E->sms, cudaDevAttrMultiProcessorCount, device);
    memset(E->h_glob, 0, sizeof(EnsGlobal));
    E->h_glob->inc_full = E->inc_full ? 1 : 0;
    E->h_glob->epsilon = E->epsilon;
    E->h_glob->hmax = E->hmax;
    E->h_glob->ev_on = 1.0e-3;
    E->h_glob->ev_off = 1.0e-4;
    cudaMemcpy(E->d_glob, E->h_glob, sizeof(EnsGlobal), cudaMemcpyHostToDevice);
    *out = E;
    return UCG_OK;
}

void ucg_ens_destroy(ucg_ensemble *E)
{
    if (!E) return;
    cudaSetDevice(E->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    free_plan(E);
    for (EnsGeomHost &g : E->geoms) {
        void *ptrs[] = {g.A, g.rscale, g.kscale, g.vscale, g.state, g.anchor, g.par, g.ctl, g.B, g.hA, g.hbidx, g.hperm, g.hinv,
                        g.hxpos, g.hrow, g.hzdst};
        for (void *p : ptrs)
            if (p) cudaFree(p);
    }
    if (E->h_glob && E->h_glob->trace) cudaFree(E->h_glob->trace);
    if (E->d_args) cudaFree(E->d_args);
    if (E->d_glob) cudaFree(E->d_glob);
    if (E->h_glob) cudaFreeHost(E->h_glob);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
}

const char *ucg_ens_last_error(ucg_ensemble *E) { return E ? E->err.c_str() : ""; }

int ucg_ens_add_geometry(ucg_ensemble *E, ucg_ctx *c, int n_instances, int *geometry)
{
    if (!E || !c) return UCG_E_BADARG;
    if (n_instances < 1 || n_instances > 4096) return ebad(E, UCG_E_BADARG, "n_instances must be 1..4096");
    if ((int)E->geoms.size() >= MAX_GEOM) return ebad(E, UCG_E_BADARG, "too many geometries");
    // the hierarchical K when the context steps on it or holds no dense K
    const bool hier = c->hm && (c->precision == UCG_PREC_HMATRIX || c->precision == UCG_PREC_HMATRIX_SPLIT ||
                                !c->assembled || !c->K);
    if (!hier && (!c->assembled || !c->K))
        return ebad(E, UCG_E_STATE, "context has no assembled FP64 matrix and no hierarchical matrix");
    if (c->nv != 0) return ebad(E, UCG_E_UNSUPPORTED, "ensembles take fault patches only");
    if (c->device != E->device) return ebad(E, UCG_E_BADARG, "context on another device");
    ECUDA(cudaSetDevice(E->device));
    // the context's work (assembly) must be complete
    ECUDA(cudaStreamSynchronize(c->stream));
    EnsGeomHost g;
    g.np = c->nr + c->nt;
    g.m = c->m;
    g.n = c->n;
    g.ninst = n_instances;
    g.mtiles = (int)((g.m + BM - 1) / BM);
    g.kblocks = (int)((g.n + BK - 1) / BK);
    const long rows_pad = (long)g.mtiles * BM;
    const size_t aimg = (size_t)g.mtiles * g.kblocks * A_IMG;
    const long len = (long)g.ninst * 7 * g.np;
    cudaError_t e = cudaSuccess;
    if (hier) {
        ucg::HLayout L;
        ucg::hmatrix_layout(c, &L);
        g.hpl = E->hplanes;
        int st = build_hgeom(E, L, g);
        if (st) {
            void *ptrs[] = {g.hA, g.hbidx, g.hperm, g.hinv, g.hxpos, g.hrow, g.hzdst};
            for (void *p : ptrs)
                if (p) cudaFree(p);
            return st;
        }
        size_t fb = 0;
        ucg::hmatrix_info(c, nullptr, nullptr, nullptr, &fb, nullptr, nullptr);
        g.h_fp64_bytes = fb;
    } else {
        e = cudaMalloc(&g.A, aimg);
        if (e == cudaSuccess) e = cudaMalloc(&g.rscale, sizeof(float) * rows_pad);
        if (e == cudaSuccess) e = cudaMalloc(&g.kscale, sizeof(float) * (size_t)g.mtiles * g.kblocks);
    }
    if (e == cudaSuccess) e = cudaMalloc(&g.state, sizeof(double) * 12 * len);
    if (e == cudaSuccess) e = cudaMalloc(&g.anchor, sizeof(double) * 5L * g.ninst * g.np);
    if (e == cudaSuccess) e = cudaMalloc(&g.par, sizeof(double) * 7L * g.ninst * g.np);
    if (e == cudaSuccess) e = cudaMalloc(&g.ctl, sizeof(InstCtl) * g.ninst);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.state, 0, sizeof(double) * 12 * len, E->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.anchor, 0, sizeof(double) * 5L * g.ninst * g.np, E->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.par, 0, sizeof(double) * 7L * g.ninst * g.np, E->stream);
    if (e == cudaSuccess) {
        std::vector<InstCtl> ctl(g.ninst);
        memset(ctl.data(), 0, sizeof(InstCtl) * g.ninst);
        for (InstCtl &x : ctl) {
            x.need_stage1 = 1;
            x.status = UCG_E_STATE;    // no state yet: inactive until ucg_ens_set_state
        }
        e = cudaMemcpy(g.ctl, ctl.data(), sizeof(InstCtl) * g.ninst, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && !hier) {
        // K = diag(row scale) (block scale) (hi + 2^-11 lo): the contraction's
        // drain applies the block scales, the stage epilogue the row scales
        k_row_scale<<<(unsigned)((rows_pad + 7) / 8), 256, 0, E->stream>>>(c->K, g.m, g.n, rows_pad, g.rscale);
        k_block_scale<<<(unsigned)(g.mtiles * g.kblocks), 256, 0, E->stream>>>(c->K, g.m, g.n, g.kblocks, g.rscale,
                                                                              g.kscale);
        const long work = rows_pad * (long)g.kblocks * (BK / 8);
        k_pack_k<<<(unsigned)((work + 255) / 256), 256, 0, E->stream>>>(c->K, g.m, g.n, g.kblocks, rows_pad,
                                                                       g.rscale, g.kscale, g.A);
        E->launches += 3;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    if (e != cudaSuccess) {
        void *ptrs[] = {g.A, g.rscale, g.kscale, g.state, g.anchor, g.par, g.ctl, g.hA, g.hbidx, g.hperm, g.hinv, g.hxpos, g.hrow,
                        g.hzdst};
        for (void *p : ptrs)
            if (p) cudaFree(p);
        return efail(E, e, "ucg_ens_add_geometry");
    }
    free_plan(E);
    E->geoms.push_back(g);
    if (geometry) *geometry = (int)E->geoms.size() - 1;
    return UCG_OK;
}

int ucg_ens_set_friction(ucg_ensemble *E, int gi, int inst, const double *Vpl, const double *rake,
                         const double *mu0, const double *sig, const double *a, const double *b, const double *L,
                         const double *Vo, const double *damping)
{
    (void)mu0;
    (void)Vo;
    if (!geom_ok(E, gi, inst)) return E ? ebad(E, UCG_E_BADARG, "geometry/instance out of range") : UCG_E_BADARG;
    if (!Vpl || !rake || !sig || !a || !b || !L || !damping) return ebad(E, UCG_E_BADARG, "null array");
    EnsGeomHost &g = E->geoms[gi];
    const int np = g.np;
    std::vector<double> h(7L * np);
    for (int e = 0; e < np; e++) {
        h[e] = Vpl[e] * cos(rake[e]);
        h[np + e] = Vpl[e] * sin(rake[e]);
        h[2 * np + e] = a[e];
        h[3 * np + e] = b[e];
        h[4 * np + e] = sig[e];
        h[5 * np + e] = L[e];
        h[6 * np + e] = damping[e];
    }
    const long pl = (long)g.ninst * np;
    for (int q = 0; q < 7; q++)
        ECUDA(cudaMemcpy(g.par + q * pl + (long)inst * np, h.data() + (long)q * np, sizeof(double) * np,
                         cudaMemcpyHostToDevice));
    return UCG_OK;
}

int ucg_ens_set_tolerance(ucg_ensemble *E, double epsilon, double max_step)
{
    if (!E) return UCG_E_BADARG;
    if (!(epsilon > 0.0) || !(max_step > 0.0)) return ebad(E, UCG_E_BADARG, "tolerance and max step must be > 0");
    E->epsilon = epsilon;
    E->hmax = max_step;
    return UCG_OK;
}

int ucg_ens_set_state(ucg_ensemble *E, int gi, int inst, double time, const double *y, double dt_next)
{
    if (!geom_ok(E, gi, inst)) return E ? ebad(E, UCG_E_BADARG, "geometry/instance out of range") : UCG_E_BADARG;
    if (!y || !(dt_next > 0.0)) return ebad(E, UCG_E_BADARG, "null state or dt_next <= 0");
    EnsGeomHost &g = E->geoms[gi];
    const long len = 7L * g.np;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    ECUDA(cudaMemcpy(g.state + (long)inst * len, y, sizeof(double) * len, cudaMemcpyHostToDevice));
    InstCtl x;
    memset(&x, 0, sizeof x);
    x.h = dt_next;
    x.dt_next = dt_next;
    x.time = time;
    x.need_stage1 = 1;
    x.status = UCG_OK;
    x.thmin_key = ~0ull;
    ECUDA(cudaMemcpy(g.ctl + inst, &x, sizeof x, cudaMemcpyHostToDevice));
    return UCG_OK;
}

int ucg_ens_get_state(ucg_ensemble *E, int gi, int inst, double *y, double *time, double *dt_next, long *accepted,
                      long *rejected, int *status)
{
    if (!geom_ok(E, gi, inst)) return E ? ebad(E, UCG_E_BADARG, "geometry/instance out of range") : UCG_E_BADARG;
    EnsGeomHost &g = E->geoms[gi];
    const long len = 7L * g.np;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    if (y) ECUDA(cudaMemcpy(y, g.state + (long)inst * len, sizeof(double) * len, cudaMemcpyDeviceToHost));
    InstCtl x;
    ECUDA(cudaMemcpy(&x, g.ctl + inst, sizeof x, cudaMemcpyDeviceToHost));
    if (time) *time = x.time;
    if (dt_next) *dt_next = x.h;
    if (accepted) *accepted = (long)x.accepted;
    if (rejected) *rejected = (long)x.rejected;
    if (status) *status = x.status;
    return UCG_OK;
}

int ucg_ens_set_states(ucg_ensemble *E, int gi, const double *y, const double *time, const double *dt_next)
{
    if (!E || gi < 0 || gi >= (int)E->geoms.size()) return E ? ebad(E, UCG_E_BADARG, "geometry out of range") : UCG_E_BADARG;
    if (!y || !time || !dt_next) return ebad(E, UCG_E_BADARG, "null array");
    EnsGeomHost &g = E->geoms[gi];
    for (int i = 0; i < g.ninst; i++)
        if (!(dt_next[i] > 0.0)) return ebad(E, UCG_E_BADARG, "dt_next <= 0");
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    const long len = 7L * g.np * g.ninst;
    ECUDA(cudaMemcpyAsync(g.state, y, sizeof(double) * len, cudaMemcpyHostToDevice, E->stream));
    std::vector<InstCtl> x(g.ninst);
    memset(x.data(), 0, sizeof(InstCtl) * g.ninst);
    for (int i = 0; i < g.ninst; i++) {
        x[i].h = x[i].dt_next = dt_next[i];
        x[i].time = time[i];
        x[i].need_stage1 = 1;
        x[i].status = UCG_OK;
        x[i].thmin_key = ~0ull;
    }
    ECUDA(cudaMemcpyAsync(g.ctl, x.data(), sizeof(InstCtl) * g.ninst, cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaStreamSynchronize(E->stream));
    return UCG_OK;
}

int ucg_ens_set_hier_planes(ucg_ensemble *E, int planes)
{
    if (!E || (planes != 2 && planes != 3)) return E ? ebad(E, UCG_E_BADARG, "planes must be 2 or 3") : UCG_E_BADARG;
    for (const EnsGeomHost &g : E->geoms)
        if (g.hier && g.hpl != planes)
            return ebad(E, UCG_E_STATE, "the planes are fixed once a hierarchical geometry is added");
    E->hplanes = planes;
    return UCG_OK;
}

int ucg_ens_set_increment_terms(ucg_ensemble *E, int terms)
{
    if (!E || (terms != 2 && terms != 3)) return E ? ebad(E, UCG_E_BADARG, "terms must be 2 or 3") : UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    E->inc_full = terms == 3;
    E->h_glob->inc_full = E->inc_full ? 1 : 0;
    ECUDA(cudaMemcpy(&E->d_glob->inc_full, &E->h_glob->inc_full, sizeof(int), cudaMemcpyHostToDevice));
    if (E->graph) cudaGraphExecDestroy(E->graph);   // the launches differ: capture again
    E->graph = nullptr;
    return UCG_OK;
}

int ucg_ens_test_wait_timeout(ucg_ensemble *E, long wait_ns, int hold)
{
    if (!E || wait_ns < 0) return UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    E->h_glob->wait_ns = (unsigned long long)wait_ns;
    E->h_glob->test_hold = hold != 0;
    E->h_glob->err = 0;
    ECUDA(cudaMemcpy(&E->d_glob->wait_ns, &E->h_glob->wait_ns, sizeof(unsigned long long), cudaMemcpyHostToDevice));
    ECUDA(cudaMemcpy(&E->d_glob->test_hold, &E->h_glob->test_hold, sizeof(int), cudaMemcpyHostToDevice));
    ECUDA(cudaMemcpy(&E->d_glob->err, &E->h_glob->err, sizeof(int), cudaMemcpyHostToDevice));
    return UCG_OK;
}

int ucg_ens_put_states(ucg_ensemble *E, int gi, const double *y)
{
    if (!E || gi < 0 || gi >= (int)E->geoms.size()) return E ? ebad(E, UCG_E_BADARG, "geometry out of range") : UCG_E_BADARG;
    if (!y) return ebad(E, UCG_E_BADARG, "null array");
    EnsGeomHost &g = E->geoms[gi];
    ECUDA(cudaSetDevice(E->device));
    const long len = 7L * g.np, total = len * g.ninst;
    double *staged = g.state + 8 * total;   // the candidate vector: free between launches
    ECUDA(cudaMemcpyAsync(staged, y, sizeof(double) * total, cudaMemcpyHostToDevice, E->stream));
    const int blocks = (int)std::min<long>((total + 255) / 256, 4L * 148);
    ens::k_ens_put<<<blocks, 256, 0, E->stream>>>(g.state, staged, g.ctl, len, total);
    E->launches++;
    ECUDA(cudaGetLastError());
    ECUDA(cudaStreamSynchronize(E->stream));
    return UCG_OK;
}

int ucg_ens_get_states(ucg_ensemble *E, int gi, double *y, double *time, double *dt_next, long *accepted,
                       long *rejected, int *status)
{
    if (!E || gi < 0 || gi >= (int)E->geoms.size()) return E ? ebad(E, UCG_E_BADARG, "geometry out of range") : UCG_E_BADARG;
    EnsGeomHost &g = E->geoms[gi];
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    if (y) ECUDA(cudaMemcpyAsync(y, g.state, sizeof(double) * 7L * g.np * g.ninst, cudaMemcpyDeviceToHost, E->stream));
    std::vector<InstCtl> x(g.ninst);
    ECUDA(cudaMemcpyAsync(x.data(), g.ctl, sizeof(InstCtl) * g.ninst, cudaMemcpyDeviceToHost, E->stream));
    ECUDA(cudaStreamSynchronize(E->stream));
    for (int i = 0; i < g.ninst; i++) {
        if (time) time[i] = x[i].time;
        if (dt_next) dt_next[i] = x[i].h;
        if (accepted) accepted[i] = (long)x[i].accepted;
        if (rejected) rejected[i] = (long)x[i].rejected;
        if (status) status[i] = x[i].status;
    }
    return UCG_OK;
}

int ucg_ens_plan(ucg_ensemble *E, int ni, int schedule, int chunk)
{
    if (!E) return UCG_E_BADARG;
    if (E->geoms.empty()) return ebad(E, UCG_E_STATE, "ensemble has no geometry");
    if (ni != 32 && ni != 64 && ni != 128) return ebad(E, UCG_E_BADARG, "ni must be 32, 64 or 128");
    if (ni == 128 && has_dense(E))
        return ebad(E, UCG_E_UNSUPPORTED, "ni 128 is for hierarchical geometries only");
    if (ni == 128 && E->hplanes == 3)
        return ebad(E, UCG_E_UNSUPPORTED, "ni 128 takes two-plane hierarchical images only");
    if (schedule != UCG_ENS_STREAM_K && schedule != UCG_ENS_SPLIT_LPT) return ebad(E, UCG_E_BADARG, "unknown schedule");
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    return install_plan(E, ni, make_sched(E, ni, 1, schedule, chunk), make_sched(E, ni, 2, schedule, chunk));
}

int ucg_ens_tune(ucg_ensemble *E, int reps, char *report, long report_len)
{
    if (!E) return UCG_E_BADARG;
    if (E->geoms.empty()) return ebad(E, UCG_E_STATE, "ensemble has no geometry");
    if (reps < 1) reps = 5;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    int maxinst = 1;
    for (const EnsGeomHost &g : E->geoms) maxinst = std::max(maxinst, g.ninst);
    std::vector<int> nis = {default_ni(E)};
    if (maxinst > 64 && nis[0] != 64) nis.push_back(64);   // (default 128: hierarchical only)
    std::string rep;
    // the anchor's schedule (single tiles) and the increments' (pairs) are chosen
    // independently; an attempt costs one anchor and five increment contractions
    double best = 1e300;
    int best_ni = 0;
    struct Cand { int kind, chunk; };
    Cand b1{UCG_ENS_STREAM_K, 0}, b2{UCG_ENS_STREAM_K, 0};
    for (int ni : nis) {
        std::vector<Cand> cands = {{UCG_ENS_STREAM_K, 0}, {UCG_ENS_SPLIT_LPT, 0}};
        for (int ch : {8, 16, 32, 64}) cands.push_back({UCG_ENS_SPLIT_LPT, ch});
        double bf = 1e300, bh = 1e300;
        Cand c1 = cands[0], c2 = cands[0];
        for (const Cand &cd : cands) {
            const Sched s1 = make_sched(E, ni, 1, cd.kind, cd.chunk), s2 = make_sched(E, ni, 2, cd.kind, cd.chunk);
            int st = install_plan(E, ni, s1, s2);
            double ms_full = 0.0, ms_hi = 0.0;
            if (!st) st = time_contract(E, reps, &ms_full, true);
            if (!st) st = time_contract(E, reps, &ms_hi, false);
            if (st) return st;
            char line[200];
            snprintf(line, sizeof line,
                     "ni=%d %-16s anchor: %5d segments, predicted %6ld k-blocks, %.4f ms   increments (pairs): "
                     "%5d segments, predicted %6ld k-blocks, %.4f ms\n", ni, s1.name.c_str(), (int)s1.segs.size(),
                     sched_cost(s1, 2), ms_full, (int)s2.segs.size(), sched_cost(s2, 2), ms_hi);
            rep += line;
            if (ms_full < bf) { bf = ms_full; c1 = cd; }
            if (ms_hi < bh) { bh = ms_hi; c2 = cd; }
        }
        if (bf + 5.0 * bh < best) {
            best = bf + 5.0 * bh;
            best_ni = ni;
            b1 = c1;
            b2 = c2;
        }
    }
    ECUDA(cudaStreamSynchronize(E->stream));
    const int st = install_plan(E, best_ni, make_sched(E, best_ni, 1, b1.kind, b1.chunk),
                                make_sched(E, best_ni, 2, b2.kind, b2.chunk));
    if (st) return st;
    rep += "chosen: " + E->plan_name + "\n";
    E->tune_report = rep;
    if (report && report_len > 0) {
        strncpy(report, rep.c_str(), (size_t)report_len - 1);
        report[report_len - 1] = '\0';
    }
    return UCG_OK;
}

int ucg_ens_matvec(ucg_ensemble *E, int gi, const double *V, double *T, int terms)
{
    if (!E || gi < 0 || gi >= (int)(E ? E->geoms.size() : 0)) return UCG_E_BADARG;
    if (!V || !T) return ebad(E, UCG_E_BADARG, "null array");
    if (terms != 2 && terms != 3) return ebad(E, UCG_E_BADARG, "terms must be 2 or 3");
    ECUDA(cudaSetDevice(E->device));
    int st = ensure_plan(E);
    if (st) return st;
    const EnsGeomHost &g = E->geoms[gi];
    double *dV = nullptr, *dT = nullptr;
    ECUDA(cudaMalloc(&dV, sizeof(double) * g.ninst * g.n));
    cudaError_t e = cudaMalloc(&dT, sizeof(double) * g.ninst * g.m);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dV, V, sizeof(double) * g.ninst * g.n, cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess) {
        if (g.hier) {
            const long work = (long)g.ninst * g.np;
            k_pack_x_dense<<<(unsigned)((work + 255) / 256), 256, 0, E->stream>>>(E->d_args, gi, dV);
        } else {
            const long warps = (long)g.ninst * g.kblocks;
            k_pack_v_dense<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, E->stream>>>(g.B, g.vscale, E->ni,
                                                                                       g.kblocks, g.ninst, g.n, dV);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = launch_all(E, terms == 3);
    if (e == cudaSuccess) {
        const long work = (long)g.ninst * g.m;
        if (g.hier)
            k_reduce_h<<<(unsigned)((work + 255) / 256), 256, 0, E->stream>>>(E->d_args, gi, dT);
        else
            k_reduce_dense<<<(unsigned)((work + 255) / 256), 256, 0, E->stream>>>(E->d_args, gi, dT,
                                                                                 terms == 2 ? 1 : 0);
        E->launches += 2;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(T, dT, sizeof(double) * g.ninst * g.m, cudaMemcpyDeviceToHost, E->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(E->stream);
    cudaFree(dV);
    if (dT) cudaFree(dT);
    if (e != cudaSuccess) return efail(E, e, "ucg_ens_matvec");
    int derr = 0;
    ECUDA(cudaMemcpy(&derr, &E->d_glob->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (derr) return ebad(E, derr, "contraction: a bounded device wait gave up");
    return UCG_OK;
}

namespace {
// the attempt loop without the graph: the same kernels launched from the host,
// for tools that do not follow conditional graph nodes
int run_eager(ucg_ensemble *E)
{
    int be = 0, bs = 0;
    for (const EnsGeomHost &g : E->geoms) {
        be += g.ninst * ((g.np + EW_THREADS - 1) / EW_THREADS);
        bs += g.ninst * (int)((7L * g.np + ST_SPAN - 1) / ST_SPAN);
    }
    k_ens_begin<<<1, 256, 0, E->stream>>>(E->d_args);
    E->launches++;
    for (long a = 0; a < E->h_glob->budget; a++) {
        cudaError_t le = enqueue_stage<1>(E, be);
        if (le == cudaSuccess) le = enqueue_stage<2>(E, be);
        if (le == cudaSuccess) le = enqueue_stage<3>(E, be);
        if (le == cudaSuccess) le = enqueue_stage<4>(E, be);
        if (le == cudaSuccess) le = enqueue_stage<5>(E, be);
        if (le == cudaSuccess) le = enqueue_stage<6>(E, be);
        if (le != cudaSuccess) return efail(E, le, "ensemble attempt");
        k_ens_finish<<<bs, ST_THREADS, 0, E->stream>>>(E->d_args);
        k_ens_control<<<1, CTL_THREADS, 0, E->stream>>>(E->d_args, 0, 0);
        E->launches += 2;
        if ((a & 15) == 15 || a + 1 == E->h_glob->budget) {
            EnsGlobal g;
            ECUDA(cudaMemcpyAsync(&g, E->d_glob, sizeof g, cudaMemcpyDeviceToHost, E->stream));
            ECUDA(cudaStreamSynchronize(E->stream));
            if (g.active_count == 0 || g.err) break;
        }
    }
    k_ens_commit<<<bs, ST_THREADS, 0, E->stream>>>(E->d_args);
    k_ens_clear_pending<<<1, 256, 0, E->stream>>>(E->d_args);
    E->launches += 2;
    ECUDA(cudaGetLastError());
    return UCG_OK;
}
}  // namespace

int ucg_ens_use_graph(ucg_ensemble *E, int use_graph)
{
    if (!E) return UCG_E_BADARG;
    E->use_graph = use_graph != 0;
    return UCG_OK;
}

int ucg_ens_run(ucg_ensemble *E, double t_end, long max_attempts, long *attempts)
{
    if (!E) return UCG_E_BADARG;
    if (attempts) *attempts = 0;
    if (max_attempts < 1) return ebad(E, UCG_E_BADARG, "max_attempts must be >= 1");
    ECUDA(cudaSetDevice(E->device));
    int st = ensure_plan(E);
    if (st) return st;
    if (E->use_graph) {
        st = build_graph(E);
        if (st) return st;
    }
    ECUDA(cudaStreamSynchronize(E->stream));
    E->h_glob->t_end = t_end;
    E->h_glob->epsilon = E->epsilon;
    E->h_glob->hmax = E->hmax;
    E->h_glob->budget = max_attempts;
    E->h_glob->attempts = 0;
    E->h_glob->err = 0;
    ECUDA(cudaMemcpyAsync(&E->d_glob->t_end, &E->h_glob->t_end, sizeof(double) * 3, cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(&E->d_glob->budget, &E->h_glob->budget, sizeof(long long), cudaMemcpyHostToDevice, E->stream));
    ECUDA(cudaMemcpyAsync(&E->d_glob->err, &E->h_glob->err, sizeof(int), cudaMemcpyHostToDevice, E->stream));
    if (E->use_graph) {
        ECUDA(cudaGraphLaunch(E->graph, E->stream));
    } else {
        st = run_eager(E);
        if (st) return st;
    }
    ECUDA(cudaMemcpyAsync(E->h_glob, E->d_glob, sizeof(EnsGlobal), cudaMemcpyDeviceToHost, E->stream));
    ECUDA(cudaStreamSynchronize(E->stream));
    if (attempts) *attempts = (long)E->h_glob->attempts;
    if (E->h_glob->err) return ebad(E, E->h_glob->err, "contraction: a bounded device wait gave up");
    return UCG_OK;
}

int ucg_ens_set_step_model(ucg_ensemble *E, const ucg_mlp *model)
{
    if (!E) return UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    mlp_device_params(model, &E->h_glob->mlp_P, &E->h_glob->mlp_N);
    ECUDA(cudaMemcpy(&E->d_glob->mlp_P, &E->h_glob->mlp_P, sizeof(void *) * 2, cudaMemcpyHostToDevice));
    return UCG_OK;
}

int ucg_ens_record_traces(ucg_ensemble *E, long capacity)
{
    if (!E || capacity < 0) return UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    if (E->h_glob->trace) cudaFree(E->h_glob->trace);
    E->h_glob->trace = nullptr;
    E->h_glob->trace_cap = 0;
    E->h_glob->trace_n = 0;
    if (capacity > 0) {
        ECUDA(cudaMalloc(&E->h_glob->trace, sizeof(float) * TRACE_LEN * (size_t)capacity));
        E->h_glob->trace_cap = (unsigned long long)capacity;
    }
    ECUDA(cudaMemcpy(&E->d_glob->trace, &E->h_glob->trace, sizeof(float *) + 2 * sizeof(unsigned long long),
                     cudaMemcpyHostToDevice));
    return UCG_OK;
}

int ucg_ens_get_traces(ucg_ensemble *E, float *buf, long max_records, long *n_records)
{
    if (!E) return UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    unsigned long long n = 0;
    ECUDA(cudaMemcpy(&n, &E->d_glob->trace_n, sizeof n, cudaMemcpyDeviceToHost));
    n = std::min(n, E->h_glob->trace_cap);
    if (n_records) *n_records = (long)n;
    if (buf && max_records > 0 && E->h_glob->trace) {
        const unsigned long long k = std::min(n, (unsigned long long)max_records);
        ECUDA(cudaMemcpy(buf, E->h_glob->trace, sizeof(float) * TRACE_LEN * k, cudaMemcpyDeviceToHost));
    }
    return UCG_OK;
}

int ucg_ens_set_event_threshold(ucg_ensemble *E, double vmax_on, double vmax_off)
{
    if (!E) return UCG_E_BADARG;
    if (!(vmax_on > 0.0) || !(vmax_off > 0.0) || vmax_off > vmax_on)
        return ebad(E, UCG_E_BADARG, "need 0 < vmax_off <= vmax_on");
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    E->h_glob->ev_on = vmax_on;
    E->h_glob->ev_off = vmax_off;
    ECUDA(cudaMemcpy(&E->d_glob->ev_on, &E->h_glob->ev_on, 2 * sizeof(double), cudaMemcpyHostToDevice));
    return UCG_OK;
}

int ucg_ens_get_events(ucg_ensemble *E, int gi, int inst, long *n_events, double *t_first)
{
    if (!geom_ok(E, gi, inst)) return E ? ebad(E, UCG_E_BADARG, "geometry/instance out of range") : UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    InstCtl x;
    ECUDA(cudaMemcpy(&x, E->geoms[gi].ctl + inst, sizeof x, cudaMemcpyDeviceToHost));
    if (n_events) *n_events = (long)x.n_events;
    if (t_first) *t_first = x.n_events ? x.t_event : -1.0;
    return UCG_OK;
}

int ucg_ens_info(ucg_ensemble *E, long *total_attempts, int *active, long *launches, long *accepted,
                 long *rejected, double *time_sum, char *plan, long plan_len)
{
    if (!E) return UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    ECUDA(cudaStreamSynchronize(E->stream));
    EnsGlobal g;
    ECUDA(cudaMemcpy(&g, E->d_glob, sizeof g, cudaMemcpyDeviceToHost));
    long acc = 0, rej = 0;
    double ts = 0.0;
    for (const EnsGeomHost &geo : E->geoms) {
        std::vector<InstCtl> x(geo.ninst);
        ECUDA(cudaMemcpy(x.data(), geo.ctl, sizeof(InstCtl) * geo.ninst, cudaMemcpyDeviceToHost));
        for (const InstCtl &c : x) {
            acc += (long)c.accepted;
            rej += (long)c.rejected;
            ts += c.time;
        }
    }
    if (total_attempts) *total_attempts = (long)g.total_attempts;
    if (active) *active = g.active_count;
    if (launches) *launches = E->launches;
    if (accepted) *accepted = acc;
    if (rejected) *rejected = rej;
    if (time_sum) *time_sum = ts;
    if (plan && plan_len > 0) {
        strncpy(plan, E->plan_name.c_str(), (size_t)plan_len - 1);
        plan[plan_len - 1] = '\0';
    }
    return UCG_OK;
}

void *ucg_ens_stream(ucg_ensemble *E) { return E ? (void *)E->stream : nullptr; }

int ucg_ens_profile_contract(ucg_ensemble *E, int reps, double *ms_anchor, double *ms_increment)
{
    if (!E || reps < 1) return UCG_E_BADARG;
    ECUDA(cudaSetDevice(E->device));
    int st = ensure_plan(E);
    if (st) return st;
    if (ms_anchor && (st = time_contract(E, reps, ms_anchor, true))) return st;
    if (ms_increment && (st = time_contract(E, reps, ms_increment, false))) return st;
    return UCG_OK;
}

}  // extern "C"
