// Right-hand side and Cash-Karp RK4(5) stepping on the device.
//
// One attempt of RKQSm (fortran/3d/src/ode45.f90:51-108) is a fixed sequence of
// launches, captured once into a CUDA graph:
//
//   stage 1   k_prologue<1>  commit an accepted candidate, v = V(cos,sin)(rake)-Vpl
//             k_traction<1>  t = K v  fused with the rate-state / Maxwell epilogue
//   stage s   k_prologue<s>  ytmp = y + h*sum_j b_sj k_j  (BLAS-1 order of RKCKm)
//             k_traction<s>  k_s = f(ytmp)                              (s = 2..6)
//   finish    k_finish       ycand, yerr, max|yerr/yscal| (ordered-bit atomicMax)
//   control   k_control      accept/reject, step size, time, counters (1 thread)
//
// Every kernel reads the control block first and returns at once when the
// integration is inactive, or (stage 1) when the state did not change since the
// last f(y), so the same graph serves accepted and rejected attempts and many
// attempts can be queued without host round trips.
//
// The stage combinations, yout and yerr follow the reference's operation order
// with explicit round-to-nearest multiplies and adds (no FMA contraction), so
// they round exactly as the oracle's restatement of RKCKm.
//
// With the split-BF16 matrix the stages are anchored: stage 1 of a step keeps
// v1 = v(y) and t1 = K v1, and stages 2-6 multiply only the increment,
// t_s = t1 + K (v_s - v1).  The product's rounding (about 1e-5 of |K| |v|)
// then cancels from the embedded error estimate (its weights sum to zero)
// instead of dominating it on components whose state and rate are near zero,
// which at rtol 1e-8 would reject nearly every attempt.  The FP64 path keeps
// the reference's plain form.
#include <utility>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include "ucg_internal.cuh"

namespace ucg {

__device__ __constant__ double c_B[6][5] = {
    {0, 0, 0, 0, 0},
    {0.2, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
    {0.3, -0.9, 1.2, 0, 0},
    {-11.0 / 54.0, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0},
    {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};

#define C1 (37.0 / 378.0)
#define C3 (250.0 / 621.0)
#define C4 (125.0 / 594.0)
#define C6 (512.0 / 1771.0)
#define DC1 (C1 - 2825.0 / 27648.0)
#define DC3 (C3 - 18575.0 / 48384.0)
#define DC4 (C4 - 13525.0 / 55296.0)
#define DC5 (-277.0 / 14336.0)
#define DC6 (C6 - 0.25)

static const double LG10 = 2.302585092994045684017991454684364208;

struct StageArgs {
    const double *y;       // state at the start of the step
    double *ys;            // stage state written by the prologue (y itself for stage 1)
    double *k[6];
    double *v;
    double *ycand, *yerr, *yscal;
    double *v1, *t1;       // stage-1 anchor (split-BF16 matrix only)
    int anchored;
    Friction fr;
    Rheology rh;
    int np, nvol;
    long len;
};

__device__ __forceinline__ bool ctl_live(const Ctl *c) { return c->active && c->status == 0; }

// Programmatic dependent launch.  The kernels of an attempt are launched with
// programmatic stream serialization: each may be scheduled while its
// predecessor in the stream still runs, waits here (griddepcontrol.wait) until
// that predecessor has completed and its writes are visible, and at once lets
// its own successor be scheduled.  So the launch latency of every kernel of an
// attempt overlaps the previous kernel instead of adding to it (it dominates
// at small N).  Without a programmatic predecessor the wait returns at once.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *p, double x)
{
    // non-negative doubles order like their bit patterns
    atomicMax(p, (unsigned long long)__double_as_longlong(x));
}

// ---- stage prologue ------------------------------------------------------------

// stage combination for one entry with the reference BLAS-1 order
template <int S>
__device__ __forceinline__ double stage_comb(const StageArgs &a, long i, double h)
{
    const double y = a.y[i];
    if (S == 1) return y;
    if (S == 2) return __dadd_rn(y, __dmul_rn(__dmul_rn(h, c_B[1][0]), a.k[0][i]));
    double r = __dmul_rn(c_B[S - 1][0], a.k[0][i]);
#pragma unroll
    for (int j = 1; j < S - 1; j++) r = __dadd_rn(r, __dmul_rn(c_B[S - 1][j], a.k[j][i]));
    return __dadd_rn(y, __dmul_rn(h, r));
}

template <int S>
__global__ void k_prologue(StageArgs a, Ctl *ctl)
{
    pdl_enter();
    if (!ctl_live(ctl)) return;
    if (S == 1 && !ctl->need_stage1) return;
    const double h = ctl->h;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int ne = a.np + a.nvol;
    if (e >= ne) return;
    const bool patch = e < a.np;
    const long o = patch ? 7L * e : 7L * a.np + 12L * (e - a.np);
    const int w = patch ? 7 : 12;
    double *ys = a.ys;
    if (S == 1) {
        if (ctl->pending) {
            double *y = const_cast<double *>(a.y);
            for (int q = 0; q < w; q++) y[o + q] = a.ycand[o + q];
        }
    } else {
        for (int q = 0; q < w; q++) ys[o + q] = stage_comb<S>(a, o + q, h);
        if (S == 2 && ctl->need_stage1) {
            // yscal = |y| + |dt_try*dydt| + TINY (ratestate.f90:315); h == dt_try here
            for (int q = 0; q < w; q++)
                a.yscal[o + q] = fabs(a.y[o + q]) + fabs(h * a.k[0][o + q]) + 1.0e-30;
        }
    }
    const double *yy = (S == 1) ? a.y : ys;
    double *ks = a.k[S - 1];
    if (patch) {
        // ratestate.f90:667-707
        const double rake = atan2(yy[o + 3], yy[o + 2]);
        const double vel = exp(yy[o + 6] * LG10);
        const double vs = vel * cos(rake), vd = vel * sin(rake);
        ks[o + 0] = vs;
        ks[o + 1] = vd;
        double v0 = vs - a.fr.vpl_c[e], v1 = vd - a.fr.vpl_s[e];
        if (a.anchored) {
            if (S == 1) {
                a.v1[2L * e] = v0;
                a.v1[2L * e + 1] = v1;
            } else {
                v0 -= a.v1[2L * e];
                v1 -= a.v1[2L * e + 1];
            }
        }
        a.v[2L * e + 0] = v0;
        a.v[2L * e + 1] = v1;
        if (S == 1) atomic_max_pos((unsigned long long *)&ctl->vmax, vel);
        if (!isfinite(vel) || !isfinite(rake)) ctl->nonfinite = 1;
    } else {
        // viscouscycles.f90:938-995
        const int iv = e - a.np;
        double s11 = yy[o + 6], s12 = yy[o + 7], s13 = yy[o + 8];
        double s22 = yy[o + 9], s23 = yy[o + 10], s33 = yy[o + 11];
        const double p = (s11 + s22 + s33) / 3.0;
        s11 = s11 - p; s22 = s22 - p; s33 = s33 - p;
        double ev[6] = {0, 0, 0, 0, 0, 0};
        if (a.rh.nonlinear) {
            const double sII = sqrt((s11 * s11 + 2.0 * s12 * s12 + 2.0 * s13 * s13 + s22 * s22 +
                                     2.0 * s23 * s23 + s33 * s33) / 2.0);
            const double eII = a.rh.gd0[iv] * pow(sII, a.rh.npow[iv] - 1);
            ev[0] += eII * s11; ev[1] += eII * s12; ev[2] += eII * s13;
            ev[3] += eII * s22; ev[4] += eII * s23; ev[5] += eII * s33;
        }
        for (int q = 0; q < 6; q++) {
            ks[o + q] = ev[q];
            const long j = 2L * a.np + 6L * iv + q;
            double vq = ev[q] - a.rh.ebg[6L * iv + q];
            if (a.anchored) {
                if (S == 1) a.v1[j] = vq;
                else vq -= a.v1[j];
            }
            a.v[j] = vq;
        }
    }
}

// ---- traction product fused with the right-hand side ----------------------------
//
// K (m x n, row-major) times v.  A CTA owns blocks of consecutive rows: in FP64
// 12 rows, 4 patches (3 rows each) or 2 volumes (6 rows each); in the split
// forms 24.  Its 8 warps sweep interleaved column slices of a block's rows, so
// every v element loaded feeds all of them; K is streamed once.  The row
// sums are reduced across lanes and warps, and the elementwise rate-state
// (ratestate.f90:731-776) or Maxwell (viscouscycles.f90:1072-1080) epilogue of
// each owned element runs on the reduced values, writing k_s directly.

constexpr int MV_WARPS = 8;

__device__ __forceinline__ double2 ld_stream(const double *p)
{
    double2 r;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
    return r;
}

__device__ __forceinline__ void rhs_patch(const StageArgs &a, const double *yy, double *ks, int e,
                                          const double t[3])
{
    const long o = 7L * e;
    const double rake = atan2(yy[o + 3], yy[o + 2]);
    const double vel = exp(yy[o + 6] * LG10);
    const double L = a.fr.L[e], bb = a.fr.b[e], sg = a.fr.sig[e], aa = a.fr.a[e], eta = a.fr.damping[e];
    const double cr = cos(rake), sr = sin(rake);
    const double dth = (exp(-yy[o + 5] * LG10) - vel / L) / LG10;
    const double dtau = t[0] * cr + t[1] * sr;
    const double dv = (dtau - bb * sg * dth * LG10) / (aa * sg + eta * vel) / LG10;
    const double corr = eta * vel * dv * LG10;
    ks[o + 2] = t[0] - corr * cr;
    ks[o + 3] = t[1] - corr * sr;
    ks[o + 4] = t[2];
    ks[o + 5] = dth;
    ks[o + 6] = dv;
}

// Right-hand side of every patch from a traction vector already formed (the
// hierarchical product): the epilogue of k_traction without the matvec.
template <int S>
__global__ void k_rhs_t(StageArgs a, const Ctl *ctl, const double *__restrict__ t)
{
    if (!ctl_live(ctl)) return;
    if (S == 1 && !ctl->need_stage1) return;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.np) return;
    const double *yy = (S == 1) ? a.y : a.ys;
    double tr[3] = {t[3L * e], t[3L * e + 1], t[3L * e + 2]};
    if (a.anchored) {
        // anchored stages: stage 1 keeps t1 = K v1, the others add K (v - v1) to it
        for (int q = 0; q < 3; q++) {
            if (S == 1) a.t1[3L * e + q] = tr[q];
            else tr[q] += a.t1[3L * e + q];
        }
    }
    rhs_patch(a, yy, a.k[S - 1], e, tr);
}

// ---- TMA bulk-copy pipeline ------------------------------------------------------
//
// The traction product streams K once per stage evaluation and is bound by HBM
// bandwidth.  Each persistent CTA (one per SM) owns a sequence of row blocks;
// a producer warp moves K into shared memory with cp.async.bulk row copies
// (192 KB in flight: 4 stages of 48 KB in FP64, 2 of 96 KB in the split forms;
// completion counted on mbarriers) while
// 8 consumer warps multiply by v and hand the stage back.  Consumer thread
// t = 32 w + l accumulates columns c = CH k + PER t .. (PER per thread) across
// chunks, so the per-row summation order is: per-thread fused multiply-adds
// along its columns, an xor butterfly across the 32 lanes, then the 8 warps in
// order (the oracle restates exactly this order).
//
// Every mbarrier wait is bounded (about 4 s of %globaltimer); a wait that runs
// out records UCG_E_TIMEOUT in the control block and the CTA stops.

constexpr unsigned long long TM_TIMEOUT_NS = 4000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// bounded wait: false when `limit` ns pass or (abort != nullptr) another
// thread aborted
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort,
                                          unsigned long long limit = TM_TIMEOUT_NS)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    for (unsigned it = 1;; it++) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 0u) {
            if (abort && *abort) return false;
            if (gtimer() - t0 > limit) return false;
        }
    }
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// element traits: FP64 K (2 columns per thread) or split-BF16 pairs (4 per thread)
template <class KT> struct TmTraits;
// ROWS per block: 12 (4 patches or 2 volumes) in FP64; the split forms take
// 24 rows (8 patches or 4 volumes) in two 96 KB stages, which halves the
// per-block reduction and epilogue per K byte where a chunk holds 2-4 times
// more columns
template <> struct TmTraits<double> {
    static constexpr int PER = 2, CH = 512, ROWS = 12, STAGES = 4;
    using Acc = double;
};
template <> struct TmTraits<float> {   // the anchor of the split form: K/s in FP32, FP64 sums
    static constexpr int PER = 4, CH = 1024, ROWS = 24, STAGES = 2;
    using Acc = double;
};
template <> struct TmTraits<__half> {   // the fp16 plane (anchored stages 2-6): FP32 products
    static constexpr int PER = 8, CH = 2048, ROWS = 24, STAGES = 2;   // and 8-term sums, FP64 across
    using Acc = double;
};
template <class KT>
constexpr size_t tm_smem_bytes()
{
    return (size_t)TmTraits<KT>::STAGES * TmTraits<KT>::ROWS * TmTraits<KT>::CH * sizeof(KT);
}

// the thread's PER values of v for one chunk, loaded once and used for all the
// rows of the stage; then one row's contribution
template <class KT> struct TmV;
template <> struct TmV<double> { double2 x; };
template <> struct TmV<float> { double x[4]; };
template <> struct TmV<__half> { float x[8]; };   // v in FP32: the plane itself carries 2^-12
// v as loaded (one chunk ahead): the fp16 form keeps the doubles and converts
// them when the chunk is used, so that no instruction waits on the loads early
template <class KT> struct TmVRaw { TmV<KT> v; };
template <> struct TmVRaw<__half> { double x[8]; };

template <class KT>
__device__ __forceinline__ void tm_load_v(const double *v, long c, long n, TmV<KT> &vr);
template <>
__device__ __forceinline__ void tm_load_v<double>(const double *v, long c, long n, TmV<double> &vr)
{
    (void)n;
    vr.x = *reinterpret_cast<const double2 *>(v + c);
}
// c is a multiple of the values per thread (4 or 8), so away from the ragged
// end the thread's values are 16-byte aligned pairs
template <>
__device__ __forceinline__ void tm_load_v<float>(const double *v, long c, long n, TmV<float> &vr)
{
    if (c + 4 <= n) {
        const double2 a = __ldg(reinterpret_cast<const double2 *>(v + c));
        const double2 b = __ldg(reinterpret_cast<const double2 *>(v + c + 2));
        vr.x[0] = a.x; vr.x[1] = a.y; vr.x[2] = b.x; vr.x[3] = b.y;
        return;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) vr.x[q] = (c + q < n) ? v[c + q] : 0.0;
}
// the raw loads of one chunk's v (every form) and their conversion when used
template <class KT>
__device__ __forceinline__ void tm_load_raw(const double *v, long c, long n, TmVRaw<KT> &raw)
{
    tm_load_v<KT>(v, c, n, raw.v);
}
template <>
__device__ __forceinline__ void tm_load_raw<__half>(const double *v, long c, long n, TmVRaw<__half> &raw)
{
    if (c + 8 <= n) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const double2 a = __ldg(reinterpret_cast<const double2 *>(v + c + 2 * q));
            raw.x[2 * q] = a.x;
            raw.x[2 * q + 1] = a.y;
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) raw.x[q] = (c + q < n) ? v[c + q] : 0.0;
}
template <class KT>
__device__ __forceinline__ void tm_cook(const TmVRaw<KT> &raw, TmV<KT> &vr)
{
    vr = raw.v;
}
template <>
__device__ __forceinline__ void tm_cook<__half>(const TmVRaw<__half> &raw, TmV<__half> &vr)
{
#pragma unroll
    for (int q = 0; q < 8; q++) vr.x[q] = __double2float_rn(raw.x[q]);
}

template <class KT>
__device__ __forceinline__ void tm_accumulate(const KT *srow, int cl, const TmV<KT> &vr,
                                              typename TmTraits<KT>::Acc &acc);
template <>
__device__ __forceinline__ void tm_accumulate<double>(const double *srow, int cl, const TmV<double> &vr, double &acc)
{
    const double2 kv = *reinterpret_cast<const double2 *>(srow + cl);
    acc = fma(kv.y, vr.x.y, fma(kv.x, vr.x.x, acc));
}
template <>
__device__ __forceinline__ void tm_accumulate<float>(const float *srow, int cl, const TmV<float> &vr, double &acc)
{
    const float4 kv = *reinterpret_cast<const float4 *>(srow + cl);
    acc = fma((double)kv.x, vr.x[0], acc);
    acc = fma((double)kv.y, vr.x[1], acc);
    acc = fma((double)kv.z, vr.x[2], acc);
    acc = fma((double)kv.w, vr.x[3], acc);
}
// the thread's 8 products of the row in FP32 (each rounded once, 2^-24: far
// below the plane's own 2^-12), their sum added to the FP64 row sum: one
// conversion to FP64 per 8 entries instead of one per entry
template <>
__device__ __forceinline__ void tm_accumulate<__half>(const __half *srow, int cl, const TmV<__half> &vr, double &acc)
{
    const uint4 raw = *reinterpret_cast<const uint4 *>(srow + cl);
    const uint32_t w4[4] = {raw.x, raw.y, raw.z, raw.w};
    float p = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2 *>(&w4[q]));
        p = __fmaf_rn(f.x, vr.x[2 * q], p);
        p = __fmaf_rn(f.y, vr.x[2 * q + 1], p);
    }
    acc += (double)p;
}

template <int S, class KT>
__global__ void __launch_bounds__((MV_WARPS + 1) * 32, 1) k_traction(const KT *__restrict__ K, long n, long ldk,
        const float *__restrict__ scale, StageArgs a, Ctl *ctl, int pblocks, int vblocks)
{
    using Tr = TmTraits<KT>;
    using Acc = typename Tr::Acc;
    constexpr int CH = Tr::CH, PER = Tr::PER, ROWS = Tr::ROWS, STAGES = Tr::STAGES;
    constexpr int PB = ROWS / 3, VB = ROWS / 6;   // patches, volumes per block
    pdl_enter();
    if (!ctl_live(ctl)) return;
    if (S == 1 && !ctl->need_stage1) return;
    extern __shared__ __align__(128) unsigned char tm_smem[];
    KT *stage = reinterpret_cast<KT *>(tm_smem);
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
    // row sums of a block, double-buffered: the few threads that run a
    // block's epilogue read one buffer while the other warps already
    // accumulate the next block into the other; the next block's barrier
    // orders the epilogue before its buffer comes round again
    __shared__ double red[2][MV_WARPS][ROWS];
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nblk = pblocks + vblocks;
    const long nch = (n + CH - 1) / CH;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], MV_WARPS);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto block_rows = [&](int blk, long &row0, int &nrows, int &e0, int &nel, bool &patch) {
        patch = blk < pblocks;
        if (patch) {
            e0 = blk * PB; nel = min(PB, a.np - e0); row0 = 3L * e0; nrows = 3 * nel;
        } else {
            e0 = (blk - pblocks) * VB; nel = min(VB, a.nvol - e0); row0 = 3L * a.np + 6L * e0; nrows = 6 * nel;
        }
    };

    const unsigned long long wait_lim = ctl->wait_ns ? ctl->wait_ns : TM_TIMEOUT_NS;
    if (warp == MV_WARPS) {
        // producer: one lane issues the row copies of each (block, chunk) item
        if (lane == 0) {
            long item = 0;
            // (test_hold: the first CTA issues nothing, its consumers' waits run out)
            const bool hold = ctl->test_hold && blockIdx.x == 0;
            for (int blk = blockIdx.x; blk < nblk && !abort_flag && !hold; blk += gridDim.x) {
                long row0; int nrows, e0, nel; bool patch;
                block_rows(blk, row0, nrows, e0, nel, patch);
                for (long ch = 0; ch < nch; ch++, item++) {
                    const int s = (int)(item % STAGES);
                    const uint32_t ph = (uint32_t)((item / STAGES) & 1);
                    if (!mbar_wait(&empty[s], ph ^ 1u, &abort_flag)) {
                        abort_flag = 1;
                        ctl->status = UCG_E_TIMEOUT;
                        break;
                    }
                    const long c0 = ch * CH;
                    const long w = min((long)CH, ldk - c0);
                    const uint32_t rowbytes = (uint32_t)(w * sizeof(KT));
                    mbar_expect_tx(&full[s], rowbytes * nrows);
                    KT *dst = stage + (size_t)s * ROWS * CH;
                    for (int r = 0; r < nrows; r++)
                        bulk_g2s(dst + (size_t)r * CH, K + (row0 + r) * ldk + c0, rowbytes, &full[s]);
                }
            }
            // items are issued in order, so the last copies into each stage are
            // those of the last STAGES items: they land before the CTA may exit,
            // also when the consumers gave up on them (bounded at the normal limit)
            for (long i = item > STAGES ? item - STAGES : 0; i < item; i++)
                mbar_wait(&full[i % STAGES], (uint32_t)((i / STAGES) & 1), nullptr);
        }
        return;
    }

    // consumers
    const double *yy = (S == 1) ? a.y : a.ys;
    double *ks = a.k[S - 1];
    long item = 0;
    const int t = threadIdx.x;
    int rb = 0;
    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x, rb ^= 1) {
        long row0; int nrows, e0, nel; bool patch;
        block_rows(blk, row0, nrows, e0, nel, patch);
        Acc acc[ROWS];
#pragma unroll
        for (int r = 0; r < ROWS; r++) acc[r] = Acc(0);
        // v does not depend on the stage: each chunk's values are loaded one
        // chunk ahead, so their latency overlaps the previous chunk's products
        const int cl = PER * t;
        TmVRaw<KT> vn;
        if (cl < n) tm_load_raw<KT>(a.v, cl, n, vn);
        for (long ch = 0; ch < nch; ch++, item++) {
            const int s = (int)(item % STAGES);
            const uint32_t ph = (uint32_t)((item / STAGES) & 1);
            // on a timed-out wait every consumer keeps walking the same item
            // sequence without computing, so all of them reach each named barrier
            const long c = ch * CH + cl;
            TmV<KT> vr;
            if (c < n) tm_cook<KT>(vn, vr);
            if (c + CH < n) tm_load_raw<KT>(a.v, c + CH, n, vn);
            const bool ready = !abort_flag && mbar_wait(&full[s], ph, &abort_flag, wait_lim);
            if (!ready && !abort_flag) {
                abort_flag = 1;
                ctl->status = UCG_E_TIMEOUT;
            }
            const KT *src = stage + (size_t)s * ROWS * CH;
            if (ready && c < n) {
#pragma unroll
                for (int r = 0; r < ROWS; r++)
                    if (r < nrows) tm_accumulate<KT>(src + (size_t)r * CH, cl, vr, acc[r]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
        double rs[ROWS];
#pragma unroll
        for (int r = 0; r < ROWS; r++) {
            Acc x = acc[r];
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            rs[r] = (double)x;
        }
        if (lane == 0) {
#pragma unroll
            for (int r = 0; r < ROWS; r++) red[rb][warp][r] = rs[r];
        }
        consumer_sync();
        if (t < nel && !abort_flag) {
            const int q = t;
            if (patch) {
                double tr[3];
                for (int c3 = 0; c3 < 3; c3++) {
                    double sum = 0.0;
                    for (int w = 0; w < MV_WARPS; w++) sum += red[rb][w][3 * q + c3];
                    tr[c3] = scale ? sum * (double)scale[row0 + 3 * q + c3] : sum;
                    if (a.anchored) {
                        const long row = row0 + 3 * q + c3;
                        if (S == 1) a.t1[row] = tr[c3];
                        else tr[c3] += a.t1[row];
                    }
                }
                rhs_patch(a, yy, ks, e0 + q, tr);
            } else {
                const long o = 7L * a.np + 12L * (e0 + q);
                for (int c6 = 0; c6 < 6; c6++) {
                    double sum = 0.0;
                    for (int w = 0; w < MV_WARPS; w++) sum += red[rb][w][6 * q + c6];
                    double sv = scale ? sum * (double)scale[row0 + 6 * q + c6] : sum;
                    if (a.anchored) {
                        const long row = row0 + 6 * q + c6;
                        if (S == 1) a.t1[row] = sv;
                        else sv += a.t1[row];
                    }
                    ks[o + 6 + c6] = sv;
                }
            }
        }
    }
}

// ---- finish: candidate, error estimate, error norm ------------------------------

__global__ void k_finish(StageArgs a, Ctl *ctl)
{
    pdl_enter();
    if (!ctl_live(ctl)) return;
    const double h = ctl->h;
    double mx = 0.0;
    bool bad = false;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < a.len; i += (long)gridDim.x * blockDim.x) {
        const double k1 = a.k[0][i], k3 = a.k[2][i], k4 = a.k[3][i], k5 = a.k[4][i], k6 = a.k[5][i];
        // ode45.f90:184-200
        double r = __dmul_rn(C1, k1);
        r = __dadd_rn(r, __dmul_rn(C3, k3));
        r = __dadd_rn(r, __dmul_rn(C4, k4));
        r = __dadd_rn(r, __dmul_rn(C6, k6));
        const double yc = __dadd_rn(a.y[i], __dmul_rn(h, r));
        double e = __dmul_rn(DC1, k1);
        e = __dadd_rn(e, __dmul_rn(DC3, k3));
        e = __dadd_rn(e, __dmul_rn(DC4, k4));
        e = __dadd_rn(e, __dmul_rn(DC5, k5));
        e = __dadd_rn(e, __dmul_rn(DC6, k6));
        e = __dmul_rn(h, e);
        a.ycand[i] = yc;
        a.yerr[i] = e;
        // MAXVAL semantics: a NaN ratio (0/0) does not raise the maximum; an
        // infinite one does and drives the step to underflow as in the
        // reference.  A non-finite candidate state is reported as such.
        const double q = fabs(e / a.yscal[i]);
        if (!isfinite(yc)) bad = true;
        mx = fmax(mx, q);
    }
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    bad = __any_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        if (mx > 0.0) atomic_max_pos(&ctl->errbits, mx);
        if (bad) ctl->nonfinite = 1;
    }
}

// ---- control: RKQSm decision ---------------------------------------------------

__global__ void k_control(Ctl *ctl)
{
    pdl_enter();
    if (!ctl_live(ctl)) return;
    const double SAFETY = 0.7, PGROW = -0.2, PSHRNK = -0.15, ERRCON = 1.89e-4;
    double errmax = __longlong_as_double((long long)ctl->errbits);
    ctl->errbits = 0ull;
    if (ctl->nonfinite) {
        ctl->status = UCG_E_NONFINITE;
        ctl->active = 0;
        return;
    }
    errmax = errmax / ctl->epsilon;
    double h = ctl->h;
    if (errmax > 1.0) {
        h = h * SAFETY * pow(errmax, PSHRNK);
        if (h < 0.5 * h) h = 0.5 * h;   // never taken (ode45.f90:83)
        ctl->h = h;
        ctl->clamped = 0;   // a shrunk step stays short of t_stop
        ctl->rejected += 1;
        ctl->need_stage1 = 0;
        ctl->pending = 0;
        const double tnew = 0.0 + h;     // the main loop passes t0 = 0 (ratestate.f90:317)
        if (tnew == 0.0) {
            ctl->status = UCG_E_STEP_UNDERFLOW;
            ctl->active = 0;
        }
    } else {
        double hnext;
        if (errmax > ERRCON) hnext = SAFETY * h * pow(errmax, PGROW);
        else hnext = 10.0 * h;
        if (hnext > ctl->hmax) hnext = ctl->hmax;
        ctl->hdid = h;
        ctl->time = ctl->clamped ? ctl->t_stop : ctl->time + h;
        ctl->dt_next = hnext;
        ctl->h = hnext;
        ctl->clamped = 0;
        if (ctl->stop_on && ctl->time < ctl->t_stop && ctl->time + hnext > ctl->t_stop) {
            ctl->h = ctl->t_stop - ctl->time;
            ctl->clamped = 1;
        }
        ctl->accepted += 1;
        ctl->pending = 1;
        ctl->vmax = 0.0;
        ctl->need_stage1 = 1;
        if (ctl->time >= ctl->t_end || ctl->accepted >= ctl->step_target) ctl->active = 0;
    }
}

// one output record at the start of a step (after stage 1: y and its rate k1)
__global__ void k_record(StageArgs a, const Ctl *ctl, Rec *rec)
{
    pdl_enter();
    if (!rec->enabled || !ctl_live(ctl) || !ctl->need_stage1) return;
    const long long step = ctl->accepted - rec->base;
    if (step < 0 || step % rec->every) return;
    const long long idx = step / rec->every;
    double *r = rec->buf + (idx % rec->cap) * rec->len;
    const int t = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
    if (t == 0) {
        r[0] = ctl->time;
        r[1] = ctl->hdid;
        r[2] = ctl->vmax;
        r[3] = (double)ctl->accepted;
    }
    // listed elements: state then rate, 7 per patch / 12 per volume, in a slot of 24
    for (int j = t; j < rec->nelem * 24; j += nt) {
        const int e = rec->elem[j / 24], q = j % 24;
        const bool patch = e < a.np;
        const int w = patch ? 7 : 12;
        const long o = patch ? 7L * e : 7L * a.np + 12L * (e - a.np);
        double v = 0.0;
        if (q < w) v = a.y[o + q];
        else if (q >= 12 && q - 12 < w) v = a.k[0][o + q - 12];
        r[4 + j] = v;
    }
    // observation-point displacements: row k of O against the slip (patches)
    // and the strain (volumes) of the state, one warp per row
    const int warp = t >> 5, nw = nt >> 5;
    double *ro = r + 4 + 24 * rec->nelem;
    for (int k = warp; k < 3 * rec->nobs; k += nw) {
        double sf, sl;
        observe_row(rec->O + (long)k * (2L * a.np + 6L * a.nvol), a.np, a.nvol, a.y, sf, sl);
        if ((t & 31) == 0) {
            const int p = k / 3, c = k % 3;
            if (rec->per_point == 3) {
                ro[3 * p + c] = sf + sl;
            } else {
                double d, df, dl;
                observe_split(c, sf, sl, d, df, dl);
                ro[9 * p + c] = d;
                ro[9 * p + 3 + c] = df;
                ro[9 * p + 6 + c] = dl;
            }
        }
    }
    if (t == 0) rec->written = idx + 1;
}

__global__ void k_commit(StageArgs a, const Ctl *ctl)
{
    pdl_enter();
    if (!ctl->pending) return;
    double *y = const_cast<double *>(a.y);
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < a.len; i += (long)gridDim.x * blockDim.x)
        y[i] = a.ycand[i];
}

__global__ void k_clear_pending(Ctl *ctl)
{
    pdl_enter();
    ctl->pending = 0;
}

// ---- host side -----------------------------------------------------------------

bool rk_anchored(const ucg_ctx *c)
{
    return ((c->precision == UCG_PREC_SPLIT_BF16 || c->precision == UCG_PREC_SPLIT_PAIR) && c->Ksp != nullptr) ||
           c->precision == UCG_PREC_HMATRIX_SPLIT;
}

// the attempt graph holds device addresses of the matrix and parameter arrays;
// whoever frees or replaces one of them drops the graph first
void rk_drop_graph(ucg_ctx *c)
{
    if (!c->attempt_graph) return;
    cudaStreamSynchronize(c->stream);
    cudaGraphExecDestroy(c->attempt_graph);
    c->attempt_graph = nullptr;
}

static StageArgs stage_args(ucg_ctx *c, int s)
{
    StageArgs a;
    a.y = c->st.y;
    a.ys = (s == 1) ? c->st.y : c->st.ytmp;
    for (int j = 0; j < 6; j++) a.k[j] = c->st.k[j];
    a.v = c->st.v;
    a.ycand = c->st.ycand;
    a.yerr = c->st.yerr;
    a.yscal = c->st.yscal;
    a.v1 = c->st.v1;
    a.t1 = c->st.t1;
    a.anchored = rk_anchored(c) ? 1 : 0;
    a.fr = c->fr;
    a.rh = c->rh;
    a.np = c->nr + c->nt;
    a.nvol = c->nv;
    a.len = c->state_len;
    return a;
}

int rk_alloc(ucg_ctx *c)
{
    rk_free(c);
    const long len = c->state_len;
    double **bufs[] = {&c->st.y, &c->st.ycand, &c->st.ytmp, &c->st.yerr, &c->st.yscal,
                       &c->st.k[0], &c->st.k[1], &c->st.k[2], &c->st.k[3], &c->st.k[4], &c->st.k[5]};
    for (double **b : bufs) {
        if (cudaMalloc(b, sizeof(double) * (len + 2)) != cudaSuccess) return UCG_E_OOM;
        cudaMemsetAsync(*b, 0, sizeof(double) * (len + 2), c->stream);
    }
    if (cudaMalloc(&c->st.v, sizeof(double) * (c->n + 2)) != cudaSuccess) return UCG_E_OOM;
    if (cudaMalloc(&c->st.v1, sizeof(double) * (c->n + 2)) != cudaSuccess) return UCG_E_OOM;
    if (cudaMalloc(&c->st.t1, sizeof(double) * (c->m + 2)) != cudaSuccess) return UCG_E_OOM;
    if (cudaMalloc(&c->ctl, sizeof(Ctl)) != cudaSuccess) return UCG_E_OOM;
    if (cudaMalloc(&c->rec, sizeof(Rec)) != cudaSuccess) return UCG_E_OOM;
    {
        Rec off{};
        UCG_CUDA(cudaMemcpyAsync(c->rec, &off, sizeof(Rec), cudaMemcpyHostToDevice, c->stream));
        c->rec_host = off;
    }
    if (cudaMallocHost(&c->ctl_host, sizeof(Ctl)) != cudaSuccess) return UCG_E_OOM;
    if (cudaMallocHost(&c->pin, sizeof(double) * (2 * len + 8)) != cudaSuccess) return UCG_E_OOM;
    memset(c->ctl_host, 0, sizeof(Ctl));
    c->ctl_host->epsilon = c->epsilon;
    c->ctl_host->hmax = c->hmax;
    UCG_CUDA(cudaMemcpyAsync(c->ctl, c->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    return UCG_OK;
}

void rk_free(ucg_ctx *c)
{
    double **bufs[] = {&c->st.y, &c->st.ycand, &c->st.ytmp, &c->st.yerr, &c->st.yscal,
                       &c->st.k[0], &c->st.k[1], &c->st.k[2], &c->st.k[3], &c->st.k[4], &c->st.k[5],
                       &c->st.v, &c->st.v1, &c->st.t1};
    for (double **b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
    }
    if (c->ctl) cudaFree(c->ctl);
    c->ctl = nullptr;
    if (c->rec) cudaFree(c->rec);
    c->rec = nullptr;
    if (c->rec_buf) cudaFree(c->rec_buf);
    c->rec_buf = nullptr;
    if (c->rec_elem) cudaFree(c->rec_elem);
    c->rec_elem = nullptr;
    c->rec_host = Rec{};
    c->rec_drained = 0;
    if (c->pert) cudaFree(c->pert);
    c->pert = nullptr;
    if (c->ctl_host) cudaFreeHost(c->ctl_host);
    c->ctl_host = nullptr;
    if (c->pin) cudaFreeHost(c->pin);
    c->pin = nullptr;
    if (c->attempt_graph) cudaGraphExecDestroy(c->attempt_graph);
    c->attempt_graph = nullptr;
}

// the blocks of ROWS rows (patches first, then volumes) and the grid
template <class KT>
static int traction_grid(ucg_ctx *c, int *pb, int *vb)
{
    constexpr int PB = TmTraits<KT>::ROWS / 3, VB = TmTraits<KT>::ROWS / 6;
    const int np = c->nr + c->nt;
    *pb = (np + PB - 1) / PB;
    *vb = (c->nv + VB - 1) / VB;
    const int blocks = *pb + *vb;
    const int cap = c->sms;
    return blocks < cap ? blocks : cap;
}

template <int S, class KT>
static void launch_traction_t(ucg_ctx *c, const StageArgs &a, const KT *K, long ldk, const float *scale)
{
    int pb, vb;
    const int grid = traction_grid<KT>(c, &pb, &vb);
    const size_t smem = tm_smem_bytes<KT>();
    auto kfn = k_traction<S, KT>;
    cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    launch_pdl(kfn, dim3(grid), dim3((MV_WARPS + 1) * 32), smem, c->stream, K, c->n, ldk, scale, a, c->ctl, pb, vb);
}

template <int S>
static void launch_traction(ucg_ctx *c, const StageArgs &a)
{
    if (S > 1 && c->precision == UCG_PREC_SPLIT_BF16 && rk_anchored(c) && c->Khi_plane) {
        // anchored stages multiply the increments by the fp16 plane
        launch_traction_t<S, __half>(c, a, c->Khi_plane, c->ldk_split, c->Kscale);
    } else if ((c->precision == UCG_PREC_SPLIT_BF16 || c->precision == UCG_PREC_SPLIT_PAIR) && c->Ksp) {
        launch_traction_t<S, float>(c, a, c->Ksp, c->ldk_split, c->Kscale);
    } else {
        launch_traction_t<S, double>(c, a, c->K, c->n, nullptr);
    }
}

template <int S>
static void enqueue_stage(ucg_ctx *c)
{
    const int ne = c->nr + c->nt + c->nv;
    StageArgs a = stage_args(c, S);
    launch_pdl(k_prologue<S>, dim3((ne + 127) / 128), dim3(128), 0, c->stream, a, c->ctl);
    c->launches.count += 1;
    if (c->precision == UCG_PREC_HMATRIX || c->precision == UCG_PREC_HMATRIX_SPLIT) {
        double *t = hmatrix_t(c);
        if (c->precision == UCG_PREC_HMATRIX) hmatrix_apply(c, c->st.v, t);
        else hmatrix_apply_split(c, c->st.v, t, true);     // every stage on the FP32 planes (hi + lo)
        k_rhs_t<S><<<(c->nr + c->nt + 127) / 128, 128, 0, c->stream>>>(a, c->ctl, t);
        c->launches.count += 1;
        return;
    }
    launch_traction<S>(c, a);
    c->launches.count += 1;
}

static void enqueue_attempt_raw(ucg_ctx *c)
{
    enqueue_stage<1>(c);
    // the recorder joins the attempt (and its graph) only while recording is on
    if (c->rec_host.enabled) {
        launch_pdl(k_record, dim3(c->sms), dim3(256), 0, c->stream, stage_args(c, 1), c->ctl, c->rec);
        c->launches.count += 1;
    }
    enqueue_stage<2>(c);
    enqueue_stage<3>(c);
    enqueue_stage<4>(c);
    enqueue_stage<5>(c);
    enqueue_stage<6>(c);
    StageArgs a = stage_args(c, 6);
    const int fin_grid = (int)((c->state_len + 255) / 256 < (long)c->sms * 4 ? (c->state_len + 255) / 256 : c->sms * 4);
    launch_pdl(k_finish, dim3(fin_grid > 0 ? fin_grid : 1), dim3(256), 0, c->stream, a, c->ctl);
    launch_pdl(k_control, dim3(1), dim3(1), 0, c->stream, c->ctl);
    c->launches.count += 2;
}

void rk_enqueue_attempt(ucg_ctx *c)
{
    if (!c->attempt_graph || c->graph_precision != c->precision) {
        if (c->attempt_graph) cudaGraphExecDestroy(c->attempt_graph);
        c->attempt_graph = nullptr;
        cudaGraph_t g;
        long before = c->launches.count;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            enqueue_attempt_raw(c);
            c->graph_launches = c->launches.count - before;
            if (cudaStreamEndCapture(c->stream, &g) == cudaSuccess) {
                if (cudaGraphInstantiate(&c->attempt_graph, g, 0) != cudaSuccess) c->attempt_graph = nullptr;
                cudaGraphDestroy(g);
            }
        }
        c->launches.count = before;
        c->graph_precision = c->precision;
        cudaGetLastError();
    }
    if (c->attempt_graph) {
        cudaGraphLaunch(c->attempt_graph, c->stream);
        c->launches.count += c->graph_launches;
    } else {
        enqueue_attempt_raw(c);
    }
}

void rk_enqueue_commit(ucg_ctx *c)
{
    StageArgs a = stage_args(c, 1);
    launch_pdl(k_commit, dim3((unsigned)((c->state_len + 255) / 256)), dim3(256), 0, c->stream, a, c->ctl);
    launch_pdl(k_clear_pending, dim3(1), dim3(1), 0, c->stream, c->ctl);
    c->launches.count += 2;
}

// Mean device time of the stage-2 traction launch (the dominant kernel), timed
// with events on the context stream.  The control block is made live for the
// measurement and restored afterwards.
int rk_profile_traction(ucg_ctx *c, int reps, double *ms)
{
    Ctl *h = c->ctl_host;
    UCG_CUDA(cudaMemcpyAsync(h, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    Ctl saved = *h;
    h->active = 1;
    h->status = 0;
    UCG_CUDA(cudaMemcpyAsync(c->ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    StageArgs a = stage_args(c, 2);
    cudaEvent_t e0, e1;
    UCG_CUDA(cudaEventCreate(&e0));
    UCG_CUDA(cudaEventCreate(&e1));
    UCG_CUDA(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < reps; r++) {
        launch_traction<2>(c, a);
    }
    c->launches.count += reps;
    UCG_CUDA(cudaEventRecord(e1, c->stream));
    UCG_CUDA(cudaEventSynchronize(e1));
    float t = 0.0f;
    UCG_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = (double)t / reps;
    *h = saved;
    UCG_CUDA(cudaMemcpyAsync(c->ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

// A coseismic perturbation of the state: slip (2 per patch) and eigenstrain
// (6 per volume) increments u, and the stress they cause, K u, added to the
// tractions (3 per patch) and stresses (6 per volume).  One warp per row of K.
__global__ void k_perturb(const double *__restrict__ K, long m, long n, int np, const double *__restrict__ u,
                          double *__restrict__ y)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x, nt = (long)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (long r = t >> 5; r < m; r += nt >> 5) {
        const double *Kr = K + r * n;
        double s = 0.0;
        for (long c = lane; c < n; c += 32) s = fma(Kr[c], u[c], s);
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) {
            const long i = r < 3L * np ? 7L * (r / 3) + 2 + r % 3
                                       : 7L * np + 12L * ((r - 3L * np) / 6) + 6 + (r - 3L * np) % 6;
            y[i] += s;
        }
    }
    for (long c = t; c < n; c += nt) {
        const long i = c < 2L * np ? 7L * (c >> 1) + (c & 1) : 7L * np + 12L * ((c - 2L * np) / 6) + (c - 2L * np) % 6;
        y[i] += u[c];
    }
}

// the same with the stress change t = H u already formed (hierarchical matrix)
__global__ void k_perturb_t(long m, long n, int np, const double *__restrict__ t, const double *__restrict__ u,
                            double *__restrict__ y)
{
    const long i0 = (long)blockIdx.x * blockDim.x + threadIdx.x, nt = (long)gridDim.x * blockDim.x;
    for (long r = i0; r < m; r += nt) y[7L * (r / 3) + 2 + r % 3] += t[r];
    for (long c = i0; c < n; c += nt) y[7L * (c >> 1) + (c & 1)] += u[c];
}

int rk_perturb(ucg_ctx *c, const double *u)
{
    if (!c->K && !(c->hm && c->nv == 0)) return UCG_E_STATE;
    if (!c->pert) UCG_CUDA(cudaMalloc(&c->pert, sizeof(double) * c->n));
    UCG_CUDA(cudaMemcpyAsync(c->pert, u, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream));
    const int blocks = (int)std::min<long>((c->m + 7) / 8, 8L * c->sms);
    if (c->K) {
        k_perturb<<<blocks, 256, 0, c->stream>>>(c->K, c->m, c->n, c->nr + c->nt, c->pert, c->st.y);
    } else {
        double *t = hmatrix_t(c);
        hmatrix_apply(c, c->pert, t);
        k_perturb_t<<<blocks, 256, 0, c->stream>>>(c->m, c->n, c->nr + c->nt, t, c->pert, c->st.y);
    }
    c->launches.count++;
    UCG_CUDA(cudaGetLastError());
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

// f(y) for the state currently in st.y into st.k[0]
int rk_odefun(ucg_ctx *c)
{
    Ctl *h = c->ctl_host;
    UCG_CUDA(cudaMemcpyAsync(h, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    h->active = 1;
    h->status = 0;
    h->need_stage1 = 1;
    h->pending = 0;
    h->vmax = 0.0;
    h->nonfinite = 0;
    UCG_CUDA(cudaMemcpyAsync(c->ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    enqueue_stage<1>(c);
    UCG_CUDA(cudaGetLastError());
    UCG_CUDA(cudaMemcpyAsync(h, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    if (h->status) return h->status;
    return h->nonfinite ? UCG_E_NONFINITE : UCG_OK;
}

// fault injection for the tests of the bounded waits
int rk_test_wait_timeout(ucg_ctx *c, unsigned long long wait_ns, int hold)
{
    Ctl *h = c->ctl_host;
    UCG_CUDA(cudaMemcpyAsync(h, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    h->wait_ns = wait_ns;
    h->test_hold = hold;
    h->status = 0;
    UCG_CUDA(cudaMemcpyAsync(c->ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

// ---- allocation-free right-hand side --------------------------------------------
//
// ucg_odefun_noalloc evaluates dydt = f(y) for a fault model whose matrix, state,
// friction parameters and output all live in caller-owned device memory, for
// callers that cannot allocate device memory at the point of the call (code
// running under an external memory manager or an allocation-free real-time
// loop, which must not call cudaMalloc or pull in an allocating library).  The
// only working storage it needs -- the source velocity vector v and the control
// block the kernels read -- lives in the fixed array below.  The array is part
// of the loaded library: every GPU that loads libucg.so holds its 8 MB until
// the process exits.  Calls share it, so calls that overlap on the GPU (on
// different streams without ordering) race on v; the array keeps the last
// call's contents, and the control block is reset at the start of every call.

namespace {

constexpr long NOALLOC_MAX_N = 1L << 20;                // source DOFs (2 per patch)
constexpr long NOALLOC_CTL_DOUBLES = (sizeof(Ctl) + sizeof(double) - 1) / sizeof(double);

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_N + NOALLOC_CTL_DOUBLES];

__global__ void k_noalloc_ctl_reset(Ctl *ctl)
{
    Ctl z;
    memset(&z, 0, sizeof z);
    z.active = 1;
    z.need_stage1 = 1;
    z.step_target = 1;
    z.t_end = 1.0e300;
    *ctl = z;
}

// the call's outcome into the caller's status word, after the other kernels:
// a wait that gave up (UCG_E_TIMEOUT), a NaN/Inf met on the way, or UCG_OK
__global__ void k_noalloc_status(const Ctl *ctl, int *status)
{
    *status = ctl->status ? ctl->status : (ctl->nonfinite ? UCG_E_NONFINITE : UCG_OK);
}

inline bool aligned_to(const void *p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace

}  // namespace ucg

extern "C" int ucg_odefun_noalloc(const double *K, long n, long m, int np, const double *y,
                                  const double *Vpl_cos_rake, const double *Vpl_sin_rake,
                                  const double *a, const double *b, const double *sig, const double *L,
                                  const double *damping, double *dydt, void *stream, int *status)
{
    using namespace ucg;
    const double *dp[] = {y, dydt, Vpl_cos_rake, Vpl_sin_rake, a, b, sig, L, damping};
    if (!K) return UCG_E_BADARG;
    for (const double *p : dp)
        if (!p || !aligned_to(p, sizeof(double))) return UCG_E_BADARG;
    // K's rows go to shared memory by bulk copies, whose source must sit on a
    // 16-byte boundary (n is even, so every row then does)
    if (!aligned_to(K, 16)) return UCG_E_BADARG;
    if (status && !aligned_to(status, sizeof(int))) return UCG_E_BADARG;
    if (np <= 0 || n != 2L * np || m != 3L * np) return UCG_E_BADARG;
    if (n > NOALLOC_MAX_N) return UCG_E_BADARG;   // beyond the fixed scratch: 2^20 source DOFs
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return UCG_E_NODEVICE;
    // the host-side name of the array is not a device address: resolve it on
    // every call with the calling device current (no allocation; the first call
    // on a device may load the module)
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return UCG_E_CUDA;
    double *v = static_cast<double *>(p);
    Ctl *ctl = reinterpret_cast<Ctl *>(v + NOALLOC_MAX_N);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    StageArgs sa{};
    sa.y = y;
    sa.ys = const_cast<double *>(y);   // stage 1 reads y and writes nothing into it
    for (int j = 0; j < 6; j++) sa.k[j] = dydt;
    sa.v = v;
    sa.fr.vpl_c = const_cast<double *>(Vpl_cos_rake);
    sa.fr.vpl_s = const_cast<double *>(Vpl_sin_rake);
    sa.fr.a = const_cast<double *>(a);
    sa.fr.b = const_cast<double *>(b);
    sa.fr.sig = const_cast<double *>(sig);
    sa.fr.L = const_cast<double *>(L);
    sa.fr.damping = const_cast<double *>(damping);
    sa.np = np;
    sa.nvol = 0;
    sa.len = 7L * np;

    int dcount = 0;
    if (cudaDeviceGetAttribute(&dcount, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || dcount <= 0)
        return UCG_E_CUDA;
    const size_t smem = tm_smem_bytes<double>();
    auto kfn = k_traction<1, double>;
    if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return UCG_E_CUDA;
    k_noalloc_ctl_reset<<<1, 1, 0, st>>>(ctl);
    k_prologue<1><<<(np + 127) / 128, 128, 0, st>>>(sa, ctl);
    const int pb = (np + 3) / 4;
    const int grid = pb < dcount ? pb : dcount;
    kfn<<<grid, (MV_WARPS + 1) * 32, smem, st>>>(K, n, n, nullptr, sa, ctl, pb, 0);
    if (status) k_noalloc_status<<<1, 1, 0, st>>>(ctl, status);
    return cudaGetLastError() == cudaSuccess ? UCG_OK : UCG_E_CUDA;
}
