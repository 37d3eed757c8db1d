// Hierarchical (H-matrix) approximation of K for fault models, built and
// applied on the device.
//
// The reference's MATLAB toolbox runs large models through a hierarchical
// matrix (matlab/+unicycle/+ode/+hmmvp/rateandstate.m:71-143, the hmmvp
// library); the Fortran drivers hold K dense.  Here:
//
//   ordering   patches are permuted by a cluster tree: recursive bisection of
//              their centres along the longest extent of the cluster, down to
//              `leaf` patches; every cluster is a contiguous range of the
//              permutation.
//   blocks     a pair of clusters (tau, sigma) is admissible when
//              max(diam tau, diam sigma) <= eta dist(tau, sigma) (bounding boxes
//              of the patches' vertices) and the block fits the build scratch;
//              admissible pairs become low-rank blocks, pairs of leaves that are
//              not admissible dense blocks, other pairs are split (the non-leaf
//              side, or both).
//   build      each block is assembled densely on the device into scratch by the
//              same pair kernels as K (assemble_block), so K itself is never
//              held: N beyond what a dense K fits in HBM works.  A low-rank
//              block is compressed by adaptive cross approximation with partial
//              pivoting (one CTA per block) to relative accuracy eps, then
//              checked against the dense block on a pseudo-random probe
//              vector; a block that fails the check, or whose factors would not
//              be smaller, is kept dense.
//   storage    FP64.  V is stored rank-major (k x n); the rows of U and of the
//              dense blocks are repacked into panels, one per row leaf and chunk
//              of at most 16 KB, each a column-major (rows x columns) slab.
//   product    t = H v: v is gathered into the permuted order (every block's
//              columns become a contiguous slice); z_b = V_b^T v_sigma for every
//              low-rank block (one warp per rank vector); one CTA per chunk
//              copies its panel into shared memory with one bulk copy and one
//              thread per row multiplies it by the matching slices of v or z;
//              a last kernel adds a leaf's chunks in order and writes K's row
//              order.  Every stored byte is read once per product and the
//              summation order is fixed (deterministic).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cuda_bf16.h>
#include <cstring>
#include <numeric>
#include <vector>
#include "ucg_internal.cuh"
#include "blocks.cuh"

namespace ucg {

struct HBlock {              // a block in the permuted element order
    int r0, r1, s0, s1;      // receiver and source element ranges
    int lowrank;             // 1: low-rank candidate (admissible)
};

struct HLowRank {            // device descriptor of a stored low-rank block
    const double *U, *V;     // k x m and k x n, rank-major
    int k, m, n, s0;         // rank, rows, columns, first source element (permuted)
    int r0;                  // first receiver element (permuted)
    int zoff;                // offset of its z in the product's workspace
    long vsoff;              // offset of its V in the split (bf16 hi / lo) copy
};

struct HLeafTerm {           // the rows of one row leaf in one block (or a range of its columns)
    const double *A;         // while building: the block's column-major rows at the leaf (stride lda)
    int lda;                 // while building: the block's m
    int cols;                // columns of this piece
    int xsel;                // 0: dense columns times xp; 1: U columns times z
    long xoff;               // first entry of xp (dense) or z (low-rank) multiplying the piece
};

struct HChunk {              // consecutive terms [q0, q1) of one row leaf, packed contiguously
    int leaf, q0, q1;
    int bytes;               // of its panel (a multiple of 16)
    long off;                // panel offset (doubles)
};

struct HMat {
    int np = 0, leaf = 0;
    double eta = 0, eps = 0;
    std::vector<int> perm;               // permuted position -> element
    int *perm_d = nullptr;
    // storage
    std::vector<void *> allocs;
    size_t bytes = 0;                    // stored factors and dense blocks
    long n_dense = 0, n_lowrank = 0, n_fallback = 0;
    int max_rank = 0;
    double build_ms = 0;
    // product
    HLowRank *lr_d = nullptr;            // low-rank descriptors
    int2 *items_d = nullptr;             // (block, rank index) work items of the first kernel
    long n_items = 0;
    HLeafTerm *terms_d = nullptr;        // per row leaf, its terms (consecutive)
    HChunk *chunks_d = nullptr;          // work of the row kernel
    int *leaf_chunk_d = nullptr;         // per row leaf, its chunks (CSR)
    int n_chunks = 0;
    int *leaf_e0_d = nullptr;            // row leaves: element ranges (permuted)
    int n_leaves = 0, max_leaf = 0;
    double *z_d = nullptr;               // low-rank workspace
    long nz = 0;
    double *part_d = nullptr;            // partial row sums (chunk, row)
    double *xp_d = nullptr;              // the product's input in the permuted order
    double *panel = nullptr;             // the row data of every chunk, chunk after chunk
    long panel_len = 0;                  // doubles
    std::vector<HLowRank> lr_h;          // host copy of the low-rank descriptors
    std::vector<int> leaf_e0_h, leaf_term0_h;   // host copies of the leaves and their term ranges
    std::vector<HLeafTerm> terms_h;
    std::vector<long> term_poff_h;       // panel offset (doubles) of every term
    // split copies (hi and lo bf16 of every value) for UCG_PREC_HMATRIX_SPLIT
    __nv_bfloat16 *ph = nullptr, *pl = nullptr, *vh = nullptr, *vl = nullptr;
    int *status_d = nullptr;             // nonzero: a bulk copy of the row kernel timed out
    double *t_d = nullptr;               // product output (K's row order)
};

namespace {

// ---- cluster tree and block tree (host) -------------------------------------------

struct Node {
    int e0, e1;
    double lo[3], hi[3];
    int c[2];
};

struct TreeBuilder {
    const std::vector<double> &box, &ctr;
    std::vector<int> &perm;
    std::vector<Node> nodes;
    int leaf;

    int build(int e0, int e1)
    {
        Node nd;
        nd.e0 = e0;
        nd.e1 = e1;
        nd.c[0] = nd.c[1] = -1;
        for (int k = 0; k < 3; k++) {
            nd.lo[k] = INFINITY;
            nd.hi[k] = -INFINITY;
        }
        double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int i = e0; i < e1; i++) {
            const int e = perm[i];
            for (int k = 0; k < 3; k++) {
                nd.lo[k] = std::min(nd.lo[k], box[6L * e + k]);
                nd.hi[k] = std::max(nd.hi[k], box[6L * e + 3 + k]);
                clo[k] = std::min(clo[k], ctr[3L * e + k]);
                chi[k] = std::max(chi[k], ctr[3L * e + k]);
            }
        }
        const int id = (int)nodes.size();
        nodes.push_back(nd);
        if (e1 - e0 > leaf) {
            int ax = 0;
            for (int k = 1; k < 3; k++)
                if (chi[k] - clo[k] > chi[ax] - clo[ax]) ax = k;
            const int mid = e0 + (e1 - e0) / 2;
            std::nth_element(perm.begin() + e0, perm.begin() + mid, perm.begin() + e1,
                             [&](int a, int b) { return ctr[3L * a + ax] < ctr[3L * b + ax]; });
            const int a = build(e0, mid);
            const int b = build(mid, e1);
            nodes[id].c[0] = a;
            nodes[id].c[1] = b;
        }
        return id;
    }
};

double diam(const Node &a)
{
    double s = 0;
    for (int k = 0; k < 3; k++) s += (a.hi[k] - a.lo[k]) * (a.hi[k] - a.lo[k]);
    return std::sqrt(s);
}

double dist(const Node &a, const Node &b)
{
    double s = 0;
    for (int k = 0; k < 3; k++) {
        const double d = std::max(0.0, std::max(a.lo[k] - b.hi[k], b.lo[k] - a.hi[k]));
        s += d * d;
    }
    return std::sqrt(s);
}

void block_tree(const std::vector<Node> &nd, int t, int s, double eta, double max_entries, std::vector<HBlock> &out)
{
    const Node &a = nd[t], &b = nd[s];
    const bool la = a.c[0] < 0, lb = b.c[0] < 0;
    const double entries = 6.0 * (a.e1 - a.e0) * (double)(b.e1 - b.e0);
    const bool fits = entries <= max_entries || (la && lb);
    if (fits && std::max(diam(a), diam(b)) <= eta * dist(a, b)) {
        out.push_back({a.e0, a.e1, b.e0, b.e1, 1});
        return;
    }
    if (la && lb) {
        out.push_back({a.e0, a.e1, b.e0, b.e1, 0});
    } else if (la) {
        block_tree(nd, t, b.c[0], eta, max_entries, out);
        block_tree(nd, t, b.c[1], eta, max_entries, out);
    } else if (lb) {
        block_tree(nd, a.c[0], s, eta, max_entries, out);
        block_tree(nd, a.c[1], s, eta, max_entries, out);
    } else {
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) block_tree(nd, a.c[i], b.c[j], eta, max_entries, out);
    }
}

// ---- adaptive cross approximation (device) --------------------------------------------

struct AcaJob {
    const double *B;         // dense block, row-major m x n
    int m, n, kmax;
    double *U, *V;           // kmax x m, kmax x n
    unsigned char *used;     // m row flags
    int *rank;               // out: rank, or -1 when the block stays dense
    double *err;             // out: relative probe error
};

constexpr int ACA_THREADS = 256;
constexpr int ACA_KMAX = 256;

__device__ double aca_probe(long j)
{
    // deterministic pseudo-random value in [-1, 1] (splitmix64 of j)
    unsigned long long x = (unsigned long long)j * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    x ^= x >> 31;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    return (double)(x >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// block-wide sum (every thread gets the result)
__device__ double block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < ACA_THREADS / 32; i++) s += sh[i];
    return s;
}

// block-wide argmax of v >= 0 (ties: lowest index); bi < 0 where no thread had a candidate
__device__ void block_argmax(double v, int idx, double *shv, int *shi, double &bv, int &bi)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (oi >= 0 && (idx < 0 || ov > v || (ov == v && oi < idx))) {
            v = ov;
            idx = oi;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        shv[w] = v;
        shi[w] = idx;
    }
    __syncthreads();
    bv = -1.0;
    bi = -1;
    for (int i = 0; i < ACA_THREADS / 32; i++)
        if (shi[i] >= 0 && (bi < 0 || shv[i] > bv || (shv[i] == bv && shi[i] < bi))) {
            bv = shv[i];
            bi = shi[i];
        }
}

__global__ void __launch_bounds__(ACA_THREADS) k_aca(const AcaJob *jobs, double eps, double check)
{
    const AcaJob J = jobs[blockIdx.x];
    __shared__ double shv[ACA_THREADS / 32];
    __shared__ int shi[ACA_THREADS / 32];
    __shared__ double zs[ACA_KMAX];
    const int m = J.m, n = J.n, tid = threadIdx.x;
    const double *B = J.B;
    for (int i = tid; i < m; i += ACA_THREADS) J.used[i] = 0;
    __syncthreads();
    int k = 0, row = m / 2, misses = 0;
    double frob2 = 0.0;
    while (k < J.kmax) {
        double *v = J.V + (long)k * n;
        double *u = J.U + (long)k * m;
        // residual of the row; its largest entry picks the pivot column
        double best = -1.0;
        int bj = -1;
        for (int j = tid; j < n; j += ACA_THREADS) {
            double r = B[(long)row * n + j];
            for (int l = 0; l < k; l++) r -= J.U[(long)l * m + row] * J.V[(long)l * n + j];
            v[j] = r;
            if (fabs(r) > best) { best = fabs(r); bj = j; }
        }
        if (tid == 0) J.used[row] = 1;
        double pv;
        int pj;
        block_argmax(best, bj, shv, shi, pv, pj);
        if (!(pv > 0.0)) {
            // a zero residual row: try the next unused one
            if (++misses > 16) break;
            int nr = -1;
            for (int i = 0; i < m; i++) {
                const int cand = (row + 1 + i) % m;
                if (!J.used[cand]) { nr = cand; break; }
            }
            __syncthreads();
            if (nr < 0) break;
            row = nr;
            continue;
        }
        const double p = v[pj];
        __syncthreads();
        for (int j = tid; j < n; j += ACA_THREADS) v[j] = v[j] / p;
        // residual of the pivot column
        for (int i = tid; i < m; i += ACA_THREADS) {
            double r = B[(long)i * n + pj];
            for (int l = 0; l < k; l++) r -= J.V[(long)l * n + pj] * J.U[(long)l * m + i];
            u[i] = r;
        }
        __syncthreads();
        // ||S_k||_F^2 update: |u|^2 |v|^2 + 2 sum_l (u_l . u)(v_l . v)
        double a = 0.0, b = 0.0;
        for (int i = tid; i < m; i += ACA_THREADS) a += u[i] * u[i];
        for (int j = tid; j < n; j += ACA_THREADS) b += v[j] * v[j];
        const double nu2 = block_sum(a, shv), nv2 = block_sum(b, shv);
        double cross = 0.0;
        for (int l = 0; l < k; l++) {
            double cu = 0.0, cv = 0.0;
            for (int i = tid; i < m; i += ACA_THREADS) cu += J.U[(long)l * m + i] * u[i];
            for (int j = tid; j < n; j += ACA_THREADS) cv += J.V[(long)l * n + j] * v[j];
            const double su = block_sum(cu, shv);
            cross += su * block_sum(cv, shv);
        }
        frob2 += nu2 * nv2 + 2.0 * cross;
        k++;
        if (sqrt(nu2 * nv2) <= eps * sqrt(fabs(frob2))) break;
        // next row: the largest entry of the new column among the unused rows
        best = -1.0;
        int bi = -1;
        for (int i = tid; i < m; i += ACA_THREADS)
            if (!J.used[i] && fabs(u[i]) > best) { best = fabs(u[i]); bi = i; }
        int ni;
        block_argmax(best, bi, shv, shi, pv, ni);
        if (ni < 0) break;
        row = ni;
    }
    // probe: || B w - U (V^T w) || / || B w || for a pseudo-random w
    const int kk = k;
    for (int l = 0; l < kk; l++) {
        double s = 0.0;
        for (int j = tid; j < n; j += ACA_THREADS) s += J.V[(long)l * n + j] * aca_probe(j);
        s = block_sum(s, shv);
        if (tid == 0) zs[l] = s;
    }
    __syncthreads();
    const int w = tid >> 5, lane = tid & 31;
    double e2 = 0.0, y2 = 0.0;
    for (int i = w; i < m; i += ACA_THREADS / 32) {
        double s = 0.0;
        for (int j = lane; j < n; j += 32) s += B[(long)i * n + j] * aca_probe(j);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        double a = 0.0;
        for (int l = lane; l < kk; l += 32) a += J.U[(long)l * m + i] * zs[l];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        e2 += (s - a) * (s - a);
        y2 += s * s;
    }
    // every lane of a warp holds the same sums; count lane 0's
    const double te = block_sum(lane == 0 ? e2 : 0.0, shv);
    const double ty = block_sum(lane == 0 ? y2 : 0.0, shv);
    if (tid == 0) {
        const double err = ty > 0.0 ? sqrt(te / ty) : (te > 0.0 ? INFINITY : 0.0);
        *J.err = err;
        const bool smaller = (double)kk * (m + n) < 0.5 * (double)m * n;
        *J.rank = (err <= check && smaller) ? kk : -1;
    }
}

// row-major m x n -> column-major
__global__ void k_to_colmajor(const double *__restrict__ a, int m, int n, double *__restrict__ b)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)m * n) return;
    const long j = t / m, i = t % m;
    b[t] = a[i * n + j];
}

// ---- the product --------------------------------------------------------------------

// v in the permuted element order (so that every block's columns are a
// contiguous range of xp)
__global__ void k_hm_gather(const int *__restrict__ perm, int np, const double *__restrict__ v,
                            double *__restrict__ xp)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    reinterpret_cast<double2 *>(xp)[i] = reinterpret_cast<const double2 *>(v)[perm[i]];
}

// z_b[l] = V_b[l, :] . xp(sigma_b): one warp per (block, rank index)
__global__ void k_hm_z(const HLowRank *__restrict__ lr, const int2 *__restrict__ items, long n_items,
                       const double *__restrict__ xp, double *__restrict__ z)
{
    const long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n_items) return;
    const int2 it = items[w];
    const HLowRank b = lr[it.x];
    const double2 *Vl = reinterpret_cast<const double2 *>(b.V + (long)it.y * b.n);
    const double2 *x = reinterpret_cast<const double2 *>(xp + 2L * b.s0);
    double s0 = 0.0, s1 = 0.0;
    for (int j = lane; j < (b.n >> 1); j += 32) {
        const double2 a = Vl[j], xx = x[j];
        s0 = fma(a.x, xx.x, s0);
        s1 = fma(a.y, xx.y, s1);
    }
    double s = s0 + s1;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) z[b.zoff + it.y] = s;
}

// Partial row sums over one chunk of a row leaf's terms: the chunk's panel
// (at most HM_CHUNK_BYTES, contiguous) arrives in shared memory by one bulk
// copy; then one thread per row multiplies its rows of the pieces by their
// slices of xp (dense) or z (low-rank).  k_hm_reduce adds a leaf's chunks in
// order.  Many small CTAs per SM keep many copies in flight.  The wait for the
// copy is bounded (about 4 s); when it runs out the chunk writes NaN, which the
// integrator reports as a non-finite rate, and the kernel flags status.
constexpr long HM_CHUNK_BYTES = 16 * 1024;
constexpr unsigned long long HM_TIMEOUT_NS = 4000000000ull;

__device__ __forceinline__ uint32_t hm_smem(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool hm_try(uint64_t *bar)
{
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(hm_smem(bar)) : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool hm_wait(uint64_t *bar)
{
    if (hm_try(bar)) return true;
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (unsigned it = 1;; it++) {
        if (hm_try(bar)) return true;
        if ((it & 255u) == 0u) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (t - t0 > HM_TIMEOUT_NS) return false;
        }
    }
}

__global__ void __launch_bounds__(128) k_hm_rows(const HLeafTerm *__restrict__ terms,
        const HChunk *__restrict__ chunks, const int *__restrict__ leaf_e0, const double *__restrict__ panel,
        const double *__restrict__ xp, const double *__restrict__ z, double *__restrict__ part, int rows_max,
        int *status)
{
    extern __shared__ __align__(128) double sm[];
    __shared__ __align__(8) uint64_t bar;
    const HChunk ch = chunks[blockIdx.x];
    const int rows = 3 * (leaf_e0[ch.leaf + 1] - leaf_e0[ch.leaf]);
    const int i = threadIdx.x;
    if (ch.bytes == 0) {
        if (i < rows) part[(long)blockIdx.x * rows_max + i] = 0.0;
        return;
    }
    if (i == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(hm_smem(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (i == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(hm_smem(&bar)), "r"(ch.bytes)
                     : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(hm_smem(sm)), "l"(panel + ch.off), "r"(ch.bytes), "r"(hm_smem(&bar)) : "memory");
    }
    const bool ok = hm_wait(&bar);
    if (!ok) {
        if (i == 0) atomicExch(status, 1);
        if (i < rows) part[(long)blockIdx.x * rows_max + i] = nan("");
        hm_wait(&bar);   // the copy may still land in this CTA's shared memory: wait once more (bounded)
        return;
    }
    if (i >= rows) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    long off = 0;
    for (int q = ch.q0; q < ch.q1; q++) {
        const HLeafTerm T = terms[q];
        const double *x = (T.xsel ? z : xp) + T.xoff;
        const double *col = sm + off + i;
        int j = 0;
        for (; j + 3 < T.cols; j += 4) {
            a0 = fma(col[j * rows], x[j], a0);
            a1 = fma(col[(j + 1) * rows], x[j + 1], a1);
            a2 = fma(col[(j + 2) * rows], x[j + 2], a2);
            a3 = fma(col[(j + 3) * rows], x[j + 3], a3);
        }
        for (; j < T.cols; j++) a0 = fma(col[j * rows], x[j], a0);
        off += ((long)rows * T.cols + 7) & ~7L;
    }
    part[(long)blockIdx.x * rows_max + i] = (a0 + a1) + (a2 + a3);
}

// ---- split (hi + lo) form ---------------------------------------------------------------
//
// Every stored value x is kept as its FP32 rounding split into two 16-bit
// planes: hi, the upper half (a bf16 number: sign, exponent, 7 significand
// bits) and lo, the lower 16 significand bits.  hi and lo together give the
// FP32 value exactly (relative error <= 2^-24); the anchored Runge-Kutta
// stages read both for every stage (4 bytes per value, half the FP64 stream)
// and sum in FP64.

__device__ __forceinline__ void split32(double v, __nv_bfloat16 &hi, __nv_bfloat16 &lo)
{
    const uint32_t b = __float_as_uint(__double2float_rn(v));
    hi = __ushort_as_bfloat16((unsigned short)(b >> 16));
    lo = __ushort_as_bfloat16((unsigned short)(b & 0xffffu));
}
__device__ __forceinline__ float join32(__nv_bfloat16 hi, __nv_bfloat16 lo)
{
    return __uint_as_float(((uint32_t)__bfloat16_as_ushort(hi) << 16) | (uint32_t)__bfloat16_as_ushort(lo));
}

__global__ void k_split_flat(const double *__restrict__ x, long n, __nv_bfloat16 *__restrict__ hi,
                             __nv_bfloat16 *__restrict__ lo)
{
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
        split32(x[t], hi[t], lo[t]);
}

struct SplitJob {
    const double *src;
    long n, dst;
};

__global__ void k_split_jobs(const SplitJob *__restrict__ jobs, __nv_bfloat16 *__restrict__ hi,
                             __nv_bfloat16 *__restrict__ lo)
{
    const SplitJob J = jobs[blockIdx.x];
    for (long t = threadIdx.x; t < J.n; t += blockDim.x) split32(J.src[t], hi[J.dst + t], lo[J.dst + t]);
}

template <bool LO>
__global__ void k_hm_z_split(const HLowRank *__restrict__ lr, const int2 *__restrict__ items, long n_items,
                             const double *__restrict__ xp, const __nv_bfloat16 *__restrict__ vh,
                             const __nv_bfloat16 *__restrict__ vl, double *__restrict__ z)
{
    const long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n_items) return;
    const int2 it = items[w];
    const HLowRank b = lr[it.x];
    const long o = b.vsoff + (long)it.y * b.n;
    const __nv_bfloat162 *h2 = reinterpret_cast<const __nv_bfloat162 *>(vh + o);
    const __nv_bfloat162 *l2 = reinterpret_cast<const __nv_bfloat162 *>(vl + o);
    const double2 *x = reinterpret_cast<const double2 *>(xp + 2L * b.s0);
    double s0 = 0.0, s1 = 0.0;
    for (int j = lane; j < (b.n >> 1); j += 32) {
        const double2 xx = x[j];
        double a0, a1;
        if (LO) {
            a0 = join32(h2[j].x, l2[j].x);
            a1 = join32(h2[j].y, l2[j].y);
        } else {
            const float2 a = __bfloat1622float2(h2[j]);
            a0 = a.x;
            a1 = a.y;
        }
        s0 = fma(a0, xx.x, s0);
        s1 = fma(a1, xx.y, s1);
    }
    double s = s0 + s1;
    for (int o2 = 16; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o2);
    if (lane == 0) z[b.zoff + it.y] = s;
}

// k_hm_rows on the split panels: the chunk's hi (and lo) bf16 values arrive by
// bulk copy (a chunk of e values is 2 e bytes per half)
template <bool LO>
__global__ void __launch_bounds__(128) k_hm_rows_split(const HLeafTerm *__restrict__ terms,
        const HChunk *__restrict__ chunks, const int *__restrict__ leaf_e0, const __nv_bfloat16 *__restrict__ ph,
        const __nv_bfloat16 *__restrict__ pl, const double *__restrict__ xp, const double *__restrict__ z,
        double *__restrict__ part, int rows_max, int *status)
{
    extern __shared__ __align__(128) __nv_bfloat16 sb[];
    __shared__ __align__(8) uint64_t bar;
    const HChunk ch = chunks[blockIdx.x];
    const int rows = 3 * (leaf_e0[ch.leaf + 1] - leaf_e0[ch.leaf]);
    const int i = threadIdx.x;
    const long nel = ch.bytes / 8;            // values in the chunk
    const uint32_t half = (uint32_t)(2 * nel);
    if (nel == 0) {
        if (i < rows) part[(long)blockIdx.x * rows_max + i] = 0.0;
        return;
    }
    if (i == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(hm_smem(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (i == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(hm_smem(&bar)),
                     "r"(LO ? 2 * half : half) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(hm_smem(sb)), "l"(ph + ch.off), "r"(half), "r"(hm_smem(&bar)) : "memory");
        if (LO)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         ::"r"(hm_smem(sb + nel)), "l"(pl + ch.off), "r"(half), "r"(hm_smem(&bar)) : "memory");
    }
    const bool ok = hm_wait(&bar);
    if (!__syncthreads_and(ok ? 1 : 0)) {
        if (i == 0) atomicExch(status, 1);
        if (i < rows) part[(long)blockIdx.x * rows_max + i] = nan("");
        hm_wait(&bar);
        return;
    }
    if (i >= rows) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    long off = 0;
    for (int q = ch.q0; q < ch.q1; q++) {
        const HLeafTerm T = terms[q];
        const double *x = (T.xsel ? z : xp) + T.xoff;
        const __nv_bfloat16 *col = sb + off + i;
        auto val = [&](int j) -> double {
            if (LO) return (double)join32(col[(long)j * rows], col[nel + (long)j * rows]);
            return (double)__bfloat162float(col[(long)j * rows]);
        };
        int j = 0;
        for (; j + 3 < T.cols; j += 4) {
            a0 = fma(val(j), x[j], a0);
            a1 = fma(val(j + 1), x[j + 1], a1);
            a2 = fma(val(j + 2), x[j + 2], a2);
            a3 = fma(val(j + 3), x[j + 3], a3);
        }
        for (; j < T.cols; j++) a0 = fma(val(j), x[j], a0);
        off += ((long)rows * T.cols + 7) & ~7L;
    }
    part[(long)blockIdx.x * rows_max + i] = (a0 + a1) + (a2 + a3);
}

struct PackJob {
    const double *src;       // column-major, leading dimension lda
    int lda, rows, cols;
    long dst;                // offset of the rows x cols panel
};

__global__ void k_pack(const PackJob *__restrict__ jobs, double *__restrict__ panel)
{
    const PackJob J = jobs[blockIdx.x];
    const long tot = (long)J.rows * J.cols;
    for (long t = threadIdx.x; t < tot; t += blockDim.x) {
        const long j = t / J.rows, i = t % J.rows;
        panel[J.dst + t] = J.src[j * J.lda + i];
    }
}

// t for one row leaf: blockDim / gs groups of gs threads (gs >= rows) each add
// every ng-th chunk of the leaf, then group 0 adds the groups' sums in order.
__global__ void k_hm_reduce(const int *__restrict__ leaf_e0, const int *__restrict__ leaf_chunk,
                            const int *__restrict__ perm, const double *__restrict__ part, int rows_max,
                            double *__restrict__ t, int gs)
{
    extern __shared__ double sh[];
    const int L = blockIdx.x;
    const int e0 = leaf_e0[L], rows = 3 * (leaf_e0[L + 1] - e0);
    const int c0 = leaf_chunk[L], c1 = leaf_chunk[L + 1];
    const int ng = blockDim.x / gs, g = threadIdx.x / gs, i = threadIdx.x % gs;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    if (i < rows) {
        int c = c0 + g;
        for (; c + 3 * ng < c1; c += 4 * ng) {
            s0 += part[(long)c * rows_max + i];
            s1 += part[(long)(c + ng) * rows_max + i];
            s2 += part[(long)(c + 2 * ng) * rows_max + i];
            s3 += part[(long)(c + 3 * ng) * rows_max + i];
        }
        for (; c < c1; c += ng) s0 += part[(long)c * rows_max + i];
    }
    sh[threadIdx.x] = (s0 + s1) + (s2 + s3);
    __syncthreads();
    if (g == 0 && i < rows) {
        double s = 0.0;
        for (int k = 0; k < ng; k++) s += sh[k * gs + i];
        t[3L * perm[e0 + i / 3] + i % 3] = s;
    }
}

}  // namespace

// ---- host entry points ---------------------------------------------------------------

void hmatrix_free(ucg_ctx *c)
{
    HMat *h = c->hm;
    if (!h) return;
    rk_drop_graph(c);
    cudaStreamSynchronize(c->stream);
    for (void *p : h->allocs) cudaFree(p);
    void *ps[] = {h->perm_d, h->lr_d, h->items_d, h->terms_d, h->chunks_d, h->leaf_chunk_d, h->leaf_e0_d, h->z_d,
                  h->t_d, h->part_d, h->xp_d, h->status_d, h->ph, h->pl, h->vh, h->vl};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete h;
    c->hm = nullptr;
}

int hmatrix_build(ucg_ctx *c, int okada_mode, double eta, double eps, int leaf)
{
    hmatrix_free(c);
    const int np = c->nr + c->nt;
    BlockSources bs;
    int rc = block_sources_build(c, okada_mode, &bs);
    if (rc) {
        c->err = "hierarchical matrix: one patch family (rectangles or triangles) and no volumes";
        return rc;
    }
    HMat *h = new HMat();
    c->hm = h;
    h->np = np;
    h->leaf = leaf;
    h->eta = eta;
    h->eps = eps;
    cudaEvent_t ev0, ev1;
    UCG_CUDA(cudaEventCreate(&ev0));
    UCG_CUDA(cudaEventCreate(&ev1));
    UCG_CUDA(cudaEventRecord(ev0, c->stream));

    // cluster tree and blocks; the build scratch bounds the size of a block
    std::vector<double> box, ctr;
    element_boxes(c, box, ctr);
    h->perm.resize(np);
    std::iota(h->perm.begin(), h->perm.end(), 0);
    TreeBuilder tb{box, ctr, h->perm, {}, leaf};
    tb.build(0, np);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t scratch = std::min<size_t>((size_t)8 << 30, free_b / 4);
    std::vector<HBlock> blocks;
    block_tree(tb.nodes, 0, 0, eta, 0.4 * (double)scratch / sizeof(double), blocks);
    std::vector<int> leaf_e0;
    for (const Node &nd : tb.nodes)
        if (nd.c[0] < 0) leaf_e0.push_back(nd.e0);
    std::sort(leaf_e0.begin(), leaf_e0.end());
    h->n_leaves = (int)leaf_e0.size();
    leaf_e0.push_back(np);
    for (int L = 0; L < h->n_leaves; L++) h->max_leaf = std::max(h->max_leaf, leaf_e0[L + 1] - leaf_e0[L]);
    UCG_CUDA(cudaMalloc(&h->perm_d, sizeof(int) * np));
    UCG_CUDA(cudaMemcpy(h->perm_d, h->perm.data(), sizeof(int) * np, cudaMemcpyHostToDevice));

    double *sc = nullptr;
    UCG_CUDA(cudaMalloc(&sc, scratch));
    struct Done {
        int b;            // block index
        int rank;         // -1: dense
        const double *A;  // dense (column-major) or U
        const double *V;
    };
    std::vector<Done> done;
    // storage: bump allocation over large device chunks; pool 0 keeps V, pool 1
    // holds U and the dense blocks until they are repacked into row panels
    const size_t CHUNK = (size_t)256 << 20;
    size_t chunk_left[2] = {0, 0};
    char *chunk_ptr[2] = {nullptr, nullptr};
    std::vector<void *> temp_allocs;
    auto store = [&](int pool, size_t bytes, double **out) -> int {
        bytes = (bytes + 255) & ~(size_t)255;
        if (bytes > chunk_left[pool]) {
            const size_t sz = std::max(bytes, CHUNK);
            void *p = nullptr;
            cudaError_t e = cudaMalloc(&p, sz);
            if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc(hierarchical matrix storage)");
            (pool == 0 ? h->allocs : temp_allocs).push_back(p);
            chunk_ptr[pool] = (char *)p;
            chunk_left[pool] = sz;
        }
        *out = (double *)chunk_ptr[pool];
        chunk_ptr[pool] += bytes;
        chunk_left[pool] -= bytes;
        return UCG_OK;
    };
    const int MAXJOBS = 4096;
    AcaJob *jobs_d = nullptr;
    int *ranks_d = nullptr;
    double *errs_d = nullptr;
    UCG_CUDA(cudaMalloc(&jobs_d, sizeof(AcaJob) * MAXJOBS));
    UCG_CUDA(cudaMalloc(&ranks_d, sizeof(int) * MAXJOBS));
    UCG_CUDA(cudaMalloc(&errs_d, sizeof(double) * MAXJOBS));
    auto cleanup = [&]() {
        cudaStreamSynchronize(c->stream);
        cudaFree(sc);
        cudaFree(jobs_d);
        cudaFree(ranks_d);
        cudaFree(errs_d);
        block_sources_free(&bs);
    };

    // the blocks in batches that fit the scratch
    size_t bi = 0;
    std::vector<AcaJob> jobs;
    std::vector<int> job_block;
    while (bi < blocks.size()) {
        size_t off = 0;   // in doubles
        jobs.clear();
        job_block.clear();
        std::vector<std::pair<int, size_t>> dense_in_batch;
        while (bi < blocks.size() && (int)jobs.size() < MAXJOBS) {
            const HBlock &B = blocks[bi];
            const long m = 3L * (B.r1 - B.r0), n = 2L * (B.s1 - B.s0);
            const int kmax = (int)std::min<long>(ACA_KMAX, std::min(m, n));
            size_t need = (size_t)m * n + (B.lowrank ? (size_t)kmax * (m + n) + (m + 7) / 8 + 2 : 0);
            need = (need + 31) & ~(size_t)31;
            if ((off + need) * sizeof(double) > scratch) {
                if (off == 0) {
                    cleanup();
                    c->err = "hierarchical matrix: a dense leaf block exceeds the build scratch (use a smaller leaf)";
                    return UCG_E_OOM;
                }
                break;
            }
            double *Bd = sc + off;
            assemble_block(c, bs, h->perm_d + B.r0, B.r1 - B.r0, h->perm_d + B.s0, B.s1 - B.s0, Bd);
            if (B.lowrank) {
                AcaJob J;
                J.B = Bd;
                J.m = (int)m;
                J.n = (int)n;
                J.kmax = kmax;
                J.U = Bd + (size_t)m * n;
                J.V = J.U + (size_t)kmax * m;
                J.used = (unsigned char *)(J.V + (size_t)kmax * n);
                J.rank = ranks_d + jobs.size();
                J.err = errs_d + jobs.size();
                jobs.push_back(J);
                job_block.push_back((int)bi);
            } else {
                dense_in_batch.push_back({(int)bi, off});
            }
            off += need;
            bi++;
        }
        if ((rc = (int)cudaGetLastError())) {
            cleanup();
            return cuda_fail(c, (cudaError_t)rc, "hierarchical matrix block assembly");
        }
        std::vector<int> ranks(jobs.size());
        if (!jobs.empty()) {
            cudaMemcpyAsync(jobs_d, jobs.data(), sizeof(AcaJob) * jobs.size(), cudaMemcpyHostToDevice, c->stream);
            k_aca<<<(int)jobs.size(), ACA_THREADS, 0, c->stream>>>(jobs_d, eps, 10.0 * eps);
            c->launches.count++;
            cudaMemcpyAsync(ranks.data(), ranks_d, sizeof(int) * jobs.size(), cudaMemcpyDeviceToHost, c->stream);
        }
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            cleanup();
            return cuda_fail(c, e, "hierarchical matrix compression");
        }
        // keep the factors of the compressed blocks and column-major copies of the dense ones
        auto keep_dense = [&](int b, const double *src) -> int {
            const HBlock &B = blocks[b];
            const int m = 3 * (B.r1 - B.r0), n = 2 * (B.s1 - B.s0);
            double *d = nullptr;
            int r = store(1, sizeof(double) * (size_t)m * n, &d);
            if (r) return r;
            const long tot = (long)m * n;
            k_to_colmajor<<<(int)((tot + 255) / 256), 256, 0, c->stream>>>(src, m, n, d);
            c->launches.count++;
            h->bytes += sizeof(double) * (size_t)m * n;
            done.push_back({b, -1, d, nullptr});
            return UCG_OK;
        };
        for (auto &d : dense_in_batch) {
            if ((rc = keep_dense(d.first, sc + d.second))) {
                cleanup();
                return rc;
            }
            h->n_dense++;
        }
        for (size_t q = 0; q < jobs.size(); q++) {
            const int b = job_block[q], k = ranks[q];
            if (k < 0) {
                if ((rc = keep_dense(b, jobs[q].B))) {
                    cleanup();
                    return rc;
                }
                h->n_fallback++;
                continue;
            }
            const AcaJob &J = jobs[q];
            double *U = nullptr, *V = nullptr;
            if ((rc = store(1, sizeof(double) * (size_t)k * J.m, &U)) || (rc = store(0, sizeof(double) * (size_t)k * J.n, &V))) {
                cleanup();
                return rc;
            }
            if (k > 0) {
                cudaMemcpyAsync(U, J.U, sizeof(double) * (size_t)k * J.m, cudaMemcpyDeviceToDevice, c->stream);
                cudaMemcpyAsync(V, J.V, sizeof(double) * (size_t)k * J.n, cudaMemcpyDeviceToDevice, c->stream);
            }
            h->bytes += sizeof(double) * (size_t)k * (J.m + J.n);
            h->n_lowrank++;
            h->max_rank = std::max(h->max_rank, k);
            done.push_back({b, k, U, V});
        }
        e = cudaStreamSynchronize(c->stream);   // the scratch is reused by the next batch
        if (e != cudaSuccess) {
            cleanup();
            return cuda_fail(c, e, "hierarchical matrix storage");
        }
    }
    cleanup();

    // product structures, in block-tree order (fixed summation order)
    std::vector<HLowRank> lr;
    std::vector<int2> items;
    std::vector<std::vector<HLeafTerm>> per_leaf(h->n_leaves);
    long zoff = 0;
    auto leaf_of = [&](int e) {
        return (int)(std::upper_bound(leaf_e0.begin(), leaf_e0.end() - 1, e) - leaf_e0.begin()) - 1;
    };
    std::sort(done.begin(), done.end(), [](const Done &a, const Done &b) { return a.b < b.b; });
    for (const Done &d : done) {
        const HBlock &B = blocks[d.b];
        const int m = 3 * (B.r1 - B.r0), n = 2 * (B.s1 - B.s0);
        if (d.rank < 0) {
            for (int L = leaf_of(B.r0); L < h->n_leaves && leaf_e0[L] < B.r1; L++)
                per_leaf[L].push_back({d.A + 3L * (leaf_e0[L] - B.r0), m, n, 0, 2L * B.s0});
        } else if (d.rank > 0) {
            const int id = (int)lr.size();
            lr.push_back({d.A, d.V, d.rank, m, n, B.s0, B.r0, (int)zoff});
            for (int l = 0; l < d.rank; l++) items.push_back(make_int2(id, l));
            for (int L = leaf_of(B.r0); L < h->n_leaves && leaf_e0[L] < B.r1; L++)
                per_leaf[L].push_back({d.A + 3L * (leaf_e0[L] - B.r0), m, d.rank, 1, zoff});
            zoff += d.rank;
        }
    }
    // terms cut into column pieces and grouped into chunks of at most
    // HM_CHUNK_BYTES; every piece's rows are packed into one panel, chunk after
    // chunk, each piece padded to 16 bytes
    std::vector<HLeafTerm> terms;
    std::vector<HChunk> chunks;
    std::vector<int> leaf_chunk(1, 0);
    std::vector<PackJob> pk;
    long poff = 0;
    for (int L = 0; L < h->n_leaves; L++) {
        const int rows = 3 * (leaf_e0[L + 1] - leaf_e0[L]);
        const int maxc = (int)std::max<long>(1, HM_CHUNK_BYTES / (8L * rows + 16));
        HChunk ch{L, (int)terms.size(), (int)terms.size(), 0, poff};
        for (const HLeafTerm &T : per_leaf[L]) {
            for (int c0 = 0; c0 < T.cols; c0 += maxc) {
                const int nc = std::min(maxc, T.cols - c0);
                const long sz = ((long)rows * nc + 7) & ~7L;   // padded to 8 elements (64 / 16 bytes)
                if (ch.bytes + 8L * sz > HM_CHUNK_BYTES) {
                    chunks.push_back(ch);
                    ch = HChunk{L, (int)terms.size(), (int)terms.size(), 0, poff};
                }
                HLeafTerm P = T;
                P.cols = nc;
                P.xoff = T.xoff + c0;
                pk.push_back({T.A + (long)c0 * T.lda, T.lda, rows, nc, poff});
                terms.push_back(P);
                poff += sz;
                ch.q1 = (int)terms.size();
                ch.bytes += (int)(8L * sz);
            }
        }
        chunks.push_back(ch);   // possibly empty: the leaf's rows are then zero
        leaf_chunk.push_back((int)chunks.size());
    }
    h->n_chunks = (int)chunks.size();
    h->leaf_e0_h = leaf_e0;
    h->leaf_term0_h.assign(1, 0);
    for (int L = 0; L < h->n_leaves; L++) h->leaf_term0_h.push_back(chunks[leaf_chunk[L + 1] - 1].q1);
    h->term_poff_h.resize(pk.size());
    for (size_t q = 0; q < pk.size(); q++) h->term_poff_h[q] = pk[q].dst;
    {
        double *panel = nullptr;
        UCG_CUDA(cudaMalloc(&panel, sizeof(double) * std::max<long>(poff, 2)));
        h->allocs.push_back(panel);
        h->panel = panel;
        h->panel_len = poff;
        if (!pk.empty()) {
            PackJob *pk_d = nullptr;
            UCG_CUDA(cudaMalloc(&pk_d, sizeof(PackJob) * pk.size()));
            UCG_CUDA(cudaMemcpy(pk_d, pk.data(), sizeof(PackJob) * pk.size(), cudaMemcpyHostToDevice));
            k_pack<<<(int)pk.size(), 256, 0, c->stream>>>(pk_d, panel);
            c->launches.count++;
            UCG_CUDA(cudaStreamSynchronize(c->stream));
            cudaFree(pk_d);
        }
        for (void *p : temp_allocs) cudaFree(p);
        for (HLowRank &b : lr) b.U = nullptr;   // the product reads U from the panels
        for (HLeafTerm &T : terms) T.A = nullptr;
        h->terms_h = terms;
    }
    h->n_items = (long)items.size();
    h->nz = std::max<long>(zoff, 1);
    UCG_CUDA(cudaMalloc(&h->lr_d, sizeof(HLowRank) * std::max<size_t>(lr.size(), 1)));
    UCG_CUDA(cudaMalloc(&h->items_d, sizeof(int2) * std::max<size_t>(items.size(), 1)));
    UCG_CUDA(cudaMalloc(&h->terms_d, sizeof(HLeafTerm) * std::max<size_t>(terms.size(), 1)));
    UCG_CUDA(cudaMalloc(&h->chunks_d, sizeof(HChunk) * chunks.size()));
    UCG_CUDA(cudaMalloc(&h->leaf_chunk_d, sizeof(int) * leaf_chunk.size()));
    UCG_CUDA(cudaMalloc(&h->leaf_e0_d, sizeof(int) * leaf_e0.size()));
    UCG_CUDA(cudaMalloc(&h->z_d, sizeof(double) * h->nz));
    UCG_CUDA(cudaMalloc(&h->t_d, sizeof(double) * (3L * np + 2)));
    UCG_CUDA(cudaMalloc(&h->xp_d, sizeof(double) * (2L * np + 2)));
    UCG_CUDA(cudaFuncSetAttribute(k_hm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HM_CHUNK_BYTES));
    UCG_CUDA(cudaMalloc(&h->status_d, sizeof(int)));
    UCG_CUDA(cudaMemset(h->status_d, 0, sizeof(int)));
    UCG_CUDA(cudaMalloc(&h->part_d, sizeof(double) * (size_t)h->n_chunks * 3 * h->max_leaf));
    {
        long vs = 0;
        for (HLowRank &b : lr) {
            b.vsoff = vs;
            vs += (long)b.k * b.n;
        }
    }
    h->lr_h = lr;
    if (!lr.empty()) UCG_CUDA(cudaMemcpy(h->lr_d, lr.data(), sizeof(HLowRank) * lr.size(), cudaMemcpyHostToDevice));
    if (!items.empty())
        UCG_CUDA(cudaMemcpy(h->items_d, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice));
    if (!terms.empty())
        UCG_CUDA(cudaMemcpy(h->terms_d, terms.data(), sizeof(HLeafTerm) * terms.size(), cudaMemcpyHostToDevice));
    UCG_CUDA(cudaMemcpy(h->chunks_d, chunks.data(), sizeof(HChunk) * chunks.size(), cudaMemcpyHostToDevice));
    UCG_CUDA(cudaMemcpy(h->leaf_chunk_d, leaf_chunk.data(), sizeof(int) * leaf_chunk.size(), cudaMemcpyHostToDevice));
    UCG_CUDA(cudaMemcpy(h->leaf_e0_d, leaf_e0.data(), sizeof(int) * leaf_e0.size(), cudaMemcpyHostToDevice));
    UCG_CUDA(cudaEventRecord(ev1, c->stream));
    UCG_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    h->build_ms = ms;
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    return UCG_OK;
}

// t = H v (K's row order), enqueued on the context stream
void hmatrix_apply(ucg_ctx *c, const double *v, double *t)
{
    HMat *h = c->hm;
    k_hm_gather<<<(h->np + 255) / 256, 256, 0, c->stream>>>(h->perm_d, h->np, v, h->xp_d);
    if (h->n_items > 0) {
        const long threads = h->n_items * 32;
        k_hm_z<<<(int)((threads + 255) / 256), 256, 0, c->stream>>>(h->lr_d, h->items_d, h->n_items, h->xp_d,
                                                                    h->z_d);
        c->launches.count++;
    }
    const int rows = 3 * h->max_leaf;
    k_hm_rows<<<h->n_chunks, ((rows + 31) / 32) * 32, HM_CHUNK_BYTES, c->stream>>>(
        h->terms_d, h->chunks_d, h->leaf_e0_d, h->panel, h->xp_d, h->z_d, h->part_d, rows, h->status_d);
    const int gs = ((rows + 31) / 32) * 32, nthr = std::max(gs, (1024 / gs) * gs);
    k_hm_reduce<<<h->n_leaves, nthr, sizeof(double) * nthr, c->stream>>>(h->leaf_e0_d, h->leaf_chunk_d, h->perm_d,
                                                                         h->part_d, rows, t, gs);
    c->launches.count += 3;
}

// hi / lo planes of the FP32 copies of the panels and of V (once; kept with the matrix)
int hmatrix_split_build(ucg_ctx *c)
{
    HMat *h = c->hm;
    if (!h) return UCG_E_STATE;
    if (h->ph) return UCG_OK;
    long vn = 0;
    for (const HLowRank &b : h->lr_h) vn += (long)b.k * b.n;
    const long pn = std::max<long>(h->panel_len, 8);
    UCG_CUDA(cudaMalloc(&h->ph, sizeof(__nv_bfloat16) * pn));
    UCG_CUDA(cudaMalloc(&h->pl, sizeof(__nv_bfloat16) * pn));
    UCG_CUDA(cudaMalloc(&h->vh, sizeof(__nv_bfloat16) * std::max<long>(vn, 8)));
    UCG_CUDA(cudaMalloc(&h->vl, sizeof(__nv_bfloat16) * std::max<long>(vn, 8)));
    if (h->panel_len > 0) {
        k_split_flat<<<8 * c->sms, 256, 0, c->stream>>>(h->panel, h->panel_len, h->ph, h->pl);
        c->launches.count++;
    }
    std::vector<SplitJob> jobs;
    for (const HLowRank &b : h->lr_h)
        if (b.k > 0) jobs.push_back({b.V, (long)b.k * b.n, b.vsoff});
    if (!jobs.empty()) {
        SplitJob *jd = nullptr;
        UCG_CUDA(cudaMalloc(&jd, sizeof(SplitJob) * jobs.size()));
        UCG_CUDA(cudaMemcpy(jd, jobs.data(), sizeof(SplitJob) * jobs.size(), cudaMemcpyHostToDevice));
        k_split_jobs<<<(int)jobs.size(), 256, 0, c->stream>>>(jd, h->vh, h->vl);
        c->launches.count++;
        UCG_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(jd);
    }
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

// t = H v on the split copies: hi + lo (lo = true) or hi alone
void hmatrix_apply_split(ucg_ctx *c, const double *v, double *t, bool lo)
{
    HMat *h = c->hm;
    k_hm_gather<<<(h->np + 255) / 256, 256, 0, c->stream>>>(h->perm_d, h->np, v, h->xp_d);
    if (h->n_items > 0) {
        const long threads = h->n_items * 32;
        if (lo)
            k_hm_z_split<true><<<(int)((threads + 255) / 256), 256, 0, c->stream>>>(h->lr_d, h->items_d, h->n_items,
                                                                                 h->xp_d, h->vh, h->vl, h->z_d);
        else
            k_hm_z_split<false><<<(int)((threads + 255) / 256), 256, 0, c->stream>>>(h->lr_d, h->items_d, h->n_items,
                                                                                  h->xp_d, h->vh, h->vl, h->z_d);
        c->launches.count++;
    }
    const int rows = 3 * h->max_leaf;
    const int thr = ((rows + 31) / 32) * 32;
    const size_t smem = (size_t)(lo ? 2 : 1) * 2 * (HM_CHUNK_BYTES / 8);
    if (lo)
        k_hm_rows_split<true><<<h->n_chunks, thr, smem, c->stream>>>(h->terms_d, h->chunks_d, h->leaf_e0_d, h->ph,
                                                                     h->pl, h->xp_d, h->z_d, h->part_d, rows,
                                                                     h->status_d);
    else
        k_hm_rows_split<false><<<h->n_chunks, thr, smem, c->stream>>>(h->terms_d, h->chunks_d, h->leaf_e0_d, h->ph,
                                                                      h->pl, h->xp_d, h->z_d, h->part_d, rows,
                                                                      h->status_d);
    const int gs = thr, nthr = std::max(gs, (1024 / gs) * gs);
    k_hm_reduce<<<h->n_leaves, nthr, sizeof(double) * nthr, c->stream>>>(h->leaf_e0_d, h->leaf_chunk_d, h->perm_d,
                                                                         h->part_d, rows, t, gs);
    c->launches.count += 3;
}

double *hmatrix_t(ucg_ctx *c) { return c->hm ? c->hm->t_d : nullptr; }

bool hmatrix_layout(const ucg_ctx *c, HLayout *out)
{
    const HMat *h = c->hm;
    if (!h) return false;
    out->np = h->np;
    out->n_leaves = h->n_leaves;
    out->perm = h->perm;
    out->leaf_e0 = h->leaf_e0_h;
    out->leaf_term0 = h->leaf_term0_h;
    out->terms.clear();
    for (size_t q = 0; q < h->terms_h.size(); q++) {
        const HLeafTerm &T = h->terms_h[q];
        out->terms.push_back({h->term_poff_h[q], T.cols, T.xsel, T.xoff});
    }
    out->lr.clear();
    for (const HLowRank &b : h->lr_h) out->lr.push_back({b.V, b.k, b.n, b.s0, b.zoff, b.r0, b.m});
    out->panel = h->panel;
    return true;
}

void hmatrix_info(const ucg_ctx *c, long *n_dense, long *n_lowrank, long *n_fallback, size_t *bytes, int *max_rank,
                  double *build_ms)
{
    const HMat *h = c->hm;
    if (n_dense) *n_dense = h ? h->n_dense + h->n_fallback : 0;
    if (n_lowrank) *n_lowrank = h ? h->n_lowrank : 0;
    if (n_fallback) *n_fallback = h ? h->n_fallback : 0;
    if (bytes) *bytes = h ? h->bytes : 0;
    if (max_rank) *max_rank = h ? h->max_rank : 0;
    if (build_ms) *build_ms = h ? h->build_ms : 0.0;
}

}  // namespace ucg
