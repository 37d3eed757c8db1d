// Internal state of a libucg context and the host-side launch wrappers shared
// by the translation units of the library.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <string>
#include <vector>
#include "../../include/ucg.h"

namespace ucg {
struct HMat;

// Device-resident integrator control block (one per context).
struct Ctl {
    double h;          // step size of the current attempt
    double time;       // simulated time
    double dt_next;    // suggested next step (RKQSm hnext)
    double hdid;       // last accepted step
    double t_end;      // stop when time >= t_end
    double epsilon;    // ode45 `epsilon`
    double hmax;       // ode45 `maximumTimeStep`
    unsigned long long errbits;   // max |yerr/yscal| as ordered bits (non-negative)
    long long accepted, rejected, step_target;
    int need_stage1;   // state changed: evaluate f(y) and yscal
    int pending;       // accepted candidate not yet copied into y
    int status;        // UCG_OK / UCG_E_STEP_UNDERFLOW / UCG_E_NONFINITE
    int active;        // 0 once t_end or step_target is reached
    int nonfinite;     // set by kernels that meet a NaN/Inf
    double vmax;       // max patch velocity at the last f(y)
    // landing on a perturbation time: with stop_on set, no step crosses t_stop;
    // the step that reaches it ends exactly on it (clamped marks that attempt)
    double t_stop;
    int stop_on, clamped;
    // fault injection for tests of the bounded waits (ucg_test_wait_timeout):
    // wait_ns != 0 replaces the 4 s limit of the traction product's waits;
    // test_hold makes the product's first CTA issue no copies, so that its
    // consumers wait on data that never comes and give up
    unsigned long long wait_ns;
    int test_hold, pad_;
};

// Device-side output recorder (the reference's export/exportPoints,
// ratestate.f90:405-537): at the start of every `every`-th accepted step, one
// record of time, dt_done, max V, the state and rate of the listed elements and
// the observation-point displacements O u, written into a ring buffer.
struct Rec {
    double *buf;            // cap records of len doubles
    long long cap, base;    // ring capacity; accepted steps when recording started
    long long written;      // records written since recording started
    const int *elem;        // listed elements (0-based, patches then volumes)
    const double *O;        // 3 nobs x n observation-point displacement kernels (row-major)
    int every, nelem, nobs, len;
    int per_point;          // 3 (total) or, with volumes, 9 (total, faulting, flow)
    int enabled;
};

// Displacement of observation-point row Ok (one row of O) for the state y
// (exportPoints: slip of every patch, strain of every volume): the sums over
// the fault columns (sf) and over the volume columns (sl), reduced over the
// warp; every lane of the calling warp receives both.
__device__ inline void observe_row(const double *__restrict__ Ok, int np, int nvol, const double *__restrict__ y,
                                   double &sf, double &sl)
{
    const int lane = threadIdx.x & 31;
    const long nf = 2L * np, n = nf + 6L * nvol;
    double a = 0.0, b = 0.0;
    for (long c = lane; c < nf; c += 32) a = fma(Ok[c], y[7L * (c >> 1) + (c & 1)], a);
    for (long c = nf + lane; c < n; c += 32) {
        const long v = c - nf;
        b = fma(Ok[c], y[7L * np + 12L * (v / 6) + v % 6], b);
    }
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, off);
        b += __shfl_xor_sync(0xffffffffu, b, off);
    }
    sf = a;
    sl = b;
}

// The three displacement sets of viscouscycles' exportPoints from the two
// partial sums of component c: total (O), "faulting" (Of) and "flow" (Ol).
// buildO (greens.f90:423-430) stores a volume's vertical column in Of rather
// than Ol, so the down component of the faulting set includes the volumes'
// and the flow set's down component is zero; kept for identical output.
__device__ __forceinline__ void observe_split(int c, double sf, double sl, double &d, double &df, double &dl)
{
    d = sf + sl;
    df = (c == 2) ? sf + sl : sf;
    dl = (c == 2) ? 0.0 : sl;
}

// Per-element constitutive data, structure of arrays.
struct Friction {
    double *vpl_c, *vpl_s;   // Vpl*cos(rake), Vpl*sin(rake)
    double *a, *b, *sig, *L, *damping;
};
struct Rheology {
    double *ebg;             // 6 per volume
    double *gd0;             // ngammadot0m
    double *npow;            // npowerm
    int nonlinear;
};

// Cash-Karp stage buffers and state.
struct Stages {
    double *y, *ycand, *ytmp, *yerr, *yscal;
    double *k[6];            // k[0] = dydt (stage 1), k[1..5] = AK2..AK6
    double *v;               // source-DOF velocity / strain-rate vector (n)
    double *t;               // receiver traction / stress (m) for odefun reads
    double *v1, *t1;         // stage-1 anchor of the split-BF16 product (n, m)
};

struct Launches {
    long count = 0;
};

}  // namespace ucg

struct ucg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    double mu = 0, lambda = 0;
    int driver = UCG_DRIVER_RATESTATE;
    std::string err;

    // host copies of geometry
    int nr = 0, nt = 0, nv = 0, nve = 0;
    std::vector<double> rx, rL, rW, rstrike, rdip;
    std::vector<int> ti1, ti2, ti3;
    std::vector<double> tvert;
    std::vector<double> vx, vL, vT, vW, vstrike;

    // matrix: K row-major (m rows = receiver DOFs, n cols = source DOFs)
    long n = 0, m = 0;
    double *K = nullptr;
    int okada_mode = -1;
    bool assembled = false;
    double asm_ms[3] = {0.0, 0.0, 0.0};   // device time of the last assembly: rect, tri, vol sources
    int precision = UCG_PREC_FP64;
    bool keep_fp64 = true;
    float *Ksp = nullptr;                            // K/s in FP32: bf16 hi bits + 16-bit lo extension
    __half *Khi_plane = nullptr;                     // fp16 of K/s (stage increments), same row stride
    float *Kscale = nullptr;   // per row
    long ldk_split = 0;        // row stride of the split matrix (n padded to a multiple of 8)

    // receivers: 12 doubles per element (xc, sv, dv, nv)
    double *rcv = nullptr;

    // constitutive parameters (host copies for the state initialisation)
    std::vector<double> hVpl, hrake, hmu0, hsig, ha, hb, hL, hVo, hdamp;
    std::vector<double> hebg, hgd0, hnpow;
    bool have_friction = false, have_rheology = false;
    ucg::Friction fr{};
    ucg::Rheology rh{};
    size_t cap_fr[7] = {0, 0, 0, 0, 0, 0, 0};   // allocated lengths of the arrays above
    size_t cap_rh[3] = {0, 0, 0};

    // integrator
    double epsilon = 1.0e-6;
    double hmax = 1.7976931348623158e308;
    ucg::Stages st{};
    ucg::Ctl *ctl = nullptr;     // device
    ucg::Ctl *ctl_host = nullptr; // pinned mirror
    ucg::Rec *rec = nullptr;      // device recorder block (allocated with the integrator)
    ucg::Rec rec_host{};          // host copy of its settings
    long long rec_drained = 0;    // records handed to the caller
    int *rec_elem = nullptr;      // device copy of the listed elements
    double *rec_buf = nullptr;
    // observation points (north, east, down) and their displacement kernels
    std::vector<double> obs_x;
    double *obs_dev = nullptr;
    double *O = nullptr;         // 3 nobs x n, row-major
    size_t O_bytes = 0;
    bool O_ready = false;
    double obs_ms = 0.0;         // device time of the last O assembly
    double *pin = nullptr;       // pinned staging (state length * 2)
    long state_len = 0;
    bool state_ready = false;

    // coseismic perturbations (ucg_add_event): applied by ucg_run when the
    // integration reaches their time; u has the source-DOF layout of K's columns
    struct Event {
        double time;
        std::vector<double> u;
        bool applied;
    };
    std::vector<Event> events;
    double *pert = nullptr;      // device copy of the perturbation being applied (n)

    ucg::HMat *hm = nullptr;     // hierarchical approximation of K (hmatrix.cu)

    cudaGraphExec_t attempt_graph = nullptr;
    int graph_precision = -1;
    long graph_launches = 0;     // kernels in one launch of the attempt graph
    int sms = 148;

    ucg::Launches launches;
};

namespace ucg {

// assemble.cu
int assemble_matrix(ucg_ctx *c, int okada_mode);
int assemble_observation(ucg_ctx *c, int okada_mode);   // O for c->obs_x (sets O_ready)
// rk.cu
int rk_alloc(ucg_ctx *c);
void rk_free(ucg_ctx *c);
int rk_odefun(ucg_ctx *c);                  // k[0] = f(y) on device, sets vmax
int rk_test_wait_timeout(ucg_ctx *c, unsigned long long wait_ns, int hold);
int rk_profile_traction(ucg_ctx *c, int reps, double *ms);
void rk_enqueue_attempt(ucg_ctx *c);        // one Cash-Karp attempt + control
void rk_enqueue_commit(ucg_ctx *c);         // copy a pending candidate into y
bool rk_anchored(const ucg_ctx *c);         // stages contract increments over the stage-1 anchor
int rk_perturb(ucg_ctx *c, const double *u); // y += slip/strain u and the stress change K u (host u)
void rk_drop_graph(ucg_ctx *c);             // before freeing anything the attempt graph reads
int split_bf16_build(ucg_ctx *c);
void split_bf16_free(ucg_ctx *c);
// hmatrix.cu
int hmatrix_build(ucg_ctx *c, int okada_mode, double eta, double eps, int leaf);
void hmatrix_free(ucg_ctx *c);
void hmatrix_apply(ucg_ctx *c, const double *v, double *t);   // t = H v, K's row order
int hmatrix_split_build(ucg_ctx *c);                          // bf16 hi / lo copies (UCG_PREC_HMATRIX_SPLIT)
void hmatrix_apply_split(ucg_ctx *c, const double *v, double *t, bool lo);
double *hmatrix_t(ucg_ctx *c);                                 // the product's output buffer
void hmatrix_info(const ucg_ctx *c, long *n_dense, long *n_lowrank, long *n_fallback, size_t *bytes,
                  int *max_rank, double *build_ms);

// The structure of a built hierarchical matrix, for consumers that lay its
// stored values out again (the ensemble's tensor-core images).  Host vectors;
// the value pointers are device addresses owned by the matrix.
struct HLayout {
    struct Term {                // one column piece of a row leaf's row panel
        long poff;               // offset (doubles) of its rows x cols column-major slab in `panel`
        int cols;
        int xsel;                // 0: columns of the permuted input xp; 1: rank entries of z
        long xoff;               // first xp column or z entry
    };
    struct LowRank {             // a stored low-rank block
        const double *V;         // k x n, rank-major
        int k, n, s0, zoff;      // rank, columns, first source element (permuted), z offset
        int r0, m;               // first receiver element (permuted), rows
    };
    int np = 0, n_leaves = 0;
    std::vector<int> perm;       // permuted position -> element
    std::vector<int> leaf_e0;    // n_leaves + 1 element offsets of the row (and column) leaves
    std::vector<int> leaf_term0; // n_leaves + 1 offsets into terms
    std::vector<Term> terms;
    std::vector<LowRank> lr;
    const double *panel = nullptr;
};
bool hmatrix_layout(const ucg_ctx *c, HLayout *out);

// mlp.cu: device addresses of a step-size model's FP16 weights and standardisation
}  // namespace ucg
namespace ucg { namespace mlp { struct Norm; } }
namespace ucg {
void mlp_device_params(const ucg_mlp *m, const __half **P, const mlp::Norm **N);

// error helper: records the CUDA error text and maps to a status
int cuda_fail(ucg_ctx *c, cudaError_t e, const char *what);
#define UCG_CUDA(call)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return ucg::cuda_fail(c, e_, #call); \
    } while (0)

}  // namespace ucg
