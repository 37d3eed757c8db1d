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
};

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
    __nv_bfloat16 *Khi = nullptr, *Klo = nullptr;   // Khi: interleaved (hi, lo) pairs
    __nv_bfloat16 *Khi_plane = nullptr;              // hi alone, same row stride
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
    double *pin = nullptr;       // pinned staging (state length * 2)
    long state_len = 0;
    bool state_ready = false;

    cudaGraphExec_t attempt_graph = nullptr;
    int graph_precision = -1;
    int sms = 148;

    ucg::Launches launches;
};

namespace ucg {

// assemble.cu
int assemble_matrix(ucg_ctx *c, int okada_mode);
// rk.cu
int rk_alloc(ucg_ctx *c);
void rk_free(ucg_ctx *c);
int rk_odefun(ucg_ctx *c);                  // k[0] = f(y) on device, sets vmax
int rk_profile_traction(ucg_ctx *c, int reps, double *ms);
void rk_enqueue_attempt(ucg_ctx *c);        // one Cash-Karp attempt + control
void rk_enqueue_commit(ucg_ctx *c);         // copy a pending candidate into y
bool rk_anchored(const ucg_ctx *c);         // stages contract increments over the stage-1 anchor
void rk_drop_graph(ucg_ctx *c);             // before freeing anything the attempt graph reads
int split_bf16_build(ucg_ctx *c);
void split_bf16_free(ucg_ctx *c);

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
