// C ABI of libucg.so (include/ucg.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include "ucg_internal.cuh"
#include "strainvolume.cuh"

using namespace ucg;

namespace ucg {
int cuda_fail(ucg_ctx *c, cudaError_t e, const char *what)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    if (c) c->err = buf;
    if (e == cudaErrorMemoryAllocation) return UCG_E_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return UCG_E_NODEVICE;
    return UCG_E_CUDA;
}
}  // namespace ucg

static int bad(ucg_ctx *c, const char *msg)
{
    if (c) c->err = msg;
    return UCG_E_BADARG;
}

static int set_err(ucg_ctx *c, int status, const char *msg)
{
    if (c) c->err = msg;
    return status;
}

extern "C" {

const char *ucg_strerror(int s)
{
    switch (s) {
    case UCG_OK: return "ok";
    case UCG_E_BADARG: return "invalid argument";
    case UCG_E_CUDA: return "CUDA error";
    case UCG_E_OOM: return "out of device memory";
    case UCG_E_STEP_UNDERFLOW: return "stepsize underflow in RKQS";
    case UCG_E_NONFINITE: return "non-finite state or rate";
    case UCG_E_TIMEOUT: return "device wait timed out";
    case UCG_E_STATE: return "call out of order";
    case UCG_E_UNSUPPORTED: return "unsupported";
    case UCG_E_NODEVICE: return "no usable CUDA device";
    default: return "unknown status";
    }
}

const char *ucg_last_error(ucg_ctx *c) { return c ? c->err.c_str() : ""; }

int ucg_create(ucg_ctx **out, int device, double mu, double lambda, int flags)
{
    if (!out) return UCG_E_BADARG;
    *out = nullptr;
    if (!(mu > 0.0) || !std::isfinite(lambda) || !(lambda + mu > 0.0)) return UCG_E_BADARG;
    if (flags != UCG_DRIVER_RATESTATE && flags != UCG_DRIVER_VISCOUSCYCLES) return UCG_E_BADARG;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return UCG_E_NODEVICE;
    if (device < 0 || device >= count) return UCG_E_BADARG;
    ucg_ctx *c = new (std::nothrow) ucg_ctx();
    if (!c) return UCG_E_OOM;
    c->device = device;
    c->mu = mu;
    c->lambda = lambda;
    c->driver = flags;
    if ((e = cudaSetDevice(device)) != cudaSuccess || (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        int s = cuda_fail(c, e, "ucg_create");
        delete c;
        return s;
    }
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return UCG_OK;
}

static void free_observation(ucg_ctx *c)
{
    if (c->O) cudaFree(c->O);
    if (c->obs_dev) cudaFree(c->obs_dev);
    c->O = nullptr;
    c->obs_dev = nullptr;
    c->O_bytes = 0;
    c->O_ready = false;
}

static void free_params(ucg_ctx *c)
{
    double **p[] = {&c->fr.vpl_c, &c->fr.vpl_s, &c->fr.a, &c->fr.b, &c->fr.sig, &c->fr.L, &c->fr.damping,
                    &c->rh.ebg, &c->rh.gd0, &c->rh.npow};
    rk_drop_graph(c);
    for (double **q : p) {
        if (*q) cudaFree(*q);
        *q = nullptr;
    }
    for (size_t &n : c->cap_fr) n = 0;
    for (size_t &n : c->cap_rh) n = 0;
}

void ucg_destroy(ucg_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    rk_free(c);
    split_bf16_free(c);
    free_params(c);
    free_observation(c);
    hmatrix_free(c);
    if (c->K) cudaFree(c->K);
    if (c->rcv) cudaFree(c->rcv);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static void invalidate(ucg_ctx *c)
{
    c->assembled = false;
    c->state_ready = false;
    rk_free(c);
    split_bf16_free(c);
    free_observation(c);
    hmatrix_free(c);
    if (c->precision == UCG_PREC_HMATRIX || c->precision == UCG_PREC_HMATRIX_SPLIT) c->precision = UCG_PREC_FP64;
}

int ucg_set_rectangles(ucg_ctx *c, int n, const double *x, const double *L, const double *W,
                       const double *strike, const double *dip)
{
    if (!c || n < 0) return UCG_E_BADARG;
    if (n > 0 && (!x || !L || !W || !strike || !dip)) return bad(c, "null array");
    for (int i = 0; i < n; i++)
        if (!(L[i] > 0.0) || !(W[i] > 0.0) || !std::isfinite(strike[i]) || !std::isfinite(dip[i]) ||
            !std::isfinite(x[3 * i]) || !std::isfinite(x[3 * i + 1]) || !std::isfinite(x[3 * i + 2]))
            return bad(c, "invalid rectangle geometry");
    c->nr = n;
    c->rx.assign(x, x + 3L * n);
    c->rL.assign(L, L + n);
    c->rW.assign(W, W + n);
    c->rstrike.assign(strike, strike + n);
    c->rdip.assign(dip, dip + n);
    invalidate(c);
    c->have_friction = false;
    return UCG_OK;
}

int ucg_set_triangles(ucg_ctx *c, int n, const int *i1, const int *i2, const int *i3, int nve,
                      const double *v)
{
    if (!c || n < 0 || nve < 0) return UCG_E_BADARG;
    if (n > 0 && (!i1 || !i2 || !i3 || !v)) return bad(c, "null array");
    for (int j = 0; j < n; j++) {
        const int ids[3] = {i1[j], i2[j], i3[j]};
        for (int k = 0; k < 3; k++)
            if (ids[k] < 1 || ids[k] > nve) return bad(c, "triangle vertex index out of range (1-based)");
        if (ids[0] == ids[1] || ids[1] == ids[2] || ids[0] == ids[2]) return bad(c, "degenerate triangle");
    }
    for (long k = 0; k < 3L * nve; k++)
        if (!std::isfinite(v[k])) return bad(c, "non-finite vertex");
    c->nt = n;
    c->nve = nve;
    c->ti1.assign(i1, i1 + n);
    c->ti2.assign(i2, i2 + n);
    c->ti3.assign(i3, i3 + n);
    c->tvert.assign(v, v + 3L * nve);
    invalidate(c);
    c->have_friction = false;
    return UCG_OK;
}

int ucg_set_volumes(ucg_ctx *c, int n, const double *x, const double *L, const double *T,
                    const double *W, const double *strike)
{
    if (!c || n < 0) return UCG_E_BADARG;
    if (n > 0 && (!x || !L || !T || !W || !strike)) return bad(c, "null array");
    for (int i = 0; i < n; i++) {
        if (!(L[i] > 0.0) || !(T[i] > 0.0) || !(W[i] > 0.0) || !std::isfinite(strike[i]))
            return bad(c, "invalid strain-volume geometry");
        // strainvolume.f90:1064-1072 stops on a negative source depth
        if (!(x[3 * i + 2] >= 0.0)) return bad(c, "strain-volume depth (q3) must be positive");
    }
    if (n > 0 && !kVolumesBuilt) return set_err(c, UCG_E_UNSUPPORTED, "strain volumes not built");
    c->nv = n;
    c->vx.assign(x, x + 3L * n);
    c->vL.assign(L, L + n);
    c->vT.assign(T, T + n);
    c->vW.assign(W, W + n);
    c->vstrike.assign(strike, strike + n);
    invalidate(c);
    c->have_rheology = false;
    return UCG_OK;
}

// Parameter arrays are rewritten in place when their length is unchanged: the
// captured attempt graph holds their device addresses, so they must stay valid.
// A new length (new geometry) reallocates and drops the graph.
static int upload(ucg_ctx *c, double **dst, size_t *cap, const std::vector<double> &h)
{
    if (*dst && *cap == h.size()) {
        if (!h.empty())
            UCG_CUDA(cudaMemcpyAsync(*dst, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->stream));
        return UCG_OK;
    }
    rk_drop_graph(c);
    if (*dst) cudaFree(*dst);
    *dst = nullptr;
    *cap = 0;
    if (h.empty()) return UCG_OK;
    UCG_CUDA(cudaMalloc(dst, sizeof(double) * h.size()));
    *cap = h.size();
    UCG_CUDA(cudaMemcpyAsync(*dst, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->stream));
    return UCG_OK;
}

int ucg_set_friction(ucg_ctx *c, const double *Vpl, const double *rake, const double *mu0,
                     const double *sig, const double *a, const double *b, const double *L,
                     const double *Vo, const double *damping)
{
    if (!c) return UCG_E_BADARG;
    const int np = c->nr + c->nt;
    if (np > 0 && (!Vpl || !rake || !mu0 || !sig || !a || !b || !L || !Vo || !damping))
        return bad(c, "null array");
    UCG_CUDA(cudaSetDevice(c->device));
    std::vector<double> vc(np), vs(np), va(a, a + np), vb(b, b + np), vsg(sig, sig + np), vL(L, L + np),
        vd(damping, damping + np);
    for (int i = 0; i < np; i++) {
        if (!(L[i] > 0.0) || !std::isfinite(Vpl[i]) || !std::isfinite(rake[i]))
            return bad(c, "invalid friction parameters");
        vc[i] = Vpl[i] * cos(rake[i]);
        vs[i] = Vpl[i] * sin(rake[i]);
    }
    int rc;
    size_t *cap = c->cap_fr;
    if ((rc = upload(c, &c->fr.vpl_c, &cap[0], vc)) || (rc = upload(c, &c->fr.vpl_s, &cap[1], vs)) ||
        (rc = upload(c, &c->fr.a, &cap[2], va)) || (rc = upload(c, &c->fr.b, &cap[3], vb)) ||
        (rc = upload(c, &c->fr.sig, &cap[4], vsg)) || (rc = upload(c, &c->fr.L, &cap[5], vL)) ||
        (rc = upload(c, &c->fr.damping, &cap[6], vd)))
        return rc;
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    c->hVpl.assign(Vpl, Vpl + np);
    c->hrake.assign(rake, rake + np);
    c->hmu0.assign(mu0, mu0 + np);
    c->hsig.assign(sig, sig + np);
    c->ha.assign(a, a + np);
    c->hb.assign(b, b + np);
    c->hL.assign(L, L + np);
    c->hVo.assign(Vo, Vo + np);
    c->hdamp.assign(damping, damping + np);
    c->have_friction = true;
    return UCG_OK;
}

int ucg_set_rheology(ucg_ctx *c, const double *e_bg, const double *gammadot0m, const double *npowerm,
                     int nonlinear_maxwell)
{
    if (!c) return UCG_E_BADARG;
    const int nv = c->nv;
    if (nv > 0 && (!e_bg || !gammadot0m || !npowerm)) return bad(c, "null array");
    UCG_CUDA(cudaSetDevice(c->device));
    std::vector<double> e(e_bg, e_bg + 6L * nv), g(gammadot0m, gammadot0m + nv), p(npowerm, npowerm + nv);
    int rc;
    if ((rc = upload(c, &c->rh.ebg, &c->cap_rh[0], e)) || (rc = upload(c, &c->rh.gd0, &c->cap_rh[1], g)) ||
        (rc = upload(c, &c->rh.npow, &c->cap_rh[2], p)))
        return rc;
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    c->hebg = e;
    c->hgd0 = g;
    c->hnpow = p;
    if (c->rh.nonlinear != (nonlinear_maxwell != 0)) rk_drop_graph(c);   // captured by value
    c->rh.nonlinear = nonlinear_maxwell != 0;
    c->have_rheology = true;
    return UCG_OK;
}

int ucg_assemble(ucg_ctx *c, int okada_mode)
{
    if (!c) return UCG_E_BADARG;
    if (okada_mode != UCG_OKADA_FP64 && okada_mode != UCG_OKADA_REF32IO) return bad(c, "okada_mode");
    if (c->nr + c->nt + c->nv == 0) return set_err(c, UCG_E_STATE, "no elements");
    rk_drop_graph(c);
    split_bf16_free(c);
    int rc = assemble_matrix(c, okada_mode);
    if (rc) return rc;
    if (c->precision == UCG_PREC_SPLIT_BF16 || c->precision == UCG_PREC_SPLIT_PAIR) return split_bf16_build(c);
    return UCG_OK;
}

int ucg_assembly_times(ucg_ctx *c, double *rect_ms, double *tri_ms, double *vol_ms)
{
    if (!c) return UCG_E_BADARG;
    if (!c->assembled) return set_err(c, UCG_E_STATE, "matrix not assembled");
    if (rect_ms) *rect_ms = c->asm_ms[0];
    if (tri_ms) *tri_ms = c->asm_ms[1];
    if (vol_ms) *vol_ms = c->asm_ms[2];
    return UCG_OK;
}

int ucg_dims(ucg_ctx *c, long *n, long *m)
{
    if (!c) return UCG_E_BADARG;
    const int np = c->nr + c->nt;
    if (n) *n = 2L * np + 6L * c->nv;
    if (m) *m = 3L * np + 6L * c->nv;
    return UCG_OK;
}

int ucg_copy_G(ucg_ctx *c, double *G, long ld, long k0, long k1)
{
    if (!c || !G) return UCG_E_BADARG;
    if (!c->assembled || !c->K) return set_err(c, UCG_E_STATE, "matrix not assembled (or FP64 copy released)");
    if (ld < c->n || k0 < 0 || k1 > c->m || k0 > k1) return bad(c, "copy range");
    UCG_CUDA(cudaSetDevice(c->device));
    UCG_CUDA(cudaMemcpy2DAsync(G, sizeof(double) * ld, c->K + k0 * c->n, sizeof(double) * c->n,
                               sizeof(double) * c->n, k1 - k0, cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

int ucg_set_precision(ucg_ctx *c, int precision)
{
    if (!c) return UCG_E_BADARG;
    if (precision != UCG_PREC_FP64 && precision != UCG_PREC_SPLIT_BF16 && precision != UCG_PREC_SPLIT_PAIR &&
        precision != UCG_PREC_HMATRIX &&
        precision != UCG_PREC_HMATRIX_SPLIT)
        return bad(c, "precision");
    if (precision == UCG_PREC_HMATRIX || precision == UCG_PREC_HMATRIX_SPLIT) {
        if (!c->hm) return set_err(c, UCG_E_STATE, "build the hierarchical matrix first (ucg_build_hmatrix)");
        if (precision == UCG_PREC_HMATRIX_SPLIT) {
            UCG_CUDA(cudaSetDevice(c->device));
            int rc = hmatrix_split_build(c);
            if (rc) return rc;
        }
        c->precision = precision;
        return UCG_OK;
    }
    if (precision == UCG_PREC_FP64 && c->assembled && !c->K)
        return set_err(c, UCG_E_STATE, "FP64 matrix was released; re-assemble");
    c->precision = precision;
    if ((precision == UCG_PREC_SPLIT_BF16 || precision == UCG_PREC_SPLIT_PAIR) && c->assembled && !c->Ksp)
        return split_bf16_build(c);
    return UCG_OK;
}

int ucg_keep_fp64(ucg_ctx *c, int keep)
{
    if (!c) return UCG_E_BADARG;
    c->keep_fp64 = keep != 0;
    if (!c->keep_fp64 && c->Ksp && c->K) {
        rk_drop_graph(c);
        cudaStreamSynchronize(c->stream);
        cudaFree(c->K);
        c->K = nullptr;
    }
    return UCG_OK;
}

long ucg_state_len(ucg_ctx *c)
{
    if (!c) return -1;
    return 7L * (c->nr + c->nt) + 12L * c->nv;
}

int ucg_init_state(ucg_ctx *c, double *y, const double *nGm, const double *nQm, const double *nRm,
                   const double *To)
{
    if (!c || !y) return UCG_E_BADARG;
    if (!c->have_friction && c->nr + c->nt > 0) return set_err(c, UCG_E_STATE, "friction not set");
    if (c->nv > 0 && (!c->have_rheology || !nGm || !nQm || !nRm || !To))
        return set_err(c, UCG_E_STATE, "rheology / volume initial-stress parameters missing");
    // initStateVector (ratestate.f90:548-610; viscouscycles.f90:710-820): O(N)
    // host arithmetic on the parameters kept at ucg_set_friction / ucg_set_rheology
    const double lg10 = log(10.0);
    const bool visc = c->driver == UCG_DRIVER_VISCOUSCYCLES;
    const int np = c->nr + c->nt;
    for (int i = 0; i < np; i++) {
        double *yy = y + 7L * i;
        double tau = c->hsig[i] * (c->hmu0[i] + (c->ha[i] - c->hb[i]) * log(c->hVpl[i] / c->hVo[i]));
        tau = visc ? tau + c->hdamp[i] * c->hVpl[i] : tau - c->hdamp[i] * c->hVpl[i];
        yy[0] = 0.0;
        yy[1] = 0.0;
        yy[2] = tau * cos(c->hrake[i]);
        yy[3] = tau * sin(c->hrake[i]);
        yy[4] = 0.0;
        yy[5] = log(c->hL[i] / c->hVpl[i]) / lg10;
        yy[6] = log(c->hVpl[i] * (visc ? 0.98 : 0.99)) / lg10;
    }
    for (int i = 0; i < c->nv; i++) {
        double *yy = y + 7L * np + 12L * i;
        const double *e = &c->hebg[6L * i];
        const double eps = sqrt((e[0] * e[0] + 2 * e[1] * e[1] + 2 * e[2] * e[2] + e[3] * e[3] +
                                 2 * e[4] * e[4] + e[5] * e[5]) / 2.0);
        for (int k = 0; k < 6; k++) yy[k] = 0.0;
        if (0.0 < eps) {
            const double tau = nGm[i] * pow(eps / c->hgd0[i] * exp(nQm[i] / (nRm[i] * To[i])), 1.0 / c->hnpow[i]);
            for (int k = 0; k < 6; k++) yy[6 + k] = tau * e[k] / eps;
        } else {
            for (int k = 0; k < 6; k++) yy[6 + k] = 0.0;
        }
    }
    return UCG_OK;
}

static int ensure_state(ucg_ctx *c)
{
    if (!c->assembled && !c->hm) return set_err(c, UCG_E_STATE, "matrix not assembled");
    if (c->nr + c->nt > 0 && !c->have_friction) return set_err(c, UCG_E_STATE, "friction not set");
    if (c->nv > 0 && !c->have_rheology) return set_err(c, UCG_E_STATE, "rheology not set");
    if (c->precision == UCG_PREC_FP64 && !c->K) return set_err(c, UCG_E_STATE, "FP64 matrix released or not assembled");
    if ((c->precision == UCG_PREC_HMATRIX || c->precision == UCG_PREC_HMATRIX_SPLIT) && !c->hm)
        return set_err(c, UCG_E_STATE, "hierarchical matrix not built");
    if (!c->state_ready) {
        c->state_len = ucg_state_len(c);
        int rc = rk_alloc(c);
        if (rc) return set_err(c, rc, "state allocation failed");
        c->state_ready = true;
    }
    return UCG_OK;
}

static int pull_ctl(ucg_ctx *c)
{
    UCG_CUDA(cudaMemcpyAsync(c->ctl_host, c->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

static int push_ctl(ucg_ctx *c)
{
    UCG_CUDA(cudaMemcpyAsync(c->ctl, c->ctl_host, sizeof(Ctl), cudaMemcpyHostToDevice, c->stream));
    return UCG_OK;
}

static int put_vec(ucg_ctx *c, double *dst, const double *src)
{
    memcpy(c->pin, src, sizeof(double) * c->state_len);
    UCG_CUDA(cudaMemcpyAsync(dst, c->pin, sizeof(double) * c->state_len, cudaMemcpyHostToDevice, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

static int obs_per_point(const ucg_ctx *c) { return c->nv > 0 ? 9 : 3; }

long ucg_record_len(ucg_ctx *c)
{
    if (!c) return 0;
    if (c->rec_host.enabled) return c->rec_host.len;
    const int nobs = c->O_ready ? (int)(c->obs_x.size() / 3) : 0;
    return 4L + 24L * c->rec_host.nelem + (long)obs_per_point(c) * nobs;
}

int ucg_record(ucg_ctx *c, int every, const int *elements, int nelem, long capacity)
{
    if (!c) return UCG_E_BADARG;
    if (capacity < 0 || every < 1 || nelem < 0 || (nelem > 0 && !elements)) return bad(c, "recording arguments");
    const int ne = c->nr + c->nt + c->nv;
    for (int j = 0; j < nelem; j++)
        if (elements[j] < 0 || elements[j] >= ne) return bad(c, "recorded element out of range");
    int rc = ensure_state(c);
    if (rc) return rc;
    UCG_CUDA(cudaSetDevice(c->device));
    if ((rc = pull_ctl(c))) return rc;
    if (c->rec_buf) cudaFree(c->rec_buf);
    if (c->rec_elem) cudaFree(c->rec_elem);
    c->rec_buf = nullptr;
    c->rec_elem = nullptr;
    Rec r{};
    if (capacity > 0) {
        const int nobs = c->O_ready ? (int)(c->obs_x.size() / 3) : 0;
        r.per_point = obs_per_point(c);
        r.len = 4 + 24 * nelem + r.per_point * nobs;
        UCG_CUDA(cudaMalloc(&c->rec_buf, sizeof(double) * (size_t)r.len * (size_t)capacity));
        if (nelem > 0) {
            UCG_CUDA(cudaMalloc(&c->rec_elem, sizeof(int) * nelem));
            UCG_CUDA(cudaMemcpy(c->rec_elem, elements, sizeof(int) * nelem, cudaMemcpyHostToDevice));
        }
        r.buf = c->rec_buf;
        r.cap = capacity;
        r.base = c->ctl_host->accepted;
        r.elem = c->rec_elem;
        r.O = nobs ? c->O : nullptr;
        r.every = every;
        r.nelem = nelem;
        r.nobs = nobs;
        r.enabled = 1;
    }
    if (c->rec_host.enabled != r.enabled) rk_drop_graph(c);   // the attempt gains / loses k_record
    c->rec_host = r;
    c->rec_drained = 0;
    UCG_CUDA(cudaMemcpyAsync(c->rec, &c->rec_host, sizeof(Rec), cudaMemcpyHostToDevice, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    return UCG_OK;
}

int ucg_records(ucg_ctx *c, double *out, long max_records, long *n_records, long *lost)
{
    if (!c || (!out && max_records > 0)) return UCG_E_BADARG;
    if (n_records) *n_records = 0;
    if (lost) *lost = 0;
    if (!c->rec || !c->rec_host.enabled) return UCG_OK;
    UCG_CUDA(cudaSetDevice(c->device));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    long long written = 0;
    UCG_CUDA(cudaMemcpy(&written, &c->rec->written, sizeof written, cudaMemcpyDeviceToHost));
    const long long cap = c->rec_host.cap, len = c->rec_host.len;
    long long start = c->rec_drained;
    if (written - start > cap) {
        if (lost) *lost = (long)(written - start - cap);
        start = written - cap;
    }
    const long long k = std::min<long long>(written - start, max_records);
    for (long long j = 0; j < k;) {
        const long long slot = (start + j) % cap, run = std::min(k - j, cap - slot);
        UCG_CUDA(cudaMemcpy(out + j * len, c->rec_buf + slot * len, sizeof(double) * run * len,
                            cudaMemcpyDeviceToHost));
        j += run;
    }
    c->rec_drained = start + k;
    if (n_records) *n_records = (long)k;
    return UCG_OK;
}

// stop a recording whose layout depends on the observation points
static int stop_recording(ucg_ctx *c)
{
    if (!c->rec || !c->rec_host.enabled) return UCG_OK;
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    rk_drop_graph(c);
    c->rec_host = Rec{};
    UCG_CUDA(cudaMemcpy(c->rec, &c->rec_host, sizeof(Rec), cudaMemcpyHostToDevice));
    if (c->rec_buf) cudaFree(c->rec_buf);
    if (c->rec_elem) cudaFree(c->rec_elem);
    c->rec_buf = nullptr;
    c->rec_elem = nullptr;
    c->rec_drained = 0;
    return UCG_OK;
}

int ucg_set_observation_points(ucg_ctx *c, int nobs, const double *x)
{
    if (!c || nobs < 0 || (nobs > 0 && !x)) return UCG_E_BADARG;
    for (long i = 0; i < 3L * nobs; i++)
        if (!std::isfinite(x[i])) return bad(c, "non-finite observation point");
    UCG_CUDA(cudaSetDevice(c->device));
    int rc = stop_recording(c);
    if (rc) return rc;
    free_observation(c);
    c->obs_x.assign(x, x + 3L * nobs);
    return UCG_OK;
}

int ucg_build_O(ucg_ctx *c, int okada_mode)
{
    if (!c) return UCG_E_BADARG;
    if (okada_mode != UCG_OKADA_FP64 && okada_mode != UCG_OKADA_REF32IO) return bad(c, "okada_mode");
    if (c->nr + c->nt + c->nv == 0) return set_err(c, UCG_E_STATE, "no elements");
    if (c->obs_x.empty()) return set_err(c, UCG_E_STATE, "no observation points");
    UCG_CUDA(cudaSetDevice(c->device));
    int rc = stop_recording(c);
    if (rc) return rc;
    c->O_ready = false;
    return assemble_observation(c, okada_mode);
}

int ucg_observation_info(ucg_ctx *c, int *nobs, int *per_point, double *build_ms)
{
    if (!c) return UCG_E_BADARG;
    if (nobs) *nobs = (int)(c->obs_x.size() / 3);
    if (per_point) *per_point = obs_per_point(c);
    if (build_ms) *build_ms = c->O_ready ? c->obs_ms : 0.0;
    return UCG_OK;
}

int ucg_copy_O(ucg_ctx *c, double *O)
{
    if (!c || !O) return UCG_E_BADARG;
    if (!c->O_ready) return set_err(c, UCG_E_STATE, "O not built");
    UCG_CUDA(cudaSetDevice(c->device));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    UCG_CUDA(cudaMemcpy(O, c->O, c->O_bytes, cudaMemcpyDeviceToHost));
    return UCG_OK;
}

// d (and the faulting / flow sets) at every point, one warp per row of O
__global__ void k_observe_state(const double *__restrict__ O, int np, int nvol, int nobs,
                                const double *__restrict__ y, double *d, double *df, double *dl)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const long n = 2L * np + 6L * nvol;
    for (int k = warp; k < 3 * nobs; k += nw) {
        double sf, sl;
        observe_row(O + (long)k * n, np, nvol, y, sf, sl);
        if ((threadIdx.x & 31) == 0) observe_split(k % 3, sf, sl, d[k], df[k], dl[k]);
    }
}

int ucg_displacements(ucg_ctx *c, const double *y, double *d, double *d_fault, double *d_flow)
{
    if (!c || !y || !d) return UCG_E_BADARG;
    if (!c->O_ready) return set_err(c, UCG_E_STATE, "O not built");
    UCG_CUDA(cudaSetDevice(c->device));
    const long len = 7L * (c->nr + c->nt) + 12L * c->nv;
    const int nobs = (int)(c->obs_x.size() / 3);
    const long rows = 3L * nobs;
    double *buf = nullptr;
    UCG_CUDA(cudaMalloc(&buf, sizeof(double) * (len + 3 * rows)));
    cudaError_t e = cudaMemcpyAsync(buf, y, sizeof(double) * len, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        const int blocks = (int)std::min<long>((rows + 7) / 8, (long)c->sms * 8);
        k_observe_state<<<blocks, 256, 0, c->stream>>>(c->O, c->nr + c->nt, c->nv, nobs, buf, buf + len,
                                                       buf + len + rows, buf + len + 2 * rows);
        c->launches.count++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(d, buf + len, sizeof(double) * rows, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && d_fault)
        e = cudaMemcpyAsync(d_fault, buf + len + rows, sizeof(double) * rows, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess && d_flow)
        e = cudaMemcpyAsync(d_flow, buf + len + 2 * rows, sizeof(double) * rows, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (e != cudaSuccess) return cuda_fail(c, e, "ucg_displacements");
    return UCG_OK;
}

int ucg_build_hmatrix(ucg_ctx *c, int okada_mode, double eta, double eps, int leaf)
{
    if (!c) return UCG_E_BADARG;
    if (okada_mode != UCG_OKADA_FP64 && okada_mode != UCG_OKADA_REF32IO) return bad(c, "okada_mode");
    if (!(eta > 0.0) || !(eps > 0.0 && eps < 1.0) || leaf < 4) return bad(c, "hierarchical matrix parameters");
    if (c->nr + c->nt == 0) return set_err(c, UCG_E_STATE, "no elements");
    UCG_CUDA(cudaSetDevice(c->device));
    rk_drop_graph(c);
    const long n = 2L * (c->nr + c->nt) + 6L * c->nv, m = 3L * (c->nr + c->nt) + 6L * c->nv;
    if (c->state_ready && (c->n != n || c->m != m)) {
        rk_free(c);
        c->state_ready = false;
    }
    c->n = n;
    c->m = m;
    return hmatrix_build(c, okada_mode, eta, eps, leaf);
}

int ucg_hmatrix_info(ucg_ctx *c, long *n_dense, long *n_lowrank, long *bytes, int *max_rank, double *build_ms)
{
    if (!c) return UCG_E_BADARG;
    if (!c->hm) return set_err(c, UCG_E_STATE, "hierarchical matrix not built");
    size_t b = 0;
    hmatrix_info(c, n_dense, n_lowrank, nullptr, &b, max_rank, build_ms);
    if (bytes) *bytes = (long)b;
    return UCG_OK;
}

int ucg_hmatrix_matvec(ucg_ctx *c, const double *x, double *y)
{
    if (!c || !x || !y) return UCG_E_BADARG;
    if (!c->hm) return set_err(c, UCG_E_STATE, "hierarchical matrix not built");
    UCG_CUDA(cudaSetDevice(c->device));
    double *xd = nullptr;
    UCG_CUDA(cudaMalloc(&xd, sizeof(double) * (c->n + 2)));
    cudaError_t e = cudaMemcpyAsync(xd, x, sizeof(double) * c->n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        double *t = hmatrix_t(c);
        hmatrix_apply(c, xd, t);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(y, t, sizeof(double) * c->m, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    }
    cudaFree(xd);
    if (e != cudaSuccess) return cuda_fail(c, e, "ucg_hmatrix_matvec");
    return UCG_OK;
}

int ucg_hmatrix_profile(ucg_ctx *c, int reps, double *ms)
{
    if (!c || reps <= 0 || !ms) return UCG_E_BADARG;
    if (!c->hm) return set_err(c, UCG_E_STATE, "hierarchical matrix not built");
    UCG_CUDA(cudaSetDevice(c->device));
    double *xd = nullptr;
    UCG_CUDA(cudaMalloc(&xd, sizeof(double) * (c->n + 2)));
    UCG_CUDA(cudaMemsetAsync(xd, 0, sizeof(double) * (c->n + 2), c->stream));
    cudaEvent_t e0, e1;
    UCG_CUDA(cudaEventCreate(&e0));
    UCG_CUDA(cudaEventCreate(&e1));
    double *t = hmatrix_t(c);
    hmatrix_apply(c, xd, t);   // warm-up
    UCG_CUDA(cudaEventRecord(e0, c->stream));
    for (int r = 0; r < reps; r++) hmatrix_apply(c, xd, t);
    UCG_CUDA(cudaEventRecord(e1, c->stream));
    UCG_CUDA(cudaEventSynchronize(e1));
    float f = 0.0f;
    cudaEventElapsedTime(&f, e0, e1);
    *ms = (double)f / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(xd);
    return UCG_OK;
}

int ucg_odefun(ucg_ctx *c, double t, const double *y, double *dydt, double *vmax)
{
    (void)t;
    if (!c || !y || !dydt) return UCG_E_BADARG;
    int rc = ensure_state(c);
    if (rc) return rc;
    UCG_CUDA(cudaSetDevice(c->device));
    if ((rc = put_vec(c, c->st.y, y))) return rc;
    rc = rk_odefun(c);
    UCG_CUDA(cudaMemcpyAsync(c->pin, c->st.k[0], sizeof(double) * c->state_len, cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    memcpy(dydt, c->pin, sizeof(double) * c->state_len);
    if (vmax) *vmax = c->ctl_host->vmax;
    c->ctl_host->need_stage1 = 1;   // device y is the caller's; next step re-evaluates
    return rc;
}

int ucg_set_tolerance(ucg_ctx *c, double epsilon, double max_step)
{
    if (!c || !(epsilon > 0.0) || !(max_step > 0.0)) return UCG_E_BADARG;
    c->epsilon = epsilon;
    c->hmax = max_step;
    if (c->ctl_host) {
        int rc = pull_ctl(c);
        if (rc) return rc;
        c->ctl_host->epsilon = epsilon;
        c->ctl_host->hmax = max_step;
        return push_ctl(c);
    }
    return UCG_OK;
}

// run queued attempts until `target` accepted steps (or inactive); polls the
// control block every `batch` attempts
static int drive(ucg_ctx *c, int batch)
{
    for (;;) {
        for (int i = 0; i < batch; i++) rk_enqueue_attempt(c);
        int rc = pull_ctl(c);
        if (rc) return rc;
        if (!c->ctl_host->active || c->ctl_host->status) break;
    }
    rk_enqueue_commit(c);
    return pull_ctl(c);
}

int ucg_rkqs(ucg_ctx *c, double *t, double *y, const double *dydt, const double *yscal, double htry,
             double *hdid, double *hnext, long *nrej)
{
    if (!c || !t || !y || !dydt || !yscal || !hdid || !hnext) return UCG_E_BADARG;
    if (!(htry > 0.0)) return bad(c, "htry must be positive");
    int rc = ensure_state(c);
    if (rc) return rc;
    UCG_CUDA(cudaSetDevice(c->device));
    if ((rc = put_vec(c, c->st.y, y))) return rc;
    // anchored stages need the stage-1 product of this y even though the
    // caller supplies dydt
    if (rk_anchored(c) && (rc = rk_odefun(c))) return set_err(c, rc, ucg_strerror(rc));
    if ((rc = put_vec(c, c->st.k[0], dydt)) || (rc = put_vec(c, c->st.yscal, yscal))) return rc;
    if ((rc = pull_ctl(c))) return rc;
    Ctl *h = c->ctl_host;
    const long acc0 = h->accepted, rej0 = h->rejected;
    h->h = htry;
    h->time = *t;
    h->t_end = INFINITY;
    h->step_target = acc0 + 1;
    h->need_stage1 = 0;
    h->pending = 0;
    h->status = 0;
    h->active = 1;
    h->nonfinite = 0;
    h->errbits = 0;
    h->epsilon = c->epsilon;
    h->hmax = c->hmax;
    if ((rc = push_ctl(c))) return rc;
    if ((rc = drive(c, 1))) return rc;
    if (nrej) *nrej = h->rejected - rej0;
    if (h->status) return set_err(c, h->status, ucg_strerror(h->status));
    UCG_CUDA(cudaMemcpyAsync(c->pin, c->st.y, sizeof(double) * c->state_len, cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    memcpy(y, c->pin, sizeof(double) * c->state_len);
    *hdid = h->hdid;
    *hnext = h->dt_next;
    *t = h->time;
    h->need_stage1 = 1;
    return UCG_OK;
}

int ucg_step(ucg_ctx *c, double *time, double *y, double *dydt, double *dt_next, double *dt_done, long *nrej)
{
    if (!c || !time || !y || !dydt || !dt_next || !dt_done) return UCG_E_BADARG;
    if (!(*dt_next > 0.0)) return bad(c, "dt_next must be positive");
    int rc = ensure_state(c);
    if (rc) return rc;
    UCG_CUDA(cudaSetDevice(c->device));
    if ((rc = put_vec(c, c->st.y, y))) return rc;
    Ctl *h = c->ctl_host;
    if ((rc = pull_ctl(c))) return rc;
    const long rej0 = h->rejected;
    h->h = *dt_next;
    h->time = *time;
    h->t_end = INFINITY;
    h->step_target = h->accepted + 1;
    h->need_stage1 = 1;
    h->pending = 0;
    h->status = 0;
    h->active = 1;
    h->nonfinite = 0;
    h->errbits = 0;
    h->vmax = 0.0;
    h->epsilon = c->epsilon;
    h->hmax = c->hmax;
    if ((rc = push_ctl(c))) return rc;
    if ((rc = drive(c, 1))) return rc;
    if (nrej) *nrej = h->rejected - rej0;
    if (h->status) return set_err(c, h->status, ucg_strerror(h->status));
    UCG_CUDA(cudaMemcpyAsync(c->pin, c->st.y, sizeof(double) * c->state_len, cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaMemcpyAsync(c->pin + c->state_len, c->st.k[0], sizeof(double) * c->state_len,
                             cudaMemcpyDeviceToHost, c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    memcpy(y, c->pin, sizeof(double) * c->state_len);
    memcpy(dydt, c->pin + c->state_len, sizeof(double) * c->state_len);
    *time = h->time;
    *dt_done = h->hdid;
    *dt_next = h->dt_next;
    return UCG_OK;
}

int ucg_set_state(ucg_ctx *c, const double *y, double time, double dt_next)
{
    if (!c || !y || !(dt_next > 0.0)) return UCG_E_BADARG;
    int rc = ensure_state(c);
    if (rc) return rc;
    UCG_CUDA(cudaSetDevice(c->device));
    if ((rc = put_vec(c, c->st.y, y))) return rc;
    if ((rc = pull_ctl(c))) return rc;
    Ctl *h = c->ctl_host;
    h->time = time;
    h->h = dt_next;
    h->dt_next = dt_next;
    h->clamped = 0;
    // perturbations at or after the new time are pending again
    for (auto &ev : c->events) ev.applied = ev.time < time;
    h->need_stage1 = 1;
    h->pending = 0;
    h->status = 0;
    h->nonfinite = 0;
    h->errbits = 0;
    h->epsilon = c->epsilon;
    h->hmax = c->hmax;
    return push_ctl(c);
}

int ucg_get_state(ucg_ctx *c, double *y, double *time, double *dt_next, long *accepted, long *rejected)
{
    if (!c) return UCG_E_BADARG;
    if (!c->state_ready) return set_err(c, UCG_E_STATE, "no device state");
    UCG_CUDA(cudaSetDevice(c->device));
    int rc = pull_ctl(c);
    if (rc) return rc;
    if (y) {
        UCG_CUDA(cudaMemcpyAsync(c->pin, c->st.y, sizeof(double) * c->state_len, cudaMemcpyDeviceToHost, c->stream));
        UCG_CUDA(cudaStreamSynchronize(c->stream));
        memcpy(y, c->pin, sizeof(double) * c->state_len);
    }
    if (time) *time = c->ctl_host->time;
    if (dt_next) *dt_next = c->ctl_host->h;
    if (accepted) *accepted = c->ctl_host->accepted;
    if (rejected) *rejected = c->ctl_host->rejected;
    return UCG_OK;
}

// apply every pending perturbation whose time has been reached; the next step
// restarts from the reference's initial tentative step
static int apply_due_events(ucg_ctx *c)
{
    Ctl *h = c->ctl_host;
    for (auto &ev : c->events) {
        if (ev.applied || ev.time > h->time) continue;
        int rc = rk_perturb(c, ev.u.data());
        if (rc) return set_err(c, rc, "perturbations need the FP64 matrix (keep_fp64)");
        ev.applied = true;
        h->need_stage1 = 1;
        h->pending = 0;
        h->h = std::min(1.0e-3, c->hmax);
        h->dt_next = h->h;
        h->clamped = 0;
    }
    return UCG_OK;
}

int ucg_run(ucg_ctx *c, double t_end, long max_steps, long *steps)
{
    if (!c || max_steps < 0) return UCG_E_BADARG;
    if (!c->state_ready) return set_err(c, UCG_E_STATE, "call ucg_set_state first");
    UCG_CUDA(cudaSetDevice(c->device));
    int rc = pull_ctl(c);
    if (rc) return rc;
    Ctl *h = c->ctl_host;
    const long acc0 = h->accepted;
    if (max_steps == 0 || h->time >= t_end) {
        if (steps) *steps = 0;
        return UCG_OK;
    }
    // segments between perturbation times: each ends exactly on the next
    // pending perturbation, which is applied before the following segment
    for (;;) {
        if ((rc = apply_due_events(c))) return rc;
        double t_next = INFINITY;
        for (const auto &ev : c->events)
            if (!ev.applied && ev.time > h->time) t_next = std::min(t_next, ev.time);
        const bool stop = t_next < t_end;
        h->t_end = stop ? t_next : t_end;
        h->stop_on = stop ? 1 : 0;
        h->t_stop = stop ? t_next : 0.0;
        h->clamped = 0;
        if (stop && h->time + h->h > t_next) {
            h->h = t_next - h->time;
            h->clamped = 1;
        }
        h->step_target = acc0 + max_steps;
        h->status = 0;
        h->active = 1;
        h->nonfinite = 0;
        h->epsilon = c->epsilon;
        h->hmax = c->hmax;
        if ((rc = push_ctl(c))) return rc;
        // queue attempts in batches sized to the remaining steps
        const long left = acc0 + max_steps - h->accepted;
        rc = drive(c, left < 32 ? (int)left : 32);
        if (rc) return rc;
        if (h->status || !stop || h->accepted >= acc0 + max_steps || h->time < t_next) break;
    }
    h->stop_on = 0;
    h->clamped = 0;
    if ((rc = push_ctl(c))) return rc;
    if (steps) *steps = h->accepted - acc0;
    if (h->status) return set_err(c, h->status, ucg_strerror(h->status));
    return UCG_OK;
}

int ucg_add_event(ucg_ctx *c, double time, const double *u)
{
    if (!c || !u || !std::isfinite(time)) return UCG_E_BADARG;
    const long n = 2L * (c->nr + c->nt) + 6L * c->nv;
    if (n == 0) return set_err(c, UCG_E_STATE, "no elements");
    for (long i = 0; i < n; i++)
        if (!std::isfinite(u[i])) return bad(c, "non-finite perturbation");
    ucg_ctx::Event ev{time, std::vector<double>(u, u + n), false};
    auto it = c->events.begin();
    while (it != c->events.end() && it->time <= time) ++it;
    c->events.insert(it, ev);
    return UCG_OK;
}

int ucg_clear_events(ucg_ctx *c)
{
    if (!c) return UCG_E_BADARG;
    c->events.clear();
    return UCG_OK;
}

int ucg_apply_perturbation(ucg_ctx *c, const double *u)
{
    if (!c || !u) return UCG_E_BADARG;
    if (!c->state_ready) return set_err(c, UCG_E_STATE, "call ucg_set_state first");
    UCG_CUDA(cudaSetDevice(c->device));
    int rc = pull_ctl(c);
    if (rc) return rc;
    if ((rc = rk_perturb(c, u))) return set_err(c, rc, "perturbations need the FP64 matrix (keep_fp64)");
    c->ctl_host->need_stage1 = 1;
    c->ctl_host->pending = 0;
    return push_ctl(c);
}

long ucg_launch_count(ucg_ctx *c) { return c ? c->launches.count : -1; }

void *ucg_stream(ucg_ctx *c) { return c ? (void *)c->stream : nullptr; }

int ucg_profile_traction(ucg_ctx *c, int reps, double *ms)
{
    if (!c || reps <= 0 || !ms) return UCG_E_BADARG;
    if (!c->state_ready) return set_err(c, UCG_E_STATE, "no device state");
    UCG_CUDA(cudaSetDevice(c->device));
    return rk_profile_traction(c, reps, ms);
}

int ucg_test_wait_timeout(ucg_ctx *c, long wait_ns, int hold)
{
    if (!c || wait_ns < 0) return UCG_E_BADARG;
    int rc = ensure_state(c);
    if (rc) return rc;
    UCG_CUDA(cudaSetDevice(c->device));
    rk_drop_graph(c);   // the captured attempt reads the control block anyway; start clean
    return rk_test_wait_timeout(c, (unsigned long long)wait_ns, hold != 0);
}

}  // extern "C"
