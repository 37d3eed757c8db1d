// Training and inference of the step-size perceptron (mlp.cuh) on the device,
// with hand-written kernels:
//
//   k_mlp_grad    one CTA per 128 samples, one thread per sample: forward pass
//                 with FP16 weights and activations (weights staged in shared
//                 memory, activations stored feature-major so that the threads
//                 of a warp read consecutive words), squared-error loss,
//                 backward pass per sample, then the weight gradients as
//                 sums over the CTA's samples (each thread owns a set of
//                 weights and loops over the samples), added to the global
//                 FP32 gradient with one atomic per weight and CTA.
//   k_mlp_adam    Adam on the FP32 master weights, refreshes the FP16 copy and
//                 clears the gradient.
//   k_mlp_predict the controllers' own single-sample evaluation
//                 (mlp::eval_warp), one warp per sample.
//
// Loss: 0.5 (y_hat - label_hat)^2 averaged over the batch, in standardised
// units.  Training data are the integrator's own traces (ensemble.cu records
// them); the label of a trace is the step size that would have met half the
// tolerance on the next step's first attempt (log10 h + 0.2 log10(0.5/errmax),
// limited to a factor 10 either way).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <numeric>
#include <random>
#include <string>
#include <vector>
#include "ucg_internal.cuh"
#include "mlp.cuh"

namespace ucg {
namespace mlp {

constexpr int TB = 128;          // samples (threads) per CTA
constexpr int ZS = TB + 1;       // padded row of FP32 per-feature arrays
constexpr int AS = TB + 2;       // padded row of FP16 per-feature arrays

struct GradSmem {
    __half w[NPARAM + 1];
    __half a0[NIN][AS];
    __half a1[NH][AS], a2[NH][AS], a3[NH][AS];
    float z1[NH][ZS], z2[NH][ZS], z3[NH][ZS];   // pre-activations, then their gradients
    float dout[TB];
    float loss[TB / 32];
};

__global__ void __launch_bounds__(TB) k_mlp_grad(const __half *__restrict__ P, const Norm *__restrict__ Nn,
                                                  const float *__restrict__ X, const float *__restrict__ Y,
                                                  const int *__restrict__ idx, long n, float inv_batch,
                                                  float *__restrict__ G, double *__restrict__ loss_sum)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem &S = *reinterpret_cast<GradSmem *>(smem_raw);
    const Norm N = *Nn;
    const int s = threadIdx.x;
    for (int p = s; p < NPARAM; p += TB) S.w[p] = P[p];
    const long j = blockIdx.x * (long)TB + s;
    const bool valid = j < n;
    const long r = valid ? (idx ? (long)idx[j] : j) : 0;
    for (int i = 0; i < NIN; i++)
        S.a0[i][s] = __float2half(valid ? (X[r * NIN + i] - N.xm[i]) / N.xs[i] : 0.0f);
    __syncthreads();

    // forward
    for (int o = 0; o < NH; o++) {
        float z = __half2float(S.w[OFF_B1 + o]);
        for (int i = 0; i < NIN; i++) z += __half2float(S.w[OFF_W1 + o * NIN + i]) * __half2float(S.a0[i][s]);
        S.z1[o][s] = z;
        S.a1[o][s] = __float2half(gelu_f(z));
    }
    for (int o = 0; o < NH; o++) {
        float z = __half2float(S.w[OFF_B2 + o]);
        for (int i = 0; i < NH; i++) z += __half2float(S.w[OFF_W2 + o * NH + i]) * __half2float(S.a1[i][s]);
        S.z2[o][s] = z;
        S.a2[o][s] = __float2half(gelu_f(z));
    }
    float out = __half2float(S.w[OFF_B4]);
    for (int o = 0; o < NH; o++) {
        float z = __half2float(S.w[OFF_B3 + o]);
        for (int i = 0; i < NH; i++) z += __half2float(S.w[OFF_W3 + o * NH + i]) * __half2float(S.a2[i][s]);
        S.z3[o][s] = z;
        const __half a = __float2half(gelu_f(z));
        S.a3[o][s] = a;
        out += __half2float(S.w[OFF_W4 + o]) * __half2float(a);
    }
    const float d = valid ? out - (Y[r] - N.ym) / N.ys : 0.0f;
    S.dout[s] = d;
    float l = 0.5f * d * d;
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if ((s & 31) == 0) S.loss[s >> 5] = l;

    // backward, per sample: dz3, dz2, dz1 overwrite z3, z2, z1
    for (int o = 0; o < NH; o++) S.z3[o][s] = d * __half2float(S.w[OFF_W4 + o]) * gelu_df(S.z3[o][s]);
    for (int i = 0; i < NH; i++) {
        float g = 0.0f;
        for (int o = 0; o < NH; o++) g += __half2float(S.w[OFF_W3 + o * NH + i]) * S.z3[o][s];
        S.z2[i][s] = g * gelu_df(S.z2[i][s]);
    }
    for (int i = 0; i < NH; i++) {
        float g = 0.0f;
        for (int o = 0; o < NH; o++) g += __half2float(S.w[OFF_W2 + o * NH + i]) * S.z2[o][s];
        S.z1[i][s] = g * gelu_df(S.z1[i][s]);
    }
    __syncthreads();

    // weight gradients: sums over this CTA's samples
    for (int p = s; p < NPARAM; p += TB) {
        float g = 0.0f;
        if (p < OFF_B1) {
            const int o = p / NIN, i = p % NIN;
            for (int t = 0; t < TB; t++) g += S.z1[o][t] * __half2float(S.a0[i][t]);
        } else if (p < OFF_W2) {
            const int o = p - OFF_B1;
            for (int t = 0; t < TB; t++) g += S.z1[o][t];
        } else if (p < OFF_B2) {
            const int o = (p - OFF_W2) / NH, i = (p - OFF_W2) % NH;
            for (int t = 0; t < TB; t++) g += S.z2[o][t] * __half2float(S.a1[i][t]);
        } else if (p < OFF_W3) {
            const int o = p - OFF_B2;
            for (int t = 0; t < TB; t++) g += S.z2[o][t];
        } else if (p < OFF_B3) {
            const int o = (p - OFF_W3) / NH, i = (p - OFF_W3) % NH;
            for (int t = 0; t < TB; t++) g += S.z3[o][t] * __half2float(S.a2[i][t]);
        } else if (p < OFF_W4) {
            const int o = p - OFF_B3;
            for (int t = 0; t < TB; t++) g += S.z3[o][t];
        } else if (p < OFF_B4) {
            const int i = p - OFF_W4;
            for (int t = 0; t < TB; t++) g += S.dout[t] * __half2float(S.a3[i][t]);
        } else {
            for (int t = 0; t < TB; t++) g += S.dout[t];
        }
        atomicAdd(&G[p], g * inv_batch);
    }
    if (s == 0) {
        double ls = 0.0;
        for (int w = 0; w < TB / 32; w++) ls += S.loss[w];
        atomicAdd(loss_sum, ls);
    }
}

__global__ void k_mlp_adam(float *__restrict__ W, float *__restrict__ M, float *__restrict__ V,
                           float *__restrict__ G, __half *__restrict__ P, float lr, float b1, float b2, float eps,
                           float c1, float c2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NPARAM) return;
    const float g = G[p];
    const float m = b1 * M[p] + (1.0f - b1) * g;
    const float v = b2 * V[p] + (1.0f - b2) * g * g;
    M[p] = m;
    V[p] = v;
    const float w = W[p] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    W[p] = w;
    P[p] = __float2half(w);
    G[p] = 0.0f;
}

__global__ void k_mlp_to_half(const float *__restrict__ W, __half *__restrict__ P)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < NPARAM) P[p] = __float2half(W[p]);
}

// FP16 weights in the inference layout (transposed hidden blocks)
__global__ void k_mlp_inference_copy(const __half *__restrict__ P, __half *__restrict__ T)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < NPARAM) T[to_inference_index(p)] = P[p];
}

// one warp per sample, the controllers' evaluation
__global__ void k_mlp_predict(const __half *__restrict__ P, const Norm *__restrict__ Nn, const float *__restrict__ X,
                              long n, float *__restrict__ Y)
{
    const long j = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5;
    if (j >= n) return;
    float x[NIN];
    for (int i = 0; i < NIN; i++) x[i] = X[j * NIN + i];
    const float y = eval_warp(P, *Nn, x);
    if ((threadIdx.x & 31) == 0) Y[j] = y;
}

}  // namespace mlp
}  // namespace ucg

using namespace ucg;
using namespace ucg::mlp;

struct ucg_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    float *W = nullptr, *M = nullptr, *V = nullptr, *G = nullptr;   // FP32 master, Adam moments, gradient
    __half *P = nullptr;                                            // FP16 weights the kernels use
    __half *T = nullptr;                                            // the same, inference layout
    Norm *norm = nullptr;                                           // device
    Norm hnorm{};
    double *loss = nullptr;
    float *X = nullptr, *Y = nullptr;                               // training set (device)
    int *idx = nullptr;
    long n = 0;
    long adam_t = 0;
};

namespace {

int mfail(ucg_mlp *m, cudaError_t e, const char *what)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    m->err = buf;
    return e == cudaErrorMemoryAllocation ? UCG_E_OOM : UCG_E_CUDA;
}
#define MCUDA(call)                                             \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return mfail(m, e_, #call);      \
    } while (0)

constexpr size_t GRAD_SMEM = sizeof(GradSmem);

int launch_grad(ucg_mlp *m, long count, const int *idx, float inv_batch)
{
    const unsigned blocks = (unsigned)((count + TB - 1) / TB);
    k_mlp_grad<<<blocks, TB, GRAD_SMEM, m->stream>>>(m->P, m->norm, m->X, m->Y, idx, count, inv_batch, m->G,
                                                      m->loss);
    return cudaGetLastError() == cudaSuccess ? UCG_OK : mfail(m, cudaGetLastError(), "k_mlp_grad");
}

}  // namespace

extern "C" {

int ucg_mlp_create(ucg_mlp **out, int device, unsigned long long seed)
{
    if (!out) return UCG_E_BADARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return UCG_E_NODEVICE;
    if (device < 0 || device >= count) return UCG_E_BADARG;
    ucg_mlp *m = new (std::nothrow) ucg_mlp();
    if (!m) return UCG_E_OOM;
    m->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
    float **f32[] = {&m->W, &m->M, &m->V, &m->G};
    for (float **p : f32)
        if (e == cudaSuccess) e = cudaMalloc(p, sizeof(float) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&m->P, sizeof(__half) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&m->T, sizeof(__half) * NPARAM);
    if (e == cudaSuccess) e = cudaMalloc(&m->norm, sizeof(Norm));
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(double));
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)GRAD_SMEM);
    if (e != cudaSuccess) {
        delete m;
        return e == cudaErrorMemoryAllocation ? UCG_E_OOM : UCG_E_CUDA;
    }
    // He-style initialisation, deterministic in the seed
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.0f, 1.0f);
    std::vector<float> w(NPARAM, 0.0f);
    for (int p = OFF_W1; p < OFF_B1; p++) w[p] = nd(rng) * std::sqrt(2.0f / NIN);
    for (int p = OFF_W2; p < OFF_B2; p++) w[p] = nd(rng) * std::sqrt(2.0f / NH);
    for (int p = OFF_W3; p < OFF_B3; p++) w[p] = nd(rng) * std::sqrt(2.0f / NH);
    for (int p = OFF_W4; p < OFF_B4; p++) w[p] = nd(rng) * std::sqrt(1.0f / NH);
    for (int i = 0; i < NIN; i++) {
        m->hnorm.xm[i] = 0.0f;
        m->hnorm.xs[i] = 1.0f;
    }
    m->hnorm.ym = 0.0f;
    m->hnorm.ys = 1.0f;
    cudaMemcpy(m->W, w.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice);
    cudaMemset(m->M, 0, sizeof(float) * NPARAM);
    cudaMemset(m->V, 0, sizeof(float) * NPARAM);
    cudaMemset(m->G, 0, sizeof(float) * NPARAM);
    cudaMemcpy(m->norm, &m->hnorm, sizeof(Norm), cudaMemcpyHostToDevice);
    k_mlp_to_half<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->W, m->P);
    k_mlp_inference_copy<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->P, m->T);
    cudaStreamSynchronize(m->stream);
    *out = m;
    return UCG_OK;
}

void ucg_mlp_destroy(ucg_mlp *m)
{
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    void *ptrs[] = {m->W, m->M, m->V, m->G, m->P, m->T, m->norm, m->loss, m->X, m->Y, m->idx};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
}

const char *ucg_mlp_last_error(ucg_mlp *m) { return m ? m->err.c_str() : ""; }

int ucg_mlp_set_params(ucg_mlp *m, const float *params, const float *norm)
{
    if (!m) return UCG_E_BADARG;
    MCUDA(cudaSetDevice(m->device));
    MCUDA(cudaStreamSynchronize(m->stream));
    if (params) {
        MCUDA(cudaMemcpy(m->W, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
        k_mlp_to_half<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->W, m->P);
        k_mlp_inference_copy<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->P, m->T);
        MCUDA(cudaGetLastError());
        MCUDA(cudaMemset(m->M, 0, sizeof(float) * NPARAM));
        MCUDA(cudaMemset(m->V, 0, sizeof(float) * NPARAM));
        m->adam_t = 0;
    }
    if (norm) {
        for (int i = 0; i < NIN; i++) {
            if (!(norm[NIN + i] > 0.0f)) {
                m->err = "input deviations must be > 0";
                return UCG_E_BADARG;
            }
        }
        if (!(norm[2 * NIN + 1] > 0.0f)) {
            m->err = "output deviation must be > 0";
            return UCG_E_BADARG;
        }
        memcpy(m->hnorm.xm, norm, sizeof(float) * NIN);
        memcpy(m->hnorm.xs, norm + NIN, sizeof(float) * NIN);
        m->hnorm.ym = norm[2 * NIN];
        m->hnorm.ys = norm[2 * NIN + 1];
        MCUDA(cudaMemcpy(m->norm, &m->hnorm, sizeof(Norm), cudaMemcpyHostToDevice));
    }
    MCUDA(cudaStreamSynchronize(m->stream));
    return UCG_OK;
}

int ucg_mlp_get_params(ucg_mlp *m, float *params, float *norm)
{
    if (!m) return UCG_E_BADARG;
    MCUDA(cudaSetDevice(m->device));
    MCUDA(cudaStreamSynchronize(m->stream));
    if (params) MCUDA(cudaMemcpy(params, m->W, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
    if (norm) {
        memcpy(norm, m->hnorm.xm, sizeof(float) * NIN);
        memcpy(norm + NIN, m->hnorm.xs, sizeof(float) * NIN);
        norm[2 * NIN] = m->hnorm.ym;
        norm[2 * NIN + 1] = m->hnorm.ys;
    }
    return UCG_OK;
}

int ucg_mlp_set_data(ucg_mlp *m, const float *x, const float *y, long n, int standardise)
{
    if (!m || !x || !y || n < 1) return UCG_E_BADARG;
    MCUDA(cudaSetDevice(m->device));
    MCUDA(cudaStreamSynchronize(m->stream));
    void *old[] = {m->X, m->Y, m->idx};
    for (void *p : old)
        if (p) cudaFree(p);
    m->X = m->Y = nullptr;
    m->idx = nullptr;
    m->n = 0;
    MCUDA(cudaMalloc(&m->X, sizeof(float) * NIN * n));
    MCUDA(cudaMalloc(&m->Y, sizeof(float) * n));
    MCUDA(cudaMalloc(&m->idx, sizeof(int) * n));
    MCUDA(cudaMemcpy(m->X, x, sizeof(float) * NIN * n, cudaMemcpyHostToDevice));
    MCUDA(cudaMemcpy(m->Y, y, sizeof(float) * n, cudaMemcpyHostToDevice));
    m->n = n;
    if (standardise) {
        // means and deviations of the training set (FP64 sums)
        for (int i = 0; i < NIN + 1; i++) {
            double s = 0.0, s2 = 0.0;
            for (long r = 0; r < n; r++) {
                const double v = i < NIN ? x[r * NIN + i] : y[r];
                s += v;
                s2 += v * v;
            }
            const double mean = s / n, var = std::max(s2 / n - mean * mean, 0.0);
            const float sd = (float)std::max(std::sqrt(var), 1e-3);
            if (i < NIN) {
                m->hnorm.xm[i] = (float)mean;
                m->hnorm.xs[i] = sd;
            } else {
                m->hnorm.ym = (float)mean;
                m->hnorm.ys = sd;
            }
        }
        MCUDA(cudaMemcpy(m->norm, &m->hnorm, sizeof(Norm), cudaMemcpyHostToDevice));
    }
    return UCG_OK;
}

int ucg_mlp_gradient(ucg_mlp *m, long offset, long count, float *grad, double *loss)
{
    if (!m || !grad || offset < 0 || count < 1 || offset + count > m->n) return UCG_E_BADARG;
    MCUDA(cudaSetDevice(m->device));
    std::vector<int> ids(count);
    std::iota(ids.begin(), ids.end(), (int)offset);
    MCUDA(cudaMemcpyAsync(m->idx, ids.data(), sizeof(int) * count, cudaMemcpyHostToDevice, m->stream));
    MCUDA(cudaMemsetAsync(m->G, 0, sizeof(float) * NPARAM, m->stream));
    MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
    int st = launch_grad(m, count, m->idx, 1.0f / (float)count);
    if (st) return st;
    double l = 0.0;
    MCUDA(cudaMemcpyAsync(grad, m->G, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, m->stream));
    MCUDA(cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    MCUDA(cudaMemsetAsync(m->G, 0, sizeof(float) * NPARAM, m->stream));
    MCUDA(cudaStreamSynchronize(m->stream));
    if (loss) *loss = l / count;
    return UCG_OK;
}

int ucg_mlp_train(ucg_mlp *m, int epochs, int batch, float lr, unsigned long long seed, float *epoch_loss)
{
    if (!m || epochs < 1 || batch < 1 || !(lr > 0.0f) || m->n < 1) return UCG_E_BADARG;
    MCUDA(cudaSetDevice(m->device));
    std::mt19937_64 rng(seed);
    std::vector<int> perm(m->n);
    std::iota(perm.begin(), perm.end(), 0);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        MCUDA(cudaMemcpyAsync(m->idx, perm.data(), sizeof(int) * m->n, cudaMemcpyHostToDevice, m->stream));
        MCUDA(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
        for (long off = 0; off < m->n; off += batch) {
            const long cnt = std::min((long)batch, m->n - off);
            const unsigned blocks = (unsigned)((cnt + TB - 1) / TB);
            k_mlp_grad<<<blocks, TB, GRAD_SMEM, m->stream>>>(m->P, m->norm, m->X, m->Y, m->idx + off, cnt,
                                                              1.0f / (float)cnt, m->G, m->loss);
            m->adam_t++;
            const float c1 = 1.0f - std::pow(b1, (float)m->adam_t), c2 = 1.0f - std::pow(b2, (float)m->adam_t);
            k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->W, m->M, m->V, m->G, m->P, lr, b1, b2, eps,
                                                                   c1, c2);
        }
        MCUDA(cudaGetLastError());
        double l = 0.0;
        MCUDA(cudaMemcpyAsync(&l, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
        MCUDA(cudaStreamSynchronize(m->stream));
        if (epoch_loss) epoch_loss[ep] = (float)(l / m->n);
    }
    k_mlp_inference_copy<<<(NPARAM + 255) / 256, 256, 0, m->stream>>>(m->P, m->T);
    MCUDA(cudaGetLastError());
    MCUDA(cudaStreamSynchronize(m->stream));
    return UCG_OK;
}

int ucg_mlp_predict(ucg_mlp *m, const float *x, long n, float *y)
{
    if (!m || !x || !y || n < 1) return UCG_E_BADARG;
    MCUDA(cudaSetDevice(m->device));
    float *dx = nullptr, *dy = nullptr;
    MCUDA(cudaMalloc(&dx, sizeof(float) * NIN * n));
    cudaError_t e = cudaMalloc(&dy, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, x, sizeof(float) * NIN * n, cudaMemcpyHostToDevice, m->stream);
    if (e == cudaSuccess) {
        k_mlp_predict<<<(unsigned)((n + 3) / 4), 128, 0, m->stream>>>(m->T, m->norm, dx, n, dy);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(dx);
    if (dy) cudaFree(dy);
    return e == cudaSuccess ? UCG_OK : mfail(m, e, "ucg_mlp_predict");
}

}  // extern "C"

namespace ucg {
// device addresses of a model's FP16 weights and standardisation, for the controllers
void mlp_device_params(const ucg_mlp *m, const __half **P, const mlp::Norm **N)
{
    *P = m ? m->T : nullptr;
    *N = m ? m->norm : nullptr;
}
}  // namespace ucg
