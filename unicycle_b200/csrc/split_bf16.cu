// Split storage of the traction matrix for the single-instance split path:
// K = diag(s) k with a per-row scale s_r = max_c |K_rc| (FP32, rounded up so
// that |k| <= 1), stored twice:
//   * the pair plane: k in FP32, i.e. a bf16 hi part (its upper 16 bits) and a
//     16-bit lo extension of the significand (its lower 16 bits): 4 bytes per
//     entry, half the FP64 stream, relative error <= 2^-24 per entry.  The
//     stage-1 anchor of every step reads it and sums in FP64;
//   * the increment plane: fp16(k) rounded to nearest, 2 bytes per entry
//     (relative error <= 2^-11 down to 2^-14 of the row maximum, an absolute
//     2^-25 of it below), which the anchored stages 2-6 multiply against the
//     velocity increments.
#include <cmath>
#include <cmath>
#include "ucg_internal.cuh"

namespace ucg {

__global__ void k_row_absmax(const double *__restrict__ K, long n, float *__restrict__ scale)
{
    const long r = blockIdx.x;
    const double *row = K + r * n;
    double m = 0.0;
    for (long c = threadIdx.x; c < n; c += blockDim.x) m = fmax(m, fabs(row[c]));
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t = fmax(t, wm[w]);
        // round the scale up to FP32 so that |K/s| <= 1
        float s = (float)t;
        if ((double)s < t) s = nextafterf(s, INFINITY);
        scale[r] = (t > 0.0) ? s : 1.0f;
    }
}

// out has row stride ldk >= n; the padding columns hold zeros
__global__ void k_split(const double *__restrict__ K, long n, long ldk, long total, const float *__restrict__ scale,
                        float *__restrict__ out, __half *__restrict__ out_hi)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long r = i / ldk, cc = i - r * ldk;
        if (cc >= n) {
            out[i] = 0.0f;
            out_hi[i] = __float2half_rn(0.0f);
            continue;
        }
        const double x = K[r * n + cc] / (double)scale[r];
        out[i] = __double2float_rn(x);
        out_hi[i] = __double2half(x);
    }
}

int split_bf16_build(ucg_ctx *c)
{
    if (!c->K) return UCG_E_STATE;
    split_bf16_free(c);
    UCG_CUDA(cudaSetDevice(c->device));
    c->ldk_split = (c->n + 7) / 8 * 8;
    const long total = c->ldk_split * c->m;
    cudaError_t e = cudaMalloc(&c->Ksp, sizeof(float) * (size_t)total);
    if (e != cudaSuccess) { c->Ksp = nullptr; return cuda_fail(c, e, "cudaMalloc(split K)"); }
    e = cudaMalloc(&c->Khi_plane, sizeof(__half) * (size_t)total);
    if (e != cudaSuccess) { c->Khi_plane = nullptr; return cuda_fail(c, e, "cudaMalloc(split K hi plane)"); }
    UCG_CUDA(cudaMalloc(&c->Kscale, sizeof(float) * (size_t)c->m));
    k_row_absmax<<<(unsigned)c->m, 256, 0, c->stream>>>(c->K, c->n, c->Kscale);
    const int grid = c->sms * 16;
    k_split<<<grid, 256, 0, c->stream>>>(c->K, c->n, c->ldk_split, total, c->Kscale, c->Ksp, c->Khi_plane);
    c->launches.count += 2;
    UCG_CUDA(cudaGetLastError());
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    if (!c->keep_fp64) {
        cudaFree(c->K);
        c->K = nullptr;
    }
    return UCG_OK;
}

void split_bf16_free(ucg_ctx *c)
{
    if (c->Ksp || c->Kscale) rk_drop_graph(c);
    if (c->Ksp) cudaFree(c->Ksp);
    if (c->Khi_plane) cudaFree(c->Khi_plane);
    if (c->Kscale) cudaFree(c->Kscale);
    c->Ksp = nullptr;
    c->Khi_plane = nullptr;
    c->Kscale = nullptr;
}

}  // namespace ucg
