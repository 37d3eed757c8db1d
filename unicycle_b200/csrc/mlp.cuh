// Learned step-size proposal: a small multilayer perceptron
//   11 inputs -> 64 -> 64 -> 64 (GELU) -> 1
// whose output is log10 of the next Runge-Kutta step size.  Inputs, in order:
//   log10 max V over the patches at the start of the step,
//   min log10 theta over the patches at the start of the step,
//   log10 of the last 8 accepted step sizes (most recent first),
//   log10 max(errmax, 1e-12) of the step just accepted (errmax = max|yerr/yscal|/epsilon).
// Inputs are standardised with the training set's means and deviations, which
// travel with the weights.  Weights and activations are FP16, sums are FP32;
// training keeps FP32 master weights (mlp.cu).  The embedded error estimate still
// decides: a proposal is only the first try of the next step, and a rejected
// proposal is shrunk by the plain RKQSm rule.
#pragma once
#include <cuda_fp16.h>

namespace ucg {
namespace mlp {

constexpr int NIN = 11, NH = 64;
constexpr int OFF_W1 = 0;                        // [NH][NIN]
constexpr int OFF_B1 = OFF_W1 + NH * NIN;        // [NH]
constexpr int OFF_W2 = OFF_B1 + NH;              // [NH][NH]
constexpr int OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH;              // [NH][NH]
constexpr int OFF_B3 = OFF_W3 + NH * NH;
constexpr int OFF_W4 = OFF_B3 + NH;              // [NH]
constexpr int OFF_B4 = OFF_W4 + NH;              // [1]
constexpr int NPARAM = OFF_B4 + 1;               // 9,153

// standardisation: x_hat = (x - xm) / xs, output log10 dt = y_hat * ys + ym
struct Norm {
    float xm[NIN], xs[NIN];
    float ym, ys;
};

__host__ __device__ inline float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__host__ __device__ inline float gelu_df(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Inference layout: the same blocks with W1, W2, W3 transposed ([in][out]),
// so that the 32 lanes of a warp read 32 consecutive outputs' weights.
__host__ __device__ inline int to_inference_index(int p)
{
    if (p < OFF_B1) return OFF_W1 + (p % NIN) * NH + p / NIN;
    if (p >= OFF_W2 && p < OFF_B2) return OFF_W2 + ((p - OFF_W2) % NH) * NH + (p - OFF_W2) / NH;
    if (p >= OFF_W3 && p < OFF_B3) return OFF_W3 + ((p - OFF_W3) % NH) * NH + (p - OFF_W3) / NH;
    return p;
}

// One sample, one warp, weights T in the inference layout (global or shared
// memory): lane l owns outputs l and l + 32 of every hidden layer, activations
// travel by shuffles; each output's sum runs over its inputs in order, the last
// layer's dot product is reduced across the warp.
__device__ inline float eval_warp(const __half *T, const Norm &N, const float x[NIN])
{
    const int l = threadIdx.x & 31;
    float a0[NIN];
#pragma unroll
    for (int i = 0; i < NIN; i++) a0[i] = __half2float(__float2half((x[i] - N.xm[i]) / N.xs[i]));
    float lo, hi;
    {
        float z0 = __half2float(T[OFF_B1 + l]), z1 = __half2float(T[OFF_B1 + l + 32]);
#pragma unroll
        for (int i = 0; i < NIN; i++) {
            z0 += __half2float(T[OFF_W1 + i * NH + l]) * a0[i];
            z1 += __half2float(T[OFF_W1 + i * NH + l + 32]) * a0[i];
        }
        lo = __half2float(__float2half(gelu_f(z0)));
        hi = __half2float(__float2half(gelu_f(z1)));
    }
#pragma unroll
    for (int layer = 0; layer < 2; layer++) {
        const int ow = layer == 0 ? OFF_W2 : OFF_W3, ob = layer == 0 ? OFF_B2 : OFF_B3;
        float z0 = __half2float(T[ob + l]), z1 = __half2float(T[ob + l + 32]);
        for (int i = 0; i < NH; i++) {
            const float a = __shfl_sync(0xffffffffu, i < 32 ? lo : hi, i & 31);
            z0 += __half2float(T[ow + i * NH + l]) * a;
            z1 += __half2float(T[ow + i * NH + l + 32]) * a;
        }
        lo = __half2float(__float2half(gelu_f(z0)));
        hi = __half2float(__float2half(gelu_f(z1)));
    }
    float out = __half2float(T[OFF_W4 + l]) * lo + __half2float(T[OFF_W4 + l + 32]) * hi;
    for (int off = 16; off > 0; off >>= 1) out += __shfl_xor_sync(0xffffffffu, out, off);
    return (out + __half2float(T[OFF_B4])) * N.ys + N.ym;
}

// feature vector from the controller's state at an accepted step
__device__ inline void features(double vmax, double thmin, const double hist[8], double errmax, float x[NIN])
{
    x[0] = (float)log10(fmax(vmax, 1e-300));
    x[1] = (float)thmin;
#pragma unroll
    for (int k = 0; k < 8; k++) x[2 + k] = (float)log10(fmax(hist[k], 1e-300));
    x[10] = (float)log10(fmax(errmax, 1e-12));
}

// order-preserving 64-bit key of a double (for atomicMin/atomicMax of signed values)
__device__ __forceinline__ unsigned long long ord_key(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_val(unsigned long long k)
{
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

}  // namespace mlp
}  // namespace ucg
