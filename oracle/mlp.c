/*
 * Oracle: the step-size perceptron (unicycle_b200/csrc/mlp.cuh), forward pass,
 * squared-error loss and backward pass on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  No reference counterpart: the
 * learned step-size proposal is new.  The network is restated from its
 * definition (11 -> 64 -> 64 -> 64 GELU -> 1, loss 0.5 (y_hat - label_hat)^2
 * averaged over the samples, standardised units), and the backward pass is the
 * chain rule written out by hand, independently of the device kernels.
 * With fp16 != 0 the weights, the standardised inputs and the three activation
 * vectors are rounded to binary16 at the same points as the device (which
 * accumulates in binary32); sums are binary64 here.  With fp16 == 0 everything
 * is binary64, so that finite differences of the loss pin the backward pass
 * (tests/test_oracle_mlp.py).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"

#define NIN 11
#define NH 64
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + NH * NIN)
#define OFF_W2 (OFF_B1 + NH)
#define OFF_B2 (OFF_W2 + NH * NH)
#define OFF_W3 (OFF_B2 + NH)
#define OFF_B3 (OFF_W3 + NH * NH)
#define OFF_W4 (OFF_B3 + NH)
#define OFF_B4 (OFF_W4 + NH)
#define NPARAM (OFF_B4 + 1)

static double rnd16(double x, int on) { return on ? (double)(_Float16)(float)x : x; }
static double gelu(double z) { return 0.5 * z * (1.0 + erf(z / sqrt(2.0))); }
static double dgelu(double z)
{
    return 0.5 * (1.0 + erf(z / sqrt(2.0))) + z * exp(-0.5 * z * z) / sqrt(2.0 * M_PI);
}

int orc_mlp_nparam(void) { return NPARAM; }

/* norm: xm[11], xs[11], ym, ys.  grad (may be NULL) receives d mean-loss / d param. */
void orc_mlp_loss_grad(const float *params, const float *norm, const float *X, const float *Y, long n,
                       int fp16, double *grad, double *loss)
{
    double w[NPARAM];
    for (int p = 0; p < NPARAM; p++) w[p] = rnd16(params[p], fp16);
    if (grad) memset(grad, 0, sizeof(double) * NPARAM);
    double L = 0.0;
    for (long r = 0; r < n; r++) {
        double a0[NIN], z1[NH], a1[NH], z2[NH], a2[NH], z3[NH], a3[NH];
        for (int i = 0; i < NIN; i++) a0[i] = rnd16((X[r * NIN + i] - norm[i]) / norm[NIN + i], fp16);
        for (int o = 0; o < NH; o++) {
            double z = w[OFF_B1 + o];
            for (int i = 0; i < NIN; i++) z += w[OFF_W1 + o * NIN + i] * a0[i];
            z1[o] = z;
            a1[o] = rnd16(gelu(z), fp16);
        }
        for (int o = 0; o < NH; o++) {
            double z = w[OFF_B2 + o];
            for (int i = 0; i < NH; i++) z += w[OFF_W2 + o * NH + i] * a1[i];
            z2[o] = z;
            a2[o] = rnd16(gelu(z), fp16);
        }
        double out = w[OFF_B4];
        for (int o = 0; o < NH; o++) {
            double z = w[OFF_B3 + o];
            for (int i = 0; i < NH; i++) z += w[OFF_W3 + o * NH + i] * a2[i];
            z3[o] = z;
            a3[o] = rnd16(gelu(z), fp16);
            out += w[OFF_W4 + o] * a3[o];
        }
        const double d = out - (Y[r] - norm[2 * NIN]) / norm[2 * NIN + 1];
        L += 0.5 * d * d;
        if (!grad) continue;
        double dz3[NH], dz2[NH], dz1[NH];
        for (int o = 0; o < NH; o++) {
            grad[OFF_W4 + o] += d * a3[o];
            dz3[o] = d * w[OFF_W4 + o] * dgelu(z3[o]);
        }
        grad[OFF_B4] += d;
        for (int i = 0; i < NH; i++) {
            double g = 0.0;
            for (int o = 0; o < NH; o++) g += w[OFF_W3 + o * NH + i] * dz3[o];
            dz2[i] = g * dgelu(z2[i]);
        }
        for (int i = 0; i < NH; i++) {
            double g = 0.0;
            for (int o = 0; o < NH; o++) g += w[OFF_W2 + o * NH + i] * dz2[o];
            dz1[i] = g * dgelu(z1[i]);
        }
        for (int o = 0; o < NH; o++) {
            for (int i = 0; i < NH; i++) {
                grad[OFF_W3 + o * NH + i] += dz3[o] * a2[i];
                grad[OFF_W2 + o * NH + i] += dz2[o] * a1[i];
            }
            for (int i = 0; i < NIN; i++) grad[OFF_W1 + o * NIN + i] += dz1[o] * a0[i];
            grad[OFF_B3 + o] += dz3[o];
            grad[OFF_B2 + o] += dz2[o];
            grad[OFF_B1 + o] += dz1[o];
        }
    }
    if (grad)
        for (int p = 0; p < NPARAM; p++) grad[p] /= (double)n;
    if (loss) *loss = L / (double)n;
}

/* log10 of the proposed step for raw inputs X (n x 11) */
void orc_mlp_predict(const float *params, const float *norm, const float *X, long n, int fp16, double *out)
{
    double w[NPARAM];
    for (int p = 0; p < NPARAM; p++) w[p] = rnd16(params[p], fp16);
    for (long r = 0; r < n; r++) {
        double a0[NIN], a1[NH], a2[NH];
        for (int i = 0; i < NIN; i++) a0[i] = rnd16((X[r * NIN + i] - norm[i]) / norm[NIN + i], fp16);
        for (int o = 0; o < NH; o++) {
            double z = w[OFF_B1 + o];
            for (int i = 0; i < NIN; i++) z += w[OFF_W1 + o * NIN + i] * a0[i];
            a1[o] = rnd16(gelu(z), fp16);
        }
        for (int o = 0; o < NH; o++) {
            double z = w[OFF_B2 + o];
            for (int i = 0; i < NH; i++) z += w[OFF_W2 + o * NH + i] * a1[i];
            a2[o] = rnd16(gelu(z), fp16);
        }
        double y = w[OFF_B4];
        for (int o = 0; o < NH; o++) {
            double z = w[OFF_B3 + o];
            for (int i = 0; i < NH; i++) z += w[OFF_W3 + o * NH + i] * a2[i];
            y += w[OFF_W4 + o] * rnd16(gelu(z), fp16);
        }
        out[r] = y * norm[2 * NIN + 1] + norm[2 * NIN];
    }
}
