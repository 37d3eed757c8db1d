// Assembly of the stress-interaction matrix K on the device.
//
// K is row-major with m rows (receiver force DOFs) and n columns (source DOFs);
// row k of K is column k of the reference's G(n,m) (fortran/3d/src/greens.f90:
// 73-275), so the reference layout is a plain copy:
//   rows:    patches 3 per element (ts, td, tn), volumes 6 (s11'..s33'),
//            elements ordered rectangles, triangles, volumes;
//   columns: rectangles 2 per source (strike, dip slip), triangles 2, volumes 6
//            (unit eigenstrain 11, 12, 13, 22, 23, 33), component fastest.
//
// One thread per (receiver, source) pair computes every unit component of the
// source at once, sharing the pair geometry, and writes them as contiguous
// columns: a warp covers 32 consecutive sources of one receiver, so each of its
// row stores is one coalesced 512-byte (patches) segment.  Per-source constants
// (frames, the REAL*4-rounded DC3D inputs, the Nikkhoo-Walter records) are built
// once on the host and read through the read-only path.
#include <cmath>
#include <cstring>
#include "ucg_internal.cuh"
#include "okada92.cuh"
#include "nikkhoo15.cuh"
#include "strainvolume.cuh"
#include "blocks.cuh"

namespace ucg {

// ---- receivers -----------------------------------------------------------------

// receiver record: xc[3], sv[3], dv[3], nv[3]
enum { RC_X = 0, RC_S = 3, RC_D = 6, RC_N = 9, RC_SIZE = 12 };

__device__ __forceinline__ void traction3(const double *r, const double s[6], double t[3])
{
    // okada92.f90:390-398
    const double n0 = r[RC_N], n1 = r[RC_N + 1], n2 = r[RC_N + 2];
    const double a = n0 * s[0] + n1 * s[1] + n2 * s[2];
    const double b = n0 * s[1] + n1 * s[3] + n2 * s[4];
    const double c = n0 * s[2] + n1 * s[4] + n2 * s[5];
    t[0] = a * r[RC_S] + b * r[RC_S + 1] + c * r[RC_S + 2];
    t[1] = a * r[RC_D] + b * r[RC_D + 1] + c * r[RC_D + 2];
    t[2] = a * n0 + b * n1 + c * n2;
}

__device__ __forceinline__ void stress6(const double *r, const double s[6], double o[6])
{
    // okada92.f90:445-462
    const double *sv = r + RC_S, *dv = r + RC_D, *nv = r + RC_N;
    const double sa = sv[0] * s[0] + sv[1] * s[1] + sv[2] * s[2];
    const double sb = sv[0] * s[1] + sv[1] * s[3] + sv[2] * s[4];
    const double sc = sv[0] * s[2] + sv[1] * s[4] + sv[2] * s[5];
    const double na = nv[0] * s[0] + nv[1] * s[1] + nv[2] * s[2];
    const double nb = nv[0] * s[1] + nv[1] * s[3] + nv[2] * s[4];
    const double nc = nv[0] * s[2] + nv[1] * s[4] + nv[2] * s[5];
    const double da = -dv[0] * s[0] - dv[1] * s[1] - dv[2] * s[2];
    const double db = -dv[0] * s[1] - dv[1] * s[3] - dv[2] * s[4];
    const double dc = -dv[0] * s[2] - dv[1] * s[4] - dv[2] * s[5];
    o[0] = sa * sv[0] + sb * sv[1] + sc * sv[2];
    o[1] = sa * nv[0] + sb * nv[1] + sc * nv[2];
    o[2] = -sa * dv[0] - sb * dv[1] - sc * dv[2];
    o[3] = na * nv[0] + nb * nv[1] + nc * nv[2];
    o[4] = -na * dv[0] - nb * dv[1] - nc * dv[2];
    o[5] = -da * dv[0] - db * dv[1] - dc * dv[2];
}

struct RcvInfo {
    long row;   // first row of K
    int nrow;   // 3 (patch) or 6 (volume)
};

__device__ __forceinline__ RcvInfo rcv_info(int e, int np)
{
    RcvInfo ri;
    if (e < np) { ri.row = 3L * e; ri.nrow = 3; }
    else { ri.row = 3L * np + 6L * (e - np); ri.nrow = 6; }
    return ri;
}

// write (ACC = false) or add (ACC = true) the 2 slip columns, one double2 per
// row, of a patch source
template <bool ACC = false>
__device__ __forceinline__ void store_patch_source(double *K, long n, long col, const double *rc,
                                                   const RcvInfo &ri, const double sS[6],
                                                   const double sD[6])
{
    double oS[6], oD[6];
    if (ri.nrow == 3) {
        traction3(rc, sS, oS);
        traction3(rc, sD, oD);
    } else {
        stress6(rc, sS, oS);
        stress6(rc, sD, oD);
    }
#pragma unroll
    for (int c = 0; c < 6; c++) {
        if (c < ri.nrow) {
            double2 *p = reinterpret_cast<double2 *>(K + (ri.row + c) * n + col);
            if (ACC) {
                const double2 o = *p;
                *p = make_double2(o.x + oS[c], o.y + oD[c]);
            } else {
                *p = make_double2(oS[c], oD[c]);
            }
        }
    }
}

// ---- rectangles (Okada 1992) -------------------------------------------------

enum { RS_Q1 = 0, RS_Q2, RS_CS, RS_SS, RS_DEPTH, RS_AL2, RS_AW1, RS_SD, RS_CD, RS_SDSD, RS_CDCD,
       RS_SDCD, RS_SIZE };

// Stress (s11, s12, s13, s22, s23, s33 for strike and dip slip) at receiver
// point (x1, x2, x3) of one rectangle record sr (okada92.f90:121-205).
template <bool R32>
__device__ __forceinline__ void rect_pair_sig(const double sr[RS_SIZE], const OkDip &dp, double x1, double x2,
                                              double x3, const OkMed &med, double mu, double lambda,
                                              double sig[2][6])
{
    const double csst = sr[RS_CS], ssst = sr[RS_SS];
    double x = (x1 - sr[RS_Q1]) * csst + (x2 - sr[RS_Q2]) * ssst;
    double y = (x1 - sr[RS_Q1]) * ssst - (x2 - sr[RS_Q2]) * csst;
    double z = -x3;
    if (R32) {
        x = (double)__double2float_rn(x);
        y = (double)__double2float_rn(y);
        z = (double)__double2float_rn(z);
    }
    double gs[9], gd[9];
    ok_dc3d_grad<R32>(med, dp, x, y, z, sr[RS_DEPTH], sr[RS_AL2], sr[RS_AW1], gs, gd);
#pragma unroll
    for (int t = 0; t < 2; t++) {
        const double *g = t ? gd : gs;
        // okada92.f90:165-205: rotate the gradient back from the strike frame
        const double uxx = g[0], uyx = g[1], uzx = g[2], uxy = g[3], uyy = g[4], uzy = g[5];
        const double uxz = g[6], uyz = g[7], uzz = g[8];
        const double uxxr = (csst * uxx + ssst * uyx) * csst - (-csst * uxy - ssst * uyy) * ssst;
        const double uxyr = (csst * uxx + ssst * uyx) * ssst + (-csst * uxy - ssst * uyy) * csst;
        const double uxzr = -csst * uxz + ssst * uyz;
        const double uyxr = (ssst * uxx - csst * uyx) * csst - (-ssst * uxy + csst * uyy) * ssst;
        const double uyyr = (ssst * uxx - csst * uyx) * ssst + (-ssst * uxy + csst * uyy) * csst;
        const double uyzr = -ssst * uxz + csst * uyz;
        const double uzxr = -csst * uzx - ssst * uzy;
        const double uzyr = -ssst * uzx + csst * uzy;
        const double e11 = uxxr, e12 = (uxyr + uyxr) / 2.0, e13 = (uxzr + uzxr) / 2.0;
        const double e22 = uyyr, e23 = (uyzr + uzyr) / 2.0, e33 = uzz;
        const double ekk = e11 + e22 + e33;
        sig[t][0] = lambda * ekk + 2.0 * mu * e11;
        sig[t][1] = 2.0 * mu * e12;
        sig[t][2] = 2.0 * mu * e13;
        sig[t][3] = lambda * ekk + 2.0 * mu * e22;
        sig[t][4] = 2.0 * mu * e23;
        sig[t][5] = lambda * ekk + 2.0 * mu * e33;
    }
}

__device__ __forceinline__ void rect_record(const double *__restrict__ src, int ns, int j, double sr[RS_SIZE],
                                            OkDip &dp)
{
#pragma unroll
    for (int f = 0; f < RS_SIZE; f++) sr[f] = __ldg(src + (long)f * ns + j);
    dp.sd = sr[RS_SD]; dp.cd = sr[RS_CD]; dp.sdsd = sr[RS_SDSD]; dp.cdcd = sr[RS_CDCD];
    dp.sdcd = sr[RS_SDCD];
}

template <bool R32>
__global__ void __launch_bounds__(128) k_assemble_rect(double *__restrict__ K, long n, long col0,
        const double *__restrict__ rcv, int nrcv, int np, const double *__restrict__ src, int ns,
        OkMed med, double mu, double lambda)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    double sr[RS_SIZE];
    OkDip dp;
    rect_record(src, ns, j, sr, dp);
    for (int e = blockIdx.y; e < nrcv; e += gridDim.y) {
        const double *rc = rcv + (long)e * RC_SIZE;
        double sig[2][6];
        rect_pair_sig<R32>(sr, dp, __ldg(rc + 0), __ldg(rc + 1), __ldg(rc + 2), med, mu, lambda, sig);
        double rloc[RC_SIZE];
#pragma unroll
        for (int f = 0; f < RC_SIZE; f++) rloc[f] = __ldg(rc + f);
        store_patch_source(K, n, col0 + 2L * j, rloc, rcv_info(e, np), sig[0], sig[1]);
    }
}

// ---- triangles (Nikkhoo & Walter 2015) -----------------------------------------

template <int PART>
__global__ void __launch_bounds__(128) k_assemble_tri(double *__restrict__ K, long n, long col0,
        const double *__restrict__ rcv, int nrcv, int np, const double *__restrict__ rec, int ns,
        NwConst cst)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    NwRec R{rec + j, (long)ns};
    for (int e = blockIdx.y; e < nrcv; e += gridDim.y) {
        const double *rc = rcv + (long)e * RC_SIZE;
        double rloc[RC_SIZE];
#pragma unroll
        for (int f = 0; f < RC_SIZE; f++) rloc[f] = __ldg(rc + f);
        double sS[6], sD[6];
        nw_part_stress<PART>(rloc, R, cst, sS, sD);
        store_patch_source<PART != 0>(K, n, col0 + 2L * j, rloc, rcv_info(e, np), sS, sD);
    }
}

// ---- strain volumes (Barbot, Moore & Lambert 2017) -------------------------------

__global__ void __launch_bounds__(128) k_assemble_vol(double *__restrict__ K, long n, long col0,
        const double *__restrict__ rcv, int nrcv, int np, const double *__restrict__ rec, int ns,
        double mu, double nu)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    SvRec R{rec + j, (long)ns};
    for (int e = blockIdx.y; e < nrcv; e += gridDim.y) {
        const double *rc = rcv + (long)e * RC_SIZE;
        double rloc[RC_SIZE];
#pragma unroll
        for (int f = 0; f < RC_SIZE; f++) rloc[f] = __ldg(rc + f);
        double sig[6][6];
        sv_pair_stress(rloc, R, mu, nu, sig);
        const RcvInfo ri = rcv_info(e, np);
        const long col = col0 + 6L * j;
        if (ri.nrow == 3) {
            double t[6][3];
#pragma unroll
            for (int q = 0; q < 6; q++) traction3(rloc, sig[q], t[q]);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                double *p = K + (ri.row + c) * n + col;
                reinterpret_cast<double2 *>(p)[0] = make_double2(t[0][c], t[1][c]);
                reinterpret_cast<double2 *>(p)[1] = make_double2(t[2][c], t[3][c]);
                reinterpret_cast<double2 *>(p)[2] = make_double2(t[4][c], t[5][c]);
            }
        } else {
            double o[6][6];
#pragma unroll
            for (int q = 0; q < 6; q++) stress6(rloc, sig[q], o[q]);
#pragma unroll
            for (int c = 0; c < 6; c++) {
                double *p = K + (ri.row + c) * n + col;
                reinterpret_cast<double2 *>(p)[0] = make_double2(o[0][c], o[1][c]);
                reinterpret_cast<double2 *>(p)[1] = make_double2(o[2][c], o[3][c]);
                reinterpret_cast<double2 *>(p)[2] = make_double2(o[4][c], o[5][c]);
            }
        }
    }
}

// ---- dense blocks of K for the hierarchical approximation -------------------------
//
// Rows of receivers ridx[0..nrb) (element ids, patches only: 3 traction rows
// each) against the columns of sources sidx[0..nsb) of one family (2 slip
// columns each); out is row-major (3 nrb) x (2 nsb).  The same pair kernels as
// K; the grid's y dimension strides over the receivers.

template <bool R32>
__global__ void __launch_bounds__(128) k_block_rect(double *__restrict__ out, const int *__restrict__ ridx, int nrb,
        const int *__restrict__ sidx, int nsb, const double *__restrict__ rcv, const double *__restrict__ src,
        int ns, OkMed med, double mu, double lambda)
{
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= nsb) return;
    double sr[RS_SIZE];
    OkDip dp;
    rect_record(src, ns, __ldg(sidx + jj), sr, dp);
    const long ld = 2L * nsb;
    for (int ii = blockIdx.y; ii < nrb; ii += gridDim.y) {
        const double *rc = rcv + (long)__ldg(ridx + ii) * RC_SIZE;
        double rloc[RC_SIZE];
#pragma unroll
        for (int f = 0; f < RC_SIZE; f++) rloc[f] = __ldg(rc + f);
        double sig[2][6], tS[3], tD[3];
        rect_pair_sig<R32>(sr, dp, rloc[0], rloc[1], rloc[2], med, mu, lambda, sig);
        traction3(rloc, sig[0], tS);
        traction3(rloc, sig[1], tD);
#pragma unroll
        for (int c = 0; c < 3; c++)
            *reinterpret_cast<double2 *>(out + (3L * ii + c) * ld + 2L * jj) = make_double2(tS[c], tD[c]);
    }
}

template <int PART>
__global__ void __launch_bounds__(128) k_block_tri(double *__restrict__ out, const int *__restrict__ ridx, int nrb,
        const int *__restrict__ sidx, int nsb, const double *__restrict__ rcv, const double *__restrict__ rec,
        int ns, NwConst cst)
{
    const int jj = blockIdx.x * blockDim.x + threadIdx.x;
    if (jj >= nsb) return;
    NwRec R{rec + __ldg(sidx + jj), (long)ns};
    const long ld = 2L * nsb;
    for (int ii = blockIdx.y; ii < nrb; ii += gridDim.y) {
        const double *rc = rcv + (long)__ldg(ridx + ii) * RC_SIZE;
        double rloc[RC_SIZE];
#pragma unroll
        for (int f = 0; f < RC_SIZE; f++) rloc[f] = __ldg(rc + f);
        double sS[6], sD[6], tS[3], tD[3];
        nw_part_stress<PART>(rloc, R, cst, sS, sD);
        traction3(rloc, sS, tS);
        traction3(rloc, sD, tD);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double2 *p = reinterpret_cast<double2 *>(out + (3L * ii + c) * ld + 2L * jj);
            if (PART == 0) {
                *p = make_double2(tS[c], tD[c]);
            } else {
                const double2 o = *p;
                *p = make_double2(o.x + tS[c], o.y + tD[c]);
            }
        }
    }
}

// ---- observation points: the displacement kernels O (buildO) ---------------------
//
// O is row-major with 3 nobs rows (north, east, down per point) and n columns
// (the source DOFs of K); row 3k + c is column (k, c) of the reference's
// O(n, 3 nobs) (fortran/3d/src/greens.f90:302-462).  Same launch shape as K:
// one thread per source, the grid's y dimension strides over points, and each
// row store of a warp is one coalesced segment.

template <bool R32>
__global__ void __launch_bounds__(128) k_observe_rect(double *__restrict__ O, long n, long col0,
        const double *__restrict__ obs, int nobs, const double *__restrict__ src, int ns, OkMed med)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    double sr[RS_SIZE];
#pragma unroll
    for (int f = 0; f < RS_SIZE; f++) sr[f] = __ldg(src + (long)f * ns + j);
    OkDip dp;
    dp.sd = sr[RS_SD]; dp.cd = sr[RS_CD]; dp.sdsd = sr[RS_SDSD]; dp.cdcd = sr[RS_CDCD];
    dp.sdcd = sr[RS_SDCD];
    const double csst = sr[RS_CS], ssst = sr[RS_SS];
    for (int k = blockIdx.y; k < nobs; k += gridDim.y) {
        const double x1 = __ldg(obs + 3L * k), x2 = __ldg(obs + 3L * k + 1), x3 = __ldg(obs + 3L * k + 2);
        // okada92.f90:251-290
        double x = (x1 - sr[RS_Q1]) * csst + (x2 - sr[RS_Q2]) * ssst;
        double y = (x1 - sr[RS_Q1]) * ssst - (x2 - sr[RS_Q2]) * csst;
        double z = -x3;
        if (R32) {
            x = (double)__double2float_rn(x);
            y = (double)__double2float_rn(y);
            z = (double)__double2float_rn(z);
        }
        double us[3], ud[3];
        ok_dc3d_disp<R32>(med, dp, x, y, z, sr[RS_DEPTH], sr[RS_AL2], sr[RS_AW1], us, ud);
        const double oS[3] = {us[0] * csst + us[1] * ssst, us[0] * ssst - us[1] * csst, -us[2]};
        const double oD[3] = {ud[0] * csst + ud[1] * ssst, ud[0] * ssst - ud[1] * csst, -ud[2]};
#pragma unroll
        for (int c = 0; c < 3; c++)
            *reinterpret_cast<double2 *>(O + (3L * k + c) * n + col0 + 2L * j) = make_double2(oS[c], oD[c]);
    }
}

__global__ void __launch_bounds__(128) k_observe_tri(double *__restrict__ O, long n, long col0,
        const double *__restrict__ obs, int nobs, const double *__restrict__ rec, int ns, double nu)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    NwRec R{rec + j, (long)ns};
    for (int k = blockIdx.y; k < nobs; k += gridDim.y) {
        const double xr[3] = {__ldg(obs + 3L * k), __ldg(obs + 3L * k + 1), __ldg(obs + 3L * k + 2)};
        double uS[3], uD[3];
        nw_pair_disp(xr, R, nu, uS, uD);
#pragma unroll
        for (int c = 0; c < 3; c++)
            *reinterpret_cast<double2 *>(O + (3L * k + c) * n + col0 + 2L * j) = make_double2(uS[c], uD[c]);
    }
}

__global__ void __launch_bounds__(128) k_observe_vol(double *__restrict__ O, long n, long col0,
        const double *__restrict__ obs, int nobs, const double *__restrict__ rec, int ns, double mu, double nu)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ns) return;
    SvRec R{rec + j, (long)ns};
    for (int k = blockIdx.y; k < nobs; k += gridDim.y) {
        const double xr[3] = {__ldg(obs + 3L * k), __ldg(obs + 3L * k + 1), __ldg(obs + 3L * k + 2)};
        double u[6][3];
        sv_pair_disp(xr, R, mu, nu, u);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            double2 *p = reinterpret_cast<double2 *>(O + (3L * k + c) * n + col0 + 6L * j);
            p[0] = make_double2(u[0][c], u[1][c]);
            p[1] = make_double2(u[2][c], u[3][c]);
            p[2] = make_double2(u[4][c], u[5][c]);
        }
    }
}

// ---- host side -----------------------------------------------------------------

static float f32(double v) { return (float)v; }

// receiver frames and centres: okada92.f90:59-87, nikkhoo15.f90:50-101,
// strainvolume.f90:135-163
static void build_receivers(ucg_ctx *c, std::vector<double> &r)
{
    const int ne = c->nr + c->nt + c->nv;
    r.assign((size_t)ne * RC_SIZE, 0.0);
    for (int i = 0; i < c->nr; i++) {
        double *q = &r[(size_t)i * RC_SIZE];
        const double st = c->rstrike[i], dp = c->rdip[i];
        double sv[3] = {cos(st), sin(st), 0.0};
        double dv[3] = {+sin(st) * cos(dp), -cos(st) * cos(dp), -sin(dp)};
        double nv[3] = {-sin(st) * sin(dp), +cos(st) * sin(dp), -cos(dp)};
        for (int k = 0; k < 3; k++) {
            q[RC_X + k] = c->rx[3 * i + k] + c->rL[i] / 2 * sv[k] - c->rW[i] / 2 * dv[k];
            q[RC_S + k] = sv[k]; q[RC_D + k] = dv[k]; q[RC_N + k] = nv[k];
        }
    }
    for (int j = 0; j < c->nt; j++) {
        double *q = &r[(size_t)(c->nr + j) * RC_SIZE];
        const double *A = &c->tvert[3L * (c->ti1[j] - 1)];
        const double *B = &c->tvert[3L * (c->ti2[j] - 1)];
        const double *C = &c->tvert[3L * (c->ti3[j] - 1)];
        double n[3];
        n[0] = (B[1] - A[1]) * (C[2] - A[2]) - (B[2] - A[2]) * (C[1] - A[1]);
        n[1] = (B[2] - A[2]) * (C[0] - A[0]) - (B[0] - A[0]) * (C[2] - A[2]);
        n[2] = (B[0] - A[0]) * (C[1] - A[1]) - (B[1] - A[1]) * (C[0] - A[0]);
        double norm = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int k = 0; k < 3; k++) n[k] = n[k] / norm;
        if (0.0 < n[2]) for (int k = 0; k < 3; k++) n[k] = -n[k];
        double s[3] = {cos(atan2(n[0], n[1])), -sin(atan2(n[0], n[1])), 0.0};
        double d[3] = {n[1] * s[2] - n[2] * s[1], n[2] * s[0] - n[0] * s[2], n[0] * s[1] - n[1] * s[0]};
        for (int k = 0; k < 3; k++) {
            q[RC_X + k] = (A[k] + B[k] + C[k]) / 3.0;
            q[RC_S + k] = s[k]; q[RC_D + k] = d[k]; q[RC_N + k] = n[k];
        }
    }
    for (int i = 0; i < c->nv; i++) {
        double *q = &r[(size_t)(c->nr + c->nt + i) * RC_SIZE];
        const double st = c->vstrike[i];
        double sv[3] = {cos(st), sin(st), 0.0};
        double dv[3] = {0.0, 0.0, -1.0};
        double nv[3] = {-sin(st), +cos(st), -0.0};
        for (int k = 0; k < 3; k++) {
            q[RC_X + k] = c->vx[3 * i + k] + c->vL[i] / 2 * sv[k] - c->vW[i] / 2 * dv[k];
            q[RC_S + k] = sv[k]; q[RC_D + k] = dv[k]; q[RC_N + k] = nv[k];
        }
    }
}

static void build_rect_sources(ucg_ctx *c, int mode, std::vector<double> &s)
{
    const int ns = c->nr;
    const bool r32 = (mode == UCG_OKADA_REF32IO);
    const double RAD2DEG = 57.29577951308232;
    s.assign((size_t)ns * RS_SIZE, 0.0);
    auto put = [&](int f, int j, double v) { s[(size_t)f * ns + j] = v; };
    for (int j = 0; j < ns; j++) {
        double dip = c->rdip[j] * RAD2DEG;
        double depth = c->rx[3 * j + 2], L = c->rL[j], W = c->rW[j];
        if (r32) { dip = f32(dip); depth = f32(depth); L = f32(L); W = f32(W); }
        OkDip dp = ok_dip(dip);
        put(RS_Q1, j, c->rx[3 * j + 0]);
        put(RS_Q2, j, c->rx[3 * j + 1]);
        put(RS_CS, j, cos(c->rstrike[j]));
        put(RS_SS, j, sin(c->rstrike[j]));
        put(RS_DEPTH, j, depth);
        put(RS_AL2, j, L);
        put(RS_AW1, j, -W);
        put(RS_SD, j, dp.sd);
        put(RS_CD, j, dp.cd);
        put(RS_SDSD, j, dp.sdsd);
        put(RS_CDCD, j, dp.cdcd);
        put(RS_SDCD, j, dp.sdcd);
    }
}

static void build_tri_sources(ucg_ctx *c, std::vector<double> &s)
{
    const int ns = c->nt;
    s.assign((size_t)ns * NW_SIZE, 0.0);
    std::vector<double> r(NW_SIZE);
    for (int j = 0; j < ns; j++) {
        const double *A = &c->tvert[3L * (c->ti1[j] - 1)];
        const double *B = &c->tvert[3L * (c->ti2[j] - 1)];
        const double *C = &c->tvert[3L * (c->ti3[j] - 1)];
        // NED -> ENU (nikkhoo15.f90:143-146)
        double P1[3] = {A[1], A[0], -A[2]}, P2[3] = {B[1], B[0], -B[2]}, P3[3] = {C[1], C[0], -C[2]};
        nw_prepare(P1, P2, P3, r.data());
        for (int f = 0; f < NW_SIZE; f++) s[(size_t)f * ns + j] = r[f];
    }
}

static void build_vol_sources(ucg_ctx *c, std::vector<double> &s)
{
    const int ns = c->nv;
    s.assign((size_t)ns * SV_SIZE, 0.0);
    std::vector<double> r(SV_SIZE);
    for (int j = 0; j < ns; j++) {
        sv_prepare(&c->vx[3 * j], c->vL[j], c->vT[j], c->vW[j], c->vstrike[j], r.data());
        for (int f = 0; f < SV_SIZE; f++) s[(size_t)f * ns + j] = r[f];
    }
}

int assemble_matrix(ucg_ctx *c, int okada_mode)
{
    const int ne = c->nr + c->nt + c->nv;
    const int np = c->nr + c->nt;
    const long n = 2L * np + 6L * c->nv;
    const long m = 3L * np + 6L * c->nv;
    if (ne == 0) return UCG_E_BADARG;
    UCG_CUDA(cudaSetDevice(c->device));
    if (c->K && (c->n != n || c->m != m)) {
        cudaFree(c->K);
        c->K = nullptr;
    }
    if (!c->K) {
        cudaError_t e = cudaMalloc(&c->K, sizeof(double) * (size_t)n * (size_t)m);
        if (e != cudaSuccess) {
            c->K = nullptr;
            cuda_fail(c, e, "cudaMalloc(K)");
            return UCG_E_OOM;
        }
    }
    c->n = n;
    c->m = m;
    std::vector<double> rh;
    build_receivers(c, rh);
    if (c->rcv) cudaFree(c->rcv);
    UCG_CUDA(cudaMalloc(&c->rcv, sizeof(double) * rh.size()));
    UCG_CUDA(cudaMemcpyAsync(c->rcv, rh.data(), sizeof(double) * rh.size(), cudaMemcpyHostToDevice, c->stream));

    const int TPB = 128;
    const int gy = ne < 65535 ? ne : 65535;
    double *dsrc = nullptr;
    auto upload = [&](const std::vector<double> &h) -> int {
        if (dsrc) { cudaStreamSynchronize(c->stream); cudaFree(dsrc); dsrc = nullptr; }
        UCG_CUDA(cudaMalloc(&dsrc, sizeof(double) * h.size()));
        UCG_CUDA(cudaMemcpyAsync(dsrc, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->stream));
        return UCG_OK;
    };
    int rc;
    // device time of each family's launches (ucg_assembly_times)
    cudaEvent_t ev[6];
    for (cudaEvent_t &e : ev) UCG_CUDA(cudaEventCreate(&e));
    for (double &t : c->asm_ms) t = 0.0;
    // load the kernels' code before the first event: under lazy module loading
    // a first launch would otherwise count the load in its family's time
    cudaFuncAttributes fa;
    if (c->nr) UCG_CUDA(okada_mode == UCG_OKADA_REF32IO ? cudaFuncGetAttributes(&fa, k_assemble_rect<true>)
                                                        : cudaFuncGetAttributes(&fa, k_assemble_rect<false>));
    if (c->nt) {
        UCG_CUDA(cudaFuncGetAttributes(&fa, k_assemble_tri<0>));
        UCG_CUDA(cudaFuncGetAttributes(&fa, k_assemble_tri<1>));
        UCG_CUDA(cudaFuncGetAttributes(&fa, k_assemble_tri<2>));
    }
    if (c->nv) UCG_CUDA(cudaFuncGetAttributes(&fa, k_assemble_vol));
    if (c->nr) {
        std::vector<double> s;
        build_rect_sources(c, okada_mode, s);
        if ((rc = upload(s))) return rc;
        UCG_CUDA(cudaEventRecord(ev[0], c->stream));
        const double alpha_d = (c->lambda + c->mu) / (c->lambda + 2.0 * c->mu);
        const double alpha = okada_mode == UCG_OKADA_REF32IO ? (double)f32(alpha_d) : alpha_d;
        dim3 grid((c->nr + TPB - 1) / TPB, gy);
        if (okada_mode == UCG_OKADA_REF32IO)
            k_assemble_rect<true><<<grid, TPB, 0, c->stream>>>(c->K, n, 0, c->rcv, ne, np, dsrc, c->nr,
                                                              ok_med(alpha), c->mu, c->lambda);
        else
            k_assemble_rect<false><<<grid, TPB, 0, c->stream>>>(c->K, n, 0, c->rcv, ne, np, dsrc, c->nr,
                                                               ok_med(alpha), c->mu, c->lambda);
        c->launches.count++;
        UCG_CUDA(cudaGetLastError());
        UCG_CUDA(cudaEventRecord(ev[1], c->stream));
    }
    if (c->nt) {
        std::vector<double> s;
        build_tri_sources(c, s);
        if ((rc = upload(s))) return rc;
        UCG_CUDA(cudaEventRecord(ev[2], c->stream));
        NwConst cst{c->lambda / (c->lambda + c->mu) / 2.0, c->mu, c->lambda};
        dim3 grid((c->nt + TPB - 1) / TPB, gy);
        // main TD, image TD and free-surface term in three accumulating passes
        k_assemble_tri<0><<<grid, TPB, 0, c->stream>>>(c->K, n, 2L * c->nr, c->rcv, ne, np, dsrc, c->nt, cst);
        k_assemble_tri<1><<<grid, TPB, 0, c->stream>>>(c->K, n, 2L * c->nr, c->rcv, ne, np, dsrc, c->nt, cst);
        k_assemble_tri<2><<<grid, TPB, 0, c->stream>>>(c->K, n, 2L * c->nr, c->rcv, ne, np, dsrc, c->nt, cst);
        c->launches.count += 3;
        UCG_CUDA(cudaGetLastError());
        UCG_CUDA(cudaEventRecord(ev[3], c->stream));
    }
    if (c->nv) {
        std::vector<double> s;
        build_vol_sources(c, s);
        if ((rc = upload(s))) return rc;
        UCG_CUDA(cudaEventRecord(ev[4], c->stream));
        const double nu = c->lambda / (c->lambda + c->mu) / 2.0;
        dim3 grid((c->nv + TPB - 1) / TPB, gy);
        k_assemble_vol<<<grid, TPB, 0, c->stream>>>(c->K, n, 2L * np, c->rcv, ne, np, dsrc, c->nv, c->mu, nu);
        c->launches.count++;
        UCG_CUDA(cudaGetLastError());
        UCG_CUDA(cudaEventRecord(ev[5], c->stream));
    }
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    const int have[3] = {c->nr > 0, c->nt > 0, c->nv > 0};
    for (int f = 0; f < 3; f++) {
        float ms = 0.0f;
        if (have[f] && cudaEventElapsedTime(&ms, ev[2 * f], ev[2 * f + 1]) == cudaSuccess) c->asm_ms[f] = ms;
    }
    for (cudaEvent_t &e : ev) cudaEventDestroy(e);
    if (dsrc) cudaFree(dsrc);
    c->okada_mode = okada_mode;
    c->assembled = true;
    return UCG_OK;
}

int assemble_observation(ucg_ctx *c, int okada_mode)
{
    const int np = c->nr + c->nt;
    const long n = 2L * np + 6L * c->nv;
    const int nobs = (int)(c->obs_x.size() / 3);
    if (np + c->nv == 0 || nobs == 0) return UCG_E_BADARG;
    UCG_CUDA(cudaSetDevice(c->device));
    const size_t bytes = sizeof(double) * (size_t)n * 3 * (size_t)nobs;
    if (c->O && c->O_bytes != bytes) {
        cudaFree(c->O);
        c->O = nullptr;
    }
    if (!c->O) {
        cudaError_t e = cudaMalloc(&c->O, bytes);
        if (e != cudaSuccess) {
            c->O = nullptr;
            return cuda_fail(c, e, "cudaMalloc(O)");
        }
        c->O_bytes = bytes;
    }
    if (c->obs_dev) cudaFree(c->obs_dev);
    c->obs_dev = nullptr;
    UCG_CUDA(cudaMalloc(&c->obs_dev, sizeof(double) * c->obs_x.size()));
    UCG_CUDA(cudaMemcpyAsync(c->obs_dev, c->obs_x.data(), sizeof(double) * c->obs_x.size(),
                             cudaMemcpyHostToDevice, c->stream));
    const int TPB = 128;
    const int gy = nobs < 65535 ? nobs : 65535;
    double *dsrc = nullptr;
    auto upload = [&](const std::vector<double> &h) -> int {
        if (dsrc) { cudaStreamSynchronize(c->stream); cudaFree(dsrc); dsrc = nullptr; }
        UCG_CUDA(cudaMalloc(&dsrc, sizeof(double) * h.size()));
        UCG_CUDA(cudaMemcpyAsync(dsrc, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, c->stream));
        return UCG_OK;
    };
    int rc;
    cudaEvent_t ev[2];
    for (cudaEvent_t &e : ev) UCG_CUDA(cudaEventCreate(&e));
    UCG_CUDA(cudaEventRecord(ev[0], c->stream));
    if (c->nr) {
        std::vector<double> s;
        build_rect_sources(c, okada_mode, s);
        if ((rc = upload(s))) return rc;
        const double alpha_d = (c->lambda + c->mu) / (c->lambda + 2.0 * c->mu);
        const double alpha = okada_mode == UCG_OKADA_REF32IO ? (double)f32(alpha_d) : alpha_d;
        dim3 grid((c->nr + TPB - 1) / TPB, gy);
        if (okada_mode == UCG_OKADA_REF32IO)
            k_observe_rect<true><<<grid, TPB, 0, c->stream>>>(c->O, n, 0, c->obs_dev, nobs, dsrc, c->nr, ok_med(alpha));
        else
            k_observe_rect<false><<<grid, TPB, 0, c->stream>>>(c->O, n, 0, c->obs_dev, nobs, dsrc, c->nr, ok_med(alpha));
        c->launches.count++;
        UCG_CUDA(cudaGetLastError());
    }
    if (c->nt) {
        std::vector<double> s;
        build_tri_sources(c, s);
        if ((rc = upload(s))) return rc;
        dim3 grid((c->nt + TPB - 1) / TPB, gy);
        k_observe_tri<<<grid, TPB, 0, c->stream>>>(c->O, n, 2L * c->nr, c->obs_dev, nobs, dsrc, c->nt,
                                                   c->lambda / (c->lambda + c->mu) / 2.0);
        c->launches.count++;
        UCG_CUDA(cudaGetLastError());
    }
    if (c->nv) {
        std::vector<double> s;
        build_vol_sources(c, s);
        if ((rc = upload(s))) return rc;
        dim3 grid((c->nv + TPB - 1) / TPB, gy);
        k_observe_vol<<<grid, TPB, 0, c->stream>>>(c->O, n, 2L * np, c->obs_dev, nobs, dsrc, c->nv, c->mu,
                                                   c->lambda / (c->lambda + c->mu) / 2.0);
        c->launches.count++;
        UCG_CUDA(cudaGetLastError());
    }
    UCG_CUDA(cudaEventRecord(ev[1], c->stream));
    UCG_CUDA(cudaStreamSynchronize(c->stream));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) c->obs_ms = ms;
    for (cudaEvent_t &e : ev) cudaEventDestroy(e);
    if (dsrc) cudaFree(dsrc);
    c->O_ready = true;
    return UCG_OK;
}

// ---- block sources (hierarchical approximation) -----------------------------------

int block_sources_build(ucg_ctx *c, int okada_mode, BlockSources *bs)
{
    if ((c->nr > 0) == (c->nt > 0) || c->nv > 0) return UCG_E_UNSUPPORTED;   // one patch family
    UCG_CUDA(cudaSetDevice(c->device));
    std::vector<double> rh;
    build_receivers(c, rh);
    if (c->rcv) cudaFree(c->rcv);
    c->rcv = nullptr;
    UCG_CUDA(cudaMalloc(&c->rcv, sizeof(double) * rh.size()));
    UCG_CUDA(cudaMemcpy(c->rcv, rh.data(), sizeof(double) * rh.size(), cudaMemcpyHostToDevice));
    std::vector<double> s;
    bs->family = c->nr > 0 ? 0 : 1;
    bs->okada_mode = okada_mode;
    if (bs->family == 0) {
        build_rect_sources(c, okada_mode, s);
        bs->ns = c->nr;
        const double alpha_d = (c->lambda + c->mu) / (c->lambda + 2.0 * c->mu);
        bs->med = ok_med(okada_mode == UCG_OKADA_REF32IO ? (double)f32(alpha_d) : alpha_d);
    } else {
        build_tri_sources(c, s);
        bs->ns = c->nt;
        bs->cst = NwConst{c->lambda / (c->lambda + c->mu) / 2.0, c->mu, c->lambda};
    }
    UCG_CUDA(cudaMalloc(&bs->src, sizeof(double) * s.size()));
    UCG_CUDA(cudaMemcpy(bs->src, s.data(), sizeof(double) * s.size(), cudaMemcpyHostToDevice));
    return UCG_OK;
}

void block_sources_free(BlockSources *bs)
{
    if (bs->src) cudaFree(bs->src);
    bs->src = nullptr;
}

void assemble_block(ucg_ctx *c, const BlockSources &bs, const int *ridx, int nrb, const int *sidx, int nsb,
                    double *out)
{
    const int TPB = 128;
    dim3 grid((nsb + TPB - 1) / TPB, nrb < 65535 ? nrb : 65535);
    if (bs.family == 0) {
        if (bs.okada_mode == UCG_OKADA_REF32IO)
            k_block_rect<true><<<grid, TPB, 0, c->stream>>>(out, ridx, nrb, sidx, nsb, c->rcv, bs.src, bs.ns,
                                                           bs.med, c->mu, c->lambda);
        else
            k_block_rect<false><<<grid, TPB, 0, c->stream>>>(out, ridx, nrb, sidx, nsb, c->rcv, bs.src, bs.ns,
                                                            bs.med, c->mu, c->lambda);
        c->launches.count++;
    } else {
        k_block_tri<0><<<grid, TPB, 0, c->stream>>>(out, ridx, nrb, sidx, nsb, c->rcv, bs.src, bs.ns, bs.cst);
        k_block_tri<1><<<grid, TPB, 0, c->stream>>>(out, ridx, nrb, sidx, nsb, c->rcv, bs.src, bs.ns, bs.cst);
        k_block_tri<2><<<grid, TPB, 0, c->stream>>>(out, ridx, nrb, sidx, nsb, c->rcv, bs.src, bs.ns, bs.cst);
        c->launches.count += 3;
    }
}

// element bounding boxes (lo[3], hi[3] per element, patches in K's order) and centres
void element_boxes(const ucg_ctx *c, std::vector<double> &box, std::vector<double> &ctr)
{
    const int np = c->nr + c->nt;
    box.assign(6L * np, 0.0);
    ctr.assign(3L * np, 0.0);
    for (int i = 0; i < np; i++) {
        double p[4][3];
        int nv;
        if (i < c->nr) {
            const double st = c->rstrike[i], dp = c->rdip[i];
            const double sv[3] = {cos(st), sin(st), 0.0};
            const double dv[3] = {+sin(st) * cos(dp), -cos(st) * cos(dp), -sin(dp)};
            for (int k = 0; k < 3; k++) {
                const double x = c->rx[3 * i + k];
                p[0][k] = x;
                p[1][k] = x + c->rL[i] * sv[k];
                p[2][k] = x + c->rL[i] * sv[k] - c->rW[i] * dv[k];
                p[3][k] = x - c->rW[i] * dv[k];
            }
            nv = 4;
        } else {
            const int j = i - c->nr;
            const int id[3] = {c->ti1[j] - 1, c->ti2[j] - 1, c->ti3[j] - 1};
            for (int q = 0; q < 3; q++)
                for (int k = 0; k < 3; k++) p[q][k] = c->tvert[3L * id[q] + k];
            nv = 3;
        }
        for (int k = 0; k < 3; k++) {
            double lo = p[0][k], hi = p[0][k], s = 0.0;
            for (int q = 0; q < nv; q++) {
                lo = std::fmin(lo, p[q][k]);
                hi = std::fmax(hi, p[q][k]);
                s += p[q][k];
            }
            box[6L * i + k] = lo;
            box[6L * i + 3 + k] = hi;
            ctr[3L * i + k] = s / nv;
        }
    }
}

}  // namespace ucg
