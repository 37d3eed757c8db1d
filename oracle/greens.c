/*
 * Oracle: the stress-interaction matrix G and its layout.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates
 *   fortran/3d/src/greens.f90:73-275   buildG / tractionRows / stressRows
 *   fortran/3d/src/okada92.f90:368-402 traction rotation (same in nikkhoo15.f90:208-220,
 *                                      strainvolume.f90:4690-4702)
 *   fortran/3d/src/okada92.f90:424-473 stress rotation into the receiver frame
 *
 * Layout (greens.f90:214-216, 266-271): G(n,m) column-major.  Column k is one
 * receiver force DOF: patches own 3 consecutive columns (ts, td, tn), volumes
 * own 6 (s11', s12', s13', s22', s23', s33').  Within a column the sources are
 * ordered rectangles, triangles, volumes; each patch source contributes 2 rows
 * (unit strike slip, unit dip slip) and each volume 6 rows (unit eigenstrain
 * 11, 12, 13, 22, 23, 33), component fastest.
 */
#include <math.h>
#include <stdlib.h>
#include "oracle.h"

long orc_g_rows(const orc_mesh *m) { return 2L * m->nr + 2L * m->nt + 6L * m->nv; }
long orc_g_cols(const orc_mesh *m) { return 3L * m->nr + 3L * m->nt + 6L * m->nv; }

static void traction(const double *sv, const double *dv, const double *nv,
                     const double s[6], double t[3])
{
    double s11 = s[0], s12 = s[1], s13 = s[2], s22 = s[3], s23 = s[4], s33 = s[5];
    double a = nv[0] * s11 + nv[1] * s12 + nv[2] * s13;
    double b = nv[0] * s12 + nv[1] * s22 + nv[2] * s23;
    double c = nv[0] * s13 + nv[1] * s23 + nv[2] * s33;
    t[0] = a * sv[0] + b * sv[1] + c * sv[2];
    t[1] = a * dv[0] + b * dv[1] + c * dv[2];
    t[2] = +a * nv[0] + b * nv[1] + c * nv[2];
}

static void stress_rot(const double *sv, const double *dv, const double *nv,
                       const double s[6], double o[6])
{
    double s11 = s[0], s12 = s[1], s13 = s[2], s22 = s[3], s23 = s[4], s33 = s[5];
    double sa = sv[0] * s11 + sv[1] * s12 + sv[2] * s13;
    double sb = sv[0] * s12 + sv[1] * s22 + sv[2] * s23;
    double sc = sv[0] * s13 + sv[1] * s23 + sv[2] * s33;
    double na = nv[0] * s11 + nv[1] * s12 + nv[2] * s13;
    double nb = nv[0] * s12 + nv[1] * s22 + nv[2] * s23;
    double nc = nv[0] * s13 + nv[1] * s23 + nv[2] * s33;
    double da = -dv[0] * s11 - dv[1] * s12 - dv[2] * s13;
    double db = -dv[0] * s12 - dv[1] * s22 - dv[2] * s23;
    double dc = -dv[0] * s13 - dv[1] * s23 - dv[2] * s33;
    o[0] = sa * sv[0] + sb * sv[1] + sc * sv[2];
    o[1] = sa * nv[0] + sb * nv[1] + sc * nv[2];
    o[2] = -sa * dv[0] - sb * dv[1] - sc * dv[2];
    o[3] = na * nv[0] + nb * nv[1] + nc * nv[2];
    o[4] = -na * dv[0] - nb * dv[1] - nc * dv[2];
    o[5] = -da * dv[0] - db * dv[1] - dc * dv[2];
}

/* 0: strain volumes by the closed forms (strainvolume.cc); 1: by Mindlin's
   point force over the cuboid's faces (mindlin.cc), the independent route */
static int g_volume_route = 0;
void orc_set_volume_route(int route) { g_volume_route = route; }

/* stress at x due to unit component j of source number src (global source index
   over rect, tri, vol) */
static void source_stress(const orc_mesh *m, const double *x, long src, int j, double s[6])
{
    if (src < m->nr) {
        long i = src;
        double ss = (j == 0), ds = (j == 1);
        orc_okada_stress(m->okada_mode, x[0], x[1], x[2], m->rx[3 * i], m->rx[3 * i + 1],
                         m->rx[3 * i + 2], m->rL[i], m->rW[i], m->rstrike[i], m->rdip[i],
                         ss, ds, 0.0, m->mu, m->lambda, s);
        return;
    }
    src -= m->nr;
    if (src < m->nt) {
        long i = src;
        const double *A = m->tv + 3L * (m->ti1[i] - 1);
        const double *B = m->tv + 3L * (m->ti2[i] - 1);
        const double *C = m->tv + 3L * (m->ti3[i] - 1);
        orc_nw15_stress(x[0], x[1], x[2], A, B, C, (double)(j == 0), (double)(j == 1), 0.0,
                        m->mu, m->lambda, s);
        return;
    }
    src -= m->nt;
    {
        long i = src;
        double eps[6] = {0, 0, 0, 0, 0, 0};
        eps[j] = 1.0;
        double nu = m->lambda / (m->lambda + m->mu) / 2.0;
        if (g_volume_route == 1)
            orc_bml17_stress_mindlin(x[0], x[1], x[2], m->vx[3 * i], m->vx[3 * i + 1], m->vx[3 * i + 2],
                                     m->vL[i], m->vT[i], m->vW[i], m->vstrike[i], eps, m->mu, nu, s);
        else
            orc_bml17_stress(x[0], x[1], x[2], m->vx[3 * i], m->vx[3 * i + 1], m->vx[3 * i + 2],
                             m->vL[i], m->vT[i], m->vW[i], m->vstrike[i], eps, m->mu, nu, s);
    }
}

static void receiver(const orc_mesh *m, long e, const double **x, const double **sv,
                     const double **dv, const double **nv, int *dof)
{
    if (e < m->nr) {
        *x = m->rxc + 3 * e; *sv = m->rsv + 3 * e; *dv = m->rdv + 3 * e; *nv = m->rnv + 3 * e;
        *dof = 3;
        return;
    }
    e -= m->nr;
    if (e < m->nt) {
        *x = m->txc + 3 * e; *sv = m->tsv + 3 * e; *dv = m->tdv + 3 * e; *nv = m->tnv + 3 * e;
        *dof = 3;
        return;
    }
    e -= m->nt;
    *x = m->vxc + 3 * e; *sv = m->vsv + 3 * e; *dv = m->vdv + 3 * e; *nv = m->vnv + 3 * e;
    *dof = 6;
}

void orc_build_g(const orc_mesh *m, long k0, long k1, double *G)
{
    long n = orc_g_rows(m);
    long nel = (long)m->nr + m->nt + m->nv;
    long nsrc = nel;
    long k = 0;
    for (long e = 0; e < nel && k < k1; e++) {
        const double *x, *sv, *dv, *nv;
        int dof;
        receiver(m, e, &x, &sv, &dv, &nv, &dof);
        if (k + dof <= k0) { k += dof; continue; }
        long row = 0;
        for (long src = 0; src < nsrc; src++) {
            int ncomp = (src < m->nr + m->nt) ? 2 : 6;
            for (int j = 0; j < ncomp; j++, row++) {
                double s[6], o[6];
                source_stress(m, x, src, j, s);
                if (dof == 3) traction(sv, dv, nv, s, o);
                else stress_rot(sv, dv, nv, s, o);
                for (int c = 0; c < dof; c++) {
                    long col = k + c;
                    if (col >= k0 && col < k1) G[(col - k0) * n + row] = o[c];
                }
            }
        }
        k += dof;
    }
}

double orc_flop_count(void) { return 0.0; }

/* Column block [k0,k1) of G with the receivers' columns distributed over
   threads (the reference distributes receiver rows over MPI ranks). */
void orc_build_g_omp(const orc_mesh *m, long k0, long k1, double *G, int threads)
{
    long n = orc_g_rows(m);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(dynamic, 3)
#endif
    for (long k = k0; k < k1; k += 3) {
        long e1 = k + 3 < k1 ? k + 3 : k1;
        orc_build_g(m, k, e1, G + (k - k0) * n);
    }
    (void)threads;
}

/* t = G^T v for the column-major n x m block G (DGEMV "T"), columns over threads */
void orc_dgemv_t(long n, long m, const double *G, const double *v, double *t, int threads)
{
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static)
#endif
    for (long k = 0; k < m; k++) {
        const double *col = G + k * n;
        double s = 0.0;
        for (long c = 0; c < n; c++) s += col[c] * v[c];
        t[k] = s;
    }
    (void)threads;
}

/* buildO, greens.f90:302-462: O (3 nobs rows x n source DOFs, row-major; row
   3k + c is the reference's column of observation point k, component c) holds
   the displacement (north, east, down) at each point for unit slip (strike,
   dip) on each patch and unit eigenstrain on each volume. */
void orc_build_o(const orc_mesh *m, int nobs, const double *xobs, double *O)
{
    const long n = orc_g_rows(m);
    const double nu = m->lambda / (m->lambda + m->mu) / 2.0;
    for (int k = 0; k < nobs; k++) {
        const double *x = xobs + 3L * k;
        long col = 0;
        for (long i = 0; i < m->nr; i++) {
            for (int j = 0; j < 2; j++, col++) {
                double u[3];
                orc_okada_disp(m->okada_mode, x[0], x[1], x[2], m->rx[3 * i], m->rx[3 * i + 1], m->rx[3 * i + 2],
                               m->rL[i], m->rW[i], m->rstrike[i], m->rdip[i], (double)(j == 0), (double)(j == 1),
                               0.0, m->mu, m->lambda, u);
                for (int c = 0; c < 3; c++) O[(3L * k + c) * n + col] = u[c];
            }
        }
        for (long i = 0; i < m->nt; i++) {
            const double *A = m->tv + 3L * (m->ti1[i] - 1);
            const double *B = m->tv + 3L * (m->ti2[i] - 1);
            const double *C = m->tv + 3L * (m->ti3[i] - 1);
            for (int j = 0; j < 2; j++, col++) {
                double u[3];
                orc_nw15_disp(x[0], x[1], x[2], A, B, C, (double)(j == 0), (double)(j == 1), 0.0, m->mu,
                              m->lambda, u);
                for (int c = 0; c < 3; c++) O[(3L * k + c) * n + col] = u[c];
            }
        }
        for (long i = 0; i < m->nv; i++) {
            for (int j = 0; j < 6; j++, col++) {
                double eps[6] = {0, 0, 0, 0, 0, 0}, u[3];
                eps[j] = 1.0;
                orc_bml17_disp_ned(x[0], x[1], x[2], m->vx[3 * i], m->vx[3 * i + 1], m->vx[3 * i + 2], m->vL[i],
                                   m->vT[i], m->vW[i], m->vstrike[i], eps, m->mu, nu, u);
                for (int c = 0; c < 3; c++) O[(3L * k + c) * n + col] = u[c];
            }
        }
    }
}
