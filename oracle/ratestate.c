/*
 * Oracle: rate-and-state friction with radiation damping, power-law Maxwell
 * strain volumes, and the Cash-Karp RK4(5) integrator with NR step control.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates:
 *   fortran/3d/src/ratestate.f90:548-610      initStateVector (faults)
 *   fortran/3d/src/viscouscycles.f90:710-820  initStateVector (faults + volumes)
 *   fortran/3d/src/ratestate.f90:624-778      odefun (faults)
 *   fortran/3d/src/viscouscycles.f90:834-1093 odefun (faults + volumes)
 *   fortran/3d/src/ode45.f90:116-202          RKCKm (BLAS-1 operation order kept:
 *                                             dcopy, dscal, then daxpy)
 *   fortran/3d/src/ode45.f90:51-108           RKQSm
 *   fortran/3d/src/ratestate.f90:306-326      main-loop iteration
 * The DGEMV of odefun is a plain column dot product summed in source order.
 */
#include <math.h>
#include <string.h>
#include "oracle.h"

static const double LG10 = 2.302585092994045684017991454684364208;  /* LOG(1.d1) */
#define TINY_ 1.0e-30

static long nsrc(const orc_model *md) { return 2L * md->np + 6L * md->nvol; }
static long nrcv(const orc_model *md) { return 3L * md->np + 6L * md->nvol; }

long orc_state_len(const orc_model *md) { return 7L * md->np + 12L * md->nvol; }

/*
 * The reference's DGEMV leaves the summation order of each dot product to the
 * BLAS it links.  The order matters here: the RKQS error norm is dominated by
 * state components that are zero analytically and hold only rounding residue
 * (e.g. the dip-slip rate of a pure strike-slip fault), so the accepted step
 * sizes follow the last bits of those sums.  The oracle therefore fixes one
 * order, the device kernel's: 256 partial sums (8 groups x 32 slots), slot
 * (w, l) accumulating columns c = 64 w + 2 l + 512 k two at a time with fused
 * multiply-adds; the 32 slots of a group combine by an xor butterfly
 * (distance 16, 8, 4, 2, 1) and the 8 groups are added in order.
 */
/* > 0: odefun's DGEMV runs over this many threads in a plain summation order
   (for timing the CPU baseline); 0: the fixed order below (parity) */
static int g_dgemv_threads = 0;
void orc_set_dgemv_threads(int threads) { g_dgemv_threads = threads > 0 ? threads : 0; }

double orc_dot_fixed_order(const double *col, const double *v, long n)
{
    double part[8];
    for (int w = 0; w < 8; w++) {
        double lane[32], tmp[32];
        for (int l = 0; l < 32; l++) {
            double acc = 0.0;
            for (long c = 64L * w + 2 * l; c < n; c += 512) acc = fma(col[c + 1], v[c + 1], fma(col[c], v[c], acc));
            lane[l] = acc;
        }
        for (int off = 16; off > 0; off >>= 1) {
            for (int l = 0; l < 32; l++) tmp[l] = lane[l] + lane[l ^ off];
            memcpy(lane, tmp, sizeof lane);
        }
        part[w] = lane[0];
    }
    double s = 0.0;
    for (int w = 0; w < 8; w++) s += part[w];
    return s;
}
long orc_work_len(const orc_model *md)
{
    return 10 * orc_state_len(md) + nsrc(md) + nrcv(md);
}

void orc_init_state(const orc_model *md, double *y)
{
    long len = orc_state_len(md);
    for (long i = 0; i < len; i++) y[i] = 0.0;
    for (int i = 0; i < md->np; i++) {
        double *yy = y + 7L * i;
        double tau = md->sig[i] * (md->mu0[i] + (md->a[i] - md->b[i]) * log(md->Vpl[i] / md->Vo[i]));
        /* ratestate.f90:589 subtracts the damping term, viscouscycles.f90:750 adds it */
        if (md->viscous) tau = tau + md->damping[i] * md->Vpl[i];
        else tau = tau - md->damping[i] * md->Vpl[i];
        yy[0] = 0.0;
        yy[1] = 0.0;
        yy[2] = tau * cos(md->rake[i]);
        yy[3] = tau * sin(md->rake[i]);
        yy[4] = 0.0;
        yy[5] = log(md->L[i] / md->Vpl[i]) / LG10;
        yy[6] = log(md->Vpl[i] * (md->viscous ? 0.98 : 0.99)) / LG10;
    }
    for (int i = 0; i < md->nvol; i++) {
        double *yy = y + 7L * md->np + 12L * i;
        const double *e = md->ebg + 6L * i;
        double eps = sqrt((e[0] * e[0] + 2 * e[1] * e[1] + 2 * e[2] * e[2] + e[3] * e[3]
                           + 2 * e[4] * e[4] + e[5] * e[5]) / 2.0);
        if (0.0 < eps) {
            double tau = md->nGm[i] * pow(eps / md->gammadot0m[i] * exp(md->nQm[i] / (md->nRm[i] * md->To[i])),
                                          1.0 / md->npowerm[i]);
            for (int k = 0; k < 6; k++) yy[6 + k] = tau * e[k] / eps;
        } else {
            for (int k = 0; k < 6; k++) yy[6 + k] = 0.0;
        }
        for (int k = 0; k < 6; k++) yy[k] = 0.0;
    }
}

void orc_odefun(const orc_model *md, const double *y, double *dydt, double *vmax,
                double *work)
{
    long n = nsrc(md), m = nrcv(md), len = orc_state_len(md);
    double *v = work, *t = work + n;
    double vm = 0.0;
    for (long i = 0; i < len; i++) dydt[i] = 0.0;
    /* step 1/3: slip velocity and strain rate from the state vector */
    for (int i = 0; i < md->np; i++) {
        const double *yy = y + 7L * i;
        double rake = atan2(yy[3], yy[2]);
        double velocity = exp(yy[6] * LG10);
        double vs = velocity * cos(rake), vd = velocity * sin(rake);
        vm = velocity > vm ? velocity : vm;
        dydt[7L * i + 0] = vs;
        dydt[7L * i + 1] = vd;
        v[2L * i + 0] = vs - md->Vpl[i] * cos(md->rake[i]);
        v[2L * i + 1] = vd - md->Vpl[i] * sin(md->rake[i]);
    }
    for (int i = 0; i < md->nvol; i++) {
        const double *yy = y + 7L * md->np + 12L * i;
        double s11 = yy[6], s12 = yy[7], s13 = yy[8], s22 = yy[9], s23 = yy[10], s33 = yy[11];
        double p = (s11 + s22 + s33) / 3.0;
        s11 = s11 - p; s22 = s22 - p; s33 = s33 - p;
        double e[6] = {0, 0, 0, 0, 0, 0};
        if (md->nonlinear_maxwell) {
            double sII = sqrt((s11 * s11 + 2.0 * s12 * s12 + 2.0 * s13 * s13 + s22 * s22
                               + 2.0 * s23 * s23 + s33 * s33) / 2.0);
            double eII = md->gammadot0m[i] * pow(sII, md->npowerm[i] - 1);
            e[0] += eII * s11; e[1] += eII * s12; e[2] += eII * s13;
            e[3] += eII * s22; e[4] += eII * s23; e[5] += eII * s33;
        }
        double *dd = dydt + 7L * md->np + 12L * i;
        for (int k = 0; k < 6; k++) dd[k] = e[k];
        for (int k = 0; k < 6; k++) v[2L * md->np + 6L * i + k] = e[k] - md->ebg[6L * i + k];
    }
    /* step 2/3: t = G^T v (DGEMV "T"), column k is contiguous */
    if (md->G && g_dgemv_threads > 0) {
        /* timing mode: the columns over threads, each a plain sequential dot
           (the reference leaves the order to its BLAS) */
        const double *G = md->G;
#ifdef _OPENMP
#pragma omp parallel for num_threads(g_dgemv_threads) schedule(static)
#endif
        for (long k = 0; k < m; k++) {
            const double *col = G + k * n;
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            long c = 0;
            for (; c + 4 <= n; c += 4) {
                s0 += col[c] * v[c];
                s1 += col[c + 1] * v[c + 1];
                s2 += col[c + 2] * v[c + 2];
                s3 += col[c + 3] * v[c + 3];
            }
            for (; c < n; c++) s0 += col[c] * v[c];
            t[k] = (s0 + s1) + (s2 + s3);
        }
    } else {
        for (long k = 0; k < m; k++) {
            if (!md->G) { t[k] = 0.0; continue; }
            t[k] = orc_dot_fixed_order(md->G + k * n, v, n);
        }
    }
    /* step 3/3: remaining state rates */
    for (int i = 0; i < md->np; i++) {
        const double *yy = y + 7L * i;
        const double *tt = t + 3L * i;
        double *dd = dydt + 7L * i;
        double rake = atan2(yy[3], yy[2]);
        double velocity = exp(yy[6] * LG10);
        dd[5] = (exp(-yy[5] * LG10) - velocity / md->L[i]) / LG10;
        double dtau = tt[0] * cos(rake) + tt[1] * sin(rake);
        dd[6] = (dtau - md->b[i] * md->sig[i] * dd[5] * LG10) /
                (md->a[i] * md->sig[i] + md->damping[i] * velocity) / LG10;
        double correction = md->damping[i] * velocity * dd[6] * LG10;
        dd[2] = tt[0] - correction * cos(rake);
        dd[3] = tt[1] - correction * sin(rake);
        dd[4] = tt[2];
    }
    for (int i = 0; i < md->nvol; i++) {
        double *dd = dydt + 7L * md->np + 12L * i;
        const double *tt = t + 3L * md->np + 6L * i;
        for (int k = 0; k < 6; k++) dd[6 + k] = tt[k];
    }
    if (vmax) *vmax = vm;
}

/* BLAS-1 restatements, reference BLAS loop semantics */
static void dcopy_(long n, const double *x, double *y) { memcpy(y, x, sizeof(double) * n); }
static void dscal_(long n, double a, double *x) { for (long i = 0; i < n; i++) x[i] = a * x[i]; }
static void daxpy_(long n, double a, const double *x, double *y)
{
    for (long i = 0; i < n; i++) y[i] = y[i] + a * x[i];
}

/* Cash-Karp tableau, ode45.f90:126-134 */
#define A_B21 0.2
#define A_B31 (3.0 / 40.0)
#define A_B32 (9.0 / 40.0)
#define A_B41 0.3
#define A_B42 (-0.9)
#define A_B43 1.2
#define A_B51 (-11.0 / 54.0)
#define A_B52 2.5
#define A_B53 (-70.0 / 27.0)
#define A_B54 (35.0 / 27.0)
#define A_B61 (1631.0 / 55296.0)
#define A_B62 (175.0 / 512.0)
#define A_B63 (575.0 / 13824.0)
#define A_B64 (44275.0 / 110592.0)
#define A_B65 (253.0 / 4096.0)
#define A_C1 (37.0 / 378.0)
#define A_C3 (250.0 / 621.0)
#define A_C4 (125.0 / 594.0)
#define A_C6 (512.0 / 1771.0)
#define A_DC1 (A_C1 - 2825.0 / 27648.0)
#define A_DC3 (A_C3 - 18575.0 / 48384.0)
#define A_DC4 (A_C4 - 13525.0 / 55296.0)
#define A_DC5 (-277.0 / 14336.0)
#define A_DC6 (A_C6 - 0.25)

void orc_rkck(const orc_model *md, const double *yin, const double *dydt, double h,
              double *yout, double *yerr, double *work)
{
    long n = orc_state_len(md);
    double *ak2 = work, *ak3 = ak2 + n, *ak4 = ak3 + n, *ak5 = ak4 + n, *ak6 = ak5 + n;
    double *ytmp = ak6 + n, *yrkck = ytmp + n, *w = yrkck + n;

    dcopy_(n, yin, ytmp);
    daxpy_(n, h * A_B21, dydt, ytmp);
    orc_odefun(md, ytmp, ak2, NULL, w);

    dcopy_(n, dydt, yrkck); dscal_(n, A_B31, yrkck); daxpy_(n, A_B32, ak2, yrkck);
    dcopy_(n, yin, ytmp); daxpy_(n, h, yrkck, ytmp);
    orc_odefun(md, ytmp, ak3, NULL, w);

    dcopy_(n, dydt, yrkck); dscal_(n, A_B41, yrkck); daxpy_(n, A_B42, ak2, yrkck);
    daxpy_(n, A_B43, ak3, yrkck);
    dcopy_(n, yin, ytmp); daxpy_(n, h, yrkck, ytmp);
    orc_odefun(md, ytmp, ak4, NULL, w);

    dcopy_(n, dydt, yrkck); dscal_(n, A_B51, yrkck); daxpy_(n, A_B52, ak2, yrkck);
    daxpy_(n, A_B53, ak3, yrkck); daxpy_(n, A_B54, ak4, yrkck);
    dcopy_(n, yin, ytmp); daxpy_(n, h, yrkck, ytmp);
    orc_odefun(md, ytmp, ak5, NULL, w);

    dcopy_(n, dydt, yrkck); dscal_(n, A_B61, yrkck); daxpy_(n, A_B62, ak2, yrkck);
    daxpy_(n, A_B63, ak3, yrkck); daxpy_(n, A_B64, ak4, yrkck); daxpy_(n, A_B65, ak5, yrkck);
    dcopy_(n, yin, ytmp); daxpy_(n, h, yrkck, ytmp);
    orc_odefun(md, ytmp, ak6, NULL, w);

    dcopy_(n, dydt, yrkck); dscal_(n, A_C1, yrkck); daxpy_(n, A_C3, ak3, yrkck);
    daxpy_(n, A_C4, ak4, yrkck); daxpy_(n, A_C6, ak6, yrkck);
    dcopy_(n, yin, yout); daxpy_(n, h, yrkck, yout);

    dcopy_(n, dydt, yerr); dscal_(n, A_DC1, yerr); daxpy_(n, A_DC3, ak3, yerr);
    daxpy_(n, A_DC4, ak4, yerr); daxpy_(n, A_DC5, ak5, yerr); daxpy_(n, A_DC6, ak6, yerr);
    dscal_(n, h, yerr);
}

int orc_rkqs(const orc_model *md, double *t, double *y, const double *dydt,
             const double *yscal, double htry, double epsilon, double hmax,
             double *hdid, double *hnext, long *nrej, double *work)
{
    const double SAFETY = 0.7, PGROW = -0.2, PSHRNK = -0.15, ERRCON = 1.89e-4;
    long n = orc_state_len(md);
    double *ycand = work, *yerr = ycand + n, *w = yerr + n;
    double h = htry;
    for (;;) {
        orc_rkck(md, y, dydt, h, ycand, yerr, w);
        double errmax = 0.0;
        for (long i = 0; i < n; i++) {
            double e = fabs(yerr[i] / yscal[i]);
            if (e > errmax) errmax = e;
        }
        errmax = errmax / epsilon;
        if (errmax > 1.0) {
            h = h * SAFETY * pow(errmax, PSHRNK);
            if (h < 0.5 * h) h = 0.5 * h;   /* never true; kept as in ode45.f90:83 */
            double tnew = *t + h;
            if (nrej) (*nrej)++;
            if (tnew == *t) return 4;
        } else {
            if (errmax > ERRCON) *hnext = SAFETY * h * pow(errmax, PGROW);
            else *hnext = 10.0 * h;
            if (*hnext > hmax) *hnext = hmax;
            *hdid = h;
            *t = *t + h;
            memcpy(y, ycand, sizeof(double) * n);
            return 0;
        }
    }
}

int orc_step(const orc_model *md, double *time, double *y, double *dydt,
             double *dt_next, double epsilon, double hmax, double *dt_done,
             long *nrej, double *work)
{
    long n = orc_state_len(md);
    double *yscal = work, *w = work + n;
    orc_odefun(md, y, dydt, NULL, w);
    double dt_try = *dt_next;
    for (long i = 0; i < n; i++) yscal[i] = fabs(y[i]) + fabs(dt_try * dydt[i]) + TINY_;
    double t0 = 0.0;
    int rc = orc_rkqs(md, &t0, y, dydt, yscal, dt_try, epsilon, hmax, dt_done, dt_next, nrej, w);
    if (rc) return rc;
    *time = *time + *dt_done;
    return 0;
}
