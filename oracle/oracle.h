/*
 * CPU oracle for the unicycle-b200 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the unicycle_b200 package,
 * libucg.so) links, loads or calls this code.  It is the checker: tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference arm
 * are its only users.
 *
 * Each routine restates the reference Fortran/C algorithm for one step of the
 * 3-D quasi-dynamic boundary-integral path and cites the reference lines it
 * follows (paths relative to the unicycle project root).
 *
 * Conventions shared with the reference:
 *   - coordinates are (north, east, down), angles in radians;
 *   - G is the reference's G(n,m), Fortran column-major: column k is one
 *     receiver force DOF, row c is one source DOF (fortran/3d/src/greens.f90:73-275);
 *   - patch state is 7 doubles per element, order ss,sd,ts,td,tn,log10(theta),
 *     log10(V) (fortran/3d/src/macros.f90:56-64); volume state is 12 doubles
 *     e11..e33,s11..s33 (fortran/3d/src/macros.f90:67-79).
 */
#ifndef UCG_ORACLE_H
#define UCG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Okada (1992) modes: see okada92.c. */
#define ORC_OKADA_FP64    0
#define ORC_OKADA_REF32IO 1

/* ---- okada92.c ---------------------------------------------------------- */
int  orc_dc3d(int mode, double alpha, double x, double y, double z, double depth,
              double dip_deg, double al1, double al2, double aw1, double aw2,
              double disl1, double disl2, double disl3, double u[12]);
void orc_okada_stress(int mode, double x1, double x2, double x3,
                      double q1, double q2, double q3, double L, double W,
                      double strike, double dip, double s, double d, double t,
                      double G, double lambda, double sig[6]);
void orc_okada_frames(int ns, const double *x, const double *L, const double *W,
                      const double *strike, const double *dip,
                      double *sv, double *dv, double *nv, double *xc);

/* ---- nikkhoo15.c -------------------------------------------------------- */
void orc_nw15_stress(double x1, double x2, double x3, const double P1[3],
                     const double P2[3], const double P3[3], double s, double d,
                     double t, double G, double lambda, double sig[6]);
void orc_tri_frames(int ns, int nve, const double *v, const int *i1, const int *i2,
                    const int *i3, double *sv, double *dv, double *nv, double *xc);

/* ---- strainvolume.c ----------------------------------------------------- */
void orc_bml17_stress(double x1, double x2, double x3, double q1, double q2,
                      double q3, double L, double T, double W, double theta,
                      const double eps[6], double G, double nu, double sig[6]);
void orc_vol_frames(int ns, const double *x, const double *L, const double *W,
                    const double *strike, double *sv, double *dv, double *nv,
                    double *xc);

/* ---- mindlin.cc: the same stress by Mindlin's point force integrated over the
   cuboid's faces (independent of the closed forms above) ------------------- */
void orc_bml17_stress_mindlin(double x1, double x2, double x3, double q1, double q2,
                              double q3, double L, double T, double W, double theta,
                              const double eps[6], double G, double nu, double sig[6]);
void orc_cuboid_grad_mindlin(double x1p, double x2p, double x3, double q3, double L,
                             double T, double W, const double eps[6], double G,
                             double nu, double grad[9]);
void orc_mindlin(double x, double y, double z, double c, double G, double nu, double u[9]);
/* strain-volume sources of orc_build_g / orc_build_o: 0 closed forms, 1 Mindlin route */
void orc_set_volume_route(int route);

/* ---- greens.c ----------------------------------------------------------- */
typedef struct {
    int nr, nt, nv;                 /* rectangles, triangles, volumes */
    const double *rx, *rL, *rW, *rstrike, *rdip;          /* rect geometry */
    const double *rsv, *rdv, *rnv, *rxc;                   /* rect frames   */
    int nve; const double *tv; const int *ti1, *ti2, *ti3; /* 1-based vertex ids */
    const double *tsv, *tdv, *tnv, *txc;                   /* tri frames    */
    const double *vx, *vL, *vT, *vW, *vstrike;             /* volume geometry */
    const double *vsv, *vdv, *vnv, *vxc;                   /* volume frames  */
    double mu, lambda;
    int okada_mode;
} orc_mesh;

long orc_g_rows(const orc_mesh *m);   /* n: source DOFs   */
long orc_g_cols(const orc_mesh *m);   /* m: receiver DOFs */
/* Fill columns [k0,k1) of G (column-major, leading dimension n). */
void orc_build_g(const orc_mesh *m, long k0, long k1, double *G);
void orc_build_g_omp(const orc_mesh *m, long k0, long k1, double *G, int threads);
void orc_dgemv_t(long n, long m, const double *G, const double *v, double *t, int threads);

/* ---- ratestate.c -------------------------------------------------------- */
typedef struct {
    int np;          /* patches (rect then tri) */
    int nvol;        /* strain volumes */
    const double *Vpl, *rake, *mu0, *sig, *a, *b, *L, *Vo, *damping;  /* per patch */
    const double *ebg;        /* 6 per volume: background strain rate */
    const double *gammadot0m; /* per volume */
    const double *npowerm;    /* per volume */
    const double *nGm, *nQm, *nRm, *To; /* per volume, state init only */
    int nonlinear_maxwell;    /* nNonlinearMaxwell > 0 */
    int viscous;              /* 1: viscouscycles driver conventions */
    const double *G;          /* column-major n x m, n = 2np+6nvol, m = 3np+6nvol;
                                 NULL: no interaction (t = 0), used to time the O(N) work */
} orc_model;

long orc_state_len(const orc_model *md);
/* odefun's DGEMV: threads > 0 runs the columns over that many threads with a
   plain summation order (timing the CPU baseline); 0 (default) the fixed order */
void orc_set_dgemv_threads(int threads);
/* one DGEMV dot product in the fixed summation order documented in ratestate.c */
double orc_dot_fixed_order(const double *col, const double *v, long n);
void orc_init_state(const orc_model *md, double *y);
/* odefun: dydt = f(y); vmax (may be NULL) receives max patch velocity.
   work must hold n + m doubles. */
void orc_odefun(const orc_model *md, const double *y, double *dydt, double *vmax,
                double *work);
/* RKCKm: one Cash-Karp attempt.  work: 6*len + n + m doubles. */
void orc_rkck(const orc_model *md, const double *y, const double *dydt, double h,
              double *yout, double *yerr, double *work);
/* RKQSm: step control loop.  Returns 0, or 4 on stepsize underflow.
   On success y <- accepted state, *hdid, *hnext set, *nrej += rejections. */
int  orc_rkqs(const orc_model *md, double *t, double *y, const double *dydt,
              const double *yscal, double htry, double epsilon, double hmax,
              double *hdid, double *hnext, long *nrej, double *work);
/* One iteration of the main loop (fortran/3d/src/ratestate.f90:307-326):
   odefun, yscal, RKQSm, time update.  dydt receives f(y) at the start. */
int  orc_step(const orc_model *md, double *time, double *y, double *dydt,
              double *dt_next, double epsilon, double hmax, double *dt_done,
              long *nrej, double *work);
long orc_work_len(const orc_model *md);

/* Count of floating-point operations executed by the kernels above (op-counting
   build only; 0 otherwise). */
double orc_flop_count(void);

/* displacements (north, east, down) for the observation points (buildO) */
void orc_okada_disp(int mode, double x1, double x2, double x3, double q1, double q2, double q3,
                    double L, double W, double strike, double dipd, double s, double d, double t,
                    double G, double lambda, double u[3]);
void orc_nw15_disp(double x1, double x2, double x3, const double P1[3], const double P2[3],
                   const double P3[3], double s, double d, double t, double G, double lambda, double u[3]);
void orc_bml17_disp_ned(double x1, double x2, double x3, double q1, double q2, double q3, double L,
                        double T, double W, double theta, const double eps[6], double G, double nu,
                        double u[3]);
void orc_build_o(const orc_mesh *m, int nobs, const double *xobs, double *O);

/* step-size perceptron (mlp.c): loss and gradient, predictions */
int  orc_mlp_nparam(void);
void orc_mlp_loss_grad(const float *params, const float *norm, const float *X, const float *Y, long n,
                       int fp16, double *grad, double *loss);
void orc_mlp_predict(const float *params, const float *norm, const float *X, long n, int fp16, double *out);

#ifdef __cplusplus
}
#endif
#endif
