/*
 * Oracle: stress of a uniformly strained vertical cuboid in a half-space by a
 * route independent of the Barbot, Moore & Lambert (2017) closed forms.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * A uniform eigenstrain e* in a volume V is equivalent to the body force
 * f = -div(s* chi_V), s* = lambda tr(e*) I + 2 mu e* (Eshelby): a surface force
 * s* n on the boundary of V (n the outward normal).  Its displacement is the
 * surface integral of the point-force Green's function of the half-space,
 *
 *     u_i(x) = sum over the six faces of  int G_ij(x; xi) s*_jk n_k dS(xi),
 *
 * with G from Mindlin (1936), "Force at a point in the interior of a
 * semi-infinite solid", Physics 7, 195-202 (the closed form below: the Kelvin
 * solution about the source, its image, and the terms that clear the
 * tractions on the free surface).  The faces are integrated by Gauss-Legendre
 * product rules on panels refined towards the observation point until every
 * panel lies at least 1.5 of its diagonal away from it; the displacement
 * gradient comes from evaluating the Green's function on forward-mode dual
 * numbers seeded with the observation point (exact differentiation).  Strain,
 * the removal of the eigenstrain inside the cuboid and Hooke's law are done in
 * the (north, east, down) frame, the meaning of the reference's
 * computeStressVerticalStrainVolume (fortran/3d/src/strainvolume.f90:1042-1140):
 * stress at x from eigenstrain eps given in the cuboid frame (x1' along strike
 * from the corner q, x2' across, x3 down; 0 < x1' < L, |x2'| < T/2,
 * q3 < x3 < q3 + W).
 *
 * Nothing here shares code or formulas with csrc/bml17_disp.h or the
 * reference's J integrals; the Green's function itself is checked by
 * tests/test_oracle.py (Navier's equations, traction-free surface,
 * reciprocity, Kelvin singularity).
 */
#include <cmath>
#include <vector>
#include "dual3.h"
#include "oracle.h"

namespace {

template <class T> inline T pw3(const T &a) { return a * a * a; }
template <class T> inline T pw5(const T &a) { return a * a * a * a * a; }

/* u[i][j]: displacement i at (x, y, z) (z depth, >= 0) from a unit force along
   j at (0, 0, c), c > 0; axes (north, east, down) */
template <class T>
void mindlin(const T &x, const T &y, const T &z, double c, double mu, double nu, T u[3][3])
{
    const double A = 1.0 / (16.0 * M_PI * mu * (1.0 - nu));
    const double k = 3.0 - 4.0 * nu;
    const double B = 4.0 * (1.0 - nu) * (1.0 - 2.0 * nu);
    const T zm = z - c, zp = z + c;
    const T R1 = sqrt(x * x + y * y + zm * zm);
    const T R2 = sqrt(x * x + y * y + zp * zp);
    const T P = R2 + zp;
    const T R13 = pw3(R1), R23 = pw3(R2), R25 = pw5(R2);
    const T cz = c * z;
    // horizontal forces: along x, and along y (x and y exchanged)
    const T hxx = k / R1 + 1.0 / R2 + x * x / R13 + k * x * x / R23 + 2.0 * cz / R23 * (1.0 - 3.0 * x * x / (R2 * R2)) +
                  B / P * (1.0 - x * x / (R2 * P));
    const T hyy = k / R1 + 1.0 / R2 + y * y / R13 + k * y * y / R23 + 2.0 * cz / R23 * (1.0 - 3.0 * y * y / (R2 * R2)) +
                  B / P * (1.0 - y * y / (R2 * P));
    const T hxy = x * y * (1.0 / R13 + k / R23 - 6.0 * cz / R25 - B / (R2 * P * P));
    const T hz = zm / R13 + k * zm / R23 - 6.0 * cz * zp / R25 + B / (R2 * P);
    // vertical force
    const T vh = zm / R13 + k * zm / R23 - B / (R2 * P) + 6.0 * cz * zp / R25;
    const T vzz = k / R1 + (8.0 * (1.0 - nu) * (1.0 - nu) - k) / R2 + zm * zm / R13 + (k * zp * zp - 2.0 * cz) / R23 +
                  6.0 * cz * zp * zp / R25;
    u[0][0] = A * hxx;
    u[1][0] = A * hxy;
    u[2][0] = A * x * hz;
    u[0][1] = A * hxy;
    u[1][1] = A * hyy;
    u[2][1] = A * y * hz;
    u[0][2] = A * x * vh;
    u[1][2] = A * y * vh;
    u[2][2] = A * vzz;
}

/* Gauss-Legendre nodes and weights on [-1, 1] (Newton on the Legendre
   recurrence) */
struct Gauss {
    std::vector<double> x, w;
    explicit Gauss(int n) : x(n), w(n)
    {
        for (int i = 0; i < n; i++) {
            double t = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
            for (int it = 0; it < 100; it++) {
                double p0 = 1.0, p1 = t;
                for (int k = 2; k <= n; k++) {
                    const double p2 = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
                    p0 = p1;
                    p1 = p2;
                }
                dp = n * (t * p1 - p0) / (t * t - 1.0);
                const double dt = p1 / dp;
                t -= dt;
                if (std::fabs(dt) < 1e-16) break;
            }
            x[i] = t;
            w[i] = 2.0 / ((1.0 - t * t) * dp * dp);
        }
    }
};

const Gauss &gauss()
{
    static const Gauss g(12);
    return g;
}

struct Face {
    int axis;       // the face's constant coordinate (0, 1, 2)
    double value;   // that coordinate
    double sign;    // outward normal along the axis
    int a, b;       // the two in-plane axes
};

/* the surface force s* n integrated with G over one rectangle of a face,
   refined towards the observation point; adds into g[i] (dual: gradient) */
void face_rect(const D3 obs[3], const Face &f, double a0, double a1, double b0, double b1, const double tr[3],
               double mu, double nu, int depth, D3 g[3])
{
    // distance from the observation point to the rectangle, against its size
    double p[3];
    p[f.axis] = f.value;
    const double oa = obs[f.a].v, ob = obs[f.b].v;
    p[f.a] = std::fmin(std::fmax(oa, a0), a1);
    p[f.b] = std::fmin(std::fmax(ob, b0), b1);
    double d2 = 0.0;
    for (int k = 0; k < 3; k++) d2 += (obs[k].v - p[k]) * (obs[k].v - p[k]);
    const double diag = std::sqrt((a1 - a0) * (a1 - a0) + (b1 - b0) * (b1 - b0));
    if (depth < 14 && std::sqrt(d2) < 1.5 * diag) {
        const double am = 0.5 * (a0 + a1), bm = 0.5 * (b0 + b1);
        face_rect(obs, f, a0, am, b0, bm, tr, mu, nu, depth + 1, g);
        face_rect(obs, f, am, a1, b0, bm, tr, mu, nu, depth + 1, g);
        face_rect(obs, f, a0, am, bm, b1, tr, mu, nu, depth + 1, g);
        face_rect(obs, f, am, a1, bm, b1, tr, mu, nu, depth + 1, g);
        return;
    }
    const Gauss &G = gauss();
    const int n = (int)G.x.size();
    const double ha = 0.5 * (a1 - a0), hb = 0.5 * (b1 - b0);
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < n; j++) {
            double xi[3];
            xi[f.axis] = f.value;
            xi[f.a] = 0.5 * (a0 + a1) + ha * G.x[i];
            xi[f.b] = 0.5 * (b0 + b1) + hb * G.x[j];
            const double wgt = G.w[i] * G.w[j] * ha * hb;
            D3 u[3][3];
            mindlin(obs[0] - xi[0], obs[1] - xi[1], obs[2], xi[2], mu, nu, u);
            for (int r = 0; r < 3; r++)
                g[r] += (u[r][0] * tr[0] + u[r][1] * tr[1] + u[r][2] * tr[2]) * wgt;
        }
    }
}

}  // namespace

/* displacement gradient grad[i][d] = d u_i / d x_d in the cuboid frame at the
   cuboid-frame point (x1p, x2p, x3), eigenstrain eps (cuboid frame) */
extern "C" void orc_cuboid_grad_mindlin(double x1p, double x2p, double x3, double q3, double L, double T, double W,
                                        const double eps[6], double G, double nu, double grad[9])
{
    const double lambda = 2.0 * G * nu / (1.0 - 2.0 * nu);
    const double e[3][3] = {{eps[0], eps[1], eps[2]}, {eps[1], eps[3], eps[4]}, {eps[2], eps[4], eps[5]}};
    const double tr = eps[0] + eps[3] + eps[5];
    double s[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) s[i][j] = 2.0 * G * e[i][j] + (i == j ? lambda * tr : 0.0);
    const D3 obs[3] = {D3::var(x1p, 0), D3::var(x2p, 1), D3::var(x3, 2)};
    const double lo[3] = {0.0, -0.5 * T, q3}, hi[3] = {L, 0.5 * T, q3 + W};
    D3 g[3];
    for (int ax = 0; ax < 3; ax++) {
        const int a = (ax + 1) % 3, b = (ax + 2) % 3;
        for (int side = 0; side < 2; side++) {
            const Face f{ax, side ? hi[ax] : lo[ax], side ? 1.0 : -1.0, a, b};
            const double t[3] = {s[0][ax] * f.sign, s[1][ax] * f.sign, s[2][ax] * f.sign};
            face_rect(obs, f, lo[a], hi[a], lo[b], hi[b], t, G, nu, 0, g);
        }
    }
    for (int i = 0; i < 3; i++)
        for (int d = 0; d < 3; d++) grad[3 * i + d] = g[i].d[d];
}

/* Mindlin's Green's function for tests: u[3 i + j] at (x, y, z) from a unit
   force along j at (0, 0, c) */
extern "C" void orc_mindlin(double x, double y, double z, double c, double G, double nu, double u[9])
{
    double r[3][3];
    mindlin<double>(x, y, z, c, G, nu, r);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) u[3 * i + j] = r[i][j];
}

/* stress (north, east, down; order 11, 12, 13, 22, 23, 33) at x from eigenstrain
   eps (cuboid frame) of the cuboid with corner q, dimensions L, T, W and strike
   theta: the quantity of computeStressVerticalStrainVolume
   (fortran/3d/src/strainvolume.f90:1042-1140) by the Mindlin route */
extern "C" void orc_bml17_stress_mindlin(double x1, double x2, double x3, double q1, double q2, double q3,
                                         double L, double T, double W, double theta, const double eps[6],
                                         double G, double nu, double sig[6])
{
    const double ct = std::cos(theta), st = std::sin(theta);
    const double x1p = (x1 - q1) * ct + (x2 - q2) * st;
    const double x2p = -(x1 - q1) * st + (x2 - q2) * ct;
    double gp[9];
    orc_cuboid_grad_mindlin(x1p, x2p, x3, q3, L, T, W, eps, G, nu, gp);
    // R maps cuboid-frame components to (north, east, down): columns e1', e2', e3
    const double R[3][3] = {{ct, -st, 0.0}, {st, ct, 0.0}, {0.0, 0.0, 1.0}};
    const double ep[3][3] = {{eps[0], eps[1], eps[2]}, {eps[1], eps[3], eps[4]}, {eps[2], eps[4], eps[5]}};
    const bool inside = x1p > 0.0 && x1p < L && std::fabs(x2p) < 0.5 * T && x3 > q3 && x3 < q3 + W;
    double e[3][3];
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            double sgr = 0.0, sep = 0.0;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    const double sym = 0.5 * (gp[3 * a + b] + gp[3 * b + a]);
                    sgr += R[i][a] * sym * R[j][b];
                    sep += R[i][a] * ep[a][b] * R[j][b];
                }
            e[i][j] = sgr - (inside ? sep : 0.0);
        }
    }
    const double lambda = 2.0 * G * nu / (1.0 - 2.0 * nu);
    const double kk = e[0][0] + e[1][1] + e[2][2];
    sig[0] = lambda * kk + 2.0 * G * e[0][0];
    sig[1] = 2.0 * G * e[0][1];
    sig[2] = 2.0 * G * e[0][2];
    sig[3] = lambda * kk + 2.0 * G * e[1][1];
    sig[4] = 2.0 * G * e[1][2];
    sig[5] = lambda * kk + 2.0 * G * e[2][2];
}
