/*
 * Oracle: Barbot, Moore & Lambert (2017) vertical strain volume (placeholder
 * until the J-integral restatement lands).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include <cmath>
#include "oracle.h"

extern "C" void orc_bml17_stress(double, double, double, double, double, double, double,
                                 double, double, double, const double *, double, double,
                                 double sig[6])
{
    for (int k = 0; k < 6; k++) sig[k] = NAN;
}

/* computeReferenceSystemVerticalStrainVolume, strainvolume.f90:135-163 */
extern "C" void orc_vol_frames(int ns, const double *x, const double *L, const double *W,
                               const double *strike, double *sv, double *dv, double *nv,
                               double *xc)
{
    for (int i = 0; i < ns; i++) {
        sv[3 * i + 0] = std::cos(strike[i]);
        sv[3 * i + 1] = std::sin(strike[i]);
        sv[3 * i + 2] = 0.0;
        dv[3 * i + 0] = 0.0;
        dv[3 * i + 1] = 0.0;
        dv[3 * i + 2] = -1.0;
        nv[3 * i + 0] = -std::sin(strike[i]);
        nv[3 * i + 1] = +std::cos(strike[i]);
        nv[3 * i + 2] = -0.0;
        for (int k = 0; k < 3; k++)
            xc[3 * i + k] = x[3 * i + k] + L[i] / 2 * sv[3 * i + k] - W[i] / 2 * dv[3 * i + k];
    }
}
