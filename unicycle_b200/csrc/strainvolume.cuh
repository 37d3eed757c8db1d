// Barbot, Moore & Lambert (2017) vertical cuboid strain volume, device side.
// (Interface only until the J-integral evaluation lands; ucg_set_volumes
// reports UCG_E_UNSUPPORTED meanwhile, so these are never reached.)
#pragma once
#include <cuda_runtime.h>

namespace ucg {

enum : int { SV_SIZE = 8 };
constexpr bool kVolumesBuilt = false;

struct SvRec {
    const double *__restrict__ base;
    long stride;
    __device__ __forceinline__ double operator[](int f) const { return __ldg(base + (long)f * stride); }
};

inline void sv_prepare(const double *x, double L, double T, double W, double strike, double *r)
{
    r[0] = x[0]; r[1] = x[1]; r[2] = x[2]; r[3] = L; r[4] = T; r[5] = W; r[6] = strike; r[7] = 0.0;
}

__device__ inline void sv_pair_stress(const double *, const SvRec &, double, double, double sig[6][6])
{
    for (int q = 0; q < 6; q++)
        for (int k = 0; k < 6; k++) sig[q][k] = 0.0;
}

}  // namespace ucg
