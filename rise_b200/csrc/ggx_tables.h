// ggx_tables.h -- host-side GGX energy tables and conductor Fresnel.
#pragma once

namespace rtb200 {

constexpr int kGgxLut = 32;
constexpr int kGgxFavgNodes = 21;   // Gauss-Legendre nodes of the Fresnel average

struct GgxTables {
    float ess[kGgxLut * kGgxLut];  // [alpha][mu]
    float eavg[kGgxLut];
    float msz[kGgxLut];            // per alpha row: 2 * integral of (1 - E_ss(mu)) mu dmu
    // per alpha row: integral of (1 - E_ss(mu)) mu over the segments before
    // segment k, k = 0 .. kGgxLut + 1 (the last entry is the whole integral)
    float mscum[kGgxLut * (kGgxLut + 2)];
    // Hemispherical Fresnel average as a sum over [0, 1]: nodes mu_i and
    // weights 2 mu_i w_i, for an incident index other than air's.
    float favg_x[kGgxFavgNodes], favg_w[kGgxFavgNodes];
};

// Computed once per process (thread-safe).
const GgxTables& GetGgxTables();
// Unpolarised conductor Fresnel reflectance at |cos| of the incidence angle.
double ConductorFresnel(double cosI, double ni, double nt, double kt);
// 2 * integral over [0, 1] of ConductorFresnel(mu) mu dmu (21-point Gauss-Legendre).
double ConductorFresnelAvg(double ni, double nt, double kt);

}  // namespace rtb200
