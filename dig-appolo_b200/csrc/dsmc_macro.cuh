// Per-cell macroscopic fields from raw moment sums, in the reference's
// operation order (writeAveragedMacro / guardInvalidMacro / writeLocalMacro /
// writeRecordMacro, src/ProcessDSMC.cpp:3126-3299). Every product and sum is
// rounded on its own (no fused multiply-add), as in the reference's build.
//
// Moment order: N, Σvx, Σvy, Σvz, Σv², Σ(xx,xy,yy,yz,zz,zx), Σv v²(3), ΣIr,
// Σv Ir(3). Output order: MacroIndex (src/ProcessDSMC.h:28-49).
#pragma once

#include "dsmc_device.cuh"

namespace dsmc {

__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }

__device__ __forceinline__ void macro_core(const double* m, double Np, double rho, double dr, double* out)
{
    out[0] = rho;
    const double ux = dd(m[1], Np), uy = dd(m[2], Np), uz = dd(m[3], Np);
    out[1] = ux; out[2] = uy; out[3] = uz;
    const double ux2 = dm(ux, ux), uy2 = dm(uy, uy), uz2 = dm(uz, uz);
    const double u2 = da(da(ux2, uy2), uz2);
    const double c23 = dd(2.0, 3.0), c13 = dd(1.0, 3.0);
    const double T = dm(dd(c23, Np), ds(m[4], dm(Np, u2)));
    out[4] = T;
    const double f = dd(dm(2.0, rho), Np);
    const double n23 = dm(c23, Np), n13 = dm(c13, Np);
    out[5] = dm(f, da(da(ds(ds(ds(dm(c23, m[5]), dm(c13, m[7])), dm(c13, m[9])), dm(n23, ux2)), dm(n13, uy2)), dm(n13, uz2)));
    out[6] = dm(f, ds(m[6], dm(dm(Np, ux), uy)));
    out[7] = dm(f, da(da(ds(ds(ds(dm(c23, m[7]), dm(c13, m[5])), dm(c13, m[9])), dm(n23, uy2)), dm(n13, ux2)), dm(n13, uz2)));
    out[8] = dm(f, ds(m[8], dm(dm(Np, uy), uz)));
    out[9] = dm(f, da(da(ds(ds(ds(dm(c23, m[9]), dm(c13, m[5])), dm(c13, m[7])), dm(n23, uz2)), dm(n13, ux2)), dm(n13, uy2)));
    out[10] = dm(f, ds(m[10], dm(dm(Np, uz), ux)));
    const double g = dd(rho, Np);
    out[11] = ds(dm(g, da(ds(ds(ds(m[11], dm(dm(2.0, ux), m[5])), dm(dm(2.0, uy), m[6])), dm(dm(2.0, uz), m[10])), dm(u2, m[1]))),
                 dm(dm(dm(ux, 1.5), T), rho));
    out[12] = ds(dm(g, da(ds(ds(ds(m[12], dm(dm(2.0, ux), m[6])), dm(dm(2.0, uy), m[7])), dm(dm(2.0, uz), m[8])), dm(u2, m[2]))),
                 dm(dm(dm(uy, 1.5), T), rho));
    out[13] = ds(dm(g, da(ds(ds(ds(m[13], dm(dm(2.0, ux), m[10])), dm(dm(2.0, uy), m[8])), dm(dm(2.0, uz), m[9])), dm(u2, m[3]))),
                 dm(dm(dm(uz, 1.5), T), rho));
    out[14] = dm(dd(dd(4.0, dr), Np), m[14]);
    out[15] = dm(f, ds(m[15], dm(ux, m[14])));
    out[16] = dm(f, ds(m[16], dm(uy, m[14])));
    out[17] = dm(f, ds(m[17], dm(uz, m[14])));
}

// guardInvalidMacro, src/ProcessDSMC.cpp:3194-3211
__device__ __forceinline__ void guard_invalid(double* out)
{
    bool valid = (out[0] > 0.0) && isfinite(out[0]) && (out[4] > 0.0) && isfinite(out[4]) &&
                 (out[14] > 0.0) && isfinite(out[14]);
    for (int j = 0; valid && j < 18; ++j) valid = isfinite(out[j]);
    if (!valid)
        for (int j = 0; j < 18; ++j) out[j] = 0.0;
}

// writeAveragedMacro, src/ProcessDSMC.cpp:3126-3181
__device__ __forceinline__ void averaged_macro(const double* m, double sampleCount, double S, double Neff,
                                               double nref, double dr, double* out)
{
    const double Np = m[0];
    if (!(Np > 1.0e-12) || !isfinite(Np) || !(sampleCount > 0.0) || !isfinite(sampleCount) ||
        !(S > 0.0) || !isfinite(S) || !(Neff > 0.0) || !isfinite(Neff) || !(nref > 0.0) ||
        !isfinite(nref) || !(dr > 0.0) || !isfinite(dr)) {
        for (int j = 0; j < 18; ++j) out[j] = 0.0;
        return;
    }
    const double rho = dd(dd(dm(dd(Neff, S), Np), sampleCount), nref);
    macro_core(m, Np, rho, dr, out);
    guard_invalid(out);
}

// writeLocalMacro, src/ProcessDSMC.cpp:3224-3261
__device__ __forceinline__ void local_macro_pre(const double* m, double S, double Neff, double nref, double dr,
                                                double* out)
{
    const double Nl = m[0];
    if (!(Nl > 0.0) || !isfinite(Nl)) {
        for (int j = 0; j < 18; ++j) out[j] = 0.0;
        return;
    }
    macro_core(m, Nl, dd(dm(dd(Neff, S), Nl), nref), dr, out);
}

// writeRecordMacro, src/ProcessDSMC.cpp:3264-3299 (no validity checks)
__device__ __forceinline__ void record_macro_pre(const double* m, double S, double Neff, double nref, double dr,
                                                 double* out)
{
    const double Np = m[0];
    macro_core(m, Np, dd(dm(dd(Neff, S), Np), nref), dr, out);
}

}  // namespace dsmc
