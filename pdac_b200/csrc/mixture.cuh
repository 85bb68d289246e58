// mixture.cuh -- the gas-particle mixture fields (mixture.f:32-52 with
// derived.f:220-331), computed after every step when compute_mixture is set
// (prog.f:331) and written with the output files.  Every cell, boundary
// frame included, as the reference's loops over the whole local array.
#pragma once
#include "kernels3d.cuh"

namespace pdac {

template <int D>
__global__ void k_mixture(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    const size_t n = P.ncell;
    const int ns = P.ns, ng = P.ng;
    const double rgp = F.rgp[c];
    // mixture_density (derived.f:252-267): rgp + SUM(rlk)
    double srl = 0.0;
    for (int is = 1; is <= ns; ++is) srl = srl + F.rlk[(is - 1) * n + c];
    const double rhom = rgp + srl;
    F.rhom[c] = rhom;
    // mixture_temperature (derived.f:269-296)
    const double tg = F.tg[c];
    double cgas = 0.0;
    for (int ig = 0; ig < ng; ++ig) cgas = hcapg1(P, P.gas_type[ig], tg) * GAS(F.ygc, c, ig) + cgas;
    double sts = 0.0, scp = 0.0;
    for (int is = 1; is <= ns; ++is) {
        const double rl = F.rlk[(is - 1) * n + c];
        sts = sts + rl * P.cps[is] * F.ts[(is - 1) * n + c];
        scp = scp + rl * P.cps[is];
    }
    double tm = rgp * cgas * tg + sts;
    const double den = rgp * cgas + scp;
    F.tm[c] = tm / den;
    // mixture_velocity (derived.f:314-331), one component at a time
    auto velm = [&](const double *ug, const double *us) {
        double s = 0.0;
        for (int is = 1; is <= ns; ++is) s = s + F.rlk[(is - 1) * n + c] * us[(is - 1) * n + c];
        double v = rgp * ug[c] + s;
        return v / rhom;
    };
    F.um[c] = velm(F.ug, F.us);
    if (D == 3) F.vm[c] = velm(F.vg, F.vs);
    F.wm[c] = velm(F.wg, F.ws);
    // mixture_mass_fractions (derived.f:220-250)
    const double inrhom = 1.0 / rhom;
    for (int ig = 0; ig < ng; ++ig) F.yd[ig * n + c] = GAS(F.ygc, c, ig) * rgp * inrhom;
    for (int is = 1; is <= ns; ++is) F.yd[(ng + is - 1) * n + c] = F.rlk[(is - 1) * n + c] * inrhom;
}

}  // namespace pdac
