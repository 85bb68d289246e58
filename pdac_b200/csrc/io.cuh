// io.cuh -- PDAC's files of the time loop in the reference's formats:
//   pdac.res     restart file, tapewr / taperd (io_restart.f:31-339),
//   output.NNNN  field dump, outp (outp.f:194-384), unformatted form,
//   pdac.chm     mass check line of print_mass_residuals (residuals.f:14-136).
// The files are Fortran unformatted sequential files (write_array,
// io_parallel.f:18-65, 166-230): every WRITE statement is one record of
// whole global arrays in the flat ijk order, framed by its byte length.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "kernels3d.cuh"

namespace pdac {

// ---- mass residuals, print_mass_residuals + compute_mass_flow_rate ---------
// per block partial sums of [res_g, res_s(ns), res_gc(ng), mfr, mgd,
// msd(ns), surface]; nswp and dt scale the mass that entered through
// inlet / vent cells since the start (residuals.f:79-111)
__global__ void k_mass_resid(Prm P, Fld F, int nswp, double dt, double *partial, int nq) {
    extern __shared__ double sh[];
    const int tid = threadIdx.x, ns = P.ns, ng = P.ng;
    for (int q = 0; q < nq; ++q) sh[q * blockDim.x + tid] = 0.0;
    const double pi = 4.0 * atan(1.0);
    auto S = [&](int q) -> double & { return sh[q * blockDim.x + tid]; };
    const int qg = 0, qs = 1, qgc = 1 + ns, qmfr = 1 + ns + ng, qmgd = qmfr + 1, qmsd = qmgd + 1, qsurf = qmsd + ns;
    for (int c = blockIdx.x * blockDim.x + tid; c < P.ncell; c += gridDim.x * blockDim.x) {
        int i = c % P.nx + 1, j = (c / P.nx) % P.ny + 1, k = c / (P.nx * P.ny) + 1;
        const int fl = P.flag[c];
        if (fluid(P, c)) {
            // ivf = 1 without immersed boundaries
            double volume = P.d3 ? P.dx[i] * P.dy[j] * P.dz[k] / 1.0 : P.r[i] * P.dx[i] * P.dz[k] / 1.0;
            S(qg) += F.rgp[c] * volume;
            for (int is = 1; is <= ns; ++is) S(qs + is - 1) += SOL(F.rlk, c, is) * volume;
            for (int ig = 0; ig < ng; ++ig) S(qgc + ig) += F.rgp[c] * GAS(F.ygc, c, ig) * volume;
        } else if (fl == INLET || fl == VENT) {
            double sx, sy, sz;
            if (!P.d3) { sx = P.dz[k] * P.rb[i]; sy = 0.0; sz = P.dx[i] * P.r[i]; }
            else { sx = P.dz[k] * P.dy[j]; sy = P.dx[i] * P.dz[k]; sz = P.dy[j] * P.dx[i]; }
            double flux = F.ug[c] * sx + F.wg[c] * sz;
            if (P.d3) flux = flux + F.vg[c] * sy;
            flux = F.rgp[c] * flux;
            S(qg) -= flux * nswp * dt;
            for (int is = 1; is <= ns; ++is) {
                flux = SOL(F.us, c, is) * sx + SOL(F.ws, c, is) * sz;
                if (P.d3) flux = flux + SOL(F.vs, c, is) * sy;
                flux = SOL(F.rlk, c, is) * flux;
                S(qs + is - 1) -= flux * nswp * dt;
            }
            for (int ig = 0; ig < ng; ++ig) {
                flux = F.ug[c] * sx + F.wg[c] * sz;
                if (P.d3) flux = flux + F.vg[c] * sy;
                flux = F.rgp[c] * GAS(F.ygc, c, ig) * flux;
                S(qgc + ig) -= flux * nswp * dt;
            }
        }
        // compute_mass_flow_rate (residuals.f:171-251); nothing in 2D plane geometry
        if ((fl == VENT || fl == INLET) && (P.d3 || P.itc == 1)) {
            double sz = P.d3 ? P.dy[j] * P.dx[i] : pi * P.dx[i] * (2.0 * P.rb[i] - P.dx[i]);
            double flux = F.rgp[c] * F.wg[c] * sz;
            S(qmgd) += F.rgp[c] * sz;
            for (int is = 1; is <= ns; ++is) {
                flux = flux + SOL(F.rlk, c, is) * SOL(F.ws, c, is) * sz;
                S(qmsd + is - 1) += SOL(F.rlk, c, is) * sz;
            }
            S(qmfr) += flux;
            if (flux > 0.0) S(qsurf) += sz;
        }
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (tid < s)
            for (int q = 0; q < nq; ++q) sh[q * blockDim.x + tid] += sh[q * blockDim.x + tid + s];
        __syncthreads();
    }
    if (tid == 0)
        for (int q = 0; q < nq; ++q) partial[(size_t)q * gridDim.x + blockIdx.x] = sh[q * blockDim.x];
}

// the derived fields of cnvert after a binary restart (setup.f:359-391):
// mole fractions, void fraction and gas specific heat, for every cell
__global__ void k_restart_derive(Prm P, Fld F) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.ncell) return;
    double yg[PDAC_MAXG], xg[PDAC_MAXG];
    for (int ig = 0; ig < P.ng; ++ig) yg[ig] = GAS(F.ygc, c, ig);
    mole(P, xg, yg);
    for (int ig = 0; ig < P.ng; ++ig) GAS(F.xgc, c, ig) = xg[ig];
    double rls = 0.0;
    for (int is = 1; is <= P.ns; ++is) rls = rls + SOL(F.rlk, c, is) * P.inrl[is];
    F.ep[c] = 1.0 - rls;
    double hc = 0.0;
    for (int ig = 0; ig < P.ng; ++ig) hc = hc + hcapg1(P, P.gas_type[ig], F.tg[c]) * yg[ig];
    F.cg[c] = hc;
}

namespace io {

// ---- Fortran unformatted sequential records --------------------------------
// A record is framed by a 4-byte little-endian byte count before and after
// its data.  Records longer than 2^31 - 9 bytes are split into subrecords
// (gfortran's convention): a subrecord's leading count is negated when
// another subrecord follows, its trailing count when it continues a
// previous one.
constexpr int64_t SUBREC_MAX = 2147483639;

struct Writer {
    FILE *f = nullptr;
    bool ok = true;
    explicit Writer(const char *path) { f = path ? std::fopen(path, "wb") : nullptr; ok = f != nullptr; }
    ~Writer() { if (f) std::fclose(f); }
    void raw(const void *p, size_t n) { if (ok && n && std::fwrite(p, 1, n, f) != n) ok = false; }
    void record(const void *data, size_t bytes) {
        const unsigned char *p = static_cast<const unsigned char *>(data);
        size_t left = bytes;
        bool first = true;
        do {
            size_t part = left > (size_t)SUBREC_MAX ? (size_t)SUBREC_MAX : left;
            bool more = left > part;
            int32_t lead = more ? -(int32_t)part : (int32_t)part;
            int32_t trail = first ? (int32_t)part : -(int32_t)part;
            raw(&lead, 4);
            raw(p, part);
            raw(&trail, 4);
            p += part;
            left -= part;
            first = false;
        } while (left > 0);
    }
    bool close() {
        if (f && std::fclose(f) != 0) ok = false;
        f = nullptr;
        return ok;
    }
};

struct Reader {
    FILE *f = nullptr;
    std::string err;
    explicit Reader(const char *path) {
        f = std::fopen(path, "rb");
        if (!f) err = std::string("cannot open ") + path;
    }
    ~Reader() { if (f) std::fclose(f); }
    // read one whole record of exactly `bytes` bytes into data
    bool record(void *data, size_t bytes, const char *what) {
        if (!f) return false;
        unsigned char *p = static_cast<unsigned char *>(data);
        size_t got = 0;
        for (;;) {
            int32_t m1 = 0, m2 = 0;
            if (std::fread(&m1, 4, 1, f) != 1) { err = std::string("end of file before ") + what; return false; }
            size_t part = (size_t)(m1 < 0 ? -(int64_t)m1 : m1);
            if (got + part > bytes) { err = std::string("record of ") + what + " is longer than expected"; return false; }
            if (part && std::fread(p + got, 1, part, f) != part) { err = std::string("short record ") + what; return false; }
            if (std::fread(&m2, 4, 1, f) != 1 || (m2 < 0 ? -(int64_t)m2 : m2) != (int64_t)part) {
                err = std::string("bad record framing at ") + what;
                return false;
            }
            got += part;
            if (m1 >= 0) break;
        }
        if (got != bytes) { err = std::string("record of ") + what + " has the wrong length"; return false; }
        return true;
    }
};

// ---- Fortran G editing ------------------------------------------------------
// Gw.dEe output of one REAL*8 (F2008 10.7.5.2.2): values whose magnitude,
// rounded to d significant digits, lies in [0.1, 10^d) are written in F form
// with d - s decimals (s = digits before the point) followed by e + 2
// blanks; others in E form 0.ddd...E+eee; zero as F with d - 1 decimals.
inline std::string fortran_g(double x, int w, int d, int e) {
    char buf[128];
    const int n = e + 2;
    if (x == 0.0) {
        std::snprintf(buf, sizeof buf, "%*.*f%*s", w - n, d - 1, x, n, "");
        return buf;
    }
    char eb[64];
    std::snprintf(eb, sizeof eb, "%.*e", d - 1, x);  // rounded mantissa and exponent
    const char *ep = std::strchr(eb, 'e');
    int ex = ep ? std::atoi(ep + 1) : 0;  // |x| rounded = m.mmm * 10^ex
    int s = ex + 1;
    if (s >= 0 && s <= d) {
        std::snprintf(buf, sizeof buf, "%*.*f%*s", w - n, d - s, x, n, "");
        return buf;
    }
    // E form with a leading "0.": mantissa digits of the d-digit rounding
    std::string digits;
    for (const char *q = eb; *q && q != ep; ++q)
        if (*q >= '0' && *q <= '9') digits += *q;
    char tail[16];
    std::snprintf(tail, sizeof tail, "E%c%0*d", s < 0 ? '-' : '+', e, s < 0 ? -s : s);
    std::string body = std::string(x < 0 ? "-" : "") + "0." + digits + tail;
    std::snprintf(buf, sizeof buf, "%*s", w, body.c_str());
    return buf;
}

}  // namespace io
}  // namespace pdac
