// ib.cuh -- immersed boundaries on the device: the forcing-point branch of
// the boundary pass and the ordered boundary pass it needs.
//
// The reference's boundary routine visits the cells in index order and
// updates in place (bdry.f:22-726): a fluid cell writes its wall and
// open-boundary neighbours, a forcing point (immersed or filled cell,
// bdry.f:103-204) interpolates its velocities from its neighbours (velint,
// velint3d, interp.f:321-781) and may fill a neighbour's scalar state (hn,
// interp.f:832-919).  On a flat mesh no two cells' updates touch the same
// cell and one thread per cell gives the reference's result; with
// topography they can (a wall cell of a step written from above and from
// the side, a forcing point reading a cell another one fills).  The host
// then orders the boundary cells into levels (pdac_gpu_create): every cell
// of a level is independent of the others of that level, and a cell comes
// in a later level than every cell before it in index order whose update it
// reads or overwrites, so running the levels in turn gives the reference's
// sequential result.
#pragma once
#include "kernels3d.cuh"

namespace pdac {

// forcing-point tables and coordinates on the device
struct IbDev {
    const int *fp[3];       // per axis: nfp x 6 (i, j, k, type, index_q, index_qq)
    const double *nsl[3];   // per axis: nfp x 3 (the no-slip point)
    double *vel[3];         // per axis: nfp x nph (written here, read by tilde)
    const double *x, *xb, *y, *yb, *z, *zb;  // 1-based, two cells of padding each side: a[q + 1]
    double *fc2;            // per cell: the filled_cell_2 toggle (0 or 1)
};

__device__ __forceinline__ double crd(const double *a, int q) { return a[q + 1]; }

// velint, interp.f:321-582 (2D); vel[0] gas, vel[is] class is
__device__ void velint2d_d(const Prm &P, const IbDev &B, int a, int f, int c, const double *velg, const double *vels,
                           double *vel) {
    const int *fp = B.fp[a] + (size_t)6 * f;
    const int i = fp[0], k = fp[2], kind = fp[3];
    const double nsx = B.nsl[a][(size_t)3 * f], nsz = B.nsl[a][(size_t)3 * f + 2];
    const double *cx = a == 0 ? B.xb : B.x;
    const double *cz = a == 0 ? B.z : B.zb;
    const int n = P.ncell, ns = P.ns;
    Raw2 R;
    raw2(P, c % P.nx + 1, c / P.nx + 1, R);
    const int immjkpp = R.wt, ippjkpp = R.et;  // interp.f:352-353
    auto V = [&](int cell, int ph) { return ph == 0 ? velg[cell] : vels[(size_t)(ph - 1) * n + cell]; };
    auto sq = [](double v) { return v * v; };
    for (int ph = 0; ph <= ns; ++ph) vel[ph] = 0.0;
    double h, zA, zB, alpha, beta;
    // the linear forms: h/zA against the first node, or the two-node line
    auto lin = [&](int n1, int n2, double zb_) {
        if (h <= zA) {
            for (int ph = 0; ph <= ns; ++ph) vel[ph] = -h / zA * V(n1, ph);
        } else {
            zB = zb_;
            for (int ph = 0; ph <= ns; ++ph) vel[ph] = -((zB - h) * V(n1, ph) + (h - zA) * V(n2, ph)) / (zB - zA);
        }
    };
    switch (kind) {
    case -3:
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i - 1) - nsx) + sq(crd(cz, k + 1) - nsz));
        lin(R.wt, immjkpp, h <= zA ? 0.0 : sqrt(sq(crd(cx, i - 2) - nsx) + sq(crd(cz, k + 2) - nsz)));
        break;
    case -2:
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i - 1) - nsx) + sq(crd(cz, k) - nsz));
        lin(R.w, R.ww, h <= zA ? 0.0 : sqrt(sq(crd(cx, i - 2) - nsx) + sq(crd(cz, k) - nsz)));
        break;
    case -1:
        alpha = (crd(cx, i - 1) - nsx) / (crd(cx, i - 1) - crd(cx, i));
        beta = (crd(cz, k + 1) - nsz) / (crd(cz, k + 1) - crd(cz, k));
        for (int ph = 0; ph <= ns; ++ph)
            vel[ph] = -(alpha * (1 - beta) * V(R.t, ph) + (1 - alpha) * (1 - beta) * V(R.wt, ph) +
                        (1 - alpha) * beta * V(R.w, ph)) / (alpha * beta);
        break;
    case 0:
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k + 1) - nsz));
        lin(R.t, R.tt, h <= zA ? 0.0 : sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k + 2) - nsz)));
        break;
    case 1:
        alpha = (crd(cx, i + 1) - nsx) / (crd(cx, i + 1) - crd(cx, i));
        beta = (crd(cz, k + 1) - nsz) / (crd(cz, k + 1) - crd(cz, k));
        for (int ph = 0; ph <= ns; ++ph)
            vel[ph] = -(alpha * (1 - beta) * V(R.t, ph) + (1 - alpha) * (1 - beta) * V(R.et, ph) +
                        (1 - alpha) * beta * V(R.e, ph)) / (alpha * beta);
        break;
    case 2:
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i + 1) - nsx) + sq(crd(cz, k) - nsz));
        lin(R.e, R.ee, h <= zA ? 0.0 : sqrt(sq(crd(cx, i + 2) - nsx) + sq(crd(cz, k) - nsz)));
        break;
    case 3:
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i + 1) - nsx) + sq(crd(cz, k + 1) - nsz));
        lin(R.et, ippjkpp, h <= zA ? 0.0 : sqrt(sq(crd(cx, i + 2) - nsx) + sq(crd(cz, k + 2) - nsz)));
        break;
    case 22:  // nsx < cx(i), checked at create
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i + 1) - nsx) + sq(crd(cz, k) - nsz));
        for (int ph = 0; ph <= ns; ++ph) vel[ph] = +h / zA * V(R.e, ph);
        break;
    case 21:  // nsx > cx(i), checked at create
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i - 1) - nsx) + sq(crd(cz, k) - nsz));
        for (int ph = 0; ph <= ns; ++ph) vel[ph] = +h / zA * V(R.w, ph);
        break;
    case 20:
        h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k) - nsz));
        zA = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cz, k + 1) - nsz));
        for (int ph = 0; ph <= ns; ++ph) vel[ph] = +h / zA * V(R.t, ph);
        break;
    default:
        for (int ph = 0; ph <= ns; ++ph) vel[ph] = V(c, ph);
        break;
    }
}

// the offset of a 3D forcing point's interpolation neighbour from its type
// (immb.f:937-952, 1101-1116, 1208-1230)
__device__ __forceinline__ void ib_delta3_d(int kind, int &di, int &dj, int &dk) {
    const int DI[9] = {0, -1, -1, 0, 1, 1, 1, 0, -1}, DJ[9] = {0, 0, -1, -1, -1, 0, 1, 1, 1};
    di = dj = dk = 0;
    if (kind == 0 || kind == 20) dk = 1;
    else if (kind >= 1 && kind <= 8) { di = DI[kind]; dj = DJ[kind]; }
    else if (kind >= 21 && kind <= 28) { di = DI[kind - 20]; dj = DJ[kind - 20]; }
}

// velint3d, interp.f:687-781
__device__ void velint3d_d(const Prm &P, const IbDev &B, int a, int f, const double *velg, const double *vels,
                           double *vel) {
    const int *fp = B.fp[a] + (size_t)6 * f;
    const int i = fp[0], j = fp[1], k = fp[2], kind = fp[3], q = fp[4], qq = fp[5];
    const double nsx = B.nsl[a][(size_t)3 * f], nsy = B.nsl[a][(size_t)3 * f + 1], nsz = B.nsl[a][(size_t)3 * f + 2];
    const double *cx = a == 0 ? B.xb : B.x;
    const double *cy = a == 1 ? B.yb : B.y;
    const double *cz = a == 2 ? B.zb : B.z;
    const int n = P.ncell, ns = P.ns;
    auto V = [&](int cell, int ph) { return ph == 0 ? velg[cell] : vels[(size_t)(ph - 1) * n + cell]; };
    auto sq = [](double v) { return v * v; };
    int di, dj, dk;
    ib_delta3_d(kind, di, dj, dk);
    const bool diagonal = (kind % 2 == 0) && kind != 0;
    const double h = sqrt(sq(crd(cx, i) - nsx) + sq(crd(cy, j) - nsy) + sq(crd(cz, k) - nsz));
    const double zA = sqrt(sq(crd(cx, i + di) - nsx) + sq(crd(cy, j + dj) - nsy) + sq(crd(cz, k + dk) - nsz));
    const double hzA = h / zA;
    if (kind >= 20) {
        for (int ph = 0; ph <= ns; ++ph) vel[ph] = hzA * V(q, ph);
    } else if (h <= zA || diagonal) {
        for (int ph = 0; ph <= ns; ++ph) vel[ph] = -hzA * V(q, ph);
    } else {
        const double zB = sqrt(sq(crd(cx, i + 2 * di) - nsx) + sq(crd(cy, j + 2 * dj) - nsy) + sq(crd(cz, k + 2 * dk) - nsz));
        for (int ph = 0; ph <= ns; ++ph) {
            const double v2 = -((zB - h) * V(q, ph) + (h - zA) * V(qq, ph)) / (zB - zA);
            const double v1 = -hzA * V(q, ph);
            vel[ph] = fabs(v1) < fabs(v2) ? v1 : v2;
        }
    }
}

// hn, interp.f:832-919
__device__ void hn_d(const Prm &P, const Fld &F, const IbDev &B, int m, int nn) {
    const int ns = P.ns, ng = P.ng;
    const size_t n = P.ncell;
    auto copy = [&](int dst, int src, double f, bool add) {
        auto put = [&](double *a, size_t d, size_t s_) {
            if (f == 1.0 && !add) a[d] = a[s_];
            else a[d] = add ? a[d] + f * a[s_] : f * a[s_];
        };
        put(F.p, dst, src);
        put(F.ep, dst, src);
        for (int is = 0; is < ns; ++is) put(F.rlk, is * n + dst, is * n + src);
        put(F.rgp, dst, src);
        put(F.tg, dst, src);
        for (int is = 0; is < ns; ++is) put(F.ts, is * n + dst, is * n + src);
        put(F.sieg, dst, src);
        for (int is = 0; is < ns; ++is) put(F.sies, is * n + dst, is * n + src);
        for (int ig = 0; ig < ng; ++ig) put(F.ygc, ig * n + dst, ig * n + src);
    };
    if (P.flag[m] == FILLED1) copy(m, nn, 1.0, false);
    else if (P.flag[nn] == FILLED1) copy(nn, m, 1.0, false);
    if (P.flag[m] == FILLED2) {
        const bool f = B.fc2[m] != 0.0;
        copy(m, nn, 0.5, f);
        B.fc2[m] = f ? 0.0 : 1.0;
    } else if (P.flag[nn] == FILLED2) {
        const bool f = B.fc2[nn] != 0.0;
        copy(nn, m, 0.5, f);
        B.fc2[nn] = f ? 0.0 : 1.0;
    }
}

// the forcing-point branch of the boundary pass for cell c, bdry.f:103-204
template <int D>
__device__ void ib_boundary_cell_d(const Prm &P, const Fld &F, const IbDev &B, int c) {
    double vel[PDAC_MAXP + 1];
    const size_t n = P.ncell;
    const int ns = P.ns;
    for (int a = 0; a < 3; ++a) {
        if (a == 1 && D == 2) continue;
        const int fnum = P.ib_num[a][c];
        if (fnum == 0) continue;
        const int f = fnum - 1;
        double *G = a == 0 ? F.ug : (a == 1 ? F.vg : F.wg);
        double *S = a == 0 ? F.us : (a == 1 ? F.vs : F.ws);
        if (D == 3) velint3d_d(P, B, a, f, G, S, vel);
        else velint2d_d(P, B, a, f, c, G, S, vel);
        for (int ph = 0; ph <= ns; ++ph) B.vel[a][(size_t)f * P.nph + ph] = vel[ph];
        if (B.fp[a][(size_t)6 * f + 3] >= 20) {
            int nb;
            if (D == 3) {
                int i, j, k;
                ijk_of(P, c, i, j, k);
                nb = a == 0 ? at3(P, min(i + 1, P.nx), j, k)
                            : (a == 1 ? at3(P, i, min(j + 1, P.ny), k) : at3(P, i, j, min(k + 1, P.nz)));
            } else {
                const int i = c % P.nx + 1, k = c / P.nx + 1;
                nb = a == 0 ? at2(P, min(i + 1, P.nx), k) : at2(P, i, min(k + 1, P.nz));
            }
            hn_d(P, F, B, c, nb);
        }
        G[c] = vel[0];
        for (int is = 1; is <= ns; ++is) S[(size_t)(is - 1) * n + c] = vel[is];
    }
}

// one level of the ordered boundary pass: items[lo .. hi) are cells whose
// updates are independent of each other
template <int D>
__global__ void k_boundary_items(Prm P, Fld F, IbDev B, const int *items, int lo, int hi) {
    const int t = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= hi) return;
    const int c = items[t];
    const int f0 = P.flag[c];
    if (f0 == IMMB || f0 == FILLED1 || f0 == FILLED2) ib_boundary_cell_d<D>(P, F, B, c);
    else if (D == 3) boundary_cell3d(P, F, c);
    else boundary_cell2d(P, F, c);
}

}  // namespace pdac
