// sink.cuh -- the particle sink at the ground (sink.f:22-121, isink > 0).
//
// boundary (bdry.f:73, 603-645) clears the sink and, for every fluid cell
// whose bottom neighbour is a wall or a filled cell, calls sink_update per
// solid: inside the ring rprox < r < rdist around (center_x, center_y) the
// cell takes out its downward particle flux rlk min(0, ws) / dz
// (interp.f:811), and the mass taken out over the step accumulates per
// ground column i (2D) or (i, j) (3D) in massl; a restart's column values
// (mass_loss) are added back at the column's first update.  The cells that
// update a column are visited in increasing k as the reference's cell loop
// does, by one thread per (column, solid); the ring test of each column is
// evaluated on the host from the reference's cell-centre coordinates.
#pragma once
#include "kernels3d.cuh"

namespace pdac {

struct Sink {
    double *massl, *mass_loss;  // (ntr, ns) column-major, ntr = nx (2D) or nx ny (3D)
    const int *ring;            // ntr: 1 when the column's centre lies inside the ring
    int ntr;
};

// runs after the boundary kernel: the only writes of boundary to a fluid
// cell's ws come from that cell's own earlier checks (bdry.f order: east,
// west, north, south, top, bottom), so the values seen here are those the
// reference's sink_update reads
template <int D>
__global__ void k_sink(Prm P, Fld F, Sink S, double dt) {
    unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (unsigned)S.ntr * (unsigned)P.ns) return;
    const int is = (int)(t / (unsigned)S.ntr) + 1, b = (int)(t % (unsigned)S.ntr);
    const int i = b % P.nx + 1, j = D == 3 ? b / P.nx + 1 : 1;
    const size_t n = P.ncell, off = (size_t)(is - 1) * n, sb = (size_t)(is - 1) * S.ntr + b;
    const int plane = P.nx * P.ny;
    const bool ring = S.ring[b] != 0;
    double massl = S.massl[sb];
    bool touched = false;
    for (int k = 1; k <= P.nz; ++k) {
        const int c = (i - 1) + P.nx * ((j - 1) + P.ny * (k - 1));
        const int f0 = P.flag[c];
        double sink = 0.0;
        if (k > 1 && (f0 == FLUID || f0 == DOME || f0 == BL_CELL)) {
            const int f2 = P.flag[c - plane];
            if (f2 == SLIP || f2 == NOSLIP || f2 == FILLED1 || f2 == FILLED2) {
                if (ring) {
                    const double ws = F.ws[off + c];
                    const double wst = ws < 0.0 ? ws : 0.0;  // MIN(0, ws)
                    sink = F.rlk[off + c] * wst * P.indz[k];
                }
                if (D == 3) massl = massl + sink * P.dx[i] * P.dy[j] * P.dz[k] * dt;
                else massl = massl + sink * P.dx[i] * P.dz[k] * dt;
                if (!touched) {
                    massl = S.mass_loss[sb] + massl;
                    touched = true;
                } else {
                    massl = 0.0 + massl;  // mass_loss was cleared at the first update
                }
            }
        }
        F.sink[off + c] = sink;
    }
    S.massl[sb] = massl;
    if (touched) S.mass_loss[sb] = 0.0;
}

}  // namespace pdac
