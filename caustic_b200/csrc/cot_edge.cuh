// Density line integral along one power-cell edge (used by the Newton
// solver's mass Jacobian; no counterpart in the reference, whose solvers use
// first derivatives only).
//
// Moving w_i by dw moves the edge between cells i and j towards j by
// dw / (2 |s_i - s_j|), so dmu_i/dw_j = -(integral of rho along the edge) /
// (2 |s_i - s_j|) and dmu_i/dw_i is minus the sum over the edges (Kitagawa,
// Merigot and Thibert, "Convergence of a Newton algorithm for semi-discrete
// optimal transport", J. Eur. Math. Soc. 2019, Thm 1.3).
#pragma once
#include "cot_common.cuh"

namespace cot {

// Integral of the piecewise-constant density along the segment A -> B
// (absolute coordinates inside proj_domain): the segment is cut at every
// pixel line it crosses, in parameter order, and each piece weighs the pixel
// that holds its midpoint.  The loop is bounded by the number of lines the
// segment can cross.
__device__ __forceinline__ double edge_rho_integral(const CotGeo &g, double ax, double ay, double bx, double by)
{
    const double dx = bx - ax, dy = by - ay;
    const double len = sqrt(dx * dx + dy * dy);
    if (!(len > 0.0)) return 0.0;
    // pixel units
    const double u0 = (ax - g.pd[0]) * g.ixs, v0 = (ay - g.pd[2]) * g.iys;
    const double du = dx * g.ixs, dv = dy * g.iys;
    const double u1 = u0 + du, v1 = v0 + dv;
    const int su = du > 0.0 ? 1 : -1, sv = dv > 0.0 ? 1 : -1;
    // the first line index ahead of the start in each direction
    int cu = du > 0.0 ? (int)floor(u0) + 1 : (int)ceil(u0) - 1;
    int cv = dv > 0.0 ? (int)floor(v0) + 1 : (int)ceil(v0) - 1;
    const double idu = du != 0.0 ? 1.0 / du : 0.0, idv = dv != 0.0 ? 1.0 / dv : 0.0;
    const int bound = (int)(fabs(floor(u1) - floor(u0)) + fabs(floor(v1) - floor(v0))) + 8;
    double t = 0.0, acc = 0.0;
    for (int it = 0; it < bound && t < 1.0; it++) {
        const double tu = du != 0.0 ? ((double)cu - u0) * idu : 2.0;
        const double tv = dv != 0.0 ? ((double)cv - v0) * idv : 2.0;
        const double tn = fmin(fmin(tu, tv), 1.0);
        if (tn > t) {
            const double tm = 0.5 * (t + tn);
            int ix = (int)floor(u0 + tm * du), iy = (int)floor(v0 + tm * dv);
            ix = min(max(ix, 0), g.nx - 1);
            iy = min(max(iy, 0), g.ny - 1);
            acc += g.rho[ix + (size_t)iy * g.nx] * (tn - t);
            t = tn;
        }
        if (tu <= tn) cu += su;
        if (tv <= tn) cv += sv;
    }
    return acc * len;
}

}  // namespace cot
