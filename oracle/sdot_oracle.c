/*
 * ORACLE — test infrastructure only.
 *
 * CPU restatement (plain C99 + OpenMP, FP64) of the reference semi-discrete
 * optimal-transport path of rmk523/caustic (Optimal_Transport_rl/).  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load this
 * library, and only as the checker.  The product path (libcausticot.so) never
 * links or calls it.
 *
 * Every function names the reference lines it restates.  The operation order of
 * the per-cell arithmetic (Sutherland-Hodgman clip, fan area, Green integral,
 * pixel loops) follows the reference exactly so that results agree to the last
 * few ulps; only the power-diagram construction differs: the reference calls
 * CGAL 5.5 (Regular_triangulation_2 + Voronoi_diagram_2), which is absent here.
 * The oracle instead takes each cell's regular-triangulation neighbour list
 * (computed by the Python side from the lower convex hull of the lifted sites,
 * i.e. the same triangulation CGAL builds) and intersects the half-planes.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define ORC_API __attribute__((visibility("default")))

/* Work arrays: the reference uses local arrays of max_edge_num = 400 doubles
 * (power_diagram.hpp:39, clip.cuh:95); rings above 200 vertices are rejected by
 * the line search (ot_op.cuh:376).  The oracle uses 1024 doubles so that it
 * never overflows on the cells the reference accepts. */
#define ORC_MAXD 1024

/* ---- clip.cuh:32-91: inside()/intersection() of one rectangle side ------- */
/* square layout: {xmin, ymin, xmax, ymax}; flag 0 bottom, 1 right, 2 top, 3 left */
static inline int orc_inside(const double *p, const double *sq, int flag)
{
    switch (flag) {
    case 0: return p[1] > sq[1];
    case 1: return p[0] < sq[2];
    case 2: return p[1] < sq[3];
    case 3: return p[0] > sq[0];
    }
    return 0;
}

static inline void orc_intersection(const double *s, const double *e, const double *sq, int flag, double *out)
{
    switch (flag) {
    case 0:
        out[0] = (s[0] - e[0]) * (sq[1] - e[1]) / (s[1] - e[1]) + e[0];
        out[1] = sq[1];
        break;
    case 1:
        out[1] = (s[1] - e[1]) * (sq[2] - e[0]) / (s[0] - e[0]) + e[1];
        out[0] = sq[2];
        break;
    case 2:
        out[0] = (s[0] - e[0]) * (sq[3] - e[1]) / (s[1] - e[1]) + e[0];
        out[1] = sq[3];
        break;
    case 3:
        out[1] = (s[1] - e[1]) * (sq[0] - e[0]) / (s[0] - e[0]) + e[1];
        out[0] = sq[0];
        break;
    }
}

/* ---- clip.cuh:93-149: Sutherland-Hodgman against an axis-aligned rectangle --
 * Passes in the order bottom, right, top, left with strict inequalities. */
ORC_API void orc_clip_rect(const double *poly, int n, const double *sq, double *out, int *nout)
{
    double in[ORC_MAXD];
    int len = n;
    memcpy(out, poly, sizeof(double) * 2 * (size_t)n);
    for (int j = 0; j < 4; j++) {
        memcpy(in, out, sizeof(double) * 2 * (size_t)len);
        int c = 0;
        for (int i = 0; i < len; i++) {
            int nx = (i + 1) % len;
            const double *s = in + 2 * i, *e = in + 2 * nx;
            double it[2];
            if (orc_inside(e, sq, j)) {
                if (orc_inside(s, sq, j)) {
                    out[2 * c] = e[0]; out[2 * c + 1] = e[1]; c++;
                } else {
                    orc_intersection(s, e, sq, j, it);
                    out[2 * c] = it[0]; out[2 * c + 1] = it[1]; c++;
                    out[2 * c] = e[0]; out[2 * c + 1] = e[1]; c++;
                }
            } else if (orc_inside(s, sq, j)) {
                orc_intersection(s, e, sq, j, it);
                out[2 * c] = it[0]; out[2 * c + 1] = it[1]; c++;
            }
        }
        len = c;
    }
    *nout = len;
}

/* ---- basic_function.cuh:527-539: fan shoelace area with abs -------------- */
ORC_API double orc_area(const double *p, int n)
{
    double a = 0;
    for (int i = 1; i < n - 1; i++)
        a += 0.5 * ((p[2 * i + 1] - p[1]) * (p[2 * i + 2] - p[0]) - (p[2 * i] - p[0]) * (p[2 * i + 3] - p[1]));
    if (a < 0) a = -a;
    return a;
}

/* ---- basic_function.cuh:826-854: closed-form edge term of ∫|x-s|^2 ------- */
static inline void orc_edge_ints(const double *p1, const double *p2, const double *s, double *acc)
{
    double x2mx1 = p2[0] - p1[0];
    double y1my2 = p1[1] - p2[1];
    double x1px2 = p1[0] + p2[0];
    double y1py2 = p1[1] + p2[1];
    double x12 = p1[0] * p1[0] + p2[0] * p2[0];
    double y12 = p1[1] * p1[1] + p2[1] * p2[1];
    double x12b = x12 + p1[0] * p2[0];
    double y12b = y12 + p1[1] * p2[1];
    double cr = p1[0] * p2[1] - p2[0] * p1[1];
    double x0 = s[0] * s[0];
    double y0 = s[1] * s[1];
    double iq = x2mx1 * y1py2 * y12 / 4. + (cr - 2. * s[1] * x2mx1) * y12b / 3.
              + (y0 * x2mx1 / 2. - s[1] * cr) * y1py2 + y0 * cr;
    double ip = y1my2 * x1px2 * x12 / 4. + (cr - 2. * s[0] * y1my2) * x12b / 3.
              + (x0 * y1my2 / 2. - s[0] * cr) * x1px2 + x0 * cr;
    *acc += iq + ip;
}

/* ---- basic_function.cuh:856-865: Polygon_Ints (closing edge first) -------- */
ORC_API double orc_poly_ints(const double *p, int n, const double *s)
{
    double acc = 0;
    orc_edge_ints(p + (2 * n - 2), p, s, &acc);
    for (int i = 0; i < n - 1; i++) orc_edge_ints(p + 2 * i, p + 2 * i + 2, s, &acc);
    return acc;
}

/* ---- basic_function.cuh:590-608: d_compute_center (fan of triangles) ------ */
ORC_API void orc_poly_center(const double *p, int n, double *c)
{
    c[0] = 0; c[1] = 0;
    double big = orc_area(p, n);
    for (int i = 0; i < n - 2; i++) {
        double tri[6] = {p[0], p[1], p[2 * i + 2], p[2 * i + 3], p[2 * i + 4], p[2 * i + 5]};
        double a = orc_area(tri, 3);
        c[0] += (tri[0] + tri[2] + tri[4]) / 3 * a;
        c[1] += (tri[1] + tri[3] + tri[5]) / 3 * a;
    }
    c[0] /= big;
    c[1] /= big;
}

/* Pixel range of a polygon's bounding box, basic_function.cuh:769-799. */
static void orc_pixel_range(const double *ip, int n, const double *pd, const int *size,
                            double xs, double ys, int *lx, int *ly, int *hx, int *hy)
{
    double mxx = ip[0], mxy = ip[1], mnx = ip[0], mny = ip[1];
    for (int i = 0; i < n; i++) {
        if (ip[2 * i] < mnx) mnx = ip[2 * i];
        if (ip[2 * i] > mxx) mxx = ip[2 * i];
        if (ip[2 * i + 1] < mny) mny = ip[2 * i + 1];
        if (ip[2 * i + 1] > mxy) mxy = ip[2 * i + 1];
    }
    int a = (int)floor((mnx - pd[0]) / xs);
    int b = (int)floor((mny - pd[2]) / ys);
    int c = (int)floor((mxx - pd[0]) / xs) + 1;
    int d = (int)floor((mxy - pd[2]) / ys) + 1;
    *lx = a > 0 ? a : 0;
    *ly = b > 0 ? b : 0;
    *hx = c < size[0] ? c : size[0];
    *hy = d < size[1] ? d : size[1];
}

/*
 * Per-cell mass and objective term: compute_inte (basic_function.cuh:743-824)
 * and compute_f (basic_function.cuh:867-952) evaluated over the same pixel
 * loop.  `picture` is the density after the reference's normalisation
 * (ot_op.cuh:154: picture /= sum(picture)/area_scalar), laid out
 * picture[ix + iy*size[0]].  pd = proj_domain {xmin, xmax, ymin, ymax}.
 * Rings are CSR: cell i = ring[2*start[i] .. 2*(start[i]+len[i])).
 */
ORC_API void orc_eval_cells(int n, const double *ring, const int *start, const int *len,
                            const double *xy, const double *w, const double *nu,
                            const double *picture, const int *size, const double *pd,
                            double *mu, double *f)
{
    const double xs = (pd[1] - pd[0]) / (double)size[0];
    const double ys = (pd[3] - pd[2]) / (double)size[1];
    const double ga = xs * ys;
#pragma omp parallel for schedule(dynamic, 64)
    for (int t = 0; t < n; t++) {
        double ip[ORC_MAXD], np_[ORC_MAXD];
        int inn = 0, nn = 0;
        double m = 0;
        double ft = -w[t] * nu[t];
        if (len[t] != 0) {
            double sq[4] = {pd[0], pd[2], pd[1], pd[3]};
            orc_clip_rect(ring + 2 * (size_t)start[t], len[t], sq, ip, &inn);
            if (inn >= 3) {
                int lx, ly, hx, hy;
                orc_pixel_range(ip, inn, pd, size, xs, ys, &lx, &ly, &hx, &hy);
                for (int ix = lx; ix < hx; ix++) {
                    for (int iy = ly; iy < hy; iy++) {
                        int g = ix + iy * size[0];
                        double cs[4] = {(double)ix * xs + pd[0], (double)iy * ys + pd[2],
                                        (double)(ix + 1) * xs + pd[0], (double)(iy + 1) * ys + pd[2]};
                        orc_clip_rect(ip, inn, cs, np_, &nn);
                        double a = orc_area(np_, nn);
                        m += picture[g] * a / ga;
                        if (a > 0) {
                            double sd = orc_poly_ints(np_, nn, xy + 2 * (size_t)t);
                            ft -= picture[g] / ga * (sd - w[t] * a);
                        }
                    }
                }
            }
        }
        mu[t] = m;
        f[t] = ft;
    }
}

/* compute_clip_area, basic_function.cuh:610-633 (source cell areas for ν).
 * sd = sample_domain {xmin, xmax, ymin, ymax}. */
ORC_API void orc_clip_area(int n, const double *ring, const int *start, const int *len,
                           const double *sd, double *area)
{
#pragma omp parallel for schedule(static)
    for (int t = 0; t < n; t++) {
        if (len[t] > 1) {
            double np_[ORC_MAXD];
            int nn = 0;
            double sq[4] = {sd[0], sd[2], sd[1], sd[3]};
            orc_clip_rect(ring + 2 * (size_t)start[t], len[t], sq, np_, &nn);
            area[t] = orc_area(np_, nn);
        } else {
            area[t] = 0;
        }
    }
}

/* compute_center, basic_function.cuh:1056-1191 (if_weighting selects the
 * density-weighted branch; pieces of area <= 1e-10 are skipped there). */
ORC_API void orc_center(int n, const double *ring, const int *start, const int *len,
                        const double *picture, const int *size, const double *pd,
                        int weighting, double *center, unsigned char *exist)
{
    const double xs = (pd[1] - pd[0]) / (double)size[0];
    const double ys = (pd[3] - pd[2]) / (double)size[1];
#pragma omp parallel for schedule(dynamic, 64)
    for (int t = 0; t < n; t++) {
        double ip[ORC_MAXD], np_[ORC_MAXD];
        int inn = 0, nn = 0;
        if (len[t] == 0) { exist[t] = 0; continue; }
        double sq[4] = {pd[0], pd[2], pd[1], pd[3]};
        const double *poly = ring + 2 * (size_t)start[t];
        orc_clip_rect(poly, len[t], sq, ip, &inn);
        if (!weighting) {
            if (inn >= 3) { orc_poly_center(ip, inn, center + 2 * (size_t)t); exist[t] = 1; }
            else exist[t] = 0;
            continue;
        }
        if (inn < 3) { exist[t] = 0; continue; }
        int lx, ly, hx, hy;
        orc_pixel_range(ip, inn, pd, size, xs, ys, &lx, &ly, &hx, &hy);
        double tot = 0, cx = 0, cy = 0;
        for (int ix = lx; ix < hx; ix++) {
            for (int iy = ly; iy < hy; iy++) {
                int g = ix + iy * size[0];
                double cs[4] = {(double)ix * xs + pd[0], (double)iy * ys + pd[2],
                                (double)(ix + 1) * xs + pd[0], (double)(iy + 1) * ys + pd[2]};
                orc_clip_rect(ip, inn, cs, np_, &nn);
                double a = orc_area(np_, nn);
                if (a > 1e-10) {
                    double lc[2];
                    orc_poly_center(np_, nn, lc);
                    double contrib = picture[g] * a;
                    tot += contrib;
                    cx += lc[0] * contrib;
                    cy += lc[1] * contrib;
                }
            }
        }
        if (tot != 0) {
            center[2 * t] = cx / tot;
            center[2 * t + 1] = cy / tot;
        } else {
            orc_poly_center(ip, inn, center + 2 * (size_t)t);
        }
        exist[t] = 1;
    }
}

/* render (basic_function.cuh:660-741): splat ν_i·area(cell∩pix)/area(cell)
 * into the pixel grid.  Serial accumulation keeps the oracle deterministic. */
ORC_API void orc_render(int n, const double *ring, const int *start, const int *len,
                        const double *carry, const int *size, const double *pd, double *out)
{
    const double xs = (pd[1] - pd[0]) / (double)size[0];
    const double ys = (pd[3] - pd[2]) / (double)size[1];
    for (int t = 0; t < n; t++) {
        double ip[ORC_MAXD], np_[ORC_MAXD];
        int inn = 0, nn = 0;
        if (len[t] == 0) continue;
        double sq[4] = {pd[0], pd[2], pd[1], pd[3]};
        orc_clip_rect(ring + 2 * (size_t)start[t], len[t], sq, ip, &inn);
        double big = orc_area(ip, inn);
        if (inn < 3) continue;
        int lx, ly, hx, hy;
        orc_pixel_range(ip, inn, pd, size, xs, ys, &lx, &ly, &hx, &hy);
        for (int ix = lx; ix < hx; ix++)
            for (int iy = ly; iy < hy; iy++) {
                double cs[4] = {(double)ix * xs + pd[0], (double)iy * ys + pd[2],
                                (double)(ix + 1) * xs + pd[0], (double)(iy + 1) * ys + pd[2]};
                orc_clip_rect(ip, inn, cs, np_, &nn);
                double a = orc_area(np_, nn);
                if (big != 0) out[ix + iy * size[0]] += carry[t] * a / big;
            }
    }
}

/* ------------------------------------------------------------------------
 * Power cells from neighbour lists.
 *
 * The reference's polygons_in_VD (power_diagram.cpp:8-134) walks each CGAL
 * Voronoi face.  Here each cell starts as the box rectangle (CCW) and is
 * intersected with the half-planes
 *     |x - s_i|^2 - w_i <= |x - s_j|^2 - w_j
 * for every listed neighbour j.  Each output edge carries the index of the
 * generator that produced it (-1..-4 for the box sides bottom, right, top,
 * left), so adjacency can be read off the ring.  After the topology is fixed,
 * every vertex is recomputed as the intersection of its two generator lines,
 * which is how CGAL constructs Voronoi vertices (circumcentres of the
 * triangulation's faces) rather than by repeated segment clipping.
 * box = {xmin, xmax, ymin, ymax}.
 * ------------------------------------------------------------------------ */

typedef struct { double a, b, c; } orc_line; /* a x + b y <= c */

/* Half-plane of generator j for cell i in coordinates translated to s_i
 * (x' = x - s_i), the way CGAL's weighted-circumcentre constructions work on
 * differences to one of the points:  2 e.x' <= |e|^2 - (w_j - w_i),
 * e = s_j - s_i.  Box sides use the translated box. */
static orc_line orc_gen_line(int i, int j, const double *xy, const double *w, const double *box)
{
    orc_line L;
    double xi = xy[2 * i], yi = xy[2 * i + 1];
    if (j >= 0) {
        double ex = xy[2 * j] - xi, ey = xy[2 * j + 1] - yi;
        L.a = 2.0 * ex;
        L.b = 2.0 * ey;
        L.c = (ex * ex + ey * ey) - (w[j] - w[i]);
    } else {
        switch (j) {
        case -1: L.a = 0; L.b = -1; L.c = -(box[2] - yi); break; /* y >= ymin */
        case -2: L.a = 1; L.b = 0; L.c = box[1] - xi; break;     /* x <= xmax */
        case -3: L.a = 0; L.b = 1; L.c = box[3] - yi; break;     /* y <= ymax */
        default: L.a = -1; L.b = 0; L.c = -(box[0] - xi); break; /* x >= xmin */
        }
    }
    return L;
}

/* Power difference side test in the difference form used for the predicate:
 * value > 0 means v lies strictly on j's side. */
static inline double orc_side(const orc_line *L, double x, double y)
{
    return L->a * x + L->b * y - L->c;
}

/* Returns the number of vertices written for cell i (<= cap), or -1 when the
 * ring would exceed cap.  out_xy: 2*cap doubles, out_lab: cap ints (label of
 * the edge from vertex k to k+1). */
static int orc_one_cell(int i, const int *nbr, int nn, const double *xy, const double *w,
                        const double *box, int cap, double *out_xy, int *out_lab)
{
    double px[2][ORC_MAXD / 2], py[2][ORC_MAXD / 2];
    int lab[2][ORC_MAXD / 2];
    int cur = 0, nv = 4;
    int vcap = ORC_MAXD / 2;
    const double xi = xy[2 * i], yi = xy[2 * i + 1];
    px[0][0] = box[0] - xi; py[0][0] = box[2] - yi; lab[0][0] = -1;
    px[0][1] = box[1] - xi; py[0][1] = box[2] - yi; lab[0][1] = -2;
    px[0][2] = box[1] - xi; py[0][2] = box[3] - yi; lab[0][2] = -3;
    px[0][3] = box[0] - xi; py[0][3] = box[3] - yi; lab[0][3] = -4;
    for (int k = 0; k < nn && nv > 0; k++) {
        int j = nbr[k];
        if (j == i) continue;
        orc_line L = orc_gen_line(i, j, xy, w, box);
        double d[ORC_MAXD / 2];
        int any_out = 0, any_in = 0;
        for (int v = 0; v < nv; v++) {
            d[v] = orc_side(&L, px[cur][v], py[cur][v]);
            if (d[v] > 0) any_out = 1; else any_in = 1;
        }
        if (!any_out) continue;
        if (!any_in) { nv = 0; break; }
        int nx = 1 - cur, c = 0;
        for (int v = 0; v < nv; v++) {
            int u = (v + 1) % nv;
            int in_v = d[v] <= 0, in_u = d[u] <= 0;
            if (in_v) {
                if (c >= vcap) return -1;
                px[nx][c] = px[cur][v]; py[nx][c] = py[cur][v];
                lab[nx][c] = in_u ? lab[cur][v] : lab[cur][v];
                c++;
            }
            if (in_v != in_u) {
                double t = d[v] / (d[v] - d[u]);
                if (c >= vcap) return -1;
                px[nx][c] = px[cur][v] + t * (px[cur][u] - px[cur][v]);
                py[nx][c] = py[cur][v] + t * (py[cur][u] - py[cur][v]);
                /* leaving: the new edge runs along j's line; entering: the
                 * remaining part of edge v->u keeps its old label */
                lab[nx][c] = in_v ? j : lab[cur][v];
                c++;
            }
        }
        cur = nx;
        nv = c;
    }
    if (nv > cap) return -1;
    /* recompute each vertex from its two generator lines */
    for (int v = 0; v < nv; v++) {
        int pv = (v + nv - 1) % nv;
        orc_line A = orc_gen_line(i, lab[cur][pv], xy, w, box);
        orc_line B = orc_gen_line(i, lab[cur][v], xy, w, box);
        double det = A.a * B.b - A.b * B.a;
        double x = px[cur][v], y = py[cur][v];
        if (det != 0) {
            double xx = (A.c * B.b - A.b * B.c) / det;
            double yy = (A.a * B.c - A.c * B.a) / det;
            if (isfinite(xx) && isfinite(yy)) { x = xx; y = yy; }
        }
        out_xy[2 * v] = xi + x;
        out_xy[2 * v + 1] = yi + y;
        out_lab[v] = lab[cur][v];
    }
    return nv;
}

/* Build all cells.  nbr CSR: nbr[nbr_start[i] .. nbr_start[i+1]).  Writes
 * ring_len[i] (0 for hidden or empty cells, -1 on overflow of cap), ring_xy
 * [2*cap*i ...], ring_lab[cap*i ...] in a fixed-stride layout. */
ORC_API void orc_cells(int n, const double *xy, const double *w, const int *nbr_start, const int *nbr,
                       const double *box, int cap, int *ring_len, double *ring_xy, int *ring_lab)
{
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        ring_len[i] = orc_one_cell(i, nbr + nbr_start[i], nbr_start[i + 1] - nbr_start[i], xy, w, box, cap,
                                   ring_xy + 2 * (size_t)cap * i, ring_lab + (size_t)cap * i);
    }
}

/* Brute-force cross-check for small n: every other site is a neighbour
 * candidate.  O(n^2); used only by tests. */
ORC_API void orc_cells_brute(int n, const double *xy, const double *w, const double *box, int cap,
                             int *ring_len, double *ring_xy, int *ring_lab)
{
#pragma omp parallel
    {
        int *all = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < n; i++) {
            /* nearest first keeps intermediate rings small */
            int c = 0;
            for (int j = 0; j < n; j++) all[c++] = j;
            ring_len[i] = orc_one_cell(i, all, c, xy, w, box, cap, ring_xy + 2 * (size_t)cap * i,
                                       ring_lab + (size_t)cap * i);
        }
        free(all);
    }
}

/*
 * Hessian of the masses (no counterpart in the reference, whose solvers use
 * first derivatives only): for every ring edge k of cell i whose generator is
 * a site j (lab >= 0),
 *     a_k = (integral of rho along the edge) / (2 |s_i - s_j|) = -dmu_i/dw_j,
 * and dmu_i/dw_i = sum_k a_k.  This is the classical derivative of a Laguerre
 * cell's mass (Kitagawa, Merigot and Thibert, "Convergence of a Newton
 * algorithm for semi-discrete optimal transport", J. Eur. Math. Soc. 2019,
 * Thm 1.3): moving w_i by dw moves the edge towards j by dw / (2|s_i - s_j|).
 * rho is the normalised picture per unit area (picture / pixel area); the
 * edge is cut at every pixel line it crosses and each piece weighs the pixel
 * that holds its midpoint.  Rings are fixed-stride (cap vertices per cell);
 * out has the same layout (0 for domain sides and past the ring's end).
 */
static int orc_cmp_d(const void *a, const void *b)
{
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

static double orc_segment_rho(const double *P, const double *Q, const double *picture, const int *size,
                              const double *pd, double xs, double ys)
{
    enum { TMAX = 16384 };
    double ts[TMAX];
    int nt = 0;
    const double dx = Q[0] - P[0], dy = Q[1] - P[1];
    const double len = sqrt(dx * dx + dy * dy);
    if (!(len > 0)) return 0.0;
    ts[nt++] = 0.0;
    ts[nt++] = 1.0;
    if (dx != 0.0) {
        double a = (fmin(P[0], Q[0]) - pd[0]) / xs, b = (fmax(P[0], Q[0]) - pd[0]) / xs;
        int c0 = (int)floor(a) + 1, c1 = (int)ceil(b) - 1;
        if (c0 < 0) c0 = 0;
        if (c1 > size[0]) c1 = size[0];
        for (int c = c0; c <= c1; c++) {
            if (nt >= TMAX) return NAN;  /* more crossings than the buffer holds: fail loudly */
            double t = (pd[0] + c * xs - P[0]) / dx;
            if (t > 0.0 && t < 1.0) ts[nt++] = t;
        }
    }
    if (dy != 0.0) {
        double a = (fmin(P[1], Q[1]) - pd[2]) / ys, b = (fmax(P[1], Q[1]) - pd[2]) / ys;
        int r0 = (int)floor(a) + 1, r1 = (int)ceil(b) - 1;
        if (r0 < 0) r0 = 0;
        if (r1 > size[1]) r1 = size[1];
        for (int r = r0; r <= r1; r++) {
            if (nt >= TMAX) return NAN;
            double t = (pd[2] + r * ys - P[1]) / dy;
            if (t > 0.0 && t < 1.0) ts[nt++] = t;
        }
    }
    qsort(ts, nt, sizeof(double), orc_cmp_d);
    const double ga = xs * ys;
    double acc = 0.0;
    for (int k = 0; k + 1 < nt; k++) {
        const double dt = ts[k + 1] - ts[k];
        if (!(dt > 0)) continue;
        const double tm = 0.5 * (ts[k] + ts[k + 1]);
        const double mx = P[0] + tm * dx, my = P[1] + tm * dy;
        const int ix = (int)floor((mx - pd[0]) / xs), iy = (int)floor((my - pd[2]) / ys);
        if (ix < 0 || iy < 0 || ix >= size[0] || iy >= size[1]) continue;
        acc += picture[ix + (size_t)iy * size[0]] / ga * dt;
    }
    return acc * len;
}

ORC_API void orc_edge_weights(int n, int cap, const double *ring, const int *len, const int *lab, const double *xy,
                              const double *picture, const int *size, const double *pd, double *out)
{
    const double xs = (pd[1] - pd[0]) / (double)size[0];
    const double ys = (pd[3] - pd[2]) / (double)size[1];
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        const double *R = ring + 2 * (size_t)i * cap;
        double *o = out + (size_t)i * cap;
        for (int k = 0; k < cap; k++) o[k] = 0.0;
        const int m = len[i];
        for (int k = 0; k < m; k++) {
            const int j = lab[(size_t)i * cap + k];
            if (j < 0) continue;
            const double *P = R + 2 * k, *Q = R + 2 * ((k + 1) % m);
            const double ex = xy[2 * j] - xy[2 * i], ey = xy[2 * j + 1] - xy[2 * i + 1];
            o[k] = orc_segment_rho(P, Q, picture, size, pd, xs, ys) / (2.0 * sqrt(ex * ex + ey * ey));
        }
    }
}
