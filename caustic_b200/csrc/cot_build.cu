// Problem set-up on the device (cot_set_problem): the checks and sums of the
// inputs, the bucket grid's counting sort, the static bound tree and the
// density scaling.  The host only reads a few scalars (the sites' box and the
// sums) to size the bucket grid; every array stays on the device.
//
// The reference reads its inputs on the host and normalises the picture there
// (main.cu:130-198, ot_op.cuh:81-88,154); here the same normalisation (the
// density scaled so that it sums to sum(nu), the reference's area_scalar, per
// unit pixel area) is one elementwise kernel after a fixed-order sum.
#include "cot_common.cuh"

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>

namespace cot {

#define BLD_THREADS 256
#define BLD_BLOCKS 296  // two per SM of a B200; the sums are fixed-order for any count

struct SiteStats {
    double xmin, xmax, ymin, ymax, nusum;
    long long bad_xy, bad_nu;  // smallest index of a non-finite site / non-positive mass (-1: none)
};
struct DensStats {
    double sum;
    long long bad;  // smallest index of a negative or non-finite pixel (-1: none)
};

__device__ __forceinline__ long long lmin_idx(long long a, long long b)
{
    if (a < 0) return b;
    if (b < 0) return a;
    return a < b ? a : b;
}

template <class T>
__device__ __forceinline__ T shfl_down_any(T v, int o)
{
    return __shfl_down_sync(0xffffffffu, v, o);
}

// Sites: box, sum of the masses (block-contiguous ranges, warps then blocks
// in order: the same sum for any scheduling), first bad entries.
__global__ void __launch_bounds__(BLD_THREADS) k_site_stats(int n, const double *__restrict__ xy,
                                                           const double *__restrict__ nu, double *partials,
                                                           unsigned int *ticket, SiteStats *out)
{
    __shared__ double sh[5][BLD_THREADS / 32];
    __shared__ long long shb[2][BLD_THREADS / 32];
    __shared__ bool last;
    const int per = (n + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY, s = 0.0;
    long long bxy = -1, bnu = -1;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double x = xy[2 * (size_t)i], y = xy[2 * (size_t)i + 1], m = nu[i];
        if (isfinite(x) && isfinite(y)) {
            x0 = fmin(x0, x);
            x1 = fmax(x1, x);
            y0 = fmin(y0, y);
            y1 = fmax(y1, y);
        } else if (bxy < 0) {
            bxy = i;
        }
        if (!(m > 0.0) || !isfinite(m)) {
            if (bnu < 0) bnu = i;
        } else {
            s += m;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fmin(x0, shfl_down_any(x0, o));
        x1 = fmax(x1, shfl_down_any(x1, o));
        y0 = fmin(y0, shfl_down_any(y0, o));
        y1 = fmax(y1, shfl_down_any(y1, o));
        s += shfl_down_any(s, o);
        bxy = lmin_idx(bxy, shfl_down_any(bxy, o));
        bnu = lmin_idx(bnu, shfl_down_any(bnu, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = x0;
        sh[1][wid] = x1;
        sh[2][wid] = y0;
        sh[3][wid] = y1;
        sh[4][wid] = s;
        shb[0][wid] = bxy;
        shb[1][wid] = bnu;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[5] = {INFINITY, -INFINITY, INFINITY, -INFINITY, 0.0};
        long long q[2] = {-1, -1};
        for (int k = 0; k < BLD_THREADS / 32; k++) {
            r[0] = fmin(r[0], sh[0][k]);
            r[1] = fmax(r[1], sh[1][k]);
            r[2] = fmin(r[2], sh[2][k]);
            r[3] = fmax(r[3], sh[3][k]);
            r[4] += sh[4][k];
            q[0] = lmin_idx(q[0], shb[0][k]);
            q[1] = lmin_idx(q[1], shb[1][k]);
        }
        double *p = partials + 7 * (size_t)blockIdx.x;
        for (int k = 0; k < 5; k++) p[k] = r[k];
        p[5] = (double)q[0];
        p[6] = (double)q[1];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    SiteStats o{INFINITY, -INFINITY, INFINITY, -INFINITY, 0.0, -1, -1};
    for (unsigned b = 0; b < gridDim.x; b++) {
        const double *p = partials + 7 * (size_t)b;
        o.xmin = fmin(o.xmin, __ldcg(p + 0));
        o.xmax = fmax(o.xmax, __ldcg(p + 1));
        o.ymin = fmin(o.ymin, __ldcg(p + 2));
        o.ymax = fmax(o.ymax, __ldcg(p + 3));
        o.nusum += __ldcg(p + 4);
        o.bad_xy = lmin_idx(o.bad_xy, (long long)__ldcg(p + 5));
        o.bad_nu = lmin_idx(o.bad_nu, (long long)__ldcg(p + 6));
    }
    *out = o;
    *ticket = 0u;
}

__global__ void __launch_bounds__(BLD_THREADS) k_dens_stats(long long npix, const double *__restrict__ d,
                                                           double *partials, unsigned int *ticket, DensStats *out)
{
    __shared__ double sh[BLD_THREADS / 32];
    __shared__ long long shb[BLD_THREADS / 32];
    __shared__ bool last;
    const long long per = (npix + gridDim.x - 1) / gridDim.x;
    const long long b0 = blockIdx.x * per, b1 = min(npix, b0 + per);
    double s = 0.0;
    long long bad = -1;
    for (long long p = b0 + threadIdx.x; p < b1; p += blockDim.x) {
        const double v = d[p];
        if (!(v >= 0.0) || !isfinite(v)) {
            if (bad < 0) bad = p;
        } else {
            s += v;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += shfl_down_any(s, o);
        bad = lmin_idx(bad, shfl_down_any(bad, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[wid] = s;
        shb[wid] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        long long q = -1;
        for (int k = 0; k < BLD_THREADS / 32; k++) {
            r += sh[k];
            q = lmin_idx(q, shb[k]);
        }
        partials[2 * (size_t)blockIdx.x] = r;
        partials[2 * (size_t)blockIdx.x + 1] = (double)q;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    DensStats o{0.0, -1};
    for (unsigned b = 0; b < gridDim.x; b++) {
        o.sum += __ldcg(partials + 2 * (size_t)b);
        o.bad = lmin_idx(o.bad, (long long)__ldcg(partials + 2 * (size_t)b + 1));
    }
    *out = o;
    *ticket = 0u;
}

// The bucket of every site (key) and its caller index (value) for the sort.
__global__ void k_bucket_keys(int n, const double *__restrict__ xy, double ox, double oy, double ihx, double ihy,
                              int bx, int by, int *__restrict__ keys, int *__restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int u = (int)((xy[2 * (size_t)i] - ox) * ihx), v = (int)((xy[2 * (size_t)i + 1] - oy) * ihy);
    u = min(max(u, 0), bx - 1);
    v = min(max(v, 0), by - 1);
    keys[i] = u + v * bx;
    idx[i] = i;
}

// Sites and masses in bucket order.
__global__ void k_gather_sites(int n, const int *__restrict__ perm, const int *__restrict__ sb_in,
                               const double *__restrict__ xy, const double *__restrict__ nu, double2 *__restrict__ sxy,
                               double *__restrict__ snu, int *__restrict__ sbucket, int *__restrict__ perm_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int i = perm[p];
    sxy[p] = make_double2(xy[2 * (size_t)i], xy[2 * (size_t)i + 1]);
    snu[p] = nu[i];
    sbucket[p] = sb_in[p];
    perm_out[p] = i;
}

// bstart[b] = first sorted site of bucket b (n for the end), from the sorted
// keys: position p opens every bucket after the previous site's up to its own.
__global__ void k_bstart(int n, int nb, const int *__restrict__ key, int *__restrict__ bstart)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > n) return;
    const int kp = p < n ? key[p] : nb;
    const int kq = p == 0 ? -1 : key[p - 1];
    for (int b = kq + 1; b <= kp; b++) bstart[b] = p;
}

// The box of a node's sites, widened by a relative 1e-12 and an absolute
// 1e-15 L (an empty node: half width -1).  Explicit roundings: no
// contraction, so the same bits as any other build of the same numbers.
__device__ __forceinline__ double4 boxed(double x0, double x1, double y0, double y1, double L)
{
    const double hx = __dadd_rn(__dmul_rn(__dmul_rn(0.5, __dsub_rn(x1, x0)), 1.0 + 1e-12), __dmul_rn(1e-15, L));
    const double hy = __dadd_rn(__dmul_rn(__dmul_rn(0.5, __dsub_rn(y1, y0)), 1.0 + 1e-12), __dmul_rn(1e-15, L));
    return make_double4(__dmul_rn(0.5, __dadd_rn(x0, x1)), __dmul_rn(0.5, __dadd_rn(y0, y1)), hx, hy);
}

// Level 0 of the bound tree: one warp per bucket.
__global__ void k_tree_leaves(int nb, const int *__restrict__ bstart, const double2 *__restrict__ sxy, double L,
                              double4 *__restrict__ tstat)
{
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nb) return;
    const int s0 = bstart[b], s1 = bstart[b + 1];
    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    for (int p = s0 + lane; p < s1; p += 32) {
        const double2 v = sxy[p];
        x0 = fmin(x0, v.x);
        x1 = fmax(x1, v.x);
        y0 = fmin(y0, v.y);
        y1 = fmax(y1, v.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
        x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o));
        x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
        y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o));
        y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) tstat[b] = s1 > s0 ? boxed(x0, x1, y0, y1, L) : make_double4(0.0, 0.0, -1.0, -1.0);
}

// Level l > 0: each node from its (up to) 2 x 2 children.
__global__ void k_tree_level(int off, int w, int h, int coff, int cw, int ch, double L, double4 *__restrict__ tstat)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= w * h) return;
    const int u = q % w, v = q / w;
    double x0 = INFINITY, x1 = -INFINITY, y0 = INFINITY, y1 = -INFINITY;
    for (int bb = 0; bb < 2; bb++)
        for (int aa = 0; aa < 2; aa++) {
            const int uu = 2 * u + aa, vv = 2 * v + bb;
            if (uu >= cw || vv >= ch) continue;
            const double4 c = tstat[coff + uu + vv * cw];
            if (c.z < 0.0) continue;
            x0 = fmin(x0, __dsub_rn(c.x, c.z));
            x1 = fmax(x1, __dadd_rn(c.x, c.z));
            y0 = fmin(y0, __dsub_rn(c.y, c.w));
            y1 = fmax(y1, __dadd_rn(c.y, c.w));
        }
    tstat[off + q] = x1 >= x0 ? boxed(x0, x1, y0, y1, L) : make_double4(0.0, 0.0, -1.0, -1.0);
}

// rho = (density / gray) / pixel area, in place (IEEE division: the same bits
// as the host's).
__global__ void k_density_scale(long long npix, const double *__restrict__ in, double gray, double ga,
                                double *__restrict__ rho)
{
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p < npix) rho[p] = __ddiv_rn(__ddiv_rn(in[p], gray), ga);
}

cudaError_t build_stats(int n, const double *xy, const double *nu, long long npix, const double *dens,
                        double *partials, unsigned int *ticket, void *site_out, void *dens_out, cudaStream_t s)
{
    const int bs = std::max(1, std::min(BLD_BLOCKS, (n + BLD_THREADS - 1) / BLD_THREADS));
    k_site_stats<<<bs, BLD_THREADS, 0, s>>>(n, xy, nu, partials, ticket, (SiteStats *)site_out);
    const int bd = (int)std::max<long long>(1, std::min<long long>(BLD_BLOCKS, (npix + BLD_THREADS - 1) / BLD_THREADS));
    k_dens_stats<<<bd, BLD_THREADS, 0, s>>>(npix, dens, partials + 7 * BLD_BLOCKS, ticket + 1, (DensStats *)dens_out);
    return cudaGetLastError();
}

size_t build_partials_doubles() { return 9 * BLD_BLOCKS; }

cudaError_t build_sort(int n, const double *xy, const double *nu, double ox, double oy, double ihx, double ihy,
                       int bx, int by, int *keys, int *idx, int *keys2, int *idx2, void *temp, size_t *temp_bytes,
                       double2 *sxy, double *snu, int *sbucket, int *perm, int *bstart, cudaStream_t s)
{
    const int nb = bx * by;
    int bits = 1;
    while (bits < 31 && (1 << bits) < nb) bits++;
    if (temp == nullptr) {
        // size query
        return cub::DeviceRadixSort::SortPairs(nullptr, *temp_bytes, keys, keys2, idx, idx2, n, 0, bits, s);
    }
    k_bucket_keys<<<(n + 255) / 256, 256, 0, s>>>(n, xy, ox, oy, ihx, ihy, bx, by, keys, idx);
    cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, *temp_bytes, keys, keys2, idx, idx2, n, 0, bits, s);
    if (e != cudaSuccess) return e;
    k_gather_sites<<<(n + 255) / 256, 256, 0, s>>>(n, idx2, keys2, xy, nu, sxy, snu, sbucket, perm);
    k_bstart<<<(n + 256) / 256, 256, 0, s>>>(n, nb, keys2, bstart);
    return cudaGetLastError();
}

cudaError_t build_tree(int nb, const int *bstart, const double2 *sxy, double L, int nlev, const int *off,
                       const int *lw, const int *lh, double4 *tstat, cudaStream_t s)
{
    k_tree_leaves<<<(nb + 7) / 8, 256, 0, s>>>(nb, bstart, sxy, L, tstat);
    for (int l = 1; l < nlev; l++) {
        const int cnt = lw[l] * lh[l];
        k_tree_level<<<(cnt + 255) / 256, 256, 0, s>>>(off[l], lw[l], lh[l], off[l - 1], lw[l - 1], lh[l - 1], L,
                                                       tstat);
    }
    return cudaGetLastError();
}

cudaError_t build_density(long long npix, const double *in, double gray, double ga, double *rho, cudaStream_t s)
{
    k_density_scale<<<(unsigned)((npix + 255) / 256), 256, 0, s>>>(npix, in, gray, ga, rho);
    return cudaGetLastError();
}

}  // namespace cot
