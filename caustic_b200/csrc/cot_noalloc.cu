// Allocation-free evaluation summary (cot_eval_summary_noalloc).
//
// Some callers cannot call cudaMalloc at the point where they need the
// solver's convergence numbers: code that is recording a CUDA stream capture
// (a cudaMalloc there invalidates the capture), hosts that hand the library a
// fixed memory budget and forbid allocations after start-up (plugins in
// larger applications, real-time loops where an allocation's latency and
// implicit synchronisation are not acceptable).  For them this entry point
// reduces per-cell results the caller already holds on the device (masses,
// objective terms, target masses) to the objective and the mass-error
// statistics without allocating anything: the per-block partial sums and the
// last-block ticket live in a file-scope device array of fixed size.
//
// Limits and sharing:
//  - n <= COT_NOALLOC_MAX_N (one block per COT_NOALLOC_BLOCK_ELEMS cells,
//    at most COT_NOALLOC_MAX_BLOCKS blocks); larger n is rejected;
//  - the scratch array (COT_NOALLOC_MAX_BLOCKS x 4 doubles + a counter,
//    about 32 KB) exists once on every device that loads the library and
//    stays there until the process exits;
//  - every call on a device uses the same array and leaves its contents
//    behind; the counter is cleared at the start of each call, the partial
//    sums are overwritten; two calls that overlap on the GPU (different
//    streams, no ordering between them) race on the array and give wrong
//    results -- order them on one stream or with events;
//  - the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, once per device, with that device current);
//    make that first call before any stream capture starts.
#include "../../include/causticot.h"
#include "cot_common.cuh"

#include <math.h>
#include <mutex>

#define COT_NOALLOC_THREADS 256

namespace cot {
int fail(cot_handle *h, int code, const char *what, const char *detail);
}

struct NoallocScratch {
    double partials[COT_NOALLOC_MAX_BLOCKS * 4];
    unsigned int ticket;
};

// The only scratch of the entry point.  In host code this name is a host-side
// stand-in, not a device address: kernels receive the address obtained from
// cudaGetSymbolAddress.
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

namespace {

std::mutex g_noalloc_mu;
NoallocScratch *g_noalloc_ptr[COT_NOALLOC_MAX_DEVICES] = {};

__device__ __forceinline__ double nsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double nmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block b reduces cells [b*E, (b+1)*E); the last block to finish sums the
// partials in block order, so the result does not depend on scheduling.
__global__ void __launch_bounds__(COT_NOALLOC_THREADS)
    k_summary_noalloc(const double *__restrict__ mu, const double *__restrict__ fc, const double *__restrict__ nu,
                      int n, NoallocScratch *scr, double *__restrict__ out)
{
    __shared__ double sh[4][COT_NOALLOC_THREADS / 32];
    __shared__ bool last;
    const int b0 = blockIdx.x * COT_NOALLOC_BLOCK_ELEMS;
    const int b1 = min(n, b0 + COT_NOALLOC_BLOCK_ELEMS);
    double f = 0.0, mx = 0.0, gn = 0.0, emp = 0.0;
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double g = mu[i] - nu[i];
        f += fc[i];
        const double rel = nu[i] > 0.0 ? fabs(g) / nu[i] : (g != 0.0 ? INFINITY : 0.0);
        // a NaN mass must not look converged: fmax would drop it
        mx = (rel == rel) ? fmax(mx, rel) : INFINITY;
        gn += g * g;
        emp += (mu[i] == 0.0) ? 1.0 : 0.0;
    }
    f = nsum(f);
    mx = nmax(mx);
    gn = nsum(gn);
    emp = nsum(emp);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        sh[0][wid] = f;
        sh[1][wid] = mx;
        sh[2][wid] = gn;
        sh[3][wid] = emp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) {
            r0 += sh[0][k];
            r1 = fmax(r1, sh[1][k]);
            r2 += sh[2][k];
            r3 += sh[3][k];
        }
        double *p = scr->partials + 4 * blockIdx.x;
        p[0] = r0;
        p[1] = r1;
        p[2] = r2;
        p[3] = r3;
        __threadfence();
        const unsigned int t = atomicAdd(&scr->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    const volatile double *p = scr->partials;
    double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
    for (unsigned int k = 0; k < gridDim.x; k++) {
        r0 += p[4 * k + 0];
        r1 = fmax(r1, p[4 * k + 1]);
        r2 += p[4 * k + 2];
        r3 += p[4 * k + 3];
    }
    out[0] = r0;
    out[1] = r1;
    out[2] = r2;
    out[3] = r3;
}

}  // namespace

extern "C" int cot_eval_summary_noalloc(const double *mu, const double *f_cell, const double *nu, int n,
                                        double *out, void *stream)
{
    if (!mu || !f_cell || !nu || !out)
        return cot::fail(nullptr, COT_EINVAL, "cot_eval_summary_noalloc: NULL argument", nullptr);
    if (n <= 0 || n > COT_NOALLOC_MAX_N)
        return cot::fail(nullptr, COT_EINVAL,
                         "cot_eval_summary_noalloc: n must be in 1..COT_NOALLOC_MAX_N (2097152); "
                         "the fixed scratch holds one partial sum per 2048 cells",
                         nullptr);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cot::fail(nullptr, COT_ECUDA, "cot_eval_summary_noalloc: cudaGetDevice", cudaGetErrorString(e));
    if (dev < 0 || dev >= COT_NOALLOC_MAX_DEVICES)
        return cot::fail(nullptr, COT_EINVAL, "cot_eval_summary_noalloc: device ordinal above COT_NOALLOC_MAX_DEVICES", nullptr);
    NoallocScratch *scr = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (g_noalloc_ptr[dev] == nullptr) {
            // once per device, with that device current
            e = cudaGetSymbolAddress((void **)&g_noalloc_ptr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_ptr[dev] = nullptr;
                return cot::fail(nullptr, COT_ECUDA, "cot_eval_summary_noalloc: cudaGetSymbolAddress", cudaGetErrorString(e));
            }
        }
        scr = g_noalloc_ptr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    e = cudaMemsetAsync(&scr->ticket, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return cot::fail(nullptr, COT_ECUDA, "cot_eval_summary_noalloc: clearing the counter", cudaGetErrorString(e));
    const int blocks = (n + COT_NOALLOC_BLOCK_ELEMS - 1) / COT_NOALLOC_BLOCK_ELEMS;
    k_summary_noalloc<<<blocks, COT_NOALLOC_THREADS, 0, s>>>(mu, f_cell, nu, n, scr, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cot::fail(nullptr, COT_ECUDA, "cot_eval_summary_noalloc: launch", cudaGetErrorString(e));
    return COT_OK;
}
