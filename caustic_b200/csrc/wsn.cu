// Kernels of the warm-start network: a convolutional encoder-decoder that
// maps a target image and the site layout to initial dual weights.  BF16
// operands, FP32 accumulation.  3x3 convolutions run as im2col + a tensor-core
// GEMM (tcgen05 through the CUTLASS sm100 collective templates); everything
// around them (im2col / col2im, bias + ReLU, pooling, upsampling, concat,
// loss, optimizer) is written here.  Activations are NHWC; a layer's weights
// are [Cout][9*Cin] (tap-major, channel-minor), the matrix B of the GEMM
// D[M, Cout] = cols[M, 9*Cin] * W^T.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cutlass/cutlass.h>
#include <cute/tensor.hpp>
#include <cutlass/gemm/device/gemm_universal_adapter.h>
#include <cutlass/gemm/kernel/gemm_universal.hpp>
#include <cutlass/gemm/collective/collective_builder.hpp>
#include <cutlass/epilogue/collective/collective_builder.hpp>
#include <cutlass/util/packed_stride.hpp>

#include "../../include/causticws.h"

namespace {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// GEMM: D[M,N] (fp32, row-major) = alpha * A[M,K] * B[K,N] + beta * D
// ---------------------------------------------------------------------------
// One GEMM configuration per operand layout: 128x128x64 tiles on one SM,
// fp32 accumulators in tensor memory, fp32 output.
#define WS_GEMM_CONFIG(NAME, LA, LB)                                                                                \
    namespace NAME {                                                                                                \
    using ElemAB = cutlass::bfloat16_t;                                                                            \
    using Tile = cute::Shape<cute::_128, cute::_128, cute::_64>;                                                   \
    using Cluster = cute::Shape<cute::_1, cute::_1, cute::_1>;                                                     \
    using Epilogue = cutlass::epilogue::collective::CollectiveBuilder<                                             \
        cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, Tile, Cluster,                                       \
        cutlass::epilogue::collective::EpilogueTileAuto, float, float, float, cutlass::layout::RowMajor, 4, float,  \
        cutlass::layout::RowMajor, 4, cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;          \
    using Mainloop = cutlass::gemm::collective::CollectiveBuilder<                                                 \
        cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElemAB, LA, 8, ElemAB, LB, 8, float, Tile, Cluster,  \
        cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(sizeof(Epilogue::SharedStorage))>,      \
        cutlass::gemm::collective::KernelScheduleAuto>::CollectiveOp;                                              \
    using Kernel = cutlass::gemm::kernel::GemmUniversal<cute::Shape<int, int, int, int>, Mainloop, Epilogue, void>; \
    using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;                                              \
    inline Gemm::Arguments args(int M, int N, int K, const void *A, const void *B, float *D, float alpha,          \
                                float beta)                                                                         \
    {                                                                                                              \
        auto sa = cutlass::make_cute_packed_stride(Kernel::StrideA{}, cute::make_shape(M, K, 1));                  \
        auto sb = cutlass::make_cute_packed_stride(Kernel::StrideB{}, cute::make_shape(N, K, 1));                  \
        auto sd = cutlass::make_cute_packed_stride(Kernel::StrideD{}, cute::make_shape(M, N, 1));                  \
        return Gemm::Arguments{cutlass::gemm::GemmUniversalMode::kGemm,                                            \
                               {M, N, K, 1},                                                                        \
                               {static_cast<const ElemAB *>(A), sa, static_cast<const ElemAB *>(B), sb},            \
                               {{alpha, beta}, D, sd, D, sd}};                                                      \
    }                                                                                                              \
    inline int run(int M, int N, int K, const void *A, const void *B, float *D, float alpha, float beta, void *ws, \
                   size_t ws_bytes, cudaStream_t s)                                                                \
    {                                                                                                              \
        auto a = args(M, N, K, A, B, D, alpha, beta);                                                              \
        Gemm g;                                                                                                    \
        if (g.can_implement(a) != cutlass::Status::kSuccess) return WS_EINVAL;                                    \
        if (Gemm::get_workspace_size(a) > ws_bytes) return WS_ECAPACITY;                                          \
        if (g.initialize(a, ws, s) != cutlass::Status::kSuccess) return WS_ECUDA;                                 \
        return g.run(s) == cutlass::Status::kSuccess ? WS_OK : WS_ECUDA;                                          \
    }                                                                                                              \
    inline size_t workspace(int M, int N, int K)                                                                   \
    {                                                                                                              \
        return Gemm::get_workspace_size(args(M, N, K, nullptr, nullptr, nullptr, 1.f, 0.f));                       \
    }                                                                                                              \
    }

// A[M,K] K-contiguous, B stored [N][K]  (forward: D = cols W^T)
WS_GEMM_CONFIG(GemmRC, cutlass::layout::RowMajor, cutlass::layout::ColumnMajor)
// A stored [K][M], B[K,N] N-contiguous   (weight gradient: dW = dZ^T cols)
WS_GEMM_CONFIG(GemmCR, cutlass::layout::ColumnMajor, cutlass::layout::RowMajor)
// A[M,K], B[K,N] both row-major         (input gradient: dcols = dZ W)
WS_GEMM_CONFIG(GemmRR, cutlass::layout::RowMajor, cutlass::layout::RowMajor)

constexpr int T = 256;

// ---------------------------------------------------------------------------
// im2col / col2im for 3x3, stride 1, zero padding 1, NHWC
// ---------------------------------------------------------------------------
// cols[(b*H + y)*W + x][tap*C + c] = in[b][y+dy][x+dx][c], tap = (dy+1)*3 + (dx+1)
__global__ void k_im2col(int B, int H, int W, int Cn, const bf16 *__restrict__ in, bf16 *__restrict__ cols)
{
    const long long K = 9LL * Cn;
    const long long total = (long long)B * H * W * K;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const long long row = q / K;
        const int k = (int)(q - row * K);
        const int tap = k / Cn, c = k - tap * Cn;
        const int x = (int)(row % W), y = (int)((row / W) % H), b = (int)(row / ((long long)W * H));
        const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
        bf16 v = __float2bfloat16(0.f);
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = in[(((long long)b * H + yy) * W + xx) * Cn + c];
        cols[q] = v;
    }
}

// dx[b][y][x][c] = sum over the (up to 9) output pixels that read it: a
// gather, so the sum order is fixed and no atomics are needed.
__global__ void k_col2im(int B, int H, int W, int Cn, const float *__restrict__ dcols, float *__restrict__ dx)
{
    const long long K = 9LL * Cn;
    const long long total = (long long)B * H * W * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % Cn);
        const long long pix = q / Cn;
        const int x = (int)(pix % W), y = (int)((pix / W) % H), b = (int)(pix / ((long long)W * H));
        float acc = 0.f;
        for (int tap = 0; tap < 9; tap++) {
            // output pixel (y - dy, x - dx) read this input through tap (dy, dx)
            const int oy = y - (tap / 3 - 1), ox = x - (tap % 3 - 1);
            if (oy < 0 || oy >= H || ox < 0 || ox >= W) continue;
            acc += dcols[(((long long)b * H + oy) * W + ox) * K + tap * Cn + c];
        }
        dx[q] = acc;
    }
}

// y = relu(d + bias) (bf16), pre = d + bias kept for the backward pass
__global__ void k_bias_act(long long M, int Cn, const float *__restrict__ d, const float *__restrict__ bias,
                           int relu, bf16 *__restrict__ y, float *__restrict__ pre)
{
    const long long total = M * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const float v = d[q] + bias[q % Cn];
        if (pre) pre[q] = v;
        y[q] = __float2bfloat16(relu ? fmaxf(v, 0.f) : v);
    }
}

// dz = dy * relu'(pre) in bf16 for the GEMMs
__global__ void k_act_back(long long n, int relu, const float *__restrict__ dy, const float *__restrict__ pre,
                           bf16 *__restrict__ dz, float *__restrict__ dz32)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const float g = (!relu || pre[q] > 0.f) ? dy[q] : 0.f;
        dz[q] = __float2bfloat16(g);
        if (dz32) dz32[q] = g;
    }
}

// db[c] = sum_m dz[m][c], one block per channel, fixed order
__global__ void k_colsum(long long M, int Cn, const float *__restrict__ dz, float *__restrict__ db)
{
    __shared__ float sh[T];
    const int c = blockIdx.x;
    float acc = 0.f;
    for (long long m = threadIdx.x; m < M; m += blockDim.x) acc += dz[m * Cn + c];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[c] = sh[0];
}

// 2x2 average pooling (H, W even) and its adjoint
__global__ void k_pool2(int B, int H, int W, int Cn, const bf16 *__restrict__ in, bf16 *__restrict__ out)
{
    const int Ho = H / 2, Wo = W / 2;
    const long long total = (long long)B * Ho * Wo * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % Cn);
        const long long p = q / Cn;
        const int x = (int)(p % Wo), y = (int)((p / Wo) % Ho), b = (int)(p / ((long long)Wo * Ho));
        const bf16 *src = in + (((long long)b * H + 2 * y) * W + 2 * x) * Cn + c;
        const float s = __bfloat162float(src[0]) + __bfloat162float(src[Cn]) + __bfloat162float(src[(long long)W * Cn]) +
                        __bfloat162float(src[(long long)W * Cn + Cn]);
        out[q] = __float2bfloat16(0.25f * s);
    }
}

__global__ void k_pool2_back(int B, int H, int W, int Cn, const float *__restrict__ dout, float *__restrict__ din)
{
    const long long total = (long long)B * H * W * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % Cn);
        const long long p = q / Cn;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
        din[q] = 0.25f * dout[(((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * Cn + c];
    }
}

// nearest 2x upsampling into channels [c0, c0 + Cn) of an output with Ct channels
__global__ void k_up2(int B, int H, int W, int Cn, const bf16 *__restrict__ in, int Ct, int c0, bf16 *__restrict__ out)
{
    const long long total = (long long)B * (2 * H) * (2 * W) * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % Cn);
        const long long p = q / Cn;
        const int x = (int)(p % (2 * W)), y = (int)((p / (2 * W)) % (2 * H)), b = (int)(p / (4LL * W * H));
        out[p * Ct + c0 + c] = in[(((long long)b * H + y / 2) * W + x / 2) * Cn + c];
    }
}

__global__ void k_up2_back(int B, int H, int W, int Cn, const float *__restrict__ dout, int Ct, int c0,
                           float *__restrict__ din)
{
    const long long total = (long long)B * H * W * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(q % Cn);
        const long long p = q / Cn;
        const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
        float s = 0.f;
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++)
                s += dout[(((long long)b * 2 * H + 2 * y + dy) * 2 * W + 2 * x + dx) * Ct + c0 + c];
        din[q] = s;
    }
}

// copy channels: out[p][c0 + c] = in[p][c] (a skip connection into a concat
// buffer) and the backward split din[p][c] = dout[p][c0 + c]
__global__ void k_put_channels(long long P, int Cn, const bf16 *__restrict__ in, int Ct, int c0, bf16 *__restrict__ out)
{
    const long long total = P * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x)
        out[(q / Cn) * Ct + c0 + q % Cn] = in[q];
}

__global__ void k_take_channels(long long P, int Cn, const float *__restrict__ dout, int Ct, int c0, float add,
                                float *__restrict__ din)
{
    const long long total = P * Cn;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const float v = dout[(q / Cn) * Ct + c0 + q % Cn];
        din[q] = add != 0.f ? din[q] + v : v;
    }
}

// Mean-free error per sample on a gy x gx grid: the weights are defined up
// to a constant, so prediction and target are compared after removing each
// one's mean.  With e = pred - target - mean:
//   loss_b = [ sum_i e_i^2 + lambda * sum (forward differences of e)^2 ] / (n B)
// (the second term weighs the local differences that set the cells' masses)
// and grad = d(sum_b loss_b) / d pred.
__global__ void k_mse_centered(int B, int gy, int gx, float lambda, const float *__restrict__ p,
                               const float *__restrict__ t, float *__restrict__ grad, float *__restrict__ loss_b)
{
    __shared__ float sh[T];
    const int n = gy * gx;
    const int b = blockIdx.x;
    const float *pb = p + (long long)b * n;
    const float *tb = t + (long long)b * n;
    float acc = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += pb[i] - tb[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    const float mean = sh[0] / n;
    __syncthreads();
    const float sc = 1.f / ((float)n * B);
    float l = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int x = i % gx, y = i / gx;
        const float e = pb[i] - tb[i] - mean;
        float g = 2.f * e;
        l += e * e;
        if (lambda != 0.f) {
            // differences to the right / upper neighbour (counted once) and
            // the gradient of every difference this site is part of
            if (x + 1 < gx) {
                const float d = (pb[i + 1] - tb[i + 1] - mean) - e;
                l += lambda * d * d;
                g -= 2.f * lambda * d;
            }
            if (x > 0) g += 2.f * lambda * (e - (pb[i - 1] - tb[i - 1] - mean));
            if (y + 1 < gy) {
                const float d = (pb[i + gx] - tb[i + gx] - mean) - e;
                l += lambda * d * d;
                g -= 2.f * lambda * d;
            }
            if (y > 0) g += 2.f * lambda * (e - (pb[i - gx] - tb[i - gx] - mean));
        }
        grad[(long long)b * n + i] = g * sc;
    }
    sh[threadIdx.x] = l;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) loss_b[b] = sh[0] * sc;
}

// Adam on fp32 master weights, with the bf16 copy the GEMMs read
__global__ void k_adam(long long n, float *__restrict__ w, bf16 *__restrict__ w16, const float *__restrict__ g,
                       float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        const float wq = w[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
        w[q] = wq;
        if (w16) w16[q] = __float2bfloat16(wq);
    }
}

__global__ void k_to_bf16(long long n, const float *__restrict__ x, bf16 *__restrict__ y)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        y[q] = __float2bfloat16(x[q]);
}

inline int grid_for(long long n)
{
    const long long b = (n + T - 1) / T;
    return (int)(b < 148LL * 32 ? b : 148LL * 32);
}

inline int last_error()
{
    return cudaGetLastError() == cudaSuccess ? WS_OK : WS_ECUDA;
}

}  // namespace

extern "C" {

WS_API int ws_gemm(int layout, int M, int N, int K, const void *A, const void *B, float *D, float alpha, float beta,
                   void *workspace, size_t workspace_bytes, void *stream)
{
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !D) return WS_EINVAL;
    if (K % 8 != 0) return WS_EINVAL;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    switch (layout) {
    case WS_GEMM_RC: return GemmRC::run(M, N, K, A, B, D, alpha, beta, workspace, workspace_bytes, s);
    case WS_GEMM_CR:
        if (M % 8 != 0 || N % 8 != 0) return WS_EINVAL;
        return GemmCR::run(M, N, K, A, B, D, alpha, beta, workspace, workspace_bytes, s);
    case WS_GEMM_RR:
        if (N % 8 != 0) return WS_EINVAL;
        return GemmRR::run(M, N, K, A, B, D, alpha, beta, workspace, workspace_bytes, s);
    default: return WS_EINVAL;
    }
}

WS_API size_t ws_gemm_workspace(int layout, int M, int N, int K)
{
    switch (layout) {
    case WS_GEMM_RC: return GemmRC::workspace(M, N, K);
    case WS_GEMM_CR: return GemmCR::workspace(M, N, K);
    case WS_GEMM_RR: return GemmRR::workspace(M, N, K);
    default: return 0;
    }
}

WS_API int ws_im2col(int B, int H, int W, int C, const void *in, void *cols, void *stream)
{
    const long long n = (long long)B * H * W * 9 * C;
    k_im2col<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(B, H, W, C, static_cast<const bf16 *>(in),
                                                                        static_cast<bf16 *>(cols));
    return last_error();
}

WS_API int ws_col2im(int B, int H, int W, int C, const float *dcols, float *dx, void *stream)
{
    const long long n = (long long)B * H * W * C;
    k_col2im<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(B, H, W, C, dcols, dx);
    return last_error();
}

WS_API int ws_bias_act(long long M, int C, const float *d, const float *bias, int relu, void *y, float *pre,
                       void *stream)
{
    k_bias_act<<<grid_for(M * C), T, 0, static_cast<cudaStream_t>(stream)>>>(M, C, d, bias, relu,
                                                                              static_cast<bf16 *>(y), pre);
    return last_error();
}

WS_API int ws_act_back(long long n, int relu, const float *dy, const float *pre, void *dz, float *dz32, void *stream)
{
    k_act_back<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(n, relu, dy, pre, static_cast<bf16 *>(dz),
                                                                          dz32);
    return last_error();
}

WS_API int ws_colsum(long long M, int C, const float *dz, float *db, void *stream)
{
    k_colsum<<<C, T, 0, static_cast<cudaStream_t>(stream)>>>(M, C, dz, db);
    return last_error();
}

WS_API int ws_pool2(int B, int H, int W, int C, const void *in, void *out, void *stream)
{
    if (H % 2 || W % 2) return WS_EINVAL;
    const long long n = (long long)B * (H / 2) * (W / 2) * C;
    k_pool2<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(B, H, W, C, static_cast<const bf16 *>(in),
                                                                        static_cast<bf16 *>(out));
    return last_error();
}

WS_API int ws_pool2_back(int B, int H, int W, int C, const float *dout, float *din, void *stream)
{
    if (H % 2 || W % 2) return WS_EINVAL;
    const long long n = (long long)B * H * W * C;
    k_pool2_back<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(B, H, W, C, dout, din);
    return last_error();
}

WS_API int ws_up2(int B, int H, int W, int C, const void *in, int Ct, int c0, void *out, void *stream)
{
    const long long n = (long long)B * 4 * H * W * C;
    k_up2<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(B, H, W, C, static_cast<const bf16 *>(in), Ct, c0,
                                                                      static_cast<bf16 *>(out));
    return last_error();
}

WS_API int ws_up2_back(int B, int H, int W, int C, const float *dout, int Ct, int c0, float *din, void *stream)
{
    const long long n = (long long)B * H * W * C;
    k_up2_back<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(B, H, W, C, dout, Ct, c0, din);
    return last_error();
}

WS_API int ws_put_channels(long long P, int C, const void *in, int Ct, int c0, void *out, void *stream)
{
    k_put_channels<<<grid_for(P * C), T, 0, static_cast<cudaStream_t>(stream)>>>(
        P, C, static_cast<const bf16 *>(in), Ct, c0, static_cast<bf16 *>(out));
    return last_error();
}

WS_API int ws_take_channels(long long P, int C, const float *dout, int Ct, int c0, int add, float *din, void *stream)
{
    k_take_channels<<<grid_for(P * C), T, 0, static_cast<cudaStream_t>(stream)>>>(P, C, dout, Ct, c0,
                                                                                   add ? 1.f : 0.f, din);
    return last_error();
}

WS_API int ws_mse_centered(int B, int gy, int gx, float lambda, const float *pred, const float *target, float *grad,
                           float *loss_b, void *stream)
{
    if (B <= 0 || gy <= 0 || gx <= 0) return WS_EINVAL;
    k_mse_centered<<<B, T, 0, static_cast<cudaStream_t>(stream)>>>(B, gy, gx, lambda, pred, target, grad, loss_b);
    return last_error();
}

WS_API int ws_adam(long long n, float *w, void *w16, const float *g, float *m, float *v, float lr, float b1, float b2,
                   float eps, int step, void *stream)
{
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(n, w, static_cast<bf16 *>(w16), g, m, v, lr, b1,
                                                                      b2, eps, c1, c2);
    return last_error();
}

WS_API int ws_to_bf16(long long n, const float *x, void *y, void *stream)
{
    k_to_bf16<<<grid_for(n), T, 0, static_cast<cudaStream_t>(stream)>>>(n, x, static_cast<bf16 *>(y));
    return last_error();
}

}  // extern "C"
