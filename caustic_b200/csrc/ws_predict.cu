// Learned warm start through the C ABI: cot_warmstart_load / _predict / _free
// (include/causticws.h).  The network trained by caustic_b200/warmstart.py is
// saved as a flat binary (WarmStartNet.save_bin); this file reads it, keeps
// the BF16 weights and FP32 biases on the device, prepares the inputs of one
// problem on the host exactly as warmstart.make_input does, and runs the
// forward pass with the same kernels the Python host layer strings together
// (ws_im2col, ws_gemm, ws_bias_act, ws_pool2, ws_up2, ws_put_channels).
// No counterpart in the reference: its solver starts from the previous
// outer iteration's weights or from zero (main.cu:193-198).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/causticws.h"

namespace {

std::string g_ws_err;

int werr(int code, const std::string &msg)
{
    g_ws_err = msg;
    return code;
}

struct Layer {
    int cout = 0, cin = 0, k = 0, has_bias = 0;
    __nv_bfloat16 *w16 = nullptr;  // [cout][k*k*cin]
    float *b = nullptr;            // [cout]
};

const int kInCh = 8;

}  // namespace

struct ws_net {
    int device = 0;
    int levels = 0, base = 0;
    double out_scale = 1.0;
    std::vector<int> ch;
    std::vector<Layer> layers;  // encoder convs, decoder convs, head
    // device buffers of the last forward pass, reused while the site grid
    // stays the same (a pass asks for the same buffers in the same order)
    std::vector<void *> bufs;
    std::vector<size_t> buf_bytes;
    int grid_x = 0, grid_y = 0;
};

namespace {

void free_bufs(ws_net *n)
{
    for (void *p : n->bufs) cudaFree(p);
    n->bufs.clear();
    n->buf_bytes.clear();
}

void free_net(ws_net *n)
{
    if (!n) return;
    for (auto &l : n->layers) {
        if (l.w16) cudaFree(l.w16);
        if (l.b) cudaFree(l.b);
    }
    free_bufs(n);
    delete n;
}

// Device buffers of a forward pass, handed out in request order from the
// network's list: the k-th request of a pass reuses the k-th buffer when it is
// large enough (the same grid asks for the same sizes), else it is replaced.
struct Pool {
    ws_net *net;
    size_t next = 0;
    explicit Pool(ws_net *n) : net(n) {}
    template <class T>
    T *get(size_t count, cudaError_t &e)
    {
        const size_t bytes = count * sizeof(T) > 0 ? count * sizeof(T) : 16;
        if (e != cudaSuccess) return nullptr;
        if (next < net->bufs.size() && net->buf_bytes[next] >= bytes) return static_cast<T *>(net->bufs[next++]);
        void *p = nullptr;
        e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return nullptr;
        if (next < net->bufs.size()) {
            cudaFree(net->bufs[next]);
            net->bufs[next] = p;
            net->buf_bytes[next] = bytes;
        } else {
            net->bufs.push_back(p);
            net->buf_bytes.push_back(bytes);
        }
        next++;
        return static_cast<T *>(p);
    }
};

}  // namespace

extern "C" WS_API int cot_warmstart_last_error(char *buf, size_t n)
{
    if (!buf || n == 0) return WS_EINVAL;
    std::snprintf(buf, n, "%s", g_ws_err.c_str());
    return WS_OK;
}

extern "C" WS_API int cot_warmstart_load(const char *path, int device, ws_net **out)
{
    if (!path || !out) return werr(WS_EINVAL, "cot_warmstart_load: NULL argument");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return werr(WS_EINVAL, std::string("cot_warmstart_load: cannot open ") + path);
    char magic[4];
    int hdr[3];
    double scale = 1.0;
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "CWS1", 4) == 0 &&
              std::fread(hdr, sizeof(int), 3, f) == 3 && std::fread(&scale, sizeof(double), 1, f) == 1;
    const int levels = ok ? hdr[0] : 0, base = ok ? hdr[1] : 0, nl = ok ? hdr[2] : 0;
    if (!ok || levels < 1 || levels > 8 || base < 1 || base > 1024 || nl != 4 * levels - 1) {
        std::fclose(f);
        return werr(WS_EINVAL, "cot_warmstart_load: not a warm-start network file (bad header)");
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        std::fclose(f);
        return werr(WS_ECUDA, "cot_warmstart_load: cudaSetDevice");
    }
    ws_net *n = new ws_net();
    n->device = device;
    n->levels = levels;
    n->base = base;
    n->out_scale = scale;
    for (int l = 0; l < levels; l++) n->ch.push_back(base << l);
    int rc = WS_OK;
    for (int q = 0; q < nl && rc == WS_OK; q++) {
        int meta[4];
        if (std::fread(meta, sizeof(int), 4, f) != 4) {
            rc = werr(WS_EINVAL, "cot_warmstart_load: truncated layer header");
            break;
        }
        Layer L;
        L.cout = meta[0];
        L.cin = meta[1];
        L.k = meta[2];
        L.has_bias = meta[3];
        const size_t nw = (size_t)L.cout * L.k * L.k * L.cin;
        if (L.cout <= 0 || L.cin <= 0 || (L.k != 1 && L.k != 3) || nw > (size_t)1 << 26) {
            rc = werr(WS_EINVAL, "cot_warmstart_load: bad layer shape");
            break;
        }
        std::vector<float> w(nw), b(L.has_bias ? L.cout : 0);
        if (std::fread(w.data(), sizeof(float), nw, f) != nw ||
            (L.has_bias && std::fread(b.data(), sizeof(float), L.cout, f) != (size_t)L.cout)) {
            rc = werr(WS_EINVAL, "cot_warmstart_load: truncated weights");
            break;
        }
        std::vector<__nv_bfloat16> w16(nw);
        for (size_t k = 0; k < nw; k++) w16[k] = __float2bfloat16_rn(w[k]);
        cudaError_t e = cudaMalloc(&L.w16, nw * sizeof(__nv_bfloat16));
        if (e == cudaSuccess) e = cudaMemcpy(L.w16, w16.data(), nw * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice);
        if (e == cudaSuccess && L.has_bias) {
            e = cudaMalloc(&L.b, L.cout * sizeof(float));
            if (e == cudaSuccess) e = cudaMemcpy(L.b, b.data(), L.cout * sizeof(float), cudaMemcpyHostToDevice);
        }
        n->layers.push_back(L);
        if (e != cudaSuccess) rc = werr(WS_ECUDA, std::string("cot_warmstart_load: ") + cudaGetErrorString(e));
    }
    std::fclose(f);
    if (rc != WS_OK) {
        free_net(n);
        return rc;
    }
    *out = n;
    return WS_OK;
}

extern "C" WS_API int cot_warmstart_free(ws_net *net)
{
    if (net) {
        cudaSetDevice(net->device);
        free_net(net);
    }
    return WS_OK;
}

extern "C" WS_API int cot_warmstart_predict(ws_net *net, const double *sites_xy, const double *nu, int gx, int gy,
                                            const double *density, int nx, int ny, const double proj_domain[4],
                                            double *w_out, void *stream)
{
    if (!net || !sites_xy || !nu || !density || !proj_domain || !w_out)
        return werr(WS_EINVAL, "cot_warmstart_predict: NULL argument");
    const int div = 1 << (net->levels - 1);
    if (gx <= 0 || gy <= 0 || gx % div || gy % div)
        return werr(WS_EINVAL, "cot_warmstart_predict: the site grid's sides must be multiples of 2^(levels-1)");
    if (nx <= 0 || ny <= 0 || nx % gx || ny % gy)
        return werr(WS_EINVAL, "cot_warmstart_predict: the image must be a whole number of pixels per site");
    const double *pd = proj_domain;
    if (!(pd[1] > pd[0]) || !(pd[3] > pd[2])) return werr(WS_EINVAL, "cot_warmstart_predict: empty proj_domain");
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaSetDevice(net->device) != cudaSuccess) return werr(WS_ECUDA, "cot_warmstart_predict: cudaSetDevice");
    const int n = gx * gy;
    // ---- inputs (warmstart.make_input) ------------------------------------
    double dsum = 0.0, nsum = 0.0;
    for (long long p = 0; p < (long long)nx * ny; p++) dsum += density[p];
    for (int i = 0; i < n; i++) nsum += nu[i];
    if (!(dsum > 0) || !(nsum > 0)) return werr(WS_EINVAL, "cot_warmstart_predict: density or masses sum to zero");
    const int fx = nx / gx, fy = ny / gy;
    std::vector<double> lg(n, 0.0);
    double lmean = 0.0;
    for (int b = 0; b < gy; b++)
        for (int a = 0; a < gx; a++) {
            double acc = 0.0;
            for (int y = b * fy; y < (b + 1) * fy; y++)
                for (int x = a * fx; x < (a + 1) * fx; x++) acc += density[x + (size_t)y * nx];
            const double img = acc / dsum / (fx * fy) * ((double)nx * ny);
            lg[a + b * gx] = std::log(std::max(img, 1e-12));
            lmean += lg[a + b * gx];
        }
    lmean /= n;
    std::vector<__nv_bfloat16> x((size_t)n * kInCh, __float2bfloat16_rn(0.0f));
    const double sx = pd[1] - pd[0], sy = pd[3] - pd[2];
    for (int b = 0; b < gy; b++)
        for (int a = 0; a < gx; a++) {
            const int i = a + b * gx;
            const double u = (a + 0.5) / gx, v = (b + 0.5) / gy;
            const double jx = ((sites_xy[2 * i] - pd[0]) / sx - u) * (4.0 * gx);
            const double jy = ((sites_xy[2 * i + 1] - pd[2]) / sy - v) * (4.0 * gy);
            const double lm = std::log(std::max(nu[i] / nsum * n, 1e-300));
            __nv_bfloat16 *px = &x[(size_t)i * kInCh];
            px[0] = __float2bfloat16_rn((float)(lg[i] - lmean));
            px[1] = __float2bfloat16_rn((float)jx);
            px[2] = __float2bfloat16_rn((float)jy);
            px[3] = __float2bfloat16_rn((float)lm);
        }
    // ---- forward pass (WarmStartNet.forward) ------------------------------
    if (net->grid_x != gx || net->grid_y != gy) {
        // another grid: the earlier pass's buffers are released first (a
        // buffer still being read by a pass in flight is not freed: the
        // earlier pass ended with a synchronisation)
        free_bufs(net);
        net->grid_x = gx;
        net->grid_y = gy;
    }
    Pool pool(net);
    cudaError_t e = cudaSuccess;
    auto *h = pool.get<__nv_bfloat16>(x.size(), e);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, x.data(), x.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return werr(WS_ECUDA, std::string("cot_warmstart_predict: ") + cudaGetErrorString(e));
    int rc = WS_OK;
    size_t ws_bytes = 0;
    void *wsp = nullptr;
    // one convolution: x [H][W][cin] bf16 -> fp32 d [H*W][cout]; with a bias,
    // y = act(d + b) in bf16
    auto conv = [&](const Layer &L, const __nv_bfloat16 *in, int H, int W, float **d_out) -> __nv_bfloat16 * {
        const int M = H * W, K = L.k * L.k * L.cin;
        const void *cols = in;
        if (L.k == 3) {
            auto *c = pool.get<__nv_bfloat16>((size_t)M * K, e);
            if (e != cudaSuccess) return nullptr;
            if ((rc = ws_im2col(1, H, W, L.cin, in, c, s)) != WS_OK) return nullptr;
            cols = c;
        }
        float *d = pool.get<float>((size_t)M * L.cout, e);
        const size_t need = ws_gemm_workspace(WS_GEMM_RC, M, L.cout, K);
        if (need > ws_bytes) {
            wsp = pool.get<unsigned char>(need, e);
            ws_bytes = need;
        }
        if (e != cudaSuccess) return nullptr;
        if ((rc = ws_gemm(WS_GEMM_RC, M, L.cout, K, cols, L.w16, d, 1.0f, 0.0f, need ? wsp : nullptr, need, s)) !=
            WS_OK)
            return nullptr;
        if (d_out) *d_out = d;
        if (!L.has_bias) return nullptr;
        auto *y = pool.get<__nv_bfloat16>((size_t)M * L.cout, e);
        if (e != cudaSuccess) return nullptr;
        if ((rc = ws_bias_act(M, L.cout, d, L.b, 1, y, nullptr, s)) != WS_OK) return nullptr;
        return y;
    };
    const int levels = net->levels;
    std::vector<const __nv_bfloat16 *> skips(levels);
    int H = gy, W = gx, q = 0;
    const __nv_bfloat16 *cur = h;
    for (int l = 0; l < levels; l++) {
        for (int t = 0; t < 2; t++) {
            cur = conv(net->layers[q++], cur, H, W, nullptr);
            if (!cur) goto fail;
        }
        skips[l] = cur;
        if (l < levels - 1) {
            auto *p = pool.get<__nv_bfloat16>((size_t)(H / 2) * (W / 2) * net->ch[l], e);
            if (e != cudaSuccess) goto fail;
            if ((rc = ws_pool2(1, H, W, net->ch[l], cur, p, s)) != WS_OK) goto fail;
            cur = p;
            H /= 2;
            W /= 2;
        }
    }
    for (int l = levels - 2; l >= 0; l--) {
        const int ct = net->ch[l + 1] + net->ch[l];
        auto *cat = pool.get<__nv_bfloat16>((size_t)(2 * H) * (2 * W) * ct, e);
        if (e != cudaSuccess) goto fail;
        if ((rc = ws_up2(1, H, W, net->ch[l + 1], cur, ct, 0, cat, s)) != WS_OK) goto fail;
        H *= 2;
        W *= 2;
        if ((rc = ws_put_channels((long long)H * W, net->ch[l], skips[l], ct, net->ch[l + 1], cat, s)) != WS_OK)
            goto fail;
        cur = cat;
        for (int t = 0; t < 2; t++) {
            cur = conv(net->layers[q++], cur, H, W, nullptr);
            if (!cur) goto fail;
        }
    }
    {
        float *d = nullptr;
        conv(net->layers[q++], cur, H, W, &d);  // the head: no bias, fp32 out [H*W][8]
        if (!d || rc != WS_OK || e != cudaSuccess) goto fail;
        std::vector<float> out((size_t)n * 8);
        e = cudaMemcpyAsync(out.data(), d, out.size() * sizeof(float), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) goto fail;
        double mean = 0.0;
        for (int i = 0; i < n; i++) {
            w_out[i] = (double)out[(size_t)i * 8] * net->out_scale / n;
            mean += w_out[i];
        }
        mean /= n;
        for (int i = 0; i < n; i++) w_out[i] -= mean;
        return WS_OK;
    }
fail:
    if (e != cudaSuccess) return werr(WS_ECUDA, std::string("cot_warmstart_predict: ") + cudaGetErrorString(e));
    return werr(rc != WS_OK ? rc : WS_ECUDA, "cot_warmstart_predict: a layer kernel failed");
}
