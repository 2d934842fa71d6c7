// The learned outer preconditioner inside the library (giem2g_set_preconditioner), for hosts that cannot
// run Python: the bias-free 4-level 3-D U-Net of giem2g_b200/learned.py (channels 16/32/64/64, stride-2
// 3x3x3 convolutions down, nearest upsampling and concatenation up), its weights read from the same .npz
// file, evaluated with the same kernels and the same BF16 roundings as the Python layer:
//   x = [Re v/rms, Im v/rms, (log10 sigma + 2), log10(f)/2] (channels-last, bf16)
//   every convolution = im2col (bf16) -> tcgen05 BF16 GEMM (FP32 out) -> ReLU -> bf16
//   up path = nearest upsampling (x2 in z, y, x) concatenated with the skip tensor
//   z = v + rms * (out[0:3] + i out[3:6])
// It is registered as the operator's outer right-preconditioner hook (the slot SET_RIGHT_PRECONDTIONER,
// seq_fgmres.F90:92-102, fills with the inner GMRES), so the solver's fallback rule applies unchanged.
#include <cuda_bf16.h>
#include <zlib.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include "common.cuh"
#include "ie_internal.h"

namespace {

using bf16 = __nv_bfloat16;

// ---- .npz (zip of .npy) reading --------------------------------------------------------------------
uint32_t rd32(const unsigned char *p) { return p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); }
uint16_t rd16(const unsigned char *p) { return (uint16_t)(p[0] | (p[1] << 8)); }

struct Array {
    std::vector<int> shape;
    std::vector<float> data;
};

// .npy payload: little-endian float32, C order
bool parse_npy(const std::vector<unsigned char> &b, Array &out, std::string &err)
{
    if (b.size() < 10 || std::memcmp(b.data(), "\x93NUMPY", 6) != 0) { err = "not a .npy array"; return false; }
    const int major = b[6];
    size_t hl, off;
    if (major == 1) { hl = rd16(&b[8]); off = 10; }
    else { if (b.size() < 12) { err = "short .npy header"; return false; } hl = rd32(&b[8]); off = 12; }
    if (off + hl > b.size()) { err = "short .npy header"; return false; }
    const std::string h(reinterpret_cast<const char *>(&b[off]), hl);
    if (h.find("'descr': '<f4'") == std::string::npos) { err = "weights must be float32 ('<f4')"; return false; }
    if (h.find("'fortran_order': False") == std::string::npos) { err = "weights must be C-ordered"; return false; }
    const size_t s0 = h.find("'shape': ("), s1 = h.find(')', s0);
    if (s0 == std::string::npos || s1 == std::string::npos) { err = "no shape in .npy header"; return false; }
    out.shape.clear();
    size_t n = 1;
    for (size_t i = s0 + 10; i < s1;) {
        while (i < s1 && (h[i] == ' ' || h[i] == ',')) i++;
        if (i >= s1) break;
        const int v = std::atoi(h.c_str() + i);
        out.shape.push_back(v);
        n *= (size_t)v;
        while (i < s1 && h[i] != ',') i++;
    }
    const size_t data_off = off + hl;
    if (b.size() < data_off + n * 4) { err = "truncated .npy data"; return false; }
    out.data.resize(n);
    std::memcpy(out.data.data(), &b[data_off], n * 4);
    return true;
}

// zip central directory -> name -> array (stored or deflated entries)
bool read_npz(const char *path, std::map<std::string, Array> &arrays, std::string &err)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) { err = std::string("cannot open ") + path; return false; }
    std::vector<unsigned char> z;
    unsigned char buf[1 << 16];
    size_t r;
    while ((r = std::fread(buf, 1, sizeof(buf), f)) > 0) z.insert(z.end(), buf, buf + r);
    std::fclose(f);
    if (z.size() < 22) { err = "not a zip file"; return false; }
    size_t eocd = std::string::npos;
    for (size_t i = z.size() - 22 + 1; i-- > 0;)
        if (rd32(&z[i]) == 0x06054b50u) { eocd = i; break; }
    if (eocd == std::string::npos) { err = "no zip end record"; return false; }
    const int entries = rd16(&z[eocd + 10]);
    size_t cd = rd32(&z[eocd + 16]);
    for (int e = 0; e < entries; e++) {
        if (cd + 46 > z.size() || rd32(&z[cd]) != 0x02014b50u) { err = "bad zip directory"; return false; }
        const int method = rd16(&z[cd + 10]);
        const size_t csize = rd32(&z[cd + 20]), usize = rd32(&z[cd + 24]);
        const size_t nlen = rd16(&z[cd + 28]), xlen = rd16(&z[cd + 30]), clen = rd16(&z[cd + 32]);
        const size_t loc = rd32(&z[cd + 42]);
        std::string name(reinterpret_cast<const char *>(&z[cd + 46]), nlen);
        cd += 46 + nlen + xlen + clen;
        if (loc + 30 > z.size() || rd32(&z[loc]) != 0x04034b50u) { err = "bad zip entry"; return false; }
        const size_t data = loc + 30 + rd16(&z[loc + 26]) + rd16(&z[loc + 28]);
        if (data + csize > z.size()) { err = "truncated zip entry"; return false; }
        std::vector<unsigned char> raw(usize);
        if (method == 0) {
            std::memcpy(raw.data(), &z[data], usize);
        } else if (method == 8) {
            z_stream s{};
            if (inflateInit2(&s, -MAX_WBITS) != Z_OK) { err = "inflateInit failed"; return false; }
            s.next_in = &z[data];
            s.avail_in = (uInt)csize;
            s.next_out = raw.data();
            s.avail_out = (uInt)usize;
            const int rc = inflate(&s, Z_FINISH);
            inflateEnd(&s);
            if (rc != Z_STREAM_END) { err = "inflate failed for " + name; return false; }
        } else {
            err = "unsupported zip compression";
            return false;
        }
        if (name.size() > 4 && name.compare(name.size() - 4, 4, ".npy") == 0) name.resize(name.size() - 4);
        Array a;
        if (!parse_npy(raw, a, err)) { err = name + ": " + err; return false; }
        arrays[name] = std::move(a);
    }
    return true;
}

// ---- kernels ----------------------------------------------------------------------------------------
constexpr int TPB = 256;

__global__ void k_sumsq(const double2 *__restrict__ v, long long n, double *partial)
{
    __shared__ double red[TPB / 32];
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB)
        s += v[i].x * v[i].x + v[i].y * v[i].y;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < TPB / 32; w++) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// rms = sqrt(mean |v|^2), clamped at 1e-300 (encode, learned.py)
__global__ void k_rms(const double *partial, int nb, long long n, double *rms)
{
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < nb; b++) t += partial[b];
        rms[0] = fmax(sqrt(t / (double)n), 1e-300);
    }
}

// x[cell][8] = Re, Im of v/rms (complex64), then the two model channels; v is [3][cells]
__global__ void k_encode(const double2 *__restrict__ v, const float *__restrict__ logsig, float logf,
                         const double *__restrict__ rms, bf16 *__restrict__ x, long long cells)
{
    const double r = rms[0];
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < cells; i += (long long)gridDim.x * TPB) {
        bf16 *o = x + i * 8;
        for (int c = 0; c < 3; c++) {
            const double2 a = v[c * cells + i];
            o[c] = __float2bfloat16((float)(a.x / r));
            o[3 + c] = __float2bfloat16((float)(a.y / r));
        }
        o[6] = __float2bfloat16(logsig[i]);
        o[7] = __float2bfloat16(logf);
    }
}

__global__ void k_relu_bf16(const float *__restrict__ y, bf16 *__restrict__ out, long long n)
{
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB)
        out[i] = __float2bfloat16(fmaxf(y[i], 0.f));
}

// out[z][y][x][Ca+Cs] = (a[z/2][y/2][x/2][Ca], s[z][y][x][Cs])
__global__ void k_up_concat(const bf16 *__restrict__ a, const bf16 *__restrict__ s, bf16 *__restrict__ out, int D,
                            int H, int W, int Ca, int Cs)
{
    const int C = Ca + Cs;
    const long long n = (long long)D * H * W * C;
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB) {
        const int c = (int)(i % C);
        const long long v = i / C;
        const int x = (int)(v % W), y = (int)((v / W) % H), z = (int)(v / ((long long)W * H));
        out[i] = c < Ca ? a[((((long long)(z / 2) * (H / 2) + y / 2) * (W / 2)) + x / 2) * Ca + c] : s[v * Cs + (c - Ca)];
    }
}

// z = v + rms * (out[cell][c] + i out[cell][3 + c])  (decode, learned.py)
__global__ void k_decode(const float *__restrict__ y, const double2 *__restrict__ v, const double *__restrict__ rms,
                         double2 *__restrict__ z, long long cells)
{
    const double r = rms[0];
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < cells; i += (long long)gridDim.x * TPB)
        for (int c = 0; c < 3; c++) {
            const double2 a = v[c * cells + i];
            z[c * cells + i] = make_double2(a.x + (double)y[i * 8 + c] * r, a.y + (double)y[i * 8 + 3 + c] * r);
        }
}

__global__ void k_f32_to_bf16(const float *__restrict__ a, bf16 *__restrict__ b, long long n)
{
    for (long long i = blockIdx.x * (long long)TPB + threadIdx.x; i < n; i += (long long)gridDim.x * TPB)
        b[i] = __float2bfloat16(a[i]);
}

int blocks(long long n) { return (int)std::min<long long>((n + TPB - 1) / TPB, 148LL * 16); }

struct LayerDef {
    const char *name;
    int cin, cout, stride;
};
// learned.py UNet3D.LAYERS
const LayerDef kLayers[12] = {{"in", 8, 16, 1},   {"e0", 16, 16, 1}, {"d1", 16, 32, 2}, {"e1", 32, 32, 1},
                              {"d2", 32, 64, 2},  {"e2", 64, 64, 1}, {"d3", 64, 64, 2}, {"b", 64, 64, 1},
                              {"u2", 128, 64, 1}, {"u1", 96, 32, 1}, {"u0", 48, 16, 1}, {"out", 16, 8, 1}};
int kp_of(int c) { return ((27 * c + 7) / 8) * 8; }

struct Net {
    int D = 0, H = 0, W = 0;
    bf16 *w[12] = {};
    float *logsig = nullptr;
    float logf = 0.f;
    double *partial = nullptr, *rms = nullptr;
    bf16 *x0 = nullptr, *e0 = nullptr, *e1 = nullptr, *e2 = nullptr, *t = nullptr, *b = nullptr, *u = nullptr,
         *cat = nullptr, *cols = nullptr;
    float *y = nullptr;
    int *d_err = nullptr;  // error word of the GEMM's bounded waits
    int nb = 0;
    long long calls = 0;

    ~Net()
    {
        for (auto p : w) cudaFree(p);
        void *ps[] = {logsig, partial, rms, x0, e0, e1, e2, t, b, u, cat, cols, y, d_err};
        for (void *p : ps) cudaFree(p);
    }

    // conv(layer, in [d][h][w][cin]) -> y fp32 [V'][cout]; returns V'
    int conv(int l, const bf16 *in, int d, int h, int wd, cudaStream_t st, long long *vout)
    {
        const LayerDef &L = kLayers[l];
        const int s = L.stride, kp = kp_of(L.cin);
        const int Do = (d - 1) / s + 1, Ho = (h - 1) / s + 1, Wo = (wd - 1) / s + 1;
        const long long V = (long long)Do * Ho * Wo;
        int rc = ie_im2col3d(in, cols, 1, d, h, wd, L.cin, s, kp, st);
        if (rc) return rc;
        rc = ie_gemm_bf16_tn(cols, w[l], y, (int)V, L.cout, kp, kp, kp, L.cout, 0, d_err, st);
        if (rc) return rc;
        *vout = V;
        return G2_OK;
    }
    int conv_relu(int l, const bf16 *in, int d, int h, int wd, bf16 *out, cudaStream_t st)
    {
        long long V = 0;
        int rc = conv(l, in, d, h, wd, st, &V);
        if (rc) return rc;
        const long long n = V * kLayers[l].cout;
        k_relu_bf16<<<blocks(n), TPB, 0, st>>>(y, out, n);
        return G2_OK;
    }

    int forward(const double2 *v, double2 *z, cudaStream_t st)
    {
        const long long cells = (long long)D * H * W;
        k_sumsq<<<nb, TPB, 0, st>>>(v, 3 * cells, partial);
        k_rms<<<1, 32, 0, st>>>(partial, nb, 3 * cells, rms);
        k_encode<<<blocks(cells), TPB, 0, st>>>(v, logsig, logf, rms, x0, cells);
        const int D2 = D / 2, H2 = H / 2, W2 = W / 2, D4 = D / 4, H4 = H / 4, W4 = W / 4;
        const int D8 = D / 8, H8 = H / 8, W8 = W / 8;
        int rc;
#define NET_TRY(e) if ((rc = (e)) != G2_OK) return rc
        NET_TRY(conv_relu(0, x0, D, H, W, t, st));            // in
        NET_TRY(conv_relu(1, t, D, H, W, e0, st));            // e0
        NET_TRY(conv_relu(2, e0, D, H, W, t, st));            // d1
        NET_TRY(conv_relu(3, t, D2, H2, W2, e1, st));         // e1
        NET_TRY(conv_relu(4, e1, D2, H2, W2, t, st));         // d2
        NET_TRY(conv_relu(5, t, D4, H4, W4, e2, st));         // e2
        NET_TRY(conv_relu(6, e2, D4, H4, W4, t, st));         // d3
        NET_TRY(conv_relu(7, t, D8, H8, W8, b, st));          // b
        k_up_concat<<<blocks((long long)D4 * H4 * W4 * 128), TPB, 0, st>>>(b, e2, cat, D4, H4, W4, 64, 64);
        NET_TRY(conv_relu(8, cat, D4, H4, W4, u, st));        // u2
        k_up_concat<<<blocks((long long)D2 * H2 * W2 * 96), TPB, 0, st>>>(u, e1, cat, D2, H2, W2, 64, 32);
        NET_TRY(conv_relu(9, cat, D2, H2, W2, u, st));        // u1
        k_up_concat<<<blocks(cells * 48), TPB, 0, st>>>(u, e0, cat, D, H, W, 32, 16);
        NET_TRY(conv_relu(10, cat, D, H, W, u, st));          // u0
        long long V = 0;
        NET_TRY(conv(11, u, D, H, W, st, &V));                // out (no ReLU)
#undef NET_TRY
        k_decode<<<blocks(cells), TPB, 0, st>>>(y, v, rms, z, cells);
        G2_CUDA_CHECK(cudaGetLastError());
        g2_count_launches(4 + 3 + 2 * 12 + 12);
        calls++;
        return G2_OK;
    }
};

int net_hook(void *user, const void *d_v, void *d_z, long long n, void *stream)
{
    Net *net = reinterpret_cast<Net *>(user);
    if (n != 3LL * net->D * net->H * net->W) return G2_ERR_ARG;
    return net->forward(reinterpret_cast<const double2 *>(d_v), reinterpret_cast<double2 *>(d_z),
                        reinterpret_cast<cudaStream_t>(stream));
}

}  // namespace

// giem2g_set_preconditioner body: kind 0 removes the network, 1 / 2 load it from weights_path and
// register it as the outer hook in mode 1 / 2.  The network's sigma channel comes from the operator's
// anomaly conductivity (Re csiga) and its frequency channel from the operator's omega.
int ie_set_learned_preconditioner(IeOp *op, int kind, const char *weights_path)
{
    if (op->learned) {
        cudaStreamSynchronize(op->stream);
        delete reinterpret_cast<Net *>(op->learned);
        op->learned = nullptr;
    }
    if (kind == 0) {
        op->precond_mode = 0;
        op->precond_fn = nullptr;
        op->precond_user = nullptr;
        return G2_OK;
    }
    if (!op->have_sigma || op->d_csiga == nullptr) {
        g2_set_error_msg("giem2g_set_preconditioner: set the anomaly conductivity first (the network reads log10 sigma)");
        return G2_ERR_STATE;
    }
    const int D = op->Nz, H = op->Ny, W = op->Nx;
    if (D % 8 || H % 8 || W % 8) {
        g2_set_error_msg("giem2g_set_preconditioner: the network needs Nx, Ny, Nz multiples of 8");
        return G2_ERR_UNSUPPORTED;
    }
    std::map<std::string, Array> arr;
    std::string err;
    if (!weights_path || !read_npz(weights_path, arr, err)) {
        g2_set_error_msg("giem2g_set_preconditioner: " + (weights_path ? err : std::string("no weights file")));
        return G2_ERR_ARG;
    }
    Net *net = new Net();
    net->D = D;
    net->H = H;
    net->W = W;
    const long long cells = (long long)D * H * W;
    cudaStream_t st = op->stream;
    auto fail = [&](const std::string &m, int rc) {
        g2_set_error_msg("giem2g_set_preconditioner: " + m);
        delete net;
        return rc;
    };
    for (int l = 0; l < 12; l++) {
        const LayerDef &L = kLayers[l];
        auto it = arr.find(L.name);
        const int kp = kp_of(L.cin);
        if (it == arr.end() || it->second.shape.size() != 2 || it->second.shape[0] != L.cout || it->second.shape[1] != kp)
            return fail(std::string("layer ") + L.name + " missing or of the wrong shape", G2_ERR_ARG);
        float *tmp = nullptr;
        if (cudaMalloc(&net->w[l], sizeof(bf16) * L.cout * kp) != cudaSuccess ||
            cudaMalloc(&tmp, sizeof(float) * L.cout * kp) != cudaSuccess)
            return fail("allocation failed", G2_ERR_NOMEM);
        // stream-ordered upload: a pageable cudaMemcpy may return before its DMA lands, and st is a
        // non-blocking stream that is not ordered after the legacy stream
        cudaMemcpyAsync(tmp, it->second.data.data(), sizeof(float) * L.cout * kp, cudaMemcpyHostToDevice, st);
        k_f32_to_bf16<<<blocks((long long)L.cout * kp), TPB, 0, st>>>(tmp, net->w[l], (long long)L.cout * kp);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            cudaFree(tmp);
            return fail("weight upload failed", G2_ERR_CUDA);
        }
        cudaFree(tmp);
    }
    // model_features (learned.py): (log10 sigma + 2) / 1 with sigma = Re(csiga), log10(f) / 2
    std::vector<double2> cs(cells);
    if (cudaMemcpyAsync(cs.data(), op->d_csiga, cells * sizeof(double2), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail("conductivity download failed", G2_ERR_CUDA);
    std::vector<float> ls(cells);
    for (long long i = 0; i < cells; i++) ls[i] = (float)((std::log10(cs[i].x) + 2.0) / 1.0);
    const double freq = op->omega / (2.0 * 3.14159265358979323846264338327950288);
    net->logf = (float)(std::log10(freq) / 2.0);
    // buffers: activations at full resolution hold at most 48 channels (the u0 input); the largest
    // im2col is u0's (cells x kp(48)); the largest GEMM output is cells x 16
    size_t maxcols = 0;
    {
        long long d = D, h = H, w = W;
        for (int l = 0; l < 12; l++) {
            const LayerDef &L = kLayers[l];
            const long long V = ((d - 1) / L.stride + 1) * ((h - 1) / L.stride + 1) * ((w - 1) / L.stride + 1);
            maxcols = std::max(maxcols, (size_t)V * kp_of(L.cin));
            if (l == 2 || l == 4 || l == 6) { d /= 2; h /= 2; w /= 2; }
            if (l == 7 || l == 8 || l == 9) { d *= 2; h *= 2; w *= 2; }
        }
    }
    net->nb = 148 * 4;
    bool ok = cudaMalloc(&net->logsig, sizeof(float) * cells) == cudaSuccess;
    ok = ok && cudaMalloc(&net->partial, sizeof(double) * net->nb) == cudaSuccess;
    ok = ok && cudaMalloc(&net->rms, sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&net->x0, sizeof(bf16) * cells * 8) == cudaSuccess;
    ok = ok && cudaMalloc(&net->e0, sizeof(bf16) * cells * 16) == cudaSuccess;
    ok = ok && cudaMalloc(&net->e1, sizeof(bf16) * cells / 8 * 32) == cudaSuccess;
    ok = ok && cudaMalloc(&net->e2, sizeof(bf16) * cells / 64 * 64) == cudaSuccess;
    ok = ok && cudaMalloc(&net->t, sizeof(bf16) * cells * 16) == cudaSuccess;
    ok = ok && cudaMalloc(&net->b, sizeof(bf16) * cells / 512 * 64) == cudaSuccess;
    ok = ok && cudaMalloc(&net->u, sizeof(bf16) * cells * 16) == cudaSuccess;
    ok = ok && cudaMalloc(&net->cat, sizeof(bf16) * cells * 48) == cudaSuccess;
    ok = ok && cudaMalloc(&net->cols, sizeof(bf16) * maxcols) == cudaSuccess;
    ok = ok && cudaMalloc(&net->y, sizeof(float) * cells * 16) == cudaSuccess;
    ok = ok && cudaMalloc(&net->d_err, sizeof(int)) == cudaSuccess &&
         cudaMemsetAsync(net->d_err, 0, sizeof(int), st) == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) return fail("allocation failed", G2_ERR_NOMEM);
    if (cudaMemcpyAsync(net->logsig, ls.data(), sizeof(float) * cells, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail("feature upload failed", G2_ERR_CUDA);
    op->learned = net;
    op->precond_mode = kind;
    op->precond_fn = net_hook;
    op->precond_user = net;
    op->config_gen++;
    return G2_OK;
}

// z = v + rms * net(v) once, outside a solve (giem2g_apply_preconditioner); checks the GEMM error word
int ie_learned_apply(IeOp *op, const double2 *d_v, double2 *d_z)
{
    if (!op->learned) {
        g2_set_error_msg("giem2g_apply_preconditioner: no network (giem2g_set_preconditioner)");
        return G2_ERR_STATE;
    }
    Net *net = reinterpret_cast<Net *>(op->learned);
    int rc = net->forward(d_v, d_z, op->stream);
    if (rc) return rc;
    int e = 0;
    G2_CUDA_CHECK(cudaMemcpyAsync(&e, net->d_err, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
    G2_CUDA_CHECK(cudaStreamSynchronize(op->stream));
    if (e) {
        g2_set_error_msg("giem2g_apply_preconditioner: a GEMM wait timed out");
        return G2_ERR_NUMERIC;
    }
    return G2_OK;
}

long long ie_learned_calls(const IeOp *op)
{
    return op->learned ? reinterpret_cast<const Net *>(op->learned)->calls : 0;
}

void ie_free_learned(IeOp *op)
{
    if (op->learned) {
        delete reinterpret_cast<Net *>(op->learned);
        op->learned = nullptr;
    }
}
