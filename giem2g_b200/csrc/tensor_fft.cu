// Spectral transform of the Green's tensor, FP64, on the GPU.
//
// Restates CalcFFTofIETensorGeneral / CALC_FFT_OF_TENSOR_COMPONENT (Integral_Equation_Module.F90:319-471)
// together with the mirrored distributed FFT (Distributed_FFT.F90:384-414, 507-551):
//   - the spatial lags g(lx,ly), lx<Nx, ly<Ny, are extended to a 2Nx x 2Ny circulant with the component
//     parities (sx,sy): xx(+,+) xy(-,-) yy(+,+) zz(+,+) xz(-,+) yz(+,-); lags Nx and Ny are set to zero;
//   - forward 2-D DFT (exp(-i...)), unnormalised;
//   - y-Nyquist correction G(.,ky) -= (-1)^ky G(.,Ny) on every kx, then x-Nyquist correction
//     G(kx,.) -= (-1)^kx G(Nx,.) with the alternating sign starting at +1 for kx = 0;
//   - keep kx<Nx, ky<Ny.
// With these corrections the 2Nx x 2Ny circular convolution restricted to the physical grid is the exact
// block-Toeplitz product, for even Nx and Ny.
// Pass A transforms along x (lines over lx for each (ly, element)), pass B along y with both corrections.
// Elements of a unit are interleaved in shared memory so global loads/stores are coalesced.
#include "common.cuh"
#include "ie_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int TE = 16;  // tensor elements per CTA

G2_D void elem_parity(int e, int P, int Nz, double &sx, double &sy)
{
    if (e < 4 * P) {
        const int comp = e / P;  // xx, xy, yy, zz
        sx = sy = (comp == 1) ? -1.0 : 1.0;
    } else {
        const int comp = (e - 4 * P) / (Nz * Nz);  // xz, yz
        sx = comp == 0 ? -1.0 : 1.0;
        sy = comp == 0 ? 1.0 : -1.0;
    }
}

// position of unit element e in the device layout (full blocks swizzled, see asw)
G2_HD int dev_pos(int e, int P, int Nz, int W)
{
    if (e < 4 * P) return e;
    const int li = e - 4 * P, blk = li / (Nz * Nz), rc = li - blk * Nz * Nz;
    const int r = rc % Nz, c = rc / Nz;
    return 4 * P + blk * Nz * Nz + asw(r, c, Nz, W);
}

// pass A: spatial [lx][ly][T] -> S1 [kx 0..Nx][ly][T]
__global__ void __launch_bounds__(kThreads) k_tensor_x(const double2 *__restrict__ g, double2 *__restrict__ S1,
                                                       const double2 *__restrict__ tw, int Nx, int Ny, int Nz)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *s = reinterpret_cast<double2 *>(smem_raw);
    const int P = Nz * (Nz + 1) / 2, T = 4 * P + 2 * Nz * Nz;
    const int L = 2 * Nx, lg = ilog2(L);
    const int ly = blockIdx.x, e0 = blockIdx.y * TE;
    const int ne = min(TE, T - e0);
    for (int i = threadIdx.x; i < L * TE; i += blockDim.x) s[i] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int i = threadIdx.x; i < Nx * TE; i += blockDim.x) {
        const int lx = i / TE, t = i - lx * TE;
        if (t >= ne) continue;
        double sx, sy;
        elem_parity(e0 + t, P, Nz, sx, sy);
        const double2 v = g[((size_t)lx * Ny + ly) * T + e0 + t];
        s[bitrev(lx, lg) * TE + t] = v;
        if (lx > 0) s[bitrev(L - lx, lg) * TE + t] = make_double2(sx * v.x, sx * v.y);
    }
    __syncthreads();
    smem_fft<double2, true>(s, lg, TE, 1, TE, tw, false);
    for (int i = threadIdx.x; i < (Nx + 1) * TE; i += blockDim.x) {
        const int kx = i / TE, t = i - kx * TE;
        if (t < ne) S1[((size_t)kx * Ny + ly) * T + e0 + t] = s[kx * TE + t];
    }
}

// pass B: S1 [kx][ly][T] -> out [kx][ky][T] (kx < Nx) or nyq [ky][T] (kx == Nx, when corr == nullptr)
__global__ void __launch_bounds__(kThreads) k_tensor_y(const double2 *__restrict__ S1, double2 *__restrict__ out,
                                                       const double2 *__restrict__ nyq, const double2 *__restrict__ tw,
                                                       int Nx, int Ny, int Nz, int kx_base)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *s = reinterpret_cast<double2 *>(smem_raw);
    const int P = Nz * (Nz + 1) / 2, T = 4 * P + 2 * Nz * Nz;
    const int L = 2 * Ny, lg = ilog2(L);
    const int kx = kx_base + blockIdx.x, e0 = blockIdx.y * TE;
    const int ne = min(TE, T - e0);
    for (int i = threadIdx.x; i < L * TE; i += blockDim.x) s[i] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int i = threadIdx.x; i < Ny * TE; i += blockDim.x) {
        const int ly = i / TE, t = i - ly * TE;
        if (t >= ne) continue;
        double sx, sy;
        elem_parity(e0 + t, P, Nz, sx, sy);
        const double2 v = S1[((size_t)kx * Ny + ly) * T + e0 + t];
        s[bitrev(ly, lg) * TE + t] = v;
        if (ly > 0) s[bitrev(L - ly, lg) * TE + t] = make_double2(sy * v.x, sy * v.y);
    }
    __syncthreads();
    smem_fft<double2, true>(s, lg, TE, 1, TE, tw, false);
    for (int i = threadIdx.x; i < Ny * TE; i += blockDim.x) {
        const int ky = i / TE, t = i - ky * TE;
        if (t >= ne) continue;
        const double2 ny = s[Ny * TE + t];
        const double sgn = (ky & 1) ? -1.0 : 1.0;
        double2 v = make_double2(s[ky * TE + t].x - sgn * ny.x, s[ky * TE + t].y - sgn * ny.y);
        if (nyq == nullptr) {
            out[(size_t)ky * T + e0 + t] = v;  // x-Nyquist row (plain layout, scratch)
        } else {
            const double sx = (kx & 1) ? -1.0 : 1.0;
            const double2 c = nyq[(size_t)ky * T + e0 + t];
            out[((size_t)kx * Ny + ky) * T + dev_pos(e0 + t, P, Nz, asw_width64(Nz))] =
                make_double2(v.x - sx * c.x, v.y - sx * c.y);
        }
    }
}

// complex64 copy; the full blocks move from the FP64 swizzle to the FP32 swizzle
__global__ void k_to_c64(const double2 *__restrict__ a, float2 *__restrict__ b, size_t units, int P, int Nz)
{
    const int T = 4 * P + 2 * Nz * Nz, W64 = asw_width64(Nz), W32 = asw_width32(Nz);
    const size_t n = units * T;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t u = i / T;
        const int e = (int)(i - u * T);
        const double2 v = a[u * T + dev_pos(e, P, Nz, W64)];
        b[u * T + dev_pos(e, P, Nz, W32)] = make_float2((float)v.x, (float)v.y);
    }
}

}  // namespace

int ie_tensor_spectrum(IeOp *op, cudaStream_t st)
{
    const int Nx = op->Nx, Ny = op->Ny, Nz = op->Nz, T = op->Tunit();
    if (!op->d_spatial) return G2_ERR_STATE;
    const size_t n_out = op->units() * T;
    double2 *S1 = nullptr, *nyq = nullptr;
    G2_CUDA_CHECK(cudaMalloc(&S1, (size_t)(Nx + 1) * Ny * T * sizeof(double2)));
    G2_CUDA_CHECK(cudaMalloc(&nyq, (size_t)Ny * T * sizeof(double2)));
    if (!op->d_tensor64) G2_CUDA_CHECK(cudaMalloc(&op->d_tensor64, n_out * sizeof(double2)));
    if (!op->d_tensor32) G2_CUDA_CHECK(cudaMalloc(&op->d_tensor32, n_out * sizeof(float2)));
    const size_t smx = (size_t)2 * Nx * TE * sizeof(double2), smy = (size_t)2 * Ny * TE * sizeof(double2);
    G2_CUDA_CHECK(cudaFuncSetAttribute(k_tensor_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    G2_CUDA_CHECK(cudaFuncSetAttribute(k_tensor_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    const int eb = (T + TE - 1) / TE;
    k_tensor_x<<<dim3(Ny, eb), kThreads, smx, st>>>(op->d_spatial, S1, op->d_twx64, Nx, Ny, Nz);
    k_tensor_y<<<dim3(1, eb), kThreads, smy, st>>>(S1, nyq, nullptr, op->d_twy64, Nx, Ny, Nz, Nx);
    k_tensor_y<<<dim3(Nx, eb), kThreads, smy, st>>>(S1, op->d_tensor64, nyq, op->d_twy64, Nx, Ny, Nz, 0);
    k_to_c64<<<1184, 256, 0, st>>>(op->d_tensor64, op->d_tensor32, op->units(), op->P(), Nz);
    G2_CUDA_CHECK(cudaGetLastError());
    G2_CUDA_CHECK(cudaStreamSynchronize(st));
    cudaFree(S1);
    cudaFree(nyq);
    // the reference transforms the kernel buffer in place (G_symm and G_symmT alias it), so the
    // spatial tensor does not outlive the transform there either
    cudaFree(op->d_spatial);
    op->d_spatial = nullptr;
    op->have_spatial = false;
    return G2_OK;
}
