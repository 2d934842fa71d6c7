// C ABI: the reference's giem2g_* entry points (giem2g_interfaces.F90:76-254) plus extensions.
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include "common.cuh"
#include "ie_internal.h"
#include "krylov.h"
#include "rc_internal.h"

namespace {
std::mutex g_mu;
std::string g_last_error;
int g_last_status = 0;
void (*g_logger)(const char *) = nullptr;
IeOp *g_last_op = nullptr;  // giem2g_interfaces.F90:69 keeps the last operator in tmp_ptr

int set_status(int rc)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_status = rc;
    if (rc == 0) g_last_error.clear();
    return rc;
}
IeOp *resolve(void *ie)
{
    // The reference's set_anomaly_conductivity/apply ignore their handle and use the last
    // operator (giem2g_interfaces.F90:196,212); a NULL handle selects that one here.
    return ie ? reinterpret_cast<IeOp *>(ie) : g_last_op;
}
bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// data_types_module.F90:214-242 GetLayerSingle; depth[1..Nl-1]
int get_layer(double z, int Nl, const std::vector<double> &depth)
{
    if (std::fabs(z) < 1e-15) return 0;
    if (z < 0) return -1;
    if (Nl == 1) return 1;
    int l = 1;
    if (z > depth[Nl - 1]) return Nl;
    while (z > depth[l]) l++;
    return l;
}
}  // namespace

static std::atomic<long long> g_launches{0};
void g2_count_launches(int n) { g_launches += n; }
long long g2_launch_total() { return g_launches.load(); }

void g2_log(const char *msg)
{
    if (g_logger) g_logger(msg);
    else std::fprintf(stdout, "%s\n", msg);
}
void g2_set_error_msg(const std::string &msg)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_last_error = msg;
}
void g2_set_error(const char *file, int line, const char *msg)
{
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s:%d: %s", file, line, msg);
    g2_set_error_msg(buf);
}

static int fail(int rc, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g2_set_error_msg(buf);
    return set_status(rc);
}

extern "C" {

int giem2g_last_status(void) { return g_last_status; }
long long giem2g_kernel_launch_count(void) { return g_launches.load(); }
const char *giem2g_last_error(void) { return g_last_error.c_str(); }

void giem2g_calc_data_sizes(GIEM2G_ANOMALY_TYPE anomaly, GIEM2G_DATA_TYPE *data)
{
    if (!data || anomaly.Nx <= 0 || anomaly.Ny <= 0 || anomaly.Nz <= 0) {
        fail(G2_ERR_ARG, "giem2g_calc_data_sizes: bad anomaly shape");
        return;
    }
    const long long Nx = anomaly.Nx, Ny = anomaly.Ny, Nz = anomaly.Nz;
    data->tensor_size = (long long)sizeof(IeOp) / 8;
    // CalcLocalKernelSize with every lag on one process (Integral_Equation_Module.F90:105-129)
    data->ie_kernel_buffer_length = (2 * Nz * (Nz + 1) + 2 * Nz * Nz) * Nx * Ny;
    // CalcLocalFFTSize(2Nx,2Ny,3Nz,1) (Distributed_FFT.F90:895-912)
    data->fft_buffers_length = 2 * Nx * 3 * Nz * 2 * Ny;
    IeOp *op = new IeOp();
    op->Nx = anomaly.Nx;
    op->Ny = anomaly.Ny;
    op->Nz = anomaly.Nz;
    g_last_op = op;
    data->giem2g_tensor = op;
    set_status(0);
}

void giem2g_prepare_ie_kernel(GIEM2G_ANOMALY_TYPE anomaly, GIEM2G_DATA_TYPE data)
{
    IeOp *op = reinterpret_cast<IeOp *>(data.giem2g_tensor);
    if (!op) { fail(G2_ERR_ARG, "giem2g_prepare_ie_kernel: no operator (call giem2g_calc_data_sizes first)"); return; }
    const int Nx = anomaly.Nx, Ny = anomaly.Ny, Nz = anomaly.Nz;
    if (!is_pow2(2 * Nx) || !is_pow2(2 * Ny) || 2 * Nx < 4 || 2 * Ny < 4 || 2 * Nx > 1024 || 2 * Ny > 1024) {
        fail(G2_ERR_UNSUPPORTED, "giem2g_prepare_ie_kernel: 2*Nx and 2*Ny must be powers of two in [4,1024] (got Nx=%d Ny=%d)", Nx, Ny);
        return;
    }
    const int Tmax_c128 = (227 * 1024) / 16 - 12 * Nz;
    if (Nz < 1 || 2 * Nz * (2 * Nz + 1) > Tmax_c128) {
        fail(G2_ERR_UNSUPPORTED, "giem2g_prepare_ie_kernel: Nz=%d exceeds the contraction tile limit", Nz);
        return;
    }
    if (!anomaly.z) { fail(G2_ERR_ARG, "giem2g_prepare_ie_kernel: z is NULL"); return; }
    op->Nx = Nx;
    op->Ny = Ny;
    op->Nz = Nz;
    op->dx = anomaly.dx;
    op->dy = anomaly.dy;
    const double *z = reinterpret_cast<const double *>(anomaly.z);
    op->z.assign(z, z + Nz + 1);
    op->dz.resize(Nz);
    for (int i = 0; i < Nz; i++) op->dz[i] = anomaly.dz ? reinterpret_cast<const double *>(anomaly.dz)[i] : z[i + 1] - z[i];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { fail(G2_ERR_CUDA, "no CUDA device"); return; }
    if (!op->stream && cudaStreamCreateWithFlags(&op->stream, cudaStreamNonBlocking) != cudaSuccess) {
        fail(G2_ERR_CUDA, "cudaStreamCreate failed");
        return;
    }
    cudaEventCreate(&op->ev0);
    cudaEventCreate(&op->ev1);
    cudaEventCreate(&op->evc0);
    cudaEventCreate(&op->evc1);
    {
        const char *gen = std::getenv("GIEM2G_GENERIC_CONTRACT");
        op->use_fast_contract = !(gen && gen[0] == '1');
    }
    int rc = ie_make_twiddles(op);
    if (!rc) rc = ie_alloc_scratch(op);
    if (!rc && !op->d_err) {
        if (cudaMalloc(&op->d_err, sizeof(int)) != cudaSuccess || cudaMemset(op->d_err, 0, sizeof(int)) != cudaSuccess ||
            cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess)
            rc = G2_ERR_NOMEM;
    }
    if (!rc && !op->d_csiga && cudaMalloc(&op->d_csiga, op->cells() * sizeof(double2)) != cudaSuccess) rc = G2_ERR_NOMEM;
    if (!rc && !op->d_vin) {
        if (cudaMalloc(&op->d_vin, op->nvec() * sizeof(double2)) != cudaSuccess ||
            cudaMalloc(&op->d_vout, op->nvec() * sizeof(double2)) != cudaSuccess)
            rc = G2_ERR_NOMEM;
    }
    if (rc) { fail(rc, "giem2g_prepare_ie_kernel: allocation failed (%s)", giem2g_last_error()); return; }
    g_last_op = op;
    set_status(0);
}

int giem2g_set_background(void *ie, GIEM2G_BACKGROUND_TYPE bkg, double omega)
{
    IeOp *op = resolve(ie);
    if (!op || op->z.empty()) return fail(G2_ERR_STATE, "giem2g_set_background: operator not prepared");
    if (bkg.Nl < 1 || !bkg.csigb || (bkg.Nl > 1 && !bkg.thickness)) return fail(G2_ERR_ARG, "giem2g_set_background: bad background");
    op->Nl = bkg.Nl;
    const double2 *cs = reinterpret_cast<const double2 *>(bkg.csigb);
    op->csigma.assign(cs, cs + bkg.Nl + 1);
    op->thick.clear();
    if (bkg.Nl > 1) {
        const double *th = reinterpret_cast<const double *>(bkg.thickness);
        op->thick.assign(th, th + bkg.Nl - 1);
    }
    op->omega = omega;
    // CREATE_BACKGROUND depth (giem2g_interfaces.F90:264-268), Lnumber (:163-165)
    std::vector<double> depth(bkg.Nl + 1, 0.0);
    if (bkg.Nl > 1) {
        depth[1] = op->thick[0];
        for (int i = 2; i <= bkg.Nl - 1; i++) depth[i] = depth[i - 1] + op->thick[i - 1];
    }
    const int Nz = op->Nz;
    op->Lnumber.assign(Nz + 1, 0);
    for (int i = 1; i <= Nz; i++) op->Lnumber[i] = get_layer((op->z[i - 1] + op->z[i]) / 2.0, bkg.Nl, depth);
    op->Lnumber[0] = get_layer(op->z[0] * (1.0 - 1e-7), bkg.Nl, depth);
    op->csigb.resize(Nz);
    op->sqsigb.resize(Nz);
    for (int iz = 1; iz <= Nz; iz++) {
        const int l = op->Lnumber[iz];
        if (l < 1) return fail(G2_ERR_ARG, "giem2g_set_background: anomaly cell %d is not below the surface", iz);
        op->csigb[iz - 1] = op->csigma[l];
        op->sqsigb[iz - 1] = std::sqrt(op->csigma[l].x);  // PreparePreconditioner (calc_ie_tensor_module.F90:303)
    }
    op->have_background = true;
    if (op->have_sigma) {
        int rc = ie_prepare_sigma(op, op->stream);
        if (rc) return set_status(rc);
    }
    return set_status(0);
}

void giem2g_calc_ie_kernel(void *ie, GIEM2G_BACKGROUND_TYPE bkg, GIEM2G_ANOMALY_TYPE anomaly, double omega)
{
    IeOp *op = resolve(ie);
    if (!op) { fail(G2_ERR_STATE, "giem2g_calc_ie_kernel: no operator"); return; }
    if (anomaly.Nx != op->Nx || anomaly.Ny != op->Ny || anomaly.Nz != op->Nz) {
        fail(G2_ERR_ARG, "giem2g_calc_ie_kernel: anomaly shape differs from the prepared operator");
        return;
    }
    op->dx = anomaly.dx;
    op->dy = anomaly.dy;
    if (giem2g_set_background(op, bkg, omega)) return;
    int rc = ie_green_tensor(op, op->stream);
    if (rc) { fail(rc, "giem2g_calc_ie_kernel: %s", giem2g_last_error()); return; }
    op->have_spatial = true;
    op->have_spectral = false;
    set_status(0);
}

int giem2g_set_ie_kernel_spatial(void *ie, const void *symm, const void *asym)
{
    IeOp *op = resolve(ie);
    if (!op || op->z.empty()) return fail(G2_ERR_STATE, "giem2g_set_ie_kernel_spatial: operator not prepared");
    const int P = op->P(), Nz = op->Nz, T = op->Tunit();
    const size_t U = op->units();
    if (!op->d_spatial && cudaMalloc(&op->d_spatial, U * T * sizeof(double2)) != cudaSuccess)
        return fail(G2_ERR_NOMEM, "giem2g_set_ie_kernel_spatial: cudaMalloc failed");
    std::vector<double2> h(U * T);
    const double2 *s = reinterpret_cast<const double2 *>(symm), *a = reinterpret_cast<const double2 *>(asym);
    for (size_t u = 0; u < U; u++) {
        std::memcpy(&h[u * T], s + u * 4 * P, sizeof(double2) * 4 * P);
        std::memcpy(&h[u * T + 4 * P], a + u * 2 * Nz * Nz, sizeof(double2) * 2 * Nz * Nz);
    }
    // stream-ordered: the transform that follows runs on the operator's (non-blocking) stream
    if (cudaMemcpyAsync(op->d_spatial, h.data(), U * T * sizeof(double2), cudaMemcpyHostToDevice, op->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(op->stream) != cudaSuccess)
        return fail(G2_ERR_CUDA, "giem2g_set_ie_kernel_spatial: copy failed");
    op->have_spatial = true;
    op->have_spectral = false;
    return set_status(0);
}

static int get_units(IeOp *op, const double2 *d, void *symm, void *asym, int W = 1)
{
    const int P = op->P(), Nz = op->Nz, T = op->Tunit();
    const size_t U = op->units();
    std::vector<double2> h(U * T);
    if (cudaMemcpyAsync(h.data(), d, U * T * sizeof(double2), cudaMemcpyDeviceToHost, op->stream) != cudaSuccess ||
        cudaStreamSynchronize(op->stream) != cudaSuccess)
        return fail(G2_ERR_CUDA, "tensor download failed");
    double2 *s = reinterpret_cast<double2 *>(symm), *a = reinterpret_cast<double2 *>(asym);
    for (size_t u = 0; u < U; u++) {
        std::memcpy(s + u * 4 * P, &h[u * T], sizeof(double2) * 4 * P);
        for (int blk = 0; blk < 2; blk++)
            for (int c = 0; c < Nz; c++)
                for (int r = 0; r < Nz; r++)
                    a[u * 2 * Nz * Nz + blk * Nz * Nz + c * Nz + r] = h[u * T + 4 * P + blk * Nz * Nz + asw(r, c, Nz, W)];
    }
    return set_status(0);
}

int giem2g_get_ie_kernel_spatial(void *ie, void *symm, void *asym)
{
    IeOp *op = resolve(ie);
    if (!op || !op->have_spatial) return fail(G2_ERR_STATE, "giem2g_get_ie_kernel_spatial: no spatial tensor");
    return get_units(op, op->d_spatial, symm, asym);
}

int giem2g_get_ie_kernel_spectral(void *ie, void *symm, void *asym)
{
    IeOp *op = resolve(ie);
    if (!op || !op->have_spectral) return fail(G2_ERR_STATE, "giem2g_get_ie_kernel_spectral: no spectral tensor");
    return get_units(op, op->d_tensor64, symm, asym, asw_width64(op->Nz));
}

void giem2g_calc_fft_of_ie_kernel(void *ie)
{
    IeOp *op = resolve(ie);
    if (!op || !op->have_spatial) { fail(G2_ERR_STATE, "giem2g_calc_fft_of_ie_kernel: no spatial tensor"); return; }
    int rc = ie_tensor_spectrum(op, op->stream);
    if (rc) { fail(rc, "giem2g_calc_fft_of_ie_kernel: %s", giem2g_last_error()); return; }
    op->have_spectral = true;
    set_status(0);
}

void giem2g_set_anomaly_conductivity(void *ie, void *csiga)
{
    IeOp *op = resolve(ie);
    if (!op || !op->d_csiga) { fail(G2_ERR_STATE, "giem2g_set_anomaly_conductivity: operator not prepared"); return; }
    if (!csiga) { fail(G2_ERR_ARG, "giem2g_set_anomaly_conductivity: csiga is NULL"); return; }
    if (cudaMemcpyAsync(op->d_csiga, csiga, op->cells() * sizeof(double2), cudaMemcpyHostToDevice, op->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(op->stream) != cudaSuccess) {
        fail(G2_ERR_CUDA, "giem2g_set_anomaly_conductivity: copy failed");
        return;
    }
    op->have_sigma = true;
    if (op->have_background) {
        int rc = ie_prepare_sigma(op, op->stream);
        if (rc) { fail(rc, "giem2g_set_anomaly_conductivity: %s", giem2g_last_error()); return; }
    }
    set_status(0);
}

static int check_ready(IeOp *op, const char *who)
{
    if (!op) return fail(G2_ERR_STATE, "%s: no operator", who);
    if (!op->have_spectral) return fail(G2_ERR_STATE, "%s: spectral tensor missing (giem2g_calc_fft_of_ie_kernel)", who);
    if (!op->have_sigma || !op->have_background) return fail(G2_ERR_STATE, "%s: conductivity/background missing", who);
    return 0;
}

int giem2g_apply_ie_operator_device(void *ie, const void *d_in, void *d_out, int precision)
{
    IeOp *op = resolve(ie);
    int rc = check_ready(op, "giem2g_apply_ie_operator_device");
    if (rc) return rc;
    if (precision != 0 && precision != 1)
        return fail(G2_ERR_ARG, "giem2g_apply_ie_operator_device: precision must be 0 or 1");
    cudaEventRecord(op->ev0, op->stream);
    if (precision == 0)
        rc = ie_apply_device64(op, reinterpret_cast<const double2 *>(d_in), reinterpret_cast<double2 *>(d_out), op->stream);
    else
        rc = ie_apply_device32(op, reinterpret_cast<const float2 *>(d_in), reinterpret_cast<float2 *>(d_out), op->stream);
    cudaEventRecord(op->ev1, op->stream);
    op->last_kernel_launches = ie_kernel_launch_count_apply(op, precision == 0 ? 0 : 1);
    op->mult_num++;
    if (rc) return fail(rc, "giem2g_apply_ie_operator_device: %s", giem2g_last_error());
    return set_status(0);
}

// Same result as giem2g_apply_ie_operator_device, with the apply's intermediates in the library's
// static device array (static_scratch.cu) instead of the operator's buffers: the call allocates
// nothing.  Rejects grids whose intermediates exceed the array.
int giem2g_apply_ie_operator_device_static(void *ie, const void *d_in, void *d_out, int precision)
{
    IeOp *op = resolve(ie);
    int rc = check_ready(op, "giem2g_apply_ie_operator_device_static");
    if (rc) return rc;
    if (precision != 0 && precision != 1)
        return fail(G2_ERR_ARG, "giem2g_apply_ie_operator_device_static: precision must be 0 or 1");
    void *base = nullptr;
    size_t cap = 0, n_u1 = 0;
    rc = ie_static_scratch(&base, &cap);
    if (rc) return fail(rc, "giem2g_apply_ie_operator_device_static: static scratch set-up failed: %s",
                        giem2g_last_error());
    const size_t es = precision == 0 ? sizeof(double2) : sizeof(float2);
    const size_t n_all = ie_apply_scratch_elems(op, &n_u1);
    const size_t off_uh = (n_u1 * es + 255) / 256 * 256;
    const size_t need = off_uh + (n_all - n_u1) * es;
    if (need > cap)
        return fail(G2_ERR_ARG,
                    "giem2g_apply_ie_operator_device_static: grid %dx%dx%d needs %zu bytes of scratch at precision "
                    "%d, above the static maximum of %zu bytes; use giem2g_apply_ie_operator_device",
                    op->Nx, op->Ny, op->Nz, need, precision, cap);
    unsigned char *b = static_cast<unsigned char *>(base);
    cudaEventRecord(op->ev0, op->stream);
    if (precision == 0)
        rc = ie_apply_device64_scratch(op, reinterpret_cast<const double2 *>(d_in), reinterpret_cast<double2 *>(d_out),
                                       op->stream, reinterpret_cast<double2 *>(b),
                                       reinterpret_cast<double2 *>(b + off_uh));
    else
        rc = ie_apply_device32_scratch(op, reinterpret_cast<const float2 *>(d_in), reinterpret_cast<float2 *>(d_out),
                                       op->stream, reinterpret_cast<float2 *>(b), reinterpret_cast<float2 *>(b + off_uh));
    cudaEventRecord(op->ev1, op->stream);
    op->last_kernel_launches = ie_kernel_launch_count_apply(op, precision == 0 ? 0 : 1);
    op->mult_num++;
    if (rc) return fail(rc, "giem2g_apply_ie_operator_device_static: %s", giem2g_last_error());
    return set_status(0);
}

void giem2g_apply_ie_operator(void *ie, void *in, void *out)
{
    // apply_ie_operator_module.F90:39 via giem2g_interfaces.F90:203-232: host vectors in/out
    IeOp *op = resolve(ie);
    if (check_ready(op, "giem2g_apply_ie_operator")) return;
    const size_t nb = op->nvec() * sizeof(double2);
    cudaMemcpyAsync(op->d_vin, in, nb, cudaMemcpyHostToDevice, op->stream);
    int rc;
    if (op->precision_mode == 1) {  // giem2g_set_precision(ie, 1)
        cudaEventRecord(op->ev0, op->stream);
        rc = ie_apply_host_mixed(op, op->d_vin, op->d_vout, op->stream);
        cudaEventRecord(op->ev1, op->stream);
        op->mult_num++;
        if (rc) { fail(rc, "giem2g_apply_ie_operator: %s", giem2g_last_error()); return; }
    } else {
        rc = giem2g_apply_ie_operator_device(op, op->d_vin, op->d_vout, 0);
    }
    if (rc) return;
    cudaMemcpyAsync(out, op->d_vout, nb, cudaMemcpyDeviceToHost, op->stream);
    if (cudaStreamSynchronize(op->stream) != cudaSuccess) { fail(G2_ERR_CUDA, "giem2g_apply_ie_operator: %s", cudaGetErrorString(cudaGetLastError())); return; }
    if (ie_check_device_error(op)) return;
    float ms = 0;
    cudaEventElapsedTime(&ms, op->ev0, op->ev1);
    op->apply_seconds += ms * 1e-3;
    set_status(0);
}

int giem2g_set_preconditioner(void *ie, int kind, const char *weights_path)
{
    IeOp *op = resolve(ie);
    if (!op) return fail(G2_ERR_STATE, "giem2g_set_preconditioner: no operator");
    if (kind < 0 || kind > 2) return fail(G2_ERR_ARG, "giem2g_set_preconditioner: kind must be 0, 1 or 2");
    const int rc = ie_set_learned_preconditioner(op, kind, weights_path);
    if (rc) return set_status(rc);
    return set_status(0);
}

int giem2g_apply_preconditioner(void *ie, const void *d_v, void *d_z)
{
    IeOp *op = resolve(ie);
    if (!op || !d_v || !d_z) return fail(G2_ERR_ARG, "giem2g_apply_preconditioner: null argument");
    return set_status(ie_learned_apply(op, reinterpret_cast<const double2 *>(d_v), reinterpret_cast<double2 *>(d_z)));
}

long long giem2g_preconditioner_calls(void *ie)
{
    IeOp *op = resolve(ie);
    return op ? ie_learned_calls(op) : 0;
}

int giem2g_set_precision(void *ie, int mode)
{
    IeOp *op = resolve(ie);
    if (!op) return fail(G2_ERR_STATE, "giem2g_set_precision: no operator");
    if (mode != 0 && mode != 1) return fail(G2_ERR_ARG, "giem2g_set_precision: mode must be 0 or 1");
    op->precision_mode = mode;
    return set_status(0);
}

static GIEM2G_FGMRES_CTL resolve_precision(const IeOp *op, GIEM2G_FGMRES_CTL ctl)
{
    if (ctl.precision < 0) ctl.precision = op->precision_mode;
    return ctl;
}

// Variants [0, n) are the separate-pass contraction shapes (k_fy, contraction, k_by); where the fused pass
// exists, variants [n, n + ie_ypipe_variants) select it with its own shapes instead.
static int n_contract(const IeOp *op, int precision)
{
    return precision == 2 ? ie_contract_pair_variants(op->Nz) : ie_contract_variants(precision, op->Nz);
}
static int n_ypipe(const IeOp *op, int precision)
{
    return ie_ypipe_supported(op->Nx, op->Ny, op->Nz) ? ie_ypipe_variants(precision) : 0;
}

int giem2g_set_contract_variant(void *ie, int precision, int variant)
{
    IeOp *op = resolve(ie);
    if (!op || precision < 0 || precision > 2) return fail(G2_ERR_ARG, "giem2g_set_contract_variant: bad arguments");
    const int n = n_contract(op, precision), ny = n_ypipe(op, precision);
    if (variant < 0 || (variant > 0 && variant >= n + ny))
        return fail(G2_ERR_ARG, "giem2g_set_contract_variant: variant %d of %d", variant, n + ny);
    if (variant >= n && ny > 0) {
        op->ypipe_mode[precision] = variant - n;
    } else {
        op->contract_variant[precision] = variant;
        op->ypipe_mode[precision] = -1;
    }
    op->config_gen++;
    return set_status(0);
}

int giem2g_set_kernel_timing(void *ie, int on)
{
    IeOp *op = resolve(ie);
    if (!op) return fail(G2_ERR_STATE, "giem2g_set_kernel_timing: no operator");
    op->time_contract = on != 0;
    return set_status(0);
}

double giem2g_last_contract_ms(void *ie)
{
    IeOp *op = resolve(ie);
    if (!op || !op->time_contract || cudaEventSynchronize(op->evc1) != cudaSuccess) return -1.0;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, op->evc0, op->evc1) != cudaSuccess) return -1.0;
    return ms;
}

int giem2g_set_fft_lines(void *ie, int lines)
{
    IeOp *op = resolve(ie);
    if (!op || (lines != 4 && lines != 8 && lines != 16 && lines != 32))
        return fail(G2_ERR_ARG, "giem2g_set_fft_lines: lines must be 4, 8, 16 or 32");
    op->fft_lines[0] = op->fft_lines[1] = lines;
    op->config_gen++;
    return set_status(0);
}

int giem2g_set_fft_lines_precision(void *ie, int precision, int lines)
{
    IeOp *op = resolve(ie);
    if (!op || (precision != 0 && precision != 1) || (lines != 4 && lines != 8 && lines != 16 && lines != 32))
        return fail(G2_ERR_ARG, "giem2g_set_fft_lines_precision: precision 0 or 1, lines 4, 8, 16 or 32");
    op->fft_lines[precision] = lines;
    op->config_gen++;
    return set_status(0);
}

int giem2g_contract_variants(void *ie, int precision)
{
    IeOp *op = resolve(ie);
    if (!op || precision < 0 || precision > 2) return 0;
    return n_contract(op, precision) + n_ypipe(op, precision);
}

int giem2g_check_device_error(void *ie)
{
    IeOp *op = resolve(ie);
    if (!op) return fail(G2_ERR_STATE, "giem2g_check_device_error: no operator");
    if (cudaStreamSynchronize(op->stream) != cudaSuccess) return fail(G2_ERR_CUDA, "%s", cudaGetErrorString(cudaGetLastError()));
    int rc = ie_check_device_error(op);
    return rc ? rc : set_status(0);
}

int giem2g_solve_device(void *ie, const void *d_Ebkg, void *d_Esol, const void *d_E0, GIEM2G_FGMRES_CTL ctl,
                        GIEM2G_RESULT *info)
{
    IeOp *op = resolve(ie);
    int rc = check_ready(op, "giem2g_solve_device");
    if (rc) return rc;
    if (!d_Ebkg || !d_Esol || !info) return fail(G2_ERR_ARG, "giem2g_solve_device: NULL argument");
    rc = krylov_solve_device(op, reinterpret_cast<const double2 *>(d_Ebkg), reinterpret_cast<double2 *>(d_Esol),
                             reinterpret_cast<const double2 *>(d_E0), resolve_precision(op, ctl), info);
    if (rc) return fail(rc, "giem2g_solve_device: %s", giem2g_last_error());
    return set_status(0);
}

int giem2g_solve(void *ie, const void *E_bkg, void *Esol, const void *E0, GIEM2G_FGMRES_CTL ctl, GIEM2G_RESULT *info)
{
    // SolveEquation (ie_solver_module.F90:43-114) with host arrays
    IeOp *op = resolve(ie);
    int rc = check_ready(op, "giem2g_solve");
    if (rc) return rc;
    if (!E_bkg || !Esol || !info) return fail(G2_ERR_ARG, "giem2g_solve: NULL argument");
    const size_t nb = op->nvec() * sizeof(double2);
    double2 *d_e0 = nullptr;
    if (cudaMemcpyAsync(op->d_vin, E_bkg, nb, cudaMemcpyHostToDevice, op->stream) != cudaSuccess)
        return fail(G2_ERR_CUDA, "giem2g_solve: copy failed");
    if (E0) {
        if (cudaMalloc(&d_e0, nb) != cudaSuccess) return fail(G2_ERR_NOMEM, "giem2g_solve: cudaMalloc failed");
        cudaMemcpyAsync(d_e0, E0, nb, cudaMemcpyHostToDevice, op->stream);
    }
    rc = krylov_solve_device(op, op->d_vin, op->d_vout, d_e0, resolve_precision(op, ctl), info);
    if (d_e0) cudaFree(d_e0);
    if (rc) return fail(rc, "giem2g_solve: %s", giem2g_last_error());
    if (cudaMemcpyAsync(Esol, op->d_vout, nb, cudaMemcpyDeviceToHost, op->stream) != cudaSuccess ||
        cudaStreamSynchronize(op->stream) != cudaSuccess)
        return fail(G2_ERR_CUDA, "giem2g_solve: copy back failed");
    return set_status(0);
}

void *giem2g_batch_create(void *const *ies, int n, GIEM2G_FGMRES_CTL ctl)
{
    if (!ies || n < 1) { fail(G2_ERR_ARG, "giem2g_batch_create: no operators"); return nullptr; }
    std::vector<IeOp *> ops(n);
    for (int i = 0; i < n; i++) {
        ops[i] = resolve(ies[i]);
        if (check_ready(ops[i], "giem2g_batch_create")) return nullptr;
    }
    void *b = nullptr;
    if (ctl.precision < 0) ctl.precision = ops[0]->precision_mode;
    const int rc = batch_create(ops.data(), n, ctl.fgmres_buf, ctl.gmres_buf, ctl.precision, &b);
    if (rc) { fail(rc, "giem2g_batch_create: %s", giem2g_last_error()); return nullptr; }
    set_status(0);
    return b;
}

int giem2g_batch_solve_device(void *batch, const void *const *d_Ebkg, void *const *d_Esol, const void *const *d_E0,
                              GIEM2G_FGMRES_CTL ctl, GIEM2G_RESULT *info)
{
    if (!batch || !d_Ebkg || !d_Esol || !info) return fail(G2_ERR_ARG, "giem2g_batch_solve_device: NULL argument");
    const int rc = batch_solve_device(batch, reinterpret_cast<const double2 *const *>(d_Ebkg),
                                      reinterpret_cast<double2 *const *>(d_Esol),
                                      reinterpret_cast<const double2 *const *>(d_E0), ctl, info);
    if (rc) return fail(rc, "giem2g_batch_solve_device: %s", giem2g_last_error());
    return set_status(0);
}

int giem2g_solve_batched(void *batch, const void *const *E_bkg, void *const *Esol, const void *const *E0,
                         GIEM2G_FGMRES_CTL ctl, GIEM2G_RESULT *info)
{
    // host arrays: every E_bkg[i] (and E0[i]) is copied in, every Esol[i] copied out
    if (!batch || !E_bkg || !Esol || !info) return fail(G2_ERR_ARG, "giem2g_solve_batched: NULL argument");
    double2 *stage = nullptr;
    size_t N = 0;
    int rc = batch_stage(batch, &stage, &N);
    if (rc) return fail(rc, "giem2g_solve_batched: %s", giem2g_last_error());
    const int n = batch_size(batch);
    cudaStream_t st = batch_op(batch, 0)->stream;
    std::vector<const double2 *> in(n), e0(n, nullptr);
    std::vector<double2 *> out(n);
    for (int i = 0; i < n; i++) {
        const size_t nb = batch_op(batch, i)->nvec() * sizeof(double2);
        in[i] = stage + (size_t)i * N;
        out[i] = stage + (size_t)(n + i) * N;
        if (cudaMemcpyAsync(const_cast<double2 *>(in[i]), E_bkg[i], nb, cudaMemcpyHostToDevice, st) != cudaSuccess)
            return fail(G2_ERR_CUDA, "giem2g_solve_batched: copy failed");
        if (E0 && E0[i]) {
            e0[i] = stage + (size_t)(2 * n + i) * N;
            if (cudaMemcpyAsync(const_cast<double2 *>(e0[i]), E0[i], nb, cudaMemcpyHostToDevice, st) != cudaSuccess)
                return fail(G2_ERR_CUDA, "giem2g_solve_batched: copy failed");
        }
    }
    rc = batch_solve_device(batch, in.data(), out.data(), e0.data(), ctl, info);
    if (rc) return fail(rc, "giem2g_solve_batched: %s", giem2g_last_error());
    for (int i = 0; i < n; i++) {
        if (cudaMemcpyAsync(Esol[i], out[i], batch_op(batch, i)->nvec() * sizeof(double2), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess)
            return fail(G2_ERR_CUDA, "giem2g_solve_batched: copy back failed");
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(G2_ERR_CUDA, "giem2g_solve_batched: sync failed");
    return set_status(0);
}

int giem2g_batch_misfit_history(void *batch, int i, double *out, int max_len)
{
    if (!batch || !out) return 0;
    return batch_history(batch, i, out, max_len);
}

void giem2g_batch_delete(void *batch)
{
    batch_free(batch);
    set_status(0);
}

int giem2g_apply_ie_operator_device_batch(void *ie, int nv, const void *const *d_in, void *const *d_out, int precision)
{
    IeOp *op = resolve(ie);
    int rc = check_ready(op, "giem2g_apply_ie_operator_device_batch");
    if (rc) return rc;
    if (nv < 1 || !d_in || !d_out || (precision != 0 && precision != 1))
        return fail(G2_ERR_ARG, "giem2g_apply_ie_operator_device_batch: bad arguments");
    cudaEventRecord(op->ev0, op->stream);
    int i = 0;
    if (precision == 1) {
        float2 *U1 = nullptr, *Uh = nullptr;
        for (; i + 1 < nv; i += 2) {
            if (!U1 && (rc = ie_pair_scratch(op, &U1, &Uh)))
                return fail(rc, "giem2g_apply_ie_operator_device_batch: %s", giem2g_last_error());
            rc = ie_apply_pair32(op, reinterpret_cast<const float2 *>(d_in[i]), reinterpret_cast<const float2 *>(d_in[i + 1]),
                                 reinterpret_cast<float2 *>(d_out[i]), reinterpret_cast<float2 *>(d_out[i + 1]), op->stream,
                                 U1, Uh);
            if (rc == G2_ERR_UNSUPPORTED) break;
            if (rc) return fail(rc, "giem2g_apply_ie_operator_device_batch: %s", giem2g_last_error());
            op->mult_num += 2;
        }
    }
    for (; i < nv; i++) {
        if (precision == 0)
            rc = ie_apply_device64(op, reinterpret_cast<const double2 *>(d_in[i]), reinterpret_cast<double2 *>(d_out[i]),
                                   op->stream);
        else
            rc = ie_apply_device32(op, reinterpret_cast<const float2 *>(d_in[i]), reinterpret_cast<float2 *>(d_out[i]),
                                   op->stream);
        if (rc) return fail(rc, "giem2g_apply_ie_operator_device_batch: %s", giem2g_last_error());
        op->mult_num++;
    }
    cudaEventRecord(op->ev1, op->stream);
    return set_status(0);
}

int giem2g_gemm_bf16_tn(const void *A, const void *B, float *C, int M, int N, int K, int lda, int ldb, int ldc,
                        int accumulate, int *d_err, void *stream)
{
    static int *own_err = nullptr;
    if (!d_err) {
        if (!own_err && (cudaMalloc(&own_err, sizeof(int)) != cudaSuccess || cudaMemset(own_err, 0, sizeof(int)) != cudaSuccess ||
                         cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess))
            return fail(G2_ERR_NOMEM, "giem2g_gemm_bf16_tn: error word");
        d_err = own_err;
    }
    const int rc = ie_gemm_bf16_tn(A, B, C, M, N, K, lda, ldb, ldc, accumulate, d_err,
                                   reinterpret_cast<cudaStream_t>(stream));
    if (rc) return fail(rc, "giem2g_gemm_bf16_tn: bad shape or alignment (K, lda, ldb multiples of 8; 16-byte aligned A, B)");
    return set_status(0);
}

int giem2g_im2col3d_bf16(const void *x, void *cols, int N, int D, int H, int W, int C, int stride, int Kp, void *stream)
{
    const int rc = ie_im2col3d(x, cols, N, D, H, W, C, stride, Kp, reinterpret_cast<cudaStream_t>(stream));
    if (rc) return fail(rc, "giem2g_im2col3d_bf16: bad shape (stride 1 or 2, Kp >= 27C, Kp multiple of 8)");
    return set_status(0);
}

int giem2g_col2im3d_f32(const float *dcols, float *dx, int N, int D, int H, int W, int C, int stride, int Kp,
                        void *stream)
{
    const int rc = ie_col2im3d(dcols, dx, N, D, H, W, C, stride, Kp, reinterpret_cast<cudaStream_t>(stream));
    if (rc) return fail(rc, "giem2g_col2im3d_f32: bad shape");
    return set_status(0);
}

int giem2g_set_outer_preconditioner(void *ie, int mode, giem2g_precond_fn fn, void *user)
{
    IeOp *op = resolve(ie);
    if (!op || mode < 0 || mode > 2 || (mode && !fn)) return fail(G2_ERR_ARG, "giem2g_set_outer_preconditioner: bad arguments");
    op->precond_mode = mode;
    op->precond_fn = mode ? fn : nullptr;
    op->precond_user = mode ? user : nullptr;
    return set_status(0);
}

int giem2g_get_misfit_history(void *ie, double *out, int max_len)
{
    IeOp *op = resolve(ie);
    if (!op || !out) return 0;
    return krylov_history(op, out, max_len);
}

void *giem2g_get_stream(void *ie)
{
    IeOp *op = resolve(ie);
    return op ? (void *)op->stream : nullptr;
}

double giem2g_last_apply_ms(void *ie)
{
    IeOp *op = resolve(ie);
    if (!op) return -1.0;
    float ms = -1.0f;
    if (cudaEventSynchronize(op->ev1) != cudaSuccess) return -1.0;
    cudaEventElapsedTime(&ms, op->ev0, op->ev1);
    return ms;
}

int giem2g_last_kernel_launches(void *ie)
{
    IeOp *op = resolve(ie);
    return op ? op->last_kernel_launches : 0;
}

long long giem2g_apply_count(void *ie)
{
    IeOp *op = resolve(ie);
    return op ? op->mult_num : -1;
}

void giem2g_set_logger(void (*logger)(const char *)) { g_logger = logger; }

void giem2g_print_stats(void *ie)
{
    // Integral_Equation_Module.F90:473-484 PRINT_STATS
    IeOp *op = resolve(ie);
    if (!op) return;
    char buf[256];
    g2_log("===================================================================================");
    std::snprintf(buf, sizeof(buf), "Time for multiplications:                                 %12.5e s", op->apply_seconds);
    g2_log(buf);
    std::snprintf(buf, sizeof(buf), "Average mult:                                             %12.5e s",
                  op->mult_num ? op->apply_seconds / op->mult_num : 0.0);
    g2_log(buf);
    std::snprintf(buf, sizeof(buf), "Number of matrix-vector multiplications:                  %12lld", op->mult_num);
    g2_log(buf);
    g2_log("===================================================================================");
    op->mult_num = 0;
    op->apply_seconds = 0;
}

// ---- receiver continuation (Continuation_Function_Module.F90; no C interface in the reference) ----

// depth[1..Nl-1] of a background (giem2g_interfaces.F90:264-268)
static std::vector<double> bkg_depth(const GIEM2G_BACKGROUND_TYPE &bkg)
{
    std::vector<double> depth(bkg.Nl + 1, 0.0);
    if (bkg.Nl > 1) {
        const double *th = reinterpret_cast<const double *>(bkg.thickness);
        depth[1] = th[0];
        for (int i = 2; i <= bkg.Nl - 1; i++) depth[i] = depth[i - 1] + th[i - 1];
    }
    return depth;
}

void *giem2g_rc_create(GIEM2G_BACKGROUND_TYPE bkg, GIEM2G_ANOMALY_TYPE anomaly, int Nr, const double *zrecv,
                       const double *x_shift, const double *y_shift)
{
    const int Nx = anomaly.Nx, Ny = anomaly.Ny, Nz = anomaly.Nz;
    if (Nx <= 0 || Ny <= 0 || Nz <= 0 || !is_pow2(2 * Nx) || !is_pow2(2 * Ny) || 2 * Nx > 2048 || 2 * Ny > 2048 ||
        !anomaly.z) {
        fail(G2_ERR_ARG, "giem2g_rc_create: Nx and Ny must be powers of two up to 1024");
        return nullptr;
    }
    if (Nr < 1 || !zrecv || bkg.Nl < 1 || (bkg.Nl > 1 && !bkg.thickness)) {
        fail(G2_ERR_ARG, "giem2g_rc_create: no receivers or bad background");
        return nullptr;
    }
    const double *z = reinterpret_cast<const double *>(anomaly.z);
    const std::vector<double> depth = bkg_depth(bkg);
    // PrepareRecvs (data_types_module.F90:124-152)
    std::vector<RcReceiver> rv(Nr);
    for (int i = 0; i < Nr; i++) {
        const double zr = zrecv[i];
        RcReceiver &r = rv[i];
        r.zrecv = zr;
        r.x_shift = x_shift ? x_shift[i] : 0.0;
        r.y_shift = y_shift ? y_shift[i] : 0.0;
        r.recv_layer = std::max(get_layer(zr, bkg.Nl, depth), 1);
        if (zr <= z[0]) {
            r.anom_cell = 0;
        } else if (zr >= z[Nz]) {
            r.anom_cell = Nz + 1;
        } else {
            for (int iz = 1; iz <= Nz; iz++) {
                if (std::fabs(zr / z[iz] - 1.0) < 1e-7) {
                    r.anom_cell = iz;
                    break;
                } else if (zr > z[iz - 1] && zr < z[iz]) {
                    r.zrecv = z[iz - 1];  // moved to the top border of its cell
                    r.anom_cell = iz - 1;
                    break;
                }
            }
        }
    }
    RcOp *op = rc_create(Nx, Ny, Nz, anomaly.dx, anomaly.dy, z, Nr, rv.data());
    if (!op) {
        fail(G2_ERR_NOMEM, "giem2g_rc_create: %s", giem2g_last_error());
        return nullptr;
    }
    set_status(0);
    return op;
}

int giem2g_rc_receivers(void *rc, double *zrecv, int *recv_layer, int *anom_cell)
{
    if (!rc) return fail(G2_ERR_STATE, "giem2g_rc_receivers: no operator");
    RcOp *op = reinterpret_cast<RcOp *>(rc);
    std::vector<RcReceiver> rv(rc_count(op));
    rc_receivers(op, rv.data());
    for (size_t i = 0; i < rv.size(); i++) {
        if (zrecv) zrecv[i] = rv[i].zrecv;
        if (recv_layer) recv_layer[i] = rv[i].recv_layer;
        if (anom_cell) anom_cell[i] = rv[i].anom_cell;
    }
    return set_status(0);
}

int giem2g_rc_calc_kernel(void *rc, GIEM2G_BACKGROUND_TYPE bkg, double omega)
{
    if (!rc) return fail(G2_ERR_STATE, "giem2g_rc_calc_kernel: no operator");
    if (bkg.Nl < 1 || !bkg.csigb || (bkg.Nl > 1 && !bkg.thickness)) return fail(G2_ERR_ARG, "giem2g_rc_calc_kernel: bad background");
    RcOp *op = reinterpret_cast<RcOp *>(rc);
    // Lnumber (giem2g_interfaces.F90:163-165) from the operator's cell borders
    const int Nz = rc_nz(op);
    const double *z = rc_borders(op);
    const std::vector<double> depth = bkg_depth(bkg);
    std::vector<int> L(Nz + 1);
    for (int i = 1; i <= Nz; i++) L[i] = get_layer((z[i - 1] + z[i]) / 2.0, bkg.Nl, depth);
    L[0] = get_layer(z[0] * (1.0 - 1e-7), bkg.Nl, depth);
    for (int i = 1; i <= Nz; i++)
        if (L[i] < 1) return fail(G2_ERR_ARG, "giem2g_rc_calc_kernel: anomaly cell %d is not below the surface", i);
    std::vector<RcReceiver> rv(rc_count(op));
    rc_receivers(op, rv.data());
    for (const RcReceiver &r : rv)
        if (r.recv_layer > bkg.Nl)
            return fail(G2_ERR_ARG, "giem2g_rc_calc_kernel: receivers were prepared for a background with more layers");
    std::vector<double> th;
    if (bkg.Nl > 1) th.assign(reinterpret_cast<const double *>(bkg.thickness),
                              reinterpret_cast<const double *>(bkg.thickness) + bkg.Nl - 1);
    return set_status(rc_calc_kernel(op, bkg.Nl, reinterpret_cast<const double2 *>(bkg.csigb), th.data(), omega,
                                     L.data()));
}

int giem2g_rc_calc_fft_of_kernel(void *rc)
{
    if (!rc) return fail(G2_ERR_STATE, "giem2g_rc_calc_fft_of_kernel: no operator");
    return set_status(rc_fft_kernel(reinterpret_cast<RcOp *>(rc)));
}

int giem2g_rc_get_kernel(void *rc, void *G)
{
    if (!rc || !G) return fail(G2_ERR_ARG, "giem2g_rc_get_kernel: null argument");
    return set_status(rc_copy_kernel(reinterpret_cast<RcOp *>(rc), reinterpret_cast<double2 *>(G)));
}

int giem2g_rc_set_anomaly_conductivity(void *rc, const void *csiga)
{
    if (!rc || !csiga) return fail(G2_ERR_ARG, "giem2g_rc_set_anomaly_conductivity: null argument");
    return set_status(rc_set_anomaly_conductivity(reinterpret_cast<RcOp *>(rc), reinterpret_cast<const double2 *>(csiga)));
}

int giem2g_rc_recalculate(void *rc, const void *E, void *Ea, void *Ha)
{
    if (!rc || !E || !Ea || !Ha) return fail(G2_ERR_ARG, "giem2g_rc_recalculate: null argument");
    return set_status(rc_recalculate_host(reinterpret_cast<RcOp *>(rc), reinterpret_cast<const double2 *>(E),
                                          reinterpret_cast<double2 *>(Ea), reinterpret_cast<double2 *>(Ha)));
}

int giem2g_rc_recalculate_device(void *rc, const void *d_E, void *d_Ea, void *d_Ha)
{
    if (!rc || !d_E || !d_Ea || !d_Ha) return fail(G2_ERR_ARG, "giem2g_rc_recalculate_device: null argument");
    return set_status(rc_recalculate_device(reinterpret_cast<RcOp *>(rc), reinterpret_cast<const double2 *>(d_E),
                                            reinterpret_cast<double2 *>(d_Ea), reinterpret_cast<double2 *>(d_Ha)));
}

void *giem2g_rc_get_stream(void *rc)
{
    return rc ? reinterpret_cast<void *>(rc_stream(reinterpret_cast<RcOp *>(rc))) : nullptr;
}

void giem2g_rc_delete(void *rc)
{
    rc_delete(reinterpret_cast<RcOp *>(rc));
    set_status(0);
}

void giem2g_delete_ie_operator(void *ie)
{
    IeOp *op = resolve(ie);
    if (!op) return;
    if (op->stream) cudaStreamSynchronize(op->stream);
    ie_free_learned(op);
    krylov_free(op);
    void *ptrs[] = {op->d_spatial, op->d_tensor64, op->d_tensor32, op->d_csiga, op->d_gsig64, op->d_asig64,
                    op->d_gsig32, op->d_asig32, op->d_post64, op->d_post32, op->d_twx64, op->d_twy64,
                    op->d_twx32, op->d_twy32, op->scratch.U1, op->scratch.Uhat, op->pair_scratch.U1,
                    op->pair_scratch.Uhat, op->d_vin, op->d_vout, op->d_err, op->d_vin32, op->d_vout32};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (op->ev0) cudaEventDestroy(op->ev0);
    if (op->ev1) cudaEventDestroy(op->ev1);
    if (op->evc0) cudaEventDestroy(op->evc0);
    if (op->evc1) cudaEventDestroy(op->evc1);
    if (op->stream) cudaStreamDestroy(op->stream);
    if (g_last_op == op) g_last_op = nullptr;
    delete op;
    set_status(0);
}

}  // extern "C"

int ie_check_device_error(IeOp *op)
{
    int h = 0;
    if (!op->d_err) return 0;
    if ((op->stream && cudaStreamSynchronize(op->stream) != cudaSuccess) ||
        cudaMemcpy(&h, op->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(G2_ERR_CUDA, "error-word read failed");
    if (h) {
        cudaMemset(op->d_err, 0, sizeof(int));
        cudaStreamSynchronize(cudaStreamLegacy);
        return fail(G2_ERR_NUMERIC, "device wait limit reached (code %d)", h);
    }
    return 0;
}
