// spectrum.cu -- the 2DCS analysis step after the batched pump-probe runs.
//
// The reference computes it offline in Python (util/readers_new/reader_honeycomb.py:
// 459-553, read_2D_nonlinear / compute_2d_fft): for one component c of M_local,
//   M_NL[k][t] = M01_k[t] - M0[t] - M1_k[t]          (k: delay tau_k, t: time)
//   S = flip_t( | fftshift( fft2( M_NL - mean(M_NL) ) ) | )
// Here M_NL and its mean are formed on the host in a fixed order (O(n_tau n_t)),
// the 2-D transform runs on the device through cuFFT (double complex, the data
// has a zero imaginary part), and one kernel applies |.|, the fftshift of both
// axes and the flip of the omega_t axis while copying out.
#include "cmd.h"
#include "cmd_internal.h"

#include <cuda_runtime.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace {

int fail_s(int code, const std::string& msg) { return cmd::fail(code, msg); }

// out[k][t] = | F[(k - nk/2) mod nk][((nt - 1 - t) - nt/2) mod nt] |
__global__ void shift_abs_kernel(const cufftDoubleComplex* __restrict__ F, int64_t nk, int64_t nt,
                                 double* __restrict__ out) {
    const int64_t total = nk * nt;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = e / nt, t = e - k * nt;
        const int64_t ks = ((k - nk / 2) % nk + nk) % nk;
        const int64_t tf = nt - 1 - t;
        const int64_t ts = ((tf - nt / 2) % nt + nt) % nt;
        const cufftDoubleComplex v = F[ks * nt + ts];
        out[e] = hypot(v.x, v.y);
    }
}

}  // namespace

extern "C" int cmd_nonlinear_spectrum(const double* M0, const double* M1, const double* M01, int64_t n_tau,
                                      int64_t n_t, int32_t component, double* m_nl, double* spectrum) {
    cmd::clear_error();
    if (!M0 || !M1 || !M01) return fail_s(CMD_ERR_INVALID_ARG, "NULL trajectory array");
    if (n_tau <= 0 || n_t <= 0 || n_tau > (1 << 24) || n_t > (1 << 24) || n_tau * n_t > ((int64_t)1 << 31))
        return fail_s(CMD_ERR_INVALID_ARG, "bad spectrum size");
    if (component < 0 || component > 2) return fail_s(CMD_ERR_INVALID_ARG, "component must be 0, 1 or 2");
    const int64_t n = n_tau * n_t;
    std::vector<double> nl((size_t)n);
    double sum = 0.0;
    for (int64_t k = 0; k < n_tau; ++k)
        for (int64_t t = 0; t < n_t; ++t) {
            const int64_t i = (k * n_t + t) * 3 + component;
            const double v = M01[i] - M0[t * 3 + component] - M1[i];
            nl[(size_t)(k * n_t + t)] = v;
            sum += v;
        }
    if (m_nl)
        for (int64_t e = 0; e < n; ++e) m_nl[e] = nl[(size_t)e];
    if (!spectrum) return CMD_OK;
    const double mean = sum / (double)n;
    std::vector<cufftDoubleComplex> h((size_t)n);
    for (int64_t e = 0; e < n; ++e) h[(size_t)e] = make_cuDoubleComplex(nl[(size_t)e] - mean, 0.0);
    cufftDoubleComplex* d = nullptr;
    double* dout = nullptr;
    cufftHandle plan = 0;
    bool have_plan = false;
    int rc = CMD_OK;
    auto cuda_ok = [&](cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        rc = fail_s(e == cudaErrorMemoryAllocation ? CMD_ERR_OOM : CMD_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
        return false;
    };
    do {
        if (!cuda_ok(cudaMalloc((void**)&d, (size_t)n * sizeof(cufftDoubleComplex)), "cudaMalloc")) break;
        if (!cuda_ok(cudaMalloc((void**)&dout, (size_t)n * sizeof(double)), "cudaMalloc")) break;
        if (!cuda_ok(cudaMemcpy(d, h.data(), (size_t)n * sizeof(cufftDoubleComplex), cudaMemcpyHostToDevice),
                     "cudaMemcpy"))
            break;
        if (cufftPlan2d(&plan, (int)n_tau, (int)n_t, CUFFT_Z2Z) != CUFFT_SUCCESS) {
            rc = fail_s(CMD_ERR_CUDA, "cufftPlan2d failed");
            break;
        }
        have_plan = true;
        if (cufftExecZ2Z(plan, d, d, CUFFT_FORWARD) != CUFFT_SUCCESS) {
            rc = fail_s(CMD_ERR_CUDA, "cufftExecZ2Z failed");
            break;
        }
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
        shift_abs_kernel<<<blocks, 256>>>(d, n_tau, n_t, dout);
        if (!cuda_ok(cudaGetLastError(), "shift_abs_kernel")) break;
        if (!cuda_ok(cudaMemcpy(spectrum, dout, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy"))
            break;
    } while (false);
    if (have_plan) cufftDestroy(plan);
    if (d) cudaFree(d);
    if (dout) cudaFree(dout);
    return rc;
}
