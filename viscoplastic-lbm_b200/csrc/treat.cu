// treat.cu -- report-step data treatment on the device (treatData.cpp:25-89,
// stopSim treatData.cpp:451-460).
//
// On every report step the reference copies rho and u of the whole lattice to
// the host and loops over all nodes in FP32:
//   residual = sum |u - u_old| / sum |u|   (1 when sum |u| = 0), u_old = the
//              velocity of the previous report (main.cu:430-434)
//   avgRho   = sum rho / N
//   avgUzPlanXZ[y] = sum over x, z of uz / (NX * NZ)
// and stops the run when residual < RESID_MAX or avgRho < 0.  Here the same
// quantities come from two launches over the device fields, summed in FP64
// with a fixed partition (bit-reproducible), and only 3 + NY doubles cross to
// the host.  The previous report's velocity stays on the device.
//
// Differences from the reference, on purpose: the sums are FP64 (the
// reference's FP32 running sums over 2e6 nodes keep about 3 significant
// digits of the residual), and avgUzPlanXZ is the mean of this report (the
// reference never clears it between reports, macrProc.h:39-40, so its k-th
// report holds the sum of k means; a caller who wants that adds them up).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include "sim.h"

namespace vlbm {

constexpr int TREAT_THREADS = 256;

__device__ __forceinline__ double treat_warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block (y, zc) sums over the x rows of plane y with z in its chunk:
// partials[(y * nzc + zc) * 4 + {0,1,2,3}] = sum |u - u_prev|, sum |u|,
// sum rho, sum uz.  The current velocity replaces u_prev.
__global__ void __launch_bounds__(TREAT_THREADS) k_treat_partials(const float* __restrict__ rho,
                                                                  const float* __restrict__ ux,
                                                                  const float* __restrict__ uy,
                                                                  const float* __restrict__ uz, float* prev,
                                                                  int prev_valid, int nx, int ny, int nz, int zchunk,
                                                                  double* partials) {
    const int y = blockIdx.x, zc = blockIdx.y;
    const int z0 = zc * zchunk, z1 = min(nz, z0 + zchunk);
    const long long N = (long long)nx * ny * nz;
    const long long cnt = (long long)(z1 - z0) * nx;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long k = threadIdx.x; k < cnt; k += TREAT_THREADS) {
        const int z = z0 + (int)(k / nx), x = (int)(k % nx);
        const long long n = (long long)x + (long long)nx * (y + (long long)ny * z);
        const double a = ux[n], b = uy[n], c = uz[n];
        double pa = 0.0, pb = 0.0, pc = 0.0;
        if (prev_valid) { pa = prev[n]; pb = prev[N + n]; pc = prev[2 * N + n]; }
        const double da = a - pa, db = b - pb, dc = c - pc;
        acc[0] += sqrt(da * da + db * db + dc * dc);
        acc[1] += sqrt(a * a + b * b + c * c);
        acc[2] += (double)rho[n];
        acc[3] += c;
        prev[n] = (float)a; prev[N + n] = (float)b; prev[2 * N + n] = (float)c;
    }
    __shared__ double sh[4][TREAT_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const double v = treat_warp_sum(acc[q]);
        if (lane == 0) sh[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < TREAT_THREADS / 32; ++w) s += sh[threadIdx.x][w];
        partials[((size_t)y * gridDim.y + zc) * 4 + threadIdx.x] = s;
    }
}

// One block: per-plane sums over the z chunks in order, then the global sums
// over the planes in order.  out[0..2] = sum |du|, sum |u|, sum rho;
// out[3 + y] = sum uz of plane y.
__global__ void __launch_bounds__(TREAT_THREADS) k_treat_finalize(const double* partials, int ny, int nzc,
                                                                  double* plane, double* out) {
    for (int y = threadIdx.x; y < ny; y += TREAT_THREADS) {
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        for (int zc = 0; zc < nzc; ++zc)
            for (int q = 0; q < 4; ++q) s[q] += partials[((size_t)y * nzc + zc) * 4 + q];
        for (int q = 0; q < 3; ++q) plane[(size_t)y * 3 + q] = s[q];
        out[3 + y] = s[3];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int y = 0; y < ny; ++y) s += plane[(size_t)y * 3 + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

}  // namespace vlbm

using namespace vlbm;

extern "C" vlbm_status vlbm_treat_data(vlbm_sim* s, double resid_max, vlbm_treat* out, double* avg_uz_plane_xz,
                                       int32_t ny) {
    if (!s || !out) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    if (avg_uz_plane_xz && ny != s->cfg.ny) { set_last_error("avg_uz_plane_xz must hold NY values"); return VLBM_ERR_INVALID; }
    if (!s->geometry) { set_last_error("vlbm_treat_data needs a geometry"); return VLBM_ERR_STATE; }
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    const int NX = s->cfg.nx, NY = s->cfg.ny, NZ = s->cfg.nz;
    const size_t N = (size_t)s->N;
    // about four blocks per SM of a 148-SM part, at least one plane chunk per plane
    const int want = std::max(1, std::min(NZ, (4 * 148 + NY - 1) / NY));
    const int zchunk = (NZ + want - 1) / want;
    const int nzc = (NZ + zchunk - 1) / zchunk;
    const size_t red_doubles = (size_t)NY * nzc * 4 + (size_t)NY * 3 + 3 + (size_t)NY;
    vlbm_status st = ensure_scratch(s);
    if (st != VLBM_OK) return st;
    if (!s->treat_prev) {
        e = sim_malloc(s, (void**)&s->treat_prev, 3 * N * sizeof(float));
        if (e != cudaSuccess) { s->treat_prev = nullptr; return cuda_status(e, "report velocity allocation"); }
        s->device_bytes += 3 * N * sizeof(float);
        s->treat_prev_valid = false;
    }
    if (!s->treat_red) {   // sizes depend only on the lattice, fixed for the simulation's life
        e = sim_malloc(s, (void**)&s->treat_red, red_doubles * sizeof(double));
        if (e != cudaSuccess) { s->treat_red = nullptr; return cuda_status(e, "report scratch allocation"); }
        s->device_bytes += red_doubles * sizeof(double);
    }
    float* f = s->scratch;
    st = sim_macroscopics_device(s, f, f + N, f + 2 * N, f + 3 * N, nullptr);
    if (st != VLBM_OK) return st;
    double* partials = s->treat_red;
    double* plane = partials + (size_t)NY * nzc * 4;
    double* res = plane + (size_t)NY * 3;
    k_treat_partials<<<dim3(NY, nzc), TREAT_THREADS, 0, s->stream>>>(f, f + N, f + 2 * N, f + 3 * N, s->treat_prev,
                                                                   s->treat_prev_valid ? 1 : 0, NX, NY, NZ, zchunk,
                                                                   partials);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        k_treat_finalize<<<1, TREAT_THREADS, 0, s->stream>>>(partials, NY, nzc, plane, res);
        e = cudaGetLastError();
    }
    std::vector<double> h(3 + (size_t)NY);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), res, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_status(e, "vlbm_treat_data");
    s->treat_prev_valid = true;
    out->step = s->step;
    out->residual = h[1] != 0.0 ? h[0] / h[1] : 1.0;
    out->avg_rho = h[2] / (double)N;
    out->stop = (out->residual < resid_max || out->avg_rho < 0.0) ? 1 : 0;
    if (avg_uz_plane_xz)
        for (int y = 0; y < NY; ++y) avg_uz_plane_xz[y] = h[3 + y] / ((double)NX * NZ);
    return VLBM_OK;
}
