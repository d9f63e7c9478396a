// reduce.cu -- FP64 global mass and momentum of the current state.
//
// Sums rho and rho*u = sum_i f_i c_i + F/2 over every node in double precision
// (the reference's only global reduction is the FP32 density mean of
// AuxFunctions/reduction.cu:36-98 used for DENSITY_CORRECTION; treatData.cpp
// sums on the host).  Two passes with a fixed partition: each block owns a
// chunk of REDUCE_CHUNK consecutive nodes and writes four partial sums, a
// single block then adds the partials in block order, so the result is
// bit-reproducible for a given lattice size.
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "sim.h"
#include "step_impl.cuh"

namespace vlbm {

constexpr int REDUCE_THREADS = 256;
constexpr int REDUCE_CHUNK = 4096;   // nodes per block

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <int Q, int ST, bool ODD, bool PAIRED>
__global__ void __launch_bounds__(REDUCE_THREADS) k_moment_partials(const StepParams p, double* partials) {
    const long long base = (long long)blockIdx.x * REDUCE_CHUNK;
    const long long end = base + REDUCE_CHUNK < p.N ? base + REDUCE_CHUNK : p.N;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long nn = base + threadIdx.x; nn < end; nn += REDUCE_THREADS) {
        const unsigned n = (unsigned)nn;
        const int x = (int)(n % (unsigned)p.nx);
        const unsigned t = n / (unsigned)p.nx;
        const int y = (int)(t % (unsigned)p.ny);
        const int z = (int)(t / (unsigned)p.ny);
        Nbr nb;
        nb.init(x, y, z, p.nx, p.ny, p.nz);
        float f[Q];
        uint8_t cls;
        gather<Q, ST, ODD, PAIRED>(p, n, nb, x, y, z, f, cls);
        if (cls & NODE_UNUSED) continue;   // outside the fluid
        // the gather gives deviations g_i = f_i - w_i rho0
        double rho = (double)p.rho0, jx = 0.5 * p.fx, jy = 0.5 * p.fy, jz = 0.5 * p.fz;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            rho += f[i];
            if (lat_cx(i)) jx += lat_cx(i) * (double)f[i];
            if (lat_cy(i)) jy += lat_cy(i) * (double)f[i];
            if (lat_cz(i)) jz += lat_cz(i) * (double)f[i];
        }
        acc[0] += rho; acc[1] += jx; acc[2] += jy; acc[3] += jz;
    }
    __shared__ double sh[4][REDUCE_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double v = warp_sum(acc[k]);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < REDUCE_THREADS / 32; ++w) s += sh[threadIdx.x][w];
        partials[(size_t)blockIdx.x * 4 + threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(REDUCE_THREADS) k_moment_finalize(const double* partials, int nblocks, double* out) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += REDUCE_THREADS)
        for (int k = 0; k < 4; ++k) acc[k] += partials[(size_t)b * 4 + k];
    __shared__ double sh[4][REDUCE_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double v = warp_sum(acc[k]);
        if (lane == 0) sh[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < REDUCE_THREADS / 32; ++w) s += sh[threadIdx.x][w];
        out[threadIdx.x] = s;
    }
}

int reduce_blocks(long long N) { return (int)((N + REDUCE_CHUNK - 1) / REDUCE_CHUNK); }

// Launch both passes: partials[4*reduce_blocks(N)] doubles, out[4] doubles (device).
cudaError_t launch_moments_sum(vlbm_sim* s, double* partials, double* out) {
    const StepParams p = make_params(s);
    const int nb = reduce_blocks(s->N);
    const bool odd = s->parity == 1;
#define VLBM_RED(QQ, SS)                                                                                   \
    do {                                                                                                   \
        if (p.pairH > 0) {                                                                                 \
            if (odd) k_moment_partials<QQ, SS, true, true><<<nb, REDUCE_THREADS, 0, s->stream>>>(p, partials); \
            else k_moment_partials<QQ, SS, false, true><<<nb, REDUCE_THREADS, 0, s->stream>>>(p, partials);    \
        } else {                                                                                           \
            if (odd) k_moment_partials<QQ, SS, true, false><<<nb, REDUCE_THREADS, 0, s->stream>>>(p, partials); \
            else k_moment_partials<QQ, SS, false, false><<<nb, REDUCE_THREADS, 0, s->stream>>>(p, partials);   \
        }                                                                                                  \
    } while (0)
    const int st = s->cfg.storage;
    if (s->Q == 19) {
        if (st == VLBM_STORE_F32) VLBM_RED(19, VLBM_STORE_F32);
        else if (st == VLBM_STORE_F16) VLBM_RED(19, VLBM_STORE_F16);
        else VLBM_RED(19, VLBM_STORE_BF16);
    } else {
        if (st == VLBM_STORE_F32) VLBM_RED(27, VLBM_STORE_F32);
        else if (st == VLBM_STORE_F16) VLBM_RED(27, VLBM_STORE_F16);
        else VLBM_RED(27, VLBM_STORE_BF16);
    }
#undef VLBM_RED
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_moment_finalize<<<1, REDUCE_THREADS, 0, s->stream>>>(partials, nb, out);
    return cudaGetLastError();
}

}  // namespace vlbm

using namespace vlbm;

extern "C" vlbm_status vlbm_moments_sum(vlbm_sim* s, double* out4) {
    if (!s || !out4) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    const size_t need = (size_t)4 * reduce_blocks(s->N) + 4;
    if (!s->red_scratch) {
        e = sim_malloc(s, (void**)&s->red_scratch, need * sizeof(double));
        if (e != cudaSuccess) { s->red_scratch = nullptr; return cuda_status(e, "reduction scratch allocation"); }
        s->device_bytes += need * sizeof(double);
    }
    double* partials = s->red_scratch;
    double* out = s->red_scratch + (need - 4);
    e = launch_moments_sum(s, partials, out);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out4, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return cuda_status(e, "vlbm_moments_sum");
}

// ---------------------------------------------------------------------------
// Allocation-free variant of vlbm_moments_sum.
//
// Some callers cannot call cudaMalloc when they want these sums: a serving
// process that has handed its whole HBM budget to admitted simulations, a
// host thread sampling mass and momentum between steps while the allocator is
// owned by another framework, or code that must not grow the device footprint
// after start-up.  This variant uses a fixed scratch array in the library's
// device globals instead of the per-simulation buffer that vlbm_moments_sum
// allocates on first use.  It runs the same two kernels on the same partition,
// so both entry points return bit-identical sums.
//
// The array below holds REDUCE_NOALLOC_MAX_BLOCKS partial-sum slots (4 doubles
// each) plus the 4-double result: 512 KiB + 32 B that every GPU which loads the
// library keeps until the process exits.  That caps the lattice at
// REDUCE_NOALLOC_MAX_BLOCKS * REDUCE_CHUNK = 67,108,864 nodes.  Every slot the
// finalize pass reads is written by the partial pass of the same call, so no
// part of the array has to start at zero; the array keeps the last call's
// contents.  All calls on a device share it: calls whose kernels overlap on
// the GPU (different streams, or several host threads) race and return wrong
// sums, so callers must serialise them.
constexpr int REDUCE_NOALLOC_MAX_BLOCKS = 16384;
static __device__ __align__(256) double g_reduce_noalloc_scratch[4 * REDUCE_NOALLOC_MAX_BLOCKS + 4];

namespace {
// Device address of g_reduce_noalloc_scratch per device ordinal.  In host code
// the array's name is only a host-side stand-in, so the address is taken with
// cudaGetSymbolAddress once per device, with that device current.
constexpr int kMaxDevices = 64;
double* g_noalloc_addr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

cudaError_t noalloc_scratch_address(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_reduce_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[device] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[device];
    return cudaSuccess;
}
}  // namespace

extern "C" vlbm_status vlbm_moments_sum_noalloc(vlbm_sim* s, double* out4) {
    if (!s || !out4) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    const int nb = reduce_blocks(s->N);
    if (nb > REDUCE_NOALLOC_MAX_BLOCKS) {
        set_last_error("vlbm_moments_sum_noalloc: the lattice has " + std::to_string(s->N) +
                       " nodes, more than the 67108864 its built-in scratch covers; use vlbm_moments_sum");
        return VLBM_ERR_INVALID;
    }
    cudaError_t e = cudaSetDevice(s->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    double* scratch = nullptr;
    e = noalloc_scratch_address(s->device, &scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_reduce_noalloc_scratch)");
    double* out = scratch + 4 * REDUCE_NOALLOC_MAX_BLOCKS;
    e = launch_moments_sum(s, scratch, out);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out4, out, 4 * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return cuda_status(e, "vlbm_moments_sum_noalloc");
}
