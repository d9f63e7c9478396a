// dispatch_impl.cuh -- template bodies of dispatch.h (included by step_q19.cu / step_q27.cu).
#pragma once
#include "dispatch.h"
#include "step_impl.cuh"

namespace vlbm {

inline unsigned grid_for(long long n, int block) { return (unsigned)((n + block - 1) / block); }

// Launch that may start before the previous kernel of the stream has finished
// (programmatic dependent launch), once that kernel has triggered it.  Either
// the two touch disjoint memory (the bulk grid after the step's boundary list)
// or the launched kernel waits in-kernel (griddepcontrol.wait) for the
// previous one's completion before it reads anything (the chained steps).
template <typename... Args>
cudaError_t launch_overlapped(void (*kernel)(Args...), unsigned grid, unsigned block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int Q, int OP, int RHEO, int ST>
cudaError_t step_t(const StepParams& p, bool odd, LaunchShape ls, cudaStream_t s) {
    if (p.pairH > 0) {  // z-paired layout: one thread per node pair; the listed pairs, then the bulk ones
        const unsigned g = grid_for(p.N / 2, ls.block);
        const unsigned gs = grid_for(p.n_special, 256);
        if (gs) {   // chained to the previous step (step_chain_enter)
            cudaError_t e;
            if (p.pairBlk)
                e = odd ? launch_overlapped(k_step2<Q, OP, RHEO, ST, true, true>, gs, 256, s, p)
                        : launch_overlapped(k_step2<Q, OP, RHEO, ST, false, true>, gs, 256, s, p);
            else
                e = odd ? launch_overlapped(k_step2<Q, OP, RHEO, ST, true, false>, gs, 256, s, p)
                        : launch_overlapped(k_step2<Q, OP, RHEO, ST, false, false>, gs, 256, s, p);
            if (e != cudaSuccess) return e;
            if (p.pairBlk)
                return odd ? launch_overlapped(k_step2_bulk<Q, OP, RHEO, ST, true, true>, g, ls.block, s, p)
                           : launch_overlapped(k_step2_bulk<Q, OP, RHEO, ST, false, true>, g, ls.block, s, p);
            return odd ? launch_overlapped(k_step2_bulk<Q, OP, RHEO, ST, true, false>, g, ls.block, s, p)
                       : launch_overlapped(k_step2_bulk<Q, OP, RHEO, ST, false, false>, g, ls.block, s, p);
        }
        // no boundary list: a normal launch (the bulk kernel reads before it waits)
        if (p.pairBlk) {
            if (odd) k_step2_bulk<Q, OP, RHEO, ST, true, true><<<g, ls.block, 0, s>>>(p);
            else k_step2_bulk<Q, OP, RHEO, ST, false, true><<<g, ls.block, 0, s>>>(p);
        } else {
            if (odd) k_step2_bulk<Q, OP, RHEO, ST, true, false><<<g, ls.block, 0, s>>>(p);
            else k_step2_bulk<Q, OP, RHEO, ST, false, false><<<g, ls.block, 0, s>>>(p);
        }
        return cudaGetLastError();
    }
    const unsigned g = grid_for(p.N, ls.block);   // chained to the previous step (step_chain_enter)
    return odd ? launch_overlapped(k_step<Q, OP, RHEO, ST, true>, g, ls.block, s, p)
               : launch_overlapped(k_step<Q, OP, RHEO, ST, false>, g, ls.block, s, p);
}

template <int Q, int OP, int ST>
cudaError_t step_rh(const StepParams& p, int rheo, bool odd, LaunchShape ls, cudaStream_t s) {
    switch (rheo) {
    case VLBM_NEWTONIAN: return step_t<Q, OP, VLBM_NEWTONIAN, ST>(p, odd, ls, s);
    case VLBM_BINGHAM: return step_t<Q, OP, VLBM_BINGHAM, ST>(p, odd, ls, s);
    case VLBM_POWERLAW: return step_t<Q, OP, VLBM_POWERLAW, ST>(p, odd, ls, s);
    }
    return cudaErrorInvalidValue;
}

template <int Q, int ST>
cudaError_t launch_step_st(const StepParams& p, int op, int rheo, bool odd, LaunchShape ls, cudaStream_t s) {
    if (op == VLBM_OP_BGK) return step_rh<Q, VLBM_OP_BGK, ST>(p, rheo, odd, ls, s);
    return step_rh<Q, VLBM_OP_REGULARIZED, ST>(p, rheo, odd, ls, s);
}

template <int Q, int RHEO, int ST>
cudaError_t macro_t(const MacroParams& mp, bool odd, cudaStream_t s) {
    const unsigned g = grid_for(mp.s.N, 256);
    const bool pr = mp.s.pairH > 0;
    if (odd) {
        if (pr) k_macro<Q, RHEO, ST, true, true><<<g, 256, 0, s>>>(mp);
        else k_macro<Q, RHEO, ST, true, false><<<g, 256, 0, s>>>(mp);
    } else {
        if (pr) k_macro<Q, RHEO, ST, false, true><<<g, 256, 0, s>>>(mp);
        else k_macro<Q, RHEO, ST, false, false><<<g, 256, 0, s>>>(mp);
    }
    return cudaGetLastError();
}

template <int Q, int ST>
cudaError_t launch_macro_st(const MacroParams& mp, int rheo, bool odd, cudaStream_t s) {
    switch (rheo) {
    case VLBM_NEWTONIAN: return macro_t<Q, VLBM_NEWTONIAN, ST>(mp, odd, s);
    case VLBM_BINGHAM: return macro_t<Q, VLBM_BINGHAM, ST>(mp, odd, s);
    case VLBM_POWERLAW: return macro_t<Q, VLBM_POWERLAW, ST>(mp, odd, s);
    }
    return cudaErrorInvalidValue;
}

template <int Q, int ST>
cudaError_t get_pops_t(const StepParams& p, bool odd, float* out, cudaStream_t s) {
    const unsigned g = grid_for(p.N, 256);
    const bool pr = p.pairH > 0;
    if (odd) {
        if (pr) k_get_pops<Q, ST, true, true><<<g, 256, 0, s>>>(p, out);
        else k_get_pops<Q, ST, true, false><<<g, 256, 0, s>>>(p, out);
    } else {
        if (pr) k_get_pops<Q, ST, false, true><<<g, 256, 0, s>>>(p, out);
        else k_get_pops<Q, ST, false, false><<<g, 256, 0, s>>>(p, out);
    }
    return cudaGetLastError();
}

template <int Q, int ST>
cudaError_t launch_get_pops_st(const StepParams& p, bool odd, float* out, cudaStream_t s) {
    return get_pops_t<Q, ST>(p, odd, out, s);
}

template <int Q, int ST>
cudaError_t launch_set_pops_st(const StepParams& p, const float* in, float rho, float ux, float uy, float uz,
                               cudaStream_t s) {
    const unsigned g = grid_for(p.N, 256);
    if (p.pairH > 0) k_set_pops<Q, ST, true><<<g, 256, 0, s>>>(p, in, rho, ux, uy, uz);
    else k_set_pops<Q, ST, false><<<g, 256, 0, s>>>(p, in, rho, ux, uy, uz);
    return cudaGetLastError();
}

template <int Q, int OP, int RHEO, int ST>
cudaError_t batched_t(const BatchLaunch* L, const BatchState* state, const BatchBlock* table, int ntiles, int grid,
                      bool odd, cudaStream_t s) {
    // chained to the previous launch of the stream (step_chain_enter)
    return odd ? launch_overlapped(k_step_batched<Q, OP, RHEO, ST, true>, grid, 256, s, L, state, table, ntiles)
               : launch_overlapped(k_step_batched<Q, OP, RHEO, ST, false>, grid, 256, s, L, state, table, ntiles);
}

template <int Q, int OP, int ST>
cudaError_t batched_rh(const BatchLaunch* L, const BatchState* state, const BatchBlock* table, int ntiles, int grid,
                       bool odd, int rheo, cudaStream_t s) {
    switch (rheo) {
    case VLBM_NEWTONIAN: return batched_t<Q, OP, VLBM_NEWTONIAN, ST>(L, state, table, ntiles, grid, odd, s);
    case VLBM_BINGHAM: return batched_t<Q, OP, VLBM_BINGHAM, ST>(L, state, table, ntiles, grid, odd, s);
    case VLBM_POWERLAW: return batched_t<Q, OP, VLBM_POWERLAW, ST>(L, state, table, ntiles, grid, odd, s);
    }
    return cudaErrorInvalidValue;
}

template <int Q, int ST>
cudaError_t launch_batched_st(const BatchLaunch* L, const BatchState* state, const BatchBlock* table, int ntiles,
                              int grid, bool odd, int op, int rheo, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    if (op == VLBM_OP_BGK) return batched_rh<Q, VLBM_OP_BGK, ST>(L, state, table, ntiles, grid, odd, rheo, s);
    return batched_rh<Q, VLBM_OP_REGULARIZED, ST>(L, state, table, ntiles, grid, odd, rheo, s);
}

// resident blocks per SM: the smaller of the two parities
template <int Q, int OP, int RHEO, int ST>
int occ_t() {
    int a = 0, b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_step_batched<Q, OP, RHEO, ST, false>, 256, 0) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_step_batched<Q, OP, RHEO, ST, true>, 256, 0) != cudaSuccess)
        return 0;
    return a < b ? a : b;
}

template <int Q, int OP, int ST>
int occ_rh(int rheo) {
    switch (rheo) {
    case VLBM_NEWTONIAN: return occ_t<Q, OP, VLBM_NEWTONIAN, ST>();
    case VLBM_BINGHAM: return occ_t<Q, OP, VLBM_BINGHAM, ST>();
    case VLBM_POWERLAW: return occ_t<Q, OP, VLBM_POWERLAW, ST>();
    }
    return 0;
}

template <int Q, int ST>
int batched_occupancy_st(int op, int rheo) {
    if (op == VLBM_OP_BGK) return occ_rh<Q, VLBM_OP_BGK, ST>(rheo);
    return occ_rh<Q, VLBM_OP_REGULARIZED, ST>(rheo);
}

template <int Q, int ST>
cudaError_t launch_relayout_st(const void* src, void* dst, int nx, int ny, long long N, int sH, int sB, int dH,
                               int dB, cudaStream_t s) {
    k_relayout<Q, ST><<<grid_for(N, 256), 256, 0, s>>>(src, dst, nx, ny, N, sH, sB, dH, dB);
    return cudaGetLastError();
}

template <int Q, int ST>
cudaError_t launch_halo_st(void* pop, const HaloSpec* msgs, int nx, int ny, long long N, int H, int blk,
                           bool unpack, cudaStream_t s) {
    const HaloMsg m0{msgs[0].buf, msgs[0].z, msgs[0].dz}, m1{msgs[1].buf, msgs[1].z, msgs[1].dz};
    k_halo<Q, ST><<<grid_for(2LL * halo_pops<Q>() * nx * ny, 256), 256, 0, s>>>(pop, m0, m1, nx, ny, N, H, blk,
                                                                                unpack ? 1 : 0);
    return cudaGetLastError();
}

#define VLBM_INSTANTIATE(QQ, SS)                                                                              \
    template cudaError_t launch_step_st<QQ, SS>(const StepParams&, int, int, bool, LaunchShape, cudaStream_t); \
    template cudaError_t launch_macro_st<QQ, SS>(const MacroParams&, int, bool, cudaStream_t);                 \
    template cudaError_t launch_get_pops_st<QQ, SS>(const StepParams&, bool, float*, cudaStream_t);            \
    template cudaError_t launch_set_pops_st<QQ, SS>(const StepParams&, const float*, float, float, float, float, \
                                                    cudaStream_t);                                              \
    template cudaError_t launch_batched_st<QQ, SS>(const BatchLaunch*, const BatchState*, const BatchBlock*, int,  \
                                                   int, bool, int, int, cudaStream_t);                          \
    template int batched_occupancy_st<QQ, SS>(int, int);                                                       \
    template cudaError_t launch_relayout_st<QQ, SS>(const void*, void*, int, int, long long, int, int, int, int,  \
                                                    cudaStream_t);                                              \
    template cudaError_t launch_halo_st<QQ, SS>(void*, const HaloSpec*, int, int, long long, int, int, bool,      \
                                                cudaStream_t);

}  // namespace vlbm
