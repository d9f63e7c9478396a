// dispatch.h -- host entry points into the templated kernels of step_impl.cuh.
// Each (velocity set, storage) pair is instantiated in its own translation
// unit (step_q<Q>_<storage>.cu); dispatch.cpp selects one at run time.
#pragma once
#include <cuda_runtime.h>
#include "internal.h"

namespace vlbm {

struct LaunchShape {
    int block;      // threads per block
};

template <int Q, int ST>
cudaError_t launch_step_st(const StepParams& p, int op, int rheo, bool odd, LaunchShape ls, cudaStream_t s);
template <int Q, int ST>
cudaError_t launch_macro_st(const MacroParams& mp, int rheo, bool odd, cudaStream_t s);
template <int Q, int ST>
cudaError_t launch_get_pops_st(const StepParams& p, bool odd, float* out, cudaStream_t s);
template <int Q, int ST>
cudaError_t launch_set_pops_st(const StepParams& p, const float* in, float rho, float ux, float uy, float uz,
                               cudaStream_t s);

struct BatchLaunch;
struct BatchState;
struct BatchBlock;
template <int Q, int ST>
cudaError_t launch_batched_st(const BatchLaunch* L, const BatchState* state, const BatchBlock* table, int ntiles,
                              int grid, bool odd, int op, int rheo, cudaStream_t s);

template <int Q, int ST>
cudaError_t launch_relayout_st(const void* src, void* dst, int nx, int ny, long long N, int sH, int sB, int dH,
                               int dB, cudaStream_t s);

// One z-slab halo message: buffer (nullptr = none), plane and c_z.
struct HaloSpec {
    void* buf;
    int z, dz;
};
template <int Q, int ST>
cudaError_t launch_halo_st(void* pop, const HaloSpec* msgs, int nx, int ny, long long N, int H, int blk,
                           bool unpack, cudaStream_t s);

// Run-time selection over (Q, storage).
cudaError_t launch_step(int Q, int st, const StepParams& p, int op, int rheo, bool odd, LaunchShape ls,
                        cudaStream_t s);
cudaError_t launch_macro(int Q, int st, const MacroParams& mp, int rheo, bool odd, cudaStream_t s);
cudaError_t launch_get_pops(int Q, int st, const StepParams& p, bool odd, float* out, cudaStream_t s);
cudaError_t launch_set_pops(int Q, int st, const StepParams& p, const float* in, float rho, float ux, float uy,
                            float uz, cudaStream_t s);
// One batched step of the lattices of a (Q, storage, op, rheology) group that
// share the AA parity `odd`: ntiles table entries walked by `grid` persistent
// blocks of 256 threads.
cudaError_t launch_batched(int Q, int st, const BatchLaunch* L, const BatchState* state, const BatchBlock* table,
                           int ntiles, int grid, bool odd, int op, int rheo, cudaStream_t s);
// Copy a population array from layout (sH, sB) into layout (dH, dB) (pairH and
// pairBlk of each; sH = 0 is the natural layout).
cudaError_t launch_relayout(int Q, int st, const void* src, void* dst, int nx, int ny, long long N, int sH, int sB,
                            int dH, int dB, cudaStream_t s);
// Copy two halo messages (msgs[0], msgs[1]: the populations with c_z == dz of
// plane z) between the population array (layout H, blk) and dense buffers in
// one launch (unpack: buffers -> array).
cudaError_t launch_halo(int Q, int st, void* pop, const HaloSpec* msgs, int nx, int ny, long long N, int H,
                        int blk, bool unpack, cudaStream_t s);
// Resident 256-thread blocks per SM of the batched kernel of a group.
int batched_blocks_per_sm(int Q, int st, int op, int rheo);
template <int Q, int ST>
int batched_occupancy_st(int op, int rheo);
// Advance the per-lattice step state of nslots lattices (parity, side buffer, boundary flag).
cudaError_t launch_batch_advance(BatchState* state, int nslots, cudaStream_t s);

}  // namespace vlbm
