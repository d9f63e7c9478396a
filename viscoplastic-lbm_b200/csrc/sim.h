// sim.h -- the simulation object behind the opaque vlbm_sim handle.
#pragma once
#include <cuda_runtime.h>
#include <memory>
#include <string>
#include <vector>
#include "internal.h"
#include "dispatch.h"

namespace vlbm {

struct IbmState;   // ibm.cu

struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

// Source of a simulation's device memory.  Without one a simulation uses
// cudaMalloc/cudaFree; the serving loop passes a cache that recycles the
// buffers of retired lattices, because cudaFree synchronises the whole device
// and would drain the work queued for the other lattices.
struct DeviceAllocator {
    virtual cudaError_t allocate(void** p, size_t bytes) = 0;
    virtual void release(void* p) = 0;
    // Pinned host memory for the uploads of a simulation built without host
    // waits (async_setup): held by the simulation until it is destroyed, when
    // its device work has completed.  nullptr: no staging, upload and wait.
    virtual void* staging(size_t) { return nullptr; }
    virtual void release_staging(void*) {}
    virtual ~DeviceAllocator() = default;
};

}  // namespace vlbm

struct vlbm_sim {
    vlbm_config cfg{};
    int Q = 19;
    long long N = 0;
    int store_bytes = 4;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // device state
    void* pop = nullptr;             // [Q][N] populations (AA in place)
    uint8_t* cls = nullptr;          // [N] node class
    int32_t* bc_slot = nullptr;      // [N]
    vlbm::BcRec* bc = nullptr;       // [nbc]
    int32_t* bc_node = nullptr;      // [nbc] node index of each boundary slot
    float* bc_q = nullptr;           // [nbc][8][3] interpolated bounce-back coefficients (or null)
    float* side[2] = {nullptr, nullptr};  // [Q][nbc] post-collision at boundary nodes
    int nbc = 0;
    int pairH = 0;                   // z-paired layout (NZ/2) or 0
    int pairBlk = 0;                 // z-paired pairs stored in blocks of 32 (pair_elem)
    int32_t* special_pairs = nullptr; // pair-nodes with a boundary or unused node (n_special), then a counter
    int n_special = 0;
    float* omega = nullptr;          // [N] Power-Law state
    float* fibm = nullptr;           // [3][N] IBM force (allocated with spheres)
    unsigned int* err = nullptr;     // device error word
    unsigned int* step_ctr = nullptr;  // [2] device step count by AA parity
    float* scratch = nullptr;        // [5][N] macroscopic output scratch (lazy)
    double* red_scratch = nullptr;   // FP64 reduction partials + result (lazy)
    float* treat_prev = nullptr;     // [3][N] velocity of the previous data report (lazy)
    double* treat_red = nullptr;     // data-report partial sums + results (lazy)
    bool treat_prev_valid = false;   // false: the previous velocity is zero
    size_t device_bytes = 0;

    // host state
    int parity = 0;                  // 0: natural layout, 1: swapped layout
    int side_cur = 0;                // side[side_cur] holds the last step's values
    int apply_bc = 0;                // boundary rules active for the next gather
    long long step = 0;
    bool geometry = false;
    int block = 256;                 // launch variant (threads per block)
    int variant = 0;

    vlbm::IbmState* ibm = nullptr;   // owned; released by ibm_destroy
    vlbm::DeviceAllocator* allocator = nullptr;   // not owned; nullptr: cudaMalloc/cudaFree
    // Built without host waits: set-up work stays queued on `stream` and its
    // uploads come from pinned staging buffers (allocator->staging), released
    // with the simulation.
    bool async_setup = false;
    std::vector<void*> staging;
    ~vlbm_sim();
};

namespace vlbm {

StepParams make_params(vlbm_sim* s);
// Write the host step count into the device counter slot of the current parity.
cudaError_t sync_step_ctr(vlbm_sim* s, cudaStream_t stream);
// Device memory of a simulation, through its allocator (if any).
cudaError_t sim_malloc(vlbm_sim* s, void** p, size_t bytes);
void sim_free(vlbm_sim* s, void* p);
cudaError_t alloc_with(DeviceAllocator* a, void** p, size_t bytes);
void free_with(DeviceAllocator* a, void* p);
// vlbm_create with a device-memory source (nullptr: cudaMalloc/cudaFree).
// async_setup: the set-up runs on a high-priority stream of its own without
// host waits (a server admitting a lattice while a long queue of other work
// holds the SMs); the caller orders later work after it with an event.
vlbm_status sim_create(const vlbm_config* cfg, DeviceAllocator* allocator, vlbm_sim** out,
                       bool async_setup = false);
// Upload `bytes` from host `src` to device `dst` on the simulation's stream:
// through a pinned staging copy when the simulation is built without host
// waits, else a plain copy after which the caller may wait.
cudaError_t sim_upload(vlbm_sim* s, void* dst, const void* src, size_t bytes);
// Free a simulation whose device work is known to be complete (no stream
// synchronisation).
void sim_release(vlbm_sim* s);
vlbm_status cuda_status(cudaError_t e, const char* what);
vlbm_status fluid_step(vlbm_sim* s);   // one fused step (no IBM)
vlbm_status sim_macroscopics_device(vlbm_sim* s, float* rho, float* ux, float* uy, float* uz, float* omega);
vlbm_status sim_validate_config(const vlbm_config& c, std::string& why);
// Allocate the [5][N] macroscopic scratch (rho, ux, uy, uz, omega) if needed.
vlbm_status ensure_scratch(vlbm_sim* s);

// FP64 mass/momentum reduction (reduce.cu)
int reduce_blocks(long long N);
cudaError_t launch_moments_sum(vlbm_sim* s, double* partials, double* out);

// A device range that a checkpoint saves and restores (checkpoint.cu).
struct StateRegion {
    uint32_t id;
    void* dev;
    size_t bytes;
};

// IBM hooks (ibm.cu)
void ibm_state_regions(vlbm_sim* s, std::vector<StateRegion>& out);
uint32_t ibm_record_bytes();   // bytes of one device particle record
vlbm_status ibm_step(vlbm_sim* s);
vlbm_status ibm_macroscopics_fixup(vlbm_sim* s, float* rho, float* ux, float* uy, float* uz);
void ibm_destroy(IbmState* st, DeviceAllocator* allocator);
void ibm_reset(vlbm_sim* s);
void ibm_counts(const vlbm_sim* s, int* np, int* nn);
int ibm_iterations(const vlbm_sim* s);
// IBM section of the run-information file (lbmReport.cpp:230-340); empty without spheres.
std::string ibm_info_section(const vlbm_sim* s);

}  // namespace vlbm
