// capi.cu -- C ABI of the fluid time step (include/vlbm.h).
#include <cuda_runtime.h>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>
#include "sim.h"
#include "lattice.cuh"

namespace vlbm {

static thread_local std::string g_last_error;

// Step field of getVarFilename (lbmReport.cpp:55-83): the zeros counted by its
// loop (k >= 1 while step * 10^k < 10^6, unsigned arithmetic), then the step;
// step 0 gets six zeros before its "0", so the first save reads
// ..._rho0000000.bin and later ones ..._rho000100.bin.
std::string step_field(uint32_t step) {
    std::string num;
    if (step == 0) {
        num = "000000";
    } else {
        uint32_t pot = 10;
        for (int k = 0; k < 12 && step * pot < 1000000u; ++k, pot *= 10) num.push_back('0');
    }
    return num + std::to_string(step);
}

// mkdir -p (folderSetup, lbmReport.cpp:25-52)
void mkdir_p(const std::string& dir) {
    std::string acc;
    for (size_t k = 0; k <= dir.size(); ++k) {
        if (k == dir.size() || dir[k] == '/') {
            if (!acc.empty()) mkdir(acc.c_str(), 0777);
        }
        if (k < dir.size()) acc.push_back(dir[k]);
    }
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

vlbm_status cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return VLBM_OK;
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VLBM_ERR_NOMEM : VLBM_ERR_CUDA;
}

#define VLBM_CUDA(call)                                              \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return cuda_status(e_, #call);        \
    } while (0)

static float default_scale(int storage) { return storage == VLBM_STORE_F16 ? 4096.0f : 1.0f; }

vlbm_status sim_validate_config(const vlbm_config& c, std::string& why) {
    if (c.nx < 1 || c.ny < 1 || c.nz < 1) { why = "lattice sizes must be >= 1"; return VLBM_ERR_INVALID; }
    const long long N = (long long)c.nx * c.ny * c.nz;
    if (N >= (1LL << 31)) { why = "lattice has 2^31 nodes or more"; return VLBM_ERR_INVALID; }
    if (c.vel_set != 19 && c.vel_set != 27) { why = "vel_set must be 19 or 27"; return VLBM_ERR_INVALID; }
    if (c.collision != VLBM_OP_REGULARIZED && c.collision != VLBM_OP_BGK) { why = "unknown collision operator"; return VLBM_ERR_INVALID; }
    if (c.rheology < VLBM_NEWTONIAN || c.rheology > VLBM_POWERLAW) { why = "unknown rheology"; return VLBM_ERR_INVALID; }
    if (c.storage < VLBM_STORE_F32 || c.storage > VLBM_STORE_BF16) { why = "unknown storage"; return VLBM_ERR_INVALID; }
    if (c.layout < VLBM_LAYOUT_AUTO || c.layout > VLBM_LAYOUT_ZPAIR) { why = "unknown layout"; return VLBM_ERR_INVALID; }
    if (c.rheology == VLBM_NEWTONIAN && !(c.tau > 0.5)) { why = "tau must be > 0.5"; return VLBM_ERR_INVALID; }
    if (c.rheology == VLBM_BINGHAM && !(c.eta_p > 0.0 && c.yield_stress >= 0.0)) { why = "Bingham needs eta_p > 0, yield_stress >= 0"; return VLBM_ERR_INVALID; }
    if (c.rheology == VLBM_POWERLAW && !(c.n_index > 0.0 && c.k_consistency > 0.0)) { why = "Power-Law needs n_index > 0, k_consistency > 0"; return VLBM_ERR_INVALID; }
    if (!(c.rho0 > 0.0)) { why = "rho0 must be > 0"; return VLBM_ERR_INVALID; }
    if (c.slab_nz_total != 0 &&
        !(c.nz >= 3 && c.nz <= c.slab_nz_total + 2 && c.slab_z_offset >= 0 && c.slab_z_offset < c.slab_nz_total)) {
        why = "a z-slab needs 3 <= nz <= slab_nz_total + 2 (ghost planes included) and 0 <= slab_z_offset < "
              "slab_nz_total";
        return VLBM_ERR_INVALID;
    }
    if (c.storage == VLBM_STORE_F16 && c.storage_scale > 0) {   // 2^k, 0 <= k <= 24
        int e = 0;
        const double m = std::frexp(c.storage_scale, &e);
        if (m != 0.5 || e < 1 || e > 25) { why = "FP16 storage_scale must be a power of two from 1 to 2^24"; return VLBM_ERR_INVALID; }
    }
    return VLBM_OK;
}

StepParams make_params(vlbm_sim* s) {
    StepParams p;
    std::memset(&p, 0, sizeof(p));
    const vlbm_config& c = s->cfg;
    p.pop = s->pop;
    p.cls = s->cls;
    p.bc_slot = s->bc_slot;
    p.bc = s->bc;
    p.bc_q = s->bc_q;
    p.side_prev = s->side[s->side_cur];
    p.side_next = s->side[s->side_cur ^ 1];
    p.omega = s->omega;
    p.fibm = s->fibm;
    p.err = s->err;
    p.nx = c.nx; p.ny = c.ny; p.nz = c.nz;
    p.N = s->N;
    p.nbc = s->nbc;
    p.pairH = s->pairH;
    p.pairBlk = s->pairBlk;
    p.special_pairs = s->special_pairs;
    p.n_special = s->n_special;
    p.apply_bc = s->apply_bc;
    p.ctr = s->step_ctr;
    p.omega_newt = (float)(1.0 / c.tau);                 // var.h:105 OMEGA
    p.fx = (float)c.fx; p.fy = (float)c.fy; p.fz = (float)c.fz;
    p.omega_p = (float)(1.0 / (3.0 * c.eta_p + 0.5));    // nnf.h:23 OMEGA_P
    p.yield = (float)c.yield_stress;
    p.n_index = (float)c.n_index;
    p.k_cons = (float)c.k_consistency;
    p.gamma0 = (float)c.gamma0;
    const float sc = c.storage_scale > 0 ? (float)c.storage_scale : default_scale(c.storage);
    p.scale = sc;
    p.inv_scale = 1.0f / sc;
    p.rho0 = (float)c.rho0;
    return p;
}

vlbm_status fluid_step(vlbm_sim* s) {
    StepParams p = make_params(s);
    LaunchShape ls{s->block};
    cudaError_t e = launch_step(s->Q, s->cfg.storage, p, s->cfg.collision, s->cfg.rheology, s->parity == 1, ls,
                                s->stream);
    if (e != cudaSuccess) return cuda_status(e, "fused step launch");
    s->parity ^= 1;
    s->side_cur ^= 1;
    s->apply_bc = 1;
    s->step += 1;
    return VLBM_OK;
}

cudaError_t alloc_with(DeviceAllocator* a, void** p, size_t bytes) {
    return a ? a->allocate(p, bytes) : cudaMalloc(p, bytes);
}
void free_with(DeviceAllocator* a, void* p) {
    if (!p) return;
    if (a) a->release(p);
    else cudaFree(p);
}
cudaError_t sim_malloc(vlbm_sim* s, void** p, size_t bytes) { return alloc_with(s->allocator, p, bytes); }
void sim_free(vlbm_sim* s, void* p) { free_with(s->allocator, p); }

static vlbm_status alloc_dev(vlbm_sim* s, void** p, size_t bytes) {
    cudaError_t e = sim_malloc(s, p, bytes);
    if (e != cudaSuccess) return cuda_status(e, "device allocation");
    s->device_bytes += bytes;
    return VLBM_OK;
}

// Side store of the boundary nodes at rest equilibrium.  It holds
// post-collision deviations g_i = f_i - w_i rho0, zero at rest.
__global__ void k_fill_side(float* s0, float* s1, int nbc, int Q) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)Q * nbc) return;
    s0[k] = 0.f;
    s1[k] = 0.f;
}

__global__ void k_set_step_ctr(unsigned* ctr, int parity, unsigned step) { ctr[parity & 1] = step; }

cudaError_t sync_step_ctr(vlbm_sim* s, cudaStream_t stream) {
    k_set_step_ctr<<<1, 1, 0, stream>>>(s->step_ctr, s->parity, (unsigned)s->step);
    return cudaGetLastError();
}

// Class bytes and slot indices of the boundary nodes (all others stay bulk).
__global__ void k_scatter_bc(const int32_t* bc_node, int nbc, uint8_t* cls, int32_t* bc_slot) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nbc) return;
    const int32_t n = bc_node[s];
    cls[n] = NODE_BC;
    bc_slot[n] = s;
}

// Nodes outside the fluid (map bit IS_USED clear, lbm.cu:23-24).
__global__ void k_mark_unused(const int32_t* nodes, long long count, uint8_t* cls) {
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    cls[nodes[k]] = NODE_UNUSED;
}

static vlbm_status fill_side_equilibrium(vlbm_sim* s) {
    if (s->nbc == 0) return VLBM_OK;
    const long long tot = (long long)s->Q * s->nbc;
    k_fill_side<<<(unsigned)((tot + 255) / 256), 256, 0, s->stream>>>(s->side[0], s->side[1], s->nbc, s->Q);
    VLBM_CUDA(cudaGetLastError());
    if (!s->async_setup) VLBM_CUDA(cudaStreamSynchronize(s->stream));
    return VLBM_OK;
}

// Pair-nodes m (nodes m and m + M, M = N/2) with a boundary or unused node:
// the pair step's bulk kernel leaves them to k_step2, which runs this list.
// The list is filled in any order (every node pair reads and writes only its
// own slots, so the order does not change the result).
__global__ void k_special_pairs(const uint8_t* cls, long long M, int32_t* list, int* count) {
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    if ((cls[m] | cls[m + M]) & (NODE_BC | NODE_UNUSED)) list[atomicAdd(count, 1)] = (int32_t)m;
}

// Z-paired pairs in blocks of 32: NX a multiple of 32 and the blocked
// offsets within 32 bits.
static int blocked_pairs_ok(const vlbm_sim* s) {
    return (s->cfg.nx % 32 == 0 && (s->N / 2) * s->Q < (1ll << 31)) ? 1 : 0;
}

// host_count >= 0: the number of listed pairs, known on the host (a set-up
// without host waits); else it is read back from the device.
static vlbm_status build_pair_tiles(vlbm_sim* s, long long host_count = -1) {
    if (s->pairH <= 0) return VLBM_OK;
    const long long M = s->N / 2;
    vlbm_status st;
    void* p;
    if (!s->special_pairs) {
        if ((st = alloc_dev(s, &p, (size_t)M * sizeof(int32_t) + sizeof(int32_t))) != VLBM_OK) return st;
        s->special_pairs = static_cast<int32_t*>(p);
    }
    int* count = s->special_pairs + M;   // the counter sits behind the list
    VLBM_CUDA(cudaMemsetAsync(count, 0, sizeof(int), s->stream));
    k_special_pairs<<<(unsigned)((M + 255) / 256), 256, 0, s->stream>>>(s->cls, M, s->special_pairs, count);
    VLBM_CUDA(cudaGetLastError());
    if (host_count >= 0) {
        s->n_special = (int)host_count;
        return VLBM_OK;
    }
    int n = 0;
    VLBM_CUDA(cudaMemcpyAsync(&n, count, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    s->n_special = n;
    return VLBM_OK;
}

// Install boundary tables: class bytes and slots (bulk everywhere, then the
// boundary nodes scattered on the device), the records and the side store.
static vlbm_status install_tables(vlbm_sim* s, const BcTables& t) {
    // the old tables are freed below: wait for work that may still read them
    // (a simulation set up without host waits has none yet)
    const bool wait = !s->async_setup;
    if (wait || s->geometry) VLBM_CUDA(cudaStreamSynchronize(s->stream));
    sim_free(s, s->bc); sim_free(s, s->side[0]); sim_free(s, s->side[1]); sim_free(s, s->bc_node);
    sim_free(s, s->bc_q);
    s->bc = nullptr; s->side[0] = s->side[1] = nullptr; s->bc_node = nullptr; s->bc_q = nullptr;
    s->nbc = (int)t.recs.size();
    const size_t N = (size_t)s->N;
    VLBM_CUDA(cudaMemsetAsync(s->cls, 0, (N + 3) & ~(size_t)3, s->stream));
    VLBM_CUDA(cudaMemsetAsync(s->bc_slot, 0xff, N * sizeof(int32_t), s->stream));
    if (!t.unused_nodes.empty()) {
        const long long cnt = (long long)t.unused_nodes.size();
        void* d = nullptr;
        VLBM_CUDA(cudaMallocAsync(&d, (size_t)cnt * sizeof(int32_t), s->stream));
        cudaError_t e = sim_upload(s, d, t.unused_nodes.data(), (size_t)cnt * sizeof(int32_t));
        if (e == cudaSuccess) {
            k_mark_unused<<<(unsigned)((cnt + 255) / 256), 256, 0, s->stream>>>(static_cast<const int32_t*>(d), cnt,
                                                                               s->cls);
            e = cudaGetLastError();
        }
        cudaFreeAsync(d, s->stream);
        if (e == cudaSuccess && wait) e = cudaStreamSynchronize(s->stream);   // before the host list goes away
        VLBM_CUDA(e);
    }
    if (s->nbc > 0) {
        void* p;
        vlbm_status st;
        if ((st = alloc_dev(s, &p, t.recs.size() * sizeof(BcRec))) != VLBM_OK) return st;
        s->bc = static_cast<BcRec*>(p);
        if ((st = alloc_dev(s, &p, t.bc_nodes.size() * sizeof(int32_t))) != VLBM_OK) return st;
        s->bc_node = static_cast<int32_t*>(p);
        for (int b = 0; b < 2; ++b) {
            if ((st = alloc_dev(s, &p, (size_t)s->Q * s->nbc * sizeof(float))) != VLBM_OK) return st;
            s->side[b] = static_cast<float*>(p);
        }
        VLBM_CUDA(sim_upload(s, s->bc, t.recs.data(), t.recs.size() * sizeof(BcRec)));
        VLBM_CUDA(sim_upload(s, s->bc_node, t.bc_nodes.data(), t.bc_nodes.size() * sizeof(int32_t)));
        if (!t.q8.empty()) {
            if ((st = alloc_dev(s, &p, t.q8.size() * sizeof(float))) != VLBM_OK) return st;
            s->bc_q = static_cast<float*>(p);
            VLBM_CUDA(sim_upload(s, s->bc_q, t.q8.data(), t.q8.size() * sizeof(float)));
        }
        k_scatter_bc<<<(s->nbc + 255) / 256, 256, 0, s->stream>>>(s->bc_node, s->nbc, s->cls, s->bc_slot);
        VLBM_CUDA(cudaGetLastError());
        if ((st = fill_side_equilibrium(s)) != VLBM_OK) return st;   // synchronises the stream
    } else if (wait) {
        VLBM_CUDA(cudaStreamSynchronize(s->stream));
    }
    long long listed = -1;
    if (!wait && s->pairH > 0) {   // pairs holding a boundary or unused node, counted here
        const long long M = s->N / 2;
        std::vector<char> mark((size_t)M, 0);
        listed = 0;
        for (const std::vector<int32_t>* v : {&t.bc_nodes, &t.unused_nodes})
            for (int32_t n : *v) {
                const long long m = n < M ? n : n - M;
                if (!mark[(size_t)m]) { mark[(size_t)m] = 1; ++listed; }
            }
    }
    vlbm_status st = build_pair_tiles(s, listed);
    if (st != VLBM_OK) return st;
    s->geometry = true;
    return VLBM_OK;
}

vlbm_status sim_macroscopics_device(vlbm_sim* s, float* rho, float* ux, float* uy, float* uz, float* omega) {
    MacroParams mp;
    std::memset(&mp, 0, sizeof(mp));
    mp.s = make_params(s);
    mp.rho = rho; mp.ux = ux; mp.uy = uy; mp.uz = uz; mp.omega_out = omega;
    mp.fibm_const = nullptr;
    cudaError_t e = launch_macro(s->Q, s->cfg.storage, mp, s->cfg.rheology, s->parity == 1, s->stream);
    if (e != cudaSuccess) return cuda_status(e, "macroscopics launch");
    if (s->ibm) return ibm_macroscopics_fixup(s, rho, ux, uy, uz);
    return VLBM_OK;
}

vlbm_status ensure_scratch(vlbm_sim* s) {
    if (s->scratch) return VLBM_OK;
    void* p = nullptr;
    vlbm_status st = alloc_dev(s, &p, (size_t)5 * s->N * sizeof(float));
    if (st != VLBM_OK) return st;
    s->scratch = static_cast<float*>(p);
    return VLBM_OK;
}

}  // namespace vlbm

using namespace vlbm;

vlbm_sim::~vlbm_sim() {
    if (ibm) { ibm_destroy(ibm, allocator); ibm = nullptr; }
    for (void* p : {(void*)pop, (void*)cls, (void*)bc_slot, (void*)bc, (void*)bc_node, (void*)side[0], (void*)side[1],
                    (void*)omega, (void*)fibm, (void*)err, (void*)step_ctr, (void*)scratch, (void*)red_scratch, (void*)bc_q,
                    (void*)treat_prev, (void*)treat_red, (void*)special_pairs})
        free_with(allocator, p);
    if (allocator)
        for (void* h : staging) allocator->release_staging(h);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

cudaError_t vlbm::sim_upload(vlbm_sim* s, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    if (s->async_setup && s->allocator) {
        void* h = s->allocator->staging(bytes);
        if (h) {   // pinned: the copy is queued and the host returns at once
            std::memcpy(h, src, bytes);
            s->staging.push_back(h);
            return cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, s->stream);
        }
    }
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream);
}

#define CHECK_SIM(s)                                                        \
    do {                                                                    \
        if (!(s)) { set_last_error("null simulation handle"); return VLBM_ERR_INVALID; } \
        cudaError_t e_ = cudaSetDevice((s)->device);                        \
        if (e_ != cudaSuccess) return cuda_status(e_, "cudaSetDevice");     \
    } while (0)

extern "C" {

int vlbm_abi_version(void) { return VLBM_ABI_VERSION; }
const char* vlbm_last_error(void) { return g_last_error.c_str(); }

vlbm_status vlbm_config_default(vlbm_config* c) {
    if (!c) return VLBM_ERR_INVALID;
    std::memset(c, 0, sizeof(*c));
    c->nx = c->ny = 128; c->nz = 384;      // var.h:95-100 (N=128, NZ=3N)
    c->vel_set = VLBM_D3Q19;               // var.h:19
    c->collision = VLBM_OP_REGULARIZED;    // lbm.cu:263-461
    c->rheology = VLBM_NEWTONIAN;
    c->storage = VLBM_STORE_F32;           // var.h:18 SINGLE_PRECISION
    c->device = 0;
    c->tau = 0.6;                          // var.h:104
    c->rho0 = 1.0;                         // var.h:107
    c->eta_p = 0.3;                        // nnf.h:20
    c->yield_stress = 1e-4;                // nnf.h:21
    c->n_index = 0.5;                      // nnf.h:11
    c->k_consistency = c->rho0 * (c->tau - 0.5) / 3.0;  // nnf.h:12
    c->gamma0 = 0.0;                       // nnf.h:13
    const double umax = 0.1;               // var.h:102 U_MAX
    const double ux[8] = {0, umax, 0, 0, 0, 0, 0, 0};            // var.h:114
    const double uy[8] = {0, umax / 2, -umax / 2, 0, 0, 0, 0, 0}; // var.h:115
    const double uz[8] = {0, umax, -umax, 0, 0, 0, 0, 0};        // var.h:116
    const double rb[8] = {1, 1, 1, 1, 1, 1, 1, 1};               // var.h:117 (RHO_0 first)
    for (int i = 0; i < 8; ++i) { c->ux_bc[i] = ux[i]; c->uy_bc[i] = uy[i]; c->uz_bc[i] = uz[i]; c->rho_bc[i] = rb[i]; }
    c->storage_scale = 0.0;
    return VLBM_OK;
}

vlbm_status vlbm_create(const vlbm_config* cfg, vlbm_sim** out) { return sim_create(cfg, nullptr, out); }

}  // extern "C"

void vlbm::sim_release(vlbm_sim* s) {
    if (!s) return;
    cudaSetDevice(s->device);
    delete s;
}

vlbm_status vlbm::sim_create(const vlbm_config* cfg, DeviceAllocator* allocator, vlbm_sim** out,
                             bool async_setup) {
    if (!cfg || !out) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    *out = nullptr;
    std::string why;
    vlbm_status st = sim_validate_config(*cfg, why);
    if (st != VLBM_OK) { set_last_error(why); return st; }
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    vlbm_sim* s = new vlbm_sim();
    s->allocator = allocator;
    s->cfg = *cfg;
    s->Q = cfg->vel_set;
    s->N = (long long)cfg->nx * cfg->ny * cfg->nz;
    s->store_bytes = cfg->storage == VLBM_STORE_F32 ? 4 : 2;
    s->device = cfg->device;
    {   // population layout
        const bool even_z = cfg->nz % 2 == 0;
        int lay = cfg->layout;
        // two-node threads with packed FP32x2 arithmetic pay off where the step
        // is bound by instruction issue: 2-byte storage, and D3Q27 (measured on
        // B200: D3Q27 256^3 FP32 30.1 vs 28.3k MLUPS, FP16 37.7 vs 31.8k; D3Q19
        // FP32 is at the HBM roofline either way and keeps the natural layout)
        if (lay == VLBM_LAYOUT_AUTO)
            lay = ((cfg->storage != VLBM_STORE_F32 || cfg->vel_set == 27) && even_z) ? VLBM_LAYOUT_ZPAIR
                                                                                      : VLBM_LAYOUT_NATURAL;
        if (lay == VLBM_LAYOUT_ZPAIR && !even_z) { delete s; set_last_error("the z-paired layout needs an even nz"); return VLBM_ERR_INVALID; }
        s->pairH = lay == VLBM_LAYOUT_ZPAIR ? cfg->nz / 2 : 0;
        // pairs in blocks of 32 (one warp's pair-nodes, all Q populations
        // together) where NX is a multiple of 32 and the blocked offsets fit
        // 32 bits: the pair step then addresses every population from one
        // pointer (D3Q19 FP16 256^3: 57.6k against 53.3k MLUPS)
        s->pairBlk = s->pairH > 0 ? blocked_pairs_ok(s) : 0;
    }
    s->async_setup = async_setup;
    if (async_setup) {
        // set-up kernels that run while a long queue of other work holds the
        // SMs (a server admitting a lattice) are scheduled ahead of it
        int least = 0, greatest = 0;
        e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, greatest);
    } else {
        e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    }
    if (e != cudaSuccess) { delete s; return cuda_status(e, "cudaStreamCreate"); }
    s->own_stream = true;
    const size_t N = (size_t)s->N;
    void* p;
    if ((st = alloc_dev(s, &p, (size_t)s->Q * N * s->store_bytes)) != VLBM_OK) { delete s; return st; }
    s->pop = p;
    // class bytes, padded to whole 32-bit words
    const size_t cls_bytes = (N + 3) & ~(size_t)3;
    if ((st = alloc_dev(s, &p, cls_bytes)) != VLBM_OK) { delete s; return st; }
    s->cls = static_cast<uint8_t*>(p);
    if ((st = alloc_dev(s, &p, N * sizeof(int32_t))) != VLBM_OK) { delete s; return st; }
    s->bc_slot = static_cast<int32_t*>(p);
    if ((st = alloc_dev(s, &p, sizeof(unsigned int))) != VLBM_OK) { delete s; return st; }
    s->err = static_cast<unsigned int*>(p);
    if ((st = alloc_dev(s, &p, 2 * sizeof(unsigned int))) != VLBM_OK) { delete s; return st; }
    s->step_ctr = static_cast<unsigned int*>(p);
    if (cfg->rheology == VLBM_POWERLAW) {
        if ((st = alloc_dev(s, &p, N * sizeof(float))) != VLBM_OK) { delete s; return st; }
        s->omega = static_cast<float*>(p);
    }
    cudaMemsetAsync(s->cls, 0, cls_bytes, s->stream);
    cudaMemsetAsync(s->bc_slot, 0xff, N * sizeof(int32_t), s->stream);
    cudaMemsetAsync(s->err, 0, sizeof(unsigned int), s->stream);
    st = vlbm_init_equilibrium(s, cfg->rho0, 0.0, 0.0, 0.0);
    if (st != VLBM_OK) { delete s; return st; }
    *out = s;
    return VLBM_OK;
}

extern "C" {

vlbm_status vlbm_destroy(vlbm_sim* s) {
    if (!s) return VLBM_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete s;
    return VLBM_OK;
}

vlbm_status vlbm_set_node_map(vlbm_sim* s, const uint32_t* map, size_t n) {
    CHECK_SIM(s);
    if (!map) { set_last_error("null node map"); return VLBM_ERR_INVALID; }
    std::string why;
    BcTables t;
    vlbm_status st = build_bc_tables(s->cfg, map, n, t, why);
    if (st != VLBM_OK) { set_last_error(why); return st; }
    return install_tables(s, t);
}

vlbm_status vlbm_set_builder(vlbm_sim* s, int32_t builder) {
    CHECK_SIM(s);
    std::string why;
    BcTables t;
    vlbm_status st = build_bc_tables_builder(s->cfg, builder, t, why);
    if (st != VLBM_OK) { set_last_error(why); return st; }
    return install_tables(s, t);
}

vlbm_status vlbm_init_equilibrium(vlbm_sim* s, double rho, double ux, double uy, double uz) {
    CHECK_SIM(s);
    StepParams p = make_params(s);
    VLBM_CUDA(launch_set_pops(s->Q, s->cfg.storage, p, nullptr, (float)rho, (float)ux, (float)uy, (float)uz,
                              s->stream));
    s->parity = 0;
    s->apply_bc = 0;     // the initial state carries no boundary rule (main.cu:204-213)
    s->step = 0;
    s->treat_prev_valid = false;
    VLBM_CUDA(sync_step_ctr(s, s->stream));
    if (s->fibm) VLBM_CUDA(cudaMemsetAsync(s->fibm, 0, (size_t)3 * s->N * sizeof(float), s->stream));
    if (s->nbc > 0) { vlbm_status st = fill_side_equilibrium(s); if (st != VLBM_OK) return st; }
    if (s->ibm) ibm_reset(s);
    if (!s->async_setup) VLBM_CUDA(cudaStreamSynchronize(s->stream));
    return VLBM_OK;
}

vlbm_status vlbm_step(vlbm_sim* s, uint32_t nsteps) {
    CHECK_SIM(s);
    if (!s->geometry) { set_last_error("vlbm_set_node_map must be called before vlbm_step"); return VLBM_ERR_STATE; }
    for (uint32_t k = 0; k < nsteps; ++k) {
        vlbm_status st = fluid_step(s);
        if (st != VLBM_OK) return st;
        if (s->ibm) {
            st = ibm_step(s);
            if (st != VLBM_OK) return st;
        }
    }
    return VLBM_OK;
}

vlbm_status vlbm_sync(vlbm_sim* s) {
    CHECK_SIM(s);
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    unsigned int h = 0;
    VLBM_CUDA(cudaMemcpy(&h, s->err, sizeof(h), cudaMemcpyDeviceToHost));
    if (h) {
        VLBM_CUDA(cudaMemset(s->err, 0, sizeof(unsigned int)));
        set_last_error("non-finite or non-positive density detected on the device");
        return VLBM_ERR_DIVERGED;
    }
    return VLBM_OK;
}

vlbm_status vlbm_set_stream(vlbm_sim* s, void* stream) {
    CHECK_SIM(s);
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    if (stream) {
        s->stream = static_cast<cudaStream_t>(stream);
        s->own_stream = false;
    } else {
        VLBM_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    return VLBM_OK;
}

vlbm_status vlbm_get_macroscopics_device(vlbm_sim* s, float* rho, float* ux, float* uy, float* uz, float* omega) {
    CHECK_SIM(s);
    return sim_macroscopics_device(s, rho, ux, uy, uz, omega);
}

vlbm_status vlbm_get_macroscopics(vlbm_sim* s, float* rho, float* ux, float* uy, float* uz, float* omega) {
    CHECK_SIM(s);
    vlbm_status st = ensure_scratch(s);
    if (st != VLBM_OK) return st;
    const size_t N = (size_t)s->N;
    float* d[5] = {s->scratch, s->scratch + N, s->scratch + 2 * N, s->scratch + 3 * N, s->scratch + 4 * N};
    st = sim_macroscopics_device(s, d[0], d[1], d[2], d[3], d[4]);
    if (st != VLBM_OK) return st;
    float* h[5] = {rho, ux, uy, uz, omega};
    for (int k = 0; k < 5; ++k)
        if (h[k]) VLBM_CUDA(cudaMemcpyAsync(h[k], d[k], N * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    return VLBM_OK;
}

vlbm_status vlbm_get_populations(vlbm_sim* s, float* pops, size_t n) {
    CHECK_SIM(s);
    if (!pops || n != (size_t)s->Q * s->N) { set_last_error("population buffer size must be Q*N"); return VLBM_ERR_INVALID; }
    void* d = nullptr;
    VLBM_CUDA(cudaMallocAsync(&d, n * sizeof(float), s->stream));
    StepParams p = make_params(s);
    cudaError_t e = launch_get_pops(s->Q, s->cfg.storage, p, s->parity == 1, static_cast<float*>(d), s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pops, d, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
    cudaFreeAsync(d, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return cuda_status(e, "vlbm_get_populations");
}

vlbm_status vlbm_set_populations(vlbm_sim* s, const float* pops, size_t n) {
    CHECK_SIM(s);
    if (!pops || n != (size_t)s->Q * s->N) { set_last_error("population buffer size must be Q*N"); return VLBM_ERR_INVALID; }
    void* d = nullptr;
    VLBM_CUDA(cudaMallocAsync(&d, n * sizeof(float), s->stream));
    cudaError_t e = cudaMemcpyAsync(d, pops, n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
    StepParams p = make_params(s);
    p.omega = nullptr;  // keep the omega state
    if (e == cudaSuccess) e = launch_set_pops(s->Q, s->cfg.storage, p, static_cast<const float*>(d), 0.f, 0.f, 0.f, 0.f, s->stream);
    cudaFreeAsync(d, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    s->parity = 0;
    s->apply_bc = 0;   // given populations already carry their boundary values
    s->treat_prev_valid = false;
    VLBM_CUDA(sync_step_ctr(s, s->stream));
    return cuda_status(e, "vlbm_set_populations");
}

vlbm_status vlbm_get_forces(vlbm_sim* s, float* fxyz, size_t n) {
    CHECK_SIM(s);
    if (!fxyz || n != (size_t)3 * s->N) { set_last_error("force buffer size must be 3*N"); return VLBM_ERR_INVALID; }
    const size_t N = (size_t)s->N;
    if (!s->fibm) {
        for (size_t k = 0; k < N; ++k) { fxyz[k] = (float)s->cfg.fx; fxyz[N + k] = (float)s->cfg.fy; fxyz[2 * N + k] = (float)s->cfg.fz; }
        return VLBM_OK;
    }
    VLBM_CUDA(cudaMemcpyAsync(fxyz, s->fibm, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    const float b[3] = {(float)s->cfg.fx, (float)s->cfg.fy, (float)s->cfg.fz};
    for (int a = 0; a < 3; ++a)
        for (size_t k = 0; k < N; ++k) fxyz[a * N + k] += b[a];
    return VLBM_OK;
}

vlbm_status vlbm_get_info(vlbm_sim* s, vlbm_info* info) {
    if (!s || !info) return VLBM_ERR_INVALID;
    std::memset(info, 0, sizeof(*info));
    info->nx = s->cfg.nx; info->ny = s->cfg.ny; info->nz = s->cfg.nz; info->q = s->Q;
    info->storage_bytes = s->store_bytes;
    info->step = s->step;
    info->n_bc_nodes = s->nbc;
    info->device_bytes = (int64_t)s->device_bytes;
    info->bytes_per_node_step = 2.0 * s->Q * s->store_bytes;
    info->last_kernel_variant = s->variant;
    info->layout = s->pairH == 0 ? 0 : (s->pairBlk ? 2 : 1);
    info->aa_parity = s->parity;
    ibm_counts(s, &info->n_particles, &info->n_lagrangian_nodes);
    return VLBM_OK;
}

vlbm_status vlbm_halo_bytes(vlbm_sim* s, size_t* bytes) {
    CHECK_SIM(s);
    if (!bytes) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    *bytes = (size_t)(s->Q == 19 ? 5 : 9) * s->cfg.nx * s->cfg.ny * (size_t)s->store_bytes;
    return VLBM_OK;
}

static vlbm_status halo_copy(vlbm_sim* s, const HaloSpec (&m)[2], bool unpack) {
    CHECK_SIM(s);
    if (!m[0].buf && !m[1].buf) { set_last_error("null halo message"); return VLBM_ERR_INVALID; }
    for (const HaloSpec& h : m)
        if (h.buf && (h.z < 0 || h.z >= s->cfg.nz || (h.dz != 1 && h.dz != -1))) {
            set_last_error("halo plane out of range or dz not +1 / -1");
            return VLBM_ERR_INVALID;
        }
    VLBM_CUDA(launch_halo(s->Q, s->cfg.storage, s->pop, m, s->cfg.nx, s->cfg.ny, s->N, s->pairH, s->pairBlk,
                          unpack, s->stream));
    return VLBM_OK;
}
vlbm_status vlbm_halo_pack(vlbm_sim* s, int32_t z, int32_t dz, void* dst) {
    const HaloSpec m[2] = {{dst, z, dz}, {nullptr, 0, 1}};
    return halo_copy(s, m, false);
}
vlbm_status vlbm_halo_unpack(vlbm_sim* s, int32_t z, int32_t dz, const void* src) {
    const HaloSpec m[2] = {{const_cast<void*>(src), z, dz}, {nullptr, 0, 1}};
    return halo_copy(s, m, true);
}
vlbm_status vlbm_halo_pack2(vlbm_sim* s, int32_t z0, int32_t dz0, void* dst0, int32_t z1, int32_t dz1, void* dst1) {
    const HaloSpec m[2] = {{dst0, z0, dz0}, {dst1, z1, dz1}};
    return halo_copy(s, m, false);
}
vlbm_status vlbm_halo_unpack2(vlbm_sim* s, int32_t z0, int32_t dz0, const void* src0, int32_t z1, int32_t dz1,
                              const void* src1) {
    const HaloSpec m[2] = {{const_cast<void*>(src0), z0, dz0}, {const_cast<void*>(src1), z1, dz1}};
    return halo_copy(s, m, true);
}

vlbm_status vlbm_set_variant(vlbm_sim* s, int32_t variant) {
    if (!s) return VLBM_ERR_INVALID;
    static const int blocks[] = {256, 64, 128, 256};
    if (variant < 0 || variant > 3) { set_last_error("unknown launch variant"); return VLBM_ERR_INVALID; }
    s->variant = variant;
    s->block = blocks[variant];
    return VLBM_OK;
}

// Switch the population layout of a simulation whose array already holds the
// new layout's values: pairH / pairBlk and, for the pair step, its tile lists.
static vlbm_status use_layout(vlbm_sim* s, int H, int blk) {
    s->pairH = H;
    s->pairBlk = H > 0 ? blk : 0;
    return build_pair_tiles(s);
}

vlbm_status vlbm_set_layout(vlbm_sim* s, int32_t layout) {
    CHECK_SIM(s);
    if (layout != VLBM_LAYOUT_NATURAL && layout != VLBM_LAYOUT_ZPAIR) {
        set_last_error("vlbm_set_layout takes VLBM_LAYOUT_NATURAL or VLBM_LAYOUT_ZPAIR");
        return VLBM_ERR_INVALID;
    }
    if (layout == VLBM_LAYOUT_ZPAIR && s->cfg.nz % 2 != 0) {
        set_last_error("the z-paired layout needs an even nz");
        return VLBM_ERR_INVALID;
    }
    const int H = layout == VLBM_LAYOUT_ZPAIR ? s->cfg.nz / 2 : 0;
    const int blk = H > 0 ? blocked_pairs_ok(s) : 0;
    s->cfg.layout = layout;
    if (H == s->pairH && blk == s->pairBlk) return VLBM_OK;
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    const size_t popb = (size_t)s->Q * s->N * s->store_bytes;
    void* copy = nullptr;
    VLBM_CUDA(cudaMalloc(&copy, popb));
    cudaError_t e = cudaMemcpyAsync(copy, s->pop, popb, cudaMemcpyDeviceToDevice, s->stream);
    if (e == cudaSuccess)
        e = launch_relayout(s->Q, s->cfg.storage, copy, s->pop, s->cfg.nx, s->cfg.ny, s->N, s->pairH, s->pairBlk, H,
                            blk, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    cudaFree(copy);
    if (e != cudaSuccess) return cuda_status(e, "relayout");
    return use_layout(s, H, blk);
}

// Project-written autotuner: per velocity set, storage and lattice size it
// times the launch shape (64, 128 or 256 threads per block) and, when the
// configuration leaves the layout to the library (VLBM_LAYOUT_AUTO, even NZ),
// the tile a thread advances: one node (natural layout) or the node pair (z,
// z + NZ/2) of the z-paired layout (in blocks of 32 pair-nodes where NX
// allows).  Each candidate runs whole even/odd step pairs on a copy of the
// state (moved into the candidate's layout by k_relayout, which copies the
// stored values); the state is then restored in the fastest layout and the
// fastest shape is kept.
vlbm_status vlbm_autotune(vlbm_sim* s, int32_t* chosen) {
    CHECK_SIM(s);
    if (!s->geometry) { set_last_error("set the node map before autotuning"); return VLBM_ERR_STATE; }
    VLBM_CUDA(cudaStreamSynchronize(s->stream));
    const size_t popb = (size_t)s->Q * s->N * s->store_bytes;
    const size_t sideb = (size_t)s->Q * s->nbc * sizeof(float);
    void *bp = nullptr, *bs0 = nullptr, *bs1 = nullptr, *bo = nullptr;
    VLBM_CUDA(cudaMalloc(&bp, popb));
    if (sideb) { VLBM_CUDA(cudaMalloc(&bs0, sideb)); VLBM_CUDA(cudaMalloc(&bs1, sideb)); }
    if (s->omega) VLBM_CUDA(cudaMalloc(&bo, (size_t)s->N * sizeof(float)));
    VLBM_CUDA(cudaMemcpy(bp, s->pop, popb, cudaMemcpyDeviceToDevice));
    if (sideb) { VLBM_CUDA(cudaMemcpy(bs0, s->side[0], sideb, cudaMemcpyDeviceToDevice));
                 VLBM_CUDA(cudaMemcpy(bs1, s->side[1], sideb, cudaMemcpyDeviceToDevice)); }
    if (bo) VLBM_CUDA(cudaMemcpy(bo, s->omega, (size_t)s->N * sizeof(float), cudaMemcpyDeviceToDevice));
    const int parity = s->parity, side_cur = s->side_cur, apply = s->apply_bc;
    const long long step = s->step;
    const int H0 = s->pairH, B0 = s->pairBlk;
    struct Layout { int H, blk; };
    std::vector<Layout> layouts{{H0, B0}};
    if (s->cfg.layout == VLBM_LAYOUT_AUTO && s->cfg.nz % 2 == 0) {
        if (H0 > 0) layouts.push_back({0, 0});
        else layouts.push_back({s->cfg.nz / 2, blocked_pairs_ok(s)});
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    float best = 1e30f;
    int bestv = 3;
    Layout bestl = layouts[0];
    const int reps = s->N > (1 << 22) ? 4 : 20;
    vlbm_status st = VLBM_OK;
    for (const Layout& l : layouts) {
        if (l.H != s->pairH || l.blk != s->pairBlk) {
            cudaError_t e = launch_relayout(s->Q, s->cfg.storage, bp, s->pop, s->cfg.nx, s->cfg.ny, s->N, H0, B0, l.H,
                                            l.blk, s->stream);
            if (e != cudaSuccess) { st = cuda_status(e, "relayout"); break; }
            if ((st = use_layout(s, l.H, l.blk)) != VLBM_OK) break;
        }
        for (int v = 1; v <= 3; ++v) {
            vlbm_set_variant(s, v);
            for (int w = 0; w < 2; ++w) fluid_step(s);
            cudaEventRecord(e0, s->stream);
            for (int r = 0; r < reps; ++r) fluid_step(s);
            cudaEventRecord(e1, s->stream);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; bestv = v; bestl = l; }
        }
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    if (st == VLBM_OK) {   // the saved state, in the fastest layout
        cudaError_t e = (bestl.H == H0 && bestl.blk == B0)
                            ? cudaMemcpy(s->pop, bp, popb, cudaMemcpyDeviceToDevice)
                            : launch_relayout(s->Q, s->cfg.storage, bp, s->pop, s->cfg.nx, s->cfg.ny, s->N, H0, B0,
                                              bestl.H, bestl.blk, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) st = cuda_status(e, "autotune restore");
        else if (bestl.H != s->pairH || bestl.blk != s->pairBlk) st = use_layout(s, bestl.H, bestl.blk);
    }
    if (sideb) { VLBM_CUDA(cudaMemcpy(s->side[0], bs0, sideb, cudaMemcpyDeviceToDevice));
                 VLBM_CUDA(cudaMemcpy(s->side[1], bs1, sideb, cudaMemcpyDeviceToDevice)); }
    if (bo) VLBM_CUDA(cudaMemcpy(s->omega, bo, (size_t)s->N * sizeof(float), cudaMemcpyDeviceToDevice));
    cudaFree(bp); cudaFree(bs0); cudaFree(bs1); cudaFree(bo);
    s->parity = parity; s->side_cur = side_cur; s->apply_bc = apply; s->step = step;
    sync_step_ctr(s, s->stream);
    if (st != VLBM_OK) return st;
    vlbm_set_variant(s, bestv);
    if (chosen) *chosen = bestv;
    VLBM_CUDA(cudaGetLastError());
    return VLBM_OK;
}

// lbmReport.cpp:55-83 file names: PATH/ID/ID_<var><step, 6 digits>.bin;
// saveAllMacrBin lbmReport.cpp:133-172: raw little-endian floats [NZ][NY][NX].
vlbm_status vlbm_write_macr_bin(vlbm_sim* s, const char* path_files, const char* id_sim, uint32_t step_label,
                                int32_t export_forces) {
    CHECK_SIM(s);
    if (!path_files || !id_sim) { set_last_error("null path"); return VLBM_ERR_INVALID; }
    const size_t N = (size_t)s->N;
    std::vector<float> rho(N), ux(N), uy(N), uz(N), om(N);
    bool nnf = s->cfg.rheology != VLBM_NEWTONIAN;
    vlbm_status st = vlbm_get_macroscopics(s, rho.data(), ux.data(), uy.data(), uz.data(), nnf ? om.data() : nullptr);
    if (st != VLBM_OK) return st;
    const std::string dir = std::string(path_files) + "/" + id_sim;
    vlbm::mkdir_p(dir);
    const std::string num = vlbm::step_field(step_label);
    auto write = [&](const char* var, const float* data) -> vlbm_status {
        std::string fn = dir + "/" + id_sim + "_" + var + num + ".bin";
        FILE* f = std::fopen(fn.c_str(), "wb");
        if (!f) { set_last_error("cannot open " + fn); return VLBM_ERR_IO; }
        size_t w = std::fwrite(data, sizeof(float), N, f);
        std::fclose(f);
        if (w != N) { set_last_error("short write " + fn); return VLBM_ERR_IO; }
        return VLBM_OK;
    };
    if ((st = write("rho", rho.data())) != VLBM_OK) return st;
    if ((st = write("ux", ux.data())) != VLBM_OK) return st;
    if ((st = write("uy", uy.data())) != VLBM_OK) return st;
    if ((st = write("uz", uz.data())) != VLBM_OK) return st;
    if (export_forces && s->ibm) {
        std::vector<float> fr(3 * N);
        if ((st = vlbm_get_forces(s, fr.data(), fr.size())) != VLBM_OK) return st;
        if ((st = write("fx", fr.data())) != VLBM_OK) return st;
        if ((st = write("fy", fr.data() + N)) != VLBM_OK) return st;
        if ((st = write("fz", fr.data() + 2 * N)) != VLBM_OK) return st;
    }
    if (nnf && (st = write("omega", om.data())) != VLBM_OK) return st;
    return VLBM_OK;
}

// Run-information file PATH/ID/ID_info.txt (getSimInfoString and
// saveSimInfo, lbmReport.cpp:174-386): the same sections, keys and number
// formats; MLUPS counts every node (main.cu:539-541) and the bandwidth is the
// algorithmic bytes of this library's step (one read and one write of each
// stored population) per second in units of 2^30 bytes (the reference's
// BYTES_PER_GB, main.cu:542-544, for its two-buffer scheme).
vlbm_status vlbm_write_info(vlbm_sim* s, const char* path_files, const char* id_sim, uint64_t total_steps,
                            double time_elapsed_s, int32_t report_steps, int32_t save_steps, double u_max) {
    CHECK_SIM(s);
    if (!path_files || !id_sim) { set_last_error("null path"); return VLBM_ERR_INVALID; }
    const vlbm_config& c = s->cfg;
    const double mlups = time_elapsed_s > 0 ? (double)total_steps * (double)s->N / 1e6 / time_elapsed_s : 0.0;
    const double bytes = 2.0 * s->Q * s->store_bytes * (double)s->N;
    const double bw = time_elapsed_s > 0 ? bytes * (double)total_steps / time_elapsed_s / (double)(1u << 30) : 0.0;
    std::string out;
    char b[4096];
    auto add = [&](const char* fmt, auto... args) {
        const int w = std::snprintf(b, sizeof(b), fmt, args...);
        if (w > 0) out.append(b, (size_t)(w < (int)sizeof(b) ? w : (int)sizeof(b) - 1));
    };
    add("%s", "---------------------------- SIMULATION INFORMATION ----------------------------\n");
    add("      Simulation ID: %s\n", id_sim);
    add("       Velocity set: D3Q%d\n", s->Q);
    add("%s", "          Precision: float\n");
    if (c.storage != VLBM_STORE_F32)
        add(" Population storage: %s deviations\n", c.storage == VLBM_STORE_F16 ? "float16" : "bfloat16");
    add("                 NX: %d\n                 NY: %d\n                 NZ: %d\n           NZ_TOTAL: %d\n",
        c.nx, c.ny, c.nz, c.nz);
    add("                Tau: %e\n               Umax: %e\n", c.tau, u_max);
    add("                 FX: %e\n                 FY: %e\n                 FZ: %e\n", c.fx, c.fy, c.fz);
    add("       Report steps: %d\n         Save steps: %d\n             Nsteps: %llu\n", report_steps, save_steps,
        (unsigned long long)total_steps);
    add("              MLUPS: %.1f\n          Bandwidht: %.1f (Gb/s)\n", mlups, bw);
    add("       Time elapsed: %.3f (s)\n            threads: (%d , 1, 1)\n", time_elapsed_s, s->block);
    add("%s", "--------------------------------------------------------------------------------\n");
    if (c.rheology != VLBM_NEWTONIAN) {
        add("%s", "\n------------------------------ NON NEWTONIAN FLUID -----------------------------\n");
        if (c.rheology == VLBM_POWERLAW)
            add("              Model: Power-Law\n        Power index: %e\n Consistency factor: %e\n"
                "            Gamma 0: %e\n", c.n_index, c.k_consistency, c.gamma0);
        else
            add("              Model: Bingham\n  Plastic viscosity: %e\n       Yield stress: %e\n"
                "      Plastic omega: %e\n", c.eta_p, c.yield_stress, 1.0 / (3.0 * c.eta_p + 0.5));
        add("%s", "--------------------------------------------------------------------------------\n");
    }
    out += ibm_info_section(s);
    cudaDeviceProp prop;
    VLBM_CUDA(cudaGetDeviceProperties(&prop, s->device));
    add("%s", "\n------------------------------- CUDA INFORMATION -------------------------------\n");
    add("\t      device number: %d\n\t               name: %s\n\t    multiprocessors: %d\n"
        "\t compute capability: %d.%d\n\t        ECC enabled: %d\n", s->device, prop.name,
        prop.multiProcessorCount, prop.major, prop.minor, prop.ECCEnabled);
    add("%s", "--------------------------------------------------------------------------------\n");
    const std::string dir = std::string(path_files) + "/" + id_sim;
    {   // mkdir -p (folderSetup, lbmReport.cpp:25-52)
        std::string acc;
        for (size_t k = 0; k <= dir.size(); ++k) {
            if ((k == dir.size() || dir[k] == '/') && !acc.empty()) mkdir(acc.c_str(), 0777);
            if (k < dir.size()) acc.push_back(dir[k]);
        }
    }
    const std::string fn = dir + "/" + id_sim + "_info.txt";
    FILE* f = std::fopen(fn.c_str(), "w");
    if (!f) { set_last_error("cannot open " + fn); return VLBM_ERR_IO; }
    const size_t wr = std::fwrite(out.data(), 1, out.size(), f);
    const int cl = std::fclose(f);
    if (wr != out.size() || cl != 0) { set_last_error("short write " + fn); return VLBM_ERR_IO; }
    return VLBM_OK;
}

}  // extern "C"
