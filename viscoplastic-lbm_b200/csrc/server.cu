// server.cu -- continuous-batching serving loop for many lattices on one GPU.
//
// The reference runs one compile-time configured simulation per process
// (src/CUDA/main.cu).  Here requests (each a full vlbm_config, a named builder,
// a step count and optional spheres) are queued, admitted in arrival order
// while the HBM budget and the slot limit allow, kept resident, advanced
// together, and retired at their step count:
//
//  * the small sphere-free lattices of one (velocity set, operator, rheology,
//    storage) group that share an AA parity advance in ONE persistent launch
//    of k_step_batched over a (lattice, tile) table; the side-store buffer and
//    boundary flag of each lattice live in device memory and are advanced by
//    k_batch_advance.  A sphere-free lattice that fills a wave of that kernel
//    by itself gets its own k_step launch.  Each lattice with spheres runs its
//    fluid and IBM launches on its own side stream (a graph branch that
//    overlaps the others).  A membership's first segment runs with direct
//    launches; once it has lasted a segment, one step is captured in a CUDA
//    graph per phase (steps since the tables were built, mod 2) and replayed
//    until the membership changes;
//  * pump() enqueues the steps in segments of at most kSegment steps and does
//    its host work (admission of queued requests, table rebuilds, graph
//    captures) while the GPU runs the previous segment.  A lattice that reaches
//    its step count is read out on the GPU (macroscopic ux and the divergence
//    word into pinned host memory, behind an event) and leaves the batch; when
//    the event has completed its completion is recorded and its device memory
//    goes back to the server's cache, which hands it to the next admitted
//    lattice without cudaFree (cudaFree would synchronise the device).
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>
#include "sim.h"
#include "step_impl.cuh"

namespace vlbm {

// After every lattice of the batch took its step.
__global__ void k_batch_advance(BatchState* state, int nslots) {
    // chained like the batched steps: wait for the step's last batched launch
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nslots) return;
    state[i].parity ^= 1;
    state[i].side_cur ^= 1;
    state[i].apply_bc = 1;
    state[i].step += 1;
}

cudaError_t launch_batch_advance(BatchState* state, int nslots, cudaStream_t s) {
    if (nslots <= 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((nslots + 127) / 128);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_batch_advance, state, nslots);
}

}  // namespace vlbm

using namespace vlbm;

namespace {

constexpr int kSegment = 64;          // steps enqueued between two host bookkeeping points
constexpr int kSegmentsInFlight = 8;  // the host waits when more segments are queued
constexpr size_t kKeptResults = 256;  // finished fields kept for vlbm_server_fetch

double now_s() {
    using clk = std::chrono::steady_clock;
    static const clk::time_point t0 = clk::now();
    return std::chrono::duration<double>(clk::now() - t0).count();
}

struct Pending {
    vlbm_request req;
    std::vector<vlbm_sphere> spheres;
    double submit_t;
    size_t bytes;
};

struct Resident {
    vlbm_sim* sim = nullptr;
    uint64_t tag = 0;
    uint64_t target = 0;
    double submit_t = 0, start_t = 0;
    size_t bytes = 0;
};

// Device bytes a request will hold: populations, class/slot arrays (5 B per
// node), the macroscopic read-out scratch used at retirement (20 B per node),
// the side store of the wall nodes (at most the six faces; cylinder walls are
// shorter but also carry 96 B of interpolation coefficients), the Power-Law
// state, the IBM fields and Lagrangian arrays, plus 1 MiB of small allocations.
size_t estimate_bytes(const vlbm_request& r) {
    const size_t N = (size_t)r.cfg.nx * r.cfg.ny * r.cfg.nz;
    const size_t sb = r.cfg.storage == VLBM_STORE_F32 ? 4 : 2;
    size_t b = (size_t)r.cfg.vel_set * N * sb + 25 * N + (1 << 20);
    const size_t walls = 2 * ((size_t)r.cfg.nx * r.cfg.ny + (size_t)r.cfg.ny * r.cfg.nz + (size_t)r.cfg.nx * r.cfg.nz);
    b += walls * (2 * (size_t)r.cfg.vel_set * 4 + 24);
    if (r.builder == VLBM_BUILDER_CIRCULAR_DUCT || r.builder == VLBM_BUILDER_ANNULAR_DUCT) b += walls * 96;
    if (r.cfg.rheology == VLBM_POWERLAW) b += 4 * N;
    if (r.n_spheres > 0) b += 56 * N + (size_t)r.n_spheres * 700 * 10 * 8;
    return b;
}

// The lattices of one kernel family that share the batched launches, in
// chunks of at most BATCH_MAX_SLOTS lattices of equal AA parity at the time
// the tables were built: a chunk of part b steps with parity b ^ ph at phase
// ph (steps since the rebuild, mod 2).
struct Chunk {
    int part;
    BatchLaunch L;        // the chunk's lattice parameters (uploaded to d_launch[launch_idx])
    size_t launch_idx;
    size_t table_off;
    int ntiles, grid;
};
struct Group {
    int Q, op, rheo, st;
    std::vector<Chunk> chunks;
};

// Device memory cache of the server.  Buffers released by retired lattices are
// kept and handed out again (best fit, at most 25 % + 2 MiB larger than asked);
// only trim() calls cudaFree.  A buffer is released only after the GPU has
// finished with its lattice (its read-out event completed).  The device memory
// the cache holds, live and cached together, stays within `cap` (the server's
// HBM budget) as long as the live buffers fit in it: a larger cached buffer is
// handed out only when it fits, and cached buffers are freed before a new
// allocation would pass the cap.
struct DevCache final : DeviceAllocator {
    std::multimap<size_t, void*> free_;
    std::unordered_map<void*, size_t> size_of;
    size_t free_bytes = 0, live_bytes = 0;
    size_t cap = ~(size_t)0;

    cudaError_t allocate(void** p, size_t bytes) override {
        const size_t need = (bytes + 511) & ~(size_t)511;
        auto it = free_.lower_bound(need);
        if (it != free_.end() && it->first <= need + need / 4 + ((size_t)2 << 20) &&
            (it->first == need || live_bytes + it->first <= cap)) {
            *p = it->second;
            free_bytes -= it->first;
            live_bytes += it->first;
            free_.erase(it);
            return cudaSuccess;
        }
        if (free_bytes + live_bytes + need > cap) trim(cap > live_bytes + need ? cap - live_bytes - need : 0);
        cudaError_t e = cudaMalloc(p, need);
        if (e == cudaErrorMemoryAllocation && !free_.empty()) {   // give the cached buffers back and retry
            cudaGetLastError();
            trim(0);
            e = cudaMalloc(p, need);
        }
        if (e != cudaSuccess) { *p = nullptr; return e; }
        size_of[*p] = need;
        live_bytes += need;
        return cudaSuccess;
    }
    void release(void* p) override {
        auto it = size_of.find(p);
        if (it == size_of.end()) return;
        free_.insert({it->second, p});
        free_bytes += it->second;
        live_bytes -= it->second;
    }
    // pinned staging for the uploads of admitted lattices, reused best fit
    std::multimap<size_t, void*> hfree_;
    std::vector<void*> hall_;
    std::unordered_map<void*, size_t> hsize_;
    void* staging(size_t bytes) override {
        const size_t need = (bytes + 4095) & ~(size_t)4095;
        auto it = hfree_.lower_bound(need);
        if (it != hfree_.end() && it->first <= 2 * need) {
            void* h = it->second;
            hfree_.erase(it);
            return h;
        }
        void* h = nullptr;
        if (cudaHostAlloc(&h, need, cudaHostAllocDefault) != cudaSuccess) { cudaGetLastError(); return nullptr; }
        hall_.push_back(h);
        hsize_[h] = need;
        return h;
    }
    void release_staging(void* h) override {
        auto it = hsize_.find(h);
        if (it != hsize_.end()) hfree_.insert({it->second, h});
    }
    void trim(size_t keep) {
        while (free_bytes > keep && !free_.empty()) {
            auto it = std::prev(free_.end());
            cudaFree(it->second);
            size_of.erase(it->second);
            free_bytes -= it->first;
            free_.erase(it);
        }
    }
    ~DevCache() override {
        trim(0);
        for (auto& kv : size_of) cudaFree(kv.first);   // nothing should be live here
        for (void* h : hall_) cudaFreeHost(h);
    }
};

// Pinned host buffers for read-outs, reused best fit; freed with the server.
struct PinnedPool {
    std::multimap<size_t, void*> free_;
    std::vector<void*> all;
    void* get(size_t bytes) {
        auto it = free_.lower_bound(bytes);
        if (it != free_.end() && it->first <= 2 * bytes + 4096) {
            void* p = it->second;
            free_.erase(it);
            return p;
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
        all.push_back(p);
        sizes[p] = bytes;
        return p;
    }
    void put(void* p) { if (p) free_.insert({sizes[p], p}); }
    std::unordered_map<void*, size_t> sizes;
    ~PinnedPool() { for (void* p : all) cudaFreeHost(p); }
};

// A lattice that reached its step count and is being read out.
struct Retiring {
    Resident r;
    float* d_ux = nullptr;        // device read-out of ux
    float* h_ux = nullptr;        // pinned copy
    unsigned* h_err = nullptr;    // pinned copy of the divergence word
    cudaEvent_t done = nullptr;
    vlbm_status status = VLBM_OK;
};

}  // namespace

struct vlbm_server {
    int device = 0;
    int sms = 148;
    size_t budget = 0;
    int max_resident = 64;
    cudaStream_t stream = nullptr;
    DevCache cache;
    PinnedPool pinned;
    std::deque<Pending> queue;
    std::vector<Resident> res;
    std::vector<Retiring> retiring;
    std::deque<cudaEvent_t> segments;   // one event per queued segment
    std::deque<vlbm_completion> done;
    std::deque<std::pair<uint64_t, std::vector<float>>> results;   // finished ux fields, by tag
    size_t bytes_in_use = 0;
    double lattice_updates = 0.0;
    // admit, rebuild, enqueue (incl. graph captures), wait, read-out [s];
    // batch steps, direct kernel launches, graph launches, graph captures
    double prof[16] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    // batch tables (rebuilt when the membership changes)
    bool dirty = true;
    BatchState* d_state = nullptr;
    BatchBlock* d_table = nullptr;
    BatchLaunch* d_launch = nullptr;    // one parameter block per chunk
    size_t cap_slots = 0, cap_table = 0, cap_launch = 0;
    std::vector<void*> old_tables;      // outgrown table buffers, freed with the server
    // pinned staging of the tables: a ring, so a rebuild does not wait for the
    // GPU to reach the previous upload (an entry is reused once its upload ran)
    struct Staging {
        BatchState* slots = nullptr;
        BatchBlock* table = nullptr;
        BatchLaunch* launch = nullptr;
        size_t cap_slots = 0, cap_table = 0, cap_launch = 0;
        cudaEvent_t uploaded = nullptr;
        bool pending = false;
    };
    Staging staging[4];
    int next_staging = 0;
    std::vector<void*> old_pinned;      // outgrown staging, freed with the server
    int stable_segments = 0;            // segments run since the last rebuild
    bool use_graphs = false;            // the batch's GPU step is short next to its launch cost
    long long own_launch_min_nodes = -1;  // -1: one wave of the batched kernel
    double last_launches = 0.0;         // kernel launches of the last enqueue_steps
    double capture_s = 0.0;             // host seconds in graph captures (part of enqueue)
    std::vector<Group> groups;
    int nslots = 0;
    int phase = 0;                 // steps since the last rebuild, mod 2
    std::vector<int> ibm_res;      // indices into res of lattices with spheres
    std::vector<int> own_res;      // indices into res of large sphere-free lattices
    std::vector<int> branch_res;   // both of the above: own launches on a side stream each
    std::vector<int> table_res;    // the lattices of the batched launches
    // per phase: graph of one step (captured once a membership has lasted a
    // segment; short captures, because memberships change often)
    cudaGraphExec_t graph1[2] = {nullptr, nullptr};
    // side streams of the lattices with spheres (graph branches)
    std::vector<cudaStream_t> side_streams;
    std::vector<cudaEvent_t> join_events;
    cudaEvent_t fork_event = nullptr;

    void drop_graphs() {
        for (int p = 0; p < 2; ++p) {
            if (graph1[p]) cudaGraphExecDestroy(graph1[p]);
            graph1[p] = nullptr;
        }
    }
    ~vlbm_server() {
        if (stream) cudaStreamSynchronize(stream);
        for (Resident& r : res) vlbm::sim_release(r.sim);
        for (Retiring& t : retiring) {
            vlbm::free_with(&cache, t.d_ux);
            vlbm::sim_release(t.r.sim);
            if (t.done) cudaEventDestroy(t.done);
        }
        for (cudaEvent_t e : segments) cudaEventDestroy(e);
        drop_graphs();
        cudaFree(d_state);
        cudaFree(d_table);
        cudaFree(d_launch);
        for (void* p : old_tables) cudaFree(p);
        for (Staging& g : staging) {
            if (g.slots) cudaFreeHost(g.slots);
            if (g.table) cudaFreeHost(g.table);
            if (g.launch) cudaFreeHost(g.launch);
            if (g.uploaded) cudaEventDestroy(g.uploaded);
        }
        for (void* p : old_pinned) cudaFreeHost(p);
        for (cudaStream_t t : side_streams) cudaStreamDestroy(t);
        for (cudaEvent_t e : join_events) cudaEventDestroy(e);
        if (fork_event) cudaEventDestroy(fork_event);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

vlbm_status server_rebuild(vlbm_server* sv) {
    sv->drop_graphs();
    sv->groups.clear();
    sv->ibm_res.clear();
    sv->table_res.clear();
    sv->branch_res.clear();
    sv->phase = 0;
    std::vector<BatchState> slots;
    std::vector<BatchBlock> table;
    auto key = [](const vlbm_sim* s) {
        const vlbm_config& c = s->cfg;
        return ((c.vel_set * 4 + c.collision) * 4 + c.rheology) * 4 + c.storage;
    };
    std::vector<int> order(sv->res.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const vlbm_sim *sa = sv->res[a].sim, *sb = sv->res[b].sim;
        return key(sa) != key(sb) ? key(sa) < key(sb) : sa->parity < sb->parity;
    });
    int cur = -1;
    sv->own_res.clear();
    // Lattices with spheres step on their own side stream (fluid and IBM
    // launches).  A sphere-free lattice that fills a wave of the batched kernel
    // by itself may get its own fused-step launches (parameters in the constant
    // bank, about 30 % faster per node than the batched kernel; a z-paired
    // lattice always does) on a side stream,
    // largest first, while the host time of all launches of a step stays below
    // about 60 % of the GPU time of the step; the rest share the batched
    // launches.  Estimates: 4 us of host time per launch, populations
    // streamed at 4.5 TB/s.
    std::vector<char> own(sv->res.size(), 0);
    {
        double gpu_us = 0.0, host_us = 4.0;   // the state-advance launch
        std::vector<std::pair<long long, int>> cand;
        for (size_t i = 0; i < sv->res.size(); ++i) {
            const vlbm_sim* s = sv->res[i].sim;
            gpu_us += 2.0 * s->Q * s->store_bytes * (double)s->N / 4.5e6;
            if (s->ibm) { host_us += 4.0 * (3.0 + 3.0 * std::max(1, ibm_iterations(s))); continue; }
            const long long wave = sv->own_launch_min_nodes >= 0
                                       ? sv->own_launch_min_nodes
                                       : (long long)std::max(1, batched_blocks_per_sm(s->Q, s->cfg.storage,
                                                                                      s->cfg.collision,
                                                                                      s->cfg.rheology)) *
                                             sv->sms * 256;
            if (s->N >= wave || s->pairH > 0) cand.emplace_back(s->N, (int)i);
            else host_us += 0.5;   // its share of the batched launches
        }
        std::sort(cand.begin(), cand.end(), std::greater<std::pair<long long, int>>());
        for (const auto& c : cand) {
            // a z-paired lattice cannot join the natural-layout table
            if (sv->res[c.second].sim->pairH > 0 || sv->own_launch_min_nodes >= 0 || host_us + 4.0 <= 0.6 * gpu_us) {
                own[c.second] = 1;
                host_us += 4.0;
            }
        }
    }
    for (int idx : order) {
        vlbm_sim* s = sv->res[idx].sim;
        if (s->ibm) { sv->ibm_res.push_back(idx); continue; }
        if (own[idx]) { sv->own_res.push_back(idx); continue; }
        sv->table_res.push_back(idx);
        const int k = key(s);
        if (k != cur) {
            sv->groups.push_back(Group{s->Q, s->cfg.collision, s->cfg.rheology, s->cfg.storage, {}});
            cur = k;
        }
        Group& g = sv->groups.back();
        const int part = s->parity;
        if (g.chunks.empty() || g.chunks.back().part != part ||
            (int)(slots.size() - g.chunks.back().L.state_base) >= BATCH_MAX_SLOTS) {
            g.chunks.emplace_back();
            Chunk& c = g.chunks.back();
            std::memset(&c.L, 0, sizeof(c.L));
            c.part = part;
            c.L.state_base = (int)slots.size();
            c.table_off = table.size();
            c.ntiles = 0;
            c.grid = 0;
        }
        Chunk& c = g.chunks.back();
        const int local = (int)slots.size() - c.L.state_base;
        StepParams pp = make_params(s);
        pp.side_prev = s->side[0];     // the kernel picks the current one from the state
        pp.side_next = s->side[1];
        c.L.p[local] = pp;
        BatchState bs;
        std::memset(&bs, 0, sizeof(bs));
        bs.parity = s->parity;
        bs.side_cur = s->side_cur;
        bs.apply_bc = s->apply_bc;
        bs.step = (unsigned)s->step;
        slots.push_back(bs);
        const unsigned nt = (unsigned)((s->N + BATCH_TILE - 1) / BATCH_TILE);
        for (unsigned t = 0; t < nt; ++t) table.push_back(BatchBlock{local, t * (unsigned)BATCH_TILE});
        c.ntiles += (int)nt;
    }
    std::vector<const BatchLaunch*> launch_src;   // chunk parameter blocks in upload order
    for (Group& g : sv->groups) {
        const int per_sm = std::max(1, batched_blocks_per_sm(g.Q, g.st, g.op, g.rheo));
        for (Chunk& c : g.chunks) {
            c.grid = std::min(c.ntiles, per_sm * sv->sms);
            c.launch_idx = launch_src.size();
            launch_src.push_back(&c.L);
        }
    }
    sv->branch_res = sv->ibm_res;
    sv->branch_res.insert(sv->branch_res.end(), sv->own_res.begin(), sv->own_res.end());
    // lattices with their own launches count their steps on the device (the
    // stochastic-rounding seed); one that stepped in the batched launch so far
    // resumes from its host count
    for (int idx : sv->branch_res) {
        cudaError_t e = sync_step_ctr(sv->res[idx].sim, sv->stream);
        if (e != cudaSuccess) return cuda_status(e, "step counter");
    }
    // one side stream and join event per lattice with its own launches
    while (sv->side_streams.size() < sv->branch_res.size()) {
        cudaStream_t t = nullptr;
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            if (t) cudaStreamDestroy(t);
            return cuda_status(e, "server side stream");
        }
        sv->side_streams.push_back(t);
        sv->join_events.push_back(ev);
    }
    if (!sv->fork_event) {
        cudaError_t e = cudaEventCreateWithFlags(&sv->fork_event, cudaEventDisableTiming);
        if (e != cudaSuccess) { sv->fork_event = nullptr; return cuda_status(e, "server fork event"); }
    }
    sv->nslots = (int)slots.size();
    // Grow the device tables without cudaFree (it synchronises the device):
    // outgrown buffers are kept until the server is destroyed.  The device
    // tables are rewritten in place: the upload is ordered after the queued
    // steps that still read them.
    if (slots.size() > sv->cap_slots) {
        const size_t cap = std::max<size_t>(256, slots.size() * 2);
        void* d = nullptr;
        if (cudaMalloc(&d, cap * sizeof(BatchState)) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("server slot table allocation failed");
            return VLBM_ERR_NOMEM;
        }
        if (sv->d_state) sv->old_tables.push_back(sv->d_state);
        sv->d_state = static_cast<BatchState*>(d);
        sv->cap_slots = cap;
    }
    if (table.size() > sv->cap_table) {
        const size_t cap = std::max<size_t>(1 << 16, table.size() * 2);
        void* d = nullptr;
        if (cudaMalloc(&d, cap * sizeof(BatchBlock)) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("server tile table allocation failed");
            return VLBM_ERR_NOMEM;
        }
        if (sv->d_table) sv->old_tables.push_back(sv->d_table);
        sv->d_table = static_cast<BatchBlock*>(d);
        sv->cap_table = cap;
    }
    if (launch_src.size() > sv->cap_launch) {
        const size_t cap = std::max<size_t>(16, launch_src.size() * 2);
        void* d = nullptr;
        if (cudaMalloc(&d, cap * sizeof(BatchLaunch)) != cudaSuccess) {
            cudaGetLastError();
            set_last_error("server launch table allocation failed");
            return VLBM_ERR_NOMEM;
        }
        if (sv->d_launch) sv->old_tables.push_back(sv->d_launch);
        sv->d_launch = static_cast<BatchLaunch*>(d);
        sv->cap_launch = cap;
    }
    if (!slots.empty()) {
        vlbm_server::Staging& g = sv->staging[sv->next_staging];
        sv->next_staging = (sv->next_staging + 1) % 4;
        cudaError_t e = cudaSuccess;
        if (g.pending) e = cudaEventSynchronize(g.uploaded);   // normally long complete
        g.pending = false;
        if (e == cudaSuccess && slots.size() > g.cap_slots) {
            void* h = nullptr;
            e = cudaHostAlloc(&h, sv->cap_slots * sizeof(BatchState), cudaHostAllocDefault);
            if (e == cudaSuccess) {
                if (g.slots) sv->old_pinned.push_back(g.slots);
                g.slots = static_cast<BatchState*>(h);
                g.cap_slots = sv->cap_slots;
            }
        }
        if (e == cudaSuccess && table.size() > g.cap_table) {
            void* h = nullptr;
            e = cudaHostAlloc(&h, sv->cap_table * sizeof(BatchBlock), cudaHostAllocDefault);
            if (e == cudaSuccess) {
                if (g.table) sv->old_pinned.push_back(g.table);
                g.table = static_cast<BatchBlock*>(h);
                g.cap_table = sv->cap_table;
            }
        }
        if (e == cudaSuccess && launch_src.size() > g.cap_launch) {
            void* h = nullptr;
            e = cudaHostAlloc(&h, sv->cap_launch * sizeof(BatchLaunch), cudaHostAllocDefault);
            if (e == cudaSuccess) {
                if (g.launch) sv->old_pinned.push_back(g.launch);
                g.launch = static_cast<BatchLaunch*>(h);
                g.cap_launch = sv->cap_launch;
            }
        }
        if (e == cudaSuccess && !g.uploaded) e = cudaEventCreateWithFlags(&g.uploaded, cudaEventDisableTiming);
        if (e == cudaSuccess) {
            std::memcpy(g.slots, slots.data(), slots.size() * sizeof(BatchState));
            std::memcpy(g.table, table.data(), table.size() * sizeof(BatchBlock));
            e = cudaMemcpyAsync(sv->d_state, g.slots, slots.size() * sizeof(BatchState), cudaMemcpyHostToDevice,
                                sv->stream);
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sv->d_table, g.table, table.size() * sizeof(BatchBlock), cudaMemcpyHostToDevice,
                                sv->stream);
        if (e == cudaSuccess && !launch_src.empty()) {
            for (size_t k = 0; k < launch_src.size(); ++k) std::memcpy(&g.launch[k], launch_src[k], sizeof(BatchLaunch));
            e = cudaMemcpyAsync(sv->d_launch, g.launch, launch_src.size() * sizeof(BatchLaunch),
                                cudaMemcpyHostToDevice, sv->stream);
        }
        if (e == cudaSuccess) e = cudaEventRecord(g.uploaded, sv->stream);
        if (e != cudaSuccess) return cuda_status(e, "server table upload");
        g.pending = true;
    }
    sv->stable_segments = 0;
    {   // graphs pay off where host launch time is comparable to the GPU step:
        // estimate both (about 4 us of host time per launch; the populations
        // streamed at about 4 TB/s, which the large lattices reach)
        double launches = 1.0 + (double)sv->own_res.size();
        for (const Group& g : sv->groups) launches += (double)g.chunks.size();
        double bytes = 0.0;
        for (const Resident& r : sv->res) {
            bytes += 2.0 * r.sim->Q * r.sim->store_bytes * (double)r.sim->N;
            if (r.sim->ibm) launches += 3.0 + 3.0 * std::max(1, ibm_iterations(r.sim));
        }
        const double host_us = 4.0 * launches, gpu_us = bytes / 4.0e6;
        sv->use_graphs = gpu_us < 3.0 * host_us;
    }
    sv->dirty = false;
    return VLBM_OK;
}

// Host mirror of the state every lattice advanced on the device.
void advance_host(vlbm_sim* s) {
    s->parity ^= 1;
    s->side_cur ^= 1;
    s->apply_bc = 1;
    s->step += 1;
}

// Enqueue `n` steps of every resident lattice (directly or into a stream
// capture of the server stream).  Server stream, per step: the batched launches
// of each group and parity part, the slot-state advance, then one k_step launch
// per large lattice.  Each lattice with spheres runs its n steps (fluid launch
// then IBM step) on its own side stream, forked from the server stream before
// the first step and joined after the last, so sphere lattices overlap each
// other and the batched work.  Advances the host mirrors and the phase.
vlbm_status enqueue_steps(vlbm_server* sv, int n) {
    cudaError_t e = cudaSuccess;
    if (!sv->branch_res.empty()) {
        e = cudaEventRecord(sv->fork_event, sv->stream);
        if (e != cudaSuccess) return cuda_status(e, "fork event");
    }
    double launches = 0.0;
    for (int i = 0; i < n; ++i) {
        for (const Group& g : sv->groups)
            for (const Chunk& c : g.chunks) {
                const bool odd = (c.part ^ sv->phase) != 0;
                e = launch_batched(g.Q, g.st, sv->d_launch + c.launch_idx, sv->d_state, sv->d_table + c.table_off,
                                   c.ntiles, c.grid, odd, g.op,
                                   g.rheo, sv->stream);
                if (e != cudaSuccess) return cuda_status(e, "batched step");
                launches += 1.0;
            }
        if (sv->nslots > 0) {
            e = launch_batch_advance(sv->d_state, sv->nslots, sv->stream);
            if (e != cudaSuccess) return cuda_status(e, "batch advance");
            launches += 1.0;
        }
        sv->phase ^= 1;
    }
    for (int idx : sv->table_res)
        for (int i = 0; i < n; ++i) advance_host(sv->res[idx].sim);
    // lattices with their own launches: one side stream each, forked from the
    // server stream before the first step and joined after the last
    for (size_t j = 0; j < sv->branch_res.size(); ++j) {
        vlbm_sim* s = sv->res[sv->branch_res[j]].sim;
        cudaStream_t side = sv->side_streams[j];
        e = cudaStreamWaitEvent(side, sv->fork_event, 0);
        if (e != cudaSuccess) return cuda_status(e, "fork wait");
        s->stream = side;
        vlbm_status st = VLBM_OK;
        for (int i = 0; i < n && st == VLBM_OK; ++i) {
            st = fluid_step(s);   // advances the mirror
            if (st == VLBM_OK && s->ibm) st = ibm_step(s);
        }
        launches += (double)n * (1.0 + (s->ibm ? 2.0 + 3.0 * std::max(1, ibm_iterations(s)) : 0.0));
        s->stream = sv->stream;
        if (st != VLBM_OK) return st;
        e = cudaEventRecord(sv->join_events[j], side);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sv->stream, sv->join_events[j], 0);
        if (e != cudaSuccess) return cuda_status(e, "join");
    }
    sv->last_launches = launches;
    return VLBM_OK;
}

struct HostState { int parity, side_cur, apply_bc; long long step; };

// Capture `steps` steps starting at the current phase; host mirrors and
// phase are left as they were (the replay advances them).
vlbm_status capture(vlbm_server* sv, int steps, cudaGraphExec_t* out) {
    const double t_start = now_s();
    std::vector<HostState> saved;
    for (const Resident& r : sv->res) saved.push_back({r.sim->parity, r.sim->side_cur, r.sim->apply_bc, r.sim->step});
    const int phase = sv->phase;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(sv->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_status(e, "begin capture");
    vlbm_status st = enqueue_steps(sv, steps);
    e = cudaStreamEndCapture(sv->stream, &g);
    sv->prof[8] += 1.0;
    for (size_t i = 0; i < sv->res.size(); ++i) {
        vlbm_sim* s = sv->res[i].sim;
        s->parity = saved[i].parity; s->side_cur = saved[i].side_cur;
        s->apply_bc = saved[i].apply_bc; s->step = saved[i].step;
    }
    sv->phase = phase;
    if (st != VLBM_OK) { if (g) cudaGraphDestroy(g); return st; }
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    if (g) cudaGraphDestroy(g);
    sv->capture_s += now_s() - t_start;
    return cuda_status(e, "server step graph");
}

vlbm_status replay(vlbm_server* sv, cudaGraphExec_t* slot, int steps) {
    if (!*slot) {
        vlbm_status st = capture(sv, steps, slot);
        if (st != VLBM_OK) return st;
    }
    cudaError_t e = cudaGraphLaunch(*slot, sv->stream);
    if (e != cudaSuccess) return cuda_status(e, "cudaGraphLaunch");
    sv->prof[7] += 1.0;
    for (Resident& r : sv->res)
        for (int i = 0; i < steps; ++i) advance_host(r.sim);
    sv->phase ^= steps & 1;
    return VLBM_OK;
}

vlbm_status server_steps(vlbm_server* sv, uint64_t k) {
    if (sv->res.empty() || k == 0) return VLBM_OK;
    vlbm_status st = VLBM_OK;
    uint64_t left = k;
    while (left > 0 && st == VLBM_OK) {
        // Lattices with their own launches take the boundary flag from the
        // host mirror: their first step (no boundary rule yet) runs outside
        // the graphs, whose steps all apply the rule.
        bool first = false;
        for (int idx : sv->branch_res) first |= sv->res[idx].sim->apply_bc == 0;
        if (first) {
            st = enqueue_steps(sv, 1);
            sv->prof[6] += sv->last_launches;
            left -= 1;
        } else if (!sv->use_graphs || sv->stable_segments == 0) {
            // direct launches: for a fresh membership (capturing pays off only
            // if it lasts) and for batches whose GPU step hides the launches
            st = enqueue_steps(sv, (int)left);
            sv->prof[6] += sv->last_launches;
            left = 0;
        } else {
            st = replay(sv, &sv->graph1[sv->phase], 1);
            left -= 1;
        }
    }
    for (const Resident& r : sv->res) sv->lattice_updates += (double)r.sim->N * (double)(k - left);
    sv->prof[5] += (double)(k - left);
    return st;
}

void fail_request(vlbm_server* sv, const Pending& p, vlbm_status st) {
    vlbm_completion c;
    std::memset(&c, 0, sizeof(c));
    c.tag = p.req.tag;
    c.status = st;
    c.submit_time_s = p.submit_t;
    c.start_time_s = c.finish_time_s = now_s();
    sv->done.push_back(c);
}

// Move a lattice built without host waits onto the server stream: the server
// stream waits for its set-up (an event on the lattice's own stream, which is
// released once that work completes); later calls wait as usual.
vlbm_status hand_over(vlbm_server* sv, vlbm_sim* s) {
    cudaEvent_t ready = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ready, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sv->stream, ready, 0);
    if (ready) cudaEventDestroy(ready);
    if (e != cudaSuccess) return cuda_status(e, "lattice hand-over");
    if (s->own_stream) cudaStreamDestroy(s->stream);   // released when its work completes
    s->stream = sv->stream;
    s->own_stream = false;
    s->async_setup = false;
    return VLBM_OK;
}

// Admit queued requests in arrival order while the slot limit and the HBM
// budget allow.  A new lattice is built on its own stream (its set-up copies
// and kernels do not wait for the queued batch work) from the server's memory
// cache, then moved to the server stream; it joins the batch at the next
// table rebuild.
vlbm_status server_admit(vlbm_server* sv) {
    while (!sv->queue.empty() && (int)sv->res.size() < sv->max_resident) {
        Pending& p = sv->queue.front();
        // admission by the budget: the estimate of the resident lattices, or the
        // buffers they actually hold (best-fit reuse can hand out a little more)
        if (std::max(sv->bytes_in_use, sv->cache.live_bytes) + p.bytes > sv->budget) break;
        vlbm_config cfg = p.req.cfg;
        cfg.device = sv->device;
        {   // the batched kernel streams one node per thread (natural layout);
            // lattices that always step with launches of their own (spheres, or
            // a full wave of the batched kernel by themselves) take the
            // library's layout, z-paired where that is faster
            const long long n = (long long)cfg.nx * cfg.ny * cfg.nz;
            const long long wave = sv->own_launch_min_nodes >= 0
                                       ? sv->own_launch_min_nodes
                                       : (long long)std::max(1, batched_blocks_per_sm(cfg.vel_set, cfg.storage,
                                                                                      cfg.collision, cfg.rheology)) *
                                             sv->sms * 256;
            cfg.layout = (!p.spheres.empty() || n >= wave) ? VLBM_LAYOUT_AUTO : VLBM_LAYOUT_NATURAL;
        }
        vlbm_sim* s = nullptr;
        const double a0 = now_s();
        // built without host waits on a high-priority stream of its own; the
        // server stream waits for the set-up through an event
        vlbm_status st = sim_create(&cfg, &sv->cache, &s, true);
        const double a1 = now_s();
        if (st == VLBM_OK) st = vlbm_set_builder(s, p.req.builder);
        const double a2 = now_s();
        if (st == VLBM_OK && !p.spheres.empty())
            st = vlbm_add_spheres(s, &p.req.ibm, p.spheres.data(), (int32_t)p.spheres.size());
        const double a3 = now_s();
        if (st == VLBM_OK) st = hand_over(sv, s);
        sv->prof[12] += a1 - a0;
        sv->prof[13] += a2 - a1;
        sv->prof[14] += a3 - a2;
        sv->prof[15] += now_s() - a3;
        if (st != VLBM_OK) {
            if (s) vlbm_destroy(s);
            fail_request(sv, p, st);
            sv->queue.pop_front();
            continue;
        }
        Resident r;
        r.sim = s;
        r.tag = p.req.tag;
        r.target = p.req.steps;
        r.submit_t = p.submit_t;
        r.start_t = now_s();
        r.bytes = std::max(p.bytes, s->device_bytes);   // admission used the estimate
        sv->bytes_in_use += r.bytes;
        sv->res.push_back(r);
        sv->queue.pop_front();
        sv->dirty = true;
    }
    return VLBM_OK;
}

// Lattices that reached their step count leave the batch: their ux and
// divergence word are copied to pinned memory behind an event, on the server
// stream after their last step.
vlbm_status begin_retire(vlbm_server* sv) {
    std::vector<Resident> keep;
    vlbm_status first_error = VLBM_OK;
    for (Resident& r : sv->res) {
        if ((uint64_t)r.sim->step < r.target) { keep.push_back(r); continue; }
        Retiring t;
        t.r = r;
        vlbm_sim* s = r.sim;
        const size_t N = (size_t)s->N;
        cudaError_t e = sim_malloc(s, (void**)&t.d_ux, N * sizeof(float));
        t.h_ux = static_cast<float*>(sv->pinned.get(N * sizeof(float)));
        t.h_err = static_cast<unsigned*>(sv->pinned.get(sizeof(unsigned)));
        if (e == cudaSuccess && (!t.h_ux || !t.h_err)) e = cudaErrorMemoryAllocation;
        if (e == cudaSuccess) {
            const vlbm_status st = sim_macroscopics_device(s, nullptr, t.d_ux, nullptr, nullptr, nullptr);
            if (st != VLBM_OK) e = cudaErrorLaunchFailure;
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(t.h_ux, t.d_ux, N * sizeof(float), cudaMemcpyDeviceToHost, sv->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(t.h_err, s->err, sizeof(unsigned), cudaMemcpyDeviceToHost, sv->stream);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(t.done, sv->stream);
        if (e != cudaSuccess) {
            t.status = cuda_status(e, "retirement read-out");
            if (first_error == VLBM_OK) first_error = t.status;
        }
        sv->retiring.push_back(t);
        sv->dirty = true;
    }
    sv->res.swap(keep);
    return first_error;
}

// Record the completions of the read-outs that finished (all of them when
// `wait`), release their lattices into the memory cache.
vlbm_status poll_retiring(vlbm_server* sv, bool wait) {
    std::vector<Retiring> still;
    for (Retiring& t : sv->retiring) {
        if (t.status == VLBM_OK && t.done) {
            const cudaError_t q = wait ? cudaEventSynchronize(t.done) : cudaEventQuery(t.done);
            if (q == cudaErrorNotReady) { still.push_back(t); continue; }
            if (q != cudaSuccess) t.status = cuda_status(q, "retirement read-out");
        }
        vlbm_sim* s = t.r.sim;
        const size_t N = (size_t)s->N;
        vlbm_completion c;
        std::memset(&c, 0, sizeof(c));
        c.tag = t.r.tag;
        c.submit_time_s = t.r.submit_t;
        c.start_time_s = t.r.start_t;
        c.steps = (uint64_t)s->step;
        c.status = t.status;
        std::vector<float> ux;
        if (c.status == VLBM_OK) {
            if (*t.h_err) {
                c.status = VLBM_ERR_DIVERGED;
            } else {
                ux.assign(t.h_ux, t.h_ux + N);
                double sum = 0.0;
                for (float v : ux) sum += v;
                c.mean_ux = sum / (double)N;
            }
        }
        c.finish_time_s = now_s();
        sv->done.push_back(c);
        if (!ux.empty()) {
            sv->results.emplace_back(t.r.tag, std::move(ux));
            while (sv->results.size() > kKeptResults) sv->results.pop_front();
        }
        sv->pinned.put(t.h_ux);
        sv->pinned.put(t.h_err);
        if (t.done) cudaEventDestroy(t.done);
        sim_free(s, t.d_ux);
        sim_release(s);   // the GPU is done with it: its buffers go back to the cache
        sv->bytes_in_use -= t.r.bytes;
    }
    sv->retiring.swap(still);
    return VLBM_OK;
}

// Keep at most kSegmentsInFlight segments queued ahead of the GPU.
vlbm_status end_segment(vlbm_server* sv) {
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(ev, sv->stream);
    if (e != cudaSuccess) { if (ev) cudaEventDestroy(ev); return cuda_status(e, "segment event"); }
    sv->segments.push_back(ev);
    while ((int)sv->segments.size() > kSegmentsInFlight) {
        e = cudaEventSynchronize(sv->segments.front());
        cudaEventDestroy(sv->segments.front());
        sv->segments.pop_front();
        if (e != cudaSuccess) return cuda_status(e, "segment wait");
    }
    return VLBM_OK;
}

}  // namespace

extern "C" {

vlbm_status vlbm_server_create(int device, size_t budget, int32_t max_resident, vlbm_server** out) {
    if (!out || max_resident < 1 || budget == 0) { set_last_error("invalid server arguments"); return VLBM_ERR_INVALID; }
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    vlbm_server* sv = new vlbm_server();
    sv->device = device;
    sv->budget = budget;
    sv->cache.cap = budget;
    sv->max_resident = max_resident;
    cudaDeviceGetAttribute(&sv->sms, cudaDevAttrMultiProcessorCount, device);
    e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { sv->stream = nullptr; delete sv; return cuda_status(e, "cudaStreamCreate"); }
    now_s();
    *out = sv;
    return VLBM_OK;
}

vlbm_status vlbm_server_submit(vlbm_server* sv, const vlbm_request* req) {
    if (!sv || !req) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    std::string why;
    vlbm_status st = sim_validate_config(req->cfg, why);
    if (st != VLBM_OK) { set_last_error(why); return st; }
    if (req->steps == 0) { set_last_error("a request needs at least one step"); return VLBM_ERR_INVALID; }
    if (req->n_spheres < 0 || (req->n_spheres > 0 && !req->spheres)) {
        set_last_error("bad sphere array");
        return VLBM_ERR_INVALID;
    }
    Pending p;
    p.req = *req;
    if (req->n_spheres > 0) p.spheres.assign(req->spheres, req->spheres + req->n_spheres);
    p.req.spheres = nullptr;
    p.submit_t = now_s();
    p.bytes = estimate_bytes(*req);
    if (p.bytes > sv->budget) { set_last_error("request larger than the server's HBM budget"); return VLBM_ERR_NOMEM; }
    sv->queue.push_back(std::move(p));
    return VLBM_OK;
}

vlbm_status vlbm_server_pump(vlbm_server* sv, uint32_t steps, vlbm_completion* out, int32_t max_out, int32_t* n_out) {
    if (n_out) *n_out = 0;
    if (!sv || (max_out > 0 && !out)) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    cudaError_t e = cudaSetDevice(sv->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    uint64_t left = steps;
    double t0 = now_s();
    vlbm_status st = poll_retiring(sv, false);
    double t1 = now_s();
    sv->prof[4] += t1 - t0;
    if (st == VLBM_OK) st = server_admit(sv);
    sv->prof[0] += now_s() - t1;
    while (st == VLBM_OK && left > 0) {
        if (sv->res.empty()) {
            // nothing to step: finish the read-outs, which may free memory for the queue
            if (sv->retiring.empty()) break;
            const double t0 = now_s();
            st = poll_retiring(sv, true);
            const double t1 = now_s();
            sv->prof[3] += t1 - t0;
            if (st == VLBM_OK) st = server_admit(sv);
            sv->prof[0] += now_s() - t1;
            continue;
        }
        double t0 = now_s();
        if (sv->dirty && (st = server_rebuild(sv)) != VLBM_OK) break;
        double t1 = now_s();
        sv->prof[1] += t1 - t0;
        uint64_t k = std::min<uint64_t>(left, kSegment);
        for (const Resident& r : sv->res) k = std::min<uint64_t>(k, r.target - (uint64_t)r.sim->step);
        if ((st = server_steps(sv, k)) != VLBM_OK) break;   // graph captures count as enqueue time here
        left -= k;
        if ((st = begin_retire(sv)) != VLBM_OK) break;
        t0 = now_s();
        sv->prof[2] += t0 - t1;
        if ((st = end_segment(sv)) != VLBM_OK) break;
        sv->stable_segments += 1;
        t1 = now_s();
        sv->prof[3] += t1 - t0;
        // host work while the GPU runs the queued segments
        if ((st = server_admit(sv)) != VLBM_OK) break;
        t0 = now_s();
        sv->prof[0] += t0 - t1;
        st = poll_retiring(sv, false);
        sv->prof[4] += now_s() - t0;
    }
    // an idle server hands back everything it finished
    if (st == VLBM_OK && sv->res.empty() && !sv->retiring.empty()) {
        t0 = now_s();
        st = poll_retiring(sv, true);
        sv->prof[3] += now_s() - t0;
    }
    // cached memory above the budget goes back to the device
    if (sv->cache.free_bytes + sv->cache.live_bytes > sv->budget)
        sv->cache.trim(sv->budget > sv->cache.live_bytes ? sv->budget - sv->cache.live_bytes : 0);
    int32_t n = 0;
    while (!sv->done.empty() && n < max_out) {
        out[n++] = sv->done.front();
        sv->done.pop_front();
    }
    if (n_out) *n_out = n;
    return st;
}

vlbm_status vlbm_server_stats(vlbm_server* sv, int32_t* resident, int32_t* queued, int64_t* bytes,
                              double* lattice_updates) {
    if (!sv) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    if (resident) *resident = (int32_t)(sv->res.size() + sv->retiring.size());   // lattices holding device memory
    if (queued) *queued = (int32_t)sv->queue.size();
    if (bytes) *bytes = (int64_t)sv->bytes_in_use;
    if (lattice_updates) *lattice_updates = sv->lattice_updates;
    return VLBM_OK;
}

vlbm_status vlbm_server_fetch(vlbm_server* sv, uint64_t tag, float* ux, size_t n) {
    if (!sv || !ux) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    for (auto it = sv->results.begin(); it != sv->results.end(); ++it)
        if (it->first == tag) {
            if (it->second.size() != n) { set_last_error("size mismatch"); return VLBM_ERR_INVALID; }
            std::memcpy(ux, it->second.data(), n * sizeof(float));
            sv->results.erase(it);
            return VLBM_OK;
        }
    set_last_error("no finished request with that tag is kept");
    return VLBM_ERR_NOT_FOUND;
}

vlbm_status vlbm_server_profile(vlbm_server* sv, double* seconds, int32_t n) {
    if (!sv || (n > 0 && !seconds)) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    sv->prof[9] = sv->capture_s;
    sv->prof[10] = (double)sv->cache.live_bytes;
    sv->prof[11] = (double)sv->cache.free_bytes;
    for (int32_t i = 0; i < n && i < 16; ++i) seconds[i] = sv->prof[i];
    return VLBM_OK;
}

vlbm_status vlbm_server_set_own_launch_min(vlbm_server* sv, int64_t nodes) {
    if (!sv) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    sv->own_launch_min_nodes = nodes < 0 ? -1 : nodes;
    sv->dirty = true;
    return VLBM_OK;
}

vlbm_status vlbm_server_destroy(vlbm_server* sv) {
    if (!sv) return VLBM_OK;
    cudaSetDevice(sv->device);
    if (sv->stream) cudaStreamSynchronize(sv->stream);
    delete sv;
    return VLBM_OK;
}

}  // extern "C"
