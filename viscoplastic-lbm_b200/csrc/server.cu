// server.cu -- continuous-batching serving loop for many lattices on one GPU.
//
// The reference runs one compile-time configured simulation per process
// (src/CUDA/main.cu).  Here requests (each a full vlbm_config, a named builder,
// a step count and optional spheres) are queued, admitted in arrival order
// while the HBM budget and the slot limit allow, kept resident, advanced
// together, and retired at their step count:
//
//  * every resident lattice of one (velocity set, operator, rheology, storage)
//    group advances in ONE persistent launch of k_step_batched over a
//    (lattice, tile) table; the step state of each lattice (AA parity,
//    side-store buffer, boundary flag) lives in device memory and is advanced by
//    k_batch_advance, so a step is captured once in a CUDA graph and replayed
//    until the membership changes.  Lattices with spheres run their IBM kernels
//    after the batched fluid step, launched directly;
//  * pump() runs up to the next retirement without host synchronisation, then
//    synchronises, records completion times and the volume-mean velocity,
//    frees the lattice and admits queued requests into the freed memory.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <string>
#include <vector>
#include "sim.h"
#include "step_impl.cuh"

namespace vlbm {

// After every lattice of the batch took its step.
__global__ void k_batch_advance(BatchSlot* slots, int nslots) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nslots) return;
    slots[i].parity ^= 1;
    slots[i].side_cur ^= 1;
    slots[i].apply_bc = 1;
}

cudaError_t launch_batch_advance(BatchSlot* slots, int nslots, cudaStream_t s) {
    if (nslots <= 0) return cudaSuccess;
    k_batch_advance<<<(nslots + 127) / 128, 128, 0, s>>>(slots, nslots);
    return cudaGetLastError();
}

}  // namespace vlbm

using namespace vlbm;

namespace {

constexpr int kGraphSteps = 8;        // steps per replay of the long graph
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
// the side store of the wall nodes (at most the six faces), the Power-Law
// state, the IBM fields and Lagrangian arrays, plus 1 MiB of small allocations.
size_t estimate_bytes(const vlbm_request& r) {
    const size_t N = (size_t)r.cfg.nx * r.cfg.ny * r.cfg.nz;
    const size_t sb = r.cfg.storage == VLBM_STORE_F32 ? 4 : 2;
    size_t b = (size_t)r.cfg.vel_set * N * sb + 25 * N + (1 << 20);
    const size_t walls = 2 * ((size_t)r.cfg.nx * r.cfg.ny + (size_t)r.cfg.ny * r.cfg.nz + (size_t)r.cfg.nx * r.cfg.nz);
    b += walls * (2 * (size_t)r.cfg.vel_set * 4 + 24);
    if (r.cfg.rheology == VLBM_POWERLAW) b += 4 * N;
    if (r.n_spheres > 0) b += 44 * N + (size_t)r.n_spheres * 700 * 10 * 8;
    return b;
}

struct Group {
    int Q, op, rheo, st;
    size_t table_off;
    int ntiles;
    int grid;
};

}  // namespace

struct vlbm_server {
    int device = 0;
    int sms = 148;
    size_t budget = 0;
    int max_resident = 64;
    cudaStream_t stream = nullptr;
    std::deque<Pending> queue;
    std::vector<Resident> res;
    std::deque<vlbm_completion> done;
    std::deque<std::pair<uint64_t, std::vector<float>>> results;   // finished ux fields, by tag
    size_t bytes_in_use = 0;
    double lattice_updates = 0.0;
    // batch tables (rebuilt when the membership changes)
    bool dirty = true;
    BatchSlot* d_slots = nullptr;
    BatchBlock* d_table = nullptr;
    size_t cap_slots = 0, cap_table = 0;
    std::vector<Group> groups;
    int nslots = 0;
    bool any_ibm = false;
    cudaGraphExec_t graph1 = nullptr, graphK = nullptr;   // one step, kGraphSteps steps

    void drop_graphs() {
        if (graph1) cudaGraphExecDestroy(graph1);
        if (graphK) cudaGraphExecDestroy(graphK);
        graph1 = graphK = nullptr;
    }
    ~vlbm_server() {
        for (Resident& r : res) vlbm_destroy(r.sim);
        drop_graphs();
        cudaFree(d_slots);
        cudaFree(d_table);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

vlbm_status server_rebuild(vlbm_server* sv) {
    sv->drop_graphs();
    sv->groups.clear();
    sv->any_ibm = false;
    std::vector<BatchSlot> slots;
    std::vector<BatchBlock> table;
    auto key = [](const vlbm_sim* s) {
        const vlbm_config& c = s->cfg;
        return ((c.vel_set * 4 + c.collision) * 4 + c.rheology) * 4 + c.storage;
    };
    std::vector<int> order(sv->res.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return key(sv->res[a].sim) < key(sv->res[b].sim); });
    int cur = -1;
    for (int idx : order) {
        vlbm_sim* s = sv->res[idx].sim;
        if (s->ibm) sv->any_ibm = true;
        const int k = key(s);
        if (k != cur) {
            sv->groups.push_back(Group{s->Q, s->cfg.collision, s->cfg.rheology, s->cfg.storage, table.size(), 0, 0});
            cur = k;
        }
        BatchSlot bs;
        std::memset(&bs, 0, sizeof(bs));
        bs.p = make_params(s);
        bs.side[0] = s->side[0];
        bs.side[1] = s->side[1];
        bs.parity = s->parity;
        bs.side_cur = s->side_cur;
        bs.apply_bc = s->apply_bc;
        const int slot = (int)slots.size();
        slots.push_back(bs);
        const unsigned nt = (unsigned)((s->N + BATCH_TILE - 1) / BATCH_TILE);
        for (unsigned t = 0; t < nt; ++t) table.push_back(BatchBlock{slot, t * (unsigned)BATCH_TILE});
        sv->groups.back().ntiles += (int)nt;
    }
    for (Group& g : sv->groups) {
        const int per_sm = std::max(1, batched_blocks_per_sm(g.Q, g.st, g.op, g.rheo));
        g.grid = std::min(g.ntiles, per_sm * sv->sms);
    }
    sv->nslots = (int)slots.size();
    if (slots.size() > sv->cap_slots) {
        cudaFree(sv->d_slots);
        sv->d_slots = nullptr;
        sv->cap_slots = 0;
        if (cudaMalloc(&sv->d_slots, slots.size() * 2 * sizeof(BatchSlot)) != cudaSuccess) {
            set_last_error("server slot table allocation failed");
            return VLBM_ERR_NOMEM;
        }
        sv->cap_slots = slots.size() * 2;
    }
    if (table.size() > sv->cap_table) {
        cudaFree(sv->d_table);
        sv->d_table = nullptr;
        sv->cap_table = 0;
        if (cudaMalloc(&sv->d_table, table.size() * 2 * sizeof(BatchBlock)) != cudaSuccess) {
            set_last_error("server tile table allocation failed");
            return VLBM_ERR_NOMEM;
        }
        sv->cap_table = table.size() * 2;
    }
    if (!slots.empty()) {
        // pageable sources: both copies are complete when the calls return
        cudaError_t e = cudaMemcpyAsync(sv->d_slots, slots.data(), slots.size() * sizeof(BatchSlot),
                                        cudaMemcpyHostToDevice, sv->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sv->d_table, table.data(), table.size() * sizeof(BatchBlock), cudaMemcpyHostToDevice,
                                sv->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sv->stream);
        if (e != cudaSuccess) return cuda_status(e, "server table upload");
    }
    sv->dirty = false;
    return VLBM_OK;
}

// The launches of one batched fluid step (all groups, then the state advance).
cudaError_t server_fluid_launches(vlbm_server* sv) {
    for (const Group& g : sv->groups) {
        cudaError_t e = launch_batched(g.Q, g.st, sv->d_slots, sv->d_table + g.table_off, g.ntiles, g.grid, g.op,
                                       g.rheo, sv->stream);
        if (e != cudaSuccess) return e;
    }
    return launch_batch_advance(sv->d_slots, sv->nslots, sv->stream);
}

cudaError_t capture(vlbm_server* sv, int steps, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(sv->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t le = cudaSuccess;
    for (int i = 0; i < steps && le == cudaSuccess; ++i) le = server_fluid_launches(sv);
    e = cudaStreamEndCapture(sv->stream, &g);
    if (e == cudaSuccess) e = le;
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    if (g) cudaGraphDestroy(g);
    return e;
}

// Host mirror of the state every lattice advanced on the device.
void advance_host(vlbm_sim* s) {
    s->parity ^= 1;
    s->side_cur ^= 1;
    s->apply_bc = 1;
    s->step += 1;
}

vlbm_status server_steps(vlbm_server* sv, uint64_t k) {
    if (sv->res.empty() || k == 0) return VLBM_OK;
    if (!sv->any_ibm) {
        cudaError_t e = cudaSuccess;
        if (k >= (uint64_t)kGraphSteps && !sv->graphK) e = capture(sv, kGraphSteps, &sv->graphK);
        if (e == cudaSuccess && k % kGraphSteps && !sv->graph1) e = capture(sv, 1, &sv->graph1);
        for (uint64_t i = 0; e == cudaSuccess && i < k / kGraphSteps; ++i) e = cudaGraphLaunch(sv->graphK, sv->stream);
        for (uint64_t i = 0; e == cudaSuccess && i < k % kGraphSteps; ++i) e = cudaGraphLaunch(sv->graph1, sv->stream);
        if (e != cudaSuccess) return cuda_status(e, "server step graph");
        for (Resident& r : sv->res)
            for (uint64_t i = 0; i < k; ++i) advance_host(r.sim);
    } else {
        for (uint64_t i = 0; i < k; ++i) {
            cudaError_t e = server_fluid_launches(sv);
            if (e != cudaSuccess) return cuda_status(e, "batched step");
            for (Resident& r : sv->res) {
                advance_host(r.sim);
                if (r.sim->ibm) {
                    vlbm_status st = ibm_step(r.sim);
                    if (st != VLBM_OK) return st;
                }
            }
        }
    }
    for (const Resident& r : sv->res) sv->lattice_updates += (double)r.sim->N * (double)k;
    return VLBM_OK;
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

vlbm_status server_admit(vlbm_server* sv) {
    while (!sv->queue.empty() && (int)sv->res.size() < sv->max_resident) {
        Pending& p = sv->queue.front();
        if (sv->bytes_in_use + p.bytes > sv->budget) break;
        vlbm_config cfg = p.req.cfg;
        cfg.device = sv->device;
        cfg.layout = VLBM_LAYOUT_NATURAL;   // the batched kernel streams one node per thread
        vlbm_sim* s = nullptr;
        vlbm_status st = vlbm_create(&cfg, &s);
        if (st == VLBM_OK) {
            std::vector<uint32_t> map((size_t)cfg.nx * cfg.ny * cfg.nz);
            st = vlbm_build_node_map(p.req.builder, cfg.nx, cfg.ny, cfg.nz, map.data(), map.size());
            if (st == VLBM_OK) st = vlbm_set_node_map(s, map.data(), map.size());
        }
        if (st == VLBM_OK && !p.spheres.empty())
            st = vlbm_add_spheres(s, &p.req.ibm, p.spheres.data(), (int32_t)p.spheres.size());
        if (st == VLBM_OK) st = vlbm_set_stream(s, sv->stream);
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

vlbm_status server_retire(vlbm_server* sv) {
    bool any = false;
    for (const Resident& r : sv->res) any |= (uint64_t)r.sim->step >= r.target;
    if (!any) return VLBM_OK;
    cudaError_t e = cudaStreamSynchronize(sv->stream);
    if (e != cudaSuccess) return cuda_status(e, "server sync");
    std::vector<Resident> keep;
    for (Resident& r : sv->res) {
        if ((uint64_t)r.sim->step < r.target) { keep.push_back(r); continue; }
        vlbm_completion c;
        std::memset(&c, 0, sizeof(c));
        c.tag = r.tag;
        c.submit_time_s = r.submit_t;
        c.start_time_s = r.start_t;
        c.steps = (uint64_t)r.sim->step;
        c.status = vlbm_sync(r.sim);
        std::vector<float> ux((size_t)r.sim->N);
        if (c.status == VLBM_OK)
            c.status = vlbm_get_macroscopics(r.sim, nullptr, ux.data(), nullptr, nullptr, nullptr);
        double sum = 0.0;
        for (float v : ux) sum += v;
        c.mean_ux = sum / (double)r.sim->N;
        c.finish_time_s = now_s();
        sv->done.push_back(c);
        sv->results.emplace_back(r.tag, std::move(ux));
        while (sv->results.size() > kKeptResults) sv->results.pop_front();
        sv->bytes_in_use -= r.bytes;
        vlbm_destroy(r.sim);
        sv->dirty = true;
    }
    sv->res.swap(keep);
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
    vlbm_status st = server_admit(sv);
    while (st == VLBM_OK && left > 0 && !sv->res.empty()) {
        if (sv->dirty && (st = server_rebuild(sv)) != VLBM_OK) break;
        uint64_t k = left;
        for (const Resident& r : sv->res) k = std::min<uint64_t>(k, r.target - (uint64_t)r.sim->step);
        if ((st = server_steps(sv, k)) != VLBM_OK) break;
        left -= k;
        if ((st = server_retire(sv)) != VLBM_OK) break;
        st = server_admit(sv);
    }
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
    if (resident) *resident = (int32_t)sv->res.size();
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

vlbm_status vlbm_server_destroy(vlbm_server* sv) {
    if (!sv) return VLBM_OK;
    cudaSetDevice(sv->device);
    if (sv->stream) cudaStreamSynchronize(sv->stream);
    delete sv;
    return VLBM_OK;
}

}  // extern "C"
