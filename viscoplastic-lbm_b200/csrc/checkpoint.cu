// checkpoint.cu -- save and restore the complete state of a simulation
// (simCheckpoint.cu:216-318: operateSimCheckpoint, loadSimCheckpoint,
// saveSimCheckpoint).
//
// The reference writes one raw file per array (step, particle centres, pop,
// popAux, rho, u, omega, f and the IBM node arrays) into
// PATH/ID/checkpoint/<gpu>_<name>.bin, with no header and no check of what it
// reads back.  Here the state is one self-describing image:
//
//   header      magic "VLBMCKPT", format version, the lattice shape, velocity
//               set, storage type, scale and layout, the boundary-node count,
//               a hash of the geometry (node classes, boundary records), the
//               host step state (step, AA parity, side-store index, boundary
//               flag), the device step counters (seeds of the stochastic
//               rounding), particle and Lagrangian-node counts
//   regions     (id, bytes, payload) for every device array that carries from
//               one step to the next: the population array as stored (AA
//               parity and half-precision bits included), both side stores of
//               the boundary nodes, Power-Law omega, the IBM force field, the
//               node classes (IBM force bits), and the IBM state
//   trailer     64-bit hash of everything before it
//
// A run resumed from an image continues bit for bit like the run that wrote
// it.  Loading requires a simulation created with the same shape, velocity
// set, storage and layout, with the same geometry and, with spheres, the same
// particle and node counts (the reference likewise creates its particles
// before it loads their state); everything else is taken from the image.
// The file form is PATH/ID/checkpoint/0_state.bin, with '/' separators on
// every platform (the reference's save path joins with "\\\\" on Linux).
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>
#include "sim.h"

namespace vlbm {

namespace {

constexpr char kMagic[8] = {'V', 'L', 'B', 'M', 'C', 'K', 'P', 'T'};
constexpr uint32_t kVersion = 2;   // 2: FP32 populations stored as deviations f_i - w_i rho0

struct CkptHeader {
    char magic[8];
    uint32_t version;
    uint32_t header_bytes;
    int32_t nx, ny, nz, q;
    int32_t storage, store_bytes, pair_h, nbc;   // pair_h: NZ/2 of a z-paired layout, bit 30 = blocked pairs
    float scale;
    int32_t rheology;
    int32_t parity, side_cur, apply_bc, has_omega;
    int64_t step;
    uint32_t step_ctr[2];
    int32_t np, nnodes;
    uint32_t record_bytes, n_regions;
    uint64_t geometry_hash;
    uint64_t payload_bytes;     // bytes of all regions with their headers
};

struct RegionHeader {
    uint32_t id;
    uint32_t pad;
    uint64_t bytes;
};

// 64-bit FNV-1a over 8-byte words (then the tail bytes); a corruption check,
// not a cryptographic hash.
struct Hash64 {
    uint64_t h = 1469598103934665603ull;
    void add(const void* data, size_t n) {
        const unsigned char* p = static_cast<const unsigned char*>(data);
        size_t k = 0;
        for (; k + 8 <= n; k += 8) {
            uint64_t w;
            std::memcpy(&w, p + k, 8);
            h = (h ^ w) * 1099511628211ull;
        }
        for (; k < n; ++k) h = (h ^ p[k]) * 1099511628211ull;
    }
};

// Copies are ordered on the simulation's stream (a pageable host-to-device
// cudaMemcpy may return before its DMA completes, and the stream is
// non-blocking) and waited for before the host reads or reuses the buffer.
cudaError_t ckpt_copy(vlbm_sim* s, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s->stream);
    return e == cudaSuccess ? cudaStreamSynchronize(s->stream) : e;
}

float effective_scale(const vlbm_sim* s) {
    if (s->cfg.storage_scale > 0) return (float)s->cfg.storage_scale;
    return s->cfg.storage == VLBM_STORE_F16 ? 4096.0f : 1.0f;
}

// Every device array that carries state from one step to the next.
void state_regions(vlbm_sim* s, std::vector<StateRegion>& out) {
    const size_t N = (size_t)s->N, Q = (size_t)s->Q;
    out.push_back({1, s->pop, Q * N * (size_t)s->store_bytes});
    if (s->nbc > 0) {
        out.push_back({2, s->side[0], Q * (size_t)s->nbc * sizeof(float)});
        out.push_back({3, s->side[1], Q * (size_t)s->nbc * sizeof(float)});
    }
    if (s->omega) out.push_back({4, s->omega, N * sizeof(float)});
    if (s->fibm) out.push_back({5, s->fibm, 3 * N * sizeof(float)});
    out.push_back({6, s->cls, N * sizeof(uint8_t)});
    ibm_state_regions(s, out);
}

// Geometry fingerprint: node classes without the IBM bits, boundary records
// and their node indices.
vlbm_status geometry_hash(vlbm_sim* s, uint64_t* out) {
    const size_t N = (size_t)s->N;
    std::vector<uint8_t> cls(N);
    cudaError_t e = ckpt_copy(s, cls.data(), s->cls, N, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "checkpoint: read node classes");
    for (auto& c : cls) c &= (uint8_t)~NODE_IBM_FORCE;
    Hash64 h;
    h.add(cls.data(), N);
    if (s->nbc > 0) {
        std::vector<BcRec> recs((size_t)s->nbc);
        std::vector<int32_t> nodes((size_t)s->nbc);
        e = ckpt_copy(s, recs.data(), s->bc, recs.size() * sizeof(BcRec), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = ckpt_copy(s, nodes.data(), s->bc_node, nodes.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_status(e, "checkpoint: read boundary tables");
        h.add(recs.data(), recs.size() * sizeof(BcRec));
        h.add(nodes.data(), nodes.size() * sizeof(int32_t));
    }
    *out = h.h;
    return VLBM_OK;
}

vlbm_status fill_header(vlbm_sim* s, const std::vector<StateRegion>& regions, CkptHeader* h) {
    std::memset(h, 0, sizeof(*h));
    std::memcpy(h->magic, kMagic, 8);
    h->version = kVersion;
    h->header_bytes = sizeof(CkptHeader);
    h->nx = s->cfg.nx; h->ny = s->cfg.ny; h->nz = s->cfg.nz; h->q = s->Q;
    h->storage = s->cfg.storage; h->store_bytes = s->store_bytes; h->pair_h = s->pairH | (s->pairBlk << 30); h->nbc = s->nbc;
    h->scale = effective_scale(s);
    h->rheology = s->cfg.rheology;
    h->parity = s->parity; h->side_cur = s->side_cur; h->apply_bc = s->apply_bc;
    h->has_omega = s->omega != nullptr;
    h->step = s->step;
    int np = 0, nn = 0;
    ibm_counts(s, &np, &nn);
    h->np = np; h->nnodes = nn;
    h->record_bytes = np ? ibm_record_bytes() : 0;
    h->n_regions = (uint32_t)regions.size();
    uint64_t payload = 0;
    for (const auto& r : regions) payload += sizeof(RegionHeader) + r.bytes;
    h->payload_bytes = payload;
    return geometry_hash(s, &h->geometry_hash);
}

vlbm_status ready(vlbm_sim* s) {
    if (!s) { set_last_error("null simulation handle"); return VLBM_ERR_INVALID; }
    if (!s->geometry) { set_last_error("checkpoint: the simulation has no geometry yet"); return VLBM_ERR_STATE; }
    cudaError_t e = cudaSetDevice(s->device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return cuda_status(e, "checkpoint: synchronise");
}

size_t image_bytes(const CkptHeader& h) { return sizeof(CkptHeader) + h.payload_bytes + sizeof(uint64_t); }

vlbm_status save_image(vlbm_sim* s, std::vector<unsigned char>* grow, void* buf, size_t n, size_t* needed) {
    vlbm_status st = ready(s);
    if (st != VLBM_OK) return st;
    std::vector<StateRegion> regions;
    state_regions(s, regions);
    CkptHeader h;
    if ((st = fill_header(s, regions, &h)) != VLBM_OK) return st;
    cudaError_t e = ckpt_copy(s, h.step_ctr, s->step_ctr, sizeof(h.step_ctr), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e, "checkpoint: read step counters");
    const size_t total = image_bytes(h);
    if (needed) *needed = total;
    unsigned char* out = static_cast<unsigned char*>(buf);
    if (grow) {
        grow->resize(total);
        out = grow->data();
    } else {
        if (!buf) return VLBM_OK;   // size query
        if (n < total) {
            set_last_error("checkpoint buffer too small: need " + std::to_string(total) + " bytes");
            return VLBM_ERR_INVALID;
        }
    }
    size_t off = 0;
    std::memcpy(out, &h, sizeof(h));
    off += sizeof(h);
    for (const auto& r : regions) {
        RegionHeader rh{r.id, 0u, (uint64_t)r.bytes};
        std::memcpy(out + off, &rh, sizeof(rh));
        off += sizeof(rh);
        e = ckpt_copy(s, out + off, r.dev, r.bytes, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_status(e, "checkpoint: read device state");
        off += r.bytes;
    }
    Hash64 hh;
    hh.add(out, off);
    std::memcpy(out + off, &hh.h, sizeof(uint64_t));
    return VLBM_OK;
}

vlbm_status mismatch(const std::string& what) {
    set_last_error("checkpoint does not match this simulation: " + what);
    return VLBM_ERR_INVALID;
}

vlbm_status load_image(vlbm_sim* s, const unsigned char* in, size_t n) {
    vlbm_status st = ready(s);
    if (st != VLBM_OK) return st;
    if (!in || n < sizeof(CkptHeader) + sizeof(uint64_t)) {
        set_last_error("checkpoint image is truncated");
        return VLBM_ERR_INVALID;
    }
    CkptHeader h;
    std::memcpy(&h, in, sizeof(h));
    if (std::memcmp(h.magic, kMagic, 8) != 0) { set_last_error("not a checkpoint image"); return VLBM_ERR_INVALID; }
    if (h.version != kVersion || h.header_bytes != sizeof(CkptHeader)) {
        set_last_error("checkpoint format version " + std::to_string(h.version) + " is not supported");
        return VLBM_ERR_UNSUPPORTED;
    }
    if (image_bytes(h) != n) { set_last_error("checkpoint image is truncated or has trailing bytes"); return VLBM_ERR_INVALID; }
    {
        Hash64 hh;
        hh.add(in, n - sizeof(uint64_t));
        uint64_t stored;
        std::memcpy(&stored, in + n - sizeof(uint64_t), sizeof(stored));
        if (stored != hh.h) { set_last_error("checkpoint image is corrupt (hash mismatch)"); return VLBM_ERR_INVALID; }
    }
    std::vector<StateRegion> regions;
    state_regions(s, regions);
    CkptHeader mine;
    if ((st = fill_header(s, regions, &mine)) != VLBM_OK) return st;
    if (h.nx != mine.nx || h.ny != mine.ny || h.nz != mine.nz) return mismatch("lattice size");
    if (h.q != mine.q) return mismatch("velocity set");
    if (h.storage != mine.storage || h.store_bytes != mine.store_bytes || h.scale != mine.scale)
        return mismatch("population storage");
    if (h.pair_h != mine.pair_h) return mismatch("population layout");
    if (h.nbc != mine.nbc || h.geometry_hash != mine.geometry_hash) return mismatch("geometry");
    if (h.has_omega != mine.has_omega) return mismatch("rheology state (Power-Law omega)");
    if (h.np != mine.np || h.nnodes != mine.nnodes || h.record_bytes != mine.record_bytes)
        return mismatch("spheres (particle or Lagrangian node count)");
    if (h.n_regions != mine.n_regions || h.payload_bytes != mine.payload_bytes) return mismatch("state arrays");
    if (h.parity < 0 || h.parity > 1 || h.side_cur < 0 || h.side_cur > 1 || h.step < 0)
        return mismatch("step state");
    size_t off = sizeof(CkptHeader);
    for (const auto& r : regions) {   // all region headers first: nothing is written on a mismatch
        RegionHeader rh;
        std::memcpy(&rh, in + off, sizeof(rh));
        if (rh.id != r.id || rh.bytes != r.bytes) return mismatch("state array " + std::to_string(r.id));
        off += sizeof(rh) + r.bytes;
    }
    off = sizeof(CkptHeader);
    for (const auto& r : regions) {
        off += sizeof(RegionHeader);
        cudaError_t e = ckpt_copy(s, r.dev, in + off, r.bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_status(e, "checkpoint: write device state");
        off += r.bytes;
    }
    cudaError_t e = ckpt_copy(s, s->step_ctr, h.step_ctr, sizeof(h.step_ctr), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "checkpoint: write step counters");
    s->parity = h.parity;
    s->side_cur = h.side_cur;
    s->apply_bc = h.apply_bc;
    s->step = h.step;
    return VLBM_OK;
}

std::string state_file(const char* path_files, const char* id_sim) {
    return std::string(path_files) + "/" + id_sim + "/checkpoint/0_state.bin";
}

}  // namespace

}  // namespace vlbm

using namespace vlbm;

extern "C" {

vlbm_status vlbm_checkpoint_save(vlbm_sim* s, void* buf, size_t n, size_t* needed) {
    return save_image(s, nullptr, buf, n, needed);
}

vlbm_status vlbm_checkpoint_load(vlbm_sim* s, const void* buf, size_t n) {
    return load_image(s, static_cast<const unsigned char*>(buf), n);
}

vlbm_status vlbm_save_checkpoint(vlbm_sim* s, const char* path_files, const char* id_sim) {
    if (!s) { set_last_error("null simulation handle"); return VLBM_ERR_INVALID; }
    if (!path_files || !id_sim) { set_last_error("null path"); return VLBM_ERR_INVALID; }
    std::vector<unsigned char> img;
    vlbm_status st = save_image(s, &img, nullptr, 0, nullptr);
    if (st != VLBM_OK) return st;
    const std::string dir = std::string(path_files) + "/" + id_sim + "/checkpoint";
    {   // mkdir -p (createFolder, simCheckpoint.cu:28-41)
        std::string acc;
        for (size_t k = 0; k <= dir.size(); ++k) {
            if ((k == dir.size() || dir[k] == '/') && !acc.empty()) mkdir(acc.c_str(), 0777);
            if (k < dir.size()) acc.push_back(dir[k]);
        }
    }
    const std::string fn = state_file(path_files, id_sim);
    const std::string tmp = fn + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) { set_last_error("cannot open " + tmp); return VLBM_ERR_IO; }
    const size_t w = std::fwrite(img.data(), 1, img.size(), f);
    const int c = std::fclose(f);
    if (w != img.size() || c != 0) { std::remove(tmp.c_str()); set_last_error("short write " + tmp); return VLBM_ERR_IO; }
    if (std::rename(tmp.c_str(), fn.c_str()) != 0) { set_last_error("cannot rename " + tmp); return VLBM_ERR_IO; }
    return VLBM_OK;
}

vlbm_status vlbm_load_checkpoint(vlbm_sim* s, const char* path_files, const char* id_sim) {
    if (!s) { set_last_error("null simulation handle"); return VLBM_ERR_INVALID; }
    if (!path_files || !id_sim) { set_last_error("null path"); return VLBM_ERR_INVALID; }
    const std::string fn = state_file(path_files, id_sim);
    FILE* f = std::fopen(fn.c_str(), "rb");
    if (!f) { set_last_error("no checkpoint at " + fn); return VLBM_ERR_NOT_FOUND; }
    std::vector<unsigned char> img;
    unsigned char chunk[1 << 16];
    size_t r;
    while ((r = std::fread(chunk, 1, sizeof(chunk), f)) > 0) img.insert(img.end(), chunk, chunk + r);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) { set_last_error("read error " + fn); return VLBM_ERR_IO; }
    return load_image(s, img.data(), img.size());
}

}  // extern "C"
