// geometry.cpp -- node-map builders and boundary tables (host side).
//
// The builders restate the reference's gpuBuildBoundaryConditions variants
// (src/CUDA/boundaryConditionsBuilders/*.cu) on the host and produce the same
// 32-bit words (bit layout src/CUDA/structs/nodeTypeMap.h:15-133).  The table
// builder turns such a map (or a named builder directly, visiting only the
// domain faces) into what the fused kernel reads: one BcRec and the node index
// of each boundary slot; the class bytes and slot indices are scattered on the
// device.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "internal.h"
#include "lattice.cuh"

namespace vlbm {

namespace {

uint32_t make_word(int scheme, int dir, int ux = 0, int uy = 0, int uz = 0, int rho = 0) {
    uint32_t m = 0;
    m |= 1u << VLBM_MAP_IS_USED_OFFSET;                     // setIsUsed(true)
    m |= (uint32_t)(scheme & 7) << VLBM_MAP_SCHEME_OFFSET;   // setSchemeBC
    m |= (uint32_t)(dir & 31) << VLBM_MAP_DIRECTION_OFFSET;  // setDirection
    // geometry CONCAVE (0), SAVE_POST_COL false
    m |= (uint32_t)(ux & 7) << VLBM_MAP_UX_IDX_OFFSET;
    m |= (uint32_t)(uy & 7) << VLBM_MAP_UY_IDX_OFFSET;
    m |= (uint32_t)(uz & 7) << VLBM_MAP_UZ_IDX_OFFSET;
    m |= (uint32_t)(rho & 7) << VLBM_MAP_RHO_IDX_OFFSET;
    return m;
}

// Direction code for a node touching walls on the given sides, with the
// priority of the reference builders' if-chains (S before N, W before E,
// B before F; corners, then xy edges, yz edges, xz edges, faces).
// sy: -1 south, +1 north, 0 none; sx: -1 west, +1 east; sz: -1 back, +1 front.
int combine_dir(int sy, int sx, int sz) {
    if (sy && sx && sz) {
        if (sy > 0) return sx < 0 ? (sz > 0 ? VLBM_NORTH_WEST_FRONT : VLBM_NORTH_WEST_BACK)
                                  : (sz > 0 ? VLBM_NORTH_EAST_FRONT : VLBM_NORTH_EAST_BACK);
        return sx < 0 ? (sz > 0 ? VLBM_SOUTH_WEST_FRONT : VLBM_SOUTH_WEST_BACK)
                      : (sz > 0 ? VLBM_SOUTH_EAST_FRONT : VLBM_SOUTH_EAST_BACK);
    }
    if (sy && sx) return sy > 0 ? (sx < 0 ? VLBM_NORTH_WEST : VLBM_NORTH_EAST)
                                : (sx < 0 ? VLBM_SOUTH_WEST : VLBM_SOUTH_EAST);
    if (sy && sz) return sy > 0 ? (sz > 0 ? VLBM_NORTH_FRONT : VLBM_NORTH_BACK)
                                : (sz > 0 ? VLBM_SOUTH_FRONT : VLBM_SOUTH_BACK);
    if (sx && sz) return sx < 0 ? (sz > 0 ? VLBM_WEST_FRONT : VLBM_WEST_BACK)
                                : (sz > 0 ? VLBM_EAST_FRONT : VLBM_EAST_BACK);
    if (sy) return sy > 0 ? VLBM_NORTH : VLBM_SOUTH;
    if (sx) return sx < 0 ? VLBM_WEST : VLBM_EAST;
    if (sz) return sz > 0 ? VLBM_FRONT : VLBM_BACK;
    return -1;
}

inline int side(int v, int n, bool wall) {
    if (!wall) return 0;
    if (v == 0) return -1;
    if (v == n - 1) return 1;
    return 0;
}

// Outward normals of each direction's walls (nodeTypeMap.h:59-85).
int dir_normals(int dir, int nrm[3][3]) {
    static const int faces[26] = {1, 2, 4, 8, 16, 32, 5, 9, 17, 33, 6, 10, 18, 34, 20, 36, 24, 40,
                                  21, 37, 25, 41, 22, 38, 26, 42};
    static const int f6[6][3] = {{0, 1, 0}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 0, 1}, {0, 0, -1}};
    if (dir < 0 || dir > 25) return 0;
    int k = 0;
    for (int f = 0; f < 6; ++f)
        if (faces[dir] & (1 << f)) { for (int a = 0; a < 3; ++a) nrm[k][a] = f6[f][a]; ++k; }
    return k;
}

}  // namespace

// Half-way bounce-back roles (bounceBack.cu:26-498, derived): a population
// arriving from outside through every wall of the node is replaced; one that
// crosses one wall inward and another outward keeps its streamed value (the
// reference's "dead pops").
int bb_role(int dir, int i) {
    int nrm[3][3];
    int k = dir_normals(dir, nrm);
    bool neg = false, pos = false;
    for (int a = 0; a < k; ++a) {
        int s = lat_cx(i) * nrm[a][0] + lat_cy(i) * nrm[a][1] + lat_cz(i) * nrm[a][2];
        neg |= s < 0;
        pos |= s > 0;
    }
    return (neg && pos) ? 2 : (neg ? 1 : 0);
}

// Word of node (x, y, z) for a named builder; false for an unknown builder id.
// Only nodes on the domain faces get a non-bulk word.
bool builder_word(int builder, int x, int y, int z, int nx, int ny, int nz, uint32_t& w) {
    w = make_word(VLBM_BC_NULL, 0);
    int d;
    switch (builder) {
    case VLBM_BUILDER_PERIODIC: break;
    case VLBM_BUILDER_PLATES_Y:  // parallelPlatesBounceBack_Y.cu:57-159
        if (y == 0) w = make_word(VLBM_BC_BOUNCE_BACK, VLBM_SOUTH);
        else if (y == ny - 1) w = make_word(VLBM_BC_BOUNCE_BACK, VLBM_NORTH);
        break;
    case VLBM_BUILDER_PLATES_Y_FREE_SLIP:  // parallelPlatesBounceBackFreeSlip.cu
        if (y == 0) w = make_word(VLBM_BC_BOUNCE_BACK, VLBM_SOUTH);
        else if (y == ny - 1) w = make_word(VLBM_BC_FREE_SLIP, VLBM_NORTH);
        break;
    case VLBM_BUILDER_PLATES_Y_ZOUHE:  // couetteZouHe.cu
        if (y == 0) w = make_word(VLBM_BC_VEL_ZOUHE, VLBM_SOUTH, 0, 0, 2);
        else if (y == ny - 1) w = make_word(VLBM_BC_VEL_ZOUHE, VLBM_NORTH, 0, 0, 1);
        break;
    case VLBM_BUILDER_LID_DRIVEN:  // lidDrivenBounceBack.cu:57-170 (z periodic)
    case VLBM_BUILDER_SQUARE_DUCT: {  // squareDuctBounceBack.cu (z periodic)
        d = combine_dir(side(y, ny, true), side(x, nx, true), 0);
        if (d < 0) break;
        if (builder == VLBM_BUILDER_LID_DRIVEN && d == VLBM_NORTH)
            w = make_word(VLBM_BC_VEL_BOUNCE_BACK, VLBM_NORTH, 1);
        else
            w = make_word(VLBM_BC_BOUNCE_BACK, d);
        break;
    }
    case VLBM_BUILDER_DUCT_YZ:  // walls y and z, periodic x
        d = combine_dir(side(y, ny, true), 0, side(z, nz, true));
        if (d >= 0) w = make_word(VLBM_BC_BOUNCE_BACK, d);
        break;
    case VLBM_BUILDER_CLOSED_BOX:  // closedBoxBounceBack.cu:56-208
    case VLBM_BUILDER_LID_CAVITY_CLOSED:
        d = combine_dir(side(y, ny, true), side(x, nx, true), side(z, nz, true));
        if (d < 0) break;
        if (builder == VLBM_BUILDER_LID_CAVITY_CLOSED && d == VLBM_NORTH)
            w = make_word(VLBM_BC_VEL_BOUNCE_BACK, VLBM_NORTH, 1);
        else
            w = make_word(VLBM_BC_BOUNCE_BACK, d);
        break;
    default:
        return false;
    }
    return true;
}

namespace {

bool needs_slot(uint32_t m) {
    const int scheme = (m >> VLBM_MAP_SCHEME_OFFSET) & 7;
    const bool save = (m >> VLBM_MAP_SAVE_POST_COL_OFFSET) & 1u;
    return scheme != VLBM_BC_NULL || save;
}

// Boundary records from the candidate nodes (node index, map word) of the
// nodes whose word asks for a slot, in increasing node order.  word_at(k)
// gives the word of any node (free-slip neighbours).
template <class WordAt>
vlbm_status tables_from_candidates(const vlbm_config& cfg, std::vector<std::pair<size_t, uint32_t>>& cand,
                                   WordAt word_at, BcTables& out) {
    const int Q = cfg.vel_set;
    const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
    // Free-slip reads post-collision populations of tangential neighbours
    // (freeSlip.cu:26-167); make sure those neighbours keep them.
    const size_t ncand = cand.size();
    bool added = false;
    for (size_t c = 0; c < ncand; ++c) {
        const size_t k = cand[c].first;
        const uint32_t m = cand[c].second;
        if (((m >> VLBM_MAP_SCHEME_OFFSET) & 7) != VLBM_BC_FREE_SLIP) continue;
        const int dir = (m >> VLBM_MAP_DIRECTION_OFFSET) & 31;
        if (dir > VLBM_BACK) continue;
        int nrm[3][3];
        dir_normals(dir, nrm);
        const int x = (int)(k % nx), y = (int)((k / nx) % ny), z = (int)(k / ((size_t)nx * ny));
        for (int i = 1; i < Q; ++i) {
            if (bb_role(dir, i) != 1) continue;
            int t[3] = {lat_cx(i), lat_cy(i), lat_cz(i)};
            for (int a = 0; a < 3; ++a) if (nrm[0][a] != 0) t[a] = 0;
            const int xs = ((x - t[0]) % nx + nx) % nx, ys = ((y - t[1]) % ny + ny) % ny,
                      zs = ((z - t[2]) % nz + nz) % nz;
            const size_t kn = (size_t)nx * ((size_t)ny * zs + ys) + xs;
            cand.emplace_back(kn, word_at(kn));
            added = true;
        }
    }
    if (added) {
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    }
    // bounce-back role masks per direction
    uint32_t role_mask[26];
    for (int d = 0; d < 26; ++d) {
        role_mask[d] = 0;
        for (int i = 1; i < Q; ++i)
            if (bb_role(d, i) == 1) role_mask[d] |= 1u << i;
    }
    out.recs.clear();
    out.bc_nodes.clear();
    out.recs.reserve(cand.size());
    out.bc_nodes.reserve(cand.size());
    uint32_t last_word = 0;
    BcRec last{};
    bool have_last = false;
    for (const auto& kw : cand) {
        const uint32_t m = kw.second;
        if (!have_last || m != last_word) {   // the record depends on the word only
            const int scheme = (m >> VLBM_MAP_SCHEME_OFFSET) & 7;
            const int dir = (m >> VLBM_MAP_DIRECTION_OFFSET) & 31;
            const int geo = (m >> VLBM_MAP_GEOMETRY_OFFSET) & 1;
            BcRec r;
            std::memset(&r, 0, sizeof(r));
            r.scheme = K_BC_NONE;
            r.dir = (uint8_t)dir;
            r.uw[0] = (float)cfg.ux_bc[(m >> VLBM_MAP_UX_IDX_OFFSET) & 7];
            r.uw[1] = (float)cfg.uy_bc[(m >> VLBM_MAP_UY_IDX_OFFSET) & 7];
            r.uw[2] = (float)cfg.uz_bc[(m >> VLBM_MAP_UZ_IDX_OFFSET) & 7];
            r.rhow = (float)cfg.rho_bc[(m >> VLBM_MAP_RHO_IDX_OFFSET) & 7];
            int nrm[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            dir_normals(dir, nrm);
            r.axis = nrm[0][0] != 0 ? 0 : (nrm[0][1] != 0 ? 1 : 2);
            const uint32_t mask = dir < 26 ? role_mask[dir] : 0u;
            switch (scheme) {
            case VLBM_BC_BOUNCE_BACK:
                // edges/corners act only when concave (boundaryConditionsHandler.cu:158-256)
                if (dir < VLBM_NORTH_WEST || geo == VLBM_CONCAVE) { r.scheme = K_BC_BOUNCE; r.mask = mask; }
                break;
            case VLBM_BC_VEL_BOUNCE_BACK:
                // faces only (boundaryConditionsHandler.cu:274-304); D3Q27 extends the D3Q19 rule
                if (dir <= VLBM_BACK) { r.scheme = K_BC_VEL_BOUNCE; r.mask = mask; }
                break;
            case VLBM_BC_FREE_SLIP:
                if (dir <= VLBM_BACK) { r.scheme = K_BC_FREE_SLIP; r.mask = mask; }
                break;
            case VLBM_BC_VEL_ZOUHE:
                // D3Q19 faces only; the reference compiles an empty body for D3Q27
                if (Q == 19 && dir <= VLBM_BACK) { r.scheme = K_BC_VEL_ZOUHE; r.mask = mask; }
                break;
            case VLBM_BC_PRES_ZOUHE:
                if (Q == 19 && dir <= VLBM_BACK) { r.scheme = K_BC_PRES_ZOUHE; r.mask = mask; }
                break;
            default: break;
            }
            last = r;
            last_word = m;
            have_last = true;
        }
        out.recs.push_back(last);
        out.bc_nodes.push_back((int32_t)kw.first);
    }
    return VLBM_OK;
}

}  // namespace

vlbm_status build_bc_tables(const vlbm_config& cfg, const uint32_t* map, size_t n, BcTables& out,
                            std::string& err) {
    const size_t N = (size_t)cfg.nx * cfg.ny * cfg.nz;
    if (n != N) { err = "node map size does not match nx*ny*nz"; return VLBM_ERR_INVALID; }
    std::vector<std::pair<size_t, uint32_t>> cand;
    for (size_t k = 0; k < N; ++k) {
        const uint32_t m = map[k];
        if (!((m >> VLBM_MAP_IS_USED_OFFSET) & 1u)) {
            err = "nodes marked unused (interpolated-bounce-back duct builders) are not supported";
            return VLBM_ERR_UNSUPPORTED;
        }
        const int scheme = (m >> VLBM_MAP_SCHEME_OFFSET) & 7;
        if (scheme == VLBM_BC_INTERP_BOUNCE_BACK || scheme == VLBM_BC_SPECIAL) {
            err = "interpolated bounce-back and builder-specific (SPECIAL) schemes are not supported";
            return VLBM_ERR_UNSUPPORTED;
        }
        if (needs_slot(m)) cand.emplace_back(k, m);
    }
    return tables_from_candidates(cfg, cand, [map](size_t k) { return map[k]; }, out);
}

vlbm_status build_bc_tables_builder(const vlbm_config& cfg, int builder, BcTables& out, std::string& err) {
    const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
    uint32_t w;
    if (!builder_word(builder, 0, 0, 0, nx, ny, nz, w)) { err = "unknown builder id"; return VLBM_ERR_NOT_FOUND; }
    auto word_at = [&](size_t k) {
        uint32_t m;
        builder_word(builder, (int)(k % nx), (int)((k / nx) % ny), (int)(k / ((size_t)nx * ny)), nx, ny, nz, m);
        return m;
    };
    // the builders mark domain-face nodes only: visit the six faces
    std::vector<std::pair<size_t, uint32_t>> cand;
    auto visit = [&](int x, int y, int z) {
        uint32_t m;
        builder_word(builder, x, y, z, nx, ny, nz, m);
        if (needs_slot(m)) cand.emplace_back((size_t)nx * ((size_t)ny * z + y) + x, m);
    };
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y) {
            const bool face_yz = (z == 0 || z == nz - 1 || y == 0 || y == ny - 1);
            if (face_yz) {
                for (int x = 0; x < nx; ++x) visit(x, y, z);
            } else {
                visit(0, y, z);
                if (nx > 1) visit(nx - 1, y, z);
            }
        }
    return tables_from_candidates(cfg, cand, word_at, out);
}

}  // namespace vlbm

using namespace vlbm;

extern "C" vlbm_status vlbm_build_node_map(int builder, int nx, int ny, int nz, uint32_t* map_out,
                                           size_t n) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !map_out) { set_last_error("invalid builder arguments"); return VLBM_ERR_INVALID; }
    if (n != (size_t)nx * ny * nz) { set_last_error("map size does not match nx*ny*nz"); return VLBM_ERR_INVALID; }
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                uint32_t w;
                if (!builder_word(builder, x, y, z, nx, ny, nz, w)) {
                    set_last_error("unknown builder id");
                    return VLBM_ERR_NOT_FOUND;
                }
                map_out[(size_t)nx * ((size_t)ny * z + y) + x] = w;
            }
    return VLBM_OK;
}
