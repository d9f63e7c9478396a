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
#include <cmath>
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

// Cylinder of the duct builders (var.h:142-162): radii (<= 0: the var.h
// values OUTER_RADIUS = NY/2 - 1.5, INNER_RADIUS = OUTER_RADIUS/4) and the
// centre DUCT_CENTER_X/Y in the builders' node coordinates x + 0.5, as the
// builders hold them (dfloat = float).
struct Duct {
    float R, r, cx, cy;
};
Duct duct_of(int nx, int ny, double outer, double inner) {
    Duct d;
    const double R = outer > 0 ? outer : ny / 2.0 - 1.5;
    d.R = (float)R;
    d.r = (float)(inner > 0 ? inner : R / 4.0);
    d.cx = (float)((nx - 1) / 2.0 + 0.5);
    d.cy = (float)((ny - 1) / 2.0 + 0.5);
    return d;
}

// distPoints2D (globalFunctions.h:159-162) in float.
float dist2f(float x1, float y1, float x2, float y2) {
    const float dx = x1 - x2, dy = y1 - y2;
    const float s = dx * dx + dy * dy;
    return std::sqrt(s);
}

// Word of node (x, y) of circularDuctInterpBounceBack.cu:35-123 (annular:
// annularDuctInterpBounceBack.cu:35-140); the cross-section is the same in
// every z plane.
uint32_t duct_word(bool annular, int x, int y, int nx, int ny, const Duct& d) {
    // used, no post-collision save, BC_NULL, CONCAVE, value indices 0; the
    // annular builder also sets the direction FRONT on every node
    uint32_t w = make_word(VLBM_BC_NULL, annular ? VLBM_FRONT : 0);
    const float xNode = (float)x + 0.5f, yNode = (float)y + 0.5f;
    const float dist = dist2f(xNode, yNode, d.cx, d.cy);
    const float s2 = std::sqrt(2.0f);
    auto set_interp = [&](bool inside) {
        w &= ~((7u << VLBM_MAP_SCHEME_OFFSET) | (31u << VLBM_MAP_DIRECTION_OFFSET));
        w |= (uint32_t)VLBM_BC_INTERP_BOUNCE_BACK << VLBM_MAP_SCHEME_OFFSET;
        w |= (uint32_t)(inside ? VLBM_SOUTH : VLBM_NORTH) << VLBM_MAP_DIRECTION_OFFSET;
    };
    const uint32_t save = 1u << VLBM_MAP_SAVE_POST_COL_OFFSET;
    if (!annular) {
        if (dist > d.R) return w & ~(1u << VLBM_MAP_IS_USED_OFFSET);
        if (dist > d.R - s2) set_interp(false);
        else if (dist > d.R - 2 * s2) w |= save;
        else return w;
    } else {
        if (dist > d.R || dist < d.r) w &= ~(1u << VLBM_MAP_IS_USED_OFFSET);
        else if (dist > d.R - s2) set_interp(false);
        else if (dist > d.R - 2 * s2) w |= save;
        else if (dist < d.r + s2) set_interp(true);
        else if (dist < d.r + 2 * s2) w |= save;
    }
    for (int i = 0; i < 8; ++i) {   // unknown: the node the population comes from is outside
        const float xa = xNode - (float)kInterpDirs[i][0], ya = yNode - (float)kInterpDirs[i][1];
        bool unknown = true;
        if (xa < (float)nx && xa > 0.f && ya < (float)ny && ya > 0.f) {
            const float da = dist2f(xa, ya, d.cx, d.cy);
            unknown = da > d.R || (annular && da < d.r);
        }
        if (unknown) w |= (1u << i) << VLBM_MAP_INTERP_BB_OFFSET;
    }
    return w;
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
bool builder_word(int builder, int x, int y, int z, int nx, int ny, int nz, uint32_t& w, double outer_radius,
                  double inner_radius) {
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
    case VLBM_BUILDER_CIRCULAR_DUCT:
    case VLBM_BUILDER_ANNULAR_DUCT:
        w = duct_word(builder == VLBM_BUILDER_ANNULAR_DUCT, x, y, nx, ny,
                      duct_of(nx, ny, outer_radius, inner_radius));
        break;
    default:
        return false;
    }
    return true;
}

namespace {

// A node gets a boundary slot when its word names a scheme.  SAVE_POST_COL
// alone asks the reference to keep post-collision populations for a
// neighbour's rule; here those arrive with the streamed populations (the
// interpolated bounce-back reads them at gather time), so no slot is needed.
bool needs_slot(uint32_t m) {
    if (!((m >> VLBM_MAP_IS_USED_OFFSET) & 1u)) return false;
    return ((m >> VLBM_MAP_SCHEME_OFFSET) & 7) != VLBM_BC_NULL;
}

// Normalised wall distance along a link (interpolatedBounceBack.cu:374-431,
// gpuDistNormalizedFromNodePopulationToWall_*), in double.  (x1, y1): the
// node, (x2, y2): the node the population comes from, R: the cylinder radius;
// coordinates relative to the duct axis.
double wall_a0(double x1, double y1, double x2, double y2, double R) {   // horizontal link
    const double y = y2;
    double x = std::sqrt(R * R - y * y);
    if (x2 < 0) x = -x;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1));
}
double wall_ainf(double x1, double y1, double x2, double y2, double R) {   // vertical link
    const double x = x2;
    double y = std::sqrt(R * R - x * x);
    if (y2 < 0) y = -y;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1));
}
double wall_diag(double x1, double y1, double x2, double y2, double R, bool slope_up) {   // _ap1 / _am1
    const double b = slope_up ? y1 - x1 : y1 + x1;
    const double dr = std::sqrt(2 * R * R - b * b);
    double x = slope_up ? (-b + dr) * 0.5 : (b + dr) * 0.5;
    if ((x1 > x2 && (x > x1 || x < x2)) || (x1 < x2 && (x < x1 || x > x2)))
        x = slope_up ? (-b - dr) * 0.5 : (b - dr) * 0.5;
    const double y = slope_up ? x + b : -x + b;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1)) / std::sqrt(2.0);
}

// Record of an interpolated bounce-back node (interpolatedBounceBack.cu:6-372):
// unknown populations from the in-plane direction bits; per direction the
// coefficients (A, B, K) of f_i = A f*_o + B (f*_i or f_o) + K w_i (c_i . u_w),
// (1/(2q), (q-1/2)/q, 3/q) with f*_i where q > 1/2
// (gpuInterpolatedBounceBackHigherQ), (2q, 1-2q, 6) with the streamed f_o
// otherwise (LowerQ), interpolatedBounceBack.h; and the wall velocity at the
// node: rotation about the axis plus axial velocity (the outer rotation grows
// with z/NZ as in the reference).
void interp_record(const vlbm_config& cfg, int x, int y, int z, uint32_t m, BcRec& r, float* coef /* [8][3] */) {
    const int Q = cfg.vel_set;
    const double R = cfg.duct_outer_radius > 0 ? cfg.duct_outer_radius : cfg.ny / 2.0 - 1.5;
    const double ri = cfg.duct_inner_radius > 0 ? cfg.duct_inner_radius : R / 4.0;
    const int dir = (m >> VLBM_MAP_DIRECTION_OFFSET) & 31;
    const bool inside = dir == VLBM_SOUTH;
    const unsigned bits = (m >> VLBM_MAP_INTERP_BB_OFFSET) & 0xFFu;
    const double xn = x - (cfg.nx - 1) / 2.0, yn = y - (cfg.ny - 1) / 2.0;
    const double rad = inside ? ri : R;
    std::memset(&r, 0, sizeof(r));
    r.scheme = K_BC_INTERP;
    r.dir = (uint8_t)dir;
    for (int i = 1; i < Q; ++i) {
        const int d = interp_dir_of(lat_cx(i), lat_cy(i));
        if (d >= 0 && ((bits >> d) & 1u)) r.mask |= 1u << i;
    }
    for (int d = 0; d < 8; ++d) {
        double A = 0.0, B = 0.0, K = 0.0;
        if ((bits >> d) & 1u) {
            const double x2 = xn - kInterpDirs[d][0], y2 = yn - kInterpDirs[d][1];
            double q;
            if (d == 0 || d == 2) q = wall_a0(xn, yn, x2, y2, rad);
            else if (d == 1 || d == 3) q = wall_ainf(xn, yn, x2, y2, rad);
            else q = wall_diag(xn, yn, x2, y2, rad, d == 4 || d == 6);
            if (q > 0.5) { A = 0.5 / q; B = (q - 0.5) / q; K = 3.0 / q; r.pad |= (uint8_t)(1u << d); }
            else { A = 2 * q; B = 1 - 2 * q; K = 6.0; }
        }
        coef[3 * d] = (float)A;
        coef[3 * d + 1] = (float)B;
        coef[3 * d + 2] = (float)K;
    }
    const double rr = std::sqrt(xn * xn + yn * yn);
    const double c = rr > 0 ? xn / rr : 0.0, s = rr > 0 ? yn / rr : 0.0;
    const bool slab = cfg.slab_nz_total != 0;   // z of the whole lattice for a z-slab
    const double zg = slab ? (double)((cfg.slab_z_offset + z) % cfg.slab_nz_total) : (double)z;
    const double w = inside ? cfg.duct_inner_rotation
                            : cfg.duct_outer_rotation * (zg / (double)(slab ? cfg.slab_nz_total : cfg.nz));
    r.uw[0] = (float)(-w * rad * s);
    r.uw[1] = (float)(w * rad * c);
    r.uw[2] = (float)(inside ? cfg.duct_inner_velocity : cfg.duct_outer_velocity);
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
            if (cfg.slab_nz_total != 0 && t[2] != 0) return VLBM_ERR_UNSUPPORTED;   // neighbour in another slab
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
    out.q8.clear();
    for (const auto& kw : cand) {
        const uint32_t m = kw.second;
        if (((m >> VLBM_MAP_SCHEME_OFFSET) & 7) == VLBM_BC_INTERP_BOUNCE_BACK) {   // per-node record
            const size_t k = kw.first;
            if (out.q8.empty()) out.q8.assign(24 * cand.size(), 0.f);
            BcRec r;
            interp_record(cfg, (int)(k % nx), (int)((k / nx) % ny), (int)(k / ((size_t)nx * ny)), m, r,
                          out.q8.data() + 24 * out.recs.size());
            out.recs.push_back(r);
            out.bc_nodes.push_back((int32_t)k);
            continue;
        }
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
    out.unused_nodes.clear();
    for (size_t k = 0; k < N; ++k) {
        const uint32_t m = map[k];
        if (!((m >> VLBM_MAP_IS_USED_OFFSET) & 1u)) {   // lbm.cu:23-24
            out.unused_nodes.push_back((int32_t)k);
            continue;
        }
        const int scheme = (m >> VLBM_MAP_SCHEME_OFFSET) & 7;
        if (scheme == VLBM_BC_SPECIAL) {
            err = "builder-specific (SPECIAL) schemes are not supported";
            return VLBM_ERR_UNSUPPORTED;
        }
        if (needs_slot(m)) cand.emplace_back(k, m);
    }
    const vlbm_status st = tables_from_candidates(cfg, cand, [map](size_t k) { return map[k]; }, out);
    if (st == VLBM_ERR_UNSUPPORTED)
        err = "free-slip walls normal to x or y read post-collision values of z neighbours, which a z-slab's "
              "ghost planes do not hold";
    return st;
}

vlbm_status build_bc_tables_builder(const vlbm_config& cfg, int builder, BcTables& out, std::string& err) {
    const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
    if (cfg.slab_nz_total != 0) {
        err = "a z-slab takes its node map from vlbm_build_node_map_planes, not a builder id";
        return VLBM_ERR_INVALID;
    }
    uint32_t w;
    if (!builder_word(builder, 0, 0, 0, nx, ny, nz, w)) { err = "unknown builder id"; return VLBM_ERR_NOT_FOUND; }
    auto word_at = [&](size_t k) {
        uint32_t m;
        builder_word(builder, (int)(k % nx), (int)((k / nx) % ny), (int)(k / ((size_t)nx * ny)), nx, ny, nz, m,
                     cfg.duct_outer_radius, cfg.duct_inner_radius);
        return m;
    };
    std::vector<std::pair<size_t, uint32_t>> cand;
    out.unused_nodes.clear();
    if (builder == VLBM_BUILDER_CIRCULAR_DUCT || builder == VLBM_BUILDER_ANNULAR_DUCT) {
        // the cross-section is the same in every plane: classify one, repeat it along z
        std::vector<std::pair<int, uint32_t>> plane_cand;
        std::vector<int> plane_unused;
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const uint32_t m = word_at((size_t)nx * y + x);
                if (!((m >> VLBM_MAP_IS_USED_OFFSET) & 1u)) plane_unused.push_back(nx * y + x);
                else if (needs_slot(m)) plane_cand.emplace_back(nx * y + x, m);
            }
        const size_t plane = (size_t)nx * ny;
        for (int z = 0; z < nz; ++z) {
            for (const auto& pc : plane_cand) cand.emplace_back(plane * z + pc.first, pc.second);
            for (int u : plane_unused) out.unused_nodes.push_back((int32_t)(plane * z + u));
        }
        return tables_from_candidates(cfg, cand, word_at, out);
    }
    // the other builders mark domain-face nodes only: visit the six faces
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

extern "C" vlbm_status vlbm_build_node_map_planes(int builder, int nx, int ny, int nz, int z_first, int n_planes,
                                                  uint32_t* map_out, size_t n) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || n_planes <= 0 || !map_out) {
        set_last_error("invalid builder arguments");
        return VLBM_ERR_INVALID;
    }
    if (n != (size_t)nx * ny * n_planes) { set_last_error("map size does not match nx*ny*n_planes"); return VLBM_ERR_INVALID; }
    for (int k = 0; k < n_planes; ++k) {
        const int z = (int)((((long long)z_first + k) % nz + nz) % nz);
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                uint32_t w;
                if (!builder_word(builder, x, y, z, nx, ny, nz, w)) {
                    set_last_error("unknown builder id");
                    return VLBM_ERR_NOT_FOUND;
                }
                map_out[(size_t)nx * ((size_t)ny * k + y) + x] = w;
            }
    }
    return VLBM_OK;
}

extern "C" vlbm_status vlbm_build_node_map(int builder, int nx, int ny, int nz, uint32_t* map_out, size_t n) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !map_out) { set_last_error("invalid builder arguments"); return VLBM_ERR_INVALID; }
    if (n != (size_t)nx * ny * nz) { set_last_error("map size does not match nx*ny*nz"); return VLBM_ERR_INVALID; }
    return vlbm_build_node_map_planes(builder, nx, ny, nz, 0, nz, map_out, n);
}
