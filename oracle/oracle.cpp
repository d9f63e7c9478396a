// oracle.cpp -- FP64 CPU restatement of the VISCOPLASTIC-LBM fluid time step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product:
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may load
// it.  It is never linked into libvlbm and the product never falls back to it.
//
// It restates the reference's algorithm as the reference runs it on the GPU
// (push streaming into a second buffer, ghost-plane z wrap == periodic wrap,
// then a boundary-condition pass that reads post-streaming populations and the
// post-collision populations kept at boundary nodes, then a buffer swap), in
// double precision, with OpenMP over nodes.  Paths cited are inside
// CERNN/VISCOPLASTIC-LBM (src/CUDA/...).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "../include/vlbm.h"

namespace {

// ---------------------------------------------------------------- lattice --
// src/CUDA/velocitySets/D3Q19.h:31-46 and D3Q27.h:39-56 (same ordering).
const int CX[27] = {0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 0, 0, 1,-1, 1,-1, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1};
const int CY[27] = {0, 0, 0, 1,-1, 0, 0, 1,-1, 0, 0, 1,-1,-1, 1, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1, 1,-1};
const int CZ[27] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 1,-1, 1,-1, 0, 0,-1, 1,-1, 1, 1,-1,-1, 1, 1,-1, 1,-1};

double weight(int Q, int i) {
    int s = std::abs(CX[i]) + std::abs(CY[i]) + std::abs(CZ[i]);
    if (Q == 19) { const double w[3] = {1.0 / 3, 1.0 / 18, 1.0 / 36}; return w[s]; }
    const double w[4] = {8.0 / 27, 2.0 / 27, 1.0 / 54, 1.0 / 216};
    return w[s];
}
int opposite(int Q, int i) {
    for (int j = 0; j < Q; ++j)
        if (CX[j] == -CX[i] && CY[j] == -CY[i] && CZ[j] == -CZ[i]) return j;
    return -1;
}
int find_pop(int Q, int cx, int cy, int cz) {
    for (int j = 0; j < Q; ++j)
        if (CX[j] == cx && CY[j] == cy && CZ[j] == cz) return j;
    return -1;
}

// Outward normals of the wall set named by a direction code
// (src/CUDA/structs/nodeTypeMap.h:59-85: NORTH is y=NY-1, SOUTH y=0, WEST x=0,
// EAST x=NX-1, FRONT z=NZ-1, BACK z=0, and their combinations).
int direction_normals(int dir, int n[3][3]) {
    // bit per face: N S W E F B
    static const int faces[26] = {
        /*N*/ 1, /*S*/ 2, /*W*/ 4, /*E*/ 8, /*F*/ 16, /*B*/ 32,
        /*NW*/ 1 | 4, /*NE*/ 1 | 8, /*NF*/ 1 | 16, /*NB*/ 1 | 32,
        /*SW*/ 2 | 4, /*SE*/ 2 | 8, /*SF*/ 2 | 16, /*SB*/ 2 | 32,
        /*WF*/ 4 | 16, /*WB*/ 4 | 32, /*EF*/ 8 | 16, /*EB*/ 8 | 32,
        /*NWF*/ 1 | 4 | 16, /*NWB*/ 1 | 4 | 32, /*NEF*/ 1 | 8 | 16, /*NEB*/ 1 | 8 | 32,
        /*SWF*/ 2 | 4 | 16, /*SWB*/ 2 | 4 | 32, /*SEF*/ 2 | 8 | 16, /*SEB*/ 2 | 8 | 32};
    static const int nrm[6][3] = {{0, 1, 0}, {0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 0, 1}, {0, 0, -1}};
    if (dir < 0 || dir > 25) return 0;
    int k = 0;
    for (int f = 0; f < 6; ++f)
        if (faces[dir] & (1 << f)) { for (int a = 0; a < 3; ++a) n[k][a] = nrm[f][a]; ++k; }
    return k;
}

// Half-way bounce-back at a face, edge or corner node
// (src/CUDA/boundaryConditionsSchemes/bounceBack.cu:26-498): a population that
// arrived from outside through every wall it crosses is replaced by the
// post-collision opposite of the same node; one that crosses one wall from
// outside while leaving through another ("dead pop" in the reference comments,
// e.g. bounceBack.cu:149) keeps its streamed value.
enum PopRole { KNOWN = 0, BOUNCED = 1, DEAD = 2 };
PopRole bb_role(int Q, int dir, int i) {
    (void)Q;
    int n[3][3];
    int k = direction_normals(dir, n);
    bool neg = false, pos = false;
    for (int a = 0; a < k; ++a) {
        int s = CX[i] * n[a][0] + CY[i] * n[a][1] + CZ[i] * n[a][2];
        if (s < 0) neg = true;
        if (s > 0) pos = true;
    }
    if (neg && pos) return DEAD;
    if (neg) return BOUNCED;
    return KNOWN;
}

struct Node { int x, y, z; };

struct OSim {
    vlbm_config cfg;
    int Q, nx, ny, nz;
    size_t N;
    std::vector<double> pop, popAux;  // [Q][N], idxPop without the ghost plane
    std::vector<uint32_t> map;        // reference node map
    std::vector<double> omega;        // Power-Law state / last omega (macr.omega)
    std::vector<double> fibm[3];      // per-node IBM force (macr.f minus FX..FZ)
    std::vector<size_t> bcNodes;      // setupBoundaryConditionsInfo list
    long long step = 0;
};

inline size_t idx(const OSim& s, int x, int y, int z) {
    return (size_t)s.nx * ((size_t)s.ny * z + y) + x;  // idxScalar globalFunctions.h:111-115
}
inline int wrapi(int v, int n) { v %= n; return v < 0 ? v + n : v; }

inline bool map_used(uint32_t m) { return (m >> VLBM_MAP_IS_USED_OFFSET) & 1u; }
inline int map_scheme(uint32_t m) { return (m >> VLBM_MAP_SCHEME_OFFSET) & 7u; }
inline int map_dir(uint32_t m) { return (m >> VLBM_MAP_DIRECTION_OFFSET) & 31u; }
inline int map_geo(uint32_t m) { return (m >> VLBM_MAP_GEOMETRY_OFFSET) & 1u; }
inline int map_ux(uint32_t m) { return (m >> VLBM_MAP_UX_IDX_OFFSET) & 7u; }
inline int map_uy(uint32_t m) { return (m >> VLBM_MAP_UY_IDX_OFFSET) & 7u; }
inline int map_uz(uint32_t m) { return (m >> VLBM_MAP_UZ_IDX_OFFSET) & 7u; }
inline int map_rho(uint32_t m) { return (m >> VLBM_MAP_RHO_IDX_OFFSET) & 7u; }
// nodeTypeMap.h:158-163: post-collision populations are kept at every BC node
// and at nodes flagged SAVE_POST_COL.
inline bool map_save(uint32_t m) {
    return ((m >> VLBM_MAP_SAVE_POST_COL_OFFSET) & 1u) || map_scheme(m) != VLBM_BC_NULL;
}

double feq(int Q, int i, double rho, double ux, double uy, double uz) {
    // gpu_f_eq globalFunctions.h:50-56
    double uc = ux * CX[i] + uy * CY[i] + uz * CZ[i];
    double uu = ux * ux + uy * uy + uz * uz;
    return weight(Q, i) * rho * (1.0 - 1.5 * uu + 3.0 * uc + 4.5 * uc * uc);
}

// Relaxation frequency: nnf.h:32-87 calcOmega, lbm.cu:209-222 selection.
double calc_omega(const OSim& s, double omegaOld, double auxStressMag) {
    const vlbm_config& c = s.cfg;
    if (c.rheology == VLBM_BINGHAM) {
        double omegaP = 1.0 / (3.0 * c.eta_p + 0.5);           // nnf.h:128
        return omegaP * std::max(0.0, 1.0 - c.yield_stress / auxStressMag);  // nnf.h:188
    }
    if (c.rheology == VLBM_POWERLAW) {
        double eta = ((1.0 / omegaOld) - 0.5) / 3.0;            // nnf.h:146
        double gammaDot = (1.0 - 0.5 * omegaOld) * auxStressMag / eta;  // nnf.h:149
        if (gammaDot <= c.gamma0) eta = c.k_consistency;        // nnf.h:151-153
        else eta = c.k_consistency * std::pow(gammaDot, c.n_index - 1.0);  // nnf.h:155
        return 1.0 / (0.5 + 3.0 * eta);                         // nnf.h:158
    }
    return 1.0 / c.tau;                                         // var.h:105
}

struct Moments {
    double rho, ux, uy, uz;
    double pxx, pyy, pzz, pxy, pxz, pyz;  // momNeq (off-diagonals NOT doubled)
    double aux;                            // auxStressMag
};

// lbm.cu:79-111 (rho, u with half force), lbm.cu:149-190 (momNeq),
// lbm.cu:192-208 (auxStressMag).
Moments moments(const OSim& s, const double* f, double fx, double fy, double fz) {
    Moments m{};
    double rho = 0, jx = 0, jy = 0, jz = 0, sxx = 0, syy = 0, szz = 0, sxy = 0, sxz = 0, syz = 0;
    for (int i = 0; i < s.Q; ++i) {
        rho += f[i];
        jx += f[i] * CX[i]; jy += f[i] * CY[i]; jz += f[i] * CZ[i];
        sxx += f[i] * CX[i] * CX[i]; syy += f[i] * CY[i] * CY[i]; szz += f[i] * CZ[i] * CZ[i];
        sxy += f[i] * CX[i] * CY[i]; sxz += f[i] * CX[i] * CZ[i]; syz += f[i] * CY[i] * CZ[i];
    }
    m.rho = rho;
    m.ux = (jx + 0.5 * fx) / rho;
    m.uy = (jy + 0.5 * fy) / rho;
    m.uz = (jz + 0.5 * fz) / rho;
    const double cs2 = 1.0 / 3.0;
    m.pxx = sxx - rho * (m.ux * m.ux + cs2);
    m.pyy = syy - rho * (m.uy * m.uy + cs2);
    m.pzz = szz - rho * (m.uz * m.uz + cs2);
    m.pxy = sxy - rho * m.ux * m.uy;
    m.pxz = sxz - rho * m.ux * m.uz;
    m.pyz = syz - rho * m.uy * m.uz;
    const double uFxx = m.ux * fx, uFyy = m.uy * fy, uFzz = m.uz * fz;
    const double uFxy = (m.ux * fy + m.uy * fx) / 2, uFxz = (m.ux * fz + m.uz * fx) / 2,
                 uFyz = (m.uy * fz + m.uz * fy) / 2;
    m.aux = std::sqrt(0.5 * ((m.pxx + uFxx) * (m.pxx + uFxx) + (m.pyy + uFyy) * (m.pyy + uFyy) +
                             (m.pzz + uFzz) * (m.pzz + uFzz) +
                             2 * ((m.pxy + uFxy) * (m.pxy + uFxy) + (m.pxz + uFxz) * (m.pxz + uFxz) +
                                  (m.pyz + uFyz) * (m.pyz + uFyz))));
    return m;
}

// Guo force term w_i [3(c_i - u) + 9 (c_i.u) c_i] . F
// (lbm.cu:403-461; collisionForceNoReg.txt force terms).
double guo(int Q, int i, const Moments& m, double fx, double fy, double fz) {
    double cu = CX[i] * m.ux + CY[i] * m.uy + CZ[i] * m.uz;
    double gx = 3.0 * (CX[i] - m.ux) + 9.0 * cu * CX[i];
    double gy = 3.0 * (CY[i] - m.uy) + 9.0 * cu * CY[i];
    double gz = 3.0 * (CZ[i] - m.uz) + 9.0 * cu * CZ[i];
    return weight(Q, i) * (gx * fx + gy * fy + gz * fz);
}

// One node's collision. Regularized: lbm.cu:263-461
//   f* = (1-w) * 4.5 w_i (Q_i:Pi_neq - c_i.F/3) + f_eq + (1-w/2) F_i
// BGK: collisionForceNoReg.txt:1-141
//   f* = (1-w) f + w f_eq + (1-w/2) F_i
void collide(const OSim& s, const double* f, const Moments& m, double omega,
             double fx, double fy, double fz, double* out) {
    const int Q = s.Q;
    for (int i = 0; i < Q; ++i) {
        double eq = feq(Q, i, m.rho, m.ux, m.uy, m.uz);
        double force = (1.0 - 0.5 * omega) * guo(Q, i, m, fx, fy, fz);
        if (s.cfg.collision == VLBM_OP_BGK) {
            out[i] = (1.0 - omega) * f[i] + omega * eq + force;
        } else {
            const double cx = CX[i], cy = CY[i], cz = CZ[i];
            double qpi = (cx * cx - 1.0 / 3) * m.pxx + (cy * cy - 1.0 / 3) * m.pyy +
                         (cz * cz - 1.0 / 3) * m.pzz + 2.0 * (cx * cy * m.pxy + cx * cz * m.pxz + cy * cz * m.pyz);
            double cf = (cx * fx + cy * fy + cz * fz) / 3.0;
            out[i] = (1.0 - omega) * 4.5 * weight(Q, i) * (qpi - cf) + eq + force;
        }
    }
}

// ---------------------------------------------------- boundary conditions --
// popS = post-streaming buffer (fPostStream), popC = buffer holding post-collision
// values at saving nodes (fPostCol); see lbm.cu:463-470, main.cu:352-360.
inline double& PS(OSim& s, std::vector<double>& b, int i, size_t n) { return b[(size_t)i * s.N + n]; }

void bc_bounce_back(OSim& s, std::vector<double>& popS, const std::vector<double>& popC,
                    size_t n, int dir, int geo) {
    // Edges and corners act only when CONCAVE (boundaryConditionsHandler.cu:158-256).
    if (dir >= VLBM_NORTH_WEST && geo != VLBM_CONCAVE) return;
    for (int i = 1; i < s.Q; ++i)
        if (bb_role(s.Q, dir, i) == BOUNCED)
            popS[(size_t)i * s.N + n] = popC[(size_t)opposite(s.Q, i) * s.N + n];
}

// Moving-wall bounce-back, D3Q19_VelBounceBack.cu:27-147 (D3Q19 faces only in the
// reference, boundaryConditionsHandler.cu:274; the same rule is applied to the
// D3Q27 unknowns here).  Uses POST-STREAMING populations: the known opposite and
// rho_w = sum of all streamed populations of the node.
void bc_vel_bounce_back(OSim& s, std::vector<double>& popS, size_t n, int dir,
                        double uxw, double uyw, double uzw) {
    if (dir > VLBM_BACK) return;
    double rhow = 0;
    for (int i = 0; i < s.Q; ++i) rhow += popS[(size_t)i * s.N + n];
    double tmp[27];
    for (int i = 0; i < s.Q; ++i) tmp[i] = popS[(size_t)i * s.N + n];
    for (int i = 1; i < s.Q; ++i) {
        if (bb_role(s.Q, dir, i) != BOUNCED) continue;
        int o = opposite(s.Q, i);
        double cu = CX[o] * uxw + CY[o] * uyw + CZ[o] * uzw;
        popS[(size_t)i * s.N + n] = tmp[o] - 6.0 * rhow * weight(s.Q, i) * cu;
    }
}

// Free slip, freeSlip.cu:26-167: an unknown population is the post-collision
// population with the wall-normal component reflected, taken from the node one
// tangential step back along the population's direction.
void bc_free_slip(OSim& s, std::vector<double>& popS, const std::vector<double>& popC,
                  size_t n, int x, int y, int z, int dir) {
    if (dir > VLBM_BACK) return;
    int nr[3][3];
    direction_normals(dir, nr);
    for (int i = 1; i < s.Q; ++i) {
        if (bb_role(s.Q, dir, i) != BOUNCED) continue;
        int c[3] = {CX[i], CY[i], CZ[i]};
        int r[3] = {c[0], c[1], c[2]};
        int t[3] = {c[0], c[1], c[2]};
        for (int a = 0; a < 3; ++a)
            if (nr[0][a] != 0) { r[a] = -c[a]; t[a] = 0; }
        int j = find_pop(s.Q, r[0], r[1], r[2]);
        size_t src = idx(s, wrapi(x - t[0], s.nx), wrapi(y - t[1], s.ny), wrapi(z - t[2], s.nz));
        popS[(size_t)i * s.N + n] = popC[(size_t)j * s.N + src];
    }
}

// Velocity Zou-He, D3Q19_VelZouHe.cu:27-172, transcribed per face including the
// reference's own term choices (EAST overwrites the unknowns from themselves,
// WEST uses uy_w in pop 15, BACK divides by 1+uz_w).
void bc_vel_zouhe(OSim& s, std::vector<double>& popS, size_t n, int dir,
                  double ux, double uy, double uz) {
    if (s.Q != 19) return;
    double f[19];
    for (int i = 0; i < 19; ++i) f[i] = popS[(size_t)i * s.N + n];
    double g[19];
    std::memcpy(g, f, sizeof(g));
    switch (dir) {
    case VLBM_NORTH: {
        double rw = (1 / (1 + uy)) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                      2 * (f[3] + f[7] + f[14] + f[11] + f[17]));
        double nyx = 0.5 * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10])) - ux * rw / 3;
        double nyz = 0.5 * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10])) - uz * rw / 3;
        g[4] = f[3] + rw * (-uy) / 3;
        g[8] = f[7] + rw * (-uy - ux) / 6 + nyx;
        g[13] = f[14] + rw * (-uy + ux) / 6 - nyx;
        g[12] = f[11] + rw * (-uy - uz) / 6 + nyz;
        g[18] = f[17] + rw * (-uy + uz) / 6 - nyz;
        break; }
    case VLBM_SOUTH: {
        double rw = (1 / (1 - uy)) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                      2 * (f[4] + f[13] + f[8] + f[18] + f[12]));
        double nyx = 0.5 * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10])) - ux * rw / 3;
        double nyz = 0.5 * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10])) - uz * rw / 3;
        g[3] = f[4] + rw * uy / 3;
        g[7] = f[8] + rw * (uy + ux) / 6 - nyx;
        g[14] = f[13] + rw * (uy - ux) / 6 + nyx;
        g[11] = f[12] + rw * (uy + uz) / 6 - nyz;
        g[17] = f[18] + rw * (uy - uz) / 6 + nyz;
        break; }
    case VLBM_WEST: {
        double rw = (1 / (1 - ux)) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                      2 * (f[2] + f[14] + f[8] + f[16] + f[10]));
        double nxy = 0.5 * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12])) - uy * rw / 3;
        double nxz = 0.5 * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12])) - uz * rw / 3;
        g[1] = f[2] + rw * ux / 3;
        g[13] = f[14] + rw * (ux - uy) / 6 + nxy;
        g[7] = f[8] + rw * (ux + uy) / 6 - nxy;
        g[9] = f[10] + rw * (ux + uz) / 6 - nxz;
        g[15] = f[16] + rw * (ux - uy) / 6 + nxz;
        break; }
    case VLBM_EAST: {
        double rw = (1 / (1 + ux)) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                      2 * (f[2] + f[14] + f[8] + f[16] + f[10]));
        double nxy = 0.5 * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12])) - uy * rw / 3;
        double nxz = 0.5 * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12])) - uz * rw / 3;
        g[2] = f[2] + rw * ux / 3;
        g[14] = f[14] + rw * (ux - uy) / 6 + nxy;
        g[8] = f[8] + rw * (ux + uy) / 6 - nxy;
        g[10] = f[10] + rw * (ux + uz) / 6 - nxz;
        g[16] = f[16] + rw * (ux - uy) / 6 + nxz;
        break; }
    case VLBM_FRONT: {
        double rw = (1 / (1 + uz)) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                      2 * (f[5] + f[9] + f[16] + f[11] + f[18]));
        double nzx = 0.5 * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8])) - rw * ux / 3;
        double nzy = 0.5 * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8])) - rw * uy / 3;
        g[6] = f[5] + rw * (-uz) / 3;
        g[15] = f[16] + rw * (-uz + ux) / 6 - nzx;
        g[10] = f[9] + rw * (-uz - ux) / 6 + nzx;
        g[17] = f[18] + rw * (-uz + uy) / 6 - nzy;
        g[12] = f[11] + rw * (-uz - uy) / 6 + nzy;
        break; }
    case VLBM_BACK: {
        double rw = (1 / (1 + uz)) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                      2 * (f[6] + f[15] + f[10] + f[17] + f[12]));
        double nzx = 0.5 * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8])) - rw * ux / 3;
        double nzy = 0.5 * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8])) - rw * uy / 3;
        g[5] = f[6] + rw * uz / 3;
        g[9] = f[10] + rw * (uz + ux) / 6 - nzx;
        g[16] = f[15] + rw * (uz - ux) / 6 + nzx;
        g[11] = f[12] + rw * (uz + ux) / 6 - nzy;
        g[18] = f[17] + rw * (uz - ux) / 6 + nzy;
        break; }
    default: return;
    }
    for (int i = 0; i < 19; ++i) popS[(size_t)i * s.N + n] = g[i];
}

// Pressure Zou-He, D3Q19_PresZouHe.cu:27-176 (EAST again overwrites unknowns
// from themselves, as in the reference).
void bc_pres_zouhe(OSim& s, std::vector<double>& popS, size_t n, int dir, double rw) {
    if (s.Q != 19) return;
    double f[19];
    for (int i = 0; i < 19; ++i) f[i] = popS[(size_t)i * s.N + n];
    double g[19];
    std::memcpy(g, f, sizeof(g));
    switch (dir) {
    case VLBM_NORTH: {
        double uy = -1 + (1 / rw) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                     2 * (f[3] + f[7] + f[14] + f[11] + f[17]));
        double nyx = 0.5 * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10]));
        double nyz = 0.5 * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10]));
        g[4] = f[3] + rw * (-uy) / 3;
        g[8] = f[7] + rw * (-uy) / 6 + nyx;
        g[13] = f[14] + rw * (-uy) / 6 - nyx;
        g[12] = f[11] + rw * (-uy) / 6 + nyz;
        g[18] = f[17] + rw * (-uy) / 6 - nyz;
        break; }
    case VLBM_SOUTH: {
        double uy = 1 - (1 / rw) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                    2 * (f[4] + f[13] + f[8] + f[18] + f[12]));
        double nyx = 0.5 * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10]));
        double nyz = 0.5 * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10]));
        g[3] = f[4] + rw * uy / 3;
        g[7] = f[8] + rw * uy / 6 - nyx;
        g[14] = f[13] + rw * uy / 6 + nyx;
        g[11] = f[12] + rw * uy / 6 - nyz;
        g[17] = f[18] + rw * uy / 6 + nyz;
        break; }
    case VLBM_WEST: {
        double ux = 1 - (1 / rw) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                    2 * (f[2] + f[14] + f[8] + f[16] + f[10]));
        double nxy = 0.5 * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12]));
        double nxz = 0.5 * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12]));
        g[1] = f[2] + rw * ux / 3;
        g[13] = f[14] + rw * ux / 6 + nxy;
        g[7] = f[8] + rw * ux / 6 - nxy;
        g[9] = f[10] + rw * ux / 6 - nxz;
        g[15] = f[16] + rw * ux / 6 + nxz;
        break; }
    case VLBM_EAST: {
        double ux = -1 + (1 / rw) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                     2 * (f[2] + f[14] + f[8] + f[16] + f[10]));
        double nxy = 0.5 * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12]));
        double nxz = 0.5 * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12]));
        g[2] = f[2] + rw * ux / 3;
        g[14] = f[14] + rw * ux / 6 + nxy;
        g[8] = f[8] + rw * ux / 6 - nxy;
        g[10] = f[10] + rw * ux / 6 - nxz;
        g[16] = f[16] + rw * ux / 6 + nxz;
        break; }
    case VLBM_FRONT: {
        double uz = -1 + (1 / rw) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                     2 * (f[5] + f[9] + f[16] + f[11] + f[18]));
        double nzx = 0.5 * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8]));
        double nzy = 0.5 * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8]));
        g[6] = f[5] + rw * (-uz) / 3;
        g[15] = f[16] + rw * (-uz) / 6 - nzx;
        g[10] = f[9] + rw * (-uz) / 6 + nzx;
        g[17] = f[18] + rw * (-uz) / 6 - nzy;
        g[12] = f[11] + rw * (-uz) / 6 + nzy;
        break; }
    case VLBM_BACK: {
        double uz = 1 - (1 / rw) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                    2 * (f[6] + f[10] + f[12] + f[15] + f[17]));
        double nzx = 0.5 * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8]));
        double nzy = 0.5 * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8]));
        g[5] = f[6] + rw * uz / 3;
        g[9] = f[10] + rw * uz / 6 - nzx;
        g[16] = f[15] + rw * uz / 6 + nzx;
        g[11] = f[12] + rw * uz / 6 - nzy;
        g[18] = f[17] + rw * uz / 6 + nzy;
        break; }
    default: return;
    }
    for (int i = 0; i < 19; ++i) popS[(size_t)i * s.N + n] = g[i];
}

// gpuBoundaryConditions dispatch, boundaryConditionsHandler.cu:25-79.
void apply_bc(OSim& s, std::vector<double>& popS, const std::vector<double>& popC, size_t n) {
    uint32_t m = s.map[n];
    int x = (int)(n % s.nx), y = (int)((n / s.nx) % s.ny), z = (int)(n / ((size_t)s.nx * s.ny));
    int dir = map_dir(m);
    switch (map_scheme(m)) {
    case VLBM_BC_BOUNCE_BACK: bc_bounce_back(s, popS, popC, n, dir, map_geo(m)); break;
    case VLBM_BC_VEL_BOUNCE_BACK:
        bc_vel_bounce_back(s, popS, n, dir, s.cfg.ux_bc[map_ux(m)], s.cfg.uy_bc[map_uy(m)],
                           s.cfg.uz_bc[map_uz(m)]);
        break;
    case VLBM_BC_FREE_SLIP: bc_free_slip(s, popS, popC, n, x, y, z, dir); break;
    case VLBM_BC_VEL_ZOUHE:
        bc_vel_zouhe(s, popS, n, dir, s.cfg.ux_bc[map_ux(m)], s.cfg.uy_bc[map_uy(m)], s.cfg.uz_bc[map_uz(m)]);
        break;
    case VLBM_BC_PRES_ZOUHE: bc_pres_zouhe(s, popS, n, dir, s.cfg.rho_bc[map_rho(m)]); break;
    default: break;
    }
}

}  // namespace

// ------------------------------------------------------------------ C API --
extern "C" {

struct oracle_sim;

oracle_sim* oracle_create(const vlbm_config* cfg, const uint32_t* map) {
    OSim* s = new OSim();
    s->cfg = *cfg;
    s->Q = cfg->vel_set;
    s->nx = cfg->nx; s->ny = cfg->ny; s->nz = cfg->nz;
    s->N = (size_t)s->nx * s->ny * s->nz;
    s->pop.assign((size_t)s->Q * s->N, 0.0);
    s->popAux.assign((size_t)s->Q * s->N, 0.0);
    s->map.assign(map, map + s->N);
    s->omega.assign(s->N, 0.0);  // lbmInitialization.cu:111 (omega = 0)
    for (int a = 0; a < 3; ++a) s->fibm[a].assign(s->N, 0.0);
    // lbmInitialization.cu:48-90: f = f_eq(RHO_0, 0) in both buffers
    for (int i = 0; i < s->Q; ++i) {
        double e = feq(s->Q, i, cfg->rho0, 0, 0, 0);
        std::fill(s->pop.begin() + (size_t)i * s->N, s->pop.begin() + (size_t)(i + 1) * s->N, e);
        std::fill(s->popAux.begin() + (size_t)i * s->N, s->popAux.begin() + (size_t)(i + 1) * s->N, e);
    }
    // setupBoundaryConditionsInfo (boundaryConditionsInfo.h:76-116): list of
    // nodes whose scheme is not BC_NULL.
    for (size_t n = 0; n < s->N; ++n)
        if (map_scheme(s->map[n]) != VLBM_BC_NULL) s->bcNodes.push_back(n);
    return reinterpret_cast<oracle_sim*>(s);
}

void oracle_destroy(oracle_sim* h) { delete reinterpret_cast<OSim*>(h); }

void oracle_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// One reference time step (main.cu:300-367): collide + push stream, z wrap,
// boundary conditions, swap.
void oracle_step(oracle_sim* h, int nsteps) {
    OSim& s = *reinterpret_cast<OSim*>(h);
    const int Q = s.Q;
    for (int it = 0; it < nsteps; ++it) {
#pragma omp parallel for schedule(static)
        for (long long zz = 0; zz < (long long)s.nz; ++zz) {
            double f[27], out[27];
            const int z = (int)zz;
            for (int y = 0; y < s.ny; ++y)
                for (int x = 0; x < s.nx; ++x) {
                    size_t n = idx(s, x, y, z);
                    uint32_t m = s.map[n];
                    if (!map_used(m)) continue;                    // lbm.cu:23-24
                    for (int i = 0; i < Q; ++i) f[i] = s.pop[(size_t)i * s.N + n];
                    // IBM force read and reset (lbm.cu:45-58)
                    double fx = s.cfg.fx + s.fibm[0][n], fy = s.cfg.fy + s.fibm[1][n],
                           fz = s.cfg.fz + s.fibm[2][n];
                    s.fibm[0][n] = s.fibm[1][n] = s.fibm[2][n] = 0.0;
                    Moments mo = moments(s, f, fx, fy, fz);
                    double om = calc_omega(s, s.omega[n], mo.aux);
                    s.omega[n] = om;                                  // lbm.cu:215-219
                    collide(s, f, mo, om, fx, fy, fz, out);
                    if (map_save(m))                                   // lbm.cu:463-470
                        for (int i = 0; i < Q; ++i) s.pop[(size_t)i * s.N + n] = out[i];
                    for (int i = 0; i < Q; ++i) {                      // lbm.cu:472-503
                        size_t d = idx(s, wrapi(x + CX[i], s.nx), wrapi(y + CY[i], s.ny),
                                       wrapi(z + CZ[i], s.nz));
                        s.popAux[(size_t)i * s.N + d] = out[i];
                    }
                }
        }
        // gpuApplyBC (lbm.cu:580-598): each BC node writes only its own slots.
#pragma omp parallel for schedule(static)
        for (long long k = 0; k < (long long)s.bcNodes.size(); ++k)
            apply_bc(s, s.popAux, s.pop, s.bcNodes[(size_t)k]);
        std::swap(s.pop, s.popAux);                                    // populations.h:63-70
        ++s.step;
    }
}

// Macroscopics of the current state, as gpuMacrCollisionStream saves them
// (lbm.cu:79-111, 247-261; omega per lbm.cu:209-222).  Non-mutating.
void oracle_macro(oracle_sim* h, double* rho, double* ux, double* uy, double* uz, double* omega) {
    OSim& s = *reinterpret_cast<OSim*>(h);
#pragma omp parallel for schedule(static)
    for (long long nn = 0; nn < (long long)s.N; ++nn) {
        size_t n = (size_t)nn;
        double f[27];
        for (int i = 0; i < s.Q; ++i) f[i] = s.pop[(size_t)i * s.N + n];
        double fx = s.cfg.fx + s.fibm[0][n], fy = s.cfg.fy + s.fibm[1][n], fz = s.cfg.fz + s.fibm[2][n];
        Moments mo = moments(s, f, fx, fy, fz);
        if (rho) rho[n] = mo.rho;
        if (ux) ux[n] = mo.ux;
        if (uy) uy[n] = mo.uy;
        if (uz) uz[n] = mo.uz;
        if (omega) omega[n] = calc_omega(s, s.omega[n], mo.aux);
    }
}

void oracle_get_pops(oracle_sim* h, double* out) {
    OSim& s = *reinterpret_cast<OSim*>(h);
    std::memcpy(out, s.pop.data(), s.pop.size() * sizeof(double));
}
void oracle_set_pops(oracle_sim* h, const double* in) {
    OSim& s = *reinterpret_cast<OSim*>(h);
    std::memcpy(s.pop.data(), in, s.pop.size() * sizeof(double));
}
void oracle_set_omega(oracle_sim* h, const double* in) {
    OSim& s = *reinterpret_cast<OSim*>(h);
    std::memcpy(s.omega.data(), in, s.N * sizeof(double));
}
long long oracle_step_count(oracle_sim* h) { return reinterpret_cast<OSim*>(h)->step; }

// Role of population i at a bounce-back node with direction `dir`
// (0 known, 1 bounced, 2 dead) -- exported so tests can pin the rule to the
// reference's tables.
int oracle_bb_role(int Q, int dir, int i) { return (int)bb_role(Q, dir, i); }

// Free-slip source (population index and tangential offset) for unknown i.
int oracle_free_slip_source(int Q, int dir, int i, int* off3) {
    int nr[3][3];
    direction_normals(dir, nr);
    if (bb_role(Q, dir, i) != BOUNCED) return -1;
    int c[3] = {CX[i], CY[i], CZ[i]}, r[3] = {c[0], c[1], c[2]}, t[3] = {c[0], c[1], c[2]};
    for (int a = 0; a < 3; ++a)
        if (nr[0][a] != 0) { r[a] = -c[a]; t[a] = 0; }
    for (int a = 0; a < 3; ++a) off3[a] = -t[a];
    return find_pop(Q, r[0], r[1], r[2]);
}

}  // extern "C"

extern "C" void oracle_lattice(int i, int* c3) {
    c3[0] = CX[i]; c3[1] = CY[i]; c3[2] = CZ[i];
}
extern "C" double oracle_weight(int Q, int i) { return weight(Q, i); }
