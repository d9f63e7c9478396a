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
        double omegaP = 1.0 / (3.0 * c.eta_p + 0.5);           // nnf.h:23
        return omegaP * std::max(0.0, 1.0 - c.yield_stress / auxStressMag);  // nnf.h:83
    }
    if (c.rheology == VLBM_POWERLAW) {
        // nnf.h:41-44: eta_old = (1/omega_old - 1/2)/3, gammaDot = (1 - omega_old/2)|S|/eta_old.
        // Since 1 - omega_old/2 = 3 omega_old eta_old, gammaDot = 3 omega_old |S|: the same value
        // in exact arithmetic, evaluated in that form because the quotient is 0/0 where
        // omega_old rounds to 2 (shear-thickening fluid at rest), and omega_old = 0 (the
        // initial state, lbmInitialization.cu:111) gives gammaDot = 0 as the reference's
        // |S|/inf does.
        double eta;
        const double gammaDot = 3.0 * omegaOld * auxStressMag;
        if (gammaDot <= c.gamma0) eta = c.k_consistency;        // nnf.h:46-48
        else eta = c.k_consistency * std::pow(gammaDot, c.n_index - 1.0);  // nnf.h:50
        return 1.0 / (0.5 + 3.0 * eta);                         // nnf.h:53
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

// Interpolated bounce-back on a cylinder along z, interpolatedBounceBack.cu:6-372
// (BC_RHEOMETER false, var.h:162).  Node coordinates relative to the axis
// (x - (NX-1)/2, y - (NY-1)/2); wall velocity from the rotation and axial
// velocity of the outer (direction NORTH) or inner (SOUTH) cylinder, the outer
// rotation scaled by z/NZ_TOTAL (:29-58).
double wall_dist_a0(double x1, double y1, double x2, double y2, double R) {       // :374-389
    double y = y2, x = std::sqrt(R * R - y * y);
    if (x2 < 0) x = -x;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1));
}
double wall_dist_ainf(double x1, double y1, double x2, double y2, double R) {     // :392-407
    double x = x2, y = std::sqrt(R * R - x * x);
    if (y2 < 0) y = -y;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1));
}
double wall_dist_ap1(double x1, double y1, double x2, double y2, double R) {      // :410-430
    double b = y1 - x1, dr = std::sqrt(2 * R * R - b * b), x = (-b + dr) * 0.5;
    if ((x1 > x2 && (x > x1 || x < x2)) || (x1 < x2 && (x < x1 || x > x2))) x = (-b - dr) * 0.5;
    double y = x + b;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1)) / std::sqrt(2.0);
}
double wall_dist_am1(double x1, double y1, double x2, double y2, double R) {
    double b = y1 + x1, dr = std::sqrt(2 * R * R - b * b), x = (b + dr) * 0.5;
    if ((x1 > x2 && (x > x1 || x < x2)) || (x1 < x2 && (x < x1 || x > x2))) x = (b - dr) * 0.5;
    double y = -x + b;
    return std::sqrt((x - x1) * (x - x1) + (y - y1) * (y - y1)) / std::sqrt(2.0);
}

void bc_interp_bounce_back(OSim& s, std::vector<double>& popS, const std::vector<double>& popC, size_t n,
                           int x, int y, int z, uint32_t m) {
    const vlbm_config& c = s.cfg;
    const double R = c.duct_outer_radius > 0 ? c.duct_outer_radius : c.ny / 2.0 - 1.5;
    const double r = c.duct_inner_radius > 0 ? c.duct_inner_radius : R / 4.0;
    const bool inside = map_dir(m) == VLBM_SOUTH;
    const unsigned bits = (m >> VLBM_MAP_INTERP_BB_OFFSET) & 0xFFu;
    const double xNode = x - (s.nx - 1) / 2.0, yNode = y - (s.ny - 1) / 2.0;
    const double rr = std::sqrt(xNode * xNode + yNode * yNode);
    const double cs = xNode / rr, sn = yNode / rr;
    double ux, uy, uz, radius;
    if (inside) {
        radius = r;
        ux = -c.duct_inner_rotation * r * sn;
        uy = c.duct_inner_rotation * r * cs;
        uz = c.duct_inner_velocity;
    } else {
        radius = R;
        const double w_o = c.duct_outer_rotation * ((double)z / (double)s.nz);
        ux = -w_o * R * sn;
        uy = w_o * R * cs;
        uz = c.duct_outer_velocity;
    }
    static const int dirs[8][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
    for (int d = 0; d < 8; ++d) {
        if (!((bits >> d) & 1u)) continue;
        const double x2 = xNode - dirs[d][0], y2 = yNode - dirs[d][1];
        double q;
        if (d == 0 || d == 2) q = wall_dist_a0(xNode, yNode, x2, y2, radius);
        else if (d == 1 || d == 3) q = wall_dist_ainf(xNode, yNode, x2, y2, radius);
        else if (d == 4 || d == 6) q = wall_dist_ap1(xNode, yNode, x2, y2, radius);
        else q = wall_dist_am1(xNode, yNode, x2, y2, radius);
        for (int i = 1; i < s.Q; ++i) {
            if (CX[i] != dirs[d][0] || CY[i] != dirs[d][1]) continue;
            const int o = opposite(s.Q, i);
            const double df = weight(s.Q, i) * (CX[i] * ux + CY[i] * uy + CZ[i] * uz);
            const double fBound = popC[(size_t)o * s.N + n];
            double v;
            if (q > 0.5) {   // gpuInterpolatedBounceBackHigherQ (interpolatedBounceBack.h)
                v = (0.5 / q) * fBound + ((q - 0.5) / q) * popC[(size_t)i * s.N + n] + 3.0 * df / q;
            } else {         // gpuInterpolatedBounceBackLowerQ: the opposite at the node x + c_i
                const size_t na = idx(s, wrapi(x + CX[i], s.nx), wrapi(y + CY[i], s.ny), wrapi(z + CZ[i], s.nz));
                v = 2 * q * fBound + (1 - 2 * q) * popC[(size_t)o * s.N + na] + 2 * 3.0 * df;
            }
            popS[(size_t)i * s.N + n] = v;
        }
    }
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
    case VLBM_BC_INTERP_BOUNCE_BACK: bc_interp_bounce_back(s, popS, popC, n, x, y, z, m); break;
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
        if (map_scheme(s->map[n]) != VLBM_BC_NULL && map_used(s->map[n])) s->bcNodes.push_back(n);
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
        if (!map_used(s.map[n])) {   // never updated: the initial values (lbmInitialization.cu:100-111)
            if (rho) rho[n] = s.cfg.rho0;
            if (ux) ux[n] = 0.0;
            if (uy) uy[n] = 0.0;
            if (uz) uz[n] = 0.0;
            if (omega) omega[n] = 0.0;
            continue;
        }
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

// =====================================================================
// Immersed boundary method for movable spheres (src/CUDA/IBM/), FP64.
// =====================================================================
namespace {

const int MAX_SLOTS = 13;  // MAX_ACTIVE_COLLISIONS, ibmBoundaryCondition.h:78

struct OPart {
    double pos[3], pos_old[3], vel[3], vel_old[3], w[3], w_avg[3], w_old[3], w_pos[3];
    double f[3], f_old[3], M[3], M_old[3];
    double I[6];  // xx yy zz xy xz yz
    double dP[3], dL[3];
    double S, radius, volume, density;
    int movable;
    int partner[MAX_SLOTS];
    int last[MAX_SLOTS];
    double tdisp[MAX_SLOTS][3];
};

struct ONodes {
    std::vector<double> x, y, z, S, fx, fy, fz, dfx, dfy, dfz;
    std::vector<int> pidx;
};

struct OIbm {
    OSim* fluid;
    vlbm_ibm_config ib;
    std::vector<OPart> parts;
    ONodes nodes;
    std::vector<double> mrho, mu[3], faux[3], vaux[3];  // macr rho,u and IBM auxiliaries
};

// Sphere surface mesh, Particle::makeSpherePolar (IBM/structs/particle.cpp:698-995),
// without the optional Coulomb relaxation (MESH_COULOMB 0).  Positions relative
// to the centre.
int sphere_mesh(double diameter, double mesh_scale, double breugem, std::vector<double>& px,
                std::vector<double>& py, std::vector<double>& pz, std::vector<double>& pS) {
    double r = diameter / 2.0 - breugem;
    unsigned nLayer = (unsigned)(2.0 * std::sqrt(2.0) * r / mesh_scale + 1.0);
    std::vector<unsigned> nl(nLayer + 1);
    std::vector<double> theta(nLayer + 1), zeta(nLayer + 1), S(nLayer + 1);
    unsigned total = 0;
    for (unsigned i = 0; i <= nLayer; ++i) {
        theta[i] = M_PI * ((double)i / (double)nLayer - 0.5);
        nl[i] = (unsigned)(1.5 + std::cos(theta[i]) * nLayer * std::sqrt(3.0));
        total += nl[i];
        zeta[i] = r * std::sin(theta[i]);
    }
    for (unsigned i = 0; i < nLayer; ++i) S[i] = (zeta[i] + zeta[i + 1]) / 2.0 - zeta[0];
    S[nLayer] = 2 * r;
    for (unsigned i = 0; i <= nLayer; ++i) S[i] = 2 * M_PI * r * S[i];
    for (unsigned i = nLayer; i > 0; --i) S[i] = S[i] - S[i - 1];
    S[0] = S[nLayer];
    px.assign(total, 0); py.assign(total, 0); pz.assign(total, 0); pS.assign(total, 0);
    pz[0] = r * std::sin(theta[0]);
    pS[0] = S[0];
    unsigned k = 1;
    double phase = 0.0;
    for (unsigned i = 1; i < nLayer; ++i) {
        if (i % 2 == 1) phase = phase + M_PI / nl[i];
        for (unsigned j = 0; j < nl[i]; ++j) {
            px[k] = r * std::cos(theta[i]) * std::cos((double)j * 2.0 * M_PI / nl[i] + phase);
            py[k] = r * std::cos(theta[i]) * std::sin((double)j * 2.0 * M_PI / nl[i] + phase);
            pz[k] = r * std::sin(theta[i]);
            pS[k] = S[i] / nl[i];
            ++k;
        }
    }
    pz[total - 1] = r * std::sin(theta[nLayer]);
    pS[total - 1] = S[nLayer];
    return (int)total;
}

// Peskin 4-point kernel, ibmGlobalFunctions.h:28-48 (STENCIL_4).
double stencil4(double x) {
    double a = std::fabs(x);
    if (a <= 1) return (1.0 / 8.0) * (3.0 - 2.0 * a + std::sqrt(1 + 4 * a - 4 * a * a));
    if (a <= 2.0) return (1.0 / 8.0) * (5.0 - 2.0 * a - std::sqrt(-7.0 + 12.0 * a - 4.0 * a * a));
    return 0.0;
}

// Minimum-image difference along a periodic axis (ibm.cu:349-374).
double periodic_delta(double d, double L) {
    if (std::fabs(d) > L / 2.0) d = d < 0 ? d + L : d - L;
    return d;
}

void cross(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// ---- contacts (IBM/collision/ibmCollision.cu) ----
int wall_index(const double n[3]) {  // calculateWallIndex :5-19
    return 7 + (1 - (int)n[0]) - 2 * (1 - (int)n[1]) - 3 * (1 - (int)n[2]);
}
// getCollisionIndexByPartnerID :21-31
int find_slot(const OPart& p, int partner, int step) {
    for (int i = 7; i < MAX_SLOTS; ++i)
        if (p.partner[i] == partner && step - p.last[i] <= 1) return i;
    return -1;
}
// startCollision :32-53 for particle partners.  A slot whose contact ended
// (last step older than step-1) is free again: the reference frees slots only
// in endCollision, which its lookup never reaches, so its slots run out after
// six distinct partners and the next update writes index -1.
int start_pair_slot(OPart& p, int partner, int step) {
    for (int i = 7; i < MAX_SLOTS; ++i) {
        if (p.last[i] == -1 || step - p.last[i] > 1) {
            p.partner[i] = partner;
            p.tdisp[i][0] = p.tdisp[i][1] = p.tdisp[i][2] = 0.0;
            p.last[i] = step;
            return i;
        }
    }
    return -1;
}
void update_tdisp(OPart& p, int idx, const double d[3], int step, double out[3]) {
    if (idx < 0) { out[0] = d[0]; out[1] = d[1]; out[2] = d[2]; return; }
    for (int a = 0; a < 3; ++a) p.tdisp[idx][a] += d[a];
    p.last[idx] = step;
    for (int a = 0; a < 3; ++a) out[a] = p.tdisp[idx][a];
}

struct ContactConst {
    double ss_n, sw_n, ss_t, sw_t, dpp, dpw;
};
ContactConst contact_constants(const vlbm_ibm_config& c) {
    // ibmBoundaryCondition.h:93-107
    ContactConst k;
    double Gp = c.particle_young / (2.0 + 2.0 * c.particle_poisson);
    double Gw = c.wall_young / (2.0 + 2.0 * c.wall_poisson);
    double np2 = c.particle_poisson * c.particle_poisson, nw2 = c.wall_poisson * c.wall_poisson;
    k.ss_n = (4.0 / 3.0) / ((1 - np2) / c.particle_young + (1 - np2) / c.particle_young);
    k.sw_n = (4.0 / 3.0) / ((1 - np2) / c.particle_young + (1 - nw2) / c.wall_young);
    k.ss_t = 4.0 * std::sqrt(2.0) / ((2 - c.particle_poisson) / Gp + (2 - c.particle_poisson) / Gp);
    k.sw_t = 4.0 * std::sqrt(2.0) / ((2 - c.particle_poisson) / Gp + (2 - c.wall_poisson) / Gw);
    double lpp = std::log(c.pp_restitution), lpw = std::log(c.pw_restitution);
    k.dpp = -2.0 * lpp / std::sqrt(M_PI * M_PI + lpp * lpp);
    k.dpw = -2.0 * lpw / std::sqrt(M_PI * M_PI + lpw * lpw);
    return k;
}

// sphereWallCollision :393-508
void sphere_wall(OPart& p, const double wall_normal[3], double disp, int step, const ContactConst& K,
                 double mu) {
    const double m = p.volume * p.density, r = p.radius;
    double n[3] = {-wall_normal[0], -wall_normal[1], -wall_normal[2]};
    const double* G = p.vel;
    const double kn = K.sw_n * std::sqrt(std::fabs(r));
    const double kt = K.sw_t * std::sqrt(r) * std::sqrt(std::fabs(disp));
    const double etan = K.dpw * std::sqrt(m * kn), etat = K.dpw * std::sqrt(m * kt);
    const double fkn = -kn * std::sqrt(std::fabs(disp * disp * disp));
    const double Gn = G[0] * n[0] + G[1] * n[1] + G[2] * n[2];
    const double q = std::pow(std::fabs(disp), 0.25);
    double fnv[3];
    for (int a = 0; a < 3; ++a) fnv[a] = fkn * n[a] - etan * Gn * n[a] * q;
    const double fn = std::sqrt(fnv[0] * fnv[0] + fnv[1] * fnv[1] + fnv[2] * fnv[2]);
    double wxn[3];
    cross(p.w, n, wxn);
    double Gct[3];
    for (int a = 0; a < 3; ++a) Gct[a] = G[a] + r * wxn[a] - Gn * n[a];
    double mag = std::sqrt(Gct[0] * Gct[0] + Gct[1] * Gct[1] + Gct[2] * Gct[2]);
    double t[3] = {0, 0, 0};
    if (mag != 0) for (int a = 0; a < 3; ++a) t[a] = Gct[a] / mag;
    const int idx = wall_index(n);
    double td[3];
    if (step - p.last[idx] > 1) {
        p.last[idx] = -1;                                     // endCollision
        p.tdisp[idx][0] = p.tdisp[idx][1] = p.tdisp[idx][2] = 0.0;  // startCollision
        p.last[idx] = step;
        for (int a = 0; a < 3; ++a) td[a] = Gct[a];
    } else {
        update_tdisp(p, idx, Gct, step, td);
    }
    double ft[3];
    for (int a = 0; a < 3; ++a) ft[a] = -kt * td[a] - etat * Gct[a] * std::pow(std::fabs(td[a]), 0.25);
    mag = std::sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
    if (mag > mu * std::fabs(fn)) {
        double mg[3] = {-Gct[0], -Gct[1], -Gct[2]};
        update_tdisp(p, idx, mg, step, td);
        for (int a = 0; a < 3; ++a) ft[a] = -mu * fn * t[a];
    }
    double nxf[3];
    cross(n, ft, nxf);
    for (int a = 0; a < 3; ++a) {
        p.f[a] += fnv[a] + ft[a];
        p.M[a] += r * nxf[a];
    }
}

// sphereSphereCollision :1718-1913 (column i < row j; slots live in particle i)
void sphere_sphere(OIbm& s, int i, int j, int step, const ContactConst& K) {
    OPart& pi = s.parts[i];
    OPart& pj = s.parts[j];
    const OSim& fl = *s.fluid;
    const double L[3] = {(double)fl.nx, (double)fl.ny, (double)fl.nz};
    const int wall[3] = {s.ib.wall_x, s.ib.wall_y, s.ib.wall_z};
    double d[3];
    for (int a = 0; a < 3; ++a) {
        d[a] = pi.pos[a] - pj.pos[a];
        if (!wall[a]) d[a] = periodic_delta(d[a], L[a]);
    }
    const double dist = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (dist > pi.radius + pj.radius) return;
    double n[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
    const double disp = pi.radius + pj.radius - dist;
    double G[3] = {pi.vel[0] - pj.vel[0], pi.vel[1] - pj.vel[1], pi.vel[2] - pj.vel[2]};
    const double mi = pi.volume * pi.density, mj = pj.volume * pj.density;
    const double reff = 1.0 / ((pi.radius + pj.radius) / (pi.radius * pj.radius));
    const double meff = 1.0 / ((mi + mj) / (mi * mj));
    const double kn = K.ss_n * std::sqrt(reff);
    const double kt = K.ss_t * std::sqrt(reff) * std::sqrt(std::fabs(disp));
    const double etan = K.dpp * std::sqrt(meff * kn), etat = K.dpp * std::sqrt(meff * kt);
    const double fkn = -kn * std::sqrt(std::fabs(disp * disp * disp));
    const double Gn = G[0] * n[0] + G[1] * n[1] + G[2] * n[2];
    const double q = std::pow(std::fabs(disp), 0.25);
    double fnv[3];
    for (int a = 0; a < 3; ++a) fnv[a] = fkn * n[a] - etan * Gn * n[a] * q;
    const double fn = std::sqrt(fnv[0] * fnv[0] + fnv[1] * fnv[1] + fnv[2] * fnv[2]);
    double wi[3], wj[3];
    cross(pi.w, n, wi);
    cross(pj.w, n, wj);
    double Gct[3];
    for (int a = 0; a < 3; ++a) Gct[a] = G[a] + pi.radius * wi[a] + pj.radius * wj[a] - Gn * n[a];
    double mag = std::sqrt(Gct[0] * Gct[0] + Gct[1] * Gct[1] + Gct[2] * Gct[2]);
    double t[3] = {0, 0, 0};
    if (mag != 0) for (int a = 0; a < 3; ++a) t[a] = Gct[a] / mag;
    double td[3];
    int idx = find_slot(pi, j, step);
    if (idx == -1) {
        idx = start_pair_slot(pi, j, step);
        for (int a = 0; a < 3; ++a) td[a] = Gct[a];
    } else {
        update_tdisp(pi, idx, G, step, td);  // the reference accumulates G here (:1851)
    }
    double ft[3];
    for (int a = 0; a < 3; ++a) ft[a] = -kt * td[a] - etat * Gct[a] * std::pow(std::fabs(td[a]), 0.25);
    mag = std::sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
    if (mag > s.ib.pp_friction * std::fabs(fn)) {
        double mg[3] = {-Gct[0], -Gct[1], -Gct[2]};
        update_tdisp(pi, idx, mg, step, td);
        for (int a = 0; a < 3; ++a) ft[a] = -s.ib.pp_friction * fn * t[a];
    }
    double nxf[3];
    cross(n, ft, nxf);
    for (int a = 0; a < 3; ++a) {
        const double fd = fnv[a] + ft[a];
        pi.f[a] -= fd;
        pi.M[a] += pi.radius * nxf[a];
        pj.f[a] += fd;
        pj.M[a] += pj.radius * nxf[a];
    }
}

// checkCollisionWallsSphere :187-250 (walls at coordinate 0 and N-1 of wall axes)
void sphere_walls(OIbm& s, OPart& p, int step, const ContactConst& K) {
    const OSim& fl = *s.fluid;
    const int wall[3] = {s.ib.wall_x, s.ib.wall_y, s.ib.wall_z};
    const int L[3] = {fl.nx, fl.ny, fl.nz};
    for (int a = 0; a < 3; ++a) {
        if (!wall[a]) continue;
        double nlo[3] = {0, 0, 0}, nhi[3] = {0, 0, 0};
        nlo[a] = 1;
        nhi[a] = -1;
        double dlo = p.pos[a];
        if (dlo < p.radius) sphere_wall(p, nlo, p.radius - dlo, step, K, s.ib.pw_friction);
        double dhi = (L[a] - 1) - p.pos[a];
        if (dhi < p.radius) sphere_wall(p, nhi, p.radius - dhi, step, K, s.ib.pw_friction);
    }
}

// gpuUpdateParticleCenterVelocityAndRotation, ibm.cu:755-897
void update_center(OIbm& s, OPart& p) {
    if (!p.movable) return;
    const double al = s.ib.movement_alpha;
    const double inv_v = 1.0 / p.volume;
    const double g[3] = {s.ib.gx, s.ib.gy, s.ib.gz};
    for (int a = 0; a < 3; ++a)
        p.vel[a] = p.vel_old[a] + ((p.f_old[a] * (1.0 - al) + p.f[a] * al + p.dP[a]) * inv_v +
                                   (p.density - s.ib.fluid_density) * g[a]) / p.density;
    const double* I = p.I;
    const double Ixx = I[0], Iyy = I[1], Izz = I[2], Ixy = I[3], Ixz = I[4], Iyz = I[5];
    const double det = Izz * Ixy * Ixy + Iyy * Ixz * Ixz + Ixx * Iyz * Iyz - Ixx * Iyy * Izz - 2 * Ixy * Ixz * Iyz;
    const double inv = 1.0 / det;
    double wa[3], LM[3];
    for (int a = 0; a < 3; ++a) {
        wa[a] = p.w_old[a] * (1.0 - al) + p.w_old[a] * al;
        LM[a] = p.dL[a] + (p.M[a] * al + p.M_old[a] * (1.0 - al));
    }
    const double Lx = Ixx * wa[0] + Ixy * wa[1] + Ixz * wa[2];
    const double Ly = Ixy * wa[0] + Iyy * wa[1] + Iyz * wa[2];
    const double Lz = Ixz * wa[0] + Iyz * wa[1] + Izz * wa[2];
    // torque balance with gyroscopic term: T = LM + w x... (ibm.cu:838-850), solved with I^-1
    const double bx = LM[0] + wa[2] * Ly - wa[1] * Lz;
    const double by = LM[1] + wa[0] * Lz - wa[2] * Lx;
    const double bz = LM[2] + wa[1] * Lx - wa[0] * Ly;
    double wn[3];
    wn[0] = p.w_old[0] + ((Iyz * Iyz - Iyy * Izz) * bx - (Ixy * Iyz - Ixz * Iyy) * bz - (Ixz * Iyz - Ixy * Izz) * by) * inv;
    wn[1] = p.w_old[1] + ((Ixz * Ixz - Ixx * Izz) * by - (Ixy * Ixz - Ixx * Iyz) * bz - (Ixz * Iyz - Ixy * Izz) * bx) * inv;
    wn[2] = p.w_old[2] + ((Ixy * Ixy - Ixx * Iyy) * bz - (Ixy * Ixz - Ixx * Iyz) * by - (Ixy * Iyz - Ixz * Iyy) * bx) * inv;
    // inertia rotated by the quaternion of w_avg (ibm.cu:852-860): I <- R I R^T
    const double th = std::sqrt(wa[0] * wa[0] + wa[1] * wa[1] + wa[2] * wa[2]);
    if (th > 0 && std::isfinite(1.0 / th)) {
        const double h = std::sin(th / 2.0) / th;
        const double qw = std::cos(th / 2.0), qx = wa[0] * h, qy = wa[1] * h, qz = wa[2] * h;
        const double R[3][3] = {
            {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)},
            {2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)},
            {2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)}};
        const double M3[3][3] = {{Ixx, Ixy, Ixz}, {Ixy, Iyy, Iyz}, {Ixz, Iyz, Izz}};
        double T[3][3] = {}, O[3][3] = {};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) T[a][b] += R[a][c] * M3[c][b];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                for (int c = 0; c < 3; ++c) O[a][b] += T[a][c] * R[b][c];
        p.I[0] = O[0][0]; p.I[1] = O[1][1]; p.I[2] = O[2][2];
        p.I[3] = O[0][1]; p.I[4] = O[0][2]; p.I[5] = O[1][2];
    }
    for (int a = 0; a < 3; ++a) p.w[a] = wn[a];
}

// gpuForceInterpolationSpread, ibm.cu:194-542 (STENCIL_4), serial over nodes.
void interp_spread(OIbm& s) {
    OSim& fl = *s.fluid;
    const int L[3] = {fl.nx, fl.ny, fl.nz};
    const int wall[3] = {s.ib.wall_x, s.ib.wall_y, s.ib.wall_z};
    const size_t nn = s.nodes.x.size();
    for (size_t k = 0; k < nn; ++k) {
        const double pos[3] = {s.nodes.x[k], s.nodes.y[k], s.nodes.z[k]};
        int base[3], lo[3], hi[3];
        double st[3][4];
        bool skip = false;
        for (int a = 0; a < 3; ++a) {
            if (!(std::fabs(pos[a]) < 4.0 * L[a] + 8.0)) { skip = true; base[a] = 0; continue; }  // diverged
            base[a] = (int)pos[a] - 1;   // int(x) - P_DIST + 1
            lo[a] = 0; hi[a] = 3;
            if (wall[a]) {
                hi[a] = (base[a] + 3 < L[a]) ? 3 : (L[a] - 1 - base[a]);
                lo[a] = (base[a] >= 0) ? 0 : -base[a];
            }
            if (hi[a] <= 0 || lo[a] >= 4) skip = true;  // ibm.cu:300-305
            for (int j = 0; j < 4; ++j) st[a][j] = stencil4(base[a] + j - pos[a]);
        }
        if (skip) continue;
        auto node_of = [&](int a, int v) { return wall[a] ? v : ((v % L[a]) + L[a]) % L[a]; };
        double rho = 0, ux = 0, uy = 0, uz = 0;
        for (int zk = lo[2]; zk <= hi[2]; ++zk)
            for (int yj = lo[1]; yj <= hi[1]; ++yj)
                for (int xi = lo[0]; xi <= hi[0]; ++xi) {
                    const double d = st[2][zk] * st[1][yj] * st[0][xi];
                    const size_t n = idx(fl, node_of(0, base[0] + xi), node_of(1, base[1] + yj), node_of(2, base[2] + zk));
                    rho += s.mrho[n] * d; ux += s.mu[0][n] * d; uy += s.mu[1][n] * d; uz += s.mu[2][n] * d;
                }
        OPart& pc = s.parts[s.nodes.pidx[k]];
        double dr[3];
        for (int a = 0; a < 3; ++a) {
            dr[a] = pos[a] - pc.pos[a];
            if (!wall[a]) dr[a] = periodic_delta(dr[a], L[a]);
        }
        double uc[3] = {0, 0, 0};
        if (pc.movable) {
            double wxr[3];
            cross(pc.w, dr, wxr);
            for (int a = 0; a < 3; ++a) uc[a] = pc.vel[a] + wxr[a];
        }
        const double aux = 2 * rho * s.nodes.S[k] * s.ib.thickness;
        const double dF[3] = {aux * (ux - uc[0]), aux * (uy - uc[1]), aux * (uz - uc[2])};
        for (int zk = lo[2]; zk <= hi[2]; ++zk)
            for (int yj = lo[1]; yj <= hi[1]; ++yj)
                for (int xi = lo[0]; xi <= hi[0]; ++xi) {
                    const double d = st[2][zk] * st[1][yj] * st[0][xi];
                    const size_t n = idx(fl, node_of(0, base[0] + xi), node_of(1, base[1] + yj), node_of(2, base[2] + zk));
                    const double inv_rho = 1.0 / s.mrho[n];
                    for (int a = 0; a < 3; ++a) {
                        s.faux[a][n] += -dF[a] * d;
                        s.vaux[a][n] += 0.5 * -dF[a] * d * inv_rho;
                    }
                }
        s.nodes.fx[k] += dF[0]; s.nodes.fy[k] += dF[1]; s.nodes.fz[k] += dF[2];
        s.nodes.dfx[k] = dF[0]; s.nodes.dfy[k] = dF[1]; s.nodes.dfz[k] = dF[2];
        double m[3];
        cross(dr, dF, m);
        for (int a = 0; a < 3; ++a) { pc.f[a] += dF[a]; pc.M[a] += m[a]; }
    }
}

// gpuParticleMovement ibm.cu:899-993 and gpuParticleNodeMovement ibm.cu:1044-1197
void move(OIbm& s) {
    OSim& fl = *s.fluid;
    const int L[3] = {fl.nx, fl.ny, fl.nz};
    const int wall[3] = {s.ib.wall_x, s.ib.wall_y, s.ib.wall_z};
    const double al = s.ib.movement_alpha;
    for (OPart& p : s.parts) {
        if (!p.movable) continue;
        for (int a = 0; a < 3; ++a) {
            const double dx = p.vel[a] * al + p.vel_old[a] * (1.0 - al);
            if (wall[a]) p.pos[a] += dx;
            else p.pos[a] = std::fmod(p.pos[a] + dx + L[a], (double)L[a]);
            p.w_avg[a] = p.w[a] * al + p.w_old[a] * (1.0 - al);
            p.w_pos[a] += p.w_avg[a];
        }
    }
    const size_t nn = s.nodes.x.size();
    for (size_t k = 0; k < nn; ++k) {
        const OPart& p = s.parts[s.nodes.pidx[k]];
        if (!p.movable) continue;
        double* P[3] = {&s.nodes.x[k], &s.nodes.y[k], &s.nodes.z[k]};
        const double wn = std::sqrt(p.w_avg[0] * p.w_avg[0] + p.w_avg[1] * p.w_avg[1] + p.w_avg[2] * p.w_avg[2]);
        if (wn <= 1e-8) {
            for (int a = 0; a < 3; ++a) {
                double d = p.pos[a] - p.pos_old[a];
                if (wall[a]) { *P[a] += d; continue; }
                if (std::fabs(d) > L[a] / 2.0) d = (p.pos[a] < p.pos_old[a]) ? p.pos[a] + L[a] - p.pos_old[a]
                                                                            : p.pos[a] - L[a] - p.pos_old[a];
                *P[a] = std::fmod(*P[a] + d + L[a], (double)L[a]);
            }
            continue;
        }
        double v[3];
        for (int a = 0; a < 3; ++a) {
            if (!wall[a] && std::fabs(*P[a] - p.pos_old[a]) > L[a] / 2.0)
                *P[a] += (*P[a] < p.pos_old[a]) ? L[a] : -L[a];
            v[a] = *P[a] - p.pos_old[a];
        }
        const double q0 = std::cos(0.5 * wn);
        const double qi = (p.w_avg[0] / wn) * std::sin(0.5 * wn);
        const double qj = (p.w_avg[1] / wn) * std::sin(0.5 * wn);
        const double qk = (p.w_avg[2] / wn) * std::sin(0.5 * wn);
        const double t = q0 * q0 - 0.5;
        // rotation rows as the reference writes them (ibm.cu:1170-1172; the third
        // row uses qi*qj - q0*qj where the rotation matrix has qi*qk - q0*qj)
        double np[3];
        np[0] = p.pos[0] + 2 * ((t + qi * qi) * v[0] + (qi * qj - q0 * qk) * v[1] + (qi * qk + q0 * qj) * v[2]);
        np[1] = p.pos[1] + 2 * ((qi * qj + q0 * qk) * v[0] + (t + qj * qj) * v[1] + (qj * qk - q0 * qi) * v[2]);
        np[2] = p.pos[2] + 2 * ((qi * qj - q0 * qj) * v[0] + (qj * qk + q0 * qi) * v[1] + (t + qk * qk) * v[2]);
        for (int a = 0; a < 3; ++a)
            *P[a] = wall[a] ? np[a] : std::fmod(np[a] + L[a], (double)L[a]);
    }
}

void ibm_macro_all(OIbm& s) {
    // gpuUpdateMacrIBM ibm.cu:544-648: rho, u from post-boundary populations with FX..FZ only
    OSim& fl = *s.fluid;
#pragma omp parallel for schedule(static)
    for (long long nn = 0; nn < (long long)fl.N; ++nn) {
        size_t n = (size_t)nn;
        double f[27];
        for (int i = 0; i < fl.Q; ++i) f[i] = fl.pop[(size_t)i * fl.N + n];
        Moments mo = moments(fl, f, fl.cfg.fx, fl.cfg.fy, fl.cfg.fz);
        s.mrho[n] = mo.rho;
        s.mu[0][n] = mo.ux; s.mu[1][n] = mo.uy; s.mu[2][n] = mo.uz;
        for (int a = 0; a < 3; ++a) { s.faux[a][n] = 0; s.vaux[a][n] = 0; }
    }
}

void ibm_substep(OIbm& s, int step) {
    OSim& fl = *s.fluid;
    for (OPart& p : s.parts) {  // gpuUpdateParticleOldValues ibm.cu:995-1042
        for (int a = 0; a < 3; ++a) {
            p.dP[a] = 0; p.dL[a] = 0;
            p.pos_old[a] = p.pos[a]; p.vel_old[a] = p.vel[a]; p.w_old[a] = p.w[a];
            p.f_old[a] = p.f[a]; p.f[a] = 0; p.M[a] = 0;
        }
    }
    ibm_macro_all(s);
    std::fill(s.nodes.fx.begin(), s.nodes.fx.end(), 0.0);   // gpuResetNodesForces
    std::fill(s.nodes.fy.begin(), s.nodes.fy.end(), 0.0);
    std::fill(s.nodes.fz.begin(), s.nodes.fz.end(), 0.0);
    std::fill(s.nodes.dfx.begin(), s.nodes.dfx.end(), 0.0);
    std::fill(s.nodes.dfy.begin(), s.nodes.dfy.end(), 0.0);
    std::fill(s.nodes.dfz.begin(), s.nodes.dfz.end(), 0.0);
    const ContactConst K = contact_constants(s.ib);
    const int np = (int)s.parts.size();
    // gpuParticlesCollisionHandler ibmCollision.cu:2381-2448, thread order:
    // pairs (column < row) then walls; each particle's slots are touched only
    // by its own pairs
    for (int row = 1; row < np; ++row)
        for (int col = 0; col < row; ++col) {
            if (!s.parts[col].movable && !s.parts[row].movable) continue;
            sphere_sphere(s, col, row, step, K);
        }
    for (int c = 0; c < np; ++c)
        if (s.parts[c].movable) sphere_walls(s, s.parts[c], step, K);
    for (OPart& p : s.parts) update_center(s, p);
    for (int it = 0; it < s.ib.max_iterations; ++it) {
        interp_spread(s);
        for (OPart& p : s.parts) update_center(s, p);
        // gpuEulerSumIBMAuxsReset (particleEulerNodesUpdate.cu:287-330)
        for (size_t n = 0; n < fl.N; ++n)
            for (int a = 0; a < 3; ++a) {
                s.mu[a][n] += s.vaux[a][n];
                fl.fibm[a][n] += s.faux[a][n];
                s.vaux[a][n] = 0; s.faux[a][n] = 0;
            }
    }
    move(s);
}

}  // namespace

extern "C" {

struct oracle_ibm;

oracle_ibm* oracle_ibm_create(const vlbm_config* cfg, const uint32_t* map, const vlbm_ibm_config* ib,
                              const vlbm_sphere* sp, int n) {
    OIbm* s = new OIbm();
    s->fluid = reinterpret_cast<OSim*>(oracle_create(cfg, map));
    s->ib = *ib;
    const size_t N = s->fluid->N;
    s->mrho.assign(N, 0.0);
    for (int a = 0; a < 3; ++a) { s->mu[a].assign(N, 0.0); s->faux[a].assign(N, 0.0); s->vaux[a].assign(N, 0.0); }
    for (int k = 0; k < n; ++k) {
        OPart p;
        std::memset(&p, 0, sizeof(p));
        const double r = sp[k].diameter / 2.0;
        p.radius = r;
        p.volume = r * r * r * 4 * M_PI / 3;
        p.S = 4.0 * M_PI * r * r;
        p.density = sp[k].density;
        const double c[3] = {sp[k].cx, sp[k].cy, sp[k].cz}, v[3] = {sp[k].vx, sp[k].vy, sp[k].vz},
                     w[3] = {sp[k].wx, sp[k].wy, sp[k].wz};
        for (int a = 0; a < 3; ++a) {
            p.pos[a] = p.pos_old[a] = c[a];
            p.vel[a] = p.vel_old[a] = v[a];
            p.w[a] = p.w_avg[a] = p.w_old[a] = w[a];
        }
        const double Iv = 2.0 * p.volume * p.density * r * r / 5.0;  // particle.cpp:745-751
        p.I[0] = p.I[1] = p.I[2] = Iv;
        p.movable = sp[k].movable;
        for (int i = 0; i < MAX_SLOTS; ++i) { p.partner[i] = -1; p.last[i] = -1; }
        std::vector<double> px, py, pz, pS;
        int nn = sphere_mesh(sp[k].diameter, ib->mesh_scale, ib->breugem, px, py, pz, pS);
        for (int j = 0; j < nn; ++j) {
            s->nodes.x.push_back(px[j] + c[0]);
            s->nodes.y.push_back(py[j] + c[1]);
            s->nodes.z.push_back(pz[j] + c[2]);
            s->nodes.S.push_back(pS[j]);
            s->nodes.pidx.push_back(k);
        }
        s->parts.push_back(p);
    }
    const size_t nn = s->nodes.x.size();
    for (auto* v : {&s->nodes.fx, &s->nodes.fy, &s->nodes.fz, &s->nodes.dfx, &s->nodes.dfy, &s->nodes.dfz})
        v->assign(nn, 0.0);
    return reinterpret_cast<oracle_ibm*>(s);
}

void oracle_ibm_destroy(oracle_ibm* h) {
    OIbm* s = reinterpret_cast<OIbm*>(h);
    oracle_destroy(reinterpret_cast<oracle_sim*>(s->fluid));
    delete s;
}

// One reference loop iteration per step: fluid (collision reads and resets the
// IBM force field) then immersedBoundaryMethod (main.cu:300-394).
void oracle_ibm_step(oracle_ibm* h, int nsteps) {
    OIbm* s = reinterpret_cast<OIbm*>(h);
    for (int k = 0; k < nsteps; ++k) {
        const int step = (int)s->fluid->step;
        oracle_step(reinterpret_cast<oracle_sim*>(s->fluid), 1);
        ibm_substep(*s, step);
    }
}

// macr after the IBM step: rho, u of gpuUpdateMacrIBM plus the velocity corrections.
void oracle_ibm_macro(oracle_ibm* h, double* rho, double* ux, double* uy, double* uz) {
    OIbm* s = reinterpret_cast<OIbm*>(h);
    const size_t N = s->fluid->N;
    for (size_t n = 0; n < N; ++n) {
        if (rho) rho[n] = s->mrho[n];
        if (ux) ux[n] = s->mu[0][n];
        if (uy) uy[n] = s->mu[1][n];
        if (uz) uz[n] = s->mu[2][n];
    }
}

// 24 doubles per particle: pos, vel, w, f, M, w_avg, I[6]
int oracle_ibm_particles(oracle_ibm* h, double* out, int n) {
    OIbm* s = reinterpret_cast<OIbm*>(h);
    int np = (int)s->parts.size();
    for (int k = 0; k < np && k < n; ++k) {
        const OPart& p = s->parts[k];
        double* o = out + 24 * k;
        for (int a = 0; a < 3; ++a) {
            o[a] = p.pos[a]; o[3 + a] = p.vel[a]; o[6 + a] = p.w[a]; o[9 + a] = p.f[a];
            o[12 + a] = p.M[a]; o[15 + a] = p.w_avg[a];
        }
        for (int a = 0; a < 6; ++a) o[18 + a] = p.I[a];
    }
    return np;
}

// node positions [3][n]
int oracle_ibm_nodes(oracle_ibm* h, double* out, int n) {
    OIbm* s = reinterpret_cast<OIbm*>(h);
    int nn = (int)s->nodes.x.size();
    if (out && n >= nn)
        for (int k = 0; k < nn; ++k) { out[k] = s->nodes.x[k]; out[nn + k] = s->nodes.y[k]; out[2 * nn + k] = s->nodes.z[k]; }
    return nn;
}

// Sphere mesh relative to the centre: xyz [3][n], S [n]; returns the node count.
int oracle_sphere_mesh(double diameter, double mesh_scale, double* xyz, double* S, int max) {
    std::vector<double> px, py, pz, pS;
    int n = sphere_mesh(diameter, mesh_scale, 0.0, px, py, pz, pS);
    if (xyz && S && max >= n)
        for (int k = 0; k < n; ++k) { xyz[k] = px[k]; xyz[n + k] = py[k]; xyz[2 * n + k] = pz[k]; S[k] = pS[k]; }
    return n;
}

}  // extern "C"

extern "C" void* oracle_ibm_fluid(oracle_ibm* h) { return reinterpret_cast<OIbm*>(h)->fluid; }
