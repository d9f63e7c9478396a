// internal.h -- structures shared by the host side and the kernels of libvlbm.
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include "../../include/vlbm.h"

namespace vlbm {

// Node class byte (one per lattice node, read by every fused step).
enum : uint8_t {
    NODE_BULK = 0,       // plain periodic streaming, no boundary rule
    NODE_BC = 1,         // boundary node: look up bc_slot / BcRec
    NODE_UNUSED = 2,     // outside the fluid (map bit IS_USED clear): not updated
    NODE_IBM_FORCE = 0x40 // IBM force present in the dense force field
};

// Boundary schemes as evaluated by the fused kernel.
enum : uint8_t {
    K_BC_NONE = 0,        // boundary node whose rule changes nothing (convex edge, ...)
    K_BC_BOUNCE = 1,      // half-way bounce-back from own post-collision opposite
    K_BC_VEL_BOUNCE = 2,  // moving-wall bounce-back from post-streaming opposite
    K_BC_FREE_SLIP = 3,   // specular reflection from tangential neighbours
    K_BC_VEL_ZOUHE = 4,   // D3Q19 velocity Zou-He (reference formulas)
    K_BC_PRES_ZOUHE = 5,  // D3Q19 pressure Zou-He (reference formulas)
    K_BC_INTERP = 6       // interpolated bounce-back on a cylinder (coefficients per in-plane direction)
};

#ifdef __CUDACC__
#define VLBM_HD __host__ __device__
#else
#define VLBM_HD
#endif
// In-plane (D2Q9) directions of the interpolated bounce-back bits
// (nodeTypeMap.h:100-107) and the in-plane direction of a population.
constexpr int kInterpDirs[8][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
VLBM_HD constexpr int interp_dir_of(int cx, int cy) {
    return (cx == 1 && cy == 0) ? 0 : (cx == 0 && cy == 1) ? 1 : (cx == -1 && cy == 0) ? 2
         : (cx == 0 && cy == -1) ? 3 : (cx == 1 && cy == 1) ? 4 : (cx == -1 && cy == 1) ? 5
         : (cx == -1 && cy == -1) ? 6 : (cx == 1 && cy == -1) ? 7 : -1;
}

// One record per boundary node, built on the host from the reference map.
struct BcRec {
    uint8_t scheme;      // K_BC_*
    uint8_t dir;         // VLBM_NORTH ... (direction of the reference map)
    uint8_t axis;        // wall-normal axis for faces (0 x, 1 y, 2 z)
    uint8_t pad;         // interpolated bounce-back: bit d set when q > 1/2 in in-plane direction d
    uint32_t mask;       // bit i set: population i is an unknown replaced by the rule
    float uw[3];         // wall velocity (moving wall, velocity Zou-He)
    float rhow;          // wall density (pressure Zou-He)
};
static_assert(sizeof(BcRec) == 24, "BcRec layout");

struct StepParams {
    void* pop;                  // populations [Q][N] (storage type per template)
    uint8_t* cls;               // node class bytes [N]
    const int32_t* bc_slot;     // [N], valid where cls & NODE_BC
    const BcRec* bc;            // [nbc]
    const float* bc_q;          // [nbc][8][3] interpolated bounce-back coefficients per in-plane direction
    const float* side_prev;     // post-collision of boundary nodes, previous step [Q][nbc]
    float* side_next;           // same, this step
    float* omega;               // Power-Law state: apparent viscosity eta of the last step [N]
    float* fibm;                // IBM force [3][N] (nullptr without spheres)
    unsigned int* err;          // device error word (bit 0: bad density)
    int nx, ny, nz;
    long long N;
    int nbc;
    int pairH;                  // z-paired population layout: NZ/2, or 0 for the natural layout
    int pairBlk;                // z-paired layout stored in blocks of 32 pair-nodes (NX % 32 == 0)
    // pair step: the pair-nodes that hold a boundary or unused node (run by
    // k_step2; the bulk kernel leaves them)
    const int32_t* special_pairs;
    int n_special;
    int apply_bc;               // 0 on the first step after (re)initialisation
    float omega_newt;           // 1/tau
    float fx, fy, fz;           // body force
    float omega_p, yield;       // Bingham
    float n_index, k_cons, gamma0;  // Power-Law
    float scale, inv_scale, rho0;   // deviation storage
    unsigned* ctr;                  // [2] step counter by AA parity (seeds the stochastic rounding)
};

struct MacroParams {
    StepParams s;
    float *rho, *ux, *uy, *uz, *omega_out;
    const float* fibm_const;    // IBM force to use in the half-force correction (may be null)
};

// Host-side analysis of a reference node map.
// Boundary slots in increasing node order: every listed node has class
// NODE_BC and slot index = its position; all other nodes are bulk.
struct BcTables {
    std::vector<BcRec> recs;         // [nbc]
    std::vector<int32_t> bc_nodes;   // [nbc] node index of each slot
    std::vector<float> q8;           // [nbc][8][3] interpolated bounce-back coefficients (empty without)
    std::vector<int32_t> unused_nodes;   // nodes whose map word has IS_USED clear
};

vlbm_status build_bc_tables(const vlbm_config& cfg, const uint32_t* map, size_t n, BcTables& out,
                            std::string& err);
// The same tables for a named builder, without a node map (faces only).
vlbm_status build_bc_tables_builder(const vlbm_config& cfg, int builder, BcTables& out, std::string& err);
bool builder_word(int builder, int x, int y, int z, int nx, int ny, int nz, uint32_t& w,
                  double outer_radius = 0.0, double inner_radius = 0.0);

// Role of population i at a bounce-back node with direction dir:
// 0 known, 1 replaced, 2 kept with its streamed value ("dead" population).
int bb_role(int dir, int i);

void set_last_error(const std::string& msg);
std::string step_field(uint32_t step);      // getVarFilename's step digits (capi.cu)
void mkdir_p(const std::string& dir);       // folderSetup's mkdir -p (capi.cu)

}  // namespace vlbm
