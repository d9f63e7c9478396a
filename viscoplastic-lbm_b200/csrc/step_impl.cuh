// step_impl.cuh -- the fused lattice-Boltzmann time step for sm_100a.
//
// One kernel per step does what the reference splits into four launches
// (gpuMacrCollisionStream lbm.cu:4-504, gpuPopulationsTransfer lbm.cu:601-657,
// gpuApplyBC lbm.cu:580-598 and the AB pointer swap populations.h:63-70):
//
//  * populations live in ONE array [Q][N] (SoA planes, x fastest) updated in
//    place with the AA access pattern: even steps read slot i of the node and
//    write the post-collision value of i into slot opp(i) of the same node;
//    odd steps read the value streamed towards the node from slot opp(i) of the
//    upstream neighbour and write into slot i of the downstream neighbour.
//    Every slot is read and written by exactly one thread, so no barrier is
//    needed and half the reference's population memory is used.
//  * streaming is fully periodic (index wrap, which is what the reference's
//    ghost-plane transfer amounts to on one GPU); boundary rules are applied
//    when a boundary node READS its populations, from the streamed values and
//    from a small double-buffered side store holding the post-collision
//    populations of boundary nodes from the previous step (the reference keeps
//    those in `pop` at nodes with SAVE_POST_COL, lbm.cu:463-470).  This
//    reproduces the reference's semantics exactly, including the populations it
//    leaves with their wrapped values at concave edges ("dead pops") and the
//    moving-wall rule that sums the wrapped unknowns into rho_w.
//  * collision (BGK or regularized), Guo forcing and the Bingham / Power-Law
//    relaxation are computed in FP32 registers; storage is FP32 or FP16/BF16
//    deviations (f_i - w_i*rho0)*scale.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include "internal.h"
#include "lattice.cuh"
#include "pair_math.cuh"

namespace vlbm {

// ------------------------------------------------------------- storage --
// Half-precision stores round stochastically: a deviation is rounded up in
// magnitude with probability equal to the dropped fraction, so the stored
// value is exact on average.  With round-to-nearest, a slow body-force-driven
// flow stalls: the per-step change of a population (about 3 w c.F, ~1e-6 for
// F = 5e-6) is below half an FP16 ulp of its deviation (~1e-2 x 2^-11) and is
// rounded away every step.  The random bits come from a per-thread linear
// congruential stream seeded by a hash of (node, step), so a run is
// reproducible and independent of the launch it runs in.
struct Rng {
    unsigned x;
    __device__ __forceinline__ Rng(unsigned n, unsigned seed) {
        unsigned h = n * 0x9E3779B1u + seed * 0x85EBCA77u + 0x165667B1u;
        h ^= h >> 16;
        h *= 0x7FEB352Du;
        h ^= h >> 15;
        h *= 0x846CA68Bu;
        h ^= h >> 16;
        x = h;
    }
    __device__ __forceinline__ unsigned next() { x = x * 1664525u + 1013904223u; return x; }
};

// float -> half, rounding toward zero after adding 13 random bits below the
// kept mantissa (stochastic rounding of normal values).
__device__ __forceinline__ __half half_sr(float v, unsigned r) {
    return __float2half_rz(__uint_as_float(__float_as_uint(v) + (r >> 19)));
}
// float -> bfloat16, the same with 16 random bits.
__device__ __forceinline__ __nv_bfloat16 bf16_sr(float v, unsigned r) {
    return __ushort_as_bfloat16((unsigned short)((__float_as_uint(v) + (r >> 16)) >> 16));
}

// The kernels work on deviations g_i = f_i - w_i rho0 from the rest
// equilibrium: moments are sums of small numbers and the collision produces the
// post-collision deviation directly.  Summing full populations instead (values
// w_i + small, whose trailing bits are those of w_i on every node) makes the
// FP32 rounding of rho systematic: with half-precision storage that created
// ~1e-7 of mass per node and step.  Every storage keeps deviations: FP32 g_i,
// half precision g_i * scale.  Storing the full FP32 population (the
// reference's state, ~w_i) would round the increments a slow flow gets every
// step (~1e-7 against an ulp of ~4e-9 at f ~ 0.05) on every store; the
// rounding bias built up to a -0.5 % velocity error in a 64x32x32 BGK
// Poiseuille channel at u ~ 1e-3 (the reference's own FP32 build: +0.2 %;
// FP64: 1e-4).  A deviation (~1e-4 there) keeps those increments to FP32
// precision.  Entry points that take or return populations convert.
template <int ST> struct Store;
template <> struct Store<VLBM_STORE_F32> {
    using T = float;
    static __device__ __forceinline__ float ld(const T* p, float, const StepParams&) { return *p; }
    static __device__ __forceinline__ void st(T* p, float g, float, const StepParams&, Rng&) { *p = g; }
    // a full population (initial state, user state)
    static __device__ __forceinline__ void st_abs(T* p, float v, float w, const StepParams& s) { *p = v - w * s.rho0; }
};
template <> struct Store<VLBM_STORE_F16> {
    using T = __half;
    static __device__ __forceinline__ float ld(const T* p, float, const StepParams& s) {
        return __half2float(*p) * s.inv_scale;
    }
    static __device__ __forceinline__ void st(T* p, float g, float, const StepParams& s, Rng& r) {
        *p = half_sr(g * s.scale, r.next());
    }
    static __device__ __forceinline__ void st_abs(T* p, float v, float w, const StepParams& s) {
        *p = __float2half_rn((v - w * s.rho0) * s.scale);
    }
};
template <> struct Store<VLBM_STORE_BF16> {
    using T = __nv_bfloat16;
    static __device__ __forceinline__ float ld(const T* p, float, const StepParams& s) {
        return __bfloat162float(*p) * s.inv_scale;
    }
    static __device__ __forceinline__ void st(T* p, float g, float, const StepParams& s, Rng& r) {
        *p = bf16_sr(g * s.scale, r.next());
    }
    static __device__ __forceinline__ void st_abs(T* p, float v, float w, const StepParams& s) {
        *p = __float2bfloat16_rn((v - w * s.rho0) * s.scale);
    }
};

// Reflection of population i across the plane normal to `axis`.
VLBM_HD constexpr int lat_refl(int i, int axis) {
    int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
    if (axis == 0) cx = -cx;
    else if (axis == 1) cy = -cy;
    else cz = -cz;
    for (int j = 0; j < 27; ++j)
        if (lat_cx(j) == cx && lat_cy(j) == cy && lat_cz(j) == cz) return j;
    return i;
}

// Periodic neighbour offsets of one node (in nodes).
struct Nbr {
    int xm, xp, ym, yp, zm, zp;
    __device__ __forceinline__ void init(int x, int y, int z, int nx, int ny, int nz) {
        const int nxy = nx * ny;
        xm = (x == 0) ? nx - 1 : -1;
        xp = (x == nx - 1) ? -(nx - 1) : 1;
        ym = (y == 0) ? (ny - 1) * nx : -nx;
        yp = (y == ny - 1) ? -(ny - 1) * nx : nx;
        zm = (z == 0) ? (nz - 1) * nxy : -nxy;
        zp = (z == nz - 1) ? -(nz - 1) * nxy : nxy;
    }
    // Hide the offsets from common-subexpression elimination: the store loop
    // then recomputes its sums (a few integer adds) instead of keeping the
    // load loop's 18 sums live across the collision.
    __device__ __forceinline__ void launder() {
        asm volatile("" : "+r"(xm), "+r"(xp), "+r"(ym), "+r"(yp), "+r"(zm), "+r"(zp));
    }
    // offset of the node at (x+dx, y+dy, z+dz), dx,dy,dz in {-1,0,1}
    __device__ __forceinline__ int off(int dx, int dy, int dz) const {
        return (dx > 0 ? xp : (dx < 0 ? xm : 0)) + (dy > 0 ? yp : (dy < 0 ? ym : 0)) +
               (dz > 0 ? zp : (dz < 0 ? zm : 0));
    }
};

// ------------------------------------------------- D3Q19 Zou-He (reference) --
// Velocity Zou-He, D3Q19_VelZouHe.cu:27-172, per face as the reference writes it.
__device__ __forceinline__ void zouhe_vel19(float (&f)[19], int dir, float ux, float uy, float uz) {
    float g4 = f[4], g8 = f[8], g13 = f[13], g12 = f[12], g18 = f[18];
    switch (dir) {
    case VLBM_NORTH: {
        float rw = (1.f / (1.f + uy)) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                         2.f * (f[3] + f[7] + f[14] + f[11] + f[17]));
        float nyx = 0.5f * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10])) - ux * rw / 3.f;
        float nyz = 0.5f * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10])) - uz * rw / 3.f;
        g4 = f[3] + rw * (-uy) / 3.f;
        g8 = f[7] + rw * (-uy - ux) / 6.f + nyx;
        g13 = f[14] + rw * (-uy + ux) / 6.f - nyx;
        g12 = f[11] + rw * (-uy - uz) / 6.f + nyz;
        g18 = f[17] + rw * (-uy + uz) / 6.f - nyz;
        f[4] = g4; f[8] = g8; f[13] = g13; f[12] = g12; f[18] = g18;
        break; }
    case VLBM_SOUTH: {
        float rw = (1.f / (1.f - uy)) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                         2.f * (f[4] + f[13] + f[8] + f[18] + f[12]));
        float nyx = 0.5f * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10])) - ux * rw / 3.f;
        float nyz = 0.5f * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10])) - uz * rw / 3.f;
        float a3 = f[4] + rw * uy / 3.f, a7 = f[8] + rw * (uy + ux) / 6.f - nyx,
              a14 = f[13] + rw * (uy - ux) / 6.f + nyx, a11 = f[12] + rw * (uy + uz) / 6.f - nyz,
              a17 = f[18] + rw * (uy - uz) / 6.f + nyz;
        f[3] = a3; f[7] = a7; f[14] = a14; f[11] = a11; f[17] = a17;
        break; }
    case VLBM_WEST: {
        float rw = (1.f / (1.f - ux)) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                         2.f * (f[2] + f[14] + f[8] + f[16] + f[10]));
        float nxy = 0.5f * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12])) - uy * rw / 3.f;
        float nxz = 0.5f * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12])) - uz * rw / 3.f;
        float a1 = f[2] + rw * ux / 3.f, a13 = f[14] + rw * (ux - uy) / 6.f + nxy,
              a7 = f[8] + rw * (ux + uy) / 6.f - nxy, a9 = f[10] + rw * (ux + uz) / 6.f - nxz,
              a15 = f[16] + rw * (ux - uy) / 6.f + nxz;
        f[1] = a1; f[13] = a13; f[7] = a7; f[9] = a9; f[15] = a15;
        break; }
    case VLBM_EAST: {
        float rw = (1.f / (1.f + ux)) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                         2.f * (f[2] + f[14] + f[8] + f[16] + f[10]));
        float nxy = 0.5f * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12])) - uy * rw / 3.f;
        float nxz = 0.5f * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12])) - uz * rw / 3.f;
        float a2 = f[2] + rw * ux / 3.f, a14 = f[14] + rw * (ux - uy) / 6.f + nxy,
              a8 = f[8] + rw * (ux + uy) / 6.f - nxy, a10 = f[10] + rw * (ux + uz) / 6.f - nxz,
              a16 = f[16] + rw * (ux - uy) / 6.f + nxz;
        f[2] = a2; f[14] = a14; f[8] = a8; f[10] = a10; f[16] = a16;
        break; }
    case VLBM_FRONT: {
        float rw = (1.f / (1.f + uz)) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                         2.f * (f[5] + f[9] + f[16] + f[11] + f[18]));
        float nzx = 0.5f * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8])) - rw * ux / 3.f;
        float nzy = 0.5f * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8])) - rw * uy / 3.f;
        float a6 = f[5] + rw * (-uz) / 3.f, a15 = f[16] + rw * (-uz + ux) / 6.f - nzx,
              a10 = f[9] + rw * (-uz - ux) / 6.f + nzx, a17 = f[18] + rw * (-uz + uy) / 6.f - nzy,
              a12 = f[11] + rw * (-uz - uy) / 6.f + nzy;
        f[6] = a6; f[15] = a15; f[10] = a10; f[17] = a17; f[12] = a12;
        break; }
    case VLBM_BACK: {
        float rw = (1.f / (1.f + uz)) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                         2.f * (f[6] + f[15] + f[10] + f[17] + f[12]));
        float nzx = 0.5f * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8])) - rw * ux / 3.f;
        float nzy = 0.5f * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8])) - rw * uy / 3.f;
        float a5 = f[6] + rw * uz / 3.f, a9 = f[10] + rw * (uz + ux) / 6.f - nzx,
              a16 = f[15] + rw * (uz - ux) / 6.f + nzx, a11 = f[12] + rw * (uz + ux) / 6.f - nzy,
              a18 = f[17] + rw * (uz - ux) / 6.f + nzy;
        f[5] = a5; f[9] = a9; f[16] = a16; f[11] = a11; f[18] = a18;
        break; }
    default: break;
    }
}

// Pressure Zou-He, D3Q19_PresZouHe.cu:27-176, per face as the reference writes it.
__device__ __forceinline__ void zouhe_pres19(float (&f)[19], int dir, float rw) {
    switch (dir) {
    case VLBM_NORTH: {
        float uy = -1.f + (1.f / rw) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                        2.f * (f[3] + f[7] + f[14] + f[11] + f[17]));
        float nyx = 0.5f * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10]));
        float nyz = 0.5f * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10]));
        float a4 = f[3] + rw * (-uy) / 3.f, a8 = f[7] + rw * (-uy) / 6.f + nyx,
              a13 = f[14] + rw * (-uy) / 6.f - nyx, a12 = f[11] + rw * (-uy) / 6.f + nyz,
              a18 = f[17] + rw * (-uy) / 6.f - nyz;
        f[4] = a4; f[8] = a8; f[13] = a13; f[12] = a12; f[18] = a18;
        break; }
    case VLBM_SOUTH: {
        float uy = 1.f - (1.f / rw) * (f[1] + f[2] + f[5] + f[6] + f[9] + f[15] + f[16] + f[10] + f[0] +
                                       2.f * (f[4] + f[13] + f[8] + f[18] + f[12]));
        float nyx = 0.5f * (f[1] + f[9] + f[15] - (f[2] + f[16] + f[10]));
        float nyz = 0.5f * (f[5] + f[9] + f[16] - (f[6] + f[15] + f[10]));
        float a3 = f[4] + rw * uy / 3.f, a7 = f[8] + rw * uy / 6.f - nyx, a14 = f[13] + rw * uy / 6.f + nyx,
              a11 = f[12] + rw * uy / 6.f - nyz, a17 = f[18] + rw * uy / 6.f + nyz;
        f[3] = a3; f[7] = a7; f[14] = a14; f[11] = a11; f[17] = a17;
        break; }
    case VLBM_WEST: {
        float ux = 1.f - (1.f / rw) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                       2.f * (f[2] + f[14] + f[8] + f[16] + f[10]));
        float nxy = 0.5f * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12]));
        float nxz = 0.5f * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12]));
        float a1 = f[2] + rw * ux / 3.f, a13 = f[14] + rw * ux / 6.f + nxy, a7 = f[8] + rw * ux / 6.f - nxy,
              a9 = f[10] + rw * ux / 6.f - nxz, a15 = f[16] + rw * ux / 6.f + nxz;
        f[1] = a1; f[13] = a13; f[7] = a7; f[9] = a9; f[15] = a15;
        break; }
    case VLBM_EAST: {
        float ux = -1.f + (1.f / rw) * (f[3] + f[4] + f[5] + f[6] + f[11] + f[17] + f[18] + f[12] + f[0] +
                                        2.f * (f[2] + f[14] + f[8] + f[16] + f[10]));
        float nxy = 0.5f * (f[3] + f[11] + f[17] - (f[4] + f[18] + f[12]));
        float nxz = 0.5f * (f[5] + f[18] + f[11] - (f[6] + f[17] + f[12]));
        float a2 = f[2] + rw * ux / 3.f, a14 = f[14] + rw * ux / 6.f + nxy, a8 = f[8] + rw * ux / 6.f - nxy,
              a10 = f[10] + rw * ux / 6.f - nxz, a16 = f[16] + rw * ux / 6.f + nxz;
        f[2] = a2; f[14] = a14; f[8] = a8; f[10] = a10; f[16] = a16;
        break; }
    case VLBM_FRONT: {
        float uz = -1.f + (1.f / rw) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                        2.f * (f[5] + f[9] + f[16] + f[11] + f[18]));
        float nzx = 0.5f * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8]));
        float nzy = 0.5f * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8]));
        float a6 = f[5] + rw * (-uz) / 3.f, a15 = f[16] + rw * (-uz) / 6.f - nzx,
              a10 = f[9] + rw * (-uz) / 6.f + nzx, a17 = f[18] + rw * (-uz) / 6.f - nzy,
              a12 = f[11] + rw * (-uz) / 6.f + nzy;
        f[6] = a6; f[15] = a15; f[10] = a10; f[17] = a17; f[12] = a12;
        break; }
    case VLBM_BACK: {
        float uz = 1.f - (1.f / rw) * (f[1] + f[2] + f[3] + f[4] + f[7] + f[14] + f[8] + f[13] + f[0] +
                                       2.f * (f[6] + f[10] + f[12] + f[15] + f[17]));
        float nzx = 0.5f * (f[1] + f[7] + f[13] - (f[2] + f[14] + f[8]));
        float nzy = 0.5f * (f[3] + f[7] + f[14] - (f[4] + f[13] + f[8]));
        float a5 = f[6] + rw * uz / 3.f, a9 = f[10] + rw * uz / 6.f - nzx, a16 = f[15] + rw * uz / 6.f + nzx,
              a11 = f[12] + rw * uz / 6.f - nzy, a18 = f[17] + rw * uz / 6.f + nzy;
        f[5] = a5; f[9] = a9; f[16] = a16; f[11] = a11; f[18] = a18;
        break; }
    default: break;
    }
}

// ----------------------------------------------------- boundary at gather --
template <int Q>
__device__ __forceinline__ void apply_bc(float (&f)[Q], const StepParams& p, const float* __restrict__ side_prev,
                                      int slot, int x, int y, int z, const Nbr& nb, unsigned n) {
    const BcRec r = p.bc[slot];
    const size_t nbc = (size_t)p.nbc;
    switch (r.scheme) {
    case K_BC_BOUNCE:
        // bounceBack.cu:26-498: unknown <- own post-collision opposite
#pragma unroll
        for (int i = 1; i < Q; ++i)
            if ((r.mask >> i) & 1u) f[i] = side_prev[(size_t)lat_opp(i) * nbc + slot];
        break;
    case K_BC_VEL_BOUNCE: {
        // D3Q19_VelBounceBack.cu:31-43: rho_w over all streamed populations
        // (including the wrapped unknowns), unknown <- streamed opposite
        // - 6 rho_w w_i (c_opp . u_w).  The opposite of an unknown at a face is
        // always a known population, so the update can run in place.  On
        // deviations: rho_w = rho0 + sum g, and w_opp = w_i cancels.
        float rw = 0.f;
#pragma unroll
        for (int i = 0; i < Q; ++i) rw += f[i];
        rw += p.rho0;
#pragma unroll
        for (int i = 1; i < Q; ++i)
            if ((r.mask >> i) & 1u) {
                const int o = lat_opp(i);
                const float cu = lat_cx(o) * r.uw[0] + lat_cy(o) * r.uw[1] + lat_cz(o) * r.uw[2];
                f[i] = f[o] - 6.f * rw * Lattice<Q>::w(i) * cu;
            }
        break;
    }
    case K_BC_FREE_SLIP:
        // freeSlip.cu:26-167: reflected post-collision population of the node one
        // tangential step upstream
#pragma unroll
        for (int i = 1; i < Q; ++i)
            if ((r.mask >> i) & 1u) {
                const int a = r.axis;
                const int j = a == 0 ? lat_refl(i, 0) : (a == 1 ? lat_refl(i, 1) : lat_refl(i, 2));
                const int tx = a == 0 ? 0 : lat_cx(i), ty = a == 1 ? 0 : lat_cy(i), tz = a == 2 ? 0 : lat_cz(i);
                const unsigned src = n + nb.off(-tx, -ty, -tz);
                const int sslot = p.bc_slot[src];
                f[i] = side_prev[(size_t)j * nbc + sslot];
            }
        break;
    case K_BC_VEL_ZOUHE:
    case K_BC_PRES_ZOUHE:
        if constexpr (Q == 19) {   // the reference's formulas act on full populations
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] += Lattice<Q>::w(i) * p.rho0;
            if (r.scheme == K_BC_VEL_ZOUHE) zouhe_vel19(f, r.dir, r.uw[0], r.uw[1], r.uw[2]);
            else zouhe_pres19(f, r.dir, r.rhow);
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] -= Lattice<Q>::w(i) * p.rho0;
        }
        break;
    case K_BC_INTERP: {
        // interpolatedBounceBack.cu:6-372.  For an unknown population i whose
        // link crosses the wall at normalised distance q from the node:
        //   q > 1/2:  f_i = f*_o / (2q) + (q - 1/2)/q f*_i + 3 w_i (c_i . u_w) / q
        //   q <= 1/2: f_i = 2q f*_o + (1 - 2q) f_o + 6 w_i (c_i . u_w)
        // with o the opposite, f* this node's post-collision values (side
        // store) and f_o the streamed opposite, i.e. the post-collision value
        // of the node one link inward (the reference reads it from its
        // post-collision array at x + c_i).  The host stores per in-plane
        // direction d the coefficients (A, B, K), and in r.pad the directions
        // with q > 1/2, so the rule is two FMAs without a division.  The rules
        // are affine with weights summing to one and w_o = w_i, so they hold for
        // deviations as written.
        const float* cf = p.bc_q + (size_t)slot * 24;
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            const int d = interp_dir_of(lat_cx(i), lat_cy(i));
            if (d < 0 || !((r.mask >> i) & 1u)) continue;
            const int o = lat_opp(i);
            const float so = side_prev[(size_t)o * nbc + slot];
            const float other = ((r.pad >> d) & 1u) ? side_prev[(size_t)i * nbc + slot] : f[o];
            const float cu = lat_cx(i) * r.uw[0] + lat_cy(i) * r.uw[1] + lat_cz(i) * r.uw[2];
            f[i] = cf[3 * d] * so + cf[3 * d + 1] * other + cf[3 * d + 2] * (Lattice<Q>::w(i) * cu);
        }
        break;
    }
    default: break;
    }
    (void)x; (void)y; (void)z;
}
template <int Q>
__device__ __forceinline__ void apply_bc(float (&f)[Q], const StepParams& p, int slot, int x, int y, int z,
                                      const Nbr& nb, unsigned n) {
    apply_bc<Q>(f, p, p.side_prev, slot, x, y, z, nb, n);
}

// Element index of population i of node (x, y, z) in the z-paired layouts:
// nodes z and z+H (H = NZ/2) of one (x, y) column are neighbours in memory
// (lane 0 / 1 of pair-node m).  Plain pairs: Q planes of N/2 pairs.  Blocked
// pairs (NX % 32 == 0): blocks of 32 consecutive pair-nodes, each holding
// all Q populations of its nodes, [m / 32][Q][32][2].
// layout_elem: the same for any layout, H = 0 being the natural [Q][N] one.
template <int Q>
__device__ __forceinline__ size_t layout_elem(int i, int x, int y, int z, int nx, int ny, long long N, int H,
                                              int blk) {
    if (H == 0) return (size_t)i * (size_t)N + (((size_t)z * ny + y) * nx + x);
    const int lane = z >= H ? 1 : 0;
    const int zp = z - lane * H;
    const size_t m = ((size_t)zp * ny + y) * nx + x;
    if (blk) return (((((m >> 5) * Q + (size_t)i) << 5) | (m & 31u)) << 1) | (size_t)lane;
    return (size_t)i * (size_t)N + ((m << 1) | (size_t)lane);
}
template <int Q>
__device__ __forceinline__ size_t pair_elem(const StepParams& p, int i, int x, int y, int z) {
    return layout_elem<Q>(i, x, y, z, p.nx, p.ny, p.N, p.pairH, p.pairBlk);
}

// The population array moved from one layout (sH, sB) to another (dH, dB),
// value for value: the stored bits are copied, so the state is unchanged.
template <int Q, int ST>
__global__ void __launch_bounds__(256) k_relayout(const void* src, void* dst, int nx, int ny, long long N, int sH,
                                                  int sB, int dH, int dB) {
    using T = typename Store<ST>::T;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int x = (int)(n % nx);
    const long long t = n / nx;
    const int y = (int)(t % ny), z = (int)(t / ny);
    const T* S = static_cast<const T*>(src);
    T* D = static_cast<T*>(dst);
#pragma unroll
    for (int i = 0; i < Q; ++i)
        D[layout_elem<Q>(i, x, y, z, nx, ny, N, dH, dB)] = S[layout_elem<Q>(i, x, y, z, nx, ny, N, sH, sB)];
}

// z-slab halo message: the stored values of the populations with c_z == dz of
// plane z, [k][y][x] with k counting those populations in lattice order,
// copied out of (pack) or into (unpack) the population array of any layout.
template <int Q>
constexpr int halo_pops() { return Q == 19 ? 5 : 9; }
struct HaloMsg {
    void* buf;
    int z, dz;
};
// Two messages per launch (a slab's two faces); message m covers threads
// [m * M, (m + 1) * M), M = halo_pops * nx * ny.
template <int Q, int ST>
__global__ void __launch_bounds__(256) k_halo(void* pop, HaloMsg m0, HaloMsg m1, int nx, int ny, long long N,
                                              int H, int blk, int unpack) {
    using T = typename Store<ST>::T;
    const long long plane = (long long)nx * ny;
    const long long M = halo_pops<Q>() * plane;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * M) return;
    const bool second = t >= M;
    if (second) t -= M;
    const HaloMsg& m = second ? m1 : m0;
    if (!m.buf) return;
    const int z = m.z, dz = m.dz;
    const int k = (int)(t / plane);
    const int r = (int)(t - (long long)k * plane);
    int i = 0;
#pragma unroll
    for (int j = 1, c = 0; j < Q; ++j)
        if (lat_cz(j) == dz) {
            if (c == k) i = j;
            ++c;
        }
    T* P = static_cast<T*>(pop);
    T* B = static_cast<T*>(m.buf);
    const size_t e = layout_elem<Q>(i, r % nx, r / nx, z, nx, ny, N, H, blk);
    if (unpack) P[e] = B[t];
    else B[t] = P[e];
}
__device__ __forceinline__ int wrap1(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// Gather f_i(x, t) of node n (after boundary rules).  Returns the side-store
// slot of a boundary node, -1 for bulk nodes.
template <int Q, int ST, bool ODD, bool PAIRED = false>
__device__ __forceinline__ int gather(const StepParams& p, const float* side_prev, int use_bc, unsigned n,
                                      const Nbr& nb, int x, int y, int z, float (&f)[Q], uint8_t& cls) {
    using S = Store<ST>;
    using T = typename S::T;
    const size_t N = (size_t)p.N;
    if (PAIRED) {
        const T* A = static_cast<const T*>(p.pop);
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (!ODD) {
                f[i] = S::ld(A + pair_elem<Q>(p, i, x, y, z), Lattice<Q>::w(i), p);
            } else {
                const size_t src = pair_elem<Q>(p, lat_opp(i), wrap1(x - lat_cx(i), p.nx), wrap1(y - lat_cy(i), p.ny),
                                                wrap1(z - lat_cz(i), p.nz));
                f[i] = S::ld(A + src, Lattice<Q>::w(i), p);
            }
        }
        cls = p.cls[n];
        int slot = -1;
        if (cls & NODE_BC) {
            slot = p.bc_slot[n];
            if (use_bc) apply_bc<Q>(f, p, side_prev, slot, x, y, z, nb, n);
        }
        return slot;
    }
    // walk the planes with one running pointer: plane j holds population j in
    // the natural layout (even steps) and population opp(j) after an even step
    const T* plane = static_cast<const T*>(p.pop);
#pragma unroll
    for (int j = 0; j < Q; ++j, plane += N) {
        if (!ODD) {
            f[j] = S::ld(plane + n, Lattice<Q>::w(j), p);
        } else {
            const int i = lat_opp(j);
            const unsigned src = n + nb.off(-lat_cx(i), -lat_cy(i), -lat_cz(i));
            f[i] = S::ld(plane + src, Lattice<Q>::w(i), p);
        }
    }
    cls = p.cls[n];
    int slot = -1;
    if (cls & NODE_BC) {
        slot = p.bc_slot[n];
        if (use_bc) apply_bc<Q>(f, p, side_prev, slot, x, y, z, nb, n);
    }
    return slot;
}
template <int Q, int ST, bool ODD, bool PAIRED = false>
__device__ __forceinline__ int gather(const StepParams& p, unsigned n, const Nbr& nb, int x, int y, int z,
                                      float (&f)[Q], uint8_t& cls) {
    return gather<Q, ST, ODD, PAIRED>(p, p.side_prev, p.apply_bc, n, nb, x, y, z, f, cls);
}

// Moments of a node: rho, u (with half force, lbm.cu:79-111), non-equilibrium
// second moments (lbm.cu:149-190) and the stress magnitude used by the
// rheology models (lbm.cu:192-208).
struct Mom {
    float rho, drho, ux, uy, uz;
    float pxx, pyy, pzz, pxy, pxz, pyz;
};

// Moments of the deviations g_i = f_i - w_i rho0: rho = rho0 + sum g,
// rho u = sum c g + F/2, and the non-equilibrium second moments
// Pi_ab = sum c_a c_b f - rho (u_a u_b + delta_ab / 3)
//       = sum c_a c_b g - rho u_a u_b - delta_ab (rho - rho0) / 3.
template <int Q, bool NEED_PI>
__device__ __forceinline__ Mom moments(const float (&f)[Q], float fx, float fy, float fz, float rho0) {
    // Sums over opposite pairs: e = g_i + g_opp feeds the even moments (rho,
    // second moments), o = g_i - g_opp the odd ones (momentum).
    Mom m;
    float rho = f[0], jx = 0.f, jy = 0.f, jz = 0.f;
    float sxx = 0.f, syy = 0.f, szz = 0.f, sxy = 0.f, sxz = 0.f, syz = 0.f;
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
        const float e = f[i] + f[i + 1], o = f[i] - f[i + 1];
        rho += e;
        if (cx) jx += cx * o;
        if (cy) jy += cy * o;
        if (cz) jz += cz * o;
        if (NEED_PI) {
            if (cx) sxx += e;
            if (cy) syy += e;
            if (cz) szz += e;
            if (cx && cy) sxy += cx * cy * e;
            if (cx && cz) sxz += cx * cz * e;
            if (cy && cz) syz += cy * cz * e;
        }
    }
    // correctly rounded reciprocal: u = j/rho enters every equilibrium, and a
    // biased approximate reciprocal (the hardware MUFU result is within 2 ulp
    // but not unbiased) acts like a spurious force proportional to the
    // momentum, which shifts a slow channel flow by ~1e-3 over 1e4 steps
    const float drho = rho;
    rho += rho0;
    const float inv = __frcp_rn(rho);
    m.rho = rho;
    m.drho = drho;
    m.ux = (jx + 0.5f * fx) * inv;
    m.uy = (jy + 0.5f * fy) * inv;
    m.uz = (jz + 0.5f * fz) * inv;
    if (NEED_PI) {
        const float dr3 = drho * (1.f / 3.f);
        m.pxx = sxx - rho * m.ux * m.ux - dr3;
        m.pyy = syy - rho * m.uy * m.uy - dr3;
        m.pzz = szz - rho * m.uz * m.uz - dr3;
        m.pxy = sxy - rho * m.ux * m.uy;
        m.pxz = sxz - rho * m.ux * m.uz;
        m.pyz = syz - rho * m.uy * m.uz;
    } else {
        m.pxx = m.pyy = m.pzz = m.pxy = m.pxz = m.pyz = 0.f;
    }
    return m;
}

__device__ __forceinline__ float stress_aux(const Mom& m, float fx, float fy, float fz) {
    const float a = m.pxx + m.ux * fx, b = m.pyy + m.uy * fy, c = m.pzz + m.uz * fz;
    const float d = m.pxy + 0.5f * (m.ux * fy + m.uy * fx);
    const float e = m.pxz + 0.5f * (m.ux * fz + m.uz * fx);
    const float g = m.pyz + 0.5f * (m.uy * fz + m.uz * fy);
    const float q = 0.5f * (a * a + b * b + c * c + 2.f * (d * d + e * e + g * g));
    return q > 0.f ? q * rsqrtf(q) : 0.f;  // hardware reciprocal square root (<= 2 ulp)
}

// nnf.h:32-87 calcOmega.  For Power-Law the per-node state is the apparent
// viscosity eta of the previous step (the reference stores omega,
// lbm.cu:215-219); with omega_old = 1/(1/2 + 3 eta_old) the reference's
//   eta_old = (1/omega_old - 1/2)/3,  gamma_dot = (1 - omega_old/2) |S| / eta_old
// is the same number as gamma_dot = 3 |S| / (1/2 + 3 eta_old), which stays
// finite where FP32 would round omega_old to exactly 2 (eta_old -> 0) and
// needs eta_old = +inf for the reference's initial omega = 0.
template <int RHEO>
__device__ __forceinline__ float relax(const StepParams& p, float eta_old, float aux, float& eta_new) {
    if (RHEO == VLBM_BINGHAM) {
        return p.omega_p * fmaxf(0.f, 1.f - __fdividef(p.yield, aux));
    } else if (RHEO == VLBM_POWERLAW) {
        const float gd = 3.f * aux / (0.5f + 3.f * eta_old);
        // gd^(n-1): the flow indices 0.5, 1 and 1.5 take a square root, a
        // reciprocal square root (<= 2 ulp) or nothing instead of powf
        const float e = p.n_index - 1.f;
        const float pw = e == -0.5f ? rsqrtf(gd) : (e == 0.5f ? sqrtf(gd) : (e == 0.f ? 1.f : powf(gd, e)));
        eta_new = (gd <= p.gamma0) ? p.k_cons : p.k_cons * pw;
        return 1.f / (0.5f + 3.f * eta_new);
    }
    return p.omega_newt;
}

// Collision in place: f <- f*.
//  regularized (lbm.cu:263-461):
//    f*_i = w_i [ A (Q_i:Pi - c_i.F/3) + rho(1 - 1.5u^2 + 3cu + 4.5cu^2) + B(3(c_i-u).F + 9 cu cF) ]
//    A = 4.5(1-omega), B = 1-omega/2
//  BGK (collisionForceNoReg.txt): f*_i = (1-omega) f_i + omega f_eq_i + B F_i
template <int Q, int OP>
__device__ __forceinline__ void collide(float (&f)[Q], const Mom& m, float omega, float fx, float fy, float fz) {
    // Populations i (odd index) and opp(i) = i+1 have opposite velocities: they
    // share Q_i:Pi, while c.u and c.F change sign.  Each pair is evaluated as an
    // even part E and an odd part O with f*_i = w (E + O), f*_opp = w (E - O).
    const float B = 1.f - 0.5f * omega;
    const float uu = m.ux * m.ux + m.uy * m.uy + m.uz * m.uz;
    const float uF = m.ux * fx + m.uy * fy + m.uz * fz;
    if (OP == VLBM_OP_REGULARIZED) {
        const float A = 4.5f * (1.f - omega);
        const float tr = (m.pxx + m.pyy + m.pzz) * (1.f / 3.f);
        // the rest part w_i rho0 is not formed: K0 is the deviation of rho(1 - 1.5 u^2)
        const float K0 = m.drho - 1.5f * m.rho * uu - 3.f * B * uF - A * tr;
        const float alpha = 3.f * B - A * (1.f / 3.f);
        const float r3 = 3.f * m.rho, r45 = 4.5f * m.rho, b9 = 9.f * B;
        f[0] = Lattice<Q>::w(0) * K0;
        // coefficients with the weight of each velocity class folded in
        float cK[3], cA[3], cr45[3], cb9[3], cal[3], cr3[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            // representative population of the class: 1 (axis), 7 (face), 19 (body, D3Q27 only)
            const float w = Lattice<Q>::w(k == 0 ? 1 : (k == 1 ? 7 : (Q == 27 ? 19 : 1)));
            cK[k] = w * K0; cA[k] = w * A; cr45[k] = w * r45; cb9[k] = w * b9; cal[k] = w * alpha; cr3[k] = w * r3;
        }
        const float pxy2 = 2.f * m.pxy, pxz2 = 2.f * m.pxz, pyz2 = 2.f * m.pyz;
#pragma unroll
        for (int i = 1; i < Q; i += 2) {
            const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
            const int k = lat_norm1(i) - 1;   // 0 axis, 1 face diagonal, 2 body diagonal
            float S = 0.f, cu = 0.f, cF = 0.f;
            if (cx) { S += m.pxx; cu += cx * m.ux; cF += cx * fx; }
            if (cy) { S += m.pyy; cu += cy * m.uy; cF += cy * fy; }
            if (cz) { S += m.pzz; cu += cz * m.uz; cF += cz * fz; }
            if (cx && cy) S += cx * cy * pxy2;
            if (cx && cz) S += cx * cz * pxz2;
            if (cy && cz) S += cy * cz * pyz2;
            const float E = cK[k] + cA[k] * S + cu * (cr45[k] * cu + cb9[k] * cF);
            const float O = cal[k] * cF + cr3[k] * cu;
            f[i] = E + O;
            f[i + 1] = E - O;
        }
    } else {
        const float om1 = 1.f - omega;
        // on deviations: (1 - omega) w rho0 + omega w rho0 cancels against w rho0
        const float base = omega * (m.drho - 1.5f * m.rho * uu) - 3.f * B * uF;
        const float r45 = 4.5f * omega * m.rho, r3 = 3.f * omega * m.rho, b9 = 9.f * B, b3 = 3.f * B;
        f[0] = om1 * f[0] + Lattice<Q>::w(0) * base;
#pragma unroll
        for (int i = 1; i < Q; i += 2) {
            const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
            float cu = 0.f, cF = 0.f;
            if (cx) { cu += cx * m.ux; cF += cx * fx; }
            if (cy) { cu += cy * m.uy; cF += cy * fy; }
            if (cz) { cu += cz * m.uz; cF += cz * fz; }
            const float w = Lattice<Q>::w(i);
            const float E = w * (base + cu * (r45 * cu + b9 * cF));
            const float O = w * (r3 * cu + b3 * cF);
            f[i] = om1 * f[i] + (E + O);
            f[i + 1] = om1 * f[i + 1] + (E - O);
        }
    }
}

// Everything after the gather for one node: IBM force read and reset
// (lbm.cu:45-58), moments, relaxation (lbm.cu:192-222), collision, and the
// post-collision copy of boundary nodes (lbm.cu:463-470).  `eta_old` is the
// node's Power-Law state p.omega[n], loaded by the caller ahead of the gather.
template <int Q, int OP, int RHEO>
__device__ __forceinline__ void relax_and_collide(const StepParams& p, float* side_next, unsigned n, uint8_t cls,
                                                  int slot, float (&f)[Q], float eta_old) {
    float fx = p.fx, fy = p.fy, fz = p.fz;
    if (cls & NODE_IBM_FORCE) {
        const size_t N = (size_t)p.N;
        fx += p.fibm[n]; fy += p.fibm[N + n]; fz += p.fibm[2 * N + n];
        p.fibm[n] = 0.f; p.fibm[N + n] = 0.f; p.fibm[2 * N + n] = 0.f;
        p.cls[n] = cls & (uint8_t)~NODE_IBM_FORCE;
    }
    constexpr bool NEED_PI = (OP == VLBM_OP_REGULARIZED) || (RHEO != VLBM_NEWTONIAN);
    const Mom m = moments<Q, NEED_PI>(f, fx, fy, fz, p.rho0);
    if (!(m.rho > 0.f && m.rho < 1e30f) && !(cls & NODE_UNUSED)) atomicOr(p.err, 1u);
    float omega = p.omega_newt;
    if (RHEO != VLBM_NEWTONIAN) {
        const float aux = stress_aux(m, fx, fy, fz);
        float eta = 0.f;
        omega = relax<RHEO>(p, eta_old, aux, eta);
        if (RHEO == VLBM_POWERLAW) p.omega[n] = eta;  // state update, lbm.cu:215-219
    }
    collide<Q, OP>(f, m, omega, fx, fy, fz);
    if (cls & NODE_UNUSED) {   // lbm.cu:23-24: not updated; rest equilibrium stays in its slots
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = 0.f;
    }
    if (slot >= 0) {
        const size_t nbc = (size_t)p.nbc;
#pragma unroll
        for (int i = 0; i < Q; ++i) side_next[(size_t)i * nbc + slot] = f[i];
    }
}
template <int Q, int OP, int RHEO>
__device__ __forceinline__ void relax_and_collide(const StepParams& p, unsigned n, uint8_t cls, int slot,
                                                  float (&f)[Q]) {
    relax_and_collide<Q, OP, RHEO>(p, p.side_next, n, cls, slot, f, (RHEO == VLBM_POWERLAW) ? p.omega[n] : 0.f);
}

// ------------------------------------------------------------ kernels --
// Occupancy: the odd (neighbour) step needs more address registers; capping it
// at 4 resident 256-thread blocks per SM (64 registers) keeps enough loads in
// flight to saturate HBM.
template <int Q, int OP, int RHEO, int ST, bool ODD>
__device__ __forceinline__ void step_node(const StepParams& p, const float* side_prev, float* side_next, int use_bc,
                                          unsigned seed, unsigned n) {
    using S = Store<ST>;
    using T = typename S::T;
    const int x = (int)(n % (unsigned)p.nx);
    const unsigned t = n / (unsigned)p.nx;
    const int y = (int)(t % (unsigned)p.ny);
    const int z = (int)(t / (unsigned)p.ny);
    Nbr nb;
    nb.init(x, y, z, p.nx, p.ny, p.nz);

    const float eta_old = (RHEO == VLBM_POWERLAW) ? p.omega[n] : 0.f;   // loaded with the populations
    float f[Q];
    uint8_t cls;
    const int slot = gather<Q, ST, ODD>(p, side_prev, use_bc, n, nb, x, y, z, f, cls);
    relax_and_collide<Q, OP, RHEO>(p, side_next, n, cls, slot, f, eta_old);
    nb.launder();
    Rng rng(n, seed);
    T* plane = static_cast<T*>(p.pop);
    const size_t N = (size_t)p.N;
#pragma unroll
    for (int j = 0; j < Q; ++j, plane += N) {
        if (!ODD) {  // plane j receives the post-collision value of opp(j) at this node
            const int i = lat_opp(j);
            S::st(plane + n, f[i], Lattice<Q>::w(i), p, rng);
        } else {     // plane j receives population j streamed to the downstream node
            const unsigned dst = n + nb.off(lat_cx(j), lat_cy(j), lat_cz(j));
            S::st(plane + dst, f[j], Lattice<Q>::w(j), p, rng);
        }
    }
}

// The step count that seeds the stochastic rounding lives on the device, one
// slot per AA parity: a step reads its parity's slot and block 0 writes the
// incremented count to the other parity's slot, which no thread of this step
// reads, so a replayed graph of steps keeps counting.
__device__ __forceinline__ unsigned step_seed(const StepParams& p, bool odd) {
    const unsigned s = p.ctr[odd ? 1 : 0];
    if (blockIdx.x == 0 && threadIdx.x == 0) p.ctr[odd ? 0 : 1] = s + 1;
    return s;
}

// Consecutive steps form a chain of programmatic dependents: a step's first
// kernel waits for the previous kernel in the stream to complete (and its
// writes to be visible) before it reads anything, then lets its own dependent
// be scheduled, so the next launch's latency and ramp overlap this grid's
// tail.  After a kernel that does not trigger, the wait returns at once.
__device__ __forceinline__ void step_chain_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <int Q, int OP, int RHEO, int ST, bool ODD>
__global__ void __launch_bounds__(256) k_step(const StepParams p) {
    step_chain_enter();
    const unsigned seed = step_seed(p, ODD);
    const unsigned n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (unsigned)p.N) return;
    step_node<Q, OP, RHEO, ST, ODD>(p, p.side_prev, p.side_next, p.apply_bc, seed, n);
}

// ------------------------------------------------------- batched step --
// Many lattices of one (velocity set, operator, rheology, storage) group
// advance in one launch.  The launch walks a table of tiles (lattice slot,
// first node; BATCH_TILE consecutive nodes each) with a grid-stride loop, so a
// grid of a few blocks per SM is persistent over all lattices.  The lattices'
// parameters sit in a device-resident BatchLaunch table whose address is the
// launch's argument; a block copies a lattice's parameters into shared memory
// when its tile belongs to another lattice than its previous one.  Lattices whose
// AA parity differs go to different tables (the parity is a template argument,
// as in k_step); the side-store buffer index and the boundary flag of every
// lattice live in its slot in device memory and are advanced by
// k_batch_advance after the group launches, so a captured step can be
// replayed any number of times.
constexpr int BATCH_TILE = 256;
constexpr int BATCH_MAX_SLOTS = 64;   // lattices per launch (parameters in one BatchLaunch table)

// Per-lattice state that changes every step (advanced by k_batch_advance).
struct BatchState {
    int side_cur, apply_bc, parity;
    unsigned step;      // steps taken (the stochastic-rounding seed)
};
struct BatchBlock {
    int slot;           // lattice of this tile: index into the launch's parameters
    unsigned first;     // first node of this tile
};
// Parameters of one batched launch: the step parameters of up to
// BATCH_MAX_SLOTS lattices (side_prev / side_next hold side[0] / side[1]).
// They stay in device memory between table rebuilds and the launch passes a
// pointer: 12 KB of launch arguments would cost host time on every launch,
// while a block reads a lattice's 200 bytes once per lattice change.
struct BatchLaunch {
    StepParams p[BATCH_MAX_SLOTS];
    int state_base;     // index of p[0]'s entry in the state array
};

// Resident blocks per SM the batched kernel is compiled for: D3Q19 fits five
// 256-thread blocks (51 registers), D3Q27 four (64 registers).
template <int Q> constexpr int batch_min_blocks() { return Q == 19 ? 5 : 4; }

template <int Q, int OP, int RHEO, int ST, bool ODD>
__global__ void __launch_bounds__(256, batch_min_blocks<Q>()) k_step_batched(const BatchLaunch* __restrict__ L,
                                                                            const BatchState* __restrict__ state,
                                                                            const BatchBlock* __restrict__ table,
                                                                            int ntiles) {
    step_chain_enter();   // after the previous launch of the server stream
    __shared__ StepParams sp;
    __shared__ float* sides[2];
    __shared__ int use_bc;
    __shared__ unsigned seed;
    constexpr int WORDS = (int)(sizeof(StepParams) / 4);
    static_assert(sizeof(StepParams) % 4 == 0, "StepParams is copied as 32-bit words");
    int t = blockIdx.x;
    if (t >= ntiles) return;
    BatchBlock e = table[t];
    int cur = -1;   // lattice whose parameters are in sp (block-uniform)
    for (; t < ntiles; t += gridDim.x) {
        // the next tile's entry is fetched while this one computes
        const int tn = t + gridDim.x;
        const BatchBlock en = tn < ntiles ? table[tn] : e;
        if (e.slot != cur) {   // uniform: every thread holds the same entry
            __syncthreads();   // the previous lattice's tiles are done with sp
            if (threadIdx.x < WORDS)
                reinterpret_cast<unsigned*>(&sp)[threadIdx.x] =
                    reinterpret_cast<const unsigned*>(&L->p[e.slot])[threadIdx.x];
            if (threadIdx.x == WORDS) {
                const BatchState st = state[L->state_base + e.slot];
                const StepParams& q = L->p[e.slot];
                sides[0] = st.side_cur ? const_cast<float*>(q.side_next) : const_cast<float*>(q.side_prev);
                sides[1] = st.side_cur ? const_cast<float*>(q.side_prev) : q.side_next;
                use_bc = st.apply_bc;
                seed = (unsigned)st.step;
            }
            __syncthreads();
            cur = e.slot;
        }
        const unsigned n = e.first + threadIdx.x;
        if (n < (unsigned)sp.N) step_node<Q, OP, RHEO, ST, ODD>(sp, sides[0], sides[1], use_bc, seed, n);
        e = en;
    }
}

// Macroscopics of the current state (what gpuMacrCollisionStream saves).
template <int Q, int RHEO, int ST, bool ODD, bool PAIRED>
__global__ void __launch_bounds__(256) k_macro(const MacroParams mp) {
    const StepParams& p = mp.s;
    const unsigned n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (unsigned)p.N) return;
    const int x = (int)(n % (unsigned)p.nx);
    const unsigned t = n / (unsigned)p.nx;
    const int y = (int)(t % (unsigned)p.ny);
    const int z = (int)(t / (unsigned)p.ny);
    Nbr nb;
    nb.init(x, y, z, p.nx, p.ny, p.nz);
    float f[Q];
    uint8_t cls;
    gather<Q, ST, ODD, PAIRED>(p, n, nb, x, y, z, f, cls);
    float fx = p.fx, fy = p.fy, fz = p.fz;
    if (mp.fibm_const) {
        const size_t N = (size_t)p.N;
        fx += mp.fibm_const[n]; fy += mp.fibm_const[N + n]; fz += mp.fibm_const[2 * N + n];
    }
    if (cls & NODE_UNUSED) {   // never updated: the initial macroscopics (lbmInitialization.cu:100-111)
        if (mp.rho) mp.rho[n] = p.rho0;
        if (mp.ux) mp.ux[n] = 0.f;
        if (mp.uy) mp.uy[n] = 0.f;
        if (mp.uz) mp.uz[n] = 0.f;
        if (mp.omega_out) mp.omega_out[n] = 0.f;
        return;
    }
    constexpr bool NEED_PI = RHEO != VLBM_NEWTONIAN;
    const Mom m = moments<Q, NEED_PI>(f, fx, fy, fz, p.rho0);
    if (mp.rho) mp.rho[n] = m.rho;
    if (mp.ux) mp.ux[n] = m.ux;
    if (mp.uy) mp.uy[n] = m.uy;
    if (mp.uz) mp.uz[n] = m.uz;
    if (mp.omega_out) {
        float omega = p.omega_newt;
        if (RHEO != VLBM_NEWTONIAN) {
            const float aux = stress_aux(m, fx, fy, fz);
            const float old = (RHEO == VLBM_POWERLAW) ? p.omega[n] : 0.f;
            float eta = 0.f;
            omega = relax<RHEO>(p, old, aux, eta);
        }
        mp.omega_out[n] = omega;
    }
}

// Populations f_i(x,t) after boundary rules, natural [Q][N] float layout.
template <int Q, int ST, bool ODD, bool PAIRED>
__global__ void __launch_bounds__(256) k_get_pops(const StepParams p, float* out) {
    const unsigned n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (unsigned)p.N) return;
    const int x = (int)(n % (unsigned)p.nx);
    const unsigned t = n / (unsigned)p.nx;
    const int y = (int)(t % (unsigned)p.ny);
    const int z = (int)(t / (unsigned)p.ny);
    Nbr nb;
    nb.init(x, y, z, p.nx, p.ny, p.nz);
    float f[Q];
    uint8_t cls;
    gather<Q, ST, ODD, PAIRED>(p, n, nb, x, y, z, f, cls);
#pragma unroll
    for (int i = 0; i < Q; ++i) out[(size_t)i * (size_t)p.N + n] = f[i] + Lattice<Q>::w(i) * p.rho0;
}

// Natural-layout store of given populations (equilibrium init or user state).
template <int Q, int ST, bool PAIRED>
__global__ void __launch_bounds__(256) k_set_pops(const StepParams p, const float* in, float rho, float ux,
                                                  float uy, float uz) {
    using S = Store<ST>;
    using T = typename S::T;
    const unsigned n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= (unsigned)p.N) return;
    T* A = static_cast<T*>(p.pop);
    const size_t N = (size_t)p.N;
    const int x = (int)(n % (unsigned)p.nx);
    const unsigned t = n / (unsigned)p.nx;
    const int y = (int)(t % (unsigned)p.ny), z = (int)(t / (unsigned)p.ny);
    const float uu = ux * ux + uy * uy + uz * uz;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        float v;
        if (in) {
            v = in[(size_t)i * N + n];
        } else {  // gpu_f_eq, globalFunctions.h:50-56 / lbmInitialization.cu:78-89
            const float cu = lat_cx(i) * ux + lat_cy(i) * uy + lat_cz(i) * uz;
            v = Lattice<Q>::w(i) * rho * (1.f - 1.5f * uu + 3.f * cu * (1.f + 1.5f * cu));
        }
        const size_t e = PAIRED ? pair_elem<Q>(p, i, x, y, z) : (size_t)i * N + n;
        S::st_abs(A + e, v, Lattice<Q>::w(i), p);
    }
    if (p.omega) p.omega[n] = __int_as_float(0x7f800000);  // eta = +inf <=> omega = 0 (lbmInitialization.cu:111)
}

// ------------------------------------------------- z-paired two-node step --
// Vector view of a node pair in each storage type.
template <int ST> struct Pair;
template <> struct Pair<VLBM_STORE_F32> {
    using V = float2;
    static __device__ __forceinline__ float get(const V& v, int lane, float, const StepParams&) {
        return lane ? v.y : v.x;
    }
    static __device__ __forceinline__ void set(V& v, int lane, float g, float, const StepParams&, Rng&) {
        if (lane) v.y = g; else v.x = g;
    }
    static __device__ __forceinline__ V swap(const V& v) { return make_float2(v.y, v.x); }
    // both lanes as deviations / packed from deviations (stored as they are)
    static constexpr bool kScaled = false;
    static __device__ __forceinline__ float2 get2(const V& v, float, const StepParams&) { return v; }
    static __device__ __forceinline__ float2 raw2(const V& v) { return v; }
    static __device__ __forceinline__ V pack2(float2 g, float, const StepParams&, Rng&, Rng&) { return g; }
};
template <> struct Pair<VLBM_STORE_F16> {
    using V = __half2;
    static __device__ __forceinline__ float get(const V& v, int lane, float, const StepParams& s) {
        return (lane ? __high2float(v) : __low2float(v)) * s.inv_scale;
    }
    static __device__ __forceinline__ void set(V& v, int lane, float g, float, const StepParams& s, Rng& r) {
        const __half h = half_sr(g * s.scale, r.next());
        v = lane ? __halves2half2(__low2half(v), h) : __halves2half2(h, __high2half(v));
    }
    static __device__ __forceinline__ V swap(const V& v) { return __lowhigh2highlow(v); }
    static __device__ __forceinline__ float2 get2(const V& v, float, const StepParams& s) {
        return mul2(__half22float2(v), f2(s.inv_scale));
    }
    // the stored values times `scale` (a power of two): k_step2 scales the moment
    // sums instead of every population, which gives the same bits
    static constexpr bool kScaled = true;
    static __device__ __forceinline__ float2 raw2(const V& v) { return __half22float2(v); }
    // both lanes rounded stochastically by the conversion itself (sm_100a
    // cvt.rs: the low half takes its random bits from rbits[12:0], the high
    // half from rbits[28:16]; measured, and unbiased to 1e-4 ulp over 4M
    // draws).  One draw per pair; folding its upper half into the lower gives
    // the low lane mixed bits, not the weak low bits of the congruential draw.
    // v: deviations times the storage scale (collide2's output).
    static __device__ __forceinline__ V pack2(float2 v, float, const StepParams&, Rng& r0, Rng&) {
        const unsigned r = r0.next();
        unsigned out;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(out) : "f"(v.y), "f"(v.x), "r"(r ^ (r >> 16)));
        return *reinterpret_cast<__half2*>(&out);
    }
};
template <> struct Pair<VLBM_STORE_BF16> {
    using V = __nv_bfloat162;
    static __device__ __forceinline__ float get(const V& v, int lane, float, const StepParams& s) {
        return (lane ? __high2float(v) : __low2float(v)) * s.inv_scale;
    }
    static __device__ __forceinline__ void set(V& v, int lane, float g, float, const StepParams& s, Rng& r) {
        const __nv_bfloat16 h = bf16_sr(g * s.scale, r.next());
        v = lane ? __halves2bfloat162(__low2bfloat16(v), h) : __halves2bfloat162(h, __high2bfloat16(v));
    }
    static __device__ __forceinline__ V swap(const V& v) { return __lowhigh2highlow(v); }
    static __device__ __forceinline__ float2 get2(const V& v, float, const StepParams& s) {
        return mul2(__bfloat1622float2(v), f2(s.inv_scale));
    }
    static constexpr bool kScaled = true;
    static __device__ __forceinline__ float2 raw2(const V& v) { return __bfloat1622float2(v); }
    // cvt.rs for bfloat16: random bits rbits[15:0] (low half), [31:16] (high
    // half); v: deviations times the storage scale
    static __device__ __forceinline__ V pack2(float2 v, float, const StepParams&, Rng& r0, Rng&) {
        const unsigned r = r0.next();
        unsigned out;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(out) : "f"(v.y), "f"(v.x), "r"(r ^ (r >> 16)));
        return *reinterpret_cast<const __nv_bfloat162*>(&out);
    }
};

// Neighbour offsets of a pair-node in blocked storage, in pairs: own(m') -
// own(m) with own(m) = (m / 32) * 32 Q + m % 32.  A y or z neighbour keeps m %
// 32 (rows hold whole blocks), so its offset is the pair-space offset times
// Q; an x neighbour may sit in the next or previous block.  Offsets along the
// axes add up for the diagonal neighbours.
struct BlkNbr {
    int xm, xp, ym, yp, zm, zp;
    template <int Q>
    __device__ __forceinline__ void init(const Nbr& pn, unsigned m) {
        const int own = (int)((m >> 5) * (Q * 32u) + (m & 31u));
        const unsigned a = (unsigned)((int)m + pn.xm), b = (unsigned)((int)m + pn.xp);
        xm = (int)((a >> 5) * (Q * 32u) + (a & 31u)) - own;
        xp = (int)((b >> 5) * (Q * 32u) + (b & 31u)) - own;
        ym = pn.ym * Q; yp = pn.yp * Q; zm = pn.zm * Q; zp = pn.zp * Q;
    }
    __device__ __forceinline__ void launder() {
        asm volatile("" : "+r"(xm), "+r"(xp), "+r"(ym), "+r"(yp), "+r"(zm), "+r"(zp));
    }
    __device__ __forceinline__ int off(int dx, int dy, int dz) const {
        return (dx > 0 ? xp : (dx < 0 ? xm : 0)) + (dy > 0 ? yp : (dy < 0 ? ym : 0)) +
               (dz > 0 ? zp : (dz < 0 ? zm : 0));
    }
};

// One thread advances the node pair (x, y, zp) / (x, y, zp+H), pair-node m.
// Every access is one aligned vector of the two nodes, also for the x-shifted
// neighbours of the odd step; crossing the periodic z seam swaps the two lanes.
//
// BLK (blocked pairs, NX % 32 == 0): a warp's 32 pairs are one block, whose Q
// planes follow each other, so plane j of the thread's own pair is at a
// compile-time offset (32 j) from one pointer, and a neighbour's is that plus
// one of six axis offsets formed once per thread (BlkNbr).
//
// BULK: the pair holds no boundary and no unused node, so the boundary
// rules, the side store and the unused-node path are compiled out (the bulk
// kernel then fits 64 registers for D3Q19: 4 resident blocks of 256 instead
// of 3).  A BULK thread whose class bytes, loaded with the populations, show
// such a node returns before it writes anything; k_step2 runs those pairs
// from their list.
template <int Q, int OP, int RHEO, int ST, bool ODD, bool BLK, bool BULK>
__device__ __forceinline__ void step2_pair(const StepParams& p, const unsigned seed, const unsigned m) {
    using PV = Pair<ST>;
    using V = typename PV::V;
    const int H = p.pairH;
    const int x = (int)(m % (unsigned)p.nx);
    const unsigned t = m / (unsigned)p.nx;
    const int y = (int)(t % (unsigned)p.ny);
    const int zp = (int)(t / (unsigned)p.ny);
    Nbr pn;                       // neighbour offsets in pair space
    pn.init(x, y, zp, p.nx, p.ny, H);
    const bool seam_lo = zp == 0, seam_hi = zp == H - 1;
    // node indices: (x, y, zp) is m, (x, y, zp + H) is m + N/2 (the even bulk
    // step needs neither x, y, zp nor the neighbour offsets)
    const unsigned n0 = m, n1 = m + (unsigned)(p.N >> 1);
    // the Power-Law state of both nodes, loaded with the populations
    const float eta0 = (RHEO == VLBM_POWERLAW) ? p.omega[n0] : 0.f;
    const float eta1 = (RHEO == VLBM_POWERLAW) ? p.omega[n1] : 0.f;
    const size_t Np = (size_t)p.N >> 1;   // pairs per plane (plain pairs)
    V in[Q];
    const V* __restrict__ P = reinterpret_cast<const V*>(p.pop);
    const size_t own = BLK ? (size_t)(m >> 5) * (Q * 32) + (m & 31u) : 0;
    const V* __restrict__ Pown = P + own;
    BlkNbr bn;
    if (BLK && ODD) bn.init<Q>(pn, m);
#pragma unroll
    for (int j = 0; j < Q; ++j) {
        if (BLK) {
            if (!ODD) {
                in[j] = Pown[32 * j];
            } else {
                const int i = lat_opp(j);
                in[i] = Pown[(ptrdiff_t)bn.off(-lat_cx(i), -lat_cy(i), -lat_cz(i)) + 32 * j];
            }
        } else if (!ODD) {
            in[j] = P[(size_t)j * Np + m];
        } else {
            const int i = lat_opp(j);
            in[i] = P[(size_t)j * Np + (unsigned)((int)m + pn.off(-lat_cx(i), -lat_cy(i), -lat_cz(i)))];
        }
    }
    // Crossing the z seam exchanges the lanes.  Only the two seam planes of
    // the pair space do it, and a warp lies in one plane, so one uniform
    // branch replaces a select per population.
    if (ODD && (seam_lo || seam_hi)) {
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            const int cz = lat_cz(i);
            if ((cz > 0 && seam_lo) || (cz < 0 && seam_hi)) in[i] = PV::swap(in[i]);
        }
    }
    // both nodes as float2: lane 0 is (x, y, zp), lane 1 (x, y, zp + H).  Half
    // storage is read as stored (deviation * scale); the moment sums are
    // scaled instead, and the boundary rules see scaled-back values.
    constexpr bool SC = PV::kScaled;
    float2 g[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) g[i] = PV::raw2(in[i]);
    const uint8_t c0 = p.cls[n0], c1 = p.cls[n1];
    if (BULK && ((c0 | c1) & (NODE_BC | NODE_UNUSED))) return;   // k_step2's pair
    int slot0 = -1, slot1 = -1;
    if (!BULK && ((c0 | c1) & NODE_BC)) {   // boundary rules per lane, on scalars
#pragma unroll
        for (int lane = 0; lane < 2; ++lane) {
            const uint8_t cl = lane ? c1 : c0;
            if (!(cl & NODE_BC)) continue;
            const unsigned nl = lane ? n1 : n0;
            const int zl = zp + lane * H;
            const int sl = p.bc_slot[nl];
            if (lane) slot1 = sl; else slot0 = sl;
            if (p.apply_bc) {
                float f[Q];
#pragma unroll
                for (int i = 0; i < Q; ++i) f[i] = SC ? lane_of(g[i], lane) * p.inv_scale : lane_of(g[i], lane);
                Nbr nb;
                nb.init(x, y, zl, p.nx, p.ny, p.nz);
                apply_bc<Q>(f, p, sl, x, y, zl, nb, nl);
#pragma unroll
                for (int i = 0; i < Q; ++i) set_lane(g[i], lane, SC ? f[i] * p.scale : f[i]);
            }
        }
    }
    float2 fx2 = f2(p.fx), fy2 = f2(p.fy), fz2 = f2(p.fz);
    if ((c0 | c1) & NODE_IBM_FORCE) {   // IBM force read and reset (lbm.cu:45-58)
        const size_t N = (size_t)p.N;
#pragma unroll
        for (int lane = 0; lane < 2; ++lane) {
            const uint8_t cl = lane ? c1 : c0;
            if (!(cl & NODE_IBM_FORCE)) continue;
            const unsigned nl = lane ? n1 : n0;
            set_lane(fx2, lane, p.fx + p.fibm[nl]);
            set_lane(fy2, lane, p.fy + p.fibm[N + nl]);
            set_lane(fz2, lane, p.fz + p.fibm[2 * N + nl]);
            p.fibm[nl] = 0.f; p.fibm[N + nl] = 0.f; p.fibm[2 * N + nl] = 0.f;
            p.cls[nl] = cl & (uint8_t)~NODE_IBM_FORCE;
        }
    }
    constexpr bool NEED_PI = (OP == VLBM_OP_REGULARIZED) || (RHEO != VLBM_NEWTONIAN);
    const Mom2 mm = moments2<Q, NEED_PI, SC>(g, fx2, fy2, fz2, p.rho0, p.inv_scale);
    if ((!(mm.rho.x > 0.f && mm.rho.x < 1e30f) && !(c0 & NODE_UNUSED)) ||
        (!(mm.rho.y > 0.f && mm.rho.y < 1e30f) && !(c1 & NODE_UNUSED)))
        atomicOr(p.err, 1u);
    float2 omega = f2(p.omega_newt);
    if (RHEO != VLBM_NEWTONIAN) {
        const float2 aux = stress_aux2(mm, fx2, fy2, fz2);
#pragma unroll
        for (int lane = 0; lane < 2; ++lane) {
            const unsigned nl = lane ? n1 : n0;
            float eta = 0.f;
            set_lane(omega, lane, relax<RHEO>(p, lane ? eta1 : eta0, lane_of(aux, lane), eta));
            if (RHEO == VLBM_POWERLAW) p.omega[nl] = eta;   // state update, lbm.cu:215-219
        }
    }
    // post-collision values as stored: deviations times the storage scale
    collide2<Q, OP>(g, mm, omega, fx2, fy2, fz2, SC ? p.inv_scale : 1.f, SC ? p.scale : 1.f);
    if (!BULK && ((c0 | c1) & NODE_UNUSED)) {   // lbm.cu:23-24: not updated; rest equilibrium stays in the slots
        const bool u0 = c0 & NODE_UNUSED, u1 = c1 & NODE_UNUSED;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (u0) g[i].x = 0.f;
            if (u1) g[i].y = 0.f;
        }
    }
    if (!BULK && (slot0 >= 0 || slot1 >= 0)) {   // post-collision values of boundary nodes (lbm.cu:463-470)
        const size_t nbc = (size_t)p.nbc;
#pragma unroll
        for (int i = 0; i < Q; ++i) {   // the side store keeps deviations
            if (slot0 >= 0) p.side_next[(size_t)i * nbc + slot0] = SC ? g[i].x * p.inv_scale : g[i].x;
            if (slot1 >= 0) p.side_next[(size_t)i * nbc + slot1] = SC ? g[i].y * p.inv_scale : g[i].y;
        }
    }
    // one random stream per node pair, drawn in destination-plane order; each
    // draw gives both lanes their bits (the one-node kernel has a stream per
    // node, so the two layouts round differently but equally well)
    Rng r0(n0, seed), r1(n0, seed);
#pragma unroll
    for (int j = 0; j < Q; ++j) {
        const int i = ODD ? j : lat_opp(j);
        in[i] = PV::pack2(g[i], Lattice<Q>::w(i), p, r0, r1);
    }
    if (ODD && (seam_lo || seam_hi)) {   // lanes exchanged across the z seam, as for the loads
#pragma unroll
        for (int j = 1; j < Q; ++j) {
            const int cz = lat_cz(j);
            if ((cz > 0 && seam_hi) || (cz < 0 && seam_lo)) in[j] = PV::swap(in[j]);
        }
    }
    if (ODD) pn.launder();
    if (ODD && BLK) bn.launder();
    V* __restrict__ Po = reinterpret_cast<V*>(p.pop);
    V* __restrict__ Powo = Po + own;
#pragma unroll
    for (int j = 0; j < Q; ++j) {
        if (BLK) {
            if (!ODD) Powo[32 * j] = in[lat_opp(j)];
            else Powo[(ptrdiff_t)bn.off(lat_cx(j), lat_cy(j), lat_cz(j)) + 32 * j] = in[j];
        } else if (!ODD) {
            Po[(size_t)j * Np + m] = in[lat_opp(j)];
        } else {
            Po[(size_t)j * Np + (unsigned)((int)m + pn.off(lat_cx(j), lat_cy(j), lat_cz(j)))] = in[j];
        }
    }
}

// Resident 256-thread blocks per SM asked of the bulk pair kernel (-Xptxas -v
// and timings at 256^3): regularized D3Q19 fits 64 registers for 4 blocks (0
// bytes of spill in the even step, 12-36 in the odd one); BGK keeps every
// population live across the collision and spills 40-180 bytes there, so it
// takes 3.  D3Q27 at 80 registers (3 blocks) spills 30-56 bytes: worth it for
// half storage, which is issue-bound (regularized FP16 46.5k against 42.1k
// MLUPS at 2 blocks), not for FP32, which streams at the copy bandwidth
// either way (30.0k against 30.5k), nor for BGK (64-250 bytes of spill).
template <int Q, int OP, int ST> constexpr int step2_bulk_blocks() {
    if (Q == 19) return OP == VLBM_OP_REGULARIZED ? 4 : 3;
    return (OP == VLBM_OP_REGULARIZED && ST != VLBM_STORE_F32) ? 3 : 2;
}

// The pair step over every pair; pairs with a boundary or unused node return
// (step2_pair, BULK) and are advanced by k_step2.
template <int Q, int OP, int RHEO, int ST, bool ODD, bool BLK>
__global__ void __launch_bounds__(256, step2_bulk_blocks<Q, OP, ST>()) k_step2_bulk(const StepParams p) {
    // Launched as the programmatic dependent of the step's boundary list
    // (k_step2), whose pairs it does not touch: it reads without waiting.  It
    // lets the next step's first kernel be scheduled.  One thread of the last
    // block waits for the boundary list before it exits, so this grid cannot
    // complete before the list and the next step's single wait covers both;
    // the last block runs in the grid's last wave, when the list is long done,
    // so no block holds its SM idle.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const unsigned seed = step_seed(p, ODD);
    const unsigned m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < (unsigned)(p.N >> 1)) step2_pair<Q, OP, RHEO, ST, ODD, BLK, true>(p, seed, m);
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) asm volatile("griddepcontrol.wait;" ::: "memory");
}

// The pair step over the pairs with a boundary or unused node, one thread per
// entry of the list p.special_pairs.
template <int Q, int OP, int RHEO, int ST, bool ODD, bool BLK>
__global__ void __launch_bounds__(256) k_step2(const StepParams p) {
    // The step's first kernel: it waits for the previous step, then lets the
    // bulk grid start.  The bulk grid touches other pairs only (each pair owns
    // the slots it reads and writes), so it runs while these few long
    // boundary threads are in flight instead of after them.
    step_chain_enter();
    const unsigned seed = step_seed(p, ODD);
    const unsigned k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (unsigned)p.n_special) return;
    step2_pair<Q, OP, RHEO, ST, ODD, BLK, false>(p, seed, (unsigned)p.special_pairs[k]);
}

}  // namespace vlbm
