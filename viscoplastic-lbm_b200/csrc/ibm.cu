// ibm.cu -- immersed-boundary step for movable spheres on the GPU.
//
// The reference (src/CUDA/IBM/ibm.cu:6-192) runs, after every fluid step, ~9 +
// 4*IBM_MAX_ITERATION host-synchronised launches, two of which sweep the whole
// lattice (gpuUpdateMacrIBM recomputes rho,u everywhere; gpuEulerSumIBMAuxsReset
// adds the auxiliary fields everywhere, once per iteration).  Here only the
// Eulerian nodes inside each sphere's stencil support are touched, in six
// launches per step with one forcing iteration (three more per iteration):
//
//   k_ibm_begin      one CTA per sphere: unwrapped node extent -> Eulerian
//                    box of each sphere, node forces reset (gpuResetNodesForces
//                    ibm.cu:651-668); beside it and the gather, on a stream of
//                    its own, one CTA: old values, Hertz-Mindlin contacts with
//                    deterministic slot updates and sums, predictor
//   k_ibm_gather     several CTAs per sphere: rho,u of the post-boundary
//                    populations with the constant body force
//                    (gpuUpdateMacrIBM ibm.cu:544-648) for the box nodes,
//                    written to dense fields; each node's owner becomes the
//                    lowest index of the spheres whose box holds it
//   per multi-direct-forcing iteration:
//     k_ibm_interp_spread  several CTAs per sphere, one warp per Lagrangian
//                    node with its 64 stencil points split over the lanes:
//                    Peskin 4-point interpolation (warp reduction), direct
//                    forcing, spreading with fixed-point atomics; per-CTA
//                    force/torque partials
//     k_ibm_update   one warp per sphere: partials added in a fixed order, particle velocity and
//                    rotation update; in the last iteration also the particle
//                    movement and the step clock
//     k_ibm_euler    over the boxes, each node by its owner sphere's CTAs:
//                    u += fAux/(2 rho), F += fAux, fAux = 0; in the last
//                    iteration also the Lagrangian node movement
//
// Particle state, contacts and integration are FP64; the Eulerian fields FP32.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <string>
#include <cmath>
#include <cstring>
#include <vector>
#include "sim.h"
#include "step_impl.cuh"

namespace vlbm {

constexpr int IBM_MAX_SLOTS = 13;           // MAX_ACTIVE_COLLISIONS, ibmBoundaryCondition.h:78
constexpr int IBM_THREADS = 256;
constexpr int IBM_NODES_PER_CTA = 32;       // Lagrangian nodes per CTA of k_ibm_interp_spread (4 per warp)
constexpr int IBM_MAX_SPLIT = 32;           // CTAs per sphere, at most
constexpr int IBM_MAX_PARTICLES = 1024;   // pair buffer np*np*6 doubles <= 50 MB
constexpr unsigned IBM_NO_OWNER = 0xFFFFFFFFu;   // owner[] of a node in no sphere's box

struct DPart {
    double pos[3], pos_old[3], vel[3], vel_old[3], w[3], w_avg[3], w_old[3], w_pos[3];
    double f[3], f_old[3], M[3], M_old[3], I[6], dP[3], dL[3];
    double S, radius, volume, density;
    int movable, node_begin, node_count, pad;
    int partner[IBM_MAX_SLOTS], last[IBM_MAX_SLOTS];
    double tdisp[IBM_MAX_SLOTS][3];
    int box_lo[3], box_n[3];
};

struct IbmParams {
    int np, nnodes;
    int nx, ny, nz;
    int wall[3];
    double alpha, rho_f, g[3], thickness;
    double ss_n, sw_n, ss_t, sw_t, dpp, dpw, mu_pp, mu_pw;
    float fx, fy, fz;
    int step;
};

struct IbmState {
    vlbm_ibm_config cfg{};
    IbmParams prm{};
    int np = 0, nnodes = 0;
    DPart* parts = nullptr;
    double *nx = nullptr, *ny = nullptr, *nz = nullptr, *nS = nullptr;
    double *nfx = nullptr, *nfy = nullptr, *nfz = nullptr, *ndx = nullptr, *ndy = nullptr, *ndz = nullptr;
    int* npid = nullptr;
    float* fields = nullptr;      // [4][N] rho,ux,uy,uz (IBM macroscopics)
    unsigned long long* faux = nullptr;   // [3][N] spread force, fixed point (IBM_FIX_SCALE)
    unsigned* owner = nullptr;    // [N] lowest sphere index whose box holds the node, during a step;
                                  // IBM_NO_OWNER everywhere between steps
    int* clock = nullptr;         // IBM steps taken (contact history clock)
    double* contrib = nullptr;    // [np][np][6] pair force/torque on the row particle
    double* fpart = nullptr;      // [np][split][6] per-CTA force/torque partials
    int split = 1;                // CTAs per sphere in k_ibm_interp_spread
    cudaStream_t cstream = nullptr;   // the contacts' launch, beside the boxes and the gather
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int gsplit = 1;               // CTAs per sphere in k_ibm_gather, k_ibm_euler and k_ibm_fixup
    std::vector<DPart> initial;   // for vlbm_init_equilibrium
    std::vector<double> init_nodes;
    size_t bytes = 0;
};

__device__ __forceinline__ double pdelta(double d, double L) {
    if (fabs(d) > L / 2.0) d = d < 0 ? d + L : d - L;
    return d;
}
__device__ __forceinline__ void dcross(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ int wrapi(int v, int n) { v %= n; return v < 0 ? v + n : v; }
// A box coordinate onto the lattice: box_lo is at least -1 - n (a node just
// across a periodic face) and a box spans at most the lattice, so one
// correction usually suffices; wrapi covers the rest.
__device__ __forceinline__ int wrap_box(int v, int n) {
    if (v < 0) v += n;
    else if (v >= n) v -= n;
    return ((unsigned)v < (unsigned)n) ? v : wrapi(v, n);
}

// The IBM launches of a step form one chain, each launched as a programmatic
// dependent of the one before (launch_chained): a kernel waits for its
// predecessor's completion before touching memory, then lets its own
// dependent be scheduled, so at most two kernels overlap and only their launch
// latency and ramp are hidden.
__device__ __forceinline__ void chain_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Peskin 4-point kernel (ibmGlobalFunctions.h:28-48, STENCIL_4)
__device__ __forceinline__ float stencil4(float x) {
    const float a = fabsf(x);
    if (a <= 1.f) return 0.125f * (3.f - 2.f * a + sqrtf(1.f + 4.f * a - 4.f * a * a));
    if (a <= 2.f) return 0.125f * (5.f - 2.f * a - sqrtf(-7.f + 12.f * a - 4.f * a * a));
    return 0.f;
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
    return s;  // valid in thread 0
}

// ---------------------------------------------------------------- box --
__device__ void ibm_box(const IbmParams& P, DPart* parts, int sphere, const double* X, const double* Y,
                        const double* Z, double* fx, double* fy, double* fz, double* dx, double* dy, double* dz) {
    __shared__ double sh[32];
    DPart& p = parts[sphere];
    const double L[3] = {(double)P.nx, (double)P.ny, (double)P.nz};
    const int Li[3] = {P.nx, P.ny, P.nz};
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int k = threadIdx.x; k < p.node_count; k += blockDim.x) {
        const int j = p.node_begin + k;
        const double q[3] = {X[j], Y[j], Z[j]};
        for (int a = 0; a < 3; ++a) {
            const double u = P.wall[a] ? q[a] : p.pos[a] + pdelta(q[a] - p.pos[a], L[a]);
            mn[a] = fmin(mn[a], u);
            mx[a] = fmax(mx[a], u);
        }
        fx[j] = fy[j] = fz[j] = 0.0;
        dx[j] = dy[j] = dz[j] = 0.0;
    }
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    // min/max block reductions
    for (int a = 0; a < 3; ++a) {
        double v = mn[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
        double w = mx[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_down_sync(0xffffffffu, w, o));
        __syncthreads();
        if ((threadIdx.x & 31) == 0) { sh[threadIdx.x >> 5] = v; sh[16 + (threadIdx.x >> 5)] = w; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a1 = 1e300, a2 = -1e300;
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { a1 = fmin(a1, sh[k]); a2 = fmax(a2, sh[16 + k]); }
            lo[a] = a1;
            hi[a] = a2;
        }
    }
    if (threadIdx.x == 0) {
        for (int a = 0; a < 3; ++a) {
            // stencil of a node at x covers int(x)-1 .. int(x)+2 (ibm.cu:236-240).
            // Extents are clamped in double before any integer conversion so a
            // diverged (non-finite or far-away) sphere yields an empty or
            // axis-sized box, never an out-of-range one.
            int l, h;
            const double La = (double)Li[a];
            if (!isfinite(lo[a]) || !isfinite(hi[a])) {
                l = 0; h = -1;
            } else if (P.wall[a]) {
                const double cl = fmin(fmax(lo[a], -4.0), La + 4.0), ch = fmin(fmax(hi[a], -4.0), La + 4.0);
                l = (int)floor(cl) - 1;
                h = (int)ch + 2;
                if (l < 0) l = 0;
                if (h > Li[a] - 1) h = Li[a] - 1;
            } else if (hi[a] - lo[a] + 5.0 >= La) {
                l = 0; h = Li[a] - 1;
            } else {
                l = (int)floor(lo[a]) - 1;
                h = (int)floor(hi[a]) + 3;   // +1: truncated bases of negative coordinates
            }
            p.box_lo[a] = l;
            p.box_n[a] = h >= l ? h - l + 1 : 0;
        }
    }
}

// -------------------------------------------------------------- gather --
// Box node k (x fastest) of a sphere's box, wrapped onto the lattice.  A box
// holds at most the lattice's nodes (< 2^31), so its indices are 32-bit.
__device__ __forceinline__ unsigned box_node(const IbmParams& P, const DPart& p, unsigned k) {
    const unsigned bx = (unsigned)p.box_n[0], by = (unsigned)p.box_n[1];
    const unsigned t = k / bx;
    const int ix = (int)(k - t * bx), iy = (int)(t % by), iz = (int)(t / by);
    const int x = wrap_box(p.box_lo[0] + ix, P.nx), y = wrap_box(p.box_lo[1] + iy, P.ny),
              z = wrap_box(p.box_lo[2] + iz, P.nz);
    return (unsigned)(((size_t)z * P.ny + y) * P.nx + x);
}
__device__ __forceinline__ unsigned box_size(const DPart& p) {
    return (unsigned)p.box_n[0] * (unsigned)p.box_n[1] * (unsigned)p.box_n[2];
}

// IBM macroscopics of every node of the spheres' boxes (gpuUpdateMacrIBM,
// ibm.cu:545-648, restricted to the boxes).  owner[n] becomes the lowest index
// of the spheres whose box holds node n: the Eulerian pass of each forcing
// iteration updates a node once, from that sphere's CTAs, and the last pass
// sets it back to IBM_NO_OWNER.
template <int Q, int ST, bool ODD, bool PAIRED>
__global__ void __launch_bounds__(IBM_THREADS) k_ibm_gather(StepParams sp, IbmParams P, const DPart* parts,
                                                             float* fields, unsigned* owner, int split) {
    chain_enter();
    // `split` CTAs per sphere share its box
    const unsigned sphere = blockIdx.x / split;
    const DPart& p = parts[sphere];
    const int sub = blockIdx.x % split;
    const unsigned bx = (unsigned)p.box_n[0], by = (unsigned)p.box_n[1];
    const unsigned tot = box_size(p);
    const size_t N = (size_t)sp.N;
    for (unsigned k = sub * blockDim.x + threadIdx.x; k < tot; k += split * blockDim.x) {
        const unsigned t = k / bx;
        const int ix = (int)(k - t * bx), iy = (int)(t % by), iz = (int)(t / by);
        const int x = wrap_box(p.box_lo[0] + ix, P.nx), y = wrap_box(p.box_lo[1] + iy, P.ny),
                  z = wrap_box(p.box_lo[2] + iz, P.nz);
        const unsigned n = (unsigned)(((size_t)z * P.ny + y) * P.nx + x);
        Nbr nb;
        nb.init(x, y, z, sp.nx, sp.ny, sp.nz);
        float f[Q];
        uint8_t cls;
        gather<Q, ST, ODD, PAIRED>(sp, n, nb, x, y, z, f, cls);
        const Mom m = moments<Q, false>(f, P.fx, P.fy, P.fz, sp.rho0);
        fields[n] = m.rho;
        fields[N + n] = m.ux;
        fields[2 * N + n] = m.uy;
        fields[3 * N + n] = m.uz;
        atomicMin(&owner[n], sphere);
    }
}

// ------------------------------------------------------------- contacts --
__device__ int wall_index(const double n[3]) {  // calculateWallIndex ibmCollision.cu:5-19
    return 7 + (1 - (int)n[0]) - 2 * (1 - (int)n[1]) - 3 * (1 - (int)n[2]);
}
__device__ void upd(DPart& p, int idx, const double d[3], int step, double out[3]) {
    if (idx < 0) { out[0] = d[0]; out[1] = d[1]; out[2] = d[2]; return; }
    for (int a = 0; a < 3; ++a) p.tdisp[idx][a] += d[a];
    p.last[idx] = step;
    for (int a = 0; a < 3; ++a) out[a] = p.tdisp[idx][a];
}

// sphereWallCollision ibmCollision.cu:393-508
__device__ void wall_contact(const IbmParams& P, DPart& p, const double wn[3], double disp, double accF[3],
                             double accM[3]) {
    const int step = P.step;
    const double m = p.volume * p.density, r = p.radius;
    const double n[3] = {-wn[0], -wn[1], -wn[2]};
    const double* G = p.vel;
    const double kn = P.sw_n * sqrt(fabs(r));
    const double kt = P.sw_t * sqrt(r) * sqrt(fabs(disp));
    const double etan = P.dpw * sqrt(m * kn), etat = P.dpw * sqrt(m * kt);
    const double fkn = -kn * sqrt(fabs(disp * disp * disp));
    const double Gn = G[0] * n[0] + G[1] * n[1] + G[2] * n[2];
    const double q = pow(fabs(disp), 0.25);
    double fnv[3];
    for (int a = 0; a < 3; ++a) fnv[a] = fkn * n[a] - etan * Gn * n[a] * q;
    const double fn = sqrt(fnv[0] * fnv[0] + fnv[1] * fnv[1] + fnv[2] * fnv[2]);
    double wxn[3];
    dcross(p.w, n, wxn);
    double Gct[3];
    for (int a = 0; a < 3; ++a) Gct[a] = G[a] + r * wxn[a] - Gn * n[a];
    double mag = sqrt(Gct[0] * Gct[0] + Gct[1] * Gct[1] + Gct[2] * Gct[2]);
    double t[3] = {0, 0, 0};
    if (mag != 0) for (int a = 0; a < 3; ++a) t[a] = Gct[a] / mag;
    const int idx = wall_index(n);
    double td[3];
    if (step - p.last[idx] > 1) {
        p.tdisp[idx][0] = p.tdisp[idx][1] = p.tdisp[idx][2] = 0.0;
        p.last[idx] = step;
        for (int a = 0; a < 3; ++a) td[a] = Gct[a];
    } else {
        upd(p, idx, Gct, step, td);
    }
    double ft[3];
    for (int a = 0; a < 3; ++a) ft[a] = -kt * td[a] - etat * Gct[a] * pow(fabs(td[a]), 0.25);
    mag = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
    if (mag > P.mu_pw * fabs(fn)) {
        const double mg[3] = {-Gct[0], -Gct[1], -Gct[2]};
        upd(p, idx, mg, step, td);
        for (int a = 0; a < 3; ++a) ft[a] = -P.mu_pw * fn * t[a];
    }
    double nxf[3];
    dcross(n, ft, nxf);
    for (int a = 0; a < 3; ++a) { accF[a] += fnv[a] + ft[a]; accM[a] += r * nxf[a]; }
}

// sphereSphereCollision ibmCollision.cu:1718-1913; slots kept in the lower
// index i, so one thread per i serialises all slot updates of that particle.
// Centre distance of two spheres (periodic axes wrapped), with explicit
// roundings so the contact screening and the contact itself take the same
// decision bit for bit.
__device__ __forceinline__ double centre_dist(const IbmParams& P, const DPart& pi, const DPart& pj, double d[3]) {
    const double L[3] = {(double)P.nx, (double)P.ny, (double)P.nz};
    for (int a = 0; a < 3; ++a) {
        d[a] = pi.pos[a] - pj.pos[a];
        if (!P.wall[a]) d[a] = pdelta(d[a], L[a]);
    }
    return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2])));
}
__device__ __forceinline__ bool spheres_touch(const IbmParams& P, const DPart& pi, const DPart& pj) {
    double d[3];
    return !(centre_dist(P, pi, pj, d) > pi.radius + pj.radius);
}

__device__ void pair_contact(const IbmParams& P, DPart& pi, const DPart& pj, int j, double accF[3], double accM[3],
                             double* out6) {
    const int step = P.step;
    double d[3];
    const double dist = centre_dist(P, pi, pj, d);
    if (dist > pi.radius + pj.radius) return;
    const double n[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
    const double disp = pi.radius + pj.radius - dist;
    const double G[3] = {pi.vel[0] - pj.vel[0], pi.vel[1] - pj.vel[1], pi.vel[2] - pj.vel[2]};
    const double mi = pi.volume * pi.density, mj = pj.volume * pj.density;
    const double reff = 1.0 / ((pi.radius + pj.radius) / (pi.radius * pj.radius));
    const double meff = 1.0 / ((mi + mj) / (mi * mj));
    const double kn = P.ss_n * sqrt(reff);
    const double kt = P.ss_t * sqrt(reff) * sqrt(fabs(disp));
    const double etan = P.dpp * sqrt(meff * kn), etat = P.dpp * sqrt(meff * kt);
    const double fkn = -kn * sqrt(fabs(disp * disp * disp));
    const double Gn = G[0] * n[0] + G[1] * n[1] + G[2] * n[2];
    const double q = pow(fabs(disp), 0.25);
    double fnv[3];
    for (int a = 0; a < 3; ++a) fnv[a] = fkn * n[a] - etan * Gn * n[a] * q;
    const double fn = sqrt(fnv[0] * fnv[0] + fnv[1] * fnv[1] + fnv[2] * fnv[2]);
    double wi[3], wj[3];
    dcross(pi.w, n, wi);
    dcross(pj.w, n, wj);
    double Gct[3];
    for (int a = 0; a < 3; ++a) Gct[a] = G[a] + pi.radius * wi[a] + pj.radius * wj[a] - Gn * n[a];
    double mag = sqrt(Gct[0] * Gct[0] + Gct[1] * Gct[1] + Gct[2] * Gct[2]);
    double t[3] = {0, 0, 0};
    if (mag != 0) for (int a = 0; a < 3; ++a) t[a] = Gct[a] / mag;
    double td[3];
    int idx = -1;
    for (int s = 7; s < IBM_MAX_SLOTS; ++s)
        if (pi.partner[s] == j && step - pi.last[s] <= 1) { idx = s; break; }
    if (idx == -1) {
        // startCollision (ibmCollision.cu:32-53); ended contacts free their slot
        for (int s = 7; s < IBM_MAX_SLOTS; ++s)
            if (pi.last[s] == -1 || step - pi.last[s] > 1) {
                pi.partner[s] = j;
                pi.tdisp[s][0] = pi.tdisp[s][1] = pi.tdisp[s][2] = 0.0;
                pi.last[s] = step;
                idx = s;
                break;
            }
        for (int a = 0; a < 3; ++a) td[a] = Gct[a];
    } else {
        upd(pi, idx, G, step, td);  // the reference accumulates G here (ibmCollision.cu:1851)
    }
    double ft[3];
    for (int a = 0; a < 3; ++a) ft[a] = -kt * td[a] - etat * Gct[a] * pow(fabs(td[a]), 0.25);
    mag = sqrt(ft[0] * ft[0] + ft[1] * ft[1] + ft[2] * ft[2]);
    if (mag > P.mu_pp * fabs(fn)) {
        const double mg[3] = {-Gct[0], -Gct[1], -Gct[2]};
        upd(pi, idx, mg, step, td);
        for (int a = 0; a < 3; ++a) ft[a] = -P.mu_pp * fn * t[a];
    }
    double nxf[3];
    dcross(n, ft, nxf);
    for (int a = 0; a < 3; ++a) {
        const double fd = fnv[a] + ft[a];
        accF[a] -= fd;
        accM[a] += pi.radius * nxf[a];
        out6[a] += fd;
        out6[3 + a] += pj.radius * nxf[a];
    }
}

// gpuUpdateParticleCenterVelocityAndRotation ibm.cu:755-897
__device__ void update_center(const IbmParams& P, DPart& p) {
    if (!p.movable) return;
    const double al = P.alpha;
    const double inv_v = 1.0 / p.volume;
    for (int a = 0; a < 3; ++a)
        p.vel[a] = p.vel_old[a] + ((p.f_old[a] * (1.0 - al) + p.f[a] * al + p.dP[a]) * inv_v +
                                   (p.density - P.rho_f) * P.g[a]) / p.density;
    const double Ixx = p.I[0], Iyy = p.I[1], Izz = p.I[2], Ixy = p.I[3], Ixz = p.I[4], Iyz = p.I[5];
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
    const double bx = LM[0] + wa[2] * Ly - wa[1] * Lz;
    const double by = LM[1] + wa[0] * Lz - wa[2] * Lx;
    const double bz = LM[2] + wa[1] * Lx - wa[0] * Ly;
    double wn[3];
    wn[0] = p.w_old[0] + ((Iyz * Iyz - Iyy * Izz) * bx - (Ixy * Iyz - Ixz * Iyy) * bz - (Ixz * Iyz - Ixy * Izz) * by) * inv;
    wn[1] = p.w_old[1] + ((Ixz * Ixz - Ixx * Izz) * by - (Ixy * Ixz - Ixx * Iyz) * bz - (Ixz * Iyz - Ixy * Izz) * bx) * inv;
    wn[2] = p.w_old[2] + ((Ixy * Ixy - Ixx * Iyy) * bz - (Ixy * Ixz - Ixx * Iyz) * by - (Ixy * Iyz - Ixz * Iyy) * bx) * inv;
    const double th = sqrt(wa[0] * wa[0] + wa[1] * wa[1] + wa[2] * wa[2]);
    if (th > 0.0 && isfinite(1.0 / th)) {  // I <- R I R^T, R of the quaternion of w_avg
        const double h = sin(th / 2.0) / th;
        const double qw = cos(th / 2.0), qx = wa[0] * h, qy = wa[1] * h, qz = wa[2] * h;
        const double R[3][3] = {
            {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)},
            {2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)},
            {2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)}};
        const double M3[3][3] = {{Ixx, Ixy, Ixz}, {Ixy, Iyy, Iyz}, {Ixz, Iyz, Izz}};
        double T[3][3], O[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                double s = 0;
                for (int c = 0; c < 3; ++c) s += R[a][c] * M3[c][b];
                T[a][b] = s;
            }
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                double s = 0;
                for (int c = 0; c < 3; ++c) s += T[a][c] * R[b][c];
                O[a][b] = s;
            }
        p.I[0] = O[0][0]; p.I[1] = O[1][1]; p.I[2] = O[2][2];
        p.I[3] = O[0][1]; p.I[4] = O[0][2]; p.I[5] = O[1][2];
    }
    for (int a = 0; a < 3; ++a) p.w[a] = wn[a];
}

constexpr int IBM_SCREEN_MAX = 256;   // spheres whose pair screening fits the shared bit matrix

__device__ void ibm_contacts(const IbmParams& P, DPart* parts, double* contrib) {
    // near[i][w] bit b: spheres i and 32w+b touch (the test pair_contact starts with)
    __shared__ unsigned near[IBM_SCREEN_MAX * (IBM_SCREEN_MAX / 32)];
    const int np = P.np;
    const bool screen = np <= IBM_SCREEN_MAX;
    const int W = (np + 31) >> 5;
    // gpuUpdateParticleOldValues ibm.cu:995-1042
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        DPart& p = parts[i];
        for (int a = 0; a < 3; ++a) {
            p.dP[a] = 0; p.dL[a] = 0;
            p.pos_old[a] = p.pos[a]; p.vel_old[a] = p.vel[a]; p.w_old[a] = p.w[a];
            p.f_old[a] = p.f[a]; p.f[a] = 0; p.M[a] = 0;
        }
    }
    __syncthreads();
    if (screen) {   // all pairs at once, a warp per 32 partners, one ballot per word
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int t = warp; t < np * W; t += nw) {
            const int i = t / W, w = t - i * W, k = 32 * w + lane;
            const bool hit = k < np && k != i && spheres_touch(P, parts[i], parts[k]);
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) near[i * W + w] = m;
        }
        __syncthreads();
    }
    // contacts: thread i owns particle i's slots and its walls; partners in
    // increasing index, only those that touch (the others add nothing)
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        DPart& pi = parts[i];
        double F[3] = {0, 0, 0}, Mo[3] = {0, 0, 0};
        if (screen) {
            for (int w = (i + 1) >> 5; w < W; ++w) {
                unsigned m = near[i * W + w];
                if (w == ((i + 1) >> 5)) m &= ~0u << ((i + 1) & 31);   // partners j > i
                while (m) {
                    const int j = 32 * w + __ffs(m) - 1;
                    m &= m - 1;
                    double* o = contrib + ((size_t)i * np + j) * 6;
                    for (int a = 0; a < 6; ++a) o[a] = 0.0;
                    if (!pi.movable && !parts[j].movable) continue;
                    pair_contact(P, pi, parts[j], j, F, Mo, o);
                }
            }
        } else {
            for (int j = i + 1; j < np; ++j) {
                double* o = contrib + ((size_t)i * np + j) * 6;
                for (int a = 0; a < 6; ++a) o[a] = 0.0;
                if (!pi.movable && !parts[j].movable) continue;
                pair_contact(P, pi, parts[j], j, F, Mo, o);
            }
        }
        if (pi.movable) {
            const int Li[3] = {P.nx, P.ny, P.nz};
            for (int a = 0; a < 3; ++a) {
                if (!P.wall[a]) continue;
                double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
                lo[a] = 1;
                hi[a] = -1;
                const double dlo = pi.pos[a];
                if (dlo < pi.radius) wall_contact(P, pi, lo, pi.radius - dlo, F, Mo);
                const double dhi = (Li[a] - 1) - pi.pos[a];
                if (dhi < pi.radius) wall_contact(P, pi, hi, pi.radius - dhi, F, Mo);
            }
        }
        for (int a = 0; a < 3; ++a) { pi.f[a] += F[a]; pi.M[a] += Mo[a]; }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < np; j += blockDim.x) {
        DPart& pj = parts[j];
        if (screen) {   // partners i < j that touch, in increasing index
            for (int w = 0; w <= (j >> 5) && w < W; ++w) {
                unsigned m = near[j * W + w];
                if (w == (j >> 5)) m &= (1u << (j & 31)) - 1u;
                while (m) {
                    const int i = 32 * w + __ffs(m) - 1;
                    m &= m - 1;
                    const double* o = contrib + ((size_t)i * np + j) * 6;
                    for (int a = 0; a < 3; ++a) { pj.f[a] += o[a]; pj.M[a] += o[3 + a]; }
                }
            }
        } else {
            for (int i = 0; i < j; ++i) {
                const double* o = contrib + ((size_t)i * np + j) * 6;
                for (int a = 0; a < 3; ++a) { pj.f[a] += o[a]; pj.M[a] += o[3 + a]; }
            }
        }
        update_center(P, pj);  // predictor (ibm.cu:98-103)
    }
}

// The start of the IBM step, two launches that run side by side: one CTA per
// sphere finds the Eulerian box of its sphere and resets its node forces
// (`contacts` 0, on the step's stream, followed by the gather); one CTA runs
// the old-value copy, the contacts and the predictor (`contacts` 1, on the IBM
// state's own stream, joined before the first interpolation).  They touch
// different fields: the contacts read positions only, which the boxes and the
// gather do not change.
__global__ void __launch_bounds__(IBM_THREADS) k_ibm_begin(IbmParams P, DPart* parts, const double* X, const double* Y,
                                                            const double* Z, double* fx, double* fy, double* fz,
                                                            double* dx, double* dy, double* dz, double* contrib,
                                                            const int* clock, int contacts) {
    chain_enter();
    if (!contacts) {   // one CTA per sphere
        ibm_box(P, parts, blockIdx.x, X, Y, Z, fx, fy, fz, dx, dy, dz);
        return;
    }
    // index of the fluid step just taken (main.cu:270), kept on the device so
    // a captured IBM step can be replayed
    P.step = *clock;
    ibm_contacts(P, parts, contrib);
}

// -------------------------------------------------- interpolation/spread --
// Stencil of one Lagrangian node: base index and validity range per axis.
struct NodeStencil {
    int base[3], lo[3], hi[3];
    float w[3][4];
    bool skip;
};

__device__ __forceinline__ NodeStencil node_stencil(const IbmParams& P, const DPart& p, double X, double Y, double Z) {
    NodeStencil s;
    const double pos[3] = {X, Y, Z};
    const double L[3] = {(double)P.nx, (double)P.ny, (double)P.nz};
    const int Li[3] = {P.nx, P.ny, P.nz};
    s.skip = false;
    for (int a = 0; a < 3; ++a) {
        double xu = P.wall[a] ? pos[a] : p.pos[a] + pdelta(pos[a] - p.pos[a], L[a]);
        if (!(fabs(xu) < 4.0 * L[a] + 8.0)) {  // non-finite or diverged position: no stencil
            s.skip = true;
            xu = 0.0;
        }
        // int(x) - P_DIST + 1 of the stored coordinate (ibm.cu:236-240): truncation,
        // which differs from floor for the negative coordinates a sphere's nodes
        // have across x=0 before their first movement wraps them; for periodic
        // axes the base is then shifted into the sphere-centred frame
        const double raw = s.skip ? 0.0 : pos[a];
        const int braw = (int)raw - 1;
        const double fr_raw = raw - (double)braw;
        if (P.wall[a]) {
            s.base[a] = braw;
        } else {
            const int k = (int)rint((xu - raw) / L[a]);
            s.base[a] = braw + k * Li[a];
        }
        s.lo[a] = 0;
        s.hi[a] = 3;
        if (P.wall[a]) {
            s.hi[a] = (s.base[a] + 3 < Li[a]) ? 3 : (Li[a] - 1 - s.base[a]);
            s.lo[a] = (s.base[a] >= 0) ? 0 : -s.base[a];
        }
        if (s.hi[a] <= 0 || s.lo[a] >= 4) s.skip = true;  // ibm.cu:300-305
        const float fr = (float)fr_raw;
#pragma unroll
        for (int j = 0; j < 4; ++j) s.w[a][j] = stencil4((float)j - fr);
    }
    return s;
}

// Spread force in 2^-48 fixed point, summed with 64-bit integer atomics: the
// sum does not depend on the order of the additions, so a lattice's IBM step is
// bit-reproducible from run to run and alone or among other lattices.
// Resolution 3.6e-15 per contribution (below the FP32 rounding of any
// contribution above 1e-7), range +-32768 for the sum at one node.
constexpr double IBM_FIX_SCALE = 281474976710656.0;   // 2^48
__device__ __forceinline__ unsigned long long to_fix(float v) {
    return (unsigned long long)__double2ll_rn((double)v * IBM_FIX_SCALE);
}
__device__ __forceinline__ float from_fix(unsigned long long v) {
    return (float)((double)(long long)v * (1.0 / IBM_FIX_SCALE));
}

// Lattice index of a box-relative offset: the offsets stay within one period
// of the lattice except when a periodic axis is shorter than the stencil box.
__device__ __forceinline__ int wrap_near(int v, int n) {
    if (v < 0) v += n;
    else if (v >= n) v -= n;
    if ((unsigned)v >= (unsigned)n) v = wrapi(v, n);
    return v;
}

// Interpolation, direct forcing and spreading (ibm.cu:307-541).  One warp per
// Lagrangian node, its 4x4x4 stencil split over the lanes (points q and q+32);
// a sphere's nodes are shared by IBM_SPLIT CTAs.  The interpolation reads the
// IBM macroscopic fields and the spreading adds into the auxiliary force field,
// two different arrays, so each node spreads right after its own
// interpolation, in the same warp.  Each CTA writes its sphere force/torque
// partial to fpart[sphere][split][6]; k_ibm_update adds the partials in a fixed
// order.
__global__ void __launch_bounds__(IBM_THREADS) k_ibm_interp_spread(IbmParams P, const DPart* parts, const double* X,
                                                                    const double* Y, const double* Z, const double* S,
                                                                    double* nfx, double* nfy, double* nfz, double* ndx,
                                                                    double* ndy, double* ndz, const float* fields,
                                                                    unsigned long long* faux, double* fpart,
                                                                    int split) {
    chain_enter();
    __shared__ double red[32];
    const int sphere = blockIdx.x / split, sub = blockIdx.x % split;
    const DPart& p = parts[sphere];
    const size_t N = (size_t)P.nx * P.ny * P.nz;
    const float* rho_g = fields;
    const float* ux_g = fields + N;
    const float* uy_g = fields + 2 * N;
    const float* uz_g = fields + 3 * N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = IBM_THREADS / 32;
    const double L[3] = {(double)P.nx, (double)P.ny, (double)P.nz};
    double accF[3] = {0, 0, 0}, accM[3] = {0, 0, 0};
    const int nb = p.node_count;
    for (int k = sub * warps + warp; k < nb; k += split * warps) {
        const int j = p.node_begin + k;
        const double xj = X[j], yj = Y[j], zj = Z[j];
        const NodeStencil st = node_stencil(P, p, xj, yj, zj);
        if (st.skip) {
            if (lane == 0) ndx[j] = ndy[j] = ndz[j] = 0.0;
            continue;
        }
        size_t g[2];
        float d[2];
        bool in[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int q = lane + 32 * h;
            const int xi = q & 3, yi = (q >> 2) & 3, zi = q >> 4;
            in[h] = xi >= st.lo[0] && xi <= st.hi[0] && yi >= st.lo[1] && yi <= st.hi[1] && zi >= st.lo[2] &&
                    zi <= st.hi[2];
            d[h] = (st.w[2][zi] * st.w[1][yi]) * st.w[0][xi];
            const int x = wrap_near(st.base[0] + xi, P.nx), y = wrap_near(st.base[1] + yi, P.ny),
                      z = wrap_near(st.base[2] + zi, P.nz);
            g[h] = ((size_t)z * P.ny + y) * P.nx + x;
        }
        float rho = 0.f, ux = 0.f, uy = 0.f, uz = 0.f;
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (in[h]) {
                rho += rho_g[g[h]] * d[h]; ux += ux_g[g[h]] * d[h];
                uy += uy_g[g[h]] * d[h]; uz += uz_g[g[h]] * d[h];
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rho += __shfl_xor_sync(0xffffffffu, rho, o);
            ux += __shfl_xor_sync(0xffffffffu, ux, o);
            uy += __shfl_xor_sync(0xffffffffu, uy, o);
            uz += __shfl_xor_sync(0xffffffffu, uz, o);
        }
        double dr[3] = {xj - p.pos[0], yj - p.pos[1], zj - p.pos[2]};
        for (int a = 0; a < 3; ++a)
            if (!P.wall[a]) dr[a] = pdelta(dr[a], L[a]);
        double uc[3] = {0, 0, 0};
        if (p.movable) {
            double wxr[3];
            dcross(p.w, dr, wxr);
            for (int a = 0; a < 3; ++a) uc[a] = p.vel[a] + wxr[a];
        }
        const double aux = 2.0 * (double)rho * S[j] * P.thickness;
        const double dF[3] = {aux * ((double)ux - uc[0]), aux * ((double)uy - uc[1]), aux * ((double)uz - uc[2])};
        if (lane == 0) {
            nfx[j] += dF[0]; nfy[j] += dF[1]; nfz[j] += dF[2];
            ndx[j] = dF[0]; ndy[j] = dF[1]; ndz[j] = dF[2];
            double m[3];
            dcross(dr, dF, m);
            for (int a = 0; a < 3; ++a) { accF[a] += dF[a]; accM[a] += m[a]; }
        }
        // spreading: fAux -= dF * delta (ibm.cu:478-512), in fixed point so the
        // sum is the same in any order
        const float f0 = (float)dF[0], f1 = (float)dF[1], f2 = (float)dF[2];
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (in[h]) {
                atomicAdd(&faux[g[h]], to_fix(-f0 * d[h]));
                atomicAdd(&faux[N + g[h]], to_fix(-f1 * d[h]));
                atomicAdd(&faux[2 * N + g[h]], to_fix(-f2 * d[h]));
            }
    }
    // this CTA's part of the sphere force and torque (ibm.cu:526-541)
    double tot6[6];
    for (int a = 0; a < 3; ++a) { tot6[a] = block_sum(accF[a], red); tot6[3 + a] = block_sum(accM[a], red); }
    if (threadIdx.x == 0)
        for (int a = 0; a < 6; ++a) fpart[((size_t)sphere * split + sub) * 6 + a] = tot6[a];
}

// gpuParticleMovement ibm.cu:899-993
__device__ void move_particle(const IbmParams& P, DPart& p) {
    if (!p.movable) return;
    const double L[3] = {(double)P.nx, (double)P.ny, (double)P.nz};
    for (int a = 0; a < 3; ++a) {
        const double dx = p.vel[a] * P.alpha + p.vel_old[a] * (1.0 - P.alpha);
        if (P.wall[a]) p.pos[a] += dx;
        else p.pos[a] = fmod(p.pos[a] + dx + L[a], L[a]);
        p.w_avg[a] = p.w[a] * P.alpha + p.w_old[a] * (1.0 - P.alpha);
        p.w_pos[a] += p.w_avg[a];
    }
}

// Sphere force/torque partials added in a fixed order, velocity and rotation
// update; after the last forcing iteration also the particle movement
// (gpuParticleMovement ibm.cu:899-993) and the step clock.
__global__ void k_ibm_update(IbmParams P, DPart* parts, const double* fpart, int split, int last, int* clock) {
    chain_enter();
    // one warp per sphere: lane l adds partials l, l + 32, ..., then a fixed
    // shuffle tree adds the lanes (the same order in every run)
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < P.np; i += gridDim.x * wpb) {
        DPart& p = parts[i];
        double t[6] = {0, 0, 0, 0, 0, 0};
        for (int b = lane; b < split; b += 32)
            for (int a = 0; a < 6; ++a) t[a] += fpart[((size_t)i * split + b) * 6 + a];
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t[a] += __shfl_down_sync(0xffffffffu, t[a], o);
        if (lane == 0) {
            for (int a = 0; a < 3; ++a) { p.f[a] += t[a]; p.M[a] += t[3 + a]; }
            update_center(P, p);
            if (last) move_particle(P, p);
        }
    }
    if (last && blockIdx.x == 0 && threadIdx.x == 0) *clock += 1;   // read by the next step's contacts
}

// gpuParticleNodeMovement ibm.cu:1044-1197
__device__ void move_node(const IbmParams& P, const DPart* parts, const int* pid, double* X, double* Y, double* Z,
                          int k) {
    const DPart& p = parts[pid[k]];
    if (!p.movable) return;
    const double L[3] = {(double)P.nx, (double)P.ny, (double)P.nz};
    double* Pp[3] = {&X[k], &Y[k], &Z[k]};
    const double wn = sqrt(p.w_avg[0] * p.w_avg[0] + p.w_avg[1] * p.w_avg[1] + p.w_avg[2] * p.w_avg[2]);
    if (wn <= 1e-8) {
        for (int a = 0; a < 3; ++a) {
            double d = p.pos[a] - p.pos_old[a];
            if (P.wall[a]) { *Pp[a] += d; continue; }
            if (fabs(d) > L[a] / 2.0) d = (p.pos[a] < p.pos_old[a]) ? p.pos[a] + L[a] - p.pos_old[a] : p.pos[a] - L[a] - p.pos_old[a];
            *Pp[a] = fmod(*Pp[a] + d + L[a], L[a]);
        }
        return;
    }
    double v[3];
    for (int a = 0; a < 3; ++a) {
        if (!P.wall[a] && fabs(*Pp[a] - p.pos_old[a]) > L[a] / 2.0) *Pp[a] += (*Pp[a] < p.pos_old[a]) ? L[a] : -L[a];
        v[a] = *Pp[a] - p.pos_old[a];
    }
    const double q0 = cos(0.5 * wn);
    const double qi = (p.w_avg[0] / wn) * sin(0.5 * wn), qj = (p.w_avg[1] / wn) * sin(0.5 * wn),
                 qk = (p.w_avg[2] / wn) * sin(0.5 * wn);
    const double t = q0 * q0 - 0.5;
    // rows as the reference writes them (third row: qi*qj - q0*qj, ibm.cu:1172)
    double np3[3];
    np3[0] = p.pos[0] + 2 * ((t + qi * qi) * v[0] + (qi * qj - q0 * qk) * v[1] + (qi * qk + q0 * qj) * v[2]);
    np3[1] = p.pos[1] + 2 * ((qi * qj + q0 * qk) * v[0] + (t + qj * qj) * v[1] + (qj * qk - q0 * qi) * v[2]);
    np3[2] = p.pos[2] + 2 * ((qi * qj - q0 * qj) * v[0] + (qj * qk + q0 * qi) * v[1] + (t + qk * qk) * v[2]);
    for (int a = 0; a < 3; ++a) *Pp[a] = P.wall[a] ? np3[a] : fmod(np3[a] + L[a], L[a]);
}

// Over the spheres' boxes, each node once (by the sphere owner[] names):
// u += fAux/(2 rho), F += fAux, fAux = 0 (gpuEulerSumIBMAuxsReset, restricted
// to the boxes); nodes that received no spread force are left as they are.
// After the last forcing iteration the same launch moves the Lagrangian nodes
// (gpuParticleNodeMovement ibm.cu:1044-1197), which k_ibm_update's particle
// movement precedes, and releases the owners.  `split` CTAs per sphere.
__global__ void __launch_bounds__(IBM_THREADS) k_ibm_euler(IbmParams P, float* fields, unsigned long long* faux,
                                                            float* fibm, uint8_t* cls, unsigned* owner,
                                                            const DPart* parts, const int* pid, double* X, double* Y,
                                                            double* Z, int split, int last) {
    chain_enter();
    const size_t N = (size_t)P.nx * P.ny * P.nz;
    if (last)
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P.nnodes; k += gridDim.x * blockDim.x)
            move_node(P, parts, pid, X, Y, Z, k);
    const unsigned sphere = blockIdx.x / split;
    const DPart& p = parts[sphere];
    const int sub = blockIdx.x % split;
    const unsigned tot = box_size(p);
    for (unsigned k = sub * blockDim.x + threadIdx.x; k < tot; k += split * blockDim.x) {
        const unsigned n = box_node(P, p, k);
        if (owner[n] != sphere) continue;
        if (last) owner[n] = IBM_NO_OWNER;
        const unsigned long long a0 = faux[n], a1 = faux[N + n], a2 = faux[2 * N + n];
        if ((a0 | a1 | a2) == 0ull) continue;
        const float rho = fields[n];
        const unsigned long long av[3] = {a0, a1, a2};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float v = from_fix(av[a]);
            fields[(1 + a) * N + n] += 0.5f * v / rho;
            fibm[a * N + n] += v;
            faux[a * N + n] = 0ull;
        }
        cls[n] = cls[n] | NODE_IBM_FORCE;
    }
}

// The IBM macroscopics of this step's box nodes into the caller's arrays.
__global__ void __launch_bounds__(IBM_THREADS) k_ibm_fixup(IbmParams P, const DPart* parts, const float* fields,
                                                            int split, float* rho, float* ux, float* uy, float* uz) {
    const size_t N = (size_t)P.nx * P.ny * P.nz;
    const DPart& p = parts[blockIdx.x / split];
    const int sub = blockIdx.x % split;
    const unsigned tot = box_size(p);
    for (unsigned k = sub * blockDim.x + threadIdx.x; k < tot; k += split * blockDim.x) {
        const unsigned n = box_node(P, p, k);
        if (rho) rho[n] = fields[n];
        if (ux) ux[n] = fields[N + n];
        if (uy) uy[n] = fields[2 * N + n];
        if (uz) uz[n] = fields[3 * N + n];
    }
}

// ---------------------------------------------------------------- host --
static void host_mesh(double diameter, double mesh_scale, double breugem, std::vector<double>& px,
                      std::vector<double>& py, std::vector<double>& pz, std::vector<double>& pS) {
    // Particle::makeSpherePolar (IBM/structs/particle.cpp:698-995), no Coulomb step
    const double r = diameter / 2.0 - breugem;
    const unsigned nLayer = (unsigned)(2.0 * std::sqrt(2.0) * r / mesh_scale + 1.0);
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
    for (unsigned i = 0; i <= nLayer; ++i) S[i] *= 2 * M_PI * r;
    for (unsigned i = nLayer; i > 0; --i) S[i] -= S[i - 1];
    S[0] = S[nLayer];
    px.assign(total, 0); py.assign(total, 0); pz.assign(total, 0); pS.assign(total, 0);
    pz[0] = r * std::sin(theta[0]);
    pS[0] = S[0];
    unsigned k = 1;
    double phase = 0.0;
    for (unsigned i = 1; i < nLayer; ++i) {
        if (i % 2 == 1) phase += M_PI / nl[i];
        for (unsigned j = 0; j < nl[i]; ++j, ++k) {
            const double a = (double)j * 2.0 * M_PI / nl[i] + phase;
            px[k] = r * std::cos(theta[i]) * std::cos(a);
            py[k] = r * std::cos(theta[i]) * std::sin(a);
            pz[k] = r * std::sin(theta[i]);
            pS[k] = S[i] / nl[i];
        }
    }
    pz[total - 1] = r * std::sin(theta[nLayer]);
    pS[total - 1] = S[nLayer];
}

#define IBM_CUDA(call)                                          \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_status(e_, #call);   \
    } while (0)

// A launch of the IBM chain (chain_enter): programmatic stream serialisation.
template <typename... KArgs, typename... Args>
static cudaError_t launch_chained(void (*kernel)(KArgs...), unsigned grid, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(IBM_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <int Q, int ST>
static cudaError_t launch_gather(vlbm_sim* s, IbmState* st) {
    const StepParams sp = make_params(s);
    const bool pr = sp.pairH > 0;
    if (s->parity == 1) {
        if (pr) return launch_chained(k_ibm_gather<Q, ST, true, true>, st->np * st->gsplit, s->stream, sp, st->prm, (const DPart*)st->parts, st->fields, st->owner, st->gsplit);
        else return launch_chained(k_ibm_gather<Q, ST, true, false>, st->np * st->gsplit, s->stream, sp, st->prm, (const DPart*)st->parts, st->fields, st->owner, st->gsplit);
    } else {
        if (pr) return launch_chained(k_ibm_gather<Q, ST, false, true>, st->np * st->gsplit, s->stream, sp, st->prm, (const DPart*)st->parts, st->fields, st->owner, st->gsplit);
        else return launch_chained(k_ibm_gather<Q, ST, false, false>, st->np * st->gsplit, s->stream, sp, st->prm, (const DPart*)st->parts, st->fields, st->owner, st->gsplit);
    }
    return cudaGetLastError();
}

static cudaError_t gather_dispatch(vlbm_sim* s, IbmState* st) {
    const int sto = s->cfg.storage;
    if (s->Q == 19) {
        if (sto == VLBM_STORE_F32) return launch_gather<19, VLBM_STORE_F32>(s, st);
        if (sto == VLBM_STORE_F16) return launch_gather<19, VLBM_STORE_F16>(s, st);
        return launch_gather<19, VLBM_STORE_BF16>(s, st);
    }
    if (sto == VLBM_STORE_F32) return launch_gather<27, VLBM_STORE_F32>(s, st);
    if (sto == VLBM_STORE_F16) return launch_gather<27, VLBM_STORE_F16>(s, st);
    return launch_gather<27, VLBM_STORE_BF16>(s, st);
}

vlbm_status ibm_step(vlbm_sim* s) {
    IbmState* st = s->ibm;
    if (!st || st->np == 0) return VLBM_OK;
    const IbmParams& P = st->prm;
    cudaStream_t cs = s->stream;
    // contacts on the IBM state's stream, beside the boxes and the gather
    IBM_CUDA(cudaEventRecord(st->ev_fork, cs));
    IBM_CUDA(cudaStreamWaitEvent(st->cstream, st->ev_fork, 0));
    k_ibm_begin<<<1, IBM_THREADS, 0, st->cstream>>>(P, st->parts, st->nx, st->ny, st->nz, st->nfx, st->nfy, st->nfz,
                                                     st->ndx, st->ndy, st->ndz, st->contrib, st->clock, 1);
    IBM_CUDA(cudaGetLastError());
    IBM_CUDA(cudaEventRecord(st->ev_join, st->cstream));
    k_ibm_begin<<<st->np, IBM_THREADS, 0, cs>>>(P, st->parts, st->nx, st->ny, st->nz, st->nfx, st->nfy, st->nfz,
                                                 st->ndx, st->ndy, st->ndz, st->contrib, st->clock, 0);
    IBM_CUDA(cudaGetLastError());
    IBM_CUDA(gather_dispatch(s, st));
    IBM_CUDA(cudaStreamWaitEvent(cs, st->ev_join, 0));   // the predictor before the first interpolation
    // the rest of the chain: programmatic dependents (chain_enter)
    const int iters = std::max(1, st->cfg.max_iterations);
    for (int it = 0; it < iters; ++it) {
        const int last = it == iters - 1;
        IBM_CUDA(launch_chained(k_ibm_interp_spread, st->np * st->split, cs, P, (const DPart*)st->parts,
                                (const double*)st->nx, (const double*)st->ny, (const double*)st->nz,
                                (const double*)st->nS, st->nfx, st->nfy, st->nfz, st->ndx, st->ndy, st->ndz,
                                (const float*)st->fields, st->faux, st->fpart, st->split));
        IBM_CUDA(launch_chained(k_ibm_update, (st->np + IBM_THREADS / 32 - 1) / (IBM_THREADS / 32), cs, P, st->parts,
                                (const double*)st->fpart, st->split, last, st->clock));
        IBM_CUDA(launch_chained(k_ibm_euler, st->np * st->gsplit, cs, P, st->fields, st->faux, s->fibm, s->cls,
                                st->owner, (const DPart*)st->parts, (const int*)st->npid, st->nx, st->ny, st->nz,
                                st->gsplit, last));
    }
    return VLBM_OK;
}

int ibm_iterations(const vlbm_sim* s) { return s->ibm ? s->ibm->cfg.max_iterations : 0; }

std::string ibm_info_section(const vlbm_sim* s) {
    const IbmState* st = s->ibm;
    if (!st || st->np == 0) return "";
    const vlbm_ibm_config& c = st->cfg;
    char b[2048];
    const int w = std::snprintf(
        b, sizeof(b),
        "\n------------------------------------- IBM --------------------------------------\n"
        "   Number of particles: %d\n"
        "        IBM iterations: %d\n"
        "          Stencil size: %d\n"
        "         Fluid density: %e\n"
        "                    GX: %e\n"
        "                    GY: %e\n"
        "                    GZ: %e\n"
        "            Mesh scale: %.2f\n"
        "         IBM thickness: %.2f\n"
        " IBM Breugem parameter: %.2f\n"
        " IBM Movement Disctre.: %.2f\n"
        "--------------------------------- IBM Collision --------------------------------\n"
        "\tPart-Part Frict Coef.: %.2f\n"
        "\tPart-Wall Frict Coef.: %.2f\n"
        "\tPart-Part Rest. Coef.: %.2f\n"
        "\tPart-Wall Rest. Coef.: %.2f\n"
        "\tParticle Young's Mod.: %.2f\n"
        "\tParticle Poisson Rat.: %.2f\n"
        "\t    Wall Young's Mod.: %.2f\n"
        "\t    Wall Poisson Rat.: %.2f\n"
        "--------------------------------- IBM Boundary Conditions ----------------------\n"
        "\t        IBM BC. X-Dir: %s \n"
        "\t        IBM BC. Y-Dir: %s \n"
        "\t        IBM BC. Z-Dir: %s \n"
        "--------------------------------------------------------------------------------\n",
        st->np, c.max_iterations, c.stencil, c.fluid_density, c.gx, c.gy, c.gz, c.mesh_scale, c.thickness,
        c.breugem, c.movement_alpha, c.pp_friction, c.pw_friction, c.pp_restitution, c.pw_restitution,
        c.particle_young, c.particle_poisson, c.wall_young, c.wall_poisson, c.wall_x ? "Wall" : "Periodic",
        c.wall_y ? "Wall" : "Periodic", c.wall_z ? "Wall" : "Periodic");
    return std::string(b, w > 0 ? (size_t)std::min(w, (int)sizeof(b) - 1) : 0);
}

uint32_t ibm_record_bytes() { return (uint32_t)sizeof(DPart); }

// The IBM state that carries from one step to the next: particle records
// (positions, velocities, rotation, forces of the previous step, contact
// history, the boxes of the step taken), Lagrangian nodes, the IBM
// macroscopics, and the step clock.  Per-step scratch (spread accumulators,
// box owners, pair and per-CTA partials) is zero, IBM_NO_OWNER or rewritten
// before it is read, so it is not saved.
void ibm_state_regions(vlbm_sim* s, std::vector<StateRegion>& out) {
    IbmState* st = s->ibm;
    if (!st || st->np == 0) return;
    const size_t nn = (size_t)st->nnodes, N = (size_t)s->N;
    out.push_back({100, st->parts, (size_t)st->np * sizeof(DPart)});
    uint32_t id = 101;
    for (double* p : {st->nx, st->ny, st->nz, st->nS, st->nfx, st->nfy, st->nfz, st->ndx, st->ndy, st->ndz})
        out.push_back({id++, p, nn * sizeof(double)});
    out.push_back({111, st->npid, nn * sizeof(int)});
    out.push_back({112, st->fields, 4 * N * sizeof(float)});
    out.push_back({114, st->clock, sizeof(int)});
}

void ibm_counts(const vlbm_sim* s, int* np, int* nn) {
    *np = s->ibm ? s->ibm->np : 0;
    *nn = s->ibm ? s->ibm->nnodes : 0;
}

vlbm_status ibm_macroscopics_fixup(vlbm_sim* s, float* rho, float* ux, float* uy, float* uz) {
    IbmState* st = s->ibm;
    if (!st || st->np == 0 || s->step == 0) return VLBM_OK;
    k_ibm_fixup<<<st->np * st->gsplit, IBM_THREADS, 0, s->stream>>>(st->prm, st->parts, st->fields, st->gsplit, rho,
                                                                    ux, uy, uz);
    return cuda_status(cudaGetLastError(), "ibm macroscopics fixup");
}

void ibm_destroy(IbmState* st, DeviceAllocator* a) {
    if (!st) return;
    free_with(a, st->parts);
    for (double* p : {st->nx, st->ny, st->nz, st->nS, st->nfx, st->nfy, st->nfz, st->ndx, st->ndy, st->ndz, st->contrib,
                      st->fpart})
        free_with(a, p);
    free_with(a, st->npid); free_with(a, st->fields); free_with(a, st->faux); free_with(a, st->owner);
    free_with(a, st->clock);
    if (st->ev_fork) cudaEventDestroy(st->ev_fork);
    if (st->ev_join) cudaEventDestroy(st->ev_join);
    if (st->cstream) cudaStreamDestroy(st->cstream);
    delete st;
}

void ibm_reset(vlbm_sim* s) {
    IbmState* st = s->ibm;
    if (!st) return;
    cudaMemcpyAsync(st->parts, st->initial.data(), st->initial.size() * sizeof(DPart), cudaMemcpyHostToDevice, s->stream);
    const size_t nn = (size_t)st->nnodes;
    cudaMemcpyAsync(st->nx, st->init_nodes.data(), nn * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(st->ny, st->init_nodes.data() + nn, nn * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(st->nz, st->init_nodes.data() + 2 * nn, nn * sizeof(double), cudaMemcpyHostToDevice, s->stream);
    cudaMemsetAsync(st->fields, 0, (size_t)4 * s->N * sizeof(float), s->stream);
    cudaMemsetAsync(st->faux, 0, (size_t)3 * s->N * sizeof(unsigned long long), s->stream);
    cudaMemsetAsync(st->owner, 0xFF, (size_t)s->N * sizeof(unsigned), s->stream);   // IBM_NO_OWNER
    cudaMemsetAsync(st->clock, 0, sizeof(int), s->stream);
}

}  // namespace vlbm

using namespace vlbm;

extern "C" {

vlbm_status vlbm_ibm_config_default(vlbm_ibm_config* c) {
    if (!c) return VLBM_ERR_INVALID;
    std::memset(c, 0, sizeof(*c));
    c->max_iterations = 1;       // ibmVar.h:23 IBM_MAX_ITERATION
    c->stencil = 4;              // ibmVar.h:136 STENCIL_4
    c->thickness = 1.0;          // ibmVar.h:33 IBM_THICKNESS
    c->movement_alpha = 0.5;     // ibmVar.h:95 IBM_MOVEMENT_DISCRETIZATION
    c->fluid_density = 1.0;      // ibmVar.h:110 FLUID_DENSITY
    c->gx = 0.0; c->gy = 0.0; c->gz = -5e-5;  // ibmVar.h:113-115
    c->wall_x = 0; c->wall_y = 1; c->wall_z = 0;  // ibmBoundaryCondition.h:20-56
    c->pp_friction = 0.1; c->pw_friction = 0.1;   // ibmBoundaryCondition.h:85-86
    c->pp_restitution = 0.9; c->pw_restitution = 0.9;  // ibmBoundaryCondition.h:87-88
    c->particle_young = 0.5; c->particle_poisson = 0.3;  // ibmBoundaryCondition.h:93-94
    c->wall_young = 100.0; c->wall_poisson = 0.3;        // ibmBoundaryCondition.h:97-98
    c->mesh_scale = 1.0;         // ibmVar.h:29 MESH_SCALE
    c->breugem = 0.0;            // ibmVar.h:27 BREUGEM_PARAMETER
    return VLBM_OK;
}

vlbm_status vlbm_add_spheres(vlbm_sim* s, const vlbm_ibm_config* ib, const vlbm_sphere* sp, int32_t n) {
    if (!s || !ib || (n > 0 && !sp)) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    IBM_CUDA(cudaSetDevice(s->device));
    if (s->ibm) { set_last_error("spheres were already added to this simulation"); return VLBM_ERR_STATE; }
    if (n <= 0 || n > IBM_MAX_PARTICLES) { set_last_error("sphere count must be in 1..1024"); return VLBM_ERR_INVALID; }
    if (s->cfg.slab_nz_total != 0) {
        set_last_error("spheres are not supported on a z-slab (the IBM step runs on whole lattices)");
        return VLBM_ERR_UNSUPPORTED;
    }
    if (ib->stencil != 4) {
        set_last_error("only the Peskin 4-point stencil (STENCIL_4) is supported");
        return VLBM_ERR_UNSUPPORTED;
    }
    if (ib->max_iterations < 1 || !(ib->mesh_scale > 0)) { set_last_error("max_iterations >= 1 and mesh_scale > 0 required"); return VLBM_ERR_INVALID; }
    IbmState* st = new IbmState();
    st->cfg = *ib;
    const vlbm_config& c = s->cfg;
    IbmParams& P = st->prm;
    P.np = n;
    P.nx = c.nx; P.ny = c.ny; P.nz = c.nz;
    P.wall[0] = ib->wall_x; P.wall[1] = ib->wall_y; P.wall[2] = ib->wall_z;
    P.alpha = ib->movement_alpha;
    P.rho_f = ib->fluid_density;
    P.g[0] = ib->gx; P.g[1] = ib->gy; P.g[2] = ib->gz;
    P.thickness = ib->thickness;
    {   // contact constants, ibmBoundaryCondition.h:93-107 and the damping factor of :441
        const double Gp = ib->particle_young / (2.0 + 2.0 * ib->particle_poisson);
        const double Gw = ib->wall_young / (2.0 + 2.0 * ib->wall_poisson);
        const double np2 = ib->particle_poisson * ib->particle_poisson, nw2 = ib->wall_poisson * ib->wall_poisson;
        P.ss_n = (4.0 / 3.0) / ((1 - np2) / ib->particle_young + (1 - np2) / ib->particle_young);
        P.sw_n = (4.0 / 3.0) / ((1 - np2) / ib->particle_young + (1 - nw2) / ib->wall_young);
        P.ss_t = 4.0 * std::sqrt(2.0) / ((2 - ib->particle_poisson) / Gp + (2 - ib->particle_poisson) / Gp);
        P.sw_t = 4.0 * std::sqrt(2.0) / ((2 - ib->particle_poisson) / Gp + (2 - ib->wall_poisson) / Gw);
        const double lpp = std::log(ib->pp_restitution), lpw = std::log(ib->pw_restitution);
        P.dpp = -2.0 * lpp / std::sqrt(M_PI * M_PI + lpp * lpp);
        P.dpw = -2.0 * lpw / std::sqrt(M_PI * M_PI + lpw * lpw);
        P.mu_pp = ib->pp_friction;
        P.mu_pw = ib->pw_friction;
    }
    P.fx = (float)c.fx; P.fy = (float)c.fy; P.fz = (float)c.fz;
    std::vector<DPart> parts(n);
    std::vector<double> X, Y, Z, S;
    std::vector<int> pid;
    for (int k = 0; k < n; ++k) {
        DPart& p = parts[k];
        std::memset(&p, 0, sizeof(p));
        const double r = sp[k].diameter / 2.0;
        p.radius = r;
        p.volume = r * r * r * 4 * M_PI / 3;
        p.S = 4.0 * M_PI * r * r;
        p.density = sp[k].density;
        const double cc[3] = {sp[k].cx, sp[k].cy, sp[k].cz}, v[3] = {sp[k].vx, sp[k].vy, sp[k].vz},
                     w[3] = {sp[k].wx, sp[k].wy, sp[k].wz};
        for (int a = 0; a < 3; ++a) {
            p.pos[a] = p.pos_old[a] = cc[a];
            p.vel[a] = p.vel_old[a] = v[a];
            p.w[a] = p.w_avg[a] = p.w_old[a] = w[a];
        }
        p.I[0] = p.I[1] = p.I[2] = 2.0 * p.volume * p.density * r * r / 5.0;  // particle.cpp:745-751
        p.movable = sp[k].movable;
        for (int i = 0; i < IBM_MAX_SLOTS; ++i) { p.partner[i] = -1; p.last[i] = -1; }
        std::vector<double> px, py, pz, pS;
        host_mesh(sp[k].diameter, ib->mesh_scale, ib->breugem, px, py, pz, pS);
        p.node_begin = (int)X.size();
        p.node_count = (int)px.size();
        for (size_t j = 0; j < px.size(); ++j) {
            X.push_back(px[j] + cc[0]); Y.push_back(py[j] + cc[1]); Z.push_back(pz[j] + cc[2]);
            S.push_back(pS[j]);
            pid.push_back(k);
        }
    }
    st->np = n;
    st->nnodes = (int)X.size();
    P.nnodes = st->nnodes;
    const size_t nn = X.size(), N = (size_t)s->N;
    auto dalloc = [&](void** p, size_t b) -> cudaError_t {
        cudaError_t e = sim_malloc(s, p, b);
        if (e == cudaSuccess) st->bytes += b;
        return e;
    };
    cudaError_t e = dalloc((void**)&st->parts, parts.size() * sizeof(DPart));
    double** dp[] = {&st->nx, &st->ny, &st->nz, &st->nS, &st->nfx, &st->nfy, &st->nfz, &st->ndx, &st->ndy, &st->ndz};
    for (double** d : dp)
        if (e == cudaSuccess) e = dalloc((void**)d, nn * sizeof(double));
    if (e == cudaSuccess) e = dalloc((void**)&st->npid, nn * sizeof(int));
    if (e == cudaSuccess) e = dalloc((void**)&st->fields, 4 * N * sizeof(float));
    if (e == cudaSuccess) e = dalloc((void**)&st->faux, 3 * N * sizeof(unsigned long long));
    if (e == cudaSuccess) e = dalloc((void**)&st->owner, N * sizeof(unsigned));
    if (e == cudaSuccess) e = dalloc((void**)&st->clock, sizeof(int));
    if (e == cudaSuccess) e = dalloc((void**)&st->contrib, (size_t)n * n * 6 * sizeof(double));
    {   // CTAs per sphere of the interpolation/spreading kernel: about
        // IBM_NODES_PER_CTA Lagrangian nodes each for the largest sphere
        std::vector<int> cnt(n, 0);
        for (int pk : pid) cnt[pk] += 1;
        int most = 1;
        for (int c : cnt) most = std::max(most, c);
        st->split = std::min(IBM_MAX_SPLIT, std::max(1, (most + IBM_NODES_PER_CTA - 1) / IBM_NODES_PER_CTA));
    }
    if (e == cudaSuccess) e = dalloc((void**)&st->fpart, (size_t)n * st->split * 6 * sizeof(double));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st->cstream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->ev_join, cudaEventDisableTiming);
    {   // CTAs per sphere of the box passes: about two box nodes per thread for the largest sphere
        long long maxbox = 1;
        for (int k = 0; k < n; ++k) {
            const long long side = (long long)std::ceil(sp[k].diameter) + 6;
            maxbox = std::max(maxbox, std::min<long long>(side, c.nx) * std::min<long long>(side, c.ny) *
                                          std::min<long long>(side, c.nz));
        }
        st->gsplit = (int)std::min<long long>(IBM_MAX_SPLIT, std::max<long long>(1, maxbox / (2 * IBM_THREADS)));
    }
    if (e == cudaSuccess && !s->fibm) {
        e = sim_malloc(s, (void**)&s->fibm, 3 * N * sizeof(float));
        if (e == cudaSuccess) s->device_bytes += 3 * N * sizeof(float);
    }
    if (e != cudaSuccess) { ibm_destroy(st, s->allocator); return cuda_status(e, "IBM allocation"); }
    // uploads and clears on the simulation's stream; a simulation set up
    // without host waits (a server admitting it while its batch work runs)
    // uploads from pinned staging and leaves the work queued
    const cudaStream_t ss = s->stream;
    const int clock = (int)s->step;   // the contact history clock starts at the lattice's step count
    e = sim_upload(s, st->parts, parts.data(), parts.size() * sizeof(DPart));
    if (e == cudaSuccess) e = sim_upload(s, st->nx, X.data(), nn * sizeof(double));
    if (e == cudaSuccess) e = sim_upload(s, st->ny, Y.data(), nn * sizeof(double));
    if (e == cudaSuccess) e = sim_upload(s, st->nz, Z.data(), nn * sizeof(double));
    if (e == cudaSuccess) e = sim_upload(s, st->nS, S.data(), nn * sizeof(double));
    if (e == cudaSuccess) e = sim_upload(s, st->npid, pid.data(), nn * sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(st->fields, 0, 4 * N * sizeof(float), ss);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->faux, 0, 3 * N * sizeof(unsigned long long), ss);
    if (e == cudaSuccess) e = cudaMemsetAsync(st->owner, 0xFF, N * sizeof(unsigned), ss);   // IBM_NO_OWNER
    if (e == cudaSuccess) e = sim_upload(s, st->clock, &clock, sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->fibm, 0, 3 * N * sizeof(float), ss);
    if (e == cudaSuccess && !s->async_setup) e = cudaStreamSynchronize(ss);   // the host vectors go out of scope
    if (e != cudaSuccess) { ibm_destroy(st, s->allocator); return cuda_status(e, "IBM setup"); }
    st->initial = parts;
    st->init_nodes.resize(3 * nn);
    std::memcpy(st->init_nodes.data(), X.data(), nn * sizeof(double));
    std::memcpy(st->init_nodes.data() + nn, Y.data(), nn * sizeof(double));
    std::memcpy(st->init_nodes.data() + 2 * nn, Z.data(), nn * sizeof(double));
    s->device_bytes += st->bytes;
    s->ibm = st;
    return VLBM_OK;
}

vlbm_status vlbm_get_particles(vlbm_sim* s, vlbm_particle_state* out, int32_t n) {
    if (!s || !out) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    if (!s->ibm) { set_last_error("no spheres in this simulation"); return VLBM_ERR_STATE; }
    IBM_CUDA(cudaSetDevice(s->device));
    IbmState* st = s->ibm;
    std::vector<DPart> h(st->np);
    IBM_CUDA(cudaMemcpyAsync(h.data(), st->parts, h.size() * sizeof(DPart), cudaMemcpyDeviceToHost, s->stream));
    IBM_CUDA(cudaStreamSynchronize(s->stream));
    for (int k = 0; k < n && k < st->np; ++k) {
        const DPart& p = h[k];
        vlbm_particle_state& o = out[k];
        std::memset(&o, 0, sizeof(o));
        for (int a = 0; a < 3; ++a) {
            o.pos[a] = p.pos[a]; o.vel[a] = p.vel[a]; o.w[a] = p.w[a]; o.f[a] = p.f[a]; o.M[a] = p.M[a];
            o.pos_old[a] = p.pos_old[a]; o.vel_old[a] = p.vel_old[a]; o.w_old[a] = p.w_old[a];
            o.f_old[a] = p.f_old[a]; o.M_old[a] = p.M_old[a]; o.w_avg[a] = p.w_avg[a]; o.w_pos[a] = p.w_pos[a];
        }
        for (int a = 0; a < 6; ++a) o.I[a] = p.I[a];
        o.radius = p.radius; o.volume = p.volume; o.density = p.density; o.S = p.S;
        o.movable = p.movable; o.n_nodes = p.node_count;
    }
    return VLBM_OK;
}

vlbm_status vlbm_get_lagrangian_nodes(vlbm_sim* s, double* pos, double* force, size_t n) {
    if (!s) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    if (!s->ibm) { set_last_error("no spheres in this simulation"); return VLBM_ERR_STATE; }
    IbmState* st = s->ibm;
    if (n != (size_t)st->nnodes) { set_last_error("node count mismatch"); return VLBM_ERR_INVALID; }
    IBM_CUDA(cudaSetDevice(s->device));
    const size_t b = n * sizeof(double);
    if (pos) {
        IBM_CUDA(cudaMemcpyAsync(pos, st->nx, b, cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(pos + n, st->ny, b, cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(pos + 2 * n, st->nz, b, cudaMemcpyDeviceToHost, s->stream));
    }
    if (force) {
        IBM_CUDA(cudaMemcpyAsync(force, st->nfx, b, cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(force + n, st->nfy, b, cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(force + 2 * n, st->nfz, b, cudaMemcpyDeviceToHost, s->stream));
    }
    IBM_CUDA(cudaStreamSynchronize(s->stream));
    return VLBM_OK;
}

// saveParticlesInfo (IBM/ibmReport.cpp:26-102): the particle centres and,
// optionally, the Lagrangian nodes as CSV, numbers in std::scientific (%e).
// Spheres carry the collision semi-axes (r, r, r), (0, 0, 0), (0, 0, 0) of
// makeSpherePolar (particle.cpp:778).
vlbm_status vlbm_write_particles_csv(vlbm_sim* s, const char* path_files, const char* id_sim, uint32_t step_label,
                                     int32_t save_nodes) {
    if (!s || !path_files || !id_sim) { set_last_error("null argument"); return VLBM_ERR_INVALID; }
    if (!s->ibm) { set_last_error("no spheres in this simulation"); return VLBM_ERR_STATE; }
    IbmState* st = s->ibm;
    IBM_CUDA(cudaSetDevice(s->device));
    std::vector<DPart> h(st->np);
    IBM_CUDA(cudaMemcpyAsync(h.data(), st->parts, h.size() * sizeof(DPart), cudaMemcpyDeviceToHost, s->stream));
    const size_t nn = (size_t)st->nnodes;
    std::vector<double> px(nn), py(nn), pz(nn), pS(nn);
    std::vector<int> pid(nn);
    if (save_nodes) {
        IBM_CUDA(cudaMemcpyAsync(px.data(), st->nx, nn * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(py.data(), st->ny, nn * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(pz.data(), st->nz, nn * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(pS.data(), st->nS, nn * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        IBM_CUDA(cudaMemcpyAsync(pid.data(), st->npid, nn * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    }
    IBM_CUDA(cudaStreamSynchronize(s->stream));
    const std::string dir = std::string(path_files) + "/" + id_sim;
    mkdir_p(dir);
    const std::string stem = dir + "/" + id_sim + "_";
    const std::string num = step_field(step_label);
    {
        const std::string fn = stem + "pCenters" + num + ".csv";
        FILE* f = std::fopen(fn.c_str(), "w");
        if (!f) { set_last_error("cannot open " + fn); return VLBM_ERR_IO; }
        std::fprintf(f, "p_number,step,pos_x,pos_y,pos_z,vel_x,vel_y,vel_z,w_x,w_y,w_z,f_x,f_y,f_z,M_x,M_y,M_z,"
                        "I_xx,I_yy,I_zz,I_xy,I_xz,I_yz,S,radius,volume,movable,semi1x,semi1y,semi1z,"
                        "semi2x,semi2y,semi2z,semi3x,semi3y,semi3z\n");
        for (int k = 0; k < st->np; ++k) {
            const DPart& p = h[k];
            std::fprintf(f, "%d,%u", k, step_label);
            const double* v3[5] = {p.pos, p.vel, p.w, p.f, p.M};
            for (const double* v : v3) std::fprintf(f, ",%e,%e,%e", v[0], v[1], v[2]);
            for (int a = 0; a < 6; ++a) std::fprintf(f, ",%e", p.I[a]);
            std::fprintf(f, ",%e,%e,%e,%d", p.S, p.radius, p.volume, p.movable ? 1 : 0);
            std::fprintf(f, ",%e,%e,%e,%e,%e,%e,%e,%e,%e\n", p.radius, p.radius, p.radius, 0.0, 0.0, 0.0, 0.0,
                         0.0, 0.0);
        }
        const bool bad = std::ferror(f) != 0;
        std::fclose(f);
        if (bad) { set_last_error("write failed " + fn); return VLBM_ERR_IO; }
    }
    if (save_nodes) {
        const std::string fn = stem + "pNodes" + num + ".csv";
        FILE* f = std::fopen(fn.c_str(), "w");
        if (!f) { set_last_error("cannot open " + fn); return VLBM_ERR_IO; }
        std::fprintf(f, "particle_index,pos_x,pos_y,pos_z,S\n");
        for (size_t i = 0; i < nn; ++i) std::fprintf(f, "%d,%e,%e,%e,%e\n", pid[i], px[i], py[i], pz[i], pS[i]);
        const bool bad = std::ferror(f) != 0;
        std::fclose(f);
        if (bad) { set_last_error("write failed " + fn); return VLBM_ERR_IO; }
    }
    return VLBM_OK;
}

}  // extern "C"
