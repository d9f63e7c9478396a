// pair_math.cuh -- the fused step's arithmetic for two nodes at once.
//
// The z-paired kernel (k_step2) holds the nodes (x, y, z) and (x, y, z + NZ/2)
// in the two lanes of float2 values and evaluates moments, stress magnitude
// and collision with sm_100's packed FP32x2 instructions (FFMA2 / FADD2 /
// FMUL2: two FP32 operations per issued instruction).  The kernel is limited by
// instruction issue, not by HBM, so this halves the arithmetic's share of the
// issue slots.  The formulas are those of moments(), stress_aux() and
// collide() in step_impl.cuh, on deviations g_i = f_i - w_i rho0.
#pragma once
#include <cuda_runtime.h>
#include "internal.h"
#include "lattice.cuh"

namespace vlbm {

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float lane_of(const float2& v, int lane) { return lane ? v.y : v.x; }
__device__ __forceinline__ void set_lane(float2& v, int lane, float a) {
    if (lane) v.y = a; else v.x = a;
}

struct Mom2 {
    float2 rho, drho, ux, uy, uz;
    float2 pxx, pyy, pzz, pxy, pxz, pyz;
};

// SCALED: g holds the stored half-precision values, deviations times a power
// of two (1 / inv_scale); the ten sums are scaled back instead of the Q
// populations, which gives the same bits (a power-of-two scale is exact).
template <int Q, bool NEED_PI, bool SCALED = false>
__device__ __forceinline__ Mom2 moments2(const float2 (&g)[Q], float2 fx, float2 fy, float2 fz, float rho0,
                                         float inv_scale = 1.f) {
    Mom2 m;
    float2 rho = g[0], jx = f2(0.f), jy = f2(0.f), jz = f2(0.f);
    float2 sxx = f2(0.f), syy = f2(0.f), szz = f2(0.f), sxy = f2(0.f), sxz = f2(0.f), syz = f2(0.f);
#pragma unroll
    for (int i = 1; i < Q; i += 2) {
        const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
        const float2 e = add2(g[i], g[i + 1]), o = sub2(g[i], g[i + 1]);
        rho = add2(rho, e);
        if (cx > 0) jx = add2(jx, o); else if (cx < 0) jx = sub2(jx, o);
        if (cy > 0) jy = add2(jy, o); else if (cy < 0) jy = sub2(jy, o);
        if (cz > 0) jz = add2(jz, o); else if (cz < 0) jz = sub2(jz, o);
        if (NEED_PI) {
            if (cx) sxx = add2(sxx, e);
            if (cy) syy = add2(syy, e);
            if (cz) szz = add2(szz, e);
            if (cx && cy) sxy = (cx * cy > 0) ? add2(sxy, e) : sub2(sxy, e);
            if (cx && cz) sxz = (cx * cz > 0) ? add2(sxz, e) : sub2(sxz, e);
            if (cy && cz) syz = (cy * cz > 0) ? add2(syz, e) : sub2(syz, e);
        }
    }
    if (SCALED) {
        const float2 k = f2(inv_scale);
        rho = mul2(rho, k);
        jx = mul2(jx, k); jy = mul2(jy, k); jz = mul2(jz, k);
        if (NEED_PI) {
            sxx = mul2(sxx, k); syy = mul2(syy, k); szz = mul2(szz, k);
            sxy = mul2(sxy, k); sxz = mul2(sxz, k); syz = mul2(syz, k);
        }
    }
    m.drho = rho;
    rho = add2(rho, f2(rho0));
    m.rho = rho;
    const float2 inv = make_float2(__frcp_rn(rho.x), __frcp_rn(rho.y));
    m.ux = mul2(fma2(fx, f2(0.5f), jx), inv);
    m.uy = mul2(fma2(fy, f2(0.5f), jy), inv);
    m.uz = mul2(fma2(fz, f2(0.5f), jz), inv);
    if (NEED_PI) {
        const float2 rn = mul2(rho, f2(-1.f));
        const float2 rux = mul2(rn, m.ux), ruy = mul2(rn, m.uy), ruz = mul2(rn, m.uz);
        const float2 dr3 = mul2(m.drho, f2(1.f / 3.f));
        m.pxx = fma2(rux, m.ux, sub2(sxx, dr3));
        m.pyy = fma2(ruy, m.uy, sub2(syy, dr3));
        m.pzz = fma2(ruz, m.uz, sub2(szz, dr3));
        m.pxy = fma2(rux, m.uy, sxy);
        m.pxz = fma2(rux, m.uz, sxz);
        m.pyz = fma2(ruy, m.uz, syz);
    } else {
        m.pxx = m.pyy = m.pzz = m.pxy = m.pxz = m.pyz = f2(0.f);
    }
    return m;
}

// |S| of the regularized stress with the force correction, per lane
// (the formula of stress_aux()).
__device__ __forceinline__ float2 stress_aux2(const Mom2& m, float2 fx, float2 fy, float2 fz) {
    const float2 a = fma2(m.ux, fx, m.pxx), b = fma2(m.uy, fy, m.pyy), c = fma2(m.uz, fz, m.pzz);
    const float2 h = f2(0.5f);
    const float2 d = fma2(h, fma2(m.ux, fy, mul2(m.uy, fx)), m.pxy);
    const float2 e = fma2(h, fma2(m.ux, fz, mul2(m.uz, fx)), m.pxz);
    const float2 k = fma2(h, fma2(m.uy, fz, mul2(m.uz, fy)), m.pyz);
    const float2 off = fma2(d, d, fma2(e, e, mul2(k, k)));
    const float2 q = mul2(h, fma2(a, a, fma2(b, b, fma2(c, c, add2(off, off)))));
    return make_float2(q.x > 0.f ? q.x * rsqrtf(q.x) : 0.f, q.y > 0.f ? q.y * rsqrtf(q.y) : 0.f);
}

// Collision in place on deviations, both lanes (the formulas of collide()).
// `gscale` is what the incoming g must be multiplied by to be deviations
// (inv_scale for stored half values, 1 otherwise); the result is deviations
// times `oscale` (the storage scale for half storage, 1 otherwise).  Both are
// powers of two, folded into the weights and BGK's (1 - omega) factor, which
// gives the same bits as scaling before and after.
template <int Q, int OP>
__device__ __forceinline__ void collide2(float2 (&g)[Q], const Mom2& m, float2 omega, float2 fx, float2 fy,
                                         float2 fz, float gscale = 1.f, float oscale = 1.f) {
    const float2 B = fma2(omega, f2(-0.5f), f2(1.f));
    const float2 uu = fma2(m.ux, m.ux, fma2(m.uy, m.uy, mul2(m.uz, m.uz)));
    const float2 uF = fma2(m.ux, fx, fma2(m.uy, fy, mul2(m.uz, fz)));
    const float2 BuF = mul2(B, uF);
    if (OP == VLBM_OP_REGULARIZED) {
        const float2 A = fma2(omega, f2(-4.5f), f2(4.5f));
        const float2 tr = mul2(add2(add2(m.pxx, m.pyy), m.pzz), f2(1.f / 3.f));
        float2 K0 = fma2(mul2(m.rho, uu), f2(-1.5f), m.drho);
        K0 = fma2(BuF, f2(-3.f), K0);
        K0 = sub2(K0, mul2(A, tr));
        const float2 alpha = fma2(B, f2(3.f), mul2(A, f2(-1.f / 3.f)));
        const float2 r3 = mul2(m.rho, f2(3.f)), r45 = mul2(m.rho, f2(4.5f)), b9 = mul2(B, f2(9.f));
        const float2 pxy2 = add2(m.pxy, m.pxy), pxz2 = add2(m.pxz, m.pxz), pyz2 = add2(m.pyz, m.pyz);
        g[0] = mul2(f2(Lattice<Q>::w(0) * oscale), K0);
#pragma unroll
        for (int i = 1; i < Q; i += 2) {
            const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
            float2 S = f2(0.f), cu = f2(0.f), cF = f2(0.f);
            bool first = true;
            if (cx) { S = m.pxx; first = false; cu = cx > 0 ? m.ux : mul2(m.ux, f2(-1.f)); cF = cx > 0 ? fx : mul2(fx, f2(-1.f)); }
            if (cy) {
                S = first ? m.pyy : add2(S, m.pyy);
                cu = first ? (cy > 0 ? m.uy : mul2(m.uy, f2(-1.f))) : (cy > 0 ? add2(cu, m.uy) : sub2(cu, m.uy));
                cF = first ? (cy > 0 ? fy : mul2(fy, f2(-1.f))) : (cy > 0 ? add2(cF, fy) : sub2(cF, fy));
                first = false;
            }
            if (cz) {
                S = first ? m.pzz : add2(S, m.pzz);
                cu = first ? (cz > 0 ? m.uz : mul2(m.uz, f2(-1.f))) : (cz > 0 ? add2(cu, m.uz) : sub2(cu, m.uz));
                cF = first ? (cz > 0 ? fz : mul2(fz, f2(-1.f))) : (cz > 0 ? add2(cF, fz) : sub2(cF, fz));
            }
            if (cx && cy) S = (cx * cy > 0) ? add2(S, pxy2) : sub2(S, pxy2);
            if (cx && cz) S = (cx * cz > 0) ? add2(S, pxz2) : sub2(S, pxz2);
            if (cy && cz) S = (cy * cz > 0) ? add2(S, pyz2) : sub2(S, pyz2);
            const float2 E = fma2(cu, fma2(r45, cu, mul2(b9, cF)), fma2(A, S, K0));
            const float2 O = fma2(alpha, cF, mul2(r3, cu));
            const float2 w = f2(Lattice<Q>::w(i) * oscale);
            g[i] = mul2(w, add2(E, O));
            g[i + 1] = mul2(w, sub2(E, O));
        }
    } else {
        const float2 om1 = mul2(sub2(f2(1.f), omega), f2(gscale * oscale));
        const float2 base = fma2(omega, fma2(mul2(m.rho, uu), f2(-1.5f), m.drho), mul2(BuF, f2(-3.f)));
        const float2 orho = mul2(omega, m.rho);
        const float2 r45 = mul2(orho, f2(4.5f)), r3 = mul2(orho, f2(3.f)), b9 = mul2(B, f2(9.f)),
                     b3 = mul2(B, f2(3.f));
        g[0] = fma2(om1, g[0], mul2(f2(Lattice<Q>::w(0) * oscale), base));
#pragma unroll
        for (int i = 1; i < Q; i += 2) {
            const int cx = lat_cx(i), cy = lat_cy(i), cz = lat_cz(i);
            float2 cu = f2(0.f), cF = f2(0.f);
            bool first = true;
            if (cx) { cu = cx > 0 ? m.ux : mul2(m.ux, f2(-1.f)); cF = cx > 0 ? fx : mul2(fx, f2(-1.f)); first = false; }
            if (cy) {
                cu = first ? (cy > 0 ? m.uy : mul2(m.uy, f2(-1.f))) : (cy > 0 ? add2(cu, m.uy) : sub2(cu, m.uy));
                cF = first ? (cy > 0 ? fy : mul2(fy, f2(-1.f))) : (cy > 0 ? add2(cF, fy) : sub2(cF, fy));
                first = false;
            }
            if (cz) {
                cu = first ? (cz > 0 ? m.uz : mul2(m.uz, f2(-1.f))) : (cz > 0 ? add2(cu, m.uz) : sub2(cu, m.uz));
                cF = first ? (cz > 0 ? fz : mul2(fz, f2(-1.f))) : (cz > 0 ? add2(cF, fz) : sub2(cF, fz));
            }
            const float2 w = f2(Lattice<Q>::w(i) * oscale);
            const float2 E = mul2(w, fma2(cu, fma2(r45, cu, mul2(b9, cF)), base));
            const float2 O = mul2(w, fma2(r3, cu, mul2(b3, cF)));
            g[i] = fma2(om1, g[i], add2(E, O));
            g[i + 1] = fma2(om1, g[i + 1], sub2(E, O));
        }
    }
}

}  // namespace vlbm
