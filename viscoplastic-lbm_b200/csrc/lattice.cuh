// lattice.cuh -- D3Q19 / D3Q27 velocity sets as compile-time tables.
//
// Population order and weights are those of the reference
// (src/CUDA/velocitySets/D3Q19.h:6-46, D3Q27.h:6-56) so that population
// planes, node maps and outputs are interchangeable with it.  All loops over
// populations are unrolled, so every c_i / w_i below folds into immediates.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define VLBM_HD __host__ __device__ __forceinline__
#else
#define VLBM_HD inline
#endif

namespace vlbm {

VLBM_HD constexpr int lat_cx(int i) {
    constexpr int v[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
    return v[i];
}
VLBM_HD constexpr int lat_cy(int i) {
    constexpr int v[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
    return v[i];
}
VLBM_HD constexpr int lat_cz(int i) {
    constexpr int v[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
    return v[i];
}
// Opposite population: in this ordering populations come in (+c, -c) pairs
// 1/2, 3/4, ..., 25/26.
VLBM_HD constexpr int lat_opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
VLBM_HD constexpr int lat_norm1(int i) {
    return (lat_cx(i) != 0) + (lat_cy(i) != 0) + (lat_cz(i) != 0);
}

template <int Q> struct Lattice;

template <> struct Lattice<19> {
    static constexpr int Q = 19;
    VLBM_HD static constexpr float w(int i) {
        return lat_norm1(i) == 0 ? 1.0f / 3.0f : (lat_norm1(i) == 1 ? 1.0f / 18.0f : 1.0f / 36.0f);
    }
    VLBM_HD static constexpr double wd(int i) {
        return lat_norm1(i) == 0 ? 1.0 / 3.0 : (lat_norm1(i) == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
};
template <> struct Lattice<27> {
    static constexpr int Q = 27;
    VLBM_HD static constexpr float w(int i) {
        return lat_norm1(i) == 0 ? 8.0f / 27.0f
             : (lat_norm1(i) == 1 ? 2.0f / 27.0f : (lat_norm1(i) == 2 ? 1.0f / 54.0f : 1.0f / 216.0f));
    }
    VLBM_HD static constexpr double wd(int i) {
        return lat_norm1(i) == 0 ? 8.0 / 27.0
             : (lat_norm1(i) == 1 ? 2.0 / 27.0 : (lat_norm1(i) == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
};

// Runtime weight (host code, tables).
inline double lattice_weight(int Q, int i) {
    return Q == 19 ? Lattice<19>::wd(i) : Lattice<27>::wd(i);
}
inline int lattice_find(int Q, int cx, int cy, int cz) {
    for (int j = 0; j < Q; ++j)
        if (lat_cx(j) == cx && lat_cy(j) == cy && lat_cz(j) == cz) return j;
    return -1;
}

}  // namespace vlbm
