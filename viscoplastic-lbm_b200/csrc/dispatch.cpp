// dispatch.cpp -- run-time selection of the (velocity set, storage) kernel family.
#include "dispatch.h"

namespace vlbm {

#define VLBM_SELECT(CALL)                                                          \
    if (Q == 19) {                                                                 \
        if (st == VLBM_STORE_F32) return CALL(19, VLBM_STORE_F32);                 \
        if (st == VLBM_STORE_F16) return CALL(19, VLBM_STORE_F16);                 \
        if (st == VLBM_STORE_BF16) return CALL(19, VLBM_STORE_BF16);               \
    } else if (Q == 27) {                                                          \
        if (st == VLBM_STORE_F32) return CALL(27, VLBM_STORE_F32);                 \
        if (st == VLBM_STORE_F16) return CALL(27, VLBM_STORE_F16);                 \
        if (st == VLBM_STORE_BF16) return CALL(27, VLBM_STORE_BF16);               \
    }                                                                              \
    return cudaErrorInvalidValue;

cudaError_t launch_step(int Q, int st, const StepParams& p, int op, int rheo, bool odd, LaunchShape ls,
                        cudaStream_t s) {
#define C_(QQ, SS) launch_step_st<QQ, SS>(p, op, rheo, odd, ls, s)
    VLBM_SELECT(C_)
#undef C_
}
cudaError_t launch_macro(int Q, int st, const MacroParams& mp, int rheo, bool odd, cudaStream_t s) {
#define C_(QQ, SS) launch_macro_st<QQ, SS>(mp, rheo, odd, s)
    VLBM_SELECT(C_)
#undef C_
}
cudaError_t launch_get_pops(int Q, int st, const StepParams& p, bool odd, float* out, cudaStream_t s) {
#define C_(QQ, SS) launch_get_pops_st<QQ, SS>(p, odd, out, s)
    VLBM_SELECT(C_)
#undef C_
}
cudaError_t launch_set_pops(int Q, int st, const StepParams& p, const float* in, float rho, float ux, float uy,
                            float uz, cudaStream_t s) {
#define C_(QQ, SS) launch_set_pops_st<QQ, SS>(p, in, rho, ux, uy, uz, s)
    VLBM_SELECT(C_)
#undef C_
}

cudaError_t launch_batched(int Q, int st, const BatchLaunch* L, const BatchState* state, const BatchBlock* table,
                           int ntiles, int grid, bool odd, int op, int rheo, cudaStream_t s) {
#define C_(QQ, SS) launch_batched_st<QQ, SS>(L, state, table, ntiles, grid, odd, op, rheo, s)
    VLBM_SELECT(C_)
#undef C_
}

cudaError_t launch_relayout(int Q, int st, const void* src, void* dst, int nx, int ny, long long N, int sH, int sB,
                            int dH, int dB, cudaStream_t s) {
#define C_(QQ, SS) launch_relayout_st<QQ, SS>(src, dst, nx, ny, N, sH, sB, dH, dB, s)
    VLBM_SELECT(C_)
#undef C_
}

cudaError_t launch_halo(int Q, int st, void* pop, const HaloSpec* msgs, int nx, int ny, long long N, int H,
                        int blk, bool unpack, cudaStream_t s) {
#define C_(QQ, SS) launch_halo_st<QQ, SS>(pop, msgs, nx, ny, N, H, blk, unpack, s)
    VLBM_SELECT(C_)
#undef C_
}

#define VLBM_SELECT_INT(CALL)                                                      \
    if (Q == 19) {                                                                 \
        if (st == VLBM_STORE_F32) return CALL(19, VLBM_STORE_F32);                 \
        if (st == VLBM_STORE_F16) return CALL(19, VLBM_STORE_F16);                 \
        if (st == VLBM_STORE_BF16) return CALL(19, VLBM_STORE_BF16);               \
    } else if (Q == 27) {                                                          \
        if (st == VLBM_STORE_F32) return CALL(27, VLBM_STORE_F32);                 \
        if (st == VLBM_STORE_F16) return CALL(27, VLBM_STORE_F16);                 \
        if (st == VLBM_STORE_BF16) return CALL(27, VLBM_STORE_BF16);               \
    }                                                                              \
    return 0;

int batched_blocks_per_sm(int Q, int st, int op, int rheo) {
#define C_(QQ, SS) batched_occupancy_st<QQ, SS>(op, rheo)
    VLBM_SELECT_INT(C_)
#undef C_
}

}  // namespace vlbm
