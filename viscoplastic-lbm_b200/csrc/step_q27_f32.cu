// step_q27_f32.cu -- D3Q27 kernels with F32 population storage.
#include "dispatch_impl.cuh"
namespace vlbm {
VLBM_INSTANTIATE(27, VLBM_STORE_F32)
}  // namespace vlbm
