// step_q19_f32.cu -- D3Q19 kernels with F32 population storage.
#include "dispatch_impl.cuh"
namespace vlbm {
VLBM_INSTANTIATE(19, VLBM_STORE_F32)
}  // namespace vlbm
