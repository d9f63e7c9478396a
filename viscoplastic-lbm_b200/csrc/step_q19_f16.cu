// step_q19_f16.cu -- D3Q19 kernels with F16 population storage.
#include "dispatch_impl.cuh"
namespace vlbm {
VLBM_INSTANTIATE(19, VLBM_STORE_F16)
}  // namespace vlbm
