// step_q27_f16.cu -- D3Q27 kernels with F16 population storage.
#include "dispatch_impl.cuh"
namespace vlbm {
VLBM_INSTANTIATE(27, VLBM_STORE_F16)
}  // namespace vlbm
