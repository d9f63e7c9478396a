// step_q19_bf16.cu -- D3Q19 kernels with BF16 population storage.
#include "dispatch_impl.cuh"
namespace vlbm {
VLBM_INSTANTIATE(19, VLBM_STORE_BF16)
}  // namespace vlbm
