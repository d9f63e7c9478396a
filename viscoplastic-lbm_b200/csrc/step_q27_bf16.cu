// step_q27_bf16.cu -- D3Q27 kernels with BF16 population storage.
#include "dispatch_impl.cuh"
namespace vlbm {
VLBM_INSTANTIATE(27, VLBM_STORE_BF16)
}  // namespace vlbm
