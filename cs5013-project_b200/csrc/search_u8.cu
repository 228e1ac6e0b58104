// search_u8.cu -- search kernel instantiations for StoreU8 rows (one
// translation unit per row format so they compile in parallel).
#include "search_dispatch.cuh"

namespace vann {
cudaError_t launch_search_u8(const SearchArgs& a, int variant, int num_sms, cudaStream_t st) {
    return launch_store<StoreU8>(a, variant, num_sms, st);
}
}  // namespace vann
