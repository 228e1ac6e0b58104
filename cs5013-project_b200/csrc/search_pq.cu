// search_pq.cu -- search kernel instantiations for StorePQ codes (one
// translation unit per row format so they compile in parallel).
#include "search_dispatch.cuh"

namespace vann {
cudaError_t launch_search_pq(const SearchArgs& a, int variant, int num_sms, cudaStream_t st) {
    return launch_store<StorePQ>(a, variant, num_sms, st);
}
}  // namespace vann
