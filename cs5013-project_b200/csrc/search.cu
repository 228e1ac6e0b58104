// search.cu -- dispatch of the search kernel by row format; the kernel itself
// is in search_impl.cuh, instantiated once per format in search_<format>.cu.
#include "search_dispatch.cuh"

namespace vann {

cudaError_t launch_search_f32(const SearchArgs& a, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_search_bf16(const SearchArgs& a, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_search_fp8(const SearchArgs& a, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_search_u8(const SearchArgs& a, int variant, int num_sms, cudaStream_t st);
cudaError_t launch_search_pq(const SearchArgs& a, int variant, int num_sms, cudaStream_t st);

cudaError_t launch_search(const SearchArgs& a, int store, int num_sms, cudaStream_t st, int variant) {
    switch (store) {
        case 0: return launch_search_f32(a, variant, num_sms, st);
        case 1: return launch_search_bf16(a, variant, num_sms, st);
        case 2: return launch_search_fp8(a, variant, num_sms, st);
        case 3: return launch_search_u8(a, variant, num_sms, st);
        case 4: return launch_search_pq(a, variant, num_sms, st);
        default: return cudaErrorInvalidValue;
    }
}

int search_variants() { return kSearchVariants; }

}  // namespace vann
