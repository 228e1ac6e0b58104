// search_dispatch.cuh -- picks the search kernel instantiation for a launch:
// register worklist (search_reg.cuh) for L <= 64 at D <= 128 and R <= 64,
// shared-memory worklist (search_impl.cuh) otherwise, and the launch-bound
// variant chosen by the autotuner.
#pragma once
#include "search_reg.cuh"

namespace vann {

// Launch-bound variants (minimum resident blocks per SM, i.e. a register cap)
// exist for the common shape (D <= 128, R <= 64); the autotuner picks one.
constexpr int kSearchVariants = 7;

template <typename S, int DC, int SPL, int LREG, int BEAM>
static cudaError_t launch_rw_v(const SearchArgs& a, int variant, int sms, cudaStream_t st) {
    switch (variant) {
        case 1: return launch_rw<S, DC, SPL, LREG, 4, BEAM>(a, sms, st);
        case 2: return launch_rw<S, DC, SPL, LREG, 5, BEAM>(a, sms, st);
        case 3: return launch_rw<S, DC, SPL, LREG, 7, BEAM>(a, sms, st);
        case 4: return launch_rw<S, DC, SPL, LREG, 8, BEAM>(a, sms, st);
        case 5: return launch_rw<S, DC, SPL, LREG, 9, BEAM>(a, sms, st);
        case 6: return launch_rw<S, DC, SPL, LREG, 10, BEAM>(a, sms, st);
        default: return launch_rw<S, DC, SPL, LREG, 6, BEAM>(a, sms, st);
    }
}

template <typename S, int DC, int SPL>
static cudaError_t launch_v(const SearchArgs& a, int variant, int sms, cudaStream_t st) {
    if constexpr (DC == 0 && SPL <= 2) {
        // worklist in registers for L <= 64; two parents per hop only here
        if (a.L <= 32)
            return a.beam == 2 ? launch_rw_v<S, DC, SPL, 1, 2>(a, variant, sms, st)
                               : launch_rw_v<S, DC, SPL, 1, 1>(a, variant, sms, st);
        if (a.L <= 64)
            return a.beam == 2 ? launch_rw_v<S, DC, SPL, 2, 2>(a, variant, sms, st)
                               : launch_rw_v<S, DC, SPL, 2, 1>(a, variant, sms, st);
    }
    if (a.beam == 2) return cudaErrorInvalidValue;
    if constexpr (S::kInt && DC == 0 && SPL <= 2) {
        if (a.int_queries) {  // build and insert searches over the exact uint8 copy
            switch (variant) {
                case 1: return launch_t<S, DC, SPL, 4, true>(a, sms, st);
                case 2: return launch_t<S, DC, SPL, 5, true>(a, sms, st);
                case 3: return launch_t<S, DC, SPL, 7, true>(a, sms, st);
                case 4: return launch_t<S, DC, SPL, 8, true>(a, sms, st);
                case 5: return launch_t<S, DC, SPL, 9, true>(a, sms, st);
                case 6: return launch_t<S, DC, SPL, 10, true>(a, sms, st);
                default: return launch_t<S, DC, SPL, 6, true>(a, sms, st);
            }
        }
    }
    if constexpr (DC == 0 && SPL <= 2) {
        switch (variant) {
            case 1: return launch_t<S, DC, SPL, 4>(a, sms, st);
            case 2: return launch_t<S, DC, SPL, 5>(a, sms, st);
            case 3: return launch_t<S, DC, SPL, 7>(a, sms, st);
            case 4: return launch_t<S, DC, SPL, 8>(a, sms, st);
            case 5: return launch_t<S, DC, SPL, 9>(a, sms, st);
            case 6: return launch_t<S, DC, SPL, 10>(a, sms, st);
            default: break;
        }
    }
    return launch_t<S, DC, SPL, 6>(a, sms, st);
}

template <typename S, int DC>
static cudaError_t launch_r(const SearchArgs& a, int variant, int sms, cudaStream_t st) {
    if (a.R <= 32) return launch_v<S, DC, 1>(a, variant, sms, st);
    if (a.R <= 64) return launch_v<S, DC, 2>(a, variant, sms, st);
    return launch_v<S, DC, 4>(a, variant, sms, st);
}

template <typename S>
static cudaError_t launch_store(const SearchArgs& a, int variant, int sms, cudaStream_t st) {
    if (a.D % S::kElems != 0) return cudaErrorInvalidValue;
    if (a.D <= 128) return launch_r<S, 0>(a, variant, sms, st);
    if (a.D <= 256) return launch_r<S, 1>(a, variant, sms, st);
    return launch_r<S, 2>(a, variant, sms, st);
}

}  // namespace vann
