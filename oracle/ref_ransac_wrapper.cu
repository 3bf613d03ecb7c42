// Test infrastructure: RapidSFM's RANSAC match filter kernels (RansacMatchFilter.cu, compiled
// unmodified from the reference sources; this file includes it) behind a C entry with an
// explicit seed (the reference's clock() seed reads it through the shim's seed hook).
// oracle/build_ref.sh builds it twice: with the reference's own flags (--use_fast_math) and with
// -fmad=false plus the shim's matching arithmetic mode.
#include "RansacMatchFilter.cu"

extern "C" int ref_ransac_match_filter(uint8_t* votes, float* affineScratch, const void* matches, uint32_t nbMatches,
                                       const uint32_t* bounds, uint32_t cols, uint32_t rows, uint32_t nbRansacTests,
                                       float threshold, int tryOtherSolutions, uint32_t seed, cudaStream_t stream) {
    try {
        cudaCheck(cudaMemcpyToSymbolAsync(g_rsfm_ref_seed, &seed, sizeof(seed), 0, cudaMemcpyHostToDevice, stream));
        rsfm::rmf::cudaRansacMatchFilter(votes, reinterpret_cast<kmat<float, 2, 3>*>(affineScratch),
                                         static_cast<const rsfm::rmf::PtPair*>(matches), nbMatches, bounds, cols, rows,
                                         nbRansacTests, threshold, tryOtherSolutions != 0, stream);
    } catch (...) {
        return 1;
    }
    return 0;
}
