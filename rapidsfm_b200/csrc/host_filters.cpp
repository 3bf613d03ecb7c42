// Host-side match filters with the reference semantics:
//   crossCheckMatches     bruteForceMatch.cpp:23-40  keep i when bwd[fwd[i].index].index == i,
//                                                    skip ~0u, output in query order
//   removeMatchConflicts  bruteForceMatch.cpp:42-66  per train descriptor keep the closest query
//                                                    (strict <, first query wins ties), output
//                                                    in train order
#include <cstdint>
#include <cstddef>
#include <vector>
#include "../../include/rsfm_b200.h"

extern "C" size_t rsfm_cross_check_matches(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                           const rsfm_best_match* matchesBwd, uint32_t nbTrainDesc,
                                           rsfm_valid_match* out) {
    if (!matches || !matchesBwd || !out) return 0;
    size_t n = 0;
    for (uint32_t i = 0; i < nbQueryDesc; ++i) {
        const uint32_t j = matches[i].index;
        if (j == ~0u || j >= nbTrainDesc) continue;
        if (matchesBwd[j].index == i) out[n++] = rsfm_valid_match{i, j, float(matches[i].distance)};
    }
    return n;
}

extern "C" size_t rsfm_remove_match_conflicts(const rsfm_best_match* matches, uint32_t nbQueryDesc,
                                              uint32_t nbTrainDesc, rsfm_valid_match* out) {
    if (!matches || !out) return 0;
    std::vector<rsfm_best_match> bwd(nbTrainDesc, rsfm_best_match{~0u, ~0u});
    for (uint32_t i = 0; i < nbQueryDesc; ++i) {
        const rsfm_best_match& q = matches[i];
        if (q.index == ~0u || q.index >= nbTrainDesc) continue;
        rsfm_best_match& t = bwd[q.index];
        if (q.distance < t.distance) t = rsfm_best_match{i, q.distance};
    }
    size_t n = 0;
    for (uint32_t j = 0; j < nbTrainDesc; ++j)
        if (bwd[j].index != ~0u) out[n++] = rsfm_valid_match{bwd[j].index, j, float(bwd[j].distance)};
    return n;
}
