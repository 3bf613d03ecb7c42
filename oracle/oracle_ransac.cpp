// CPU oracle for the RANSAC match filter. TEST INFRASTRUCTURE ONLY (tests/ and bench.py's CPU
// leg); nothing in the product links, loads or calls it.
//
// Restates RapidSFM's grid-cell affine RANSAC vote filter (paths relative to its source tree):
//  - cell grid and binning: RansacMatchFilter.cpp:40-66 (cellWidth = ceil(max(w, h) / cellCols),
//    cell of a match = clamp(ceil(left / cellWidth)), matches reordered cell by cell, stable)
//  - kernelFindBestAffineForCells: RansacMatchFilter.cu:196-273 (per cell, nbRansacTests
//    3-point affine fits over the 3x3 cell neighbourhood; tests t, t+128, ... on thread t;
//    glibc-style LCG minstd_rand :44-49; distinct samples by rejection; scale gate
//    det in [1/16, 16]; inlier: |A l + t - r|^2 < (threshold * min(sqrt(det), 1))^2; best per
//    thread by strictly more inliers, then the CTA tree reduction of :143-162)
//  - kernelTryBestAffineOfOtherCellsAndVote: :275-333 (every cell's model tried on every
//    neighbourhood; votes when the best has >= 6 inliers)
//  - kernelComputeVotes: :336-389 (own model; +1 vote per inlier when the count is >= 6)
// Differences by design, matched by the CUDA kernels: the RNG seed is a parameter (the reference
// seeds from clock(), so its output is not reproducible); a cell whose neighbourhood holds fewer
// than 9 matches gets the zero model (the reference leaves its scratch slot unwritten); the 3x3
// solve is Gaussian elimination with partial pivoting (the reference's solveGaussElim lives in
// the missing cuda-utils submodule). Every float operation is written out in a fixed order
// (std::fma where the kernels fuse) and built with -ffp-contract=off, so the CUDA kernels
// (explicit _rn intrinsics) match bit for bit.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr uint32_t kCta = 128;
constexpr uint32_t kMinInliers = 6;

struct Pt {
    float lx, ly, rx, ry;
};
struct Aff {
    float a[6];  // row-major 2x3: [a00 a01 a02; a10 a11 a12]
};

uint32_t lcg(uint32_t& s) {
    s = (s * 1103515245u + 12345u) & 0x7fffffffu;
    return s;
}

// 3x3 system A x = B (two right-hand sides) by Gaussian elimination with partial pivoting (first
// largest |pivot|); returns the affine [x^T] as 2x3 rows.
Aff solve3(const Pt* p) {
    float m[3][5];
    for (int i = 0; i < 3; ++i) {
        m[i][0] = p[i].lx;
        m[i][1] = p[i].ly;
        m[i][2] = 1.f;
        m[i][3] = p[i].rx;
        m[i][4] = p[i].ry;
    }
    for (int c = 0; c < 3; ++c) {
        int piv = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(m[r][c]) > std::fabs(m[piv][c])) piv = r;
        if (piv != c)
            for (int k = 0; k < 5; ++k) std::swap(m[c][k], m[piv][k]);
        for (int r = c + 1; r < 3; ++r) {
            const float f = m[r][c] / m[c][c];
            for (int k = c; k < 5; ++k) m[r][k] = m[r][k] - f * m[c][k];
        }
    }
    float x[3][2];
    for (int r = 2; r >= 0; --r)
        for (int h = 0; h < 2; ++h) {
            float v = m[r][3 + h];
            for (int k = r + 1; k < 3; ++k) v = v - m[r][k] * x[k][h];
            x[r][h] = v / m[r][r];
        }
    Aff t;
    for (int h = 0; h < 2; ++h)
        for (int k = 0; k < 3; ++k) t.a[3 * h + k] = x[k][h];
    return t;
}

float det2(const Aff& t) { return t.a[0] * t.a[4] - t.a[1] * t.a[3]; }

float sqr_threshold(const Aff& t, float threshold) {
    const float s = std::sqrt(det2(t));
    const float m = (1.f < s) ? 1.f : s;  // std::min(s, 1.f), NaN kept
    const float v = threshold * m;
    return v * v;
}

// Fused multiply-adds (std::fma rounds once, as the GPU's FMA does), in the kernels' order.
bool inlier(const Aff& t, const Pt& p, float sqrThr) {
    const float dx = std::fma(t.a[0], p.lx, std::fma(t.a[1], p.ly, t.a[2])) - p.rx;
    const float dy = std::fma(t.a[3], p.lx, std::fma(t.a[4], p.ly, t.a[5])) - p.ry;
    return std::fma(dx, dx, dy * dy) < sqrThr;
}

struct Hood {
    uint32_t start[9], size[9], sum;
    Hood(const uint32_t* bounds, uint32_t cols, uint32_t rows, uint32_t cy, uint32_t cx) {
        sum = 0;
        for (int k = 0; k < 9; ++k) {
            const int m = int(cy) - 1 + k / 3, n = int(cx) - 1 + k % 3;
            if (m >= 0 && m < int(rows) && n >= 0 && n < int(cols)) {
                const uint32_t idx = uint32_t(m) * cols + uint32_t(n);
                start[k] = bounds[idx];
                size[k] = bounds[idx + 1] - bounds[idx];
            } else {
                start[k] = size[k] = 0;
            }
            sum += size[k];
        }
    }
    uint32_t match(uint32_t idx) const {
        uint32_t acc = 0;
        for (int k = 0; k < 9; ++k) {
            if (size[k] == 0) continue;
            if (idx < acc + size[k]) return start[k] + (idx - acc);
            acc += size[k];
        }
        return ~0u;
    }
    uint32_t count(const Aff& t, const Pt* pts, float threshold) const {
        const float thr = sqr_threshold(t, threshold);
        uint32_t c = 0;
        for (int k = 0; k < 9; ++k)
            for (uint32_t i = start[k]; i < start[k] + size[k]; ++i) c += inlier(t, pts[i], thr) ? 1u : 0u;
        return c;
    }
};

// The CTA tree of RansacMatchFilter.cu:143-162: for mid = 64 .. 1, slot t < mid takes slot
// t + mid when that has strictly more inliers.
void tree_max(std::vector<uint32_t>& n, std::vector<Aff>& a) {
    for (uint32_t mid = kCta / 2; mid != 0; mid /= 2)
        for (uint32_t t = 0; t < mid; ++t)
            if (n[t] < n[t + mid]) {
                n[t] = n[t + mid];
                a[t] = a[t + mid];
            }
}

}  // namespace

extern "C" {

// Per-cell best models (affines: cols*rows x 6 floats). seed: RNG seed of thread 0 of cell 0.
void orc_ransac_models(const float* matches, const uint32_t* bounds, uint32_t cols, uint32_t rows,
                       uint32_t nbTests, float threshold, uint32_t seed, float* affines) {
    const Pt* pts = reinterpret_cast<const Pt*>(matches);
    for (uint32_t cy = 0; cy < rows; ++cy)
        for (uint32_t cx = 0; cx < cols; ++cx) {
            const uint32_t cell = cy * cols + cx;
            const Hood h(bounds, cols, rows, cy, cx);
            Aff* out = reinterpret_cast<Aff*>(affines) + cell;
            if (h.sum < 9) {
                std::memset(out, 0, sizeof(Aff));
                continue;
            }
            std::vector<uint32_t> bestN(kCta, 0);
            std::vector<Aff> bestA(kCta, Aff{{1, 0, 0, 0, 1, 0}});
            for (uint32_t t = 0; t < kCta; ++t) {
                uint32_t s = seed + (kCta * cell + t) * 22695477u;
                for (uint32_t n = t; n < nbTests; n += kCta) {
                    uint32_t idx[3];
                    uint32_t m = 0;
                    for (uint32_t draw = 0; m < 3 && draw < 64; ++draw) {  // the kernels' draw limit
                        const uint32_t v = lcg(s) % h.sum;
                        bool dup = false;
                        for (uint32_t k = 0; k < m; ++k) dup = dup || idx[k] == v;
                        if (!dup) idx[m++] = v;
                    }
                    if (m < 3) continue;
                    Pt p[3];
                    for (int k = 0; k < 3; ++k) p[k] = pts[h.match(idx[k])];
                    const Aff a = solve3(p);
                    const float d = det2(a);
                    if (d < 0.0625f || d > 16.f || !std::isfinite(d)) continue;
                    const uint32_t c = h.count(a, pts, threshold);
                    if (c > bestN[t]) {
                        bestN[t] = c;
                        bestA[t] = a;
                    }
                }
            }
            tree_max(bestN, bestA);
            *out = bestA[0];
        }
}

// Votes (u8 per match) from the models: each cell's own model (tryOther = 0) or the best of all
// cells' models on its neighbourhood (tryOther = 1, 2); +1 per inlier when >= 6 inliers. With
// tryOther = 1 the gate is the reference's (RansacMatchFilter.cu:305-330): the inlier at
// neighbourhood position i is voted for by thread i mod 128, which tests its own partial maximum
// of the CTA tree (n[t] after tree_max; only n[0] is the full maximum).
void orc_ransac_votes(const float* matches, uint32_t nbMatches, const uint32_t* bounds, uint32_t cols,
                      uint32_t rows, const float* affines, float threshold, int tryOther, uint8_t* votes) {
    const Pt* pts = reinterpret_cast<const Pt*>(matches);
    const Aff* models = reinterpret_cast<const Aff*>(affines);
    std::memset(votes, 0, nbMatches);
    const uint32_t nCells = cols * rows;
    for (uint32_t cy = 0; cy < rows; ++cy)
        for (uint32_t cx = 0; cx < cols; ++cx) {
            const uint32_t cell = cy * cols + cx;
            const Hood h(bounds, cols, rows, cy, cx);
            Aff best = models[cell];
            uint32_t bestN = 0;
            std::vector<uint32_t> gate;  // per thread (tryOther = 1)
            if (tryOther) {
                std::vector<uint32_t> n(kCta, 0);
                std::vector<Aff> a(kCta, models[cell]);
                for (uint32_t t = 0; t < kCta; ++t)
                    for (uint32_t k = t; k < nCells; k += kCta) {
                        const uint32_t c = h.count(models[k], pts, threshold);
                        if (c > n[t]) {
                            n[t] = c;
                            a[t] = models[k];
                        }
                    }
                tree_max(n, a);
                best = a[0];
                bestN = n[0];
                if (tryOther == 1) gate = n;
            } else {
                bestN = h.count(best, pts, threshold);
            }
            if (bestN < kMinInliers) continue;
            const float thr = sqr_threshold(best, threshold);
            for (uint32_t i = 0; i < h.sum; ++i) {
                if (!gate.empty() && gate[i % kCta] < kMinInliers) continue;
                const uint32_t m = h.match(i);
                if (inlier(best, pts[m], thr)) votes[m] = uint8_t(votes[m] + 1);
            }
        }
}

}  // extern "C"
