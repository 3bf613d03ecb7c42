// Minimal stand-in for cuda-utils' ptr.h (written for this project): a bounds-aware pointer made
// of (base, number of valid elements, current offset).
#pragma once
#include <cstdint>
#include "KArray.h"

namespace cudapp {
template <typename T, typename OrigType = T>
struct Ptr {
    T* base;
    uint32_t nbElems;
    int32_t offset;
    RSFM_SHIM_HD Ptr(T* b, uint32_t n, int32_t off) : base(b), nbElems(n), offset(off) {}
    RSFM_SHIM_HD bool isInBound() const { return offset >= 0 && uint32_t(offset) < nbElems; }
    RSFM_SHIM_HD T* get() const { return base + offset; }
    RSFM_SHIM_HD Ptr operator+(int32_t n) const { return Ptr(base, nbElems, offset + n); }
    RSFM_SHIM_HD T& operator*() const { return base[offset]; }
    RSFM_SHIM_HD T& operator[](int32_t i) const { return base[offset + i]; }
};
}  // namespace cudapp
