#!/usr/bin/env bash
# Builds RapidSFM's own matcher kernels (from the reference sources, unmodified, where they lie)
# into oracle/_ref/librsfm_ref.so, for sm_100a, with the reference's release flags
# (CMakeLists.txt:60-62: --use_fast_math -DNDEBUG --expt-relaxed-constexpr). The missing
# cuda-utils headers are replaced by this project's minimal stand-ins in oracle/ref_shim/.
# Test infrastructure only. Output goes to oracle/_ref/ (git-ignored; travels with the tree).
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# Location of the RapidSFM source tree: RSFM_REFERENCE_DIR, else where this build machine keeps
# it read-only. This recipe is the only file that reads the reference sources.
REF="${RSFM_REFERENCE_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/bruteForceMatchIMMA.cu" ]; then
  echo "reference sources not found at $REF; skipping" >&2
  exit 0
fi
mkdir -p "$OUT"
NVCC="${NVCC:-/usr/local/cuda/bin/nvcc}"
"$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 --use_fast_math -DNDEBUG \
  --expt-relaxed-constexpr -Xcompiler -fPIC -shared \
  -I"$HERE/ref_shim" -I"$REF" \
  -o "$OUT/librsfm_ref.so.tmp" \
  "$REF/bruteForceMatchIMMA.cu" "$REF/bruteForceMatch.cu" "$REF/bruteForceMatch.cpp" \
  "$REF/casHash/accumulateDesc.cu" "$REF/casHash/computeHash.cu" \
  "$REF/casHash/buildBuckets.cu" "$REF/casHash/findBestMatch.cu" \
  "$HERE/ref_wrapper.cu"
mv "$OUT/librsfm_ref.so.tmp" "$OUT/librsfm_ref.so"
echo "$OUT/librsfm_ref.so"
# RANSAC match filter (RansacMatchFilter.cu), twice: with the reference's flags, and with
# -fmad=false and the shim's arithmetic in the B200 kernel's order (bit-for-bit comparison).
if [ -f "$REF/RansacMatchFilter.cu" ]; then
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 --use_fast_math -DNDEBUG \
    --expt-relaxed-constexpr -Xcompiler -fPIC -shared -DRSFM_REF_SEED_HOOK \
    -I"$HERE/ref_shim" -I"$REF" -o "$OUT/librsfm_ref_ransac.so.tmp" "$HERE/ref_ransac_wrapper.cu"
  mv "$OUT/librsfm_ref_ransac.so.tmp" "$OUT/librsfm_ref_ransac.so"
  "$NVCC" -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -fmad=false -DNDEBUG \
    --expt-relaxed-constexpr -Xcompiler -fPIC -shared -DRSFM_REF_SEED_HOOK -DRSFM_SHIM_KMAT_MATCH \
    -I"$HERE/ref_shim" -I"$REF" -o "$OUT/librsfm_ref_ransac_ieee.so.tmp" "$HERE/ref_ransac_wrapper.cu"
  mv "$OUT/librsfm_ref_ransac_ieee.so.tmp" "$OUT/librsfm_ref_ransac_ieee.so"
  echo "$OUT/librsfm_ref_ransac.so $OUT/librsfm_ref_ransac_ieee.so"
fi
