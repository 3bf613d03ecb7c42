// Allocation-free variant of rsfm_bf_match (no reference counterpart).
//
// rsfm_bf_match needs one 32-bit second-best distance per query row while it runs (the row
// thresholds of the fused top-2 epilogue), and takes that scratch from a stream-ordered pool
// allocation. This entry point takes it instead from a fixed file-scope device array, so a call
// allocates no device memory at all: for callers that must not allocate (a scheduler thread that runs under a fixed
// memory budget, or code that may not touch the allocator while other work is in flight).
//
// Limits and contract:
//  - the scratch holds kNoAllocMaxRows = 1 Mi rows (4 MiB); a call whose tasks hold more query
//    rows in total returns RSFM_ERR_CAPACITY before enqueuing anything;
//  - the first call on a device (with that device current) looks up the array's device address
//    with cudaGetSymbolAddress and caches it per device; make that first call before any stream
//    capture on the device;
//  - every call shares the one array and it keeps the last call's contents; the init kernel of each
//    call sets the rows it uses to ~0u before the matcher reads them, so nothing carries over
//    between calls. Calls whose work overlaps on the GPU (different streams, no ordering between
//    them) race on the array and their results are undefined: order them on one stream.
#include "bf_internal.h"
#include "common.h"
#include <algorithm>
#include <mutex>
#include <vector>

namespace rsfm_b200 {
namespace noalloc {

constexpr size_t kNoAllocMaxRows = size_t(1) << 20;
constexpr size_t kTasksPerLaunch = bf::kMaxTasksPerLaunch;  // tasks per matcher launch, as in rsfm_bf_match
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint32_t g_second_scratch[kNoAllocMaxRows];

static std::mutex g_lock;
static uint32_t* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once per device).
static int scratch_for_current_device(uint32_t** out) {
    int dev = -1;
    RSFM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return RSFM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_lock);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        RSFM_CUDA_TRY(cudaGetSymbolAddress(&p, g_second_scratch));
        g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scratch_ptr[dev];
    return RSFM_OK;
}

}  // namespace noalloc
}  // namespace rsfm_b200

using namespace rsfm_b200;

extern "C" int rsfm_bf_match_noalloc(const rsfm_sift_bf_task* tasks, size_t nbTasks, cudaStream_t stream) {
    launch_count_reset();
    // The same argument checks as rsfm_bf_match, then the scratch limit on the total query rows.
    int st = bf::validate(tasks, nbTasks);
    if (st != RSFM_OK) return st;
    size_t total = 0;
    for (size_t t = 0; t < nbTasks; ++t) total += tasks[t].nbDescA;
    if (total > noalloc::kNoAllocMaxRows) return RSFM_ERR_CAPACITY;
    if (nbTasks == 0) return RSFM_OK;
    uint32_t* scratch = nullptr;
    st = noalloc::scratch_for_current_device(&scratch);
    if (st != RSFM_OK) return st;
    uint32_t* second[noalloc::kTasksPerLaunch];
    size_t off = 0;
    for (size_t i = 0; i < nbTasks; i += noalloc::kTasksPerLaunch) {
        const size_t n = std::min(noalloc::kTasksPerLaunch, nbTasks - i);
        for (size_t t = 0; t < n; ++t) {
            second[t] = scratch + off;
            off += tasks[i + t].nbDescA;
        }
        st = bf::launch_chunk(tasks + i, n, second, nullptr, 0, 1, stream);
        if (st != RSFM_OK) return st;
    }
    return RSFM_OK;
}
