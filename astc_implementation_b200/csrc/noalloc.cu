// Encode entry point that allocates no memory, for callers that cannot call
// cudaMalloc: code running inside a host application's own memory budget (a
// game engine or driver-side texture pipeline whose allocator owns the whole
// device heap), code running while a CUDA graph is being built elsewhere in
// the process, or plug-ins loaded into a process whose allocation policy they
// do not control.  The caller passes the input texels and the output blocks;
// every intermediate the search needs lives in one file-scope device array.
//
// Limits and sharing rules:
//  * the array is kNoallocBytes (48 MiB) and every GPU that loads this library
//    keeps it until the process exits;
//  * one call encodes at most kNoallocMaxBlocks (2048) blocks; larger images are
//    rejected with ASTCB200_TOO_LARGE (split them into tiles);
//  * all calls share the array and it keeps the last call's contents; calls
//    that overlap on the GPU (other streams, other host threads) race, so
//    callers must serialise them;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress; make that first call before any stream capture.
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "astcb200.h"
#include "kernels.h"
#include "tables.h"

namespace astcb200 {
namespace {

constexpr size_t kNoallocBytes = size_t(48) << 20;
constexpr size_t kNoallocTableBytes = size_t(2) << 20;
constexpr uint32_t kNoallocMaxBlocks = 2048;

__device__ __align__(256) uint8_t g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint8_t* g_scratch_ptr[kMaxDevices] = {};

struct HostBlob {
    TableLayout L;
    std::vector<uint8_t> bytes;
};

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace
}  // namespace astcb200

using namespace astcb200;

extern "C" int astcb200_encode_noalloc(int device, const uint8_t* d_rgba8, uint32_t width, uint32_t height,
                                       uint8_t block_x, uint8_t block_y, uint8_t* d_out_blocks, void* cuda_stream) {
    static_assert(align256(sizeof(PartPicks) * kNoallocMaxBlocks) + align256(sizeof(PBRec) * kSlotsPerBlock * kNoallocMaxBlocks) +
                      align256(sizeof(Snap) * kSlotsPerBlock * kNumCand * kNoallocMaxBlocks) + kNoallocTableBytes <= kNoallocBytes,
                  "no-allocation scratch too small for its block limit");
    if (!d_rgba8 || !d_out_blocks || width == 0 || height == 0 || device < 0 || device >= kMaxDevices) return ASTCB200_BAD_ARG;
    if (((uintptr_t)d_rgba8 & 3) || ((uintptr_t)d_out_blocks & 15)) return ASTCB200_BAD_ARG;
    if (!valid_footprint(block_x, block_y)) return ASTCB200_INVALID_FOOTPRINT;
    const uint64_t nbx = (width + block_x - 1) / block_x, nby = (height + block_y - 1) / block_y;
    if (nbx * nby > kNoallocMaxBlocks) return ASTCB200_TOO_LARGE;
    if (cudaSetDevice(device) != cudaSuccess) return ASTCB200_CUDA_ERROR;

    static std::map<int, HostBlob> blobs;
    uint8_t* base = nullptr;
    const HostBlob* hb = nullptr;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (!g_scratch_ptr[device]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ASTCB200_CUDA_ERROR;
            g_scratch_ptr[device] = static_cast<uint8_t*>(p);
        }
        base = g_scratch_ptr[device];
        HostBlob& b = blobs[block_x * 256 + block_y];
        if (b.bytes.empty() && !build_tables(block_x, block_y, b.L, b.bytes)) return ASTCB200_INVALID_FOOTPRINT;
        if (b.bytes.size() > kNoallocTableBytes) return ASTCB200_TOO_LARGE;
        hb = &b;
    }
    if (configure_kernels(hb->L) != cudaSuccess) return ASTCB200_CUDA_ERROR;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    if (cudaMemcpyAsync(base, hb->bytes.data(), hb->bytes.size(), cudaMemcpyHostToDevice, s) != cudaSuccess) return ASTCB200_CUDA_ERROR;

    KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.img = d_rgba8;
    a.width = (int)width; a.height = (int)height; a.nbx = (int)nbx; a.nby = (int)nby;
    a.block_first = 0; a.nblocks = (int)(nbx * nby);
    a.tables = base;
    a.L = hb->L;
    size_t off = kNoallocTableBytes;
    a.picks = reinterpret_cast<PartPicks*>(base + off);
    off += align256(sizeof(PartPicks) * kNoallocMaxBlocks);
    a.pbrec = reinterpret_cast<PBRec*>(base + off);
    off += align256(sizeof(PBRec) * kSlotsPerBlock * kNoallocMaxBlocks);
    a.snaps = reinterpret_cast<Snap*>(base + off);
    a.out_blocks = d_out_blocks;
    a.symbolic = nullptr;
    a.slots = kSlotsPerBlock;
    a.topn = kNumCand;
    // Every record the kernels read is written earlier in the same call (absent
    // partitioned blocks get ncand = 0, unrefined candidates err = 1e37), so the
    // previous call's contents need no clearing.
    if (launch_partition_search(a, s) != cudaSuccess) return ASTCB200_CUDA_ERROR;
    if (launch_front(a, s) != cudaSuccess) return ASTCB200_CUDA_ERROR;
    if (launch_refine(a, s) != cudaSuccess) return ASTCB200_CUDA_ERROR;
    if (launch_select_pack(a, s) != cudaSuccess) return ASTCB200_CUDA_ERROR;
    return ASTCB200_OK;
}
