// Encode entry point that allocates no memory, for callers that cannot call
// cudaMalloc: code running inside a host application's own memory budget (a
// game engine or driver-side texture pipeline whose allocator owns the whole
// device heap), or plug-ins loaded into a process whose allocation policy they
// do not control.  The caller passes the input texels and the output blocks;
// every intermediate the search needs, and the search tables of every
// footprint used so far, live in one file-scope device array.
//
// Limits and sharing rules:
//  * the array is kNoallocBytes (52 MiB); the CUDA runtime commits it on a device
//    when the first call there resolves its address (modules load lazily), and
//    the device keeps it until the process exits.  Make that first call at start-up,
//    before the caller's allocator reserves the heap: if the device has no room
//    left then, the call returns ASTCB200_OOM;
//  * one call encodes at most kNoallocMaxBlocks (2048) blocks; larger images are
//    rejected with ASTCB200_TOO_LARGE (split them into tiles);
//  * the first call on a device, and the first call of each footprint on it, do
//    set-up work: they resolve the array's address with cudaGetSymbolAddress,
//    upload that footprint's tables into the array with a synchronous copy and
//    set the kernels' shared-memory limits.  Make those first calls before any
//    stream capture.  Later calls only queue the four search kernels;
//  * all calls share the array and it keeps the last call's contents; calls
//    that overlap on the GPU (other streams, other host threads) race, so
//    callers must serialise them;
//  * the search is always the exhaustive one of the reference (no proposal
//    network, no pruning), with the reference's semantics.
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "astcb200.h"
#include "device_guard.h"
#include "kernels.h"
#include "tables.h"

namespace astcb200 {
namespace {

constexpr size_t kNoallocBytes = size_t(52) << 20;
constexpr size_t kNoallocTableBytes = size_t(8) << 20;  // every footprint's tables: 7.13 MiB
constexpr uint32_t kNoallocMaxBlocks = 2048;

__device__ __align__(256) uint8_t g_noalloc_scratch[kNoallocBytes];

constexpr int kMaxDevices = 64;
constexpr int kFootprints = 14;

struct HostBlob {
    TableLayout L;
    std::vector<uint8_t> bytes;
};

// Per device: the array's address and where each footprint's tables sit in it.
struct DeviceState {
    uint8_t* base = nullptr;
    size_t table_end = 0;
    long long table_off[kFootprints];
    DeviceState() { for (long long& o : table_off) o = -1; }
};

std::mutex g_mu;
DeviceState g_dev[kMaxDevices];
std::map<int, HostBlob> g_blobs;  // by block_x * 256 + block_y

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

int footprint_index(int bx, int by) {
    static const int fp[kFootprints][2] = {{4, 4}, {5, 4}, {5, 5}, {6, 5}, {6, 6}, {8, 5}, {8, 6},
                                           {10, 5}, {10, 6}, {8, 8}, {10, 8}, {10, 10}, {12, 10}, {12, 12}};
    for (int i = 0; i < kFootprints; i++)
        if (fp[i][0] == bx && fp[i][1] == by) return i;
    return -1;
}

int status_of(cudaError_t e) { return e == cudaErrorMemoryAllocation ? ASTCB200_OOM : ASTCB200_CUDA_ERROR; }

}  // namespace
}  // namespace astcb200

using namespace astcb200;

extern "C" int astcb200_encode_noalloc(int device, const uint8_t* d_rgba8, uint32_t width, uint32_t height,
                                       uint8_t block_x, uint8_t block_y, uint8_t* d_out_blocks, void* cuda_stream) {
    static_assert(kNoallocTableBytes + align256(sizeof(PartPicks) * kNoallocMaxBlocks) +
                          align256(sizeof(PBRec) * kSlotsPerBlock * kNoallocMaxBlocks) +
                          align256(sizeof(Snap) * kSlotsPerBlock * kNumCand * kNoallocMaxBlocks) <= kNoallocBytes,
                  "no-allocation scratch too small for its block limit");
    if (!d_rgba8 || !d_out_blocks || width == 0 || height == 0 || device < 0 || device >= kMaxDevices) return ASTCB200_BAD_ARG;
    if (((uintptr_t)d_rgba8 & 3) || ((uintptr_t)d_out_blocks & 15)) return ASTCB200_BAD_ARG;
    const int fi = footprint_index(block_x, block_y);
    if (fi < 0) return ASTCB200_INVALID_FOOTPRINT;
    const uint64_t nbx = (width + block_x - 1) / block_x, nby = (height + block_y - 1) / block_y;
    if (nbx * nby > kNoallocMaxBlocks) return ASTCB200_TOO_LARGE;
    DeviceGuard dg(device);
    if (dg.err != cudaSuccess) return ASTCB200_CUDA_ERROR;

    uint8_t* base = nullptr;
    const HostBlob* hb = nullptr;
    size_t toff = 0;
    {
        std::lock_guard<std::mutex> g(g_mu);
        DeviceState& ds = g_dev[device];
        if (!ds.base) {  // set-up, once per device
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) { cudaGetLastError(); return status_of(e); }
            ds.base = static_cast<uint8_t*>(p);
        }
        base = ds.base;
        HostBlob& b = g_blobs[block_x * 256 + block_y];
        if (b.bytes.empty() && !build_tables(block_x, block_y, b.L, b.bytes)) return ASTCB200_INVALID_FOOTPRINT;
        hb = &b;
        if (ds.table_off[fi] < 0) {  // set-up, once per footprint and device: the tables stay resident
            if (ds.table_end + align256(b.bytes.size()) > kNoallocTableBytes) return ASTCB200_TOO_LARGE;
            cudaError_t e = cudaMemcpy(base + ds.table_end, b.bytes.data(), b.bytes.size(), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = configure_kernels(b.L);
            if (e != cudaSuccess) { cudaGetLastError(); return status_of(e); }
            ds.table_off[fi] = (long long)ds.table_end;
            ds.table_end += align256(b.bytes.size());
        }
        toff = (size_t)ds.table_off[fi];
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

    KernelArgs a;
    std::memset(&a, 0, sizeof(a));
    a.img = d_rgba8;
    a.width = (int)width; a.height = (int)height; a.nbx = (int)nbx; a.nby = (int)nby;
    a.block_first = 0; a.nblocks = (int)(nbx * nby);
    a.tables = base + toff;
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
