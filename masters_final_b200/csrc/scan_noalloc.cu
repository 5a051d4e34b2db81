// Exclusive int32 scan that allocates nothing.
//
// Who needs it: code that must not allocate device memory at the time it
// runs -- for example a host program whose memory pools are sized and locked
// at start-up, an embedded or real-time caller that forbids allocation on its
// processing path, or a plugin that only receives raw buffers from its host
// application and has no allocator to draw a workspace from.  Such callers
// cannot provide the workspace that eacb_scan_excl_i32 asks for.
//
// How: the scan's look-back scratch (one status word per 4096-element tile,
// a tile counter and an error word) lives in a fixed array in device memory,
// defined below.  It is part of the library's image: every GPU that loads
// libeacb200 holds it (about 350 KiB) until the process exits.  The device
// address of that array is looked up once per device with
// cudaGetSymbolAddress (a lookup, not an allocation), on the first call made
// while that device is current; make that first call before any stream
// capture.  The address is kept for the life of the process, so a process
// that resets a device (cudaDeviceReset) must not call this entry point on
// that device afterwards.  The array is shared by every call: the parts a
// call needs are cleared at the start of the call, and two calls that run on
// the GPU at the same time (for instance on two streams) would race on it, so
// callers must serialise them.  Each call waits for its scan to finish: it
// copies the device status back to the host and synchronizes the stream.
#include "eacb_common.cuh"
#include "scan_impl.cuh"

#include <mutex>

namespace {

// n up to 2^28 elements -> 43,691 tiles of 6,144
constexpr int64_t kNoAllocMaxN = EACB_SCAN_NOALLOC_MAX_N;
constexpr int64_t kNoAllocTiles = kNoAllocMaxN / eacb::kScanTile + 1;
// layout: [0] error word, [8..16) tile counter, [256..) tile status words
constexpr size_t kNoAllocBytes = 256 + (size_t)kNoAllocTiles * sizeof(uint64_t);

static __device__ __align__(256) unsigned char g_scan_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_scan_scratch on the current device (looked up once).
int scratch_for_current_device(unsigned char **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return EACB_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return EACB_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scan_scratch) != cudaSuccess || !p) return EACB_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = (unsigned char *)g_scratch_addr[dev];
    return EACB_OK;
}

}  // namespace

extern "C" int eacb_scan_excl_i32_noalloc(const int32_t *in, int32_t *out, int64_t n, int64_t init,
                                          int64_t *d_total, uintptr_t stream)
{
    if (n < 0 || (n > 0 && (!in || !out)) || !d_total) return EACB_ERR_BAD_ARGUMENT;
    if (n > kNoAllocMaxN) return EACB_ERR_WORKSPACE;       // beyond the fixed scratch
    unsigned char *base = nullptr;
    int s = scratch_for_current_device(&base);
    if (s) return s;
    eacb::ScanScratch sc;
    sc.err = (int *)base;
    sc.counter = (int *)(base + 8);
    sc.status = (uint64_t *)(base + 256);
    sc.max_tiles = kNoAllocTiles;
    cudaStream_t st = (cudaStream_t)stream;
    // the previous call's contents are still there: clear what starts at zero
    // (scan_launch clears the tile counter and the status words it uses)
    EACB_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(int), st));
    eacb::ProfScope ps(eacb::PROF_SCAN, st);
    s = eacb::scan_launch<int32_t, int32_t>(in, out, n, init, d_total, sc, st);
    ps.done((double)n * 2.0 * sizeof(int32_t));
    if (s) return s;
    // report a device-side failure of this call (a look-back wait that gave
    // up) before returning: read the error word and wait for the scan
    int e = 0;
    EACB_CUDA(cudaMemcpyAsync(&e, sc.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    return eacb::dev_err_to_status(e);
}
