// Shared device/host helpers of libeacb200 (sm_100a only).
//
// Conventions of every entry point in include/eacb200.h:
//   * device pointers + sizes + a cudaStream_t passed as uintptr_t;
//   * scratch memory comes from a caller-owned workspace whose size is given
//     by the matching *_workspace_size() query (nothing here calls cudaMalloc);
//   * the return value is an eacb status (0 = ok, negative = error); device
//     side failures (iteration caps, bad input detected in a kernel) are
//     written to an error word in the workspace and reported on return.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/eacb200.h"

namespace eacb {
inline void count_launch(int n = 1);
// the calling thread's last failed CUDA runtime call (eacb_last_cuda_error)
void note_cuda_error(int code, const char *file, int line);
// caps the participants of the Boruvka round kernels this host thread
// launches (0 = no cap)
void set_thread_round_team(int blocks);
// Launch-shape knobs of the tuning table (csrc/tune.cu); (a, b) is the
// shape each user states.
enum TuneKnob : int {
    TUNE_TC_CTAS_PER_SM = 0,   // tensor-core labeler CTAs per SM (1, 2); a = d, b = n
    TUNE_TC_BUFFERS = 1,       // its centroid tile buffers (1, 2); a = d, b = n
    TUNE_CO_COUNT_CTAS = 2,    // co-association count pass CTAs per SM; a = P, b = n
    TUNE_CO_FILL_CTAS = 3,     // co-association fill pass CTAs per SM; a = P, b = n
    TUNE_MST_PHASE1 = 4,       // graph MST: first phase's share of the entries, per mille; a = 0, b = V
    TUNE_ROUND_TEAM = 5,       // Boruvka round kernel participants at most; a = 0 graph, 1 EAC; b = V
    TUNE_CO_DENSE = 6,         // co-association pair tiles: compare work allowed per streamed
                               // member visit (0: streaming only); a = P, b = n
    TUNE_NKNOBS = 7
};
int64_t tune_get(int knob, int64_t a, int64_t b, int64_t dflt);
}
#define EACB_CUDA(call)                                           \
    do {                                                          \
        cudaError_t _e = (call);                                  \
        if (_e != cudaSuccess) {                                  \
            eacb::note_cuda_error((int)_e, __FILE__, __LINE__);   \
            return EACB_ERR_CUDA;                                 \
        }                                                         \
    } while (0)

#define EACB_CHECK_LAUNCH()                 \
    do {                                    \
        eacb::count_launch();               \
        EACB_CUDA(cudaGetLastError());      \
    } while (0)

namespace eacb {

constexpr int kWarp = 32;

// Device error word values (written with atomicCAS so the first one sticks).
enum DevErr : int {
    DEV_OK = 0,
    DEV_SPIN_LIMIT = 1,      // a look-back wait gave up
    DEV_CHASE_LIMIT = 2,     // pointer chase exceeded its bound (not a forest)
    DEV_BAD_INPUT = 3,       // input failed a device-side check
    DEV_FIRST_OVERFLOW = 4,  // first partition's tail exceeds a row capacity
    DEV_CAPACITY = 5,        // an internal capacity was exceeded
};

__device__ __forceinline__ void set_err(int *err, int code)
{
    atomicCAS(err, 0, code);
}

inline int dev_err_to_status(int e)
{
    switch (e) {
    case DEV_OK: return EACB_OK;
    case DEV_SPIN_LIMIT: return EACB_ERR_DEVICE_WAIT;
    case DEV_CHASE_LIMIT: return EACB_ERR_NOT_CONVERGED;
    case DEV_BAD_INPUT: return EACB_ERR_BAD_INPUT;
    case DEV_FIRST_OVERFLOW: return EACB_ERR_FIRST_PARTITION_OVERFLOW;
    case DEV_CAPACITY: return EACB_ERR_WORKSPACE;
    default: return EACB_ERR_INTERNAL;
    }
}

// ---------------------------------------------------------------------------
// Workspace carving: a bump allocator over the caller's buffer.  The same
// carve sequence runs in "size" mode (base == nullptr) for the *_workspace_size
// queries, so sizes and layouts cannot drift apart.
// ---------------------------------------------------------------------------
struct Carver {
    char *base;
    size_t off;
    size_t cap;
    bool overflow;
    // a workspace that is not 256-byte aligned is refused like a short one
    // (the tensor-core and vector paths need 16-byte aligned sub-buffers)
    explicit Carver(void *b, size_t c)
        : base((char *)b), off(0), cap(c), overflow(b != nullptr && ((uintptr_t)b & 255u) != 0)
    {
    }
    template <typename T>
    T *take(size_t count)
    {
        off = (off + 255) & ~(size_t)255;
        T *p = base ? (T *)(base + off) : nullptr;
        off += count * sizeof(T);
        if (base && off > cap) overflow = true;
        return p;
    }
};

inline cudaStream_t as_stream(uintptr_t s) { return (cudaStream_t)s; }

// Raises a kernel's dynamic shared memory limit to the most the device
// allows.  Every caller sets the same value, so host threads launching the
// kernel concurrently with different requests never lower the limit under
// one another's launch (occupancy follows the request of each launch).
template <typename F>
inline cudaError_t allow_max_dyn_smem(F *func)
{
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, (const void *)func);
    if (e != cudaSuccess) return e;
    int dev = 0, optin = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) !=
        cudaSuccess)
        return e;
    return cudaFuncSetAttribute((const void *)func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)a.sharedSizeBytes);
}

inline unsigned grid_for(int64_t n, int threads, int64_t max_blocks = 148 * 32)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (unsigned)b;
}

// ---------------------------------------------------------------------------
// Warp / block scans (int64 accumulators).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t warp_incl_sum(int64_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int64_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Exclusive sum across the block; `total` receives the block sum.  The
// warp totals are combined with a Blelloch up-sweep / down-sweep in shared
// memory (work-efficient tree, 2 log2(warps) steps).
template <int THREADS>
__device__ __forceinline__ int64_t block_excl_sum(int64_t v, int64_t &total)
{
    constexpr int W = THREADS / 32;
    __shared__ int64_t tree[W];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t inc = warp_incl_sum(v);
    if (lane == 31) tree[warp] = inc;
    __syncthreads();
    if (threadIdx.x == 0) {
        // up-sweep
        for (int d = 1; d < W; d <<= 1)
            for (int i = 2 * d - 1; i < W; i += 2 * d) tree[i] += tree[i - d];
    }
    __syncthreads();
    int64_t tot = tree[W - 1];
    __syncthreads();
    if (threadIdx.x == 0) {
        tree[W - 1] = 0;
        // down-sweep
        for (int d = W >> 1; d >= 1; d >>= 1)
            for (int i = 2 * d - 1; i < W; i += 2 * d) {
                int64_t t = tree[i - d];
                tree[i - d] = tree[i];
                tree[i] += t;
            }
    }
    __syncthreads();
    int64_t r = tree[warp] + inc - v;
    total = tot;
    __syncthreads();
    return r;
}

// The same result with the warp totals combined by warp 0 in shuffles (three
// barriers, no serial steps): for the row kernels, which scan once per
// column chunk.
template <int THREADS>
__device__ __forceinline__ int64_t block_excl_sum_shfl(int64_t v, int64_t &total)
{
    constexpr int W = THREADS / 32;
    static_assert(W >= 1 && W <= 32, "one warp combines the warp totals");
    __shared__ int64_t wpre[W + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t inc = warp_incl_sum(v);
    if (lane == 31) wpre[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int64_t x = lane < W ? wpre[lane] : 0;
        const int64_t xi = warp_incl_sum(x);
        if (lane < W) wpre[lane] = xi - x;
        if (lane == 31) wpre[W] = xi;
    }
    __syncthreads();
    const int64_t r = wpre[warp] + inc - v;
    total = wpre[W];
    __syncthreads();                 // wpre is rewritten by the next call
    return r;
}

// ---------------------------------------------------------------------------
// Decoupled look-back (single-pass scan across tiles).  One 64-bit status word
// per tile: bits 63..62 = flag (0 empty, 1 aggregate, 2 inclusive prefix),
// bits 61..0 = value (two's complement, 62 bits).  Flag and value travel in
// one 64-bit access and no reader needs another tile's data, so the status
// loads and stores are relaxed (gpu scope); acquire/release ordering cost a
// fifth of the scan's bandwidth.  Tiles take their index from
// an atomic counter, so every tile a block waits on belongs to a block that is
// already running; the wait is still bounded and reports DEV_SPIN_LIMIT.
// ---------------------------------------------------------------------------
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ int64_t status_val(uint64_t s)
{
    return ((int64_t)(s << 2)) >> 2;
}

__device__ __forceinline__ void status_store(uint64_t *st, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(st), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t status_load(const uint64_t *st)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(st) : "memory");
    return v;
}

// Called by warp 0 of the block with the tile aggregate; returns (to every
// lane of warp 0) the exclusive prefix of this tile.
__device__ __forceinline__ int64_t lookback(uint64_t *status, int64_t tile, int64_t agg,
                                            int64_t init, int *err)
{
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) status_store(&status[0], kFlagInc | ((uint64_t)(init + agg) & kValMask));
        return init;
    }
    if (lane == 0) status_store(&status[tile], kFlagAgg | ((uint64_t)agg & kValMask));
    int64_t prefix = 0;
    int64_t pos = tile - 1;           // highest tile not yet folded in
    int spins = 0;
    while (true) {
        int64_t t = pos - lane;
        uint64_t s = (t >= 0) ? status_load(&status[t]) : (kFlagInc);  // t<0 never happens before an inclusive
        unsigned empty = __ballot_sync(0xffffffffu, (s >> 62) == 0);
        if (empty) {
            if (++spins > kSpinLimit) {
                if (lane == 0) set_err(err, DEV_SPIN_LIMIT);
                break;
            }
            continue;
        }
        unsigned inc = __ballot_sync(0xffffffffu, (s >> 62) == 2);
        // fold lanes [0, first inclusive] (lane 0 = tile pos)
        int stop = inc ? (__ffs(inc) - 1) : 31;
        int64_t v = (lane <= stop) ? status_val(s) : 0;
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        prefix += v;
        if (inc) break;
        pos -= 32;
    }
    if (lane == 0)
        status_store(&status[tile], kFlagInc | ((uint64_t)(prefix + agg) & kValMask));
    return prefix;
}

}  // namespace eacb

// ---------------------------------------------------------------------------
// Built-in profiling (off by default): launch counter for every kernel this
// library launches, and CUDA-event timing of tagged kernels on the stream
// they are launched on, with their algorithmic byte counts.
// ---------------------------------------------------------------------------
namespace eacb {
enum ProfTag { PROF_ROUNDS = 0, PROF_SCAN = 1, PROF_COASSOC = 2, PROF_KMEANS = 3,
               PROF_PHASE = 4, PROF_NTAGS = 8 };
struct Prof {
    int enabled;
    int64_t launches;
    double ms[PROF_NTAGS];
    double bytes[PROF_NTAGS];
    int64_t count[PROF_NTAGS];
};
Prof &prof();
// the launch counter is shared by every host thread that calls the library
inline void count_launch(int n) { __atomic_fetch_add(&prof().launches, (int64_t)n, __ATOMIC_RELAXED); }

// Times one launch when profiling is on: construct before the launch,
// call done(bytes) after it.  Synchronizes on the end event.
struct ProfScope {
    cudaEvent_t a, b;
    cudaStream_t st;
    int tag;
    bool on;
    ProfScope(int t, cudaStream_t s) : st(s), tag(t), on(prof().enabled != 0)
    {
        if (on) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, st);
        }
    }
    void done(double bytes)
    {
        if (!on) return;
        cudaEventRecord(b, st);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        prof().ms[tag] += ms;
        prof().bytes[tag] += bytes;
        prof().count[tag] += 1;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        on = false;
    }
};
}  // namespace eacb
