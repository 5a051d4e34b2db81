// Scan kernels shared by the scan entry points and by the graph/coassoc code.
#pragma once
#include "eacb_common.cuh"

namespace eacb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 24;
constexpr int64_t kScanTile = (int64_t)kScanThreads * kScanItems;

struct ScanScratch {
    uint64_t *status;
    int *counter;
    int *err;
    int64_t max_tiles;
    static ScanScratch carve(Carver &c, int64_t n, int *err = nullptr)
    {
        ScanScratch s;
        s.err = err ? err : c.take<int>(1);
        // sized for the smallest tile any single-pass kernel uses (2048)
        s.max_tiles = (n + 2047) / 2048 + 1;
        s.status = c.take<uint64_t>(s.max_tiles);
        s.counter = c.take<int>(1);
        return s;
    }
};

template <typename T> struct Vec16;
template <> struct Vec16<int32_t> { typedef int4 type; static constexpr int n = 4; };
template <> struct Vec16<int64_t> { typedef longlong2 type; static constexpr int n = 2; };

template <typename TOut>
__device__ __forceinline__ TOut narrow(int64_t v) { return (TOut)v; }
template <>
__device__ __forceinline__ int32_t narrow<int32_t>(int64_t v) { return (int32_t)(uint32_t)(uint64_t)v; }

template <typename TIn, typename TOut, bool VEC>
__global__ void __launch_bounds__(kScanThreads)
k_scan(const TIn *__restrict__ in, TOut *__restrict__ out, int64_t n, int64_t init,
       uint64_t *status, int *counter, int64_t *total, int *err, const int64_t *d_n = nullptr)
{
    __shared__ int s_tile;
    __shared__ int64_t s_prefix;
    // with d_n the length is read on the device and the grid is sized for
    // the largest length: surplus blocks take tile ids past the end and leave
    if (d_n) n = *d_n;
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile * kScanTile >= n && !(n == 0 && tile == 0)) return;
    if (n == 0) {
        if (threadIdx.x == 0 && total) *total = init;
        return;
    }
    const int64_t base = tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    TIn v[kScanItems];
    const bool full = base + kScanItems <= n;
    if (VEC && full) {
        typedef typename Vec16<TIn>::type V;
        const V *p = reinterpret_cast<const V *>(in + base);
#pragma unroll
        for (int i = 0; i < kScanItems / Vec16<TIn>::n; ++i) {
            V x = __ldcs(p + i);
            memcpy(&v[i * Vec16<TIn>::n], &x, sizeof(V));
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) v[i] = (base + i < n) ? in[base + i] : TIn(0);
    }
    int64_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) sum += (int64_t)v[i];
    int64_t agg;
    int64_t excl = block_excl_sum<kScanThreads>(sum, agg);
    if (threadIdx.x < 32) {
        int64_t pre = lookback(status, tile, agg, init, err);
        if (threadIdx.x == 0) s_prefix = pre;
    }
    __syncthreads();
    int64_t run = s_prefix + excl;
    TOut o[kScanItems];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        o[i] = narrow<TOut>(run);
        run += (int64_t)v[i];
    }
    if (VEC && full) {
        typedef typename Vec16<TOut>::type V;
        V *p = reinterpret_cast<V *>(out + base);
#pragma unroll
        for (int i = 0; i < kScanItems / Vec16<TOut>::n; ++i) {
            V x;
            memcpy(&x, &o[i * Vec16<TOut>::n], sizeof(V));
            __stcs(p + i, x);
        }
    } else {
#pragma unroll
        for (int i = 0; i < kScanItems; ++i)
            if (base + i < n) out[base + i] = o[i];
    }
    const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (tile == ntiles - 1 && threadIdx.x == 0 && total) *total = s_prefix + agg;
}

__global__ void k_set_i64(int64_t *p, int64_t v);

// Clears look-back state with a kernel (usable where memset nodes are not).
__global__ void k_clear_status(uint64_t *status, int64_t n, int *counter);

// Scan whose length is read on the device (*d_n <= max_n); no memset calls,
// so it can be captured into a conditional graph body.  With clear = false
// the caller's previous kernel has already zeroed the look-back state
// (status words [0, ceil(max_n / kScanTile)) and the tile counter).
template <typename TIn, typename TOut>
inline int scan_launch_dev(const TIn *in, TOut *out, const int64_t *d_n, int64_t max_n,
                           int64_t init, int64_t *d_total, const ScanScratch &s, cudaStream_t st,
                           bool clear = true)
{
    const int64_t ntiles = (max_n + kScanTile - 1) / kScanTile;
    const int64_t grid = ntiles > 0 ? ntiles : 1;
    if (clear) {
        k_clear_status<<<grid_for(grid, 256, 148 * 4), 256, 0, st>>>(s.status, grid, s.counter);
        EACB_CHECK_LAUNCH();
    }
    if (((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0))
        k_scan<TIn, TOut, true><<<(unsigned)grid, kScanThreads, 0, st>>>(
            in, out, max_n, init, s.status, s.counter, d_total, s.err, d_n);
    else
        k_scan<TIn, TOut, false><<<(unsigned)grid, kScanThreads, 0, st>>>(
            in, out, max_n, init, s.status, s.counter, d_total, s.err, d_n);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

template <typename TIn, typename TOut>
inline int scan_launch(const TIn *in, TOut *out, int64_t n, int64_t init, int64_t *d_total,
                       const ScanScratch &s, cudaStream_t st)
{
    if (n == 0) {
        if (d_total) {
            k_set_i64<<<1, 1, 0, st>>>(d_total, init);
            EACB_CHECK_LAUNCH();
        }
        return EACB_OK;
    }
    const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (ntiles > (int64_t)0x7fffffff) return EACB_ERR_UNSUPPORTED;
    EACB_CUDA(cudaMemsetAsync(s.status, 0, sizeof(uint64_t) * ntiles, st));
    EACB_CUDA(cudaMemsetAsync(s.counter, 0, sizeof(int), st));
    const bool vec = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0);
    if (vec)
        k_scan<TIn, TOut, true><<<(unsigned)ntiles, kScanThreads, 0, st>>>(
            in, out, n, init, s.status, s.counter, d_total, s.err);
    else
        k_scan<TIn, TOut, false><<<(unsigned)ntiles, kScanThreads, 0, st>>>(
            in, out, n, init, s.status, s.counter, d_total, s.err);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

}  // namespace eacb
