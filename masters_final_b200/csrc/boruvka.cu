// Boruvka minimum spanning forest, connected components and the EAC final
// clustering (lifetime cut) on B200.
//
// Reference: MyML/MyML/graph/mst.py:417-809 (boruvka_minho_gpu and kernels),
// MyML/MyML/graph/connected_components.py:176-345, MyML/MyML/EAC/eac.py:199-391.
//
// Design (not the reference's):
//  * Every directed edge is ONE 64-bit word: weight-order bits | min(u,v) |
//    max(u,v) | direction bit, with u, v the ORIGINAL endpoints.  A round
//    never rewrites edges; it only drops the ones that became internal.  The
//    current endpoints are label[u], label[v] (label = original vertex ->
//    current supervertex, kept for all original vertices, L2 resident).
//  * Min-edge selection is an atomicMin of a 64-bit selection key per
//    supervertex: (weight, min, max) for the MST -- a strict total order, so
//    the forest is unique -- or (weight, destination supervertex) for the
//    reference's connected-components numbering.  Lanes of a warp holding
//    edges of the same supervertex are pre-reduced with a segmented shuffle
//    scan, so one atomic is issued per run, not per edge.
//  * Contraction is a single-pass, order-preserving stream compaction
//    (decoupled look-back over 2048-edge tiles) fused with the NEXT round's
//    min-edge selection: each edge is read once and written once per round.
//  * Mutual picks are broken towards the larger id like the reference; roots
//    are found by a bounded pointer chase with path halving; supervertices are
//    renumbered by an exclusive scan of the root flags (root order), which is
//    the reference's numbering.
#include "eacb_common.cuh"
#include "scan_impl.cuh"

#include <algorithm>
#include <vector>

namespace eacb {

enum { SEL_MST = 0, SEL_CC = 1 };

struct Pack {
    int vbits;
    int wshift;      // 2*vbits + 1
    uint64_t vmask;
    __host__ __device__ uint32_t a(uint64_t k) const { return (uint32_t)((k >> (vbits + 1)) & vmask); }
    __host__ __device__ uint32_t b(uint64_t k) const { return (uint32_t)((k >> 1) & vmask); }
    __host__ __device__ uint32_t w(uint64_t k) const { return (uint32_t)(k >> wshift); }
    __host__ __device__ uint32_t src(uint64_t k) const { return (k & 1) ? b(k) : a(k); }
    __host__ __device__ uint32_t dst(uint64_t k) const { return (k & 1) ? a(k) : b(k); }
    __host__ __device__ uint64_t make(uint32_t w, uint32_t u, uint32_t v) const
    {
        uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
        return ((uint64_t)w << wshift) | ((uint64_t)lo << (vbits + 1)) | ((uint64_t)hi << 1) |
               (uint64_t)(u > v);
    }
    // MST selection key (weight, min, max) and its decoding
    __host__ __device__ uint64_t mst_sel(uint64_t k) const { return k >> 1; }
    __host__ __device__ uint32_t sel_a(uint64_t s) const { return (uint32_t)((s >> vbits) & vmask); }
    __host__ __device__ uint32_t sel_b(uint64_t s) const { return (uint32_t)(s & vmask); }
    __host__ __device__ uint32_t sel_w(uint64_t s) const { return (uint32_t)(s >> (2 * vbits)); }
};

static int make_pack(int32_t n_vertices, int wbits, Pack &pk)
{
    int vbits = 1;
    while (vbits < 31 && ((int64_t)1 << vbits) < (int64_t)n_vertices) vbits++;
    if (wbits + 2 * vbits + 1 > 64) return EACB_ERR_UNSUPPORTED;
    pk.vbits = vbits;
    pk.wshift = 2 * vbits + 1;
    pk.vmask = ((uint64_t)1 << vbits) - 1;
    return EACB_OK;
}

static int dtype_bits(int dt)
{
    switch (dt) {
    case EACB_U8: return 8;
    case EACB_U16: return 16;
    case EACB_I32: case EACB_U32: case EACB_F32: return 32;
    default: return -1;
    }
}

// Order-preserving unsigned image of a weight.
__device__ __forceinline__ uint32_t wword(uint8_t x) { return x; }
__device__ __forceinline__ uint32_t wword(uint16_t x) { return x; }
__device__ __forceinline__ uint32_t wword(uint32_t x) { return x; }
__device__ __forceinline__ uint32_t wword(int32_t x) { return (uint32_t)x ^ 0x80000000u; }
__device__ __forceinline__ uint32_t wword(float x)
{
    uint32_t u = __float_as_uint(x == 0.0f ? 0.0f : x);   // -0 == +0
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

constexpr uint64_t kNone = ~0ull;

// atomicMin that is skipped when the candidate cannot lower the slot.  Within
// a kernel the slots only decrease, so a (possibly older) L2 value that the
// candidate does not beat means the atomic would change nothing; late
// rounds, whose few supervertices receive most edges, then issue few atomics.
__device__ __forceinline__ void min_if_lower(unsigned long long *slot, uint64_t v)
{
    if (v < __ldcg(slot)) atomicMin(slot, (unsigned long long)v);
}

// One atomicMin per run of equal `su` among consecutive lanes.
__device__ __forceinline__ void seg_min_atomic(bool valid, int32_t su, uint64_t sel,
                                               unsigned long long *best)
{
    const int lane = threadIdx.x & 31;
    int32_t key = valid ? su : -1 - lane;
    int32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
    bool head = (lane == 0) || (prev != key);
    unsigned heads = __ballot_sync(0xffffffffu, head);
    int start = 31 - __clz(heads & ((2u << lane) - 1u));
    uint64_t m = valid ? sel : kNone;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t o = __shfl_up_sync(0xffffffffu, m, d);
        if (lane - d >= start) m = (o < m) ? o : m;
    }
    int32_t next = __shfl_down_sync(0xffffffffu, key, 1);
    bool tail = (lane == 31) || (next != key);
    if (valid && tail) min_if_lower(&best[su], m);
}

constexpr int kET = 256;   // edge-tile threads
constexpr int kEI = 8;     // edges per thread (striped): 2048 edges per tile
constexpr int64_t kETile = (int64_t)kET * kEI;

// Edge sources for the tile kernel ------------------------------------------
// Each source splits an edge into fetch() (independent global loads, issued
// for all items of a thread before any is used) and resolve() (the dependent
// work), so a thread keeps all its loads in flight at once.
// (a) the current edge array: fetch the word, resolve its endpoints'
//     supervertices (two gathers from the L2-resident label array)
struct SrcEdges {
    typedef uint64_t Raw;
    const uint64_t *e;
    const int32_t *label;
    Pack pk;
    uint32_t V0;
    __device__ __forceinline__ void fetch(int64_t i, Raw &r) const { r = __ldcs(e + i); }
    __device__ __forceinline__ bool resolve(const Raw &r, uint64_t &k, int32_t &su, int32_t &sv,
                                            uint32_t &w) const
    {
        k = r;
        if (pk.a(k) >= V0 || pk.b(k) >= V0) return false;   // dead words (never real edges)
        su = label[pk.src(k)];
        sv = label[pk.dst(k)];
        w = pk.w(k);
        return su != sv;
    }
};

// (b) both directions of undirected keys (MST selection keys) below a weight cap
struct SrcForest {
    typedef uint64_t Raw;
    const uint64_t *keys;   // selection keys (w, a, b)
    int64_t n_keys;
    int64_t wmax;           // keep weights <= wmax (-1 keeps none)
    Pack pk;
    __device__ __forceinline__ void fetch(int64_t i, Raw &r) const
    {
        r = keys[i < n_keys ? i : i - n_keys];
    }
    // resolve() needs the item index for the direction: passed through k
    __device__ __forceinline__ bool resolve_dir(const Raw &s, bool reverse, uint64_t &k,
                                                int32_t &su, int32_t &sv, uint32_t &w) const
    {
        w = pk.sel_w(s);
        if ((int64_t)w > wmax) return false;
        const uint32_t a = pk.sel_a(s), b = pk.sel_b(s);
        k = (s << 1) | (uint64_t)reverse;
        su = (int32_t)(reverse ? b : a);
        sv = (int32_t)(reverse ? a : b);
        return true;
    }
};

template <typename Src>
__device__ __forceinline__ bool resolve_item(const Src &src, const typename Src::Raw &r,
                                             int64_t i, uint64_t &k, int32_t &su, int32_t &sv,
                                             uint32_t &w)
{
    return src.resolve(r, k, su, sv, w);
}

template <>
__device__ __forceinline__ bool resolve_item<SrcForest>(const SrcForest &src, const uint64_t &r,
                                                        int64_t i, uint64_t &k, int32_t &su,
                                                        int32_t &sv, uint32_t &w)
{
    return src.resolve_dir(r, i >= src.n_keys, k, su, sv, w);
}

// Tile kernel: keep-filter + order-preserving compaction + fused min-edge
// selection for the next round.  eout may equal the source array (in-place
// contraction): a tile writes only after its prefix is known, i.e. after
// every earlier tile has read its input, and never past its own input end.
template <int MODE, typename Src>
__global__ void __launch_bounds__(kET)
k_edge_tile(Src src, int64_t n_in, uint64_t *eout, unsigned long long *best,
            uint64_t *status, int *counter, int64_t *d_count, int *err,
            const int64_t *d_n = nullptr)
{
    __shared__ int s_tile;
    __shared__ int s_off[kEI][kET / 32];
    __shared__ int64_t s_prefix;
    // with d_n the edge count is read on the device and the blocks loop over
    // tiles (persistent grid); tile ids are taken in increasing order, so
    // every tile a block waits on is held by a running block
    if (d_n) n_in = *d_n;
    const int64_t n_tiles = (n_in + kETile - 1) / kETile;
    for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int64_t tile = s_tile;
    __syncthreads();
    if (tile >= n_tiles) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = tile * kETile;
    typename Src::Raw raw[kEI];
#pragma unroll
    for (int it = 0; it < kEI; ++it) {
        const int64_t i = base + (int64_t)it * kET + threadIdx.x;
        if (i < n_in) src.fetch(i, raw[it]);
    }
    uint64_t k[kEI];
    int32_t su[kEI], sv[kEI];
    uint32_t w[kEI];
    bool keep[kEI];
#pragma unroll
    for (int it = 0; it < kEI; ++it) {
        const int64_t i = base + (int64_t)it * kET + threadIdx.x;
        su[it] = sv[it] = 0;
        w[it] = 0;
        k[it] = 0;
        keep[it] = (i < n_in) && resolve_item(src, raw[it], i, k[it], su[it], sv[it], w[it]);
    }
    unsigned bal[kEI];
#pragma unroll
    for (int it = 0; it < kEI; ++it) {
        bal[it] = __ballot_sync(0xffffffffu, keep[it]);
        if (lane == 0) s_off[it][warp] = __popc(bal[it]);
        const uint64_t sel =
            MODE == SEL_MST ? (k[it] >> 1) : (((uint64_t)w[it] << 32) | (uint32_t)sv[it]);
        seg_min_atomic(keep[it], su[it], sel, best);
    }
    __syncthreads();
    if (warp == 0) {
        // exclusive scan of the kEI x 8 per-warp counts in (item, warp) order
        constexpr int N = kEI * (kET / 32);
        constexpr int PER = N / 32;
        int c[PER];
        int sum = 0;
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            int idx = lane * PER + q;
            c[q] = s_off[idx / (kET / 32)][idx % (kET / 32)];
            sum += c[q];
        }
        int incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int o = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += o;
        }
        int run = incl - sum;
        int tot = __shfl_sync(0xffffffffu, incl, 31);
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            int idx = lane * PER + q;
            s_off[idx / (kET / 32)][idx % (kET / 32)] = run;
            run += c[q];
        }
        int64_t pre = lookback(status, tile, tot, 0, err);
        if (lane == 0) {
            s_prefix = pre;
            const int64_t ntiles = (n_in + kETile - 1) / kETile;
            if (tile == ntiles - 1) *d_count = pre + tot;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < kEI; ++it) {
        if (bal[it] & (1u << lane)) {
            int64_t pos = s_prefix + s_off[it][warp] + __popc(bal[it] & lt);
            eout[pos] = k[it];
        }
    }
    if (!d_n) return;            // one tile per block
    __syncthreads();             // shared state is reused by the next tile
    }
}

// Round-0 edges straight from a symmetric CSR, one warp per row: entry e
// becomes edge word e (a self loop or an entry outside every row stays a dead
// word, dropped by the first contraction); the row's minimum selection key is
// one atomicMin.
template <int MODE, typename WT>
__global__ void k_edges_csr(const int32_t *first, const int32_t *deg, const int32_t *dest,
                            const WT *weight, int32_t V, int64_t E, Pack pk, uint64_t *eout,
                            unsigned long long *best, int *err)
{
    const int lane = threadIdx.x & 31;
    for (int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < V;
         u += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t f = first[u], d = deg[u];
        if (f < 0 || d < 0 || f + d > E) {
            if (lane == 0) set_err(err, DEV_BAD_INPUT);
            continue;
        }
        uint64_t m = kNone;
        for (int64_t e = f + lane; e < f + d; e += 32) {
            const int32_t v = dest[e];
            if (v < 0 || v >= V) {
                set_err(err, DEV_BAD_INPUT);
                continue;
            }
            if (v == (int32_t)u) continue;          // self loop: stays dead
            const uint32_t w = wword(weight[e]);
            const uint64_t k = pk.make(w, (uint32_t)u, (uint32_t)v);
            eout[e] = k;
            const uint64_t sel = MODE == SEL_MST ? (k >> 1) : (((uint64_t)w << 32) | (uint32_t)v);
            m = sel < m ? sel : m;
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const uint64_t x = __shfl_xor_sync(0xffffffffu, m, o);
            m = x < m ? x : m;
        }
        if (lane == 0 && m != kNone) atomicMin(&best[u], (unsigned long long)m);
    }
}

// ---------------------------------------------------------------------------
// Weight phases (MST mode).  For a strict total order of the edges, the
// minimum spanning forest of the edges up to a key is exactly the MST
// restricted to those edges (Kruskal's prefix property).  So the forest is
// grown phase by phase over weight ranges: a phase contracts the edges of its
// range whose endpoints are still in different components, then the next
// phase starts from those components.  Heavy edges that the light ones made
// internal are dropped by one filtering read instead of being carried through
// every round.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t wbucket(uint32_t w, int wbits)
{
    return wbits <= 8 ? w : (w >> (wbits - 8));
}

// 256-bin histograms.  Weights are heavily skewed (most co-association
// dissimilarities sit in a few top bins), so a shared atomic per element
// would serialise on those bins: lanes of a warp holding the same bin combine
// first (match_any), and every warp owns a private copy of the bins.
constexpr int kHistThreads = 256;

__device__ __forceinline__ void hist_add(unsigned *h, uint32_t b, bool valid)
{
    const unsigned act = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const unsigned peers = __match_any_sync(act, b);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[b], (unsigned)__popc(peers));
}

__device__ __forceinline__ void hist_flush(unsigned (*h)[256], unsigned long long *hist)
{
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        unsigned long long t = 0;
        for (int w = 0; w < kHistThreads / 32; ++w) t += h[w][b];
        if (t) atomicAdd(&hist[b], t);
    }
}

template <typename WT>
__global__ void __launch_bounds__(kHistThreads)
k_whist_csr(const WT *weight, int64_t E, int wbits, unsigned long long *hist)
{
    __shared__ unsigned h[kHistThreads / 32][256];
    for (int i = threadIdx.x; i < (kHistThreads / 32) * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    unsigned *mine = h[threadIdx.x >> 5];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // the loop bound is warp-uniform (match_any needs the whole warp)
    for (int64_t e0 = (int64_t)blockIdx.x * blockDim.x; e0 < E; e0 += stride) {
        const int64_t e = e0 + threadIdx.x;
        const bool ok = e < E;
        hist_add(mine, ok ? wbucket(wword(weight[e]), wbits) & 255 : 0, ok);
    }
    hist_flush(h, hist);
}

// uint8 weights, 16 per thread per step (128-bit loads).  Every lane owns a
// private column of 256 counters (bank = lane, so no conflicts and no
// atomics): counts[warp][bin][lane], 32 KB per warp, two warps per block.
constexpr int kHist8Threads = 64;
constexpr size_t kHist8Smem = (size_t)(kHist8Threads / 32) * 256 * 32 * sizeof(uint32_t);
__global__ void __launch_bounds__(kHist8Threads, 1)
k_whist_u8(const uint8_t *w, int64_t n, unsigned long long *hist)
{
    extern __shared__ uint32_t hs[];
    for (int i = threadIdx.x; i < (kHist8Threads / 32) * 256 * 32; i += blockDim.x) hs[i] = 0;
    __syncthreads();
    uint32_t *mine = hs + (threadIdx.x >> 5) * 256 * 32 + (threadIdx.x & 31);
    int64_t head = (int64_t)((16 - ((uintptr_t)w & 15)) & 15);
    if (head > n) head = n;
    const int64_t nv = (n - head) >> 4;               // whole 16-byte vectors
    const uint4 *v = reinterpret_cast<const uint4 *>(w + head);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    auto add16 = [&](const uint4 &x) {
        const uint32_t wd[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int k = 0; k < 16; ++k)     // no-return adds: equal bytes do not serialise
            atomicAdd(&mine[((wd[k >> 2] >> (8 * (k & 3))) & 255u) * 32], 1u);
    };
    // few warps fit beside the private columns, so each thread keeps eight
    // 16-byte loads in flight
    constexpr int kU = 8;
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; q + (kU - 1) * stride < nv; q += kU * stride) {
        uint4 x[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) x[u] = __ldcs(v + q + u * stride);
        // all eight loads are issued before the first is consumed
#pragma unroll
        for (int u = 0; u < kU; ++u)
            asm volatile("" : "+r"(x[u].x), "+r"(x[u].y), "+r"(x[u].z), "+r"(x[u].w));
#pragma unroll
        for (int u = 0; u < kU; ++u) add16(x[u]);
    }
    for (; q < nv; q += stride) add16(__ldcs(v + q));
    // the unaligned head and the ragged tail (< 32 bytes), by the first block
    if (blockIdx.x == 0) {
        const int64_t tail0 = head + (nv << 4);
        const int64_t rest = head + (n - tail0);
        const int64_t t = threadIdx.x;
        if (t < rest) mine[(uint32_t)w[t < head ? t : tail0 + (t - head)] * 32] += 1;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x) {
        unsigned long long tot = 0;
        for (int wp = 0; wp < kHist8Threads / 32; ++wp)
            for (int l = 0; l < 32; ++l) tot += hs[(wp * 256 + b) * 32 + l];
        if (tot) atomicAdd(&hist[b], tot);
    }
}

static int launch_whist_u8(const uint8_t *w, int64_t n, unsigned long long *hist, cudaStream_t st)
{
    EACB_CUDA(allow_max_dyn_smem(k_whist_u8));
    k_whist_u8<<<grid_for((n + 15) / 16, kHist8Threads, 148 * 3), kHist8Threads, kHist8Smem,
                 st>>>(w, n, hist);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

// Phase builds: the edges of a weight-bucket range (lo, hi] whose endpoints
// are in different components, appended to eout, with the first round's
// minimum-edge selection.  The rows of a block step reserve their output
// slots with one atomicAdd, which keeps the shared cursor off the critical
// path.  Edge order is not deterministic, results are: selection uses a
// strict total order.
constexpr int kPhThreads = 256;
constexpr int kPhWarps = kPhThreads / 32;

// Exclusive offsets of the block's per-warp counts in s_cnt and one
// reservation of mult * total slots.  A reservation that would pass `cap`
// (the output capacity) writes nothing and raises DEV_CAPACITY; it returns
// false to every thread of the block.
__device__ __forceinline__ bool phase_reserve(int64_t *s_cnt, unsigned long long *s_base,
                                              unsigned long long *cursor, int mult,
                                              unsigned long long cap, int *err)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t tot = 0;
        for (int w = 0; w < kPhWarps; ++w) {
            const int64_t c = s_cnt[w];
            s_cnt[w] = tot;
            tot += c;
        }
        const unsigned long long need = (unsigned long long)(mult * tot);
        const unsigned long long b = tot ? atomicAdd(cursor, need) : 0ull;
        *s_base = b;
        s_ok = b + need <= cap;
        if (!s_ok) set_err(err, DEV_CAPACITY);
    }
    __syncthreads();
    return s_ok != 0;
}

// Graph rows are short (degrees), so a warp takes 32 consecutive rows per
// block step, one row per lane for the row data.  When the 32 rows lie back
// to back in the CSR (the usual layout), the warp walks their entries as one
// flat range, 32 entries per step, each lane finding its entry's row among
// the lanes' row starts (a 5-step shuffle search): the dependent loads of
// all 32 rows overlap instead of running row after row.  Otherwise it walks
// the rows one by one.  Kept words are staged in shared memory; the block
// reserves once per step and copies them out coalesced (a warp whose
// staging fills up flushes it on its own).
constexpr int kPhStage = 512;            // staged words per warp

__device__ __forceinline__ void phase_flush_warp(const uint64_t *stage, int cnt, uint64_t *eout,
                                                 unsigned long long *cursor,
                                                 unsigned long long cap, int *err)
{
    const int lane = threadIdx.x & 31;
    unsigned long long b = 0;
    if (lane == 0) b = atomicAdd(cursor, (unsigned long long)cnt);
    b = __shfl_sync(0xffffffffu, b, 0);
    if (b + cnt > cap) {
        if (lane == 0) set_err(err, DEV_CAPACITY);
        return;
    }
    for (int i = lane; i < cnt; i += 32) eout[b + i] = stage[i];
}

// Appends one candidate per lane to the warp's staging (flushing first when
// it would overflow).
__device__ __forceinline__ void phase_stage(bool keep, uint64_t k, uint64_t *stage, int &cnt,
                                            uint64_t *eout, unsigned long long *cursor,
                                            unsigned long long cap, int *err)
{
    const int lane = threadIdx.x & 31;
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int nb = __popc(bal);
    if (cnt + nb > kPhStage) {
        __syncwarp();
        phase_flush_warp(stage, cnt, eout, cursor, cap, err);
        __syncwarp();
        cnt = 0;
    }
    if (keep) stage[cnt + __popc(bal & ((1u << lane) - 1u))] = k;
    cnt += nb;
}

template <typename WT>
__global__ void __launch_bounds__(kPhThreads)
k_phase_csr(const int32_t *first, const int32_t *deg, const int32_t *dest, const WT *weight,
            int32_t V, int64_t E, int wbits, int lo, int hi, const int *dev_lohi, int slot,
            const int32_t *label, Pack pk, uint64_t *eout, unsigned long long *cursor,
            unsigned long long cap, unsigned long long *best, int *err)
{
    if (dev_lohi) {
        lo = dev_lohi[2 * slot];
        hi = dev_lohi[2 * slot + 1];
    }
    __shared__ uint64_t stage_all[kPhWarps][kPhStage];
    __shared__ int64_t s_cnt[kPhWarps];
    __shared__ unsigned long long s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *stage = stage_all[warp];
    const int64_t step = (int64_t)kPhWarps * 32;
    // entry test: the candidate word of entry e of row u (supervertex lu)
    auto test = [&](int64_t e, int64_t u, int32_t lu, uint64_t &k) -> bool {
        const int32_t v = dest[e];
        if (v < 0 || v >= V) {
            set_err(err, DEV_BAD_INPUT);
            return false;
        }
        if (v == (int32_t)u) return false;
        const uint32_t w = wword(weight[e]);
        const int bk = (int)wbucket(w, wbits);
        if (bk <= lo || bk > hi || label[v] == lu) return false;
        k = pk.make(w, (uint32_t)u, (uint32_t)v);
        return true;
    };
    for (int64_t r0 = (int64_t)blockIdx.x * step; r0 < V; r0 += (int64_t)gridDim.x * step) {
        const int64_t u0 = r0 + (int64_t)warp * 32;
        const int nrows = u0 >= V ? 0 : (int)(V - u0 < 32 ? V - u0 : 32);
        int64_t f = 0, d = 0;
        int32_t lu = 0;
        if (lane < nrows) {
            f = first[u0 + lane];
            d = deg[u0 + lane];
            if (f < 0 || d < 0 || f + d > E) {
                set_err(err, DEV_BAD_INPUT);
                f = 0;
                d = 0;
            }
            lu = label[u0 + lane];
        }
        // rows back to back?  (row l + 1 starts where row l ends)
        const int64_t f_next = __shfl_down_sync(0xffffffffu, f, 1);
        const bool linked = lane + 1 >= nrows || f_next == f + d;
        const int64_t e_begin = __shfl_sync(0xffffffffu, f, 0);
        const int64_t e_end = nrows > 0 ? __shfl_sync(0xffffffffu, f + d, nrows - 1) : 0;
        const bool flat = __all_sync(0xffffffffu, linked) && nrows > 0 &&
                          e_end - e_begin < ((int64_t)1 << 30);
        int cnt = 0;
        if (flat) {
            const int32_t frel = (int32_t)(f - e_begin);      // row starts, warp-relative
            // four 32-entry slices per step, the loads of all in flight together
            constexpr int S = 4;
            for (int64_t e0 = e_begin; e0 < e_end; e0 += 32 * S) {
                int64_t e[S];
                int r[S];
                int32_t lr[S], v[S];
                uint32_t w[S];
                bool in[S];
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    e[q] = e0 + 32 * q + lane;
                    in[q] = e[q] < e_end;
                    const int32_t erel = (int32_t)(e[q] - e_begin);
                    // row of entry e: the last row starting at or before e
                    int rr = 0;
#pragma unroll
                    for (int st = 16; st >= 1; st >>= 1) {
                        const int c = rr + st;
                        const int32_t fs = __shfl_sync(0xffffffffu, frel, c & 31);
                        if (c < nrows && fs <= erel) rr = c;
                    }
                    r[q] = rr;
                    lr[q] = __shfl_sync(0xffffffffu, lu, rr);
                    v[q] = in[q] ? dest[e[q]] : -1;
                    w[q] = in[q] ? wword(weight[e[q]]) : 0u;
                }
                bool cand[S];
                int32_t lv[S];
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    cand[q] = false;
                    if (in[q]) {
                        if (v[q] < 0 || v[q] >= V) {
                            set_err(err, DEV_BAD_INPUT);
                        } else if (v[q] != (int32_t)(u0 + r[q])) {
                            const int bk = (int)wbucket(w[q], wbits);
                            cand[q] = bk > lo && bk <= hi;
                        }
                    }
                    lv[q] = cand[q] ? label[v[q]] : 0;
                }
#pragma unroll
                for (int q = 0; q < S; ++q) {
                    const bool keep = cand[q] && lv[q] != lr[q];
                    const uint64_t k =
                        keep ? pk.make(w[q], (uint32_t)(u0 + r[q]), (uint32_t)v[q]) : 0ull;
                    phase_stage(keep, k, stage, cnt, eout, cursor, cap, err);
                    if (keep) min_if_lower(&best[lr[q]], k >> 1);
                }
            }
        } else {
            for (int rr = 0; rr < nrows; ++rr) {
                const int64_t fr = __shfl_sync(0xffffffffu, f, rr);
                const int64_t dr = __shfl_sync(0xffffffffu, d, rr);
                const int32_t lr = __shfl_sync(0xffffffffu, lu, rr);
                for (int64_t e0 = fr; e0 < fr + dr; e0 += 32) {
                    const int64_t e = e0 + lane;
                    uint64_t k = 0;
                    const bool keep = e < fr + dr && test(e, u0 + rr, lr, k);
                    phase_stage(keep, k, stage, cnt, eout, cursor, cap, err);
                    if (keep) min_if_lower(&best[lr], k >> 1);
                }
            }
        }
        if (lane == 0) s_cnt[warp] = cnt;
        const bool fits = phase_reserve(s_cnt, &s_base, cursor, 1, cap, err);
        if (fits) {
            const unsigned long long at = s_base + (unsigned long long)s_cnt[warp];
            for (int i = lane; i < cnt; i += 32) eout[at + i] = stage[i];
        }
        __syncthreads();          // staging and s_cnt are reused by the next step
    }
}

// Same for an upper-triangle CSR with uint8 weights: both directions of each
// kept entry.  Co-association rows are long (thousands of entries), so a
// warp takes one row and walks it in 128-entry groups, each lane taking four
// consecutive entries: their four weights (one word) are read first, and the
// four column indices (16 bytes) only when one of the weights falls in the
// phase's range, so a phase over a narrow range reads little more than the
// weight array; only those entries gather the other end's label.  A first
// walk (four groups in flight) counts the kept entries, the warp reserves
// 2 x that many words with one atomic, and a second walk over the (now
// cached) row writes them: per group its i -> j words, then its j -> i words,
// runs of equal source for the min-edge selection of later rounds.  Each
// entry is checked (j > i, j < n) in the phase whose range holds its weight.
__global__ void __launch_bounds__(kPhThreads, 4)
k_phase_upper(const int64_t *indptr, const int32_t *indices, const uint8_t *w, int32_t n,
              int64_t nnz, int lo, int hi, int dense, int64_t row0, int64_t row1,
              const int32_t *label, Pack pk, uint64_t *eout, unsigned long long *cursor,
              unsigned long long cap, unsigned long long *best, unsigned long long *khist,
              int *err)
{
    constexpr int G = 4;
    __shared__ unsigned s_kh[256];           // kept entries per weight, this block
    for (int b = threadIdx.x; b < 256; b += blockDim.x) s_kh[b] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * kPhWarps;
    for (int64_t i = row0 + (int64_t)blockIdx.x * kPhWarps + (threadIdx.x >> 5); i < row1;
         i += nwarps) {
        const int64_t s = indptr[i], e_end = indptr[i + 1];
        if (s < 0 || e_end < s || e_end > nnz) {
            if (lane == 0) set_err(err, DEV_BAD_INPUT);
            continue;
        }
        if (s == e_end) continue;
        const int32_t li = label[i];
        const int64_t a0 = s & ~(int64_t)3;        // groups start on 16-byte index boundaries
        // weights of the lane's entries e .. e+3 (zero outside the arrays)
        auto wload = [&](int64_t e) -> uint32_t {
            if (e >= e_end) return 0u;
            if (e + 3 < nnz) return __ldg(reinterpret_cast<const uint32_t *>(w + e));
            uint32_t v = 0u;
            for (int q = 0; q < 4 && e + q < nnz; ++q) v |= (uint32_t)w[e + q] << (8 * q);
            return v;
        };
        // bit q: entry e+q is in the row with its weight in (lo, hi]; four
        // byte compares at once, the row's bounds only in its edge groups
        const uint32_t lo4 = 0x01010101u * (uint32_t)(lo + 1), hi4 = 0x01010101u * (uint32_t)hi;
        auto cmask = [&](int64_t e, uint32_t wv) -> unsigned {
            uint32_t m = __vcmpgeu4(wv, lo4) & __vcmpleu4(wv, hi4);
            if (e < s || e + 4 > e_end) {
                const int64_t a = s - e, b = e_end - e;     // valid bytes [a, b)
                const int qa = a < 0 ? 0 : (a > 4 ? 4 : (int)a);
                const int qb = b < 0 ? 0 : (b > 4 ? 4 : (int)b);
                const uint32_t va = qa >= 4 ? 0u : 0xffffffffu << (8 * qa);
                const uint32_t vb = qb <= 0 ? 0u : 0xffffffffu >> (8 * (4 - qb));
                m &= va & vb;
            }
            return ((m >> 7) & 1u) | ((m >> 14) & 2u) | ((m >> 21) & 4u) | ((m >> 28) & 8u);
        };
        // the indices of the entries in cm (all four in a dense phase)
        auto jload = [&](int64_t e, unsigned cm) -> int4 {
            if (dense) cm = e < e_end ? 15u : 0u;
            if (!cm) return make_int4(0, 0, 0, 0);
            if (e + 3 < nnz) return __ldg(reinterpret_cast<const int4 *>(indices + e));
            int32_t t[4] = {0, 0, 0, 0};
            for (int q = 0; q < 4; ++q)
                if (((cm >> q) & 1u) && e + q < nnz) t[q] = indices[e + q];
            return make_int4(t[0], t[1], t[2], t[3]);
        };
        // bit q: candidate q is kept (other end in another component); lj
        // receives the candidates' other-end labels
        auto keep = [&](unsigned cm, const int4 &jv, int32_t (&lj)[4]) -> unsigned {
            const int32_t jj[4] = {jv.x, jv.y, jv.z, jv.w};
            unsigned c2 = cm;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (((cm >> q) & 1u) && (jj[q] <= i || jj[q] >= n)) {
                    set_err(err, DEV_BAD_INPUT);
                    c2 &= ~(1u << q);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) lj[q] = ((c2 >> q) & 1u) ? label[jj[q]] : li;
            unsigned km = 0u;
#pragma unroll
            for (int q = 0; q < 4; ++q) km |= (lj[q] != li ? 1u : 0u) << q;
            return km;
        };
        int cnt = 0;
        for (int64_t g = a0; g < e_end; g += 128 * G) {
            uint32_t wv[G];
            unsigned cm[G];
            int4 jv[G];
            if (dense) {
                // most entries are in range: the indices are read beside the
                // weights instead of after them
#pragma unroll
                for (int u = 0; u < G; ++u) {
                    wv[u] = wload(g + 128 * u + 4 * lane);
                    jv[u] = jload(g + 128 * u + 4 * lane, 0u);
                }
#pragma unroll
                for (int u = 0; u < G; ++u) cm[u] = cmask(g + 128 * u + 4 * lane, wv[u]);
            } else {
#pragma unroll
                for (int u = 0; u < G; ++u) wv[u] = wload(g + 128 * u + 4 * lane);
#pragma unroll
                for (int u = 0; u < G; ++u) {
                    cm[u] = cmask(g + 128 * u + 4 * lane, wv[u]);
                    jv[u] = jload(g + 128 * u + 4 * lane, cm[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < G; ++u) {
                int32_t lj[4];
                const unsigned km = keep(cm[u], jv[u], lj);
                cnt += __popc(km);
                for (unsigned b = km; b; b &= b - 1u)
                    atomicAdd(&s_kh[(wv[u] >> (8 * (__ffs(b) - 1))) & 255u], 1u);
            }
        }
        cnt = __reduce_add_sync(0xffffffffu, cnt);
        if (cnt == 0) continue;
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(cursor, 2ull * (unsigned long long)cnt);
        at = __shfl_sync(0xffffffffu, at, 0);
        if (at + 2ull * (unsigned long long)cnt > cap) {
            if (lane == 0) set_err(err, DEV_CAPACITY);
            continue;
        }
        uint64_t m = kNone;
        for (int64_t g = a0; g < e_end; g += 128) {
            const int64_t e = g + 4 * lane;
            const uint32_t wv = wload(e);
            const unsigned cm = cmask(e, wv);
            const int4 jv = jload(e, cm);
            int32_t lj[4];
            const unsigned km = keep(cm, jv, lj);
            const int c = __popc(km);
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += o;
            }
            const int tot = __shfl_sync(0xffffffffu, incl, 31);
            if (tot == 0) continue;
            unsigned long long p = at + (unsigned long long)(incl - c);
            const int32_t jj[4] = {jv.x, jv.y, jv.z, jv.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!((km >> q) & 1u)) continue;
                const uint64_t k = pk.make((wv >> (8 * q)) & 255u, (uint32_t)i, (uint32_t)jj[q]);
                eout[p] = k;
                eout[p + tot] = k | 1ull;
                m = (k >> 1) < m ? (k >> 1) : m;
                min_if_lower(&best[lj[q]], k >> 1);
                ++p;
            }
            at += 2ull * (unsigned long long)tot;
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const uint64_t x = __shfl_xor_sync(0xffffffffu, m, o);
            m = x < m ? x : m;
        }
        if (lane == 0 && m != kNone) min_if_lower(&best[li], m);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < 256; b += blockDim.x)
        if (s_kh[b]) atomicAdd(&khist[b], (unsigned long long)s_kh[b]);
}

// One phase: the entries with weight bucket in (lo, hi] of rows [r0, r1);
// with slot >= 0 the range is read on the device from the plan's slot.
struct Phase {
    int lo, hi;
    int64_t r0, r1;
    int slot;
};

// Phase ranges (lo, hi] of weight buckets: cut the bucket histogram at the
// given cumulative fractions of the entries.
__host__ __device__ static int phase_ranges(const unsigned long long *hist, const double *fracs,
                                            int nf, int *lo, int *hi)
{
    unsigned long long tot = 0;
    for (int b = 0; b < 256; ++b) tot += hist[b];
    int np = 0, prev = -1;
    unsigned long long acc = 0;
    int b = 0;
    for (int f = 0; f < nf; ++f) {
        const double target = fracs[f] * (double)tot;
        while (b < 255 && (double)(acc + hist[b]) < target) acc += hist[b++];
        const int cut = (f == nf - 1) ? 255 : b;
        if (cut > prev) {
            lo[np] = prev;
            hi[np] = cut;
            np++;
            prev = cut;
        }
        if (cut == 255) break;
        acc += hist[b];
        b++;
    }
    if (prev < 255) {
        lo[np] = prev;
        hi[np] = 255;
        np++;
    }
    return np;
}

// The weight phases of an MST on the device (no host read): ranges (lo, hi]
// at cumulative fractions 1/8, 1/2, 1 of the histogram, one slot each in
// lohi (an unused slot holds the empty range (255, 255]).
constexpr int kPhaseSlots = 3;
__global__ void k_phase_plan(const unsigned long long *hist, int *lohi)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double fracs[kPhaseSlots] = {0.125, 0.5, 1.0};
    int lo[8], hi[8];
    const int np = phase_ranges(hist, fracs, kPhaseSlots, lo, hi);
    for (int q = 0; q < kPhaseSlots; ++q) {
        lohi[2 * q] = q < np ? lo[q] : 255;
        lohi[2 * q + 1] = q < np ? hi[q] : 255;
    }
}

__global__ void k_iota(int32_t *a, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        a[i] = (int32_t)i;
}

constexpr int kMaxRounds = 96;   // Boruvka rounds per phase (halving: 96 is never reached)

// Round state kept on the device, so that a round needs no host value and
// the rounds can loop inside one CUDA graph (see Engine::run):
enum : int {
    C_E_NEXT = 0,     // edges after this round's contraction (filter total)
    C_V_NEXT = 1,     // supervertices after this round (root-scan total)
    C_EMIT = 2,       // forest edges emitted this round (emit-scan total)
    C_CURSOR = 3,     // phase-build output cursor
    C_V = 4,          // supervertices at the start of the round
    C_E = 5,          // edges at the start of the round
    C_NMST = 6,       // forest edges emitted so far (all phases)
    C_ROUNDS = 7,     // rounds run in this phase
    C_DONE = 8,       // 1 once the phase has converged
    C_ROUNDS_ALL = 9, // rounds run since the engine's reset (all phases)
    C_COUNT = 16
};

// successor of each supervertex from its selected key
template <int MODE>
__global__ void k_select(const unsigned long long *best, int32_t *succ, const int64_t *dV,
                         const int32_t *label, Pack pk)
{
    const int64_t V = *dV;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < V;
         s += (int64_t)gridDim.x * blockDim.x) {
        uint64_t b = best[s];
        int32_t t = (int32_t)s;
        if (b != kNone) {
            if (MODE == SEL_CC) {
                t = (int32_t)(uint32_t)b;
            } else {
                int32_t la = label[pk.sel_a(b)], lb = label[pk.sel_b(b)];
                t = (la == (int32_t)s) ? lb : la;
            }
        }
        succ[s] = t;
    }
}

// Look-back state of the next single-pass kernel, cleared by the kernel
// before it (one launch fewer per scan).
__device__ __forceinline__ void clear_lookback(uint64_t *status, int64_t n_status, int *counter)
{
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t i = t0; i < n_status; i += (int64_t)gridDim.x * blockDim.x) status[i] = 0;
    if (t0 == 0) *counter = 0;
}

// mutual picks: the smaller id drops its edge (MyML/MyML/graph/mst.py:283-305)
__global__ void k_mirror(const int32_t *succ, int32_t *color, int32_t *emit, const int64_t *dV,
                         uint64_t *status, int64_t n_status, int *counter)
{
    const int64_t V = *dV;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < V;
         s += (int64_t)gridDim.x * blockDim.x) {
        int32_t t = succ[s];
        bool has = t != (int32_t)s;
        bool drop = has && succ[t] == (int32_t)s && (int32_t)s < t;
        color[s] = (has && !drop) ? t : (int32_t)s;
        if (emit) emit[s] = (has && !drop) ? 1 : 0;
    }
    clear_lookback(status, n_status, counter);
}

// One pass per supervertex s: (MST) emits its selected edge at its scanned
// position, appended after the forest edges of earlier rounds; finds its root
// by pointer chasing with path halving, bounded (a non-forest errors); flags
// roots for the renumbering scan.  A halving step replaces c's parent p by
// its grandparent g only if c still points at p (compare-and-swap): a plain
// store could overwrite the root that c's own thread already stored, leaving
// c on a non-root.  s is a root exactly when its own chase ends at s.
__global__ void k_jump(int32_t *color, const int64_t *dV, int *err,
                       const unsigned long long *best, int32_t *flag, const int32_t *pos,
                       uint64_t *out, const int64_t *d_base, uint64_t *status, int64_t n_status,
                       int *counter)
{
    const int64_t V = *dV;
    uint64_t *o = out ? out + *d_base : nullptr;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < V;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (o && flag[s]) o[pos[s]] = best[s];
        int32_t c = color[s];
        int64_t guard = 0;
        while (true) {
            int32_t p = color[c];
            if (p == c) break;
            int32_t g = color[p];
            if (g != p) atomicCAS(&color[c], p, g);
            c = g;
            if (++guard > (int64_t)V + 64) {
                set_err(err, DEV_CHASE_LIMIT);
                break;
            }
        }
        color[s] = c;
        flag[s] = c == (int32_t)s;
    }
    clear_lookback(status, n_status, counter);
}

// Relabels every original vertex to its new supervertex id, and clears the
// next round's selection (Vn supervertices) and the contraction's look-back
// state.
__global__ void k_relabel(int32_t *label, const int32_t *color, const int32_t *newid, int64_t V0,
                          unsigned long long *best, const int64_t *dVn, uint64_t *status,
                          int64_t n_status, int *counter, int64_t *d_count)
{
    const int64_t Vn = *dVn;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t x = t0; x < V0; x += stride) label[x] = newid[color[label[x]]];
    for (int64_t x = t0; x < Vn; x += stride) best[x] = kNone;
    clear_lookback(status, n_status, counter);
    if (t0 == 0) *d_count = 0;
}

// Start of a phase queued without a host read: its edge count is the
// build's cursor, its supervertex count the previous phase's result (V0
// for the first phase).
__global__ void k_phase_begin(int64_t *cnt, int64_t V0, int first_phase)
{
    if (threadIdx.x == 0) {
        if (first_phase) cnt[C_V] = V0;
        cnt[C_E] = cnt[C_CURSOR];
        cnt[C_ROUNDS] = 0;
        cnt[C_DONE] = 0;
    }
}

__global__ void k_round_begin(int64_t *cnt, int64_t V, int64_t E)
{
    if (threadIdx.x == 0) {
        cnt[C_V] = V;
        cnt[C_E] = E;
        cnt[C_ROUNDS] = 0;
        cnt[C_DONE] = 0;
    }
}

// End of a round: advance the sizes and decide whether another round runs.
// cnt[C_DONE]: 0 = continue, 1 = converged (one supervertex or no edge
// left), 2 = no contraction (an error), 3 = round limit, 4 = device error.
// Inside a graph, the loop condition is cleared when the phase is done.
// A phase that stops without converging (no contraction, or the round limit
// when that limit is not a deliberate stop) also raises DEV_CHASE_LIMIT, so
// phases queued after it report the failure at the end.
__global__ void k_round_end(int64_t *cnt, int is_mst, int max_rounds, int *err,
                            cudaGraphConditionalHandle h, int use_handle)
{
    if (threadIdx.x != 0) return;
    const int64_t V = cnt[C_V], Vn = cnt[C_V_NEXT], En = cnt[C_E_NEXT];
    if (is_mst) cnt[C_NMST] += cnt[C_EMIT];
    const int64_t r = ++cnt[C_ROUNDS];
    ++cnt[C_ROUNDS_ALL];
    int64_t done = 0;
    if (*(volatile const int *)err) done = 4;
    else if (Vn <= 1 || En == 0) done = 1;
    else if (Vn >= V) done = 2;
    else if (r >= max_rounds) done = 3;
    if (done == 2 || (done == 3 && max_rounds >= kMaxRounds)) set_err(err, DEV_CHASE_LIMIT);
    cnt[C_DONE] = done;
    cnt[C_V] = Vn;
    cnt[C_E] = En;
    if (use_handle) cudaGraphSetConditional(h, done ? 0u : 1u);
}

// MST selection key -> index of its entry in row min(u,v) of a symmetric CSR
// (the smallest index with the key's destination and weight).  One thread
// per key scans the row, four entries per step with their loads in flight:
// graph rows are short, and a thread per key keeps every key's dependent
// loads (key -> row extent -> entries) overlapping with all the others.
template <typename WT>
__global__ void k_key2eid(const uint64_t *keys, int64_t n_keys, const int32_t *first,
                          const int32_t *deg, const int32_t *dest, const WT *weight, Pack pk,
                          int32_t *out, int *err)
{
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n_keys;
         q += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t s = keys[q];
        const int32_t a = (int32_t)pk.sel_a(s), b = (int32_t)pk.sel_b(s);
        const uint32_t w = pk.sel_w(s);
        const int64_t f = first[a], d = deg[a];
        int64_t found = -1;
        for (int64_t e0 = f; e0 < f + d && found < 0; e0 += 4) {
            int32_t v[4];
            uint32_t ww[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int64_t e = e0 + i;
                v[i] = e < f + d ? dest[e] : -1;
                ww[i] = e < f + d ? wword(weight[e]) : 0u;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (found < 0 && v[i] == b && ww[i] == w) found = e0 + i;
        }
        if (found < 0) set_err(err, DEV_BAD_INPUT);   // graph not symmetric
        out[q] = (int32_t)found;
    }
}

// ---------------------------------------------------------------------------
// Host-side engine
// ---------------------------------------------------------------------------
struct Engine {
    int *err;
    int64_t *cnt;             // round state, indexed by C_E_NEXT .. C_DONE
    uint64_t *ea, *eb;
    int32_t *label;
    unsigned long long *best;
    int32_t *succ, *color, *flag, *pos;
    uint64_t *mst;
    unsigned long long *hist; // 256 weight buckets
    int *lohi;                // the device phase plan (k_phase_plan)
    ScanScratch scan;
    int32_t V0;
    int64_t Emax;
    int64_t mst_base = 0;     // forest edges emitted by earlier phases
    int max_rounds = kMaxRounds;   // lowered only by the round-trace debug entry point

    static Engine carve(Carver &c, int32_t V0, int64_t Emax)
    {
        Engine g;
        g.err = c.take<int>(1);
        g.cnt = c.take<int64_t>(C_COUNT);
        g.hist = c.take<unsigned long long>(256);
        g.lohi = c.take<int>(2 * kPhaseSlots);
        g.V0 = V0;
        g.Emax = Emax;
        // one edge array (contraction is in place); eb holds the two
        // directions of a forest (at most 2 V0 words) for the final clustering
        g.ea = c.take<uint64_t>(Emax > 0 ? Emax : 1);
        g.eb = c.take<uint64_t>(2 * (size_t)V0);
        g.label = c.take<int32_t>(V0);
        g.best = c.take<unsigned long long>(V0);
        g.succ = c.take<int32_t>(V0);
        g.color = c.take<int32_t>(V0);
        g.flag = c.take<int32_t>(V0);
        g.pos = c.take<int32_t>(V0);
        g.mst = c.take<uint64_t>(V0);
        g.scan = ScanScratch::carve(c, Emax > V0 ? Emax : V0, g.err);
        return g;
    }

    int read_counts(cudaStream_t st, int64_t h[3])
    {
        int e = 0;
        EACB_CUDA(cudaMemcpyAsync(h, cnt, 3 * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaStreamSynchronize(st));
        return dev_err_to_status(e);
    }

    // MST by weight phases (see k_phase_csr).  `hist` must hold the 256-bucket
    // weight histogram; build(lo, hi) launches one phase's edge build into ea
    // (slots reserved through cnt[C_CURSOR]) with its selection into best.
    int read_hist(cudaStream_t st, unsigned long long h[256])
    {
        EACB_CUDA(cudaMemcpyAsync(h, hist, 256 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaStreamSynchronize(st));
        return EACB_OK;
    }

    template <typename Build>
    int run_phased(Pack pk, const std::vector<Phase> &plan, Build build, cudaStream_t st,
                   int64_t *n_mst_out, int64_t *n_comp_out)
    {
        if (prof().enabled == 0 && max_rounds >= kMaxRounds) {
            int per_round = 0;
            cudaGraphExec_t exec = round_graph<SEL_MST>(pk, &per_round);
            if (exec) return run_phased_graph(plan, build, exec, per_round, st, n_mst_out,
                                              n_comp_out);
        }
        int32_t V = V0;
        mst_base = 0;
        for (const Phase &ph : plan) {
            EACB_CUDA(cudaMemsetAsync(best, 0xff, sizeof(uint64_t) * V, st));
            EACB_CUDA(cudaMemsetAsync(&cnt[C_CURSOR], 0, sizeof(int64_t), st));
            EACB_CUDA(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned long long), st));
            int s = build(ph);
            if (s) return s;
            int64_t Ep = 0;
            int e = 0;
            EACB_CUDA(cudaMemcpyAsync(&Ep, &cnt[C_CURSOR], sizeof(int64_t), cudaMemcpyDeviceToHost,
                                      st));
            EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaStreamSynchronize(st));
            if (e) return dev_err_to_status(e);
            if (Ep > Emax) return EACB_ERR_INTERNAL;
            if (prof().enabled) prof().bytes[PROF_PHASE] += 8.0 * (double)Ep;   // words written
            int64_t nm = 0, nc = 0;
            if ((s = run<SEL_MST>(pk, Ep, V, st, &nm, &nc))) return s;
            mst_base += nm;
            V = (int32_t)nc;
            if (V <= 1) break;
        }
        *n_mst_out = mst_base;
        *n_comp_out = V;
        return EACB_OK;
    }

    // Phases in order with a host read after each build (the final
    // clustering): the edge array holds a phase's usual output, and a phase
    // whose kept entries overflow it is discarded and redone as the pieces
    // split() cuts from the build's per-weight kept counts, in order.
    template <typename Build, typename Split>
    int run_phased_retry(Pack pk, std::vector<Phase> plan, Build build, Split split,
                         cudaStream_t st, int64_t *n_mst_out, int64_t *n_comp_out)
    {
        int32_t V = V0;
        mst_base = 0;
        size_t q = 0;
        while (q < plan.size()) {
            const Phase ph = plan[q];
            EACB_CUDA(cudaMemsetAsync(best, 0xff, sizeof(uint64_t) * V, st));
            EACB_CUDA(cudaMemsetAsync(&cnt[C_CURSOR], 0, sizeof(int64_t), st));
            EACB_CUDA(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned long long), st));
            int s = build(ph);
            if (s) return s;
            int64_t Ep = 0;
            int e = 0;
            EACB_CUDA(cudaMemcpyAsync(&Ep, &cnt[C_CURSOR], sizeof(int64_t), cudaMemcpyDeviceToHost,
                                      st));
            EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaStreamSynchronize(st));
            if (e == DEV_CAPACITY) {
                // the build still counted every kept entry, per weight, in
                // hist: the pieces are cut from those counts
                unsigned long long kh[256];
                EACB_CUDA(cudaMemcpyAsync(kh, hist, sizeof(kh), cudaMemcpyDeviceToHost, st));
                EACB_CUDA(cudaStreamSynchronize(st));
                std::vector<Phase> pieces;
                if ((s = split(ph, kh, pieces))) return s;
                EACB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
                plan.erase(plan.begin() + (ptrdiff_t)q);
                plan.insert(plan.begin() + (ptrdiff_t)q, pieces.begin(), pieces.end());
                continue;
            }
            if (e) return dev_err_to_status(e);
            if (Ep > Emax) return EACB_ERR_INTERNAL;
            if (prof().enabled) prof().bytes[PROF_PHASE] += 8.0 * (double)Ep;   // words written
            int64_t nm = 0, nc = 0;
            if ((s = run<SEL_MST>(pk, Ep, V, st, &nm, &nc))) return s;
            mst_base += nm;
            V = (int32_t)nc;
            ++q;
            if (V <= 1) break;
        }
        *n_mst_out = mst_base;
        *n_comp_out = V;
        return EACB_OK;
    }

    // All phases queued back to back with no host read in between: a phase's
    // edge count and supervertex count stay on the device (k_phase_begin),
    // an empty phase runs one no-op round, and one read at the end gives the
    // forest size, the component count and any error.
    template <typename Build>
    int run_phased_graph(const std::vector<Phase> &plan, Build build, cudaGraphExec_t exec,
                         int per_round, cudaStream_t st, int64_t *n_mst_out, int64_t *n_comp_out)
    {
        for (size_t q = 0; q < plan.size(); ++q) {
            EACB_CUDA(cudaMemsetAsync(best, 0xff, sizeof(uint64_t) * V0, st));
            EACB_CUDA(cudaMemsetAsync(&cnt[C_CURSOR], 0, sizeof(int64_t), st));
            int s = build(plan[q]);
            if (s) return s;
            k_phase_begin<<<1, 32, 0, st>>>(cnt, V0, q == 0 ? 1 : 0);
            EACB_CHECK_LAUNCH();
            EACB_CUDA(cudaGraphLaunch(exec, st));
        }
        int64_t after[C_COUNT];
        int e = 0;
        EACB_CUDA(cudaMemcpyAsync(after, cnt, sizeof(after), cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaStreamSynchronize(st));
        count_launch((int)(after[C_ROUNDS_ALL] * per_round));
        if (e) return dev_err_to_status(e);
        mst_base = after[C_NMST];
        *n_mst_out = after[C_NMST];
        *n_comp_out = plan.empty() ? V0 : after[C_V];
        return EACB_OK;
    }

    int reset(cudaStream_t st)
    {
        EACB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        EACB_CUDA(cudaMemsetAsync(cnt, 0, C_COUNT * sizeof(int64_t), st));
        EACB_CUDA(cudaMemsetAsync(best, 0xff, sizeof(uint64_t) * V0, st));
        k_iota<<<grid_for(V0, 256), 256, 0, st>>>(label, V0);
        EACB_CHECK_LAUNCH();
        return EACB_OK;
    }

    template <int MODE, typename Src>
    int filter(const Src &src, int64_t n_in, uint64_t *out, cudaStream_t st)
    {
        if (n_in == 0) {
            EACB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int64_t), st));
            return EACB_OK;
        }
        const int64_t ntiles = (n_in + kETile - 1) / kETile;
        EACB_CUDA(cudaMemsetAsync(scan.status, 0, sizeof(uint64_t) * ntiles, st));
        EACB_CUDA(cudaMemsetAsync(scan.counter, 0, sizeof(int), st));
        k_edge_tile<MODE, Src><<<(unsigned)ntiles, kET, 0, st>>>(
            src, n_in, out, best, scan.status, scan.counter, cnt, err);
        EACB_CHECK_LAUNCH();
        return EACB_OK;
    }

    int edge_grid() const
    {
        const int64_t t = (Emax + kETile - 1) / kETile;
        return (int)(t < 148 * 8 ? (t > 0 ? t : 1) : 148 * 8);
    }

    // One Boruvka round with every size read on the device (cnt[C_V],
    // cnt[C_E]); identical launch shapes every round, so the sequence can be
    // captured once into a CUDA graph.  With use_handle the last kernel sets
    // the graph's loop condition.  Returns the kernels it launches per round
    // in *per_round.
    template <int MODE>
    int enqueue_round(Pack pk, cudaStream_t st, int use_handle, cudaGraphConditionalHandle h,
                      bool timed_filter, int *per_round)
    {
        const unsigned gv = 296;
        int launches = 0;
        // look-back status words: scans over V0, the contraction over Emax
        const int64_t vtiles = (V0 + kScanTile - 1) / kScanTile;
        const int64_t etiles = (Emax + kETile - 1) / kETile;
        k_select<MODE><<<gv, 256, 0, st>>>(best, succ, &cnt[C_V], label, pk);
        EACB_CHECK_LAUNCH();
        k_mirror<<<gv, 256, 0, st>>>(succ, color, MODE == SEL_MST ? flag : nullptr, &cnt[C_V],
                                     scan.status, vtiles, scan.counter);
        EACB_CHECK_LAUNCH();
        launches += 2;
        if (MODE == SEL_MST) {
            int s = scan_launch_dev<int32_t, int32_t>(flag, pos, &cnt[C_V], V0, 0, &cnt[C_EMIT],
                                                      scan, st, false);
            if (s) return s;
            launches += 1;
        }
        k_jump<<<gv, 256, 0, st>>>(color, &cnt[C_V], err, best, flag, pos,
                                   MODE == SEL_MST ? mst : nullptr, &cnt[C_NMST], scan.status,
                                   vtiles, scan.counter);
        EACB_CHECK_LAUNCH();
        int s = scan_launch_dev<int32_t, int32_t>(flag, pos, &cnt[C_V], V0, 0, &cnt[C_V_NEXT],
                                                  scan, st, false);
        if (s) return s;
        k_relabel<<<grid_for(V0, 256), 256, 0, st>>>(label, color, pos, V0, best, &cnt[C_V_NEXT],
                                                       scan.status, etiles > 0 ? etiles : 1,
                                                       scan.counter, &cnt[C_E_NEXT]);
        EACB_CHECK_LAUNCH();
        launches += 3;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        if (timed_filter) {
            cudaEventCreate(&ev0);
            cudaEventCreate(&ev1);
            cudaEventRecord(ev0, st);
        }
        SrcEdges se{ea, label, pk, (uint32_t)V0};
        k_edge_tile<MODE, SrcEdges><<<edge_grid(), kET, 0, st>>>(
            se, 0, ea, best, scan.status, scan.counter, &cnt[C_E_NEXT], err, &cnt[C_E]);
        EACB_CHECK_LAUNCH();
        if (timed_filter) {
            cudaEventRecord(ev1, st);
            timed_ev0 = ev0;
            timed_ev1 = ev1;
        }
        k_round_end<<<1, 32, 0, st>>>(cnt, MODE == SEL_MST ? 1 : 0, max_rounds, err, h, use_handle);
        EACB_CHECK_LAUNCH();
        launches += 2;
        if (per_round) *per_round = launches;
        return EACB_OK;
    }

    cudaEvent_t timed_ev0 = nullptr, timed_ev1 = nullptr;

    template <int MODE>
    cudaGraphExec_t round_graph(Pack pk, int *per_round);

    // Rounds; edges of round 0 are in `ea` (E0 of them) and `best` holds
    // their selection; supervertex ids are [0, V_start) under `label`.  The
    // rounds run inside one CUDA graph that loops on the device (conditional
    // WHILE node) until the phase converges; with profiling on (per-launch
    // CUDA events) or a round limit they are driven from the host instead.
    // On return: label = component of every vertex, *n_comp = number of
    // components, *n_mst = forest edges emitted by these rounds.
    template <int MODE>
    int run(Pack pk, int64_t E0, int32_t V_start, cudaStream_t st, int64_t *n_mst_out,
            int64_t *n_comp_out)
    {
        if (E0 == 0) {                 // nothing to contract: components stay as they are
            *n_mst_out = 0;
            *n_comp_out = V_start;
            return EACB_OK;
        }
        int64_t before[C_COUNT];
        EACB_CUDA(cudaMemcpyAsync(before, cnt, sizeof(before), cudaMemcpyDeviceToHost, st));
        k_round_begin<<<1, 32, 0, st>>>(cnt, V_start, E0);
        EACB_CHECK_LAUNCH();
        int per_round = 0;
        const bool host_driven = prof().enabled != 0 || max_rounds < kMaxRounds;
        cudaGraphExec_t exec = host_driven ? nullptr : round_graph<MODE>(pk, &per_round);
        int64_t after[C_COUNT];
        int e = 0;
        if (exec) {
            EACB_CUDA(cudaGraphLaunch(exec, st));
            EACB_CUDA(cudaMemcpyAsync(after, cnt, sizeof(after), cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaStreamSynchronize(st));
            count_launch((int)(after[C_ROUNDS] * per_round));
        } else {
            for (int round = 0; round < max_rounds; ++round) {
                const bool timed = prof().enabled != 0;
                int64_t E_in = 0;
                if (timed)
                    EACB_CUDA(cudaMemcpyAsync(&E_in, &cnt[C_E], sizeof(int64_t),
                                              cudaMemcpyDeviceToHost, st));
                int s = enqueue_round<MODE>(pk, st, 0, 0, timed, &per_round);
                if (s) return s;
                EACB_CUDA(cudaMemcpyAsync(after, cnt, sizeof(after), cudaMemcpyDeviceToHost, st));
                EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
                EACB_CUDA(cudaStreamSynchronize(st));
                if (timed) {
                    // algorithmic HBM bytes of one contraction: every edge word
                    // read once, every surviving edge word written once
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, timed_ev0, timed_ev1);
                    prof().ms[PROF_EDGE_TILE] += ms;
                    prof().bytes[PROF_EDGE_TILE] +=
                        8.0 * (double)E_in + 8.0 * (double)after[C_E_NEXT];
                    prof().count[PROF_EDGE_TILE] += 1;
                    cudaEventDestroy(timed_ev0);
                    cudaEventDestroy(timed_ev1);
                }
                if (e || after[C_DONE]) break;
            }
        }
        if (e) return dev_err_to_status(e);
        const int64_t done = after[C_DONE];
        if (done == 2) return EACB_ERR_NOT_CONVERGED;                 // no progress
        if (done == 0 || done == 3) {                                  // round cap
            if (max_rounds >= kMaxRounds) return EACB_ERR_NOT_CONVERGED;
        }
        *n_mst_out = after[C_NMST] - before[C_NMST];
        *n_comp_out = after[C_V];
        return EACB_OK;
    }
};

// Cache of instantiated round graphs, keyed by everything the captured
// kernels see (workspace layout, sizes, mode, key packing, device).
struct GraphKey {
    const void *base;
    int64_t V0, Emax;
    int mode, vbits, dev, max_rounds;
    bool operator==(const GraphKey &o) const
    {
        return base == o.base && V0 == o.V0 && Emax == o.Emax && mode == o.mode &&
               vbits == o.vbits && dev == o.dev && max_rounds == o.max_rounds;
    }
};
struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    int per_round;
};
// One cache per host thread: an entry is only ever launched by the thread
// that built it, so no other thread can destroy a graph in use.
struct GraphCache {
    std::vector<GraphEntry> v;
    ~GraphCache()
    {
        for (auto &g : v) cudaGraphExecDestroy(g.exec);
    }
};
static thread_local GraphCache t_graphs;

// Builds (once per key) the graph: a conditional WHILE node whose body is
// one round; the body's last kernel clears the condition when the phase has
// converged.  Returns nullptr if this driver cannot build it (the host then
// drives the rounds).
template <int MODE>
cudaGraphExec_t Engine::round_graph(Pack pk, int *per_round)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    GraphKey key{(const void *)err, V0, Emax, MODE, pk.vbits, dev, max_rounds};
    for (auto &g : t_graphs.v)
        if (g.key == key) {
            *per_round = g.per_round;
            return g.exec;
        }
    cudaStream_t cs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int pr = 0;
    bool ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess &&
              cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle h = 0;
    if (ok) ok = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) ==
                 cudaSuccess;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node = nullptr;
    if (ok) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
    }
    if (ok) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            const int s = enqueue_round<MODE>(pk, cs, 1, h, false, &pr);
            count_launch(-pr);                // capturing launches nothing
            cudaGraph_t out = nullptr;
            ok = cudaStreamEndCapture(cs, &out) == cudaSuccess && s == EACB_OK;
        }
    }
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (cs) cudaStreamDestroy(cs);
    cudaGetLastError();                       // a failed build leaves no sticky error
    if (!ok) {
        if (exec) cudaGraphExecDestroy(exec);
        return nullptr;
    }
    if (t_graphs.v.size() >= 16) {
        cudaGraphExecDestroy(t_graphs.v.front().exec);
        t_graphs.v.erase(t_graphs.v.begin());
    }
    t_graphs.v.push_back(GraphEntry{key, exec, pr});
    *per_round = pr;
    return exec;
}

static int g_debug_rounds = 0;   // 0 = off; else rounds to run (round-trace test entry)

template <typename WT>
static int csr_graph_run(int mode, const int32_t *dest, const WT *weight, int wbits,
                         const int32_t *first, const int32_t *deg, int32_t V, int64_t E,
                         int32_t *mst_out, int64_t *host_n_mst, int32_t *labels_out,
                         int64_t *host_n_comp, void *ws, size_t ws_bytes, cudaStream_t st)
{
    Pack pk;
    int s = make_pack(V, wbits, pk);
    if (s) return s;
    Carver c(ws, ws_bytes);
    Engine g = Engine::carve(c, V, E);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    if ((s = g.reset(st))) return s;
    int64_t h[3];
    int64_t n_mst = 0, n_comp = 0;
    if (g_debug_rounds > 0) g.max_rounds = g_debug_rounds;
    const unsigned gr = grid_for((int64_t)V * 32, 256);
    if (mode == SEL_MST && g_debug_rounds == 0) {
        // weight phases over the bucket histogram of the entries
        EACB_CUDA(cudaMemsetAsync(g.hist, 0, 256 * sizeof(unsigned long long), st));
        if (E > 0) {
            if (sizeof(WT) == 1) {
                if ((s = launch_whist_u8((const uint8_t *)weight, E, g.hist, st))) return s;
            } else {
                k_whist_csr<WT><<<grid_for(E, kHistThreads, 148 * 8), kHistThreads, 0, st>>>(
                    weight, E, wbits, g.hist);
            }
            EACB_CHECK_LAUNCH();
        }
        // the phase plan stays on the device: the whole MST is queued without
        // a host read until its end
        k_phase_plan<<<1, 32, 0, st>>>(g.hist, g.lohi);
        EACB_CHECK_LAUNCH();
        std::vector<Phase> plan;
        for (int q = 0; q < kPhaseSlots; ++q) plan.push_back(Phase{0, 0, 0, V, q});
        // a phase holds a subset of the E entries: the edge array always fits
        auto build = [&](const Phase &ph) -> int {
            if (E == 0) return EACB_OK;
            ProfScope ps(PROF_PHASE, st);
            k_phase_csr<WT><<<gr, kPhThreads, 0, st>>>(
                first, deg, dest, weight, V, E, wbits, 0, 0, g.lohi, ph.slot, g.label, pk, g.ea,
                (unsigned long long *)&g.cnt[C_CURSOR], (unsigned long long)g.Emax, g.best,
                g.err);
            EACB_CHECK_LAUNCH();
            // compulsory reads: row extents and labels (12 B per row), dest and
            // weight (4 + sizeof(WT) B per entry); the written words follow
            ps.done(12.0 * V + (4.0 + sizeof(WT)) * (double)E);
            return EACB_OK;
        };
        if ((s = g.run_phased(pk, plan, build, st, &n_mst, &n_comp))) return s;
    } else {
        if (E > 0) {
            // dead words everywhere first: entries outside every row, self loops
            EACB_CUDA(cudaMemsetAsync(g.ea, 0xff, sizeof(uint64_t) * E, st));
            if (mode == SEL_MST)
                k_edges_csr<SEL_MST, WT><<<gr, 256, 0, st>>>(first, deg, dest, weight, V, E, pk,
                                                             g.ea, g.best, g.err);
            else
                k_edges_csr<SEL_CC, WT><<<gr, 256, 0, st>>>(first, deg, dest, weight, V, E, pk,
                                                            g.ea, g.best, g.err);
            EACB_CHECK_LAUNCH();
        }
        if ((s = g.read_counts(st, h))) return s;      // input validity before the rounds
        if (mode == SEL_MST) s = g.run<SEL_MST>(pk, E, V, st, &n_mst, &n_comp);
        else s = g.run<SEL_CC>(pk, E, V, st, &n_mst, &n_comp);
        if (s) return s;
    }
    if (mode == SEL_MST) {
        if (n_mst > 0) {
            k_key2eid<WT><<<grid_for(n_mst, 256), 256, 0, st>>>(g.mst, n_mst, first, deg, dest,
                                                                      weight, pk, mst_out, g.err);
            EACB_CHECK_LAUNCH();
        }
        if ((s = g.read_counts(st, h))) return s;
        *host_n_mst = n_mst;
    } else {
        EACB_CUDA(cudaMemcpyAsync(labels_out, g.label, sizeof(int32_t) * V,
                                  cudaMemcpyDeviceToDevice, st));
        *host_n_comp = n_comp;
    }
    if (g_debug_rounds > 0 && labels_out && mode == SEL_MST)
        EACB_CUDA(cudaMemcpyAsync(labels_out, g.label, sizeof(int32_t) * V,
                                  cudaMemcpyDeviceToDevice, st));
    return EACB_OK;
}

static int csr_dispatch(int mode, const int32_t *dest, const void *weight, int dt,
                        const int32_t *first, const int32_t *deg, int32_t V, int64_t E,
                        int32_t *mst_out, int64_t *host_n_mst, int32_t *labels,
                        int64_t *host_n_comp, void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (V <= 0 || E < 0 || !first || !deg || (E > 0 && (!dest || !weight)) || !ws)
        return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    const int wb = dtype_bits(dt);
    switch (dt) {
    case EACB_U8:
        return csr_graph_run<uint8_t>(mode, dest, (const uint8_t *)weight, wb, first, deg, V, E,
                                      mst_out, host_n_mst, labels, host_n_comp, ws, ws_bytes, st);
    case EACB_U16:
        return csr_graph_run<uint16_t>(mode, dest, (const uint16_t *)weight, wb, first, deg, V, E,
                                       mst_out, host_n_mst, labels, host_n_comp, ws, ws_bytes, st);
    case EACB_I32:
        return csr_graph_run<int32_t>(mode, dest, (const int32_t *)weight, wb, first, deg, V, E,
                                      mst_out, host_n_mst, labels, host_n_comp, ws, ws_bytes, st);
    case EACB_U32:
        return csr_graph_run<uint32_t>(mode, dest, (const uint32_t *)weight, wb, first, deg, V, E,
                                       mst_out, host_n_mst, labels, host_n_comp, ws, ws_bytes, st);
    case EACB_F32:
        return csr_graph_run<float>(mode, dest, (const float *)weight, wb, first, deg, V, E,
                                    mst_out, host_n_mst, labels, host_n_comp, ws, ws_bytes, st);
    default:
        return EACB_ERR_BAD_ARGUMENT;
    }
}

// ---------------------------------------------------------------------------
// Final clustering helpers
// ---------------------------------------------------------------------------
__global__ void k_weight_hist(const uint64_t *keys, int64_t n, Pack pk, int64_t *hist)
{
    __shared__ int64_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd((unsigned long long *)&h[pk.sel_w(keys[i]) & 255], 1ull);
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd((unsigned long long *)&hist[i], (unsigned long long)h[i]);
}

struct CutPlan {
    int64_t status;      // 0 ok, else an eacb status
    int64_t n_clusters;  // nc_stable
    int64_t wmax;        // keep forest edges with weight <= wmax (-1: none)
    int64_t need_labels;
};

// The lifetime rule of MyML/MyML/EAC/eac.py:366-391 and the cut decision of
// :220-265, evaluated on the 256-bin histogram of the uint8 MST weights
// (sorted weights are the bins expanded in order).
__global__ void k_cut_plan(const int64_t *hist, int64_t n_mst, int32_t n, int32_t max_dist,
                           int32_t n_clusters, CutPlan *plan)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CutPlan p{0, 0, 255, 0};
    const int64_t n_disc = (int64_t)n - n_mst;
    int64_t nc;
    int64_t thr = 255;
    if (n_clusters == 0) {
        if (n_mst < 2) { p.status = EACB_ERR_VALUE; *plan = p; return; }
        // lifetimes = differences of consecutive sorted weights; zero ones
        // exist iff some bin holds two or more edges
        bool has_zero = false;
        int prev = -1, wlast = 0;
        int best_gap = 0, m_w = -1;
        for (int b = 0; b < 256; ++b) {
            int64_t c = hist[b];
            if (!c) continue;
            if (c >= 2) has_zero = true;
            if (prev >= 0 && b - prev > best_gap) { best_gap = b - prev; m_w = prev; }
            prev = b;
            wlast = b;
        }
        if (!has_zero) { p.status = EACB_ERR_VALUE; *plan = p; return; }
        int first_w = -1;
        for (int b = 0; b < 256; ++b) if (hist[b]) { first_w = b; break; }
        if (m_w < 0) m_w = first_w;          // all lifetimes zero: argmax = 0
        int64_t above = 0;
        for (int b = m_w + 1; b < 256; ++b) above += hist[b];
        int64_t cont = above == 0 ? 1 : above + 1;
        // th < 2 * min(zero lifetimes) never holds once a zero lifetime exists
        if (n_disc > 1) {
            int64_t disc_life = (int64_t)max_dist + 1 + 1 - wlast;
            if ((int64_t)best_gap > disc_life) cont += n_disc - 1;
            else cont = n_disc;
        }
        nc = cont;
        thr = m_w;    // the cut removes exactly the edges heavier than w[m]
    } else {
        nc = n_clusters;
        if (nc > n_disc) {
            // cut the (nc - n_disc) heaviest forest edges; supported when that
            // boundary falls between two weight bins (no tie to split)
            const int64_t n_cuts = nc - n_disc;
            int64_t acc = 0;
            thr = 255;
            for (int b = 255; b >= 0 && acc < n_cuts; --b) {
                if (acc + hist[b] > n_cuts) { p.status = EACB_ERR_UNSUPPORTED; *plan = p; return; }
                acc += hist[b];
                thr = b - 1;
            }
        }
    }
    p.n_clusters = nc;
    p.wmax = (nc > n_disc) ? thr : 255;
    p.need_labels = nc > 1;
    *plan = p;
}

__global__ void k_comp_min(const int32_t *label, int32_t n, int32_t *cmin)
{
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * blockDim.x)
        atomicMin(&cmin[label[x]], (int32_t)x);
}

__global__ void k_first_flag(const int32_t *label, const int32_t *cmin, int32_t n, int32_t *flag)
{
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * blockDim.x)
        flag[x] = cmin[label[x]] == (int32_t)x;
}

__global__ void k_canon(const int32_t *label, const int32_t *cmin, const int32_t *pos, int32_t n,
                        int32_t *out)
{
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * blockDim.x)
        out[x] = pos[cmin[label[x]]];
}

}  // namespace eacb

using namespace eacb;

// Test hook: the next graph calls stop after `rounds` Boruvka rounds (0 =
// run to completion) so tests can compare per-round state.
extern "C" void eacb_debug_set_rounds(int rounds) { g_debug_rounds = rounds; }

extern "C" size_t eacb_boruvka_workspace_size(int32_t n_vertices, int64_t n_edges)
{
    Carver c(nullptr, 0);
    Engine::carve(c, n_vertices, n_edges);
    return c.off;
}

extern "C" int eacb_boruvka_mst(const int32_t *dest, const void *weight, int weight_dtype,
                                const int32_t *first_edge, const int32_t *out_degree,
                                int32_t n_vertices, int64_t n_edges, int32_t *mst_out,
                                int64_t *host_n_mst, void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (!host_n_mst || (!mst_out && n_vertices > 1)) return EACB_ERR_BAD_ARGUMENT;
    int64_t dummy = 0;
    return csr_dispatch(SEL_MST, dest, weight, weight_dtype, first_edge, out_degree, n_vertices,
                        n_edges, mst_out, host_n_mst, nullptr, &dummy, ws, ws_bytes, stream);
}

extern "C" int eacb_connected_components(const int32_t *dest, const void *weight,
                                         int weight_dtype, const int32_t *first_edge,
                                         const int32_t *out_degree, int32_t n_vertices,
                                         int64_t n_edges, int32_t *labels, int64_t *host_n_comps,
                                         void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (!labels || !host_n_comps) return EACB_ERR_BAD_ARGUMENT;
    int64_t dummy = 0;
    return csr_dispatch(SEL_CC, dest, weight, weight_dtype, first_edge, out_degree, n_vertices,
                        n_edges, nullptr, &dummy, labels, host_n_comps, ws, ws_bytes, stream);
}

// Edge words of the final clustering: every entry's two directions when the
// matrix is small, else 256 words per point (at least 2^20): room for the
// usual output of a phase, not its worst case (a phase that overflows is
// redone in pieces), so a matrix of thousands of entries per row does not
// need an edge array of its own size.
static int64_t final_edge_cap(int32_t n, int64_t nnz)
{
    const int64_t all = 2 * (nnz > (int64_t)n ? nnz : (int64_t)n);
    const int64_t usual = 256 * (int64_t)n > ((int64_t)1 << 20) ? 256 * (int64_t)n : ((int64_t)1 << 20);
    return all < usual ? all : usual;
}

// Phases of the final clustering, lightest weights first: the weight ranges
// whose cumulative entry counts reach 8n, 32n, 128n, 512n, 2048n and all
// entries.  A co-association matrix holds thousands of entries per row, and
// the lightest few per point already join most points: later phases keep
// only entries between different components, so they write few edges, and a
// phase over a narrow range reads little more than the weights.
static void plan_final_phases(const unsigned long long h[256], int32_t n, std::vector<Phase> &plan)
{
    unsigned long long tot = 0;
    for (int b = 0; b < 256; ++b) tot += h[b];
    const double t = tot ? (double)tot : 1.0;
    double fracs[6];
    for (int f = 0; f < 5; ++f) fracs[f] = std::min(1.0, (double)(8 << (2 * f)) * n / t);
    fracs[5] = 1.0;
    int lo[8], hi[8];
    const int np = phase_ranges(h, fracs, 6, lo, hi);
    for (int q = 0; q < np; ++q) plan.push_back(Phase{lo[q], hi[q], 0, n, -1});
}

// Pieces of a phase whose kept entries did not fit the edge array, from the
// kept entries per weight that its build counted (kh; upper bounds for the
// pieces, whose components only merge): consecutive weights while their
// kept entries fit, and a weight that alone does not fit split into row
// ranges of equal entry counts (the order (w, a, b) keeps a row range of one
// weight contiguous).  Host row pointers are fetched on the first row split.
static int split_final_phase(const Phase &ph, const unsigned long long kh[256], int64_t cap_entries,
                             const int64_t *d_indptr, int32_t n, std::vector<int64_t> &ip,
                             cudaStream_t st, std::vector<Phase> &out)
{
    const unsigned long long cap = (unsigned long long)(cap_entries / 8 * 7);
    if (ph.r0 != 0 || ph.r1 != n) {
        // a row range of one weight: halve the rows
        if (ph.r1 - ph.r0 < 2) return EACB_ERR_INTERNAL;
        const int64_t m = ph.r0 + (ph.r1 - ph.r0) / 2;
        out.push_back(Phase{ph.lo, ph.hi, ph.r0, m, -1});
        out.push_back(Phase{ph.lo, ph.hi, m, ph.r1, -1});
        return EACB_OK;
    }
    int start = ph.lo;
    unsigned long long acc = 0;
    for (int w = ph.lo + 1; w <= ph.hi; ++w) {
        if (kh[w] <= cap && acc + kh[w] <= cap) {
            acc += kh[w];
            continue;
        }
        if (w - 1 > start) out.push_back(Phase{start, w - 1, 0, n, -1});
        if (kh[w] <= cap) {                    // w opens the next piece
            start = w - 1;
            acc = kh[w];
            continue;
        }
        // weight w alone: rows in pieces of about equal entry counts
        if (ip.empty()) {
            ip.resize((size_t)n + 1);
            EACB_CUDA(cudaMemcpyAsync(ip.data(), d_indptr, sizeof(int64_t) * ((size_t)n + 1),
                                      cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaStreamSynchronize(st));
        }
        const int64_t parts = (int64_t)((kh[w] + cap - 1) / cap);
        const double piece = (double)ip[n] / (double)parts;
        int64_t r = 0;
        while (r < n) {
            int64_t e = r + 1;
            while (e < n && (double)(ip[e + 1] - ip[r]) <= piece) ++e;
            out.push_back(Phase{w - 1, w, r, e, -1});
            r = e;
        }
        start = w;
        acc = 0;
    }
    if (ph.hi > start) out.push_back(Phase{start, ph.hi, 0, n, -1});
    if (out.size() == 1 && out[0].lo == ph.lo && out[0].hi == ph.hi) {
        // the counts say it fits (it cannot have overflowed): split anyway
        out.clear();
        if (ph.hi - ph.lo < 2) return EACB_ERR_INTERNAL;
        const int m = ph.lo + (ph.hi - ph.lo) / 2;
        out.push_back(Phase{ph.lo, m, 0, n, -1});
        out.push_back(Phase{m, ph.hi, 0, n, -1});
    }
    return EACB_OK;
}

static void carve_final(Carver &c, int32_t n, int64_t nnz, Engine *g, int64_t **hist,
                        CutPlan **plan, int32_t **cmin)
{
    *g = Engine::carve(c, n, final_edge_cap(n, nnz));
    *hist = c.take<int64_t>(256);
    *plan = c.take<CutPlan>(1);
    *cmin = c.take<int32_t>(n);
}

extern "C" size_t eacb_final_clustering_workspace_size(int32_t n, int64_t nnz)
{
    Carver c(nullptr, 0);
    Engine g;
    int64_t *h;
    CutPlan *p;
    int32_t *m;
    carve_final(c, n, nnz, &g, &h, &p, &m);
    return c.off;
}

extern "C" int eacb_final_clustering(const int64_t *indptr, const int32_t *indices,
                                     const uint8_t *diassoc, int32_t n, int64_t nnz,
                                     int32_t max_dist, int32_t n_clusters, int32_t *labels,
                                     int64_t *host_n_fclusts, int32_t *host_labels_valid,
                                     void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (n <= 0 || nnz < 0 || !indptr || (nnz > 0 && (!indices || !diassoc)) || !labels ||
        !host_n_fclusts || !host_labels_valid || !ws || n_clusters < 0)
        return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Pack pk;
    int s = make_pack(n, 8, pk);
    if (s) return s;
    Carver c(ws, ws_bytes);
    Engine g;
    int64_t *hist;
    CutPlan *plan;
    int32_t *cmin;
    carve_final(c, n, nnz, &g, &hist, &plan, &cmin);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    if ((s = g.reset(st))) return s;
    // 1. minimum spanning forest of the dissimilarity graph, by weight phases
    EACB_CUDA(cudaMemsetAsync(g.hist, 0, 256 * sizeof(unsigned long long), st));
    if (nnz > 0) {
        if ((s = launch_whist_u8(diassoc, nnz, g.hist, st))) return s;
    }
    int64_t n_mst = 0, n_comp = 0;
    unsigned long long wh[256];
    if ((s = g.read_hist(st, wh))) return s;
    std::vector<Phase> phases;
    plan_final_phases(wh, n, phases);
    unsigned long long wtot = 0;
    for (int b = 0; b < 256; ++b) wtot += wh[b];
    // a phase whose range holds over a quarter of the entries reads every
    // 16-byte run of indices anyway
    auto dense = [&](const Phase &ph) -> int {
        unsigned long long in = 0;
        for (int b = ph.lo + 1; b <= ph.hi; ++b) in += wh[b];
        return 4 * in > wtot ? 1 : 0;
    };
    auto build = [&](const Phase &ph) -> int {
        if (nnz == 0) return EACB_OK;
        ProfScope ps(PROF_PHASE, st);
        k_phase_upper<<<grid_for((ph.r1 - ph.r0) * 32, kPhThreads), kPhThreads, 0, st>>>(
            indptr, indices, diassoc, n, nnz, ph.lo, ph.hi, dense(ph), ph.r0, ph.r1, g.label, pk, g.ea,
            (unsigned long long *)&g.cnt[C_CURSOR], (unsigned long long)g.Emax, g.best, g.hist,
            g.err);
        EACB_CHECK_LAUNCH();
        // compulsory reads: row pointers and labels (12 B per row), column and
        // weight (5 B per entry; a row-range phase is counted in proportion to
        // its rows); the written words follow
        const double rows = (double)(ph.r1 - ph.r0);
        ps.done(12.0 * rows + 5.0 * (double)nnz * (rows / (double)n));
        return EACB_OK;
    };
    std::vector<int64_t> hip;
    auto split = [&](const Phase &ph, const unsigned long long kh[256], std::vector<Phase> &out) {
        return split_final_phase(ph, kh, g.Emax / 2, indptr, n, hip, st, out);
    };
    if ((s = g.run_phased_retry(pk, phases, build, split, st, &n_mst, &n_comp))) return s;
    // 2. lifetime rule on the weight histogram
    EACB_CUDA(cudaMemsetAsync(hist, 0, 256 * sizeof(int64_t), st));
    if (n_mst > 0) {
        k_weight_hist<<<grid_for(n_mst, 256, 148 * 4), 256, 0, st>>>(g.mst, n_mst, pk, hist);
        EACB_CHECK_LAUNCH();
    }
    k_cut_plan<<<1, 32, 0, st>>>(hist, n_mst, n, max_dist, n_clusters, plan);
    EACB_CHECK_LAUNCH();
    CutPlan hp;
    EACB_CUDA(cudaMemcpyAsync(&hp, plan, sizeof(CutPlan), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    if (hp.status) return (int)hp.status;
    *host_n_fclusts = hp.n_clusters;
    if (!hp.need_labels) {
        *host_labels_valid = 0;
        *host_n_fclusts = 1;
        return EACB_OK;
    }
    // 3. components of the forest without the cut edges (the forest keys
    //    move to ea: the second run reuses the engine's buffers)
    EACB_CUDA(cudaMemcpyAsync(g.ea, g.mst, sizeof(uint64_t) * n_mst, cudaMemcpyDeviceToDevice, st));
    if ((s = g.reset(st))) return s;
    // the forest edges (both directions) go from ea[0, n_mst) into eb
    SrcForest sf{g.ea, n_mst, hp.wmax, pk};
    if ((s = g.filter<SEL_CC>(sf, 2 * n_mst, g.eb, st))) return s;
    int64_t h[3];
    if ((s = g.read_counts(st, h))) return s;
    // run() starts from ea: swap roles by copying (forest is small)
    EACB_CUDA(cudaMemcpyAsync(g.ea, g.eb, sizeof(uint64_t) * h[0], cudaMemcpyDeviceToDevice, st));
    int64_t nm2 = 0, nc2 = 0;
    if ((s = g.run<SEL_CC>(pk, h[0], n, st, &nm2, &nc2))) return s;
    // 4. number components by their smallest member
    EACB_CUDA(cudaMemsetAsync(cmin, 0x7f, sizeof(int32_t) * n, st));
    const unsigned gn = grid_for(n, 256);
    k_comp_min<<<gn, 256, 0, st>>>(g.label, n, cmin);
    EACB_CHECK_LAUNCH();
    k_first_flag<<<gn, 256, 0, st>>>(g.label, cmin, n, g.flag);
    EACB_CHECK_LAUNCH();
    if ((s = scan_launch<int32_t, int32_t>(g.flag, g.pos, n, 0, &g.cnt[1], g.scan, st))) return s;
    k_canon<<<gn, 256, 0, st>>>(g.label, cmin, g.pos, n, labels);
    EACB_CHECK_LAUNCH();
    if ((s = g.read_counts(st, h))) return s;
    *host_n_fclusts = h[1];
    *host_labels_valid = 1;
    return EACB_OK;
}

// ---------------------------------------------------------------------------
// The final clustering's two steps as separate calls.
// ---------------------------------------------------------------------------
__global__ void k_check_labels(const int32_t *labels, int32_t n, int *err)
{
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * blockDim.x)
        if (labels[x] < 0 || labels[x] >= n) set_err(err, DEV_BAD_INPUT);
}

extern "C" size_t eacb_lifetime_cut_workspace_size(void)
{
    Carver c(nullptr, 0);
    c.take<unsigned long long>(256);
    c.take<CutPlan>(1);
    return c.off;
}

// lifetime_n_clusters (MyML/MyML/EAC/eac.py:366-391) and the cut decision of
// sp_sl_lifetime (:220-265) on the uint8 weights of a minimum spanning forest
// of n points (any order).  *host_n_clusters receives the number of clusters;
// *host_threshold the largest forest weight kept (-1: none, 255: all).
extern "C" int eacb_lifetime_cut(const uint8_t *mst_weights, int64_t n_mst, int32_t n,
                                 int32_t max_dist, int32_t n_clusters, int64_t *host_n_clusters,
                                 int32_t *host_threshold, void *ws, size_t ws_bytes,
                                 uintptr_t stream)
{
    if (n <= 0 || n_mst < 0 || n_mst >= n || (n_mst > 0 && !mst_weights) || n_clusters < 0 ||
        !host_n_clusters || !host_threshold || !ws)
        return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    unsigned long long *hist = c.take<unsigned long long>(256);
    CutPlan *plan = c.take<CutPlan>(1);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned long long), st));
    if (n_mst > 0) {
        const int s = launch_whist_u8(mst_weights, n_mst, hist, st);
        if (s) return s;
    }
    k_cut_plan<<<1, 32, 0, st>>>((const int64_t *)hist, n_mst, n, max_dist, n_clusters, plan);
    EACB_CHECK_LAUNCH();
    CutPlan hp;
    EACB_CUDA(cudaMemcpyAsync(&hp, plan, sizeof(CutPlan), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    if (hp.status) return (int)hp.status;
    *host_n_clusters = hp.n_clusters;
    *host_threshold = (int32_t)hp.wmax;
    return EACB_OK;
}

extern "C" size_t eacb_relabel_canonical_workspace_size(int32_t n)
{
    Carver c(nullptr, 0);
    c.take<int>(1);
    c.take<int64_t>(1);
    c.take<int32_t>(n);
    c.take<int32_t>(n);
    c.take<int32_t>(n);
    ScanScratch::carve(c, n);
    return c.off;
}

// Numbers the groups of a labelling by their smallest member (the group of
// point 0 is 0, the next group to appear is 1, ...): the numbering scipy's
// connected_components gives, which the final labels use.  labels_in holds
// n group ids in [0, n); labels_out may equal labels_in.
extern "C" int eacb_relabel_canonical(const int32_t *labels_in, int32_t n, int32_t *labels_out,
                                      int64_t *host_n_groups, void *ws, size_t ws_bytes,
                                      uintptr_t stream)
{
    if (!labels_in || n <= 0 || !labels_out || !host_n_groups || !ws) return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    int *err = c.take<int>(1);
    int64_t *total = c.take<int64_t>(1);
    int32_t *cmin = c.take<int32_t>(n);
    int32_t *flag = c.take<int32_t>(n);
    int32_t *pos = c.take<int32_t>(n);
    ScanScratch scan = ScanScratch::carve(c, n, err);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    EACB_CUDA(cudaMemsetAsync(cmin, 0x7f, sizeof(int32_t) * n, st));
    const unsigned gn = grid_for(n, 256);
    k_check_labels<<<gn, 256, 0, st>>>(labels_in, n, err);
    EACB_CHECK_LAUNCH();
    int e = 0;
    EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    if (e) return dev_err_to_status(e);
    k_comp_min<<<gn, 256, 0, st>>>(labels_in, n, cmin);
    EACB_CHECK_LAUNCH();
    k_first_flag<<<gn, 256, 0, st>>>(labels_in, cmin, n, flag);
    EACB_CHECK_LAUNCH();
    int s = scan_launch<int32_t, int32_t>(flag, pos, n, 0, total, scan, st);
    if (s) return s;
    k_canon<<<gn, 256, 0, st>>>(labels_in, cmin, pos, n, labels_out);
    EACB_CHECK_LAUNCH();
    int64_t ng = 0;
    EACB_CUDA(cudaMemcpyAsync(&ng, total, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    if (e) return dev_err_to_status(e);
    *host_n_groups = ng;
    return EACB_OK;
}
