// Boruvka minimum spanning forest, connected components and the EAC final
// clustering (lifetime cut) on B200.
//
// Reference: MyML/MyML/graph/mst.py:417-809 (boruvka_minho_gpu and kernels),
// MyML/MyML/graph/connected_components.py:176-345, MyML/MyML/EAC/eac.py:199-391.
//
// Design (not the reference's):
//  * Every undirected edge is ONE 64-bit word: weight-order bits | min(u,v) |
//    max(u,v) | the entry's offset in the row of min(u,v) (graph MST; the
//    spare bits) | direction, with u, v the ORIGINAL endpoints, offered to the selection
//    slots of both its ends.  A round never rewrites edges; it only drops the
//    ones that became internal.  The current endpoints are the roots of u
//    and v in a union-find forest over the original vertices.
//  * Min-edge selection is an atomicMin of a 64-bit selection key per
//    supervertex: (weight, min, max) for the MST -- a strict total order, so
//    the forest is unique -- or (weight, other end's supervertex) for the
//    reference's connected-components numbering.  Lanes of a warp holding
//    edges of the same supervertex are pre-reduced with a segmented shuffle
//    scan, so one atomic is issued per run, not per edge.
//  * All Boruvka rounds of a phase run in ONE persistent kernel (k_rounds):
//    a cooperative grid whose blocks meet at bounded grid barriers, or a
//    single block for small graphs.  Contraction is fused with the NEXT
//    round's min-edge selection: each edge is read once and written at most
//    once per round.
//  * Mutual picks are broken towards the larger id like the reference; roots
//    are found by a bounded pointer chase with path halving; supervertices are
//    renumbered in root order, which is the reference's numbering.
//  * The MST grows by weight phases (Kruskal's prefix property), so heavy
//    edges that lighter ones made internal are dropped by one filtering read.
#include "eacb_common.cuh"
#include "scan_impl.cuh"

#include <algorithm>
#include <vector>

namespace eacb {

enum { SEL_MST = 0, SEL_CC = 1 };

struct Pack {
    int vbits;
    int obits;       // row-offset bits (0: none)
    int wshift;      // 2*vbits + obits + 1
    uint64_t vmask;
    uint64_t omask;  // (1 << obits) - 1: also the "offset not recorded" value
    __host__ __device__ uint32_t a(uint64_t k) const { return (uint32_t)((k >> (vbits + obits + 1)) & vmask); }
    __host__ __device__ uint32_t b(uint64_t k) const { return (uint32_t)((k >> (obits + 1)) & vmask); }
    __host__ __device__ uint32_t w(uint64_t k) const { return (uint32_t)(k >> wshift); }
    __host__ __device__ uint32_t src(uint64_t k) const { return (k & 1) ? b(k) : a(k); }
    __host__ __device__ uint32_t dst(uint64_t k) const { return (k & 1) ? a(k) : b(k); }
    // off: where the entry min -> max sits in the row of min (omask: not
    // recorded); it is the lowest field of the selection key, so among
    // parallel entries of one row the first one wins
    __host__ __device__ uint64_t make(uint32_t w, uint32_t u, uint32_t v, uint64_t off) const
    {
        uint32_t lo = u < v ? u : v, hi = u < v ? v : u;
        return ((uint64_t)w << wshift) | ((uint64_t)lo << (vbits + obits + 1)) |
               ((uint64_t)hi << (obits + 1)) | ((off & omask) << 1) | (uint64_t)(u > v);
    }
    __host__ __device__ uint64_t make(uint32_t w, uint32_t u, uint32_t v) const
    {
        return make(w, u, v, omask);
    }
    // MST selection key (weight, min, max, offset) and its decoding
    __host__ __device__ uint64_t mst_sel(uint64_t k) const { return k >> 1; }
    __host__ __device__ uint32_t sel_a(uint64_t s) const { return (uint32_t)((s >> (vbits + obits)) & vmask); }
    __host__ __device__ uint32_t sel_b(uint64_t s) const { return (uint32_t)((s >> obits) & vmask); }
    __host__ __device__ uint32_t sel_w(uint64_t s) const { return (uint32_t)(s >> (2 * vbits + obits)); }
    __host__ __device__ uint64_t sel_off(uint64_t s) const { return s & omask; }
};

// with_offsets: the bits left over in the word hold the entry's row offset
// (a graph MST returns entry ids: k_key2eid reads them instead of searching
// the row).
static int make_pack(int32_t n_vertices, int wbits, Pack &pk, bool with_offsets = false)
{
    int vbits = 1;
    while (vbits < 31 && ((int64_t)1 << vbits) < (int64_t)n_vertices) vbits++;
    if (wbits + 2 * vbits + 1 > 64) return EACB_ERR_UNSUPPORTED;
    const int spare = 64 - (wbits + 2 * vbits + 1);
    pk.vbits = vbits;
    pk.obits = with_offsets ? (spare < 24 ? spare : 24) : 0;
    pk.wshift = 2 * vbits + pk.obits + 1;
    pk.vmask = ((uint64_t)1 << vbits) - 1;
    pk.omask = ((uint64_t)1 << pk.obits) - 1;
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

// An offer that never waits: a reduction with no return value.  For kernels
// whose slots each receive few offers (a graph's first phase: a vertex is
// offered its incident edges only), where the check load of min_if_lower
// would put an L2 round trip between consecutive offers of a thread.
__device__ __forceinline__ void offer_min(unsigned long long *slot, uint64_t v, bool check)
{
    if (check) min_if_lower(slot, v);
    else atomicMin(slot, (unsigned long long)v);
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
// Undirected keys (MST selection keys) below a weight cap, one word each
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
    return src.resolve_dir(r, false, k, su, sv, w);
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
        // the word stands for both directions: the other end's offer
        if (keep[it])
            min_if_lower(&best[sv[it]],
                         MODE == SEL_MST ? (k[it] >> 1)
                                         : (((uint64_t)w[it] << 32) | (uint32_t)su[it]));
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
// minimum-edge selection.  Output slots are reserved with one atomicAdd per
// block step (the identity phase) or per warp staging flush, which keeps the
// shared cursor off the critical path.  Edge order is not deterministic,
// results are: selection uses a strict total order.
// the final clustering merges its remaining weight phases once fewer than
// one component per this many points is left
constexpr int64_t kMergeBelow = 64;
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
// to back in the CSR (the usual layout) and their entries fit the warp's
// row staging, the warp copies the whole range into shared memory with
// coalesced 16-byte loads and each lane then walks its own row there, with
// no per-entry row search: an inexpensive test records the kept entries,
// and a dense pass builds and offers their words (see kPhChunk).  A longer
// back-to-back range is walked as one flat
// range, 32 entries per step, each lane finding its entry's row among the
// lanes' row starts (a 5-step shuffle search).  Otherwise the warp walks
// the rows one by one.  Kept words are staged in shared memory.  In the
// identity phase (every row read) the block reserves once per step and
// copies them out coalesced; a later phase, which skips most rows, has no
// block barrier: each warp flushes its staging when it fills up and at the
// end.
constexpr int kPhStage = 256;            // staged words per warp
constexpr int kPhChunk = 8;              // entries per row between dense passes
constexpr int kPhRec = 32 * kPhChunk;    // kept-entry records per warp (dynamic shared memory)
constexpr size_t kPhRecBytes = (size_t)kPhWarps * kPhRec * sizeof(int32_t);
constexpr int kPhRowBytes = 3840;        // row staging per warp: entries x (4 + sizeof(WT))

template <typename WT>
struct RowCap {
    static constexpr int value = (kPhRowBytes / (4 + (int)sizeof(WT))) & ~15;
};

// Copies entries [e_begin, e_end) of src (E entries) into the warp's dst and
// returns the entry index that dst[0] holds: 16-byte vectors from the
// aligned vector at or before e_begin when src is 16-byte aligned (every
// vector read lies inside [0, E)), else one entry per lane.  The caller
// checks that e_end - e_begin + 16 / sizeof(T) - 1 <= CAP.
template <typename T, int CAP>
__device__ __forceinline__ int64_t warp_copy_range(const T *src, int64_t e_begin, int64_t e_end,
                                                   int64_t E, T *dst)
{
    constexpr int VEC = 16 / (int)sizeof(T);
    constexpr int NV = (CAP / VEC + 31) / 32;      // vectors per lane at most
    constexpr int NB = 3;                          // vectors in flight per lane
    const int lane = threadIdx.x & 31;
    if (((uintptr_t)src & 15) == 0) {
        const int64_t base = e_begin & ~(int64_t)(VEC - 1);
        const int nv = (int)((e_end - base + VEC - 1) / VEC);
#pragma unroll
        for (int k0 = 0; k0 < NV; k0 += NB) {
            if (lane + 32 * k0 >= nv) break;
            uint4 x[NB];
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                const int i = lane + 32 * (k0 + k);
                const int64_t e = base + (int64_t)i * VEC;
                if (i < nv && e + VEC <= E) {
                    x[k] = __ldg(reinterpret_cast<const uint4 *>(src + e));
                } else {
                    T t[VEC];
#pragma unroll
                    for (int q = 0; q < VEC; ++q) t[q] = (i < nv && e + q < E) ? src[e + q] : T(0);
                    memcpy(&x[k], t, 16);
                }
            }
#pragma unroll
            for (int k = 0; k < NB; ++k) {
                const int i = lane + 32 * (k0 + k);
                if (i < nv) *reinterpret_cast<uint4 *>(dst + (int64_t)i * VEC) = x[k];
            }
        }
        return base;
    }
    for (int64_t i = lane; i < e_end - e_begin; i += 32) dst[i] = src[e_begin + i];
    return e_begin;
}

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

// identity: the first phase (every vertex its own root: no label is read,
// and every entry is checked once for a destination out of range, and
// counted into sym[0] (u < v) or sym[1] (u > v): a symmetric graph has as
// many of each).  Its selection offers are reductions with no check load: a
// vertex is offered its own incident edges only.
// skip_root (device int, or null; -1 = none): a later phase skips the rows of
// that root -- the giant component the earlier phases built -- and emits
// both directions of each kept entry whose other end lies in it, so the
// giant still sees every edge it has to another component (each such edge is
// found once, from the row outside the giant).
template <int MODE, typename WT>
__global__ void __launch_bounds__(kPhThreads, 4)
k_phase_csr(const int32_t *first, const int32_t *deg, const int32_t *dest, const WT *weight,
            int32_t V, int64_t E, int wbits, int lo, int hi, const int *dev_lohi, int slot,
            int identity, const int32_t *skip_root, const int32_t *label, Pack pk,
            uint64_t *eout, unsigned long long *cursor, unsigned long long cap,
            unsigned long long *best, unsigned long long *sym, int *err)
{
    unsigned n_lt = 0, n_gt = 0;             // this lane's entries by direction (the warp sum is 32-bit)
    if (dev_lohi) {
        lo = dev_lohi[2 * slot];
        hi = dev_lohi[2 * slot + 1];
    }
    const int32_t skip = skip_root ? *skip_root : -1;
    constexpr int kCap = RowCap<WT>::value;
    __shared__ uint64_t stage_all[kPhWarps][kPhStage];
    __shared__ __align__(16) int32_t rdest_all[kPhWarps][kCap];
    __shared__ __align__(16) WT rw_all[kPhWarps][kCap];
    __shared__ int64_t s_cnt[kPhWarps];
    __shared__ unsigned long long s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *stage = stage_all[warp];
    int32_t *rdest = rdest_all[warp];
    WT *rw = rw_all[warp];
    extern __shared__ int32_t ph_rec[];      // kPhWarps x kPhRec kept-entry records
    int32_t *rec = ph_rec + warp * kPhRec;
    const int64_t step = (int64_t)kPhWarps * 32;
    auto root_of = [&](int32_t v) -> int32_t { return identity ? v : label[v]; };
    // a kept entry u -> v (roots lu != lv) becomes one word for the
    // undirected edge: written from the row of its smaller end, or from the
    // only row read when v lies in the skipped giant; its key is offered to
    // both ends (MST: (weight, min, max); CC: (weight, other end's root))
    // (off: the entry's offset in row u, recorded when u is the smaller end)
    auto emit = [&](bool kept, uint32_t w, int32_t u, int32_t v, int32_t lu, int32_t lv,
                    int64_t off, int &cnt) {
        const bool keep = kept && (u < v || lv == skip);
        const uint64_t k =
            keep ? pk.make(w, (uint32_t)u, (uint32_t)v,
                           (u < v && (uint64_t)off < pk.omask) ? (uint64_t)off : pk.omask)
                 : 0ull;
        phase_stage(keep, k, stage, cnt, eout, cursor, cap, err);
        if (keep) {
            offer_min(&best[lu], MODE == SEL_MST ? (k >> 1) : (((uint64_t)w << 32) | (uint32_t)lv),
                      !identity);
            offer_min(&best[lv], MODE == SEL_MST ? (k >> 1) : (((uint64_t)w << 32) | (uint32_t)lu),
                      !identity);
        }
    };
    int cnt = 0;                         // staged words (carried across steps without identity)
    // the next step's row labels are loaded one step ahead (a later phase
    // spends most steps on this load alone: its rows are mostly skipped)
    auto row_label = [&](int64_t r) -> int32_t {
        const int64_t u = r + (int64_t)warp * 32 + lane;
        return (identity || u >= V) ? (int32_t)u : label[u];
    };
    int32_t lu_next = row_label((int64_t)blockIdx.x * step);
    for (int64_t r0 = (int64_t)blockIdx.x * step; r0 < V; r0 += (int64_t)gridDim.x * step) {
        const int64_t u0 = r0 + (int64_t)warp * 32;
        const int nrows = u0 >= V ? 0 : (int)(V - u0 < 32 ? V - u0 : 32);
        int64_t f = 0, d = 0;
        int32_t lu = 0;
        bool live = false;
        const int32_t lu_this = lu_next;
        lu_next = row_label(r0 + (int64_t)gridDim.x * step);
        if (lane < nrows) {
            lu = lu_this;
            live = lu != skip;
            if (live) {
                f = first[u0 + lane];
                d = deg[u0 + lane];
                if (f < 0 || d < 0 || f + d > E) {
                    set_err(err, DEV_BAD_INPUT);
                    f = 0;
                    d = 0;
                }
            }
        }
        if (__any_sync(0xffffffffu, live)) {
            // rows back to back?  (row l + 1 starts where row l ends; a
            // skipped row must not break the range, so it counts as empty
            // only when the whole warp is flat over the live rows)
            const int64_t f_next = __shfl_down_sync(0xffffffffu, f, 1);
            const bool nl = __shfl_down_sync(0xffffffffu, live, 1);
            const bool linked = lane + 1 >= nrows || !live || !nl || f_next == f + d;
            const unsigned lmask = __ballot_sync(0xffffffffu, live);
            const int lfirst = __ffs(lmask) - 1, llast = 31 - __clz(lmask);
            const int64_t e_begin = __shfl_sync(0xffffffffu, f, lfirst);
            const int64_t e_end = __shfl_sync(0xffffffffu, f + d, llast);
            const bool flat = __all_sync(0xffffffffu, linked) && lmask == (nrows >= 32 ? 0xffffffffu : ((1u << nrows) - 1u)) &&
                              e_end - e_begin < ((int64_t)1 << 30);
            // the whole range fits the row staging (with the slack of the
            // aligned first vector of either array)
            constexpr int kSlack = 16 / (int)(sizeof(WT) < 4 ? sizeof(WT) : 4) - 1;
            if (flat && e_end - e_begin + kSlack <= kCap) {
                const int64_t db = warp_copy_range<int32_t, kCap>(dest, e_begin, e_end, E, rdest);
                const int64_t wb = warp_copy_range<WT, kCap>(weight, e_begin, e_end, E, rw);
                __syncwarp();
                const int32_t od = (int32_t)(f - db), ow = (int32_t)(f - wb);
                const int32_t u = (int32_t)(u0 + lane);
                const int dl = (int)d;                  // 0 past the last row
                const int dmax = (int)__reduce_max_sync(0xffffffffu, (unsigned)dl);
                const unsigned below = (1u << lane) - 1u;
                // kPhChunk entries of every row at a time: a cheap test of
                // each entry records the kept ones as (row lane, offset), then
                // a dense pass over the records builds, stages and offers
                // their words with every lane busy (a phase keeps a small
                // share of the entries).  The same words and offers as
                // emit(): one word per undirected edge, offered to both ends.
                for (int j0 = 0; j0 < dmax; j0 += kPhChunk) {
                    const int j1 = j0 + kPhChunk < dmax ? j0 + kPhChunk : dmax;
                    int nrec = 0;
                    for (int j = j0; j < j1; ++j) {
                        bool keep = false;
                        if (j < dl) {
                            const int32_t v = rdest[od + j];
                            if ((uint32_t)v >= (uint32_t)V) {
                                set_err(err, DEV_BAD_INPUT);
                            } else if (v != u) {
                                if (v > u) ++n_lt; else ++n_gt;
                                const int bk = (int)wbucket(wword(rw[ow + j]), wbits);
                                if (bk > lo && bk <= hi) {
                                    const int32_t lv = root_of(v);
                                    keep = lv != lu && (u < v || lv == skip);
                                }
                            }
                        }
                        const unsigned bal = __ballot_sync(0xffffffffu, keep);
                        if (keep) rec[nrec + __popc(bal & below)] = (lane << 16) | j;
                        nrec += __popc(bal);
                    }
                    __syncwarp();
                    for (int i0 = 0; i0 < nrec; i0 += 32) {
                        const bool ok = i0 + lane < nrec;
                        const int32_t rc = ok ? rec[i0 + lane] : 0;
                        const int r = rc >> 16, jr = rc & 0xffff;
                        const int32_t odr = __shfl_sync(0xffffffffu, od, r);
                        const int32_t owr = __shfl_sync(0xffffffffu, ow, r);
                        const int32_t lur = __shfl_sync(0xffffffffu, lu, r);
                        const int32_t ur = (int32_t)(u0 + r);
                        const int32_t v = ok ? rdest[odr + jr] : 0;
                        const uint32_t w = ok ? wword(rw[owr + jr]) : 0u;
                        const int32_t lv = ok ? root_of(v) : 0;
                        const uint64_t k =
                            ok ? pk.make(w, (uint32_t)ur, (uint32_t)v,
                                         (ur < v && (uint64_t)jr < pk.omask) ? (uint64_t)jr
                                                                             : pk.omask)
                               : 0ull;
                        phase_stage(ok, k, stage, cnt, eout, cursor, cap, err);
                        if (ok) {
                            offer_min(&best[lur],
                                      MODE == SEL_MST ? (k >> 1)
                                                      : (((uint64_t)w << 32) | (uint32_t)lv),
                                      !identity);
                            offer_min(&best[lv],
                                      MODE == SEL_MST ? (k >> 1)
                                                      : (((uint64_t)w << 32) | (uint32_t)lur),
                                      !identity);
                        }
                    }
                    __syncwarp();                       // the records are reused
                }
                __syncwarp();                           // the row staging is reused
            } else if (flat) {
                const int32_t frel = (int32_t)(f - e_begin);      // row starts, warp-relative
                // four 32-entry slices per step, the loads of all in flight together
                constexpr int S = 4;
                for (int64_t e0 = e_begin; e0 < e_end; e0 += 32 * S) {
                    int64_t e[S];
                    int r[S];
                    int32_t lr[S], v[S], eo[S];
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
                        eo[q] = erel - __shfl_sync(0xffffffffu, frel, rr);   // offset in its row
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
                                if (v[q] > (int32_t)(u0 + r[q])) ++n_lt; else ++n_gt;
                                const int bk = (int)wbucket(w[q], wbits);
                                cand[q] = bk > lo && bk <= hi;
                            }
                        }
                        lv[q] = cand[q] ? root_of(v[q]) : 0;
                    }
#pragma unroll
                    for (int q = 0; q < S; ++q)
                        emit(cand[q] && lv[q] != lr[q], w[q], (int32_t)(u0 + r[q]), v[q], lr[q],
                             lv[q], eo[q], cnt);
                }
            } else {
                for (int rr = 0; rr < nrows; ++rr) {
                    if (!((lmask >> rr) & 1u)) continue;
                    const int64_t fr = __shfl_sync(0xffffffffu, f, rr);
                    const int64_t dr = __shfl_sync(0xffffffffu, d, rr);
                    const int32_t lr = __shfl_sync(0xffffffffu, lu, rr);
                    const int32_t u = (int32_t)(u0 + rr);
                    for (int64_t e0 = fr; e0 < fr + dr; e0 += 32) {
                        const int64_t e = e0 + lane;
                        bool cand = false;
                        int32_t v = -1, lv = 0;
                        uint32_t w = 0;
                        if (e < fr + dr) {
                            v = dest[e];
                            if (v < 0 || v >= V) {
                                set_err(err, DEV_BAD_INPUT);
                            } else if (v != u) {
                                if (v > u) ++n_lt; else ++n_gt;
                                w = wword(weight[e]);
                                const int bk = (int)wbucket(w, wbits);
                                cand = bk > lo && bk <= hi;
                                if (cand) lv = root_of(v);
                            }
                        }
                        emit(cand && lv != lr, w, u, v, lr, lv, e - fr, cnt);
                    }
                }
            }
        }
        if (identity) {
            // identity is uniform over the grid, so every thread of the
            // block takes the reservation's barriers
            if (lane == 0) s_cnt[warp] = cnt;
            const bool fits = phase_reserve(s_cnt, &s_base, cursor, 1, cap, err);
            if (fits) {
                const unsigned long long at = s_base + (unsigned long long)s_cnt[warp];
                for (int i = lane; i < cnt; i += 32) eout[at + i] = stage[i];
            }
            __syncthreads();      // staging and s_cnt are reused by the next step
            cnt = 0;
        }
    }
    if (!identity && cnt > 0) {
        __syncwarp();
        phase_flush_warp(stage, cnt, eout, cursor, cap, err);
    }
    if (sym) {
        n_lt = __reduce_add_sync(0xffffffffu, (unsigned)n_lt);
        n_gt = __reduce_add_sync(0xffffffffu, (unsigned)n_gt);
        if ((threadIdx.x & 31) == 0 && (n_lt | n_gt)) {
            atomicAdd(&sym[0], (unsigned long long)n_lt);
            atomicAdd(&sym[1], (unsigned long long)n_gt);
        }
    }
}

// The root holding most vertices (from a strided sample of 2048 vertices, in
// a shared-memory count table), or -1 when none holds a quarter of the
// sample: the rows a later weight phase may skip.
constexpr int kGiantSample = 2048;
__global__ void __launch_bounds__(1024)
k_pick_giant(const int32_t *label, int64_t V0, int32_t *out)
{
    constexpr int T = 2 * kGiantSample;
    __shared__ int32_t key[T];
    __shared__ int32_t cnt[T];
    __shared__ unsigned long long best;
    for (int i = threadIdx.x; i < T; i += blockDim.x) {
        key[i] = -1;
        cnt[i] = 0;
    }
    if (threadIdx.x == 0) best = 0ull;
    __syncthreads();
    const int64_t n = V0 < kGiantSample ? V0 : kGiantSample;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const int32_t r = label[(j * V0) / n];
        unsigned slot = ((uint32_t)r * 2654435761u) % T;
        for (int probe = 0; probe < T; ++probe) {
            int32_t k = key[slot];
            if (k == -1) {
                k = atomicCAS(&key[slot], -1, r);
                if (k == -1) k = r;
            }
            if (k == r) {
                atomicAdd(&cnt[slot], 1);
                break;
            }
            slot = (slot + 1) % T;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < T; i += blockDim.x)
        if (cnt[i]) atomicMax(&best, ((unsigned long long)cnt[i] << 32) | (uint32_t)key[i]);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int64_t c = (int64_t)(best >> 32);
        *out = (n > 0 && 4 * c >= n) ? (int32_t)(uint32_t)best : -1;
    }
}

// Same for an upper-triangle CSR with uint8 weights: one word per kept entry,
// offered to both ends.  Co-association rows are long (thousands of entries), so a
// warp takes one row and walks it in 128-entry groups, each lane taking four
// consecutive entries: their four weights (one word) are read first and
// tested against the phase's range four bytes at once, and the four column
// indices (16 bytes) only when one of the weights falls in the range, so a
// phase over a narrow range reads little more than the weight array; only
// those entries gather the other end's label (none in the first phase, whose
// labels are the identity).  Kept entries update the selection slots and the
// per-weight counts as they are found and are staged in shared memory in walk
// order; the warp then reserves the row's words with one atomic and copies
// the staging out.  A row with more kept entries than the staging holds
// walks again to write them.  Each entry is checked (j > i, j < n) in the
// phase whose range holds its weight.
constexpr int kUpStage = 128;      // staged edge words per warp

// bit q: byte q of w lies in [L, H], with c1 = (0x8000 - L) and c2 = (0x7fff -
// H) in both 16-bit halves: bytes 0, 2 and bytes 1, 3 are spread to 16-bit
// lanes, where bit 15 of x + c1 is x >= L and bit 15 of x + c2 is x > H
__device__ __forceinline__ unsigned bytes_in_range(uint32_t w, uint32_t c1, uint32_t c2)
{
    const uint32_t e = __byte_perm(w, 0u, 0x4240), o = __byte_perm(w, 0u, 0x4341);
    const uint32_t me = (e + c1) & ~(e + c2), mo = (o + c1) & ~(o + c2);
    return ((me >> 15) & 1u) | ((mo >> 14) & 2u) | ((me >> 29) & 4u) | ((mo >> 28) & 8u);
}

__global__ void __launch_bounds__(kPhThreads, 3)
k_phase_upper(const int64_t *indptr, const int32_t *indices, const uint8_t *w, int32_t n,
              int64_t nnz, int lo, int hi, int dense, int ident, int64_t row0, int64_t row1,
              const int32_t *label, Pack pk, uint64_t *eout, unsigned long long *cursor,
              unsigned long long cap, unsigned long long *best, unsigned long long *khist,
              int *err)
{
    constexpr int G = 4;
    __shared__ unsigned s_kh[256];           // kept entries per weight, this block
    __shared__ uint64_t stage_all[kPhWarps][kUpStage];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) s_kh[b] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    uint64_t *stage = stage_all[threadIdx.x >> 5];
    const uint32_t c1 = 0x00010001u * (uint32_t)(0x8000 - (lo + 1));
    const uint32_t c2 = 0x00010001u * (uint32_t)(0x7fff - hi);
    const int64_t nwarps = (int64_t)gridDim.x * kPhWarps;
    for (int64_t i = row0 + (int64_t)blockIdx.x * kPhWarps + (threadIdx.x >> 5); i < row1;
         i += nwarps) {
        const int64_t s = indptr[i], e_end = indptr[i + 1];
        if (s < 0 || e_end < s || e_end > nnz) {
            if (lane == 0) set_err(err, DEV_BAD_INPUT);
            continue;
        }
        if (s == e_end) continue;
        const int32_t li = ident ? (int32_t)i : label[i];
        const int64_t a0 = s & ~(int64_t)3;        // groups start on 16-byte index boundaries
        // weights of the lane's entries e .. e+3 (zero outside the arrays)
        auto wload = [&](int64_t e) -> uint32_t {
            if (e >= e_end) return 0u;
            if (e + 3 < nnz) return __ldg(reinterpret_cast<const uint32_t *>(w + e));
            uint32_t v = 0u;
            for (int q = 0; q < 4 && e + q < nnz; ++q) v |= (uint32_t)w[e + q] << (8 * q);
            return v;
        };
        // bit q: entry e+q is in the row with its weight in (lo, hi]
        auto cmask = [&](int64_t e, uint32_t wv) -> unsigned {
            unsigned m = bytes_in_range(wv, c1, c2);
            if (e < s || e + 4 > e_end) {
                const int64_t a = s - e, b = e_end - e;     // valid entries [a, b)
                const int qa = a < 0 ? 0 : (a > 4 ? 4 : (int)a);
                const int qb = b < 0 ? 0 : (b > 4 ? 4 : (int)b);
                m &= (0xfu << qa) & (0xfu >> (4 - qb));
            }
            return m;
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
            unsigned c2m = cm;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (((cm >> q) & 1u) && (jj[q] <= i || jj[q] >= n)) {
                    set_err(err, DEV_BAD_INPUT);
                    c2m &= ~(1u << q);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                lj[q] = ((c2m >> q) & 1u) ? (ident ? jj[q] : label[jj[q]]) : li;
            unsigned km = 0u;
#pragma unroll
            for (int q = 0; q < 4; ++q) km |= (lj[q] != li ? 1u : 0u) << q;
            return km;
        };
        // the row's kept words in walk order: warp prefix of the lanes' counts
        auto place = [&](unsigned km, int c, int &tot) -> int {
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int o = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += o;
            }
            tot = __shfl_sync(0xffffffffu, incl, 31);
            return incl - c;
        };
        int cnt = 0, staged = 0;
        bool spill = false;
        uint64_t m = kNone;
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
                const unsigned km = cm[u] ? keep(cm[u], jv[u], lj) : 0u;
                if (!__any_sync(0xffffffffu, km != 0u)) continue;
                const int c = __popc(km);
                int tot;
                int p = staged + place(km, c, tot);
                if (staged + tot > kUpStage) spill = true;
                const int32_t jj[4] = {jv[u].x, jv[u].y, jv[u].z, jv[u].w};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (!((km >> q) & 1u)) continue;
                    const uint32_t wq = (wv[u] >> (8 * q)) & 255u;
                    const uint64_t k = pk.make(wq, (uint32_t)i, (uint32_t)jj[q]);
                    atomicAdd(&s_kh[wq], 1u);
                    m = (k >> 1) < m ? (k >> 1) : m;
                    min_if_lower(&best[lj[q]], k >> 1);
                    if (!spill) stage[p++] = k;
                }
                staged += tot;
                cnt += c;
            }
        }
        cnt = __reduce_add_sync(0xffffffffu, cnt);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            const uint64_t x = __shfl_xor_sync(0xffffffffu, m, o);
            m = x < m ? x : m;
        }
        if (cnt == 0) continue;
        if (lane == 0 && m != kNone) min_if_lower(&best[li], m);
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(cursor, (unsigned long long)cnt);
        at = __shfl_sync(0xffffffffu, at, 0);
        if (at + (unsigned long long)cnt > cap) {
            if (lane == 0) set_err(err, DEV_CAPACITY);
            __syncwarp();
            continue;
        }
        __syncwarp();
        if (!spill) {
            for (int t = lane; t < cnt; t += 32) eout[at + t] = stage[t];
            __syncwarp();                  // the staging is reused by the next row
            continue;
        }
        // more kept entries than the staging holds: walk again to write them
        for (int64_t g = a0; g < e_end; g += 128) {
            const int64_t e = g + 4 * lane;
            const uint32_t wv = wload(e);
            const unsigned cm = cmask(e, wv);
            const int4 jv = jload(e, cm);
            int32_t lj[4];
            const unsigned km = cm ? keep(cm, jv, lj) : 0u;
            if (!__any_sync(0xffffffffu, km != 0u)) continue;
            const int c = __popc(km);
            int tot;
            unsigned long long p = at + (unsigned long long)place(km, c, tot);
            const int32_t jj[4] = {jv.x, jv.y, jv.z, jv.w};
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if ((km >> q) & 1u)
                    eout[p++] = pk.make((wv >> (8 * q)) & 255u, (uint32_t)i, (uint32_t)jj[q]);
            at += (unsigned long long)tot;
        }
        __syncwarp();
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
    int ident;            // the labels are still the identity (no merges yet)
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
// at cumulative fractions p1 (per mille of the entries; a tuning-table
// knob, default a quarter) and 1 of the histogram, one slot each in lohi
// (an unused slot holds the empty range (255, 255]).
constexpr int kPhaseSlots = 2;
__global__ void k_phase_plan(const unsigned long long *hist, int *lohi, int p1_permille)
{
    __shared__ unsigned long long h[256];
    for (int b = threadIdx.x; b < 256; b += blockDim.x) h[b] = hist[b];
    __syncthreads();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double fracs[kPhaseSlots] = {p1_permille / 1000.0, 1.0};
    int lo[8], hi[8];
    const int np = phase_ranges(h, fracs, kPhaseSlots, lo, hi);
    for (int q = 0; q < kPhaseSlots; ++q) {
        lohi[2 * q] = q < np ? lo[q] : 255;
        lohi[2 * q + 1] = q < np ? hi[q] : 255;
    }
}

constexpr int kMaxRounds = 96;   // Boruvka rounds per phase (halving: 96 is never reached)

// Round state kept on the device (int64 words), so that the phases of an MST
// can be queued back to back without a host read:
enum : int {
    C_V = 0,          // supervertices at the start of the next round
    C_E = 1,          // edge words in the round kernel's input buffer
    C_NMST = 2,       // forest edges emitted so far (all phases)
    C_CURSOR = 3,     // phase-build output cursor
    C_ROUNDS = 4,     // rounds run by the last round kernel
    C_DONE = 5,       // how the last round kernel ended (see k_rounds)
    C_ROUNDS_ALL = 6, // rounds run since the engine's reset (all phases)
    C_EBUF = 7,       // edge buffer holding the last round's survivors (0 or 1)
    C_AUX0 = 8,       // scratch totals of single-pass kernels
    C_AUX1 = 9,
    C_SYM_LT = 10,    // CSR entries u -> v with u < v (symmetry check)
    C_SYM_GT = 11,    // ... with u > v
    C_COUNT = 16
};

// ---------------------------------------------------------------------------
// Boruvka rounds: all rounds of a phase in ONE persistent kernel.
//
// Supervertices are named by an original vertex, their root: `parent` is a
// union-find forest over the original vertices (a root points to itself), so
// a round never renumbers anything and never sweeps all original vertices;
// an edge endpoint or a key endpoint finds its supervertex by following
// parent pointers (and shortens the path it walked).  Only the ACTIVE roots
// -- those with an edge to another supervertex -- are visited, from a list
// kept in increasing id order.
//
// The participants are either every block of a cooperative grid (all blocks
// resident at once, so they may wait on one another) or a single block.
// Each participant owns a contiguous chunk of the original vertices (its
// part of the active list) and a contiguous segment of the phase's edge
// words; both shrink in place.  Between the steps of a round the
// participants meet at a barrier: a bounded spin on an arrival counter for
// the grid, __syncthreads for one block.  Once few active roots and edges are
// left, the grid's other blocks leave and block 0 runs the remaining rounds
// alone for every participant's chunk and segment (no grid barriers).
// A round is
//   A. per active root s: its successor t (the root of the other end of its
//      selected key); a mutual pick (t's successor is s) is broken towards
//      the larger id, so the smaller one stays a root
//      (MyML/MyML/graph/mst.py:283-305); color[s] = t, or s.
//   B. in list order: each non-root emits its key as a forest edge (slots in
//      root-id order, from the participants' counts), finds its new root
//      (bounded chase with compare-and-swap path halving over color) and
//      points its parent there; the roots that still have an edge stay in the
//      list, and their selection slots are cleared.
//   D. contraction fused with the next round's minimum-edge selection: each
//      edge word whose endpoints now have different roots stays in its
//      segment (compacted in place: a tile's words are in registers before
//      any of the tile's survivors is written, and survivors never move past
//      their tile) and is offered to both its roots' slots (one atomicMin per
//      run of equal first root in a warp, and one for the other root).  Edge order does not matter:
//      selection uses total orders, so every result is independent of it.
// Three barriers per round.  After the last one every participant reads the
// same sizes and takes the same decision to stop:
//   C_DONE = 1 converged (no edge left), 2 no contraction (not a valid
//   graph), 3 round cap, 4 a device error.
// Root ids keep the reference's choices: its renumbering is order-preserving,
// so "smaller id" and "smallest destination" compare the same way, and its
// final component number is the rank of the root id (k_rank_roots).
// The steps handle several elements per thread at a time with all loads of
// one level issued together: they are chains of dependent gathers, so the
// independent chains in flight, not bandwidth, set their speed.
// ---------------------------------------------------------------------------
constexpr int kRT = 1024;                       // round-kernel threads per block
constexpr int kRItems = 4;                      // edge words per thread per tile
constexpr int kRV = 4;                          // vertices per thread per step
constexpr int64_t kRTile = (int64_t)kRT * kRItems;
constexpr int kRWarps = kRT / 32;
constexpr int kMaxTeam = 148 * 8;               // participants (blocks) at most
constexpr long long kBarrierSpins = 1ll << 21;  // about a second of waiting
constexpr int64_t kSoloActive = 1024;           // block 0 alone below these sizes
constexpr int64_t kSoloEdges = 8192;
constexpr int kFindLimit = 1 << 20;             // parent-chain steps (a forest is shorter)

struct GridBarrier {
    unsigned count;       // arrivals since the launch began (never reset inside one)
    unsigned pad;
};

// Grid-wide barrier of a cooperative launch.  Thread 0 of each block adds
// its arrival to a counter that only grows, with no return value, and waits
// until the counter reaches (barriers passed + 1) x blocks: no block resets
// anything, so the last arrival is the only write the others wait for.  The
// counter starts at zero (the host clears it before each launch).  The wait
// gives up after about a second (DEV_SPIN_LIMIT), or as soon as any block
// has raised an error, so a block that left early never holds the others.
// Returns false when it gave up.  The arrival is a release and the polling
// load an acquire (gpu scope); with the block barriers around them they
// order every thread's writes before the arrival and its reads after the
// wait.  The data exchanged between blocks is read with L1-bypassing loads.
__device__ __forceinline__ bool grid_barrier(GridBarrier *b, unsigned &passed, int *err)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned target = (passed + 1u) * gridDim.x;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&b->count) : "memory");
        auto count_now = [&]() -> unsigned {
            unsigned c;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(c) : "l"(&b->count) : "memory");
            return c;
        };
        int ok = 1;
        long long spins = 0;
        while ((int)(count_now() - target) < 0) {
            if (*(volatile int *)err) {
                ok = 0;
                break;
            }
            if (++spins > kBarrierSpins) {
                set_err(err, DEV_SPIN_LIMIT);
                ok = 0;
                break;
            }
            if (spins > 256) __nanosleep(32);
        }
        s_ok = ok;
    }
    __syncthreads();
    ++passed;
    return s_ok != 0;
}

struct RoundArgs {
    Pack pk;
    int64_t V0;
    uint64_t *e;                  // edge words of the phase (compacted per segment)
    int32_t *parent;              // V0: union-find parent (a root points to itself)
    unsigned long long *best;     // V0: selection slot per root
    int32_t *color;               // V0: successor, then new root, per active root
    int32_t *act;                 // V0: active roots, per participant chunk
    uint64_t *mst;                // forest keys, appended at cnt[C_NMST] (MST mode)
    int32_t *part;                // 2 x kMaxTeam: per participant (emits, merges)
    int32_t *alen;                // kMaxTeam: active roots per participant
    int64_t *seg;                 // kMaxTeam: edge words per participant segment
    int64_t *cnt;                 // C_* round state
    int64_t *trace;               // 3 x kMaxRounds: (V, E, active) per round
    GridBarrier *bar;
    int *err;
    int max_rounds;
    int from_cursor;              // edge count = cnt[C_CURSOR] (a queued phase's build)
    int first_phase;              // supervertex count = V0
};

// Roots of N vertices at once (all parent loads of one level issued
// together); each vertex whose first parent was not its root is pointed at
// the root (a benign race: every writer writes the same root).  Negative
// ids (empty lanes) are left alone: they must not all walk and rewrite the
// path of one real vertex.
// The parent loads may be served by L1: late rounds send most finds to the
// few roots left, and L2-only loads of those few lines from every SM
// serialise (a 20x slower contraction measured on a 16-NN graph).  The
// entries a round rewrites (merged roots, step B) were written before the
// barrier that precedes the finds, whose acquire fence orders the later
// loads after them; within a step the only writes are path compressions,
// so a stale value is an older ancestor and the walk still ends at the root.
template <int N>
__device__ __forceinline__ void find_batch(int32_t *parent, int32_t (&x)[N], int *err)
{
    int32_t r[N], first[N];
    bool go[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        r[i] = x[i] >= 0 ? parent[x[i]] : x[i];
        first[i] = r[i];
        go[i] = r[i] != x[i];
    }
    for (int step = 0;; ++step) {
        int32_t up[N];
        bool any = false;
#pragma unroll
        for (int i = 0; i < N; ++i) up[i] = go[i] ? parent[r[i]] : r[i];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (go[i] && up[i] != r[i]) {
                r[i] = up[i];
                any = true;
            } else {
                go[i] = false;
            }
        }
        if (!any) break;
        if (step > kFindLimit) {
            set_err(err, DEV_CHASE_LIMIT);
            break;
        }
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
        if (first[i] != x[i] && first[i] != r[i]) parent[x[i]] = r[i];
        x[i] = r[i];
    }
}

// Successors of up to kRV active roots at once (s[i] < 0: none): the root of
// the other end of each selected key, or the root itself when it selected
// nothing.
template <int MODE>
__device__ __forceinline__ void succ_batch(const RoundArgs &a, const int32_t (&s)[kRV],
                                           int32_t (&t)[kRV])
{
    uint64_t b[kRV];
#pragma unroll
    for (int i = 0; i < kRV; ++i) b[i] = s[i] >= 0 ? __ldcg(a.best + s[i]) : kNone;
    if constexpr (MODE == SEL_CC) {
#pragma unroll
        for (int i = 0; i < kRV; ++i) t[i] = b[i] == kNone ? s[i] : (int32_t)(uint32_t)b[i];
    } else {
    int32_t e[2 * kRV];
#pragma unroll
    for (int i = 0; i < kRV; ++i) {
        const bool ok = b[i] != kNone;
        e[2 * i] = ok ? (int32_t)a.pk.sel_a(b[i]) : -1;
        e[2 * i + 1] = ok ? (int32_t)a.pk.sel_b(b[i]) : -1;
    }
    find_batch<2 * kRV>(a.parent, e, a.err);
#pragma unroll
    for (int i = 0; i < kRV; ++i)
        t[i] = b[i] == kNone ? s[i] : (e[2 * i] == s[i] ? e[2 * i + 1] : e[2 * i]);
    }
}

template <int MODE, bool GRID>
__global__ void __launch_bounds__(kRT, 1)
k_rounds(RoundArgs a)
{
    __shared__ int s_off[kRItems][kRWarps];
    __shared__ int s_base;
    __shared__ int s_err;
    const int64_t P = GRID ? (int64_t)gridDim.x : 1, p = GRID ? (int64_t)blockIdx.x : 0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bool solo = !GRID;                  // one block does all the work
    int64_t Pe = P;                     // participants whose chunks and segments are in use
    unsigned passed = 0;                // grid barriers passed (the same in every block)
    auto sync = [&]() -> bool {
        if (!solo) return grid_barrier(a.bar, passed, a.err);
        __syncthreads();
        return true;
    };
    // a queued weight phase starts from its build's cursor and the previous
    // phase's supervertex count (V0 for the first phase)
    int64_t V = a.first_phase ? a.V0 : __ldcg(a.cnt + C_V);
    int64_t E = __ldcg(a.cnt + (a.from_cursor ? C_CURSOR : C_E));
    int64_t nmst = __ldcg(a.cnt + C_NMST);
    const int64_t E0 = E;
    const int64_t seg_stride = (E0 + P - 1) / P;     // edge segment of participant q
    const int64_t vchunk = (a.V0 + P - 1) / P;       // vertex chunk of participant q
    auto ebase = [&](int64_t q) { return min(E0, q * seg_stride); };
    auto vbase = [&](int64_t q) { return min(a.V0, q * vchunk); };

    // ---- active list: the roots with a selection, in id order -------------
    // (kRV consecutive vertices per thread: the loads of all in flight, one
    // block scan per kRT * kRV vertices)
    for (int64_t q = solo ? 0 : p; q < (solo ? P : p + 1); ++q) {
        const int64_t v0 = vbase(q), v1 = min(a.V0, v0 + vchunk);
        int64_t kept = 0;
        for (int64_t xb = v0; xb < v1; xb += (int64_t)kRT * kRV) {
            const int64_t x0 = xb + (int64_t)tid * kRV;
            int32_t par[kRV];
            uint64_t sel[kRV];
#pragma unroll
            for (int i = 0; i < kRV; ++i) {
                const bool in = x0 + i < v1;
                par[i] = in ? __ldcg(a.parent + x0 + i) : -1;
                sel[i] = in ? __ldcg(a.best + x0 + i) : kNone;
            }
            int c = 0;
            bool on[kRV];
#pragma unroll
            for (int i = 0; i < kRV; ++i) {
                on[i] = par[i] == (int32_t)(x0 + i) && sel[i] != kNone;
                c += on[i] ? 1 : 0;
            }
            int64_t ttot;
            int64_t at = v0 + kept + block_excl_sum_shfl<kRT>(c, ttot);
#pragma unroll
            for (int i = 0; i < kRV; ++i)
                if (on[i]) a.act[at++] = (int32_t)(x0 + i);
            kept += ttot;
        }
        const int64_t e0 = ebase(q);
        if (tid == 0) {
            a.alen[q] = (int32_t)kept;
            a.seg[q] = min(E0, e0 + seg_stride) - e0;
        }
    }
    if (tid == 0) s_err = *(volatile int *)a.err;
    __syncthreads();
    int round = 0, done = s_err ? 4 : ((E == 0 || V <= 1) ? 1 : 0);
    if (!done && !sync()) done = 4;
    int64_t Aact = 0;                                 // active roots this round
    if (!done) {
        int64_t x = 0;
        for (int64_t j = tid; j < P; j += kRT) x += __ldcg(a.alen + j);
        block_excl_sum_shfl<kRT>(x, Aact);
    }
    while (!done) {
        const int64_t q0 = solo ? 0 : p, q1 = solo ? Pe : p + 1;
        // ---- A: successors, mutual picks, per-participant counts ---------
        for (int64_t q = q0; q < q1; ++q) {
            const int32_t *al = a.act + vbase(q);
            const int64_t n = __ldcg(a.alen + q);
            int64_t mine = 0;                   // (forest edges << 32) | merges
            for (int64_t ib = tid; ib < n; ib += (int64_t)kRT * kRV) {
                int32_t s[kRV], t[kRV], tt[kRV], m[kRV];
#pragma unroll
                for (int i = 0; i < kRV; ++i) {
                    const int64_t j = ib + (int64_t)i * kRT;
                    s[i] = j < n ? __ldcg(al + j) : -1;
                }
                succ_batch<MODE>(a, s, t);
                // mutual pick: only a smaller s with a successor needs t's
#pragma unroll
                for (int i = 0; i < kRV; ++i) m[i] = (s[i] >= 0 && s[i] < t[i]) ? t[i] : -1;
                succ_batch<MODE>(a, m, tt);
#pragma unroll
                for (int i = 0; i < kRV; ++i) {
                    if (s[i] < 0) continue;
                    const bool keep = t[i] != s[i] && !(m[i] >= 0 && tt[i] == s[i]);
                    a.color[s[i]] = keep ? t[i] : s[i];
                    mine += keep ? ((MODE == SEL_MST ? (1ll << 32) : 0ll) | 1ll) : 0ll;
                }
            }
            int64_t btot;
            block_excl_sum_shfl<kRT>(mine, btot);
            if (tid == 0) {
                a.part[q] = (int32_t)(btot >> 32);             // forest edges
                a.part[kMaxTeam + q] = (int32_t)(btot & 0xffffffffll);   // merges
            }
        }
        if (!sync()) break;

        // ---- B: forest edges, new roots, the next active list -----------
        int64_t merges = 0, epre = 0;           // all merges; forest edges before q0
        {
            // both below 2^31 (at most V0 each): one scan of (merges << 32) | edges
            int64_t x = 0, tot = 0;
            for (int64_t j = tid; j < Pe; j += kRT) {
                x += (int64_t)__ldcg(a.part + kMaxTeam + j) << 32;
                if (j < q0) x += __ldcg(a.part + j);
            }
            block_excl_sum_shfl<kRT>(x, tot);
            merges = tot >> 32;
            epre = tot & 0xffffffffll;
        }
        for (int64_t q = q0; q < q1; ++q) {
            int32_t *al = a.act + vbase(q);
            const int64_t n = __ldcg(a.alen + q);
            int64_t kept = 0;
            for (int64_t base = 0; base < n; base += (int64_t)kRT * kRV) {
                // thread tid takes kRV consecutive entries, so the block scans
                // keep list order
                int32_t s[kRV], c[kRV];
                bool root[kRV], act[kRV], stay[kRV];
                int64_t fl = 0;                 // (forest edges << 32) | staying roots
                const int64_t jb = base + (int64_t)tid * kRV;
#pragma unroll
                for (int i = 0; i < kRV; ++i) {
                    const bool in = jb + i < n;
                    s[i] = in ? __ldcg(al + jb + i) : 0;
                }
#pragma unroll
                for (int i = 0; i < kRV; ++i) {
                    const bool in = jb + i < n;
                    c[i] = in ? __ldcg(a.color + s[i]) : 0;
                    root[i] = in && c[i] == s[i];
                    act[i] = in && !root[i];
                    // a root stays active only while it has an edge
                    stay[i] = root[i] && __ldcg(a.best + s[i]) != kNone;
                    fl += ((act[i] && MODE == SEL_MST) ? (1ll << 32) : 0ll) | (stay[i] ? 1ll : 0ll);
                }
                int64_t ttot;
                int64_t ex = block_excl_sum_shfl<kRT>(fl, ttot);
                __syncthreads();                // every entry of the tile is read
                int64_t ep = epre + (ex >> 32), kp = kept + (ex & 0xffffffffll);
#pragma unroll
                for (int i = 0; i < kRV; ++i) {
                    if (stay[i]) al[kp++] = s[i];
                    if (act[i] && MODE == SEL_MST) a.mst[nmst + ep++] = __ldcg(a.best + s[i]);
                }
                // new roots of the non-roots: chases interleaved
                for (int64_t guard = 0;; ++guard) {
                    bool any = false;
                    int32_t up[kRV], g[kRV];
#pragma unroll
                    for (int i = 0; i < kRV; ++i) up[i] = act[i] ? __ldcg(a.color + c[i]) : 0;
#pragma unroll
                    for (int i = 0; i < kRV; ++i) {
                        if (act[i] && up[i] == c[i]) {
                            act[i] = false;
                            a.color[s[i]] = c[i];
                            a.parent[s[i]] = c[i];
                        }
                        g[i] = act[i] ? __ldcg(a.color + up[i]) : 0;
                    }
#pragma unroll
                    for (int i = 0; i < kRV; ++i) {
                        if (!act[i]) continue;
                        if (g[i] != up[i]) atomicCAS(a.color + c[i], up[i], g[i]);
                        c[i] = g[i];
                        any = true;
                    }
                    if (!any) break;
                    if (guard > V + 64) {
                        set_err(a.err, DEV_CHASE_LIMIT);
                        break;
                    }
                }
#pragma unroll
                for (int i = 0; i < kRV; ++i)
                    if (stay[i]) a.best[s[i]] = kNone;
                kept += ttot & 0xffffffffll;
                epre += ttot >> 32;
            }
            if (tid == 0) a.alen[q] = (int32_t)kept;
        }
        if (!sync()) break;

        // ---- D: contraction of the segments, in place ---------------------
        for (int64_t q = q0; q < q1; ++q) {
            uint64_t *seg = a.e + ebase(q);
            const int64_t elen = __ldcg(a.seg + q);
            int64_t out = 0;                    // survivors written so far
            for (int64_t base = 0; base < elen; base += kRTile) {
                uint64_t k[kRItems];
#pragma unroll
                for (int it = 0; it < kRItems; ++it) {
                    const int64_t i = base + (int64_t)it * kRT + tid;
                    k[it] = i < elen ? __ldcg(seg + i) : kNone;
                }
                // dead words (self loops left by a CSR load) have a == b
                int32_t ep[2 * kRItems];
                bool ok[kRItems];
#pragma unroll
                for (int it = 0; it < kRItems; ++it) {
                    ok[it] = k[it] != kNone && a.pk.a(k[it]) < (uint64_t)a.V0 &&
                             a.pk.b(k[it]) < (uint64_t)a.V0;
                    ep[2 * it] = ok[it] ? (int32_t)a.pk.a(k[it]) : -1;
                    ep[2 * it + 1] = ok[it] ? (int32_t)a.pk.b(k[it]) : -2;
                }
                find_batch<2 * kRItems>(a.parent, ep, a.err);
                bool keep[kRItems];
                unsigned bal[kRItems];
#pragma unroll
                for (int it = 0; it < kRItems; ++it) {
                    const int32_t su = ep[2 * it], sv = ep[2 * it + 1];
                    keep[it] = ok[it] && su != sv;
                    bal[it] = __ballot_sync(0xffffffffu, keep[it]);
                    if (lane == 0) s_off[it][warp] = __popc(bal[it]);
                    // one word per undirected edge: offered to both ends
                    const uint64_t sel = MODE == SEL_MST
                                             ? (k[it] >> 1)
                                             : (((uint64_t)a.pk.w(k[it]) << 32) | (uint32_t)sv);
                    seg_min_atomic(keep[it], su, sel, a.best);
                    if (keep[it])
                        min_if_lower(&a.best[sv],
                                     MODE == SEL_MST
                                         ? (k[it] >> 1)
                                         : (((uint64_t)a.pk.w(k[it]) << 32) | (uint32_t)su));
                }
                __syncthreads();                // the tile's words are all read
                if (warp == 0) {
                    // exclusive scan of the per-(item, warp) counts in
                    // (item, warp) order
                    constexpr int N = kRItems * kRWarps;
                    constexpr int PER = N / 32;
                    int cc[PER];
                    int sum = 0;
#pragma unroll
                    for (int j = 0; j < PER; ++j) {
                        const int idx = lane * PER + j;
                        cc[j] = s_off[idx / kRWarps][idx % kRWarps];
                        sum += cc[j];
                    }
                    int incl = sum;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const int o = __shfl_up_sync(0xffffffffu, incl, d);
                        if (lane >= d) incl += o;
                    }
                    int r = incl - sum;
#pragma unroll
                    for (int j = 0; j < PER; ++j) {
                        const int idx = lane * PER + j;
                        s_off[idx / kRWarps][idx % kRWarps] = r;
                        r += cc[j];
                    }
                    if (lane == 31) s_base = incl;
                }
                __syncthreads();
                const unsigned lt = (1u << lane) - 1u;
#pragma unroll
                for (int it = 0; it < kRItems; ++it)
                    if (keep[it]) seg[out + s_off[it][warp] + __popc(bal[it] & lt)] = k[it];
                out += s_base;
                __syncthreads();                // s_off and s_base are reused
            }
            if (tid == 0) a.seg[q] = out;
        }
        if (!sync()) break;

        // ---- E: the next round's sizes, the same in every participant ----
        int64_t En = 0, An = 0;
        {
            // the error flag is read beside the counts; the scans' block
            // barriers publish s_err
            const int e_now = tid == 0 ? *(volatile int *)a.err : 0;
            int64_t x = 0, y = 0;
            for (int64_t j = tid; j < Pe; j += kRT) {
                x += __ldcg(a.seg + j);
                y += __ldcg(a.alen + j);
            }
            if (tid == 0) s_err = e_now;
            block_excl_sum_shfl<kRT>(x, En);
            block_excl_sum_shfl<kRT>(y, An);
        }
        if (p == 0 && tid == 0 && round < kMaxRounds) {
            a.trace[3 * round] = V;
            a.trace[3 * round + 1] = E;
            a.trace[3 * round + 2] = Aact;
        }
        ++round;
        nmst += MODE == SEL_MST ? merges : 0;
        if (s_err) done = 4;
        else if (En == 0) done = 1;
        else if (merges == 0) done = 2;
        else if (round >= a.max_rounds) done = 3;
        V -= merges;
        E = En;
        Aact = An;
        __syncthreads();                        // s_err is rewritten next round
        if (!done && !solo && An <= kSoloActive && En <= kSoloEdges) {
            // every block decides alike: the others leave, and block 0 moves
            // all active roots and edge words to the front of its own chunk
            // and segment, in participant order (list order = id order is
            // kept).  The participants' counts are read at once and their
            // exclusive prefixes kept in shared memory; the copy then runs
            // over the concatenated elements, kRT at a time, each element
            // finding its participant by binary search.  A destination never
            // passes its source, so each chunk is read before it is written.
            solo = true;
            if (p != 0) return;
            static_assert(2 * kRT >= kMaxTeam, "two participants per thread");
            __shared__ int64_t s_apre[kMaxTeam + 1], s_epre[kMaxTeam + 1];
            {
                const int64_t j0 = 2 * (int64_t)tid;
                const int64_t a0 = j0 < Pe ? (int64_t)__ldcg(a.alen + j0) : 0;
                const int64_t a1 = j0 + 1 < Pe ? (int64_t)__ldcg(a.alen + j0 + 1) : 0;
                const int64_t m0 = j0 < Pe ? __ldcg(a.seg + j0) : 0;
                const int64_t m1 = j0 + 1 < Pe ? __ldcg(a.seg + j0 + 1) : 0;
                int64_t at, mt;
                const int64_t ax = block_excl_sum_shfl<kRT>(a0 + a1, at);
                const int64_t mx = block_excl_sum_shfl<kRT>(m0 + m1, mt);
                if (j0 < Pe) {
                    s_apre[j0] = ax;
                    s_epre[j0] = mx;
                }
                if (j0 + 1 < Pe) {
                    s_apre[j0 + 1] = ax + a0;
                    s_epre[j0 + 1] = mx + m0;
                }
                if (tid == 0) {
                    s_apre[Pe] = at;
                    s_epre[Pe] = mt;
                }
            }
            __syncthreads();
            const int64_t ao = s_apre[Pe], eo = s_epre[Pe];
            // the participant holding concatenated element i: the last q < Pe
            // with pre[q] <= i (pre[0] = 0)
            auto owner = [&](const int64_t *pre, int64_t i) -> int64_t {
                int64_t lo = 0, hi = Pe - 1;
                while (lo < hi) {
                    const int64_t mid = (lo + hi + 1) >> 1;
                    if (pre[mid] <= i) lo = mid;
                    else hi = mid - 1;
                }
                return lo;
            };
            for (int64_t c = 0; c < ao; c += kRT) {
                const int64_t i = c + tid;
                int32_t v = 0;
                if (i < ao) {
                    const int64_t q = owner(s_apre, i);
                    v = __ldcg(a.act + vbase(q) + (i - s_apre[q]));
                }
                __syncthreads();
                if (i < ao) a.act[i] = v;
                __syncthreads();
            }
            for (int64_t c = 0; c < eo; c += kRT) {
                const int64_t i = c + tid;
                uint64_t v = 0;
                if (i < eo) {
                    const int64_t q = owner(s_epre, i);
                    v = __ldcg(a.e + ebase(q) + (i - s_epre[q]));
                }
                __syncthreads();
                if (i < eo) a.e[i] = v;
                __syncthreads();
            }
            if (tid == 0) {
                a.alen[0] = (int32_t)ao;
                a.seg[0] = eo;
            }
            Pe = 1;
            __syncthreads();
        }
    }
    if (p == 0 && tid == 0) {
        a.cnt[C_V] = V;
        a.cnt[C_E] = E;
        a.cnt[C_NMST] = nmst;
        a.cnt[C_ROUNDS] = round;
        a.cnt[C_ROUNDS_ALL] += round;
        a.cnt[C_DONE] = done;
        if (done == 2 || done == 3) set_err(a.err, DEV_CHASE_LIMIT);
    }
}

// Points every original vertex at its root (the next phase's builds and the
// final labels read roots directly).
// With next_best set, it also readies the next weight phase of a queued MST:
// every selection slot empty, the build cursor and the round kernel's barrier
// at zero (the round kernel that precedes it has ended).
__global__ void k_flatten(int32_t *parent, int64_t V0, int *err, unsigned long long *next_best,
                          int64_t *cnt, GridBarrier *bar)
{
    if (next_best && blockIdx.x == 0 && threadIdx.x == 0) {
        cnt[C_CURSOR] = 0;
        bar->count = 0;
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * 4;
    for (int64_t xb = (int64_t)blockIdx.x * blockDim.x * 4 + threadIdx.x; xb < V0; xb += stride) {
        int32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t v = xb + (int64_t)i * blockDim.x;
            r[i] = v < V0 ? (int32_t)v : -1;
            if (next_best && v < V0) next_best[v] = kNone;
        }
        find_batch<4>(parent, r, err);
    }
}

// Engine state for a new run: no error, the round state, weight histogram
// and barrier at zero, every selection slot empty, and every vertex its own
// root (parent) and its own successor (color; a root that no round visits
// keeps color[s] == s).
__global__ void k_engine_reset(int *err, int64_t *cnt, unsigned long long *hist, GridBarrier *bar,
                               unsigned long long *best, int32_t *parent, int32_t *color,
                               int64_t n)
{
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            *err = 0;
            bar->count = 0;
        }
        for (int i = threadIdx.x; i < C_COUNT; i += blockDim.x) cnt[i] = 0;
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0ull;
    }
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        best[i] = kNone;
        parent[i] = (int32_t)i;
        color[i] = (int32_t)i;
    }
}

// Sizes of a round-kernel run started from the host, and its barrier at zero.
__global__ void k_set_sizes(int64_t *cnt, int64_t V, int64_t E, GridBarrier *bar)
{
    if (threadIdx.x == 0) {
        cnt[C_V] = V;
        cnt[C_E] = E;
        bar->count = 0;
    }
}

// Component numbers = rank of the root id among all roots: the reference's
// numbering (its per-round renumbering keeps root order).  flag/pos: V0
// int32 scratch; labels may alias parent.
__global__ void k_root_flags(const int32_t *parent, int64_t V0, int32_t *flag)
{
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < V0;
         x += (int64_t)gridDim.x * blockDim.x)
        flag[x] = parent[x] == (int32_t)x;
}

__global__ void k_rank_roots(const int32_t *parent, const int32_t *pos, int64_t V0,
                             int32_t *labels)
{
    for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < V0;
         x += (int64_t)gridDim.x * blockDim.x)
        labels[x] = pos[parent[x]];
}

// Round-kernel launch shape.  Test hooks: g_round_cap lowers the rounds a
// phase may run (reaching it is an error, as for the built-in cap), and
// g_round_team forces the number of participants (1 = one block).
static int g_round_cap = 0;
static int g_round_team = 0;
// A host thread may cap the participants of the round kernels it launches
// (set_thread_round_team): the batched path runs many small instances side
// by side, each best served by a single block instead of the whole GPU.
static thread_local int t_round_team_cap = 0;

template <int MODE>
static int round_team_max(int *out)
{
    static int cached = 0;
    if (!cached) {
        int dev = 0, sms = 0, per_sm = 0;
        EACB_CUDA(cudaGetDevice(&dev));
        EACB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        EACB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rounds<MODE, true>,
                                                                kRT, 0));
        int m = sms * (per_sm > 2 ? 2 : per_sm);
        cached = m < 1 ? 1 : (m > kMaxTeam ? kMaxTeam : m);
    }
    *out = cached;
    return EACB_OK;
}

// Participants for a graph of V0 vertices and about E edge words: one per
// 4096 vertices or 16K edge words, up to the resident maximum.
template <int MODE>
static int round_team(int64_t V0, int64_t E, int kind, int *team)
{
    int mx = 1;
    int s = round_team_max<MODE>(&mx);
    if (s) return s;
    const int64_t work = std::max((V0 + 4095) / 4096, (E + 16383) / 16384);
    int t = g_round_team > 0 ? g_round_team : (int)std::min<int64_t>(work, mx);
    const int64_t cap = g_round_team > 0 ? 0 : tune_get(TUNE_ROUND_TEAM, kind, V0, 0);
    if (cap > 0) t = (int)std::min<int64_t>(t, cap);
    if (t_round_team_cap > 0) t = std::min(t, t_round_team_cap);
    *team = std::max(1, std::min(t, mx));
    return EACB_OK;
}

// MST selection key -> index of its entry in row min(u,v) of a symmetric CSR
// (the smallest index with the key's destination and weight).  A key whose
// build recorded the entry's offset in that row (the word's spare bits) is
// one load of the row start.  Otherwise one thread per key scans the row,
// with the loads of a step in flight together: graph rows are short, and a
// thread per key keeps every key's dependent loads (key -> row extent ->
// entries) overlapping with all the others.
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
        const uint64_t off = pk.sel_off(s);
        const int64_t f = first[a];
        if (off != pk.omask) {
            // the build recorded where the entry sits in row a: the first
            // such entry, since a parallel entry of the row with a smaller
            // offset has the smaller selection key
            out[q] = (int32_t)(f + (int64_t)off);
            continue;
        }
        const int64_t d = deg[a];
        int64_t found = -1;
        // the first 16 entries in one batch of loads (most rows of a k-NN
        // graph end there), the rest 8 at a time
        for (int64_t e0 = f; e0 < f + d && found < 0; e0 += (e0 == f ? 16 : 8)) {
            int32_t v[16];
            uint32_t ww[16];
            const int span = e0 == f ? 16 : 8;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int64_t e = e0 + i;
                const bool in = i < span && e < f + d;
                v[i] = in ? dest[e] : -1;
                ww[i] = in ? wword(weight[e]) : 0u;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i)
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
    int64_t *cnt;             // round state (C_*)
    uint64_t *ea;             // edge words: phase builds write them, the rounds compact them
    int32_t *label;           // union-find parent; after each phase every vertex's root
    unsigned long long *best;
    int32_t *color, *flag, *pos, *act;
    uint64_t *mst;
    unsigned long long *hist; // 256 weight buckets
    int *lohi;                // the device phase plan (k_phase_plan)
    int32_t *giant;           // root whose rows a later phase skips (k_pick_giant)
    int32_t *part;            // per-participant counts of the round kernel
    int32_t *alen;            // per-participant active roots
    int64_t *seg;             // per-participant surviving edge words
    int64_t *trace;
    GridBarrier *bar;
    ScanScratch scan;
    int32_t V0;
    int64_t Emax;
    int kind = 0;             // 0 graph MST/CC, 1 EAC final clustering (tuning shape)

    static Engine carve(Carver &c, int32_t V0, int64_t Emax)
    {
        Engine g;
        g.err = c.take<int>(1);
        g.cnt = c.take<int64_t>(C_COUNT);
        g.hist = c.take<unsigned long long>(256);
        g.lohi = c.take<int>(2 * kPhaseSlots);
        g.giant = c.take<int32_t>(1);
        g.bar = c.take<GridBarrier>(1);
        g.seg = c.take<int64_t>(kMaxTeam);
        g.trace = c.take<int64_t>(3 * kMaxRounds);
        g.part = c.take<int32_t>(2 * kMaxTeam);
        g.alen = c.take<int32_t>(kMaxTeam);
        g.V0 = V0;
        // the edge words (compacted in place by the rounds); they also hold
        // the two directions of a forest (at most 2 V0 words)
        g.Emax = std::max<int64_t>(Emax, 2 * (int64_t)V0);
        g.ea = c.take<uint64_t>(g.Emax);
        g.label = c.take<int32_t>(V0);
        g.best = c.take<unsigned long long>(V0);
        g.color = c.take<int32_t>(V0);
        g.flag = c.take<int32_t>(V0);
        g.pos = c.take<int32_t>(V0);
        g.act = c.take<int32_t>(V0);
        g.mst = c.take<uint64_t>(V0);
        g.scan = ScanScratch::carve(c, g.Emax, g.err);
        return g;
    }

    int read_counts(cudaStream_t st, int64_t h[C_COUNT])
    {
        int e = 0;
        EACB_CUDA(cudaMemcpyAsync(h, cnt, C_COUNT * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaStreamSynchronize(st));
        return dev_err_to_status(e);
    }

    int read_hist(cudaStream_t st, unsigned long long h[256])
    {
        EACB_CUDA(cudaMemcpyAsync(h, hist, 256 * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, st));
        EACB_CUDA(cudaStreamSynchronize(st));
        return EACB_OK;
    }

    int reset(cudaStream_t st)
    {
        k_engine_reset<<<grid_for(V0, 256), 256, 0, st>>>(err, cnt, hist, bar, best, label, color,
                                                         V0);
        EACB_CHECK_LAUNCH();
        return EACB_OK;
    }

    // Runs the rounds of one phase: input edges in ea (cnt[C_E] of them, or
    // cnt[C_CURSOR] with from_cursor), supervertices [0, cnt[C_V]) (V0 with
    // first_phase) with their selection in best; the barrier is at zero (the
    // reset, k_set_sizes or the previous phase's k_flatten cleared it).  One
    // launch; with profiling on it is timed, and its algorithmic bytes come
    // from the per-round sizes the kernel records.  With next_phase set, the
    // flattening after it readies the next queued phase.
    template <int MODE>
    int rounds(Pack pk, cudaStream_t st, int64_t e_hint, int from_cursor = 0,
               int first_phase = 0, bool next_phase = false)
    {
        int team = 1;
        int s = round_team<MODE>(V0, e_hint, kind, &team);
        if (s) return s;
        RoundArgs a;
        a.pk = pk;
        a.V0 = V0;
        a.e = ea;
        a.parent = label;
        a.best = best;
        a.color = color;
        a.act = act;
        a.mst = mst;
        a.part = part;
        a.alen = alen;
        a.seg = seg;
        a.cnt = cnt;
        a.trace = trace;
        a.bar = bar;
        a.err = err;
        a.max_rounds = g_round_cap > 0 ? std::min(g_round_cap, kMaxRounds) : kMaxRounds;
        a.from_cursor = from_cursor;
        a.first_phase = first_phase;
        ProfScope ps(PROF_ROUNDS, st);
        if (team == 1) {
            k_rounds<MODE, false><<<1, kRT, 0, st>>>(a);
            EACB_CHECK_LAUNCH();
        } else {
            void *args[] = {(void *)&a};
            EACB_CUDA(cudaLaunchCooperativeKernel((const void *)k_rounds<MODE, true>, dim3(team),
                                                  dim3(kRT), args, 0, st));
            count_launch();
        }
        if (ps.on) {
            // per round: each edge word read and (if it survives) written
            // back, 8 B each, with its two endpoints' parents (8 B); per
            // active root its list entry, selection slot, successor and
            // parent (20 B)
            int64_t h[C_COUNT], tr[3 * kMaxRounds];
            EACB_CUDA(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaMemcpyAsync(tr, trace, sizeof(tr), cudaMemcpyDeviceToHost, st));
            EACB_CUDA(cudaStreamSynchronize(st));
            double bytes = 0.0;
            const int64_t nr = std::min<int64_t>(h[C_ROUNDS], kMaxRounds);
            for (int64_t r = 0; r < nr; ++r) {
                const double En = r + 1 < nr ? (double)tr[3 * r + 4] : (double)h[C_E];
                bytes += 16.0 * (double)tr[3 * r + 1] + 8.0 * En + 20.0 * (double)tr[3 * r + 2];
            }
            ps.done(bytes);
        }
        // every vertex to its root, for the next phase's builds and the labels
        k_flatten<<<grid_for(V0, 256 * 4, 148 * 8), 256, 0, st>>>(
            label, V0, err, next_phase ? best : nullptr, cnt, bar);
        EACB_CHECK_LAUNCH();
        return EACB_OK;
    }

    // MST by weight phases (see k_phase_csr), all queued back to back with no
    // host read in between, right after reset(): build(ph) appends a phase's
    // edges to ea through cnt[C_CURSOR] with their selection in best; the
    // round kernel takes its edge count from the cursor, and the flattening
    // after it clears the slots, the cursor and the barrier for the next
    // phase.  One read at the end gives the forest size, the component count
    // and any error.
    template <typename Build>
    int run_phased(Pack pk, const std::vector<Phase> &plan, Build build, cudaStream_t st,
                   int64_t *n_mst_out, int64_t *n_comp_out)
    {
        for (size_t q = 0; q < plan.size(); ++q) {
            Phase ph = plan[q];
            ph.ident = q == 0;                 // no round has merged anything yet
            int s = build(ph);
            if (s) return s;
            if ((s = rounds<SEL_MST>(pk, st, Emax, 1, q == 0 ? 1 : 0, q + 1 < plan.size())))
                return s;
        }
        int64_t h[C_COUNT];
        int s = read_counts(st, h);
        if (s) return s;
        *n_mst_out = h[C_NMST];
        *n_comp_out = plan.empty() ? V0 : h[C_V];
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
        int64_t V = V0, n_mst = 0;
        size_t q = 0;
        bool merged = false;
        while (q < plan.size()) {
            Phase ph = plan[q];
            ph.ident = !merged;                // no round has merged anything yet
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
            int64_t nc = 0;
            if ((s = run<SEL_MST>(pk, Ep, V, st, &n_mst, &nc))) return s;
            merged = merged || nc < V;
            V = nc;
            ++q;
            if (V <= 1) break;
            // Few components left: the rest of the weights in one phase.
            // Each phase walks the whole matrix, and once the components are
            // few most entries join a component to itself, so the remaining
            // phases would keep few words each; a merged phase that does
            // overflow the edge array is redone in pieces like any other.
            if (q + 1 < plan.size() && V * kMergeBelow <= V0) {
                bool full = true;
                for (size_t r = q; r < plan.size(); ++r)
                    full = full && plan[r].r0 == 0 && plan[r].r1 == V0;
                if (full) {
                    const Phase rest{plan[q].lo, plan.back().hi, 0, V0, -1, 0};
                    plan.resize(q);
                    plan.push_back(rest);
                }
            }
        }
        *n_mst_out = n_mst;
        *n_comp_out = V;
        return EACB_OK;
    }

    template <int MODE, typename Src>
    int filter(const Src &src, int64_t n_in, uint64_t *out, cudaStream_t st)
    {
        if (n_in == 0) {
            EACB_CUDA(cudaMemsetAsync(&cnt[C_AUX0], 0, sizeof(int64_t), st));
            return EACB_OK;
        }
        const int64_t ntiles = (n_in + kETile - 1) / kETile;
        EACB_CUDA(cudaMemsetAsync(scan.status, 0, sizeof(uint64_t) * ntiles, st));
        EACB_CUDA(cudaMemsetAsync(scan.counter, 0, sizeof(int), st));
        k_edge_tile<MODE, Src><<<(unsigned)ntiles, kET, 0, st>>>(
            src, n_in, out, best, scan.status, scan.counter, &cnt[C_AUX0], err);
        EACB_CHECK_LAUNCH();
        return EACB_OK;
    }

    // Rounds from E0 edge words in ea (selection already in best) over
    // supervertices [0, V_start).  On return: label = component of every
    // vertex, *n_comp_out = number of components, *n_mst_total = forest
    // edges emitted since the engine's reset.
    template <int MODE>
    int run(Pack pk, int64_t E0, int64_t V_start, cudaStream_t st, int64_t *n_mst_total,
            int64_t *n_comp_out)
    {
        k_set_sizes<<<1, 32, 0, st>>>(cnt, V_start, E0, bar);
        EACB_CHECK_LAUNCH();
        int s = rounds<MODE>(pk, st, E0);
        if (s) return s;
        int64_t h[C_COUNT];
        if ((s = read_counts(st, h))) return s;
        if (h[C_DONE] != 1) return EACB_ERR_NOT_CONVERGED;
        *n_mst_total = h[C_NMST];
        *n_comp_out = h[C_V];
        return EACB_OK;
    }
};

template <typename WT>
static int csr_graph_run(int mode, const int32_t *dest, const WT *weight, int wbits,
                         const int32_t *first, const int32_t *deg, int32_t V, int64_t E,
                         int32_t *mst_out, int64_t *host_n_mst, int32_t *labels_out,
                         int64_t *host_n_comp, void *ws, size_t ws_bytes, cudaStream_t st)
{
    Pack pk;
    int s = make_pack(V, wbits, pk, mode == SEL_MST);
    if (s) return s;
    Carver c(ws, ws_bytes);
    Engine g = Engine::carve(c, V, E);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    if ((s = g.reset(st))) return s;
    int64_t h[C_COUNT];
    int64_t n_mst = 0, n_comp = 0;
    const unsigned gr = grid_for((int64_t)V * 32, 256);
    const unsigned gph = grid_for(V, kPhThreads, 148 * 4);   // phase builds: grid-stride rows
    if (mode == SEL_MST) {
        // weight phases over the bucket histogram of the entries (the reset
        // cleared it)
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
        const int p1 = (int)std::min<int64_t>(999, std::max<int64_t>(
                           1, tune_get(TUNE_MST_PHASE1, 0, V, 250)));
        k_phase_plan<<<1, 256, 0, st>>>(g.hist, g.lohi, p1);
        EACB_CHECK_LAUNCH();
        std::vector<Phase> plan;
        for (int q = 0; q < kPhaseSlots; ++q) plan.push_back(Phase{0, 0, 0, V, q});
        // a phase holds a subset of the E entries: the edge array always fits.
        // The first phase reads every row with identity labels; the later one
        // skips the rows of the giant component the first phase built
        auto build = [&](const Phase &ph) -> int {
            if (E == 0) return EACB_OK;
            if (ph.slot > 0) {
                k_pick_giant<<<1, 1024, 0, st>>>(g.label, V, g.giant);
                EACB_CHECK_LAUNCH();
            }
            ProfScope ps(PROF_PHASE, st);
            // the first phase reads every row and needs many warps to keep
            // its loads in flight; the skipping phase touches few rows
            // the kept-entry records (dynamic) on top of the static staging pass 48 KB
            EACB_CUDA(cudaFuncSetAttribute((const void *)k_phase_csr<SEL_MST, WT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kPhRecBytes));
            k_phase_csr<SEL_MST, WT><<<ph.slot == 0 ? gr : gph, kPhThreads, kPhRecBytes, st>>>(
                first, deg, dest, weight, V, E, wbits, 0, 0, g.lohi, ph.slot, ph.slot == 0 ? 1 : 0,
                ph.slot > 0 ? g.giant : nullptr, g.label, pk, g.ea,
                (unsigned long long *)&g.cnt[C_CURSOR], (unsigned long long)g.Emax, g.best,
                ph.slot == 0 ? (unsigned long long *)&g.cnt[C_SYM_LT] : nullptr, g.err);
            EACB_CHECK_LAUNCH();
            // compulsory reads: row extents and labels (12 B per row), dest and
            // weight (4 + sizeof(WT) B per entry); the written words follow
            ps.done(12.0 * V + (4.0 + sizeof(WT)) * (double)E);
            return EACB_OK;
        };
        if ((s = g.run_phased(pk, plan, build, st, &n_mst, &n_comp))) return s;
    } else {
        // every entry with identity labels: one word per undirected edge and
        // each vertex's first selection (the reference's round one)
        if (E > 0) {
            EACB_CUDA(cudaFuncSetAttribute((const void *)k_phase_csr<SEL_CC, WT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kPhRecBytes));
            k_phase_csr<SEL_CC, WT><<<gr, kPhThreads, kPhRecBytes, st>>>(
                first, deg, dest, weight, V, E, wbits, -1, 255, nullptr, 0, 1, nullptr, g.label, pk,
                g.ea, (unsigned long long *)&g.cnt[C_CURSOR], (unsigned long long)g.Emax, g.best,
                (unsigned long long *)&g.cnt[C_SYM_LT], g.err);
            EACB_CHECK_LAUNCH();
        }
        if ((s = g.read_counts(st, h))) return s;
        if (h[C_SYM_LT] != h[C_SYM_GT]) return EACB_ERR_BAD_INPUT;   // not symmetric
        if ((s = g.run<SEL_CC>(pk, h[C_CURSOR], V, st, &n_mst, &n_comp))) return s;
    }
    if (mode == SEL_MST) {
        if (n_mst > 0) {
            k_key2eid<WT><<<grid_for(n_mst, 256), 256, 0, st>>>(g.mst, n_mst, first, deg, dest,
                                                                  weight, pk, mst_out, g.err);
            EACB_CHECK_LAUNCH();
        }
        if ((s = g.read_counts(st, h))) return s;
        if (h[C_SYM_LT] != h[C_SYM_GT]) return EACB_ERR_BAD_INPUT;   // not symmetric
        *host_n_mst = n_mst;
    } else {
        // the reference's component numbers: ranks of the root ids
        const unsigned gv = grid_for(V, 256);
        k_root_flags<<<gv, 256, 0, st>>>(g.label, V, g.flag);
        EACB_CHECK_LAUNCH();
        if ((s = scan_launch<int32_t, int32_t>(g.flag, g.pos, V, 0, &g.cnt[C_AUX1], g.scan, st)))
            return s;
        k_rank_roots<<<gv, 256, 0, st>>>(g.label, g.pos, V, labels_out);
        EACB_CHECK_LAUNCH();
        if ((s = g.read_counts(st, h))) return s;
        if (h[C_AUX1] != n_comp) return EACB_ERR_INTERNAL;
        *host_n_comp = n_comp;
    }
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

// Test hooks of the Boruvka round kernel (see k_rounds): the rounds a phase
// may run (0 = the built-in cap; reaching a lower cap is reported as
// EACB_ERR_NOT_CONVERGED, like the built-in one) and its participants
// (0 = automatic, 1 = one block, more = that many cooperative blocks, at
// most the resident maximum).  Process-wide; set them only between calls.
namespace eacb {
void set_thread_round_team(int blocks) { t_round_team_cap = blocks > 0 ? blocks : 0; }
}  // namespace eacb

extern "C" void eacb_debug_set_round_cap(int rounds) { g_round_cap = rounds > 0 ? rounds : 0; }
extern "C" void eacb_debug_set_round_team(int blocks) { g_round_team = blocks > 0 ? blocks : 0; }

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

// Matrices of up to this many entries get an edge word for every entry, so
// no phase can overflow and all phases are queued with no host read between
// them (the many small matrices of batched EAC); larger ones keep the
// bounded edge array below and may redo an overflowing phase in pieces.
constexpr int64_t kFinalQueuedEntries = (int64_t)1 << 26;

// Edge words of the final clustering (one per kept entry): every entry when
// the matrix is small, else 256 words per point (at least 2^20): room for
// the usual output of a phase, not its worst case (a phase that overflows is
// redone in pieces), so a matrix of thousands of entries per row does not
// need an edge array of its own size.
static int64_t final_edge_cap(int32_t n, int64_t nnz)
{
    const int64_t all = nnz > (int64_t)n ? nnz : (int64_t)n;
    if (all <= kFinalQueuedEntries) return all;       // nothing can overflow
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
    g.kind = 1;
    if ((s = g.reset(st))) return s;
    // 1. minimum spanning forest of the dissimilarity graph, by weight phases
    //    (the reset cleared the histogram)
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
            indptr, indices, diassoc, n, nnz, ph.lo, ph.hi, dense(ph), ph.ident, ph.r0, ph.r1,
            g.label, pk, g.ea,
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
        return split_final_phase(ph, kh, g.Emax, indptr, n, hip, st, out);
    };
    if (g.Emax >= nnz) {
        if ((s = g.run_phased(pk, phases, build, st, &n_mst, &n_comp))) return s;
    } else {
        if ((s = g.run_phased_retry(pk, phases, build, split, st, &n_mst, &n_comp))) return s;
    }
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
    // 3. components of the forest without the cut edges: the kept forest
    //    keys go from mst into ea, then the rounds
    if ((s = g.reset(st))) return s;
    SrcForest sf{g.mst, n_mst, hp.wmax, pk};
    if ((s = g.filter<SEL_CC>(sf, n_mst, g.ea, st))) return s;
    int64_t h[C_COUNT];
    if ((s = g.read_counts(st, h))) return s;
    int64_t nm2 = 0, nc2 = 0;
    if ((s = g.run<SEL_CC>(pk, h[C_AUX0], n, st, &nm2, &nc2))) return s;
    // 4. number components by their smallest member
    EACB_CUDA(cudaMemsetAsync(cmin, 0x7f, sizeof(int32_t) * n, st));
    const unsigned gn = grid_for(n, 256);
    k_comp_min<<<gn, 256, 0, st>>>(g.label, n, cmin);
    EACB_CHECK_LAUNCH();
    k_first_flag<<<gn, 256, 0, st>>>(g.label, cmin, n, g.flag);
    EACB_CHECK_LAUNCH();
    if ((s = scan_launch<int32_t, int32_t>(g.flag, g.pos, n, 0, &g.cnt[C_AUX1], g.scan, st)))
        return s;
    k_canon<<<gn, 256, 0, st>>>(g.label, cmin, g.pos, n, labels);
    EACB_CHECK_LAUNCH();
    if ((s = g.read_counts(st, h))) return s;
    *host_n_fclusts = h[C_AUX1];
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
