// Sparse co-association matrix (condensed CSR of co-occurrence counts).
//
// Reference: MyML/MyML/EAC/sparse.py -- EAC_CSR.update_ensemble :154-166,
// update_cluster_fp_condensed :446-465 (first partition, no capacity check),
// update_cluster_sorted_surgical_condensed :957-1040 (sorted rows, capacity
// per row, later associations discarded), _condense :212-226.
//
// Semantics reproduced exactly: row i of the condensed matrix holds the
// columns j > i that share a cluster with i in some partition, with the count
// of such partitions.  A row keeps at most cap(i) = cap_indptr[i+1] -
// cap_indptr[i] columns: the first cap(i) distinct columns in the order
// (rank of the first partition where the pair co-occurs in processing order,
// then j); counts of discarded columns are summed into nnz_discarded.  The
// processing order is the partition with the fewest non-empty clusters
// first (lowest index on ties), then the others by index.
//
// B200 design (not the reference's insertion sort into pre-allocated rows):
//  1. per partition, cluster member lists sorted by point index are built by
//     a stable counting sort (tile histograms, one device scan over
//     (partition, cluster, tile), warp-level match_any placement); a point's
//     "tail" in a partition is then the contiguous run of its cluster's
//     member list after its own position.
//  2. pass 1, one CTA per row (persistent, dynamic row queue): the row's P
//     tails are streamed in column chunks into a shared-memory bitmap
//     (atomicOr); popcounts give the exact number of distinct columns, hence
//     the kept count min(D_i, cap(i)) and the row offsets (device scan).
//  3. pass 2, same streaming into shared-memory byte counters (one byte per
//     column, four packed per word), then a block-wide compaction of the
//     non-zero counters writes the row in column order straight into the
//     final CSR.  Rows whose distinct count exceeds their capacity are
//     redone by a rank-aware kernel: a column's rank (first partition in
//     processing order that associates it) is an atomicMin per visit, and
//     the keep rule is applied from the rank histogram.
//  4. the pair tiles (k_nbr, k_pairs): rows grouped by their
//     cluster in the partition with the most clusters are counted by
//     comparing label vectors over the group's neighbourhood instead of
//     streaming tails, when that is cheaper; the count pass keeps each
//     tile's pair counts for the fill.  Steps 2 and 3 then take only the
//     rows outside those groups (and every row over its capacity).
#include "eacb_common.cuh"
#include "scan_impl.cuh"
#include "members.cuh"

#include <cuda_fp16.h>

#include <algorithm>

namespace eacb {

constexpr int kMaxK = 8192;            // largest cluster id + 1 supported
constexpr int kRowThreads = 512;
constexpr int kBitmapBytes = 96 * 1024;        // pass 1: 786,432 columns per chunk
// pass 2 runs two 512-thread CTAs per SM, each with 96 KB of byte counters
// and a "touched" flag byte per 16 counters; the compaction reads only
// flagged counter vectors and clears what it reads, so a chunk costs no pass
// over its mostly-zero counters, and one CTA's compaction and barrier waits
// overlap the other's walk
constexpr int kFillThreads = 512;
constexpr int kFillVecs = 12;                  // counter vectors (16 columns) per thread
constexpr int kCountBytes = kFillThreads * kFillVecs * 16;   // 98,304 columns per chunk
constexpr int kFillSmem = kCountBytes + kCountBytes / 16;
constexpr int kCapCols = 16 * 1024;            // capped rows: columns per chunk
constexpr int kCapSmem = kCapCols * 5;         // byte counters + 32-bit ranks
constexpr int kMaxP = 255;
// work queues: 0 count rows, 1 fill rows, 2 capped rows, 3 row order,
// 4 neighbourhoods, 5 pair tiles (count), 6 pair tiles (fill)
constexpr int kQueues = 8;

// pair tiles: 128 rows x 128 columns, labels as FP16 pairs (exact below 2048)
constexpr int kPT = 128;
constexpr int kPairThreads = 256;
constexpr int kDenseMaxK = 2048;
constexpr int kNbrThreads = 512;
constexpr int kNbrBytes = 64 * 1024;           // neighbourhood chunk: 524,288 columns
constexpr int kMaxGroupLists = 4096;           // (partition, cluster) lists per group
// member positions fit 32 bits (P n < 2^31): cursors, ends and keys are
// int32, so two CTAs fit an SM
constexpr int kNbrSmem = kNbrBytes + kMaxGroupLists * (4 + 4 + 4);
constexpr int64_t kDenseRatioDefault = 16;
// the count pass keeps each tile's pair counts (one byte per pair, 16 KB per
// 128 x 128 tile) for the fill, in up to this many bytes per point (and at
// most kPairBytesMax); a tile that finds no room is recomputed by the fill
constexpr int64_t kPairBytesPerPoint = 8192;
constexpr int64_t kPairBytesMax = (int64_t)32 << 30;

// half2 words per point in the FP16 label copy: P rounded up to 8 partitions
__host__ __device__ constexpr int32_t pair_words(int32_t P) { return ((P + 7) / 8) * 4; }

struct CoWS {
    int *err;
    int32_t *members;     // P*n, member lists of every partition, back to back
    int32_t *mypos;       // P*n, global position of point i in its member list (-1: none)
    int32_t *cnt;         // P*K*ntiles tile counts
    int64_t *S;           // exclusive scan of cnt (+ total)
    int32_t *ncl;         // P non-empty clusters
    int32_t *order;       // P processing order
    int32_t *rowcnt;      // n kept columns per row
    int32_t *rowflag;     // n: bit 0 = distinct columns exceed the capacity,
                          //    bit 1 = the row's group takes the pair tiles
    int32_t *rowperm;     // n: the order the row kernels take rows in
    int *queue;           // work-queue counters
    unsigned long long *disc;   // discarded counts
    int *maxcnt;          // largest kept count
    int *prow;            // the partition whose clusters order the rows
    uint32_t *lt;         // n x Q: FP16 label pairs, point-major (pair tiles)
    int64_t *grp_off;     // K: a group's neighbourhood in nbr
    int32_t *grp_len;     // K: its length
    int32_t *grp_tiles;   // K (+1): pair-tile row blocks of a group (0: streamed)
    int64_t *grp_item0;   // K + 1: exclusive scan of grp_tiles
    int32_t *nbr;         // neighbourhoods, back to back
    unsigned long long *nbr_used;
    int32_t *rowlist;     // n: rows a streaming kernel takes
    int *rowlist_n;
    uint8_t *pbuf;        // pair counts of the count pass's tiles, read by the fill
    unsigned long long *pused;
    int64_t *islot;       // per pair-tile item: its place in pbuf (-1: none)
    ScanScratch scan;
    int64_t ntiles, nbr_cap, pcap, nitems_max;
    int32_t Q;            // half2 words per point in lt
    static CoWS carve(Carver &c, int32_t n, int32_t P, int32_t K)
    {
        CoWS w;
        w.err = c.take<int>(1);
        w.ntiles = ((int64_t)n + kMLTile - 1) / kMLTile;
        w.Q = pair_words(P);
        w.nbr_cap = 16 * (int64_t)n + 65536;
        w.pcap = std::min<int64_t>(kPairBytesPerPoint * (int64_t)n + (1 << 20), kPairBytesMax);
        w.nitems_max = (int64_t)n / kPT + K + 1;
        const int64_t pn = (int64_t)P * n;
        const int64_t m = (int64_t)P * K * w.ntiles;
        w.members = c.take<int32_t>(pn > 0 ? pn : 1);
        w.mypos = c.take<int32_t>(pn > 0 ? pn : 1);
        w.cnt = c.take<int32_t>(m + 1);
        w.S = c.take<int64_t>(m + 1);
        w.ncl = c.take<int32_t>(P > 0 ? P : 1);
        w.order = c.take<int32_t>(P > 0 ? P : 1);
        w.rowcnt = c.take<int32_t>(n);
        w.rowflag = c.take<int32_t>(n);
        w.rowperm = c.take<int32_t>(n);
        w.queue = c.take<int>(kQueues);
        w.disc = c.take<unsigned long long>(1);
        w.maxcnt = c.take<int>(1);
        w.prow = c.take<int>(1);
        w.lt = c.take<uint32_t>((size_t)n * w.Q);
        w.grp_off = c.take<int64_t>(K);
        w.grp_len = c.take<int32_t>(K);
        w.grp_tiles = c.take<int32_t>((size_t)K + 1);
        w.grp_item0 = c.take<int64_t>((size_t)K + 1);
        w.nbr = c.take<int32_t>(w.nbr_cap);
        w.nbr_used = c.take<unsigned long long>(1);
        w.rowlist = c.take<int32_t>(n);
        w.rowlist_n = c.take<int>(1);
        w.pbuf = c.take<uint8_t>(w.pcap);
        w.pused = c.take<unsigned long long>(1);
        w.islot = c.take<int64_t>(w.nitems_max);
        w.scan = ScanScratch::carve(c, m + 1 > n ? m + 1 : n, w.err);
        return w;
    }
};

// ------------------------------------------------------------- row tails --
struct TailCtx {
    const int32_t *labels;
    const int32_t *members;
    const int32_t *mypos;
    const int64_t *S;
    int32_t n, P, K;
    int64_t ntiles;
    // [start, end) of point i's tail in partition p (start == end: none)
    __device__ void tail(int32_t i, int32_t p, int64_t &s, int64_t &e) const
    {
        int32_t mp = mypos[(int64_t)p * n + i];
        if (mp < 0) { s = e = 0; return; }
        int32_t c = labels[(int64_t)p * n + i];
        s = (int64_t)mp + 1;
        e = S[((int64_t)p * K + c + 1) * ntiles];
    }
};

__device__ __forceinline__ int next_row(int *queue, int *s_row)
{
    if (threadIdx.x == 0) *s_row = atomicAdd(queue, 1);
    __syncthreads();
    int r = *s_row;
    __syncthreads();
    return r;
}

template <int THREADS>
__device__ __forceinline__ int64_t block_sum(int64_t v)
{
    int64_t tot;
    block_excl_sum_shfl<THREADS>(v, tot);
    return tot;
}

// Stream the tails of all partitions into [j0, jl): calls op(j, p) per
// element j of tail p, and advances the cursors ts[p] past what it consumed.
// A warp walks one tail at a time, kStreamU x 32 members per step with all
// loads issued before any is used (the walk is latency-bound: a tail
// averages a few hundred members); a tail is sorted, so the members below jl
// are a prefix of the step.
constexpr int kStreamU = 8;
// Warps take tails dynamically (*next, zeroed by the caller before the
// block's barrier), so warps that drew short tails take more of them.
template <typename IT, typename Op>
__device__ __forceinline__ void stream_chunk(const int32_t *members, IT *ts, const IT *te,
                                             int32_t P, int32_t jl, int *next, Op op)
{
    const int lane = threadIdx.x & 31;
    for (;;) {
        int p = 0;
        if (lane == 0) p = atomicAdd(next, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= P) break;
        int64_t cur = ts[p];
        const int64_t end = te[p];
        while (cur < end) {
            // 32-bit offsets from the step's base keep the per-member work to
            // a compare, a load and the op; the count taken is one reduction
            const int32_t *base = members + cur + lane;
            const int64_t left = end - cur;
            const int rem = left < kStreamU * 32 ? (int)left : kStreamU * 32;
            int32_t j[kStreamU];
#pragma unroll
            for (int u = 0; u < kStreamU; ++u)
                j[u] = u * 32 + lane < rem ? __ldg(base + u * 32) : 0x7fffffff;
            int mine = 0;
#pragma unroll
            for (int u = 0; u < kStreamU; ++u) {
                const bool ok = j[u] < jl;
                if (ok) op(j[u], p);
                mine += ok;
            }
            const int taken = __reduce_add_sync(0xffffffffu, mine);
            cur += taken;
            if (taken != kStreamU * 32) break;
        }
        if (lane == 0) ts[p] = (IT)cur;
    }
}

// ---------------------------------------------------------------- pass 1 --
__global__ void __launch_bounds__(kRowThreads)
k_rows_count(TailCtx tc, const int32_t *order, const int32_t *rows, const int *nrows,
             const int64_t *cap_indptr, int32_t *rowcnt, int32_t *rowflag, int *queue, int *err)
{
    extern __shared__ uint32_t bm[];
    __shared__ int64_t ts[kMaxP], te[kMaxP];
    __shared__ int s_row, s_next;
    const int32_t n = tc.n, P = tc.P;
    const int nr = *nrows;
    constexpr int32_t kCols = kBitmapBytes * 8;
    while (true) {
        const int qi = next_row(queue, &s_row);
        if (qi >= nr) break;
        const int i = rows[qi];
        const int64_t cap = cap_indptr[i + 1] - cap_indptr[i];
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            int64_t s, e;
            tc.tail(i, p, s, e);
            ts[p] = s;
            te[p] = e;
            if (p == order[0] && e - s > cap) set_err(err, DEV_FIRST_OVERFLOW);
        }
        __syncthreads();
        int64_t D = 0;
        for (int64_t j0 = (int64_t)i + 1; j0 < n; j0 += kCols) {
            const int32_t jl = (int32_t)((j0 + kCols < n) ? j0 + kCols : n);
            const int nvec = (int)((jl - j0 + 127) >> 7);      // 128 columns per vector
            uint4 *b4 = reinterpret_cast<uint4 *>(bm);
            for (int w = threadIdx.x; w < nvec; w += blockDim.x) b4[w] = make_uint4(0u, 0u, 0u, 0u);
            if (threadIdx.x == 0) s_next = 0;
            __syncthreads();
            const int32_t jb = (int32_t)j0;
            stream_chunk(tc.members, ts, te, P, jl, &s_next, [&](int32_t j, int) {
                const int32_t o = j - jb;
                atomicOr(&bm[o >> 5], 1u << (o & 31));
            });
            __syncthreads();
            int64_t c = 0;
            for (int w = threadIdx.x; w < nvec; w += blockDim.x) {
                const uint4 x = b4[w];
                c += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
            }
            D += block_sum<kRowThreads>(c);
        }
        if (threadIdx.x == 0) {
            rowcnt[i] = (int32_t)(D < cap ? D : cap);
            rowflag[i] = D > cap;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- pass 2 --
// Block-wide ordered compaction of a chunk's non-zero byte counters.  Thread
// t owns counter vectors [kFillVecs t, kFillVecs (t + 1)) (16 columns each)
// and their flag bytes (kFillVecs / 4 words); it counts the kept bytes of its
// flagged vectors with per-byte compare masks, places them after a block
// scan, writes them in column order and clears the vectors and flags.
__device__ __forceinline__ int64_t emit_flagged(uint32_t *ctr32, uint32_t *flag32, int32_t jb,
                                                int32_t *indices, uint8_t *data, int64_t out0,
                                                int &maxc)
{
    static_assert(kFillVecs % 4 == 0, "a thread's flags are whole words");
    uint32_t *fw = flag32 + threadIdx.x * (kFillVecs / 4);
    uint4 *cv = reinterpret_cast<uint4 *>(ctr32) + threadIdx.x * kFillVecs;
    uint32_t fm = 0;                                   // bit q: vector q flagged
#pragma unroll
    for (int k = 0; k < kFillVecs / 4; ++k) {
        const uint32_t m = __vcmpne4(fw[k], 0u);
        fm |= (((m >> 7) & 1u) | ((m >> 14) & 2u) | ((m >> 21) & 4u) | ((m >> 28) & 8u)) << (4 * k);
    }
    int mine = 0;
    for (uint32_t b = fm; b; b &= b - 1u) {
        const uint4 x = cv[__ffs(b) - 1];
        mine += (__popc(__vcmpne4(x.x, 0u)) + __popc(__vcmpne4(x.y, 0u)) +
                 __popc(__vcmpne4(x.z, 0u)) + __popc(__vcmpne4(x.w, 0u))) >> 3;
    }
    int64_t tot;
    int64_t at = out0 + block_excl_sum_shfl<kFillThreads>(mine, tot);
    for (uint32_t b = fm; b; b &= b - 1u) {
        const int v = __ffs(b) - 1;
        const uint4 x = cv[v];
        cv[v] = make_uint4(0u, 0u, 0u, 0u);
        const uint32_t w4[4] = {x.x, x.y, x.z, x.w};
        const int32_t c0 = jb + (int32_t)(threadIdx.x * kFillVecs + v) * 16;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t m = __vcmpne4(w4[q], 0u);       // 0xff in each non-zero byte
            while (m) {
                const int bb = (__ffs(m) - 1) >> 3;
                m &= ~(0xffu << (8 * bb));
                const uint32_t cnt = (w4[q] >> (8 * bb)) & 255u;
                indices[at] = c0 + q * 4 + bb;
                data[at] = (uint8_t)cnt;
                maxc = max(maxc, (int)cnt);
                at++;
            }
        }
    }
    if (fm) {
#pragma unroll
        for (int k = 0; k < kFillVecs / 4; ++k) fw[k] = 0u;
    }
    return tot;
}

__global__ void __launch_bounds__(kFillThreads, 2)
k_rows_fill(TailCtx tc, const int32_t *rows, const int *nrows, const int32_t *rowflag,
            const int64_t *indptr, int32_t *indices, uint8_t *data, int *queue, int *gmax, int *err)
{
    extern __shared__ uint32_t ctr32[];
    uint32_t *flag32 = ctr32 + kCountBytes / 4;
    uint8_t *flag = reinterpret_cast<uint8_t *>(flag32);
    __shared__ int64_t ts[kMaxP], te[kMaxP];
    __shared__ int s_row, s_next;
    const int32_t n = tc.n, P = tc.P;
    const int nr = *nrows;
    constexpr int32_t kCols = kCountBytes;
    int maxc = 0;
    // counters and flags start at zero; each compaction clears what it read
    for (int w = threadIdx.x; w < kFillSmem / 16; w += blockDim.x)
        reinterpret_cast<uint4 *>(ctr32)[w] = make_uint4(0u, 0u, 0u, 0u);
    while (true) {
        const int qi = next_row(queue, &s_row);
        if (qi >= nr) break;
        const int i = rows[qi];
        if (rowflag[i]) continue;            // uniform across the block
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            int64_t s, e;
            tc.tail(i, p, s, e);
            ts[p] = s;
            te[p] = e;
        }
        int64_t out = indptr[i];
        for (int64_t j0 = (int64_t)i + 1; j0 < n; j0 += kCols) {
            const int32_t jl = (int32_t)((j0 + kCols < n) ? j0 + kCols : n);
            if (threadIdx.x == 0) s_next = 0;
            __syncthreads();
            const int32_t jb = (int32_t)j0;
            stream_chunk(tc.members, ts, te, P, jl, &s_next, [&](int32_t j, int) {
                const int32_t o = j - jb;
                atomicAdd(&ctr32[o >> 2], 1u << (8 * (o & 3)));
                flag[o >> 4] = 1;
            });
            __syncthreads();
            out += emit_flagged(ctr32, flag32, jb, indices, data, out, maxc);
        }
        if (threadIdx.x == 0 && out != indptr[i + 1]) set_err(err, DEV_CAPACITY);
    }
    // block max -> global
    for (int d = 16; d >= 1; d >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, d));
    if ((threadIdx.x & 31) == 0) atomicMax(gmax, maxc);
}

// ------------------------------------------------------ rows over capacity --
// One CTA per flagged row.  The tails are indexed by processing position q
// (tail q is partition order[q]); a column's rank is the smallest q whose
// tail holds it, i.e. the first partition in processing order that
// associates it with the row -- an atomicMin per visit, so all tails stream
// at once as in the other passes.  Pass 0 histograms the ranks; the keep rule
// then needs r* (the rank at which the running distinct count reaches the
// capacity) and the quota of rank-r* columns that still fit; pass 1 keeps
// rank < r* and the first `quota` rank-r* columns in column order.  A row
// whose tail span fits one chunk keeps its pass-0 chunk for pass 1.
__global__ void __launch_bounds__(kRowThreads)
k_rows_capped(TailCtx tc, const int32_t *order, const int32_t *rows, const int *nrows,
              const int32_t *rowflag, const int64_t *cap_indptr, const int64_t *indptr,
              int32_t *indices, uint8_t *data, int *queue, int *gmax, unsigned long long *disc,
              int *err)
{
    extern __shared__ uint32_t sm[];
    uint32_t *ctr32 = sm;                      // kCapCols byte counters
    uint32_t *rank = sm + kCapCols / 4;        // kCapCols ranks (kNoRank: column untouched)
    constexpr uint32_t kNoRank = 0xffffffffu;
    __shared__ int64_t ts[kMaxP], te[kMaxP];
    __shared__ int hist[kMaxP + 1];
    __shared__ int s_row, s_rstar, s_quota, s_seen, s_next;
    const int32_t n = tc.n, P = tc.P;
    const int nr = *nrows;
    int maxc = 0;
    while (true) {
        const int qi = next_row(queue, &s_row);
        if (qi >= nr) break;
        const int i = rows[qi];
        if (!(rowflag[i] & 1)) continue;
        const int64_t cap = cap_indptr[i + 1] - cap_indptr[i];
        const bool one_chunk = (int64_t)n - ((int64_t)i + 1) <= kCapCols;
        for (int q = threadIdx.x; q <= P; q += blockDim.x) hist[q] = 0;
        int rs = 0, qt = 0;
        int64_t out = indptr[i];
        unsigned long long dsum = 0;
        for (int pass = 0; pass < 2; ++pass) {
            const bool stream = pass == 0 || !one_chunk;
            if (stream)
                for (int q = threadIdx.x; q < P; q += blockDim.x) {
                    int64_t s, e;
                    tc.tail(i, order[q], s, e);
                    ts[q] = s;
                    te[q] = e;
                }
            if (threadIdx.x == 0) s_seen = 0;
            __syncthreads();
            for (int64_t j0 = (int64_t)i + 1; j0 < n; j0 += kCapCols) {
                const int32_t jl = (int32_t)((j0 + kCapCols < n) ? j0 + kCapCols : n);
                const int width = (int)(jl - j0);
                if (stream) {
                    const int nw = (width + 15) >> 4 << 2;
                    for (int w = threadIdx.x; w < nw; w += blockDim.x) ctr32[w] = 0;
                    for (int o = threadIdx.x; o < width; o += blockDim.x) rank[o] = kNoRank;
                    if (threadIdx.x == 0) s_next = 0;
                    __syncthreads();
                    const int32_t jb = (int32_t)j0;
                    stream_chunk(tc.members, ts, te, P, jl, &s_next, [&](int32_t j, int q) {
                        const int32_t o = j - jb;
                        atomicAdd(&ctr32[o >> 2], 1u << (8 * (o & 3)));
                        atomicMin(&rank[o], (uint32_t)q);
                    });
                    __syncthreads();
                }
                if (pass == 0) {
                    for (int o = threadIdx.x; o < width; o += blockDim.x)
                        if (rank[o] != kNoRank) atomicAdd(&hist[rank[o]], 1);
                    __syncthreads();
                    continue;
                }
                // kept: rank < r*, or rank == r* among the first `quota` such
                // columns in column order; each thread owns a contiguous run
                const int per = (width + blockDim.x - 1) / blockDim.x;
                const int o0 = min(width, (int)threadIdx.x * per), o1 = min(width, o0 + per);
                int mystar = 0;
                for (int o = o0; o < o1; ++o) mystar += (rank[o] == (uint32_t)rs);
                int64_t tstar;
                const int64_t before = s_seen + block_excl_sum<kRowThreads>(mystar, tstar);
                int64_t seen = before;
                const uint8_t *c8 = (const uint8_t *)ctr32;
                int kept = 0;
                for (int o = o0; o < o1; ++o) {
                    const uint32_t r = rank[o];
                    if (r == kNoRank) continue;
                    const bool k = r < (uint32_t)rs || (r == (uint32_t)rs && seen < qt);
                    if (r == (uint32_t)rs) seen++;
                    if (k) kept++; else dsum += c8[o];
                }
                int64_t tk;
                int64_t at = out + block_excl_sum<kRowThreads>(kept, tk);
                seen = before;
                for (int o = o0; o < o1; ++o) {
                    const uint32_t r = rank[o];
                    if (r == kNoRank) continue;
                    const bool k = r < (uint32_t)rs || (r == (uint32_t)rs && seen < qt);
                    if (r == (uint32_t)rs) seen++;
                    if (k) {
                        indices[at] = (int32_t)j0 + o;
                        data[at] = c8[o];
                        maxc = max(maxc, (int)c8[o]);
                        at++;
                    }
                }
                out += tk;
                __syncthreads();
                if (threadIdx.x == 0) s_seen += (int)tstar;
                __syncthreads();
            }
            if (pass == 0) {
                if (threadIdx.x == 0) {
                    int64_t cum = 0;
                    int r = P, quota = 0;
                    for (int q = 0; q < P; ++q) {
                        if (cum + hist[q] >= cap) { r = q; quota = (int)(cap - cum); break; }
                        cum += hist[q];
                    }
                    s_rstar = r;
                    s_quota = quota;
                }
                __syncthreads();
                rs = s_rstar;
                qt = s_quota;
            }
        }
        if (threadIdx.x == 0 && out != indptr[i + 1]) set_err(err, DEV_CAPACITY);
        for (int d = 16; d >= 1; d >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, d);
        if ((threadIdx.x & 31) == 0 && dsum) atomicAdd(disc, dsum);
        __syncthreads();
    }
    for (int d = 16; d >= 1; d >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, d));
    if ((threadIdx.x & 31) == 0) atomicMax(gmax, maxc);
}

// ------------------------------------------------------------ pair tiles --
// The second way to the same rows.  The rows are grouped by their cluster in
// the row-order partition.  A group's neighbourhood N(g) is the sorted union
// of every cluster (any partition) that holds one of its rows, cut to the
// columns above the group's first row; every column that co-occurs with a
// row of the group lies in it.  The count of a pair (i, j) is then a
// comparison of the two label vectors: with the labels in FP16 (exact below
// 2048; -1 and padding are NaN, which equals nothing) two partitions take one
// HSET2 and one HADD2, and a 128 x 128 tile of pairs runs as a register-
// blocked product with no atomics and no scattered loads.  A group takes the
// tiles when their compare work (rows x |N(g)| x partition pairs) is at most
// `ratio` times the member visits the streaming kernels would spend on its
// rows; the others, and every row over its capacity, stay on the streaming
// kernels.  Both ways produce the same counts, columns and order.

__device__ __forceinline__ uint32_t label_half(int32_t l)
{
    return l >= 0 ? (uint32_t)__half_as_ushort(__int2half_rn(l)) : 0x7e00u;    // NaN
}

// lt[i*Q + w]: partitions (2w, 2w+1) of point i as a half2 (low half first)
__global__ void k_labels_f16(const int32_t *labels, int32_t n, int32_t P, int32_t Q,
                             uint32_t *lt)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint4 *dst = reinterpret_cast<uint4 *>(lt + i * Q);
        for (int v = 0; v < Q / 4; ++v) {
            uint32_t h[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int p = 8 * v + e;
                h[e] = label_half(p < P ? labels[(int64_t)p * n + i] : -1);
            }
            dst[v] = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16),
                                h[6] | (h[7] << 16));
        }
    }
}

struct GroupCtx {
    const int32_t *labels, *members, *mypos;
    const int64_t *S;
    const int *prow;
    int32_t n, P, K, Q;
    int64_t ntiles;
};

// first position in members[a, b) whose point is above lo
__device__ __forceinline__ int64_t first_above(const int32_t *members, int64_t a, int64_t b,
                                               int32_t lo)
{
    while (a < b) {
        const int64_t m = (a + b) >> 1;
        if (members[m] > lo) b = m; else a = m + 1;
    }
    return a;
}

// One CTA per group (dynamic queue over the row-order partition's clusters):
// the group's cluster lists, its rows' streaming cost, |N(g)| by chunked
// bitmaps, the choice of path and, for the pair tiles, N(g) itself.
__global__ void __launch_bounds__(kNbrThreads, 2)
k_nbr(GroupCtx gc, int64_t ratio, int32_t *nbr, int64_t nbr_cap, unsigned long long *nbr_used,
      int64_t *grp_off, int32_t *grp_len, int32_t *grp_tiles, int32_t *rowflag, int *queue)
{
    extern __shared__ __align__(16) uint8_t nsm[];
    uint32_t *bm = reinterpret_cast<uint32_t *>(nsm);
    int32_t *ts = reinterpret_cast<int32_t *>(nsm + kNbrBytes);
    int32_t *te = ts + kMaxGroupLists;
    int32_t *cl = te + kMaxGroupLists;
    __shared__ int s_g, s_nc, s_next, s_dense;
    __shared__ int64_t s_off;
    const int32_t n = gc.n, P = gc.P, K = gc.K;
    const int64_t nt = gc.ntiles;
    const int pr = *gc.prow;
    constexpr int32_t kCols = kNbrBytes * 8;
    for (;;) {
        const int g = next_row(queue, &s_g);
        if (g >= K) break;
        const int64_t gb = gc.S[((int64_t)pr * K + g) * nt];
        const int64_t size = gc.S[((int64_t)pr * K + g + 1) * nt] - gb;
        if (size == 0) {
            if (threadIdx.x == 0) grp_tiles[g] = 0;
            continue;
        }
        const int32_t *rows = gc.members + gb;
        const int32_t lo = rows[0];
        // 1. the clusters holding the group's rows, all partitions at once:
        // bit p*K + c of a P x K bitmap, kept in the chunk bitmap's memory
        // (unused until step 2; P*K <= 255 * 2048 bits fits its 64 KB); a
        // thread takes a row through every partition, loads in flight
        const int nwords = (int)(((int64_t)P * K + 31) >> 5);
        if (threadIdx.x == 0) s_nc = 0;
        for (int w = threadIdx.x; w < nwords; w += blockDim.x) bm[w] = 0u;
        __syncthreads();
        // the streaming kernels' member visits for the group, estimated from
        // at most 64 of its rows (it only chooses the path, never the result)
        const int64_t vstep = size > 64 ? size / 64 : 1;
        int64_t visits = 0;
        for (int64_t t = threadIdx.x; t < size; t += blockDim.x) {
            const int32_t i = rows[t];
            const bool sample = t % vstep == 0 && t / vstep < 64;
            const unsigned act = __activemask();
            const int lane = threadIdx.x & 31;
#pragma unroll 2
            for (int p = 0; p < P; ++p) {
                const int32_t c = gc.labels[(int64_t)p * n + i];
                const bool ok = c >= 0 && c < K;
                // rows of a group mostly share a cluster: one atomic per
                // distinct cluster of the warp
                const unsigned peers = __match_any_sync(act, ok ? c : -1 - lane);
                if (ok && lane == __ffs(peers) - 1) {
                    const int bit = p * K + c;
                    atomicOr(&bm[bit >> 5], 1u << (bit & 31));
                }
                if (ok && sample)
                    visits += gc.S[((int64_t)p * K + c + 1) * nt] -
                              gc.mypos[(int64_t)p * n + i] - 1;
            }
        }
        __syncthreads();
        for (int w = threadIdx.x; w < nwords; w += blockDim.x)
            for (uint32_t b = bm[w]; b; b &= b - 1u) {
                const int slot = atomicAdd(&s_nc, 1);
                if (slot < kMaxGroupLists) cl[slot] = w * 32 + __ffs(b) - 1;
            }
        __syncthreads();
        visits = block_sum<kNbrThreads>(visits) * vstep;
        const int nc = s_nc;
        bool dense = nc <= kMaxGroupLists;
        int64_t total = 0;
        for (int pass = 0; pass < 2 && dense; ++pass) {
            // cursors: each list from its first member above the group's first row
            for (int e = threadIdx.x; e < nc; e += blockDim.x) {
                const int64_t a = gc.S[(int64_t)cl[e] * nt], b = gc.S[((int64_t)cl[e] + 1) * nt];
                ts[e] = (int32_t)first_above(gc.members, a, b, lo);
                te[e] = (int32_t)b;
            }
            __syncthreads();
            int64_t at = 0;
            for (int64_t j0 = (int64_t)lo + 1; j0 < n; j0 += kCols) {
                const int32_t jl = (int32_t)((j0 + kCols < n) ? j0 + kCols : n);
                const int nvec = (int)((jl - j0 + 127) >> 7);
                uint4 *b4 = reinterpret_cast<uint4 *>(bm);
                for (int v = threadIdx.x; v < nvec; v += blockDim.x) b4[v] = make_uint4(0u, 0u, 0u, 0u);
                if (threadIdx.x == 0) s_next = 0;
                __syncthreads();
                const int32_t jb = (int32_t)j0;
                stream_chunk(gc.members, ts, te, nc, jl, &s_next, [&](int32_t j, int) {
                    const int32_t o = j - jb;
                    atomicOr(&bm[o >> 5], 1u << (o & 31));
                });
                __syncthreads();
                // each thread owns a run of vectors; pass 1 writes its columns in order
                const int per = (nvec + kNbrThreads - 1) / kNbrThreads;
                const int v0 = min(nvec, (int)threadIdx.x * per), v1 = min(nvec, v0 + per);
                int64_t c = 0;
                for (int v = v0; v < v1; ++v) {
                    const uint4 x = b4[v];
                    c += __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w);
                }
                int64_t tot;
                const int64_t pre = block_excl_sum_shfl<kNbrThreads>(c, tot);
                if (pass == 1) {
                    int32_t *out = nbr + s_off + at + pre;
                    for (int v = v0; v < v1; ++v)
                        for (int q = 0; q < 4; ++q)
                            for (uint32_t b = bm[4 * v + q]; b; b &= b - 1u)
                                *out++ = jb + 128 * v + 32 * q + __ffs(b) - 1;
                }
                at += tot;
                __syncthreads();
            }
            if (pass == 1) break;
            total = at;
            // the choice: the tiles' compare work against the streaming visits
            int64_t est = 0;
            const double span = (double)max(1, n - 1 - lo);
            for (int64_t t = threadIdx.x; t * kPT < size; t += blockDim.x)
                est += (int64_t)((double)kPT * gc.Q * (double)total *
                                 ((double)(n - 1 - rows[t * kPT]) / span));
            est = block_sum<kNbrThreads>(est);
            if (threadIdx.x == 0) {
                int d = ratio > 0 && est <= ratio * visits;
                if (d) {
                    const unsigned long long o = atomicAdd(nbr_used, (unsigned long long)total);
                    d = (int64_t)(o + total) <= nbr_cap;
                    s_off = (int64_t)o;
                }
                s_dense = d;
            }
            __syncthreads();
            dense = s_dense;
        }
        if (threadIdx.x == 0) {
            grp_tiles[g] = dense ? (int32_t)((size + kPT - 1) / kPT) : 0;
            grp_off[g] = dense ? s_off : 0;
            grp_len[g] = dense ? (int32_t)total : 0;
        }
        if (dense)
            for (int64_t t = threadIdx.x; t < size; t += blockDim.x) rowflag[rows[t]] = 2;
        __syncthreads();
    }
}

struct PairCtx {
    const uint32_t *lt;
    const int32_t *members, *nbr;
    const int64_t *S, *grp_off, *item0;
    const int32_t *grp_len;
    const int *prow;
    int32_t n, K, Q;
    int64_t ntiles;
    uint8_t *pbuf;            // kept pair counts (count pass writes, fill reads)
    int64_t pcap;
    unsigned long long *pused;
    int64_t *islot;
};

// Column c of a tile sits at slot 8 (c % 16) + c / 16, so that the eight
// slots 8tx..8tx+7 a thread reads with two 16-byte loads are the columns
// tx, tx + 16, ..., tx + 112: each group of 16 consecutive columns is then
// held by the 16 lanes of a half-warp, one column per lane.
__device__ __forceinline__ int col_slot(int c) { return ((c & 15) << 3) | (c >> 4); }

// 128 points' label pairs into s[w*128 + slot] (-1: a NaN point); idx is
// indexed by slot
__device__ __forceinline__ void load_pairs(uint32_t *s, const int32_t *idx, const uint32_t *lt,
                                           int32_t Q)
{
    for (int k = threadIdx.x; k < kPT * (Q / 4); k += blockDim.x) {
        const int r = k & (kPT - 1), v = k >> 7;
        const int32_t i = idx[r];
        const uint4 x = i >= 0 ? *reinterpret_cast<const uint4 *>(lt + (int64_t)i * Q + 4 * v)
                               : make_uint4(0x7e007e00u, 0x7e007e00u, 0x7e007e00u, 0x7e007e00u);
        s[(4 * v) * kPT + r] = x.x;
        s[(4 * v + 1) * kPT + r] = x.y;
        s[(4 * v + 2) * kPT + r] = x.z;
        s[(4 * v + 3) * kPT + r] = x.w;
    }
}

// One CTA per (group, 128-row block), from a queue over all groups' blocks.
// Thread (tx, ty) of a 16 x 16 grid owns rows 8ty..8ty+7 and columns tx +
// 16b (b = 0..7) of each tile.  A row's 16 consecutive columns 16b..16b+15
// are then one per lane of a half-warp: a ballot places its kept entries, and
// the half-warp writes them to consecutive positions with one store.
// COUNT: distinct columns per row -> rowcnt, rowflag (and the first
// partition's overflow check).  FILL: the kept entries at indptr[i].
template <bool FILL>
__global__ void __launch_bounds__(kPairThreads, 2)
k_pairs(PairCtx pc, TailCtx tc, const int32_t *order, const int64_t *cap_indptr,
        const int64_t *indptr, int32_t *rowcnt, int32_t *rowflag, int32_t *indices,
        uint8_t *data, int *queue, int *gmax, int *err)
{
    extern __shared__ __align__(16) uint32_t psm[];
    const int32_t Q = pc.Q, K = pc.K;
    uint32_t *sR = psm;
    uint32_t *sC = psm + (size_t)Q * kPT;
    __shared__ int32_t s_row[kPT], s_col[kPT];
    __shared__ int64_t s_end[kPT], s_cur[kPT];
    __shared__ int64_t s_slot;
    __shared__ int s_item, s_c0;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int pr = *pc.prow;
    const int64_t nitems = pc.item0[K];
    int maxc = 0;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int64_t t = s_item;
        if (t >= nitems) break;
        int glo = 0, ghi = K;                       // item0[glo] <= t < item0[ghi]
        while (ghi - glo > 1) {
            const int m = (glo + ghi) >> 1;
            if (pc.item0[m] <= t) glo = m; else ghi = m;
        }
        const int g = glo;
        const int64_t gb = pc.S[((int64_t)pr * K + g) * pc.ntiles];
        const int64_t size = pc.S[((int64_t)pr * K + g + 1) * pc.ntiles] - gb;
        const int64_t r0 = (t - pc.item0[g]) * kPT;
        const int nrow = (int)(size - r0 < kPT ? size - r0 : kPT);
        for (int r = threadIdx.x; r < kPT; r += blockDim.x) {
            const int32_t i = r < nrow ? pc.members[gb + r0 + r] : -1;
            s_row[r] = i;
            if (FILL) {
                s_end[r] = i >= 0 ? indptr[i + 1] : 0;
                s_cur[r] = i >= 0 ? indptr[i] : 0;
            }
        }
        __syncthreads();
        load_pairs(sR, s_row, pc.lt, Q);
        const int32_t *nb = pc.nbr + pc.grp_off[g];
        const int32_t len = pc.grp_len[g];
        if (threadIdx.x == 0) {
            int a = 0, b = len;
            const int32_t first = s_row[0];
            while (a < b) {
                const int m = (a + b) >> 1;
                if (nb[m] > first) b = m; else a = m + 1;
            }
            s_c0 = a;
            // the item's counts: a place reserved by the count pass, which
            // the fill reads instead of comparing again
            if (FILL) {
                s_slot = pc.islot[t];
            } else {
                const int64_t need = (int64_t)((len - a + kPT - 1) / kPT) * kPairThreads * 64;
                int64_t at = -1;
                if (need > 0) {
                    at = (int64_t)atomicAdd(pc.pused, (unsigned long long)need);
                    if (at + need > pc.pcap) at = -1;
                }
                pc.islot[t] = at;
                s_slot = at;
            }
        }
        // this thread's rows: a row that takes no entries compares as INT_MAX
        int32_t ri[8];
        int dcount[8];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int32_t i = s_row[8 * ty + a];
            bool live = i >= 0;
            if (FILL && live) live = !(rowflag[i] & 1);
            ri[a] = live ? i : 0x7fffffff;
            dcount[a] = 0;
        }
        __syncthreads();
        const int64_t slot = s_slot;
        for (int cb = s_c0, ci = 0; cb < len; cb += kPT, ++ci) {
            for (int c = threadIdx.x; c < kPT; c += blockDim.x)
                s_col[col_slot(c)] = cb + c < len ? nb[cb + c] : -1;
            __syncthreads();
            // the thread's 64 counts, one byte each: pw[2a + b/4] byte b%4 is
            // (row 8ty + a, column tx + 16b)
            uint32_t pw[16];
            uint4 *kept = slot >= 0 ? reinterpret_cast<uint4 *>(
                              pc.pbuf + slot + ((int64_t)ci * kPairThreads + threadIdx.x) * 64)
                                    : nullptr;
            if (FILL && slot >= 0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint4 v = kept[q];
                    pw[4 * q] = v.x;
                    pw[4 * q + 1] = v.y;
                    pw[4 * q + 2] = v.z;
                    pw[4 * q + 3] = v.w;
                }
            } else {
                load_pairs(sC, s_col, pc.lt, Q);
                __syncthreads();
                __half2 acc[8][8];
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int b = 0; b < 8; ++b) acc[a][b] = __float2half2_rn(0.f);
#pragma unroll 2
                for (int w = 0; w < Q; ++w) {
                    const uint4 ra = *reinterpret_cast<const uint4 *>(sR + w * kPT + 8 * ty);
                    const uint4 rb = *reinterpret_cast<const uint4 *>(sR + w * kPT + 8 * ty + 4);
                    const uint4 ca = *reinterpret_cast<const uint4 *>(sC + w * kPT + 8 * tx);
                    const uint4 cc = *reinterpret_cast<const uint4 *>(sC + w * kPT + 8 * tx + 4);
                    const uint32_t R[8] = {ra.x, ra.y, ra.z, ra.w, rb.x, rb.y, rb.z, rb.w};
                    const uint32_t C[8] = {ca.x, ca.y, ca.z, ca.w, cc.x, cc.y, cc.z, cc.w};
#pragma unroll
                    for (int a = 0; a < 8; ++a) {
                        const __half2 rv = *reinterpret_cast<const __half2 *>(&R[a]);
#pragma unroll
                        for (int b = 0; b < 8; ++b)
                            acc[a][b] = __hadd2(
                                acc[a][b], __heq2(rv, *reinterpret_cast<const __half2 *>(&C[b])));
                    }
                }
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        uint32_t word = 0;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const __half2 v = acc[a][4 * h + e];
                            word |= (uint32_t)(__low2float(v) + __high2float(v)) << (8 * e);
                        }
                        pw[2 * a + h] = word;
                    }
                if (!FILL && slot >= 0)
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        kept[q] = make_uint4(pw[4 * q], pw[4 * q + 1], pw[4 * q + 2], pw[4 * q + 3]);
            }
            int32_t cj[8];
#pragma unroll
            for (int b = 0; b < 8; ++b) cj[b] = s_col[8 * tx + b];
            const int half = threadIdx.x & 16;              // this half-warp's ballot bits
            const uint32_t below = (1u << tx) - 1u;
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                // the half-warp's lanes all read the cursor before the first
                // ballot and lane 0 advances it after the last
                int64_t at = FILL ? s_cur[8 * ty + a] : 0;
                const int64_t end = FILL ? s_end[8 * ty + a] : 0;
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    const int cnt = (int)((pw[2 * a + (b >> 2)] >> (8 * (b & 3))) & 255u);
                    const bool keep = cj[b] > ri[a] && cnt > 0;
                    if (FILL) {
                        const uint32_t m = (__ballot_sync(0xffffffffu, keep) >> half) & 0xffffu;
                        const int64_t pos = at + __popc(m & below);
                        if (keep && pos < end) {
                            indices[pos] = cj[b];
                            data[pos] = (uint8_t)cnt;
                            maxc = max(maxc, cnt);
                        }
                        at += __popc(m);
                    } else {
                        dcount[a] += keep;
                    }
                }
                if (FILL) {
                    __syncwarp();
                    if (tx == 0) s_cur[8 * ty + a] = at;
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int32_t i = s_row[8 * ty + a];
            if (FILL) {
                if (tx == 0 && ri[a] != 0x7fffffff && s_cur[8 * ty + a] != indptr[i + 1])
                    set_err(err, DEV_CAPACITY);
            } else {
                int d = dcount[a];
#pragma unroll
                for (int o = 8; o >= 1; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o, 16);
                if (tx == 0 && i >= 0) {
                    const int64_t cap = cap_indptr[i + 1] - cap_indptr[i];
                    rowcnt[i] = (int32_t)(d < cap ? d : cap);
                    rowflag[i] = 2 | (d > cap ? 1 : 0);
                    // the first partition in processing order takes no capacity check
                    int64_t s, e;
                    tc.tail(i, order[0], s, e);
                    if (e - s > cap) set_err(err, DEV_FIRST_OVERFLOW);
                }
            }
        }
        __syncthreads();
    }
    if (FILL) {
        for (int d = 16; d >= 1; d >>= 1) maxc = max(maxc, __shfl_xor_sync(0xffffffffu, maxc, d));
        if ((threadIdx.x & 31) == 0) atomicMax(gmax, maxc);
    }
}

// rows of the row order whose flag bits under `mask` equal `want`, kept in
// that order within each warp's 32 (the lists the streaming kernels take)
__global__ void k_pick_rows(const int32_t *rowperm, int32_t n, const int32_t *rowflag, int mask,
                            int want, int32_t *out, int *count)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t b = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~(int64_t)31; b < n;
         b += stride) {
        const int64_t q = b + lane;
        const int32_t i = q < n ? rowperm[q] : -1;
        const bool sel = i >= 0 && (rowflag[i] & mask) == want;
        const unsigned m = __ballot_sync(0xffffffffu, sel);
        int base = 0;
        if (lane == 0 && m) base = atomicAdd(count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (sel) out[base + __popc(m & ((1u << lane) - 1u))] = i;
    }
}

__global__ void k_diassoc_val(uint8_t *data, int64_t nnz, uint32_t top)
{
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x)
        data[e] = (uint8_t)(top - data[e]);
}

__global__ void k_diassoc(uint8_t *data, int64_t nnz, const int *gmax)
{
    const uint32_t top = (uint32_t)(*gmax) + 1u;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x)
        data[e] = (uint8_t)(top - data[e]);
}

// Row order of the row kernels: the points cluster by cluster of the
// partition with the most clusters (its member lists), then the points it
// leaves unlabelled.  Rows in flight then share member lists -- in that
// partition by construction, in the others mostly, since they are close
// points -- and read them from L2 instead of HBM.
__global__ void k_rowperm(const int32_t *labels, int32_t n, int32_t P, int32_t K, int64_t ntiles,
                          const int32_t *members, const int64_t *S, const int32_t *ncl,
                          int32_t *rowperm, int *counter, int *prow)
{
    int pr = 0;
    for (int p = 1; p < P; ++p)
        if (ncl[p] > ncl[pr]) pr = p;
    if (blockIdx.x == 0 && threadIdx.x == 0) *prow = pr;
    const int64_t s0 = S[(int64_t)pr * K * ntiles], s1 = S[((int64_t)pr + 1) * K * ntiles];
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < s1 - s0; q += stride)
        rowperm[q] = members[s0 + q];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (labels[(int64_t)pr * n + i] < 0) rowperm[(s1 - s0) + atomicAdd(counter, 1)] = (int32_t)i;
}

static int check_args(const int32_t *labels, int32_t n, int32_t P, int32_t K)
{
    if (!labels || n <= 0 || P <= 0 || P > kMaxP || K <= 0) return EACB_ERR_BAD_ARGUMENT;
    if (K > kMaxK) return EACB_ERR_UNSUPPORTED;
    if ((int64_t)P * n >= ((int64_t)1 << 31)) return EACB_ERR_UNSUPPORTED;
    return EACB_OK;
}

static int read_err(int *err, cudaStream_t st)
{
    int e = 0;
    EACB_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    return dev_err_to_status(e);
}

static int row_grid(int ctas_per_sm = 2)
{
    ctas_per_sm = ctas_per_sm < 1 ? 1 : (ctas_per_sm > 2 ? 2 : ctas_per_sm);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return ctas_per_sm * sms;
}

template <bool FILL>
static int launch_pairs(const CoWS &w, const TailCtx &tc, const int64_t *cap_indptr,
                        const int64_t *indptr, int32_t *indices, uint8_t *data, cudaStream_t st)
{
    const size_t smem = (size_t)2 * w.Q * kPT * sizeof(uint32_t);
    if (smem > 200 * 1024) return EACB_ERR_UNSUPPORTED;
    EACB_CUDA(allow_max_dyn_smem(k_pairs<FILL>));
    PairCtx pc{w.lt, w.members, w.nbr, w.S, w.grp_off, w.grp_item0, w.grp_len, w.prow,
               tc.n, tc.K, w.Q, w.ntiles, w.pbuf, w.pcap, w.pused, w.islot};
    if (!FILL) EACB_CUDA(cudaMemsetAsync(w.pused, 0, sizeof(unsigned long long), st));
    k_pairs<FILL><<<row_grid(2), kPairThreads, smem, st>>>(
        pc, tc, w.order, cap_indptr, indptr, w.rowcnt, w.rowflag, indices, data,
        &w.queue[FILL ? 6 : 5], w.maxcnt, w.err);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

}  // namespace eacb

using namespace eacb;

extern "C" size_t eacb_coassoc_workspace_size(int32_t n, int32_t P, int32_t K)
{
    Carver c(nullptr, 0);
    CoWS::carve(c, n, P, K);
    return c.off;
}

extern "C" int eacb_coassoc_prepare(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                                    int64_t *host_max_cluster, void *ws, size_t ws_bytes,
                                    uintptr_t stream)
{
    int s = check_args(labels, n, P, K);
    if (s) return s;
    if (!host_max_cluster || !ws) return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    CoWS w = CoWS::carve(c, n, P, K);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    EACB_CUDA(cudaMemsetAsync(w.queue, 0, kQueues * sizeof(int), st));
    const int64_t nt = w.ntiles;
    const int64_t m = (int64_t)P * K * nt;
    k_ml_count<<<(unsigned)(P * nt), 256, K * sizeof(int), st>>>(labels, n, K, nt, w.cnt, w.err);
    EACB_CHECK_LAUNCH();
    if ((s = scan_launch<int32_t, int64_t>(w.cnt, w.S, m, 0, &w.S[m], w.scan, st))) return s;
    const size_t place_smem = (size_t)K * (sizeof(int64_t) + sizeof(int32_t));
    if (place_smem > 48 * 1024)
        EACB_CUDA(allow_max_dyn_smem(k_ml_place));
    k_ml_place<<<(unsigned)(P * nt), 32, place_smem, st>>>(labels, n, K, nt, w.S, w.members,
                                                           w.mypos);
    EACB_CHECK_LAUNCH();
    EACB_CUDA(cudaMemsetAsync(w.maxcnt, 0, sizeof(int), st));
    k_ncl<<<P, 256, 0, st>>>(w.S, K, nt, w.ncl, w.maxcnt);
    EACB_CHECK_LAUNCH();
    k_order<<<1, 32, 0, st>>>(w.ncl, P, w.order);
    EACB_CHECK_LAUNCH();
    k_rowperm<<<grid_for(n, 256), 256, 0, st>>>(labels, n, P, K, nt, w.members, w.S, w.ncl,
                                                 w.rowperm, &w.queue[3], w.prow);
    EACB_CHECK_LAUNCH();
    // the path of each group (pair tiles or streaming) and the neighbourhoods
    EACB_CUDA(cudaMemsetAsync(w.rowflag, 0, sizeof(int32_t) * n, st));
    EACB_CUDA(cudaMemsetAsync(w.grp_tiles, 0, sizeof(int32_t) * ((size_t)K + 1), st));
    const int64_t ratio = K <= kDenseMaxK ? tune_get(TUNE_CO_DENSE, P, n, kDenseRatioDefault) : 0;
    if (ratio > 0) {
        k_labels_f16<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(labels, n, P, w.Q, w.lt);
        EACB_CHECK_LAUNCH();
        EACB_CUDA(cudaMemsetAsync(w.nbr_used, 0, sizeof(unsigned long long), st));
        EACB_CUDA(allow_max_dyn_smem(k_nbr));
        GroupCtx gc{labels, w.members, w.mypos, w.S, w.prow, n, P, K, w.Q, nt};
        k_nbr<<<row_grid(2), kNbrThreads, kNbrSmem, st>>>(gc, ratio, w.nbr, w.nbr_cap, w.nbr_used,
                                                          w.grp_off, w.grp_len, w.grp_tiles,
                                                          w.rowflag, &w.queue[4]);
        EACB_CHECK_LAUNCH();
    }
    if ((s = scan_launch<int32_t, int64_t>(w.grp_tiles, w.grp_item0, K, 0, &w.grp_item0[K],
                                           w.scan, st)))
        return s;
    int mc = 0;
    EACB_CUDA(cudaMemcpyAsync(&mc, w.maxcnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    if ((s = read_err(w.err, st))) return s;
    *host_max_cluster = mc;
    return EACB_OK;
}

extern "C" int eacb_coassoc_count(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                                  const int64_t *cap_indptr, int64_t *indptr, int64_t *host_nnz,
                                  void *ws, size_t ws_bytes, uintptr_t stream)
{
    int s = check_args(labels, n, P, K);
    if (s) return s;
    if (!cap_indptr || !indptr || !host_nnz || !ws) return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    CoWS w = CoWS::carve(c, n, P, K);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(w.queue, 0, kQueues * sizeof(int), st));
    TailCtx tc{labels, w.members, w.mypos, w.S, n, P, K, w.ntiles};
    EACB_CUDA(allow_max_dyn_smem(k_rows_count));
    ProfScope ps(PROF_COASSOC, st);
    if ((s = launch_pairs<false>(w, tc, cap_indptr, nullptr, nullptr, nullptr, st))) return s;
    // the streamed rows: those outside the pair tiles' groups
    EACB_CUDA(cudaMemsetAsync(w.rowlist_n, 0, sizeof(int), st));
    k_pick_rows<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(w.rowperm, n, w.rowflag, 2, 0,
                                                           w.rowlist, w.rowlist_n);
    EACB_CHECK_LAUNCH();
    k_rows_count<<<row_grid((int)tune_get(TUNE_CO_COUNT_CTAS, P, n, 2)), kRowThreads, kBitmapBytes,
                   st>>>(
        tc, w.order, w.rowlist, w.rowlist_n, cap_indptr, w.rowcnt, w.rowflag, &w.queue[0], w.err);
    EACB_CHECK_LAUNCH();
    ps.done(0.0);
    if ((s = scan_launch<int32_t, int64_t>(w.rowcnt, indptr, n, 0, &indptr[n], w.scan, st))) return s;
    EACB_CUDA(cudaMemcpyAsync(host_nnz, &indptr[n], sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    return read_err(w.err, st);
}

__global__ void k_cap_linear(int32_t n, double m, double b, int64_t ns, int64_t ne, int64_t vs,
                             int64_t ve, int64_t *y)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t v;
        if (i < ns) v = vs;
        else if (i < ne) v = (int64_t)__dadd_rn(__dmul_rn(m, (double)(int32_t)i), b);
        else v = ve;
        y[i] = v;
    }
}

__global__ void k_cap_const(int32_t n, int64_t c, int64_t *y)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
         i += (int64_t)gridDim.x * blockDim.x)
        y[i] = i * c;
}

extern "C" size_t eacb_capacity_workspace_size(int32_t n)
{
    Carver c(nullptr, 0);
    ScanScratch::carve(c, n);
    c.take<int64_t>((size_t)n + 1);
    return c.off;
}

extern "C" int eacb_capacity_linear(int32_t n, int64_t max_assocs, double n_s, double n_e,
                                    double val_s, double val_e, int64_t *cap_indptr, void *ws,
                                    size_t ws_bytes, uintptr_t stream)
{
    if (n <= 0 || max_assocs <= 0 || !cap_indptr || !ws) return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    ScanScratch sc = ScanScratch::carve(c, n);
    int64_t *y = c.take<int64_t>((size_t)n + 1);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    // the line through (n_s*n, val_s*max) and (n_e*n, val_e*max), in the
    // reference's float64 arithmetic (MyML/MyML/EAC/sparse.py:391-409)
    const double fns = n_s * n, fne = n_e * n, fvs = val_s * max_assocs, fve = val_e * max_assocs;
    const double m = (fve - fvs) / (fne - fns);
    const double b = fvs - fns * m;
    EACB_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(int), st));
    k_cap_linear<<<grid_for(n, 256), 256, 0, st>>>(n, m, b, (int64_t)fns, (int64_t)fne,
                                                    (int64_t)fvs, (int64_t)fve, y);
    EACB_CHECK_LAUNCH();
    return scan_launch<int64_t, int64_t>(y, cap_indptr, n, 0, &cap_indptr[n], sc, st);
}

extern "C" int eacb_capacity_constant(int32_t n, int64_t max_assocs, int64_t *cap_indptr,
                                      uintptr_t stream)
{
    if (n <= 0 || max_assocs <= 0 || !cap_indptr) return EACB_ERR_BAD_ARGUMENT;
    k_cap_const<<<grid_for((int64_t)n + 1, 256), 256, 0, as_stream(stream)>>>(n, max_assocs,
                                                                             cap_indptr);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

extern "C" int eacb_make_diassoc(uint8_t *data, int64_t nnz, int32_t max_val, uintptr_t stream)
{
    if (nnz < 0 || (nnz > 0 && !data)) return EACB_ERR_BAD_ARGUMENT;
    if (nnz == 0) return EACB_OK;
    k_diassoc_val<<<grid_for(nnz, 256), 256, 0, as_stream(stream)>>>(data, nnz, (uint32_t)max_val);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

extern "C" int eacb_coassoc_fill(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                                 const int64_t *cap_indptr, const int64_t *indptr,
                                 int32_t *indices, uint8_t *data, int32_t make_diassoc,
                                 int64_t *host_discarded, int32_t *host_max_count, void *ws,
                                 size_t ws_bytes, uintptr_t stream)
{
    int s = check_args(labels, n, P, K);
    if (s) return s;
    if (!cap_indptr || !indptr || !host_discarded || !host_max_count || !ws)
        return EACB_ERR_BAD_ARGUMENT;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    CoWS w = CoWS::carve(c, n, P, K);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(w.queue, 0, kQueues * sizeof(int), st));
    EACB_CUDA(cudaMemsetAsync(w.disc, 0, sizeof(unsigned long long), st));
    EACB_CUDA(cudaMemsetAsync(w.maxcnt, 0, sizeof(int), st));
    TailCtx tc{labels, w.members, w.mypos, w.S, n, P, K, w.ntiles};
    EACB_CUDA(allow_max_dyn_smem(k_rows_fill));
    EACB_CUDA(allow_max_dyn_smem(k_rows_capped));
    ProfScope ps(PROF_COASSOC, st);
    if ((s = launch_pairs<true>(w, tc, cap_indptr, indptr, indices, data, st))) return s;
    EACB_CUDA(cudaMemsetAsync(w.rowlist_n, 0, sizeof(int), st));
    k_pick_rows<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(w.rowperm, n, w.rowflag, 3, 0,
                                                           w.rowlist, w.rowlist_n);
    EACB_CHECK_LAUNCH();
    k_rows_fill<<<row_grid((int)tune_get(TUNE_CO_FILL_CTAS, P, n, 2)), kFillThreads, kFillSmem,
                  st>>>(
        tc, w.rowlist, w.rowlist_n, w.rowflag, indptr, indices, data, &w.queue[1], w.maxcnt,
        w.err);
    EACB_CHECK_LAUNCH();
    ps.done(0.0);
    // rows over their capacity, from either path
    EACB_CUDA(cudaMemsetAsync(w.rowlist_n, 0, sizeof(int), st));
    k_pick_rows<<<grid_for(n, 256, 148 * 8), 256, 0, st>>>(w.rowperm, n, w.rowflag, 1, 1,
                                                           w.rowlist, w.rowlist_n);
    EACB_CHECK_LAUNCH();
    k_rows_capped<<<row_grid(), kRowThreads, kCapSmem, st>>>(
        tc, w.order, w.rowlist, w.rowlist_n, w.rowflag, cap_indptr, indptr, indices, data,
        &w.queue[2], w.maxcnt, w.disc, w.err);
    EACB_CHECK_LAUNCH();
    int64_t nnz = 0;
    EACB_CUDA(cudaMemcpyAsync(&nnz, &indptr[n], sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    unsigned long long dh = 0;
    int mh = 0;
    EACB_CUDA(cudaMemcpyAsync(&dh, w.disc, sizeof(dh), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaMemcpyAsync(&mh, w.maxcnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    if ((s = read_err(w.err, st))) return s;
    if (make_diassoc && nnz > 0) {
        k_diassoc<<<grid_for(nnz, 256), 256, 0, st>>>(data, nnz, w.maxcnt);
        EACB_CHECK_LAUNCH();
    }
    *host_discarded = (int64_t)dh;
    *host_max_count = mh;
    return EACB_OK;
}

// One call for the whole build: member lists, the capacity layout from the
// largest cluster (max_assocs = factor x largest cluster when max_assocs is
// 0, like EAC.buildMatrix, MyML/MyML/EAC/eac.py:115-140), kept counts, then
// the rows.  indices/data hold `capacity` entries (the reference
// preallocates the capacity layout's total, sparse.py:109-138; the kept
// count never exceeds it); rows are written back to back (condensed).
static size_t coassoc_build_ws(int32_t n, int32_t P, int32_t K, size_t *co, size_t *cap_ws)
{
    *co = (eacb_coassoc_workspace_size(n, P, K) + 255) & ~(size_t)255;
    *cap_ws = (eacb_capacity_workspace_size(n) + 255) & ~(size_t)255;
    return *co + *cap_ws + (((size_t)n + 1) * sizeof(int64_t) + 255) / 256 * 256;
}

extern "C" size_t eacb_coassoc_build_workspace_size(int32_t n, int32_t P, int32_t K)
{
    size_t co, cw;
    return coassoc_build_ws(n, P, K, &co, &cw);
}

extern "C" int eacb_coassoc_build(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                                  int32_t cap_mode, int64_t max_assocs, int32_t factor,
                                  int64_t *indptr, int32_t *indices, uint8_t *data,
                                  int64_t capacity, int32_t make_diassoc, int64_t *host_nnz,
                                  int64_t *host_discarded, int32_t *host_max_count,
                                  int64_t *host_max_assocs, void *ws, size_t ws_bytes,
                                  uintptr_t stream)
{
    if (!indptr || !indices || !data || !host_nnz || !host_discarded || !host_max_count ||
        !host_max_assocs || !ws || (cap_mode != 0 && cap_mode != 1) || max_assocs < 0 ||
        (max_assocs == 0 && factor <= 0) || capacity < 0)
        return EACB_ERR_BAD_ARGUMENT;
    size_t co, cw;
    if (ws_bytes < coassoc_build_ws(n, P, K, &co, &cw)) return EACB_ERR_WORKSPACE;
    char *base = (char *)ws;
    int64_t *cap_indptr = (int64_t *)(base + co + cw);
    int64_t maxc = 0;
    int s = eacb_coassoc_prepare(labels, n, P, K, &maxc, base, co, stream);
    if (s) return s;
    const int64_t ma = max_assocs ? max_assocs : maxc * (int64_t)factor;
    *host_max_assocs = ma;
    if (cap_mode == 0)
        s = eacb_capacity_linear(n, ma, 0.05, 1.0, 1.0, 0.05, cap_indptr, base + co, cw, stream);
    else
        s = eacb_capacity_constant(n, ma, cap_indptr, stream);
    if (s) return s;
    int64_t nnz = 0;
    if ((s = eacb_coassoc_count(labels, n, P, K, cap_indptr, indptr, &nnz, base, co, stream)))
        return s;
    *host_nnz = nnz;
    if (nnz > capacity) return EACB_ERR_WORKSPACE;
    return eacb_coassoc_fill(labels, n, P, K, cap_indptr, indptr, indices, data, make_diassoc,
                             host_discarded, host_max_count, base, co, stream);
}
