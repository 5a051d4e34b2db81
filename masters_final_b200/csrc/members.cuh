// Cluster member lists by a stable counting sort (shared by the
// co-association build and the k-means centroid update).
//
// For a label matrix labels[p*n + i] in [0, K) (-1 = none), the member list of
// cluster (p, c) is the ascending list of points with that label.  Lists are
// laid out back to back in (partition, cluster) order: a tile histogram
// cnt[(p*K + c)*ntiles + tile] is scanned (exclusive, int64) into S, so that
// S[(p*K + c)*ntiles + tile] is where tile `tile`'s members of (p, c) start and
// [S[(p*K+c)*ntiles], S[(p*K+c+1)*ntiles]) is the whole list.
#pragma once
#include "eacb_common.cuh"

namespace eacb {

constexpr int kMLTile = 4096;          // points per tile in the counting sort

// ---------------------------------------------------------------- step 1 --
static __global__ void __launch_bounds__(256)
k_ml_count(const int32_t *labels, int32_t n, int32_t K, int64_t ntiles, int32_t *cnt, int *err)
{
    extern __shared__ int hist[];
    const int64_t p = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
    for (int c = threadIdx.x; c < K; c += blockDim.x) hist[c] = 0;
    __syncthreads();
    const int64_t i0 = tile * kMLTile;
    const int32_t *lp = labels + p * n;
    for (int64_t i = i0 + threadIdx.x; i < i0 + kMLTile && i < n; i += blockDim.x) {
        int32_t l = lp[i];
        if (l >= K) { set_err(err, DEV_BAD_INPUT); continue; }
        if (l >= 0) atomicAdd(&hist[l], 1);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < K; c += blockDim.x)
        cnt[((int64_t)p * K + c) * ntiles + tile] = hist[c];
}

// one warp per (partition, tile): points in index order, 32 at a time
static __global__ void __launch_bounds__(32)
k_ml_place(const int32_t *labels, int32_t n, int32_t K, int64_t ntiles, const int64_t *S,
           int32_t *members, int32_t *mypos)
{
    extern __shared__ int64_t base[];          // K tile bases, then K int32 counters
    int32_t *run = (int32_t *)(base + K);
    const int64_t p = blockIdx.x / ntiles, tile = blockIdx.x % ntiles;
    const int lane = threadIdx.x;
    for (int c = lane; c < K; c += 32) {
        base[c] = S[((int64_t)p * K + c) * ntiles + tile];
        run[c] = 0;
    }
    __syncwarp();
    const int32_t *lp = labels + p * n;
    const int64_t i0 = tile * kMLTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t c0 = i0; c0 < i0 + kMLTile && c0 < n; c0 += 32) {
        const int64_t i = c0 + lane;
        int32_t l = (i < n) ? lp[i] : -1;
        if (l >= K) l = -1;
        const bool valid = l >= 0;
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? l : -1 - lane);
        int32_t before = valid ? run[l] : 0;
        __syncwarp();
        if (valid) {
            const int r = __popc(peers & lt);
            const int64_t pos = base[l] + before + r;
            members[pos] = (int32_t)i;
            mypos[p * n + i] = (int32_t)pos;
            if (lane == 31 - __clz(peers)) run[l] = before + __popc(peers);
        } else if (i < n) {
            mypos[p * n + i] = -1;
        }
        __syncwarp();
    }
}

// non-empty clusters per partition, then the processing order
static __global__ void k_ncl(const int64_t *S, int32_t K, int64_t ntiles, int32_t *ncl, int *maxsize)
{
    __shared__ int tot, big;
    if (threadIdx.x == 0) tot = big = 0;
    __syncthreads();
    const int64_t p = blockIdx.x;
    int mine = 0, mbig = 0;
    for (int c = threadIdx.x; c < K; c += blockDim.x) {
        int64_t a = S[(p * K + c) * ntiles], b = S[(p * K + c + 1) * ntiles];
        mine += b > a;
        mbig = max(mbig, (int)(b - a));
    }
    atomicAdd(&tot, mine);
    atomicMax(&big, mbig);
    __syncthreads();
    if (threadIdx.x == 0) {
        ncl[p] = tot;
        atomicMax(maxsize, big);
    }
}

static __global__ void k_order(const int32_t *ncl, int32_t P, int32_t *order)
{
    if (threadIdx.x != 0) return;
    int first = 0;
    for (int p = 1; p < P; ++p)
        if (ncl[p] < ncl[first]) first = p;
    order[0] = first;
    int q = 1;
    for (int p = 0; p < P; ++p)
        if (p != first) order[q++] = p;
}

}  // namespace eacb
