// Batched K-Means (Lloyd) ensemble generation with the reference's exact
// arithmetic.
//
// Reference: MyML/MyML/cluster/KMeans.py -- fit :117-189, _init_centroids
// :191-201, numba_label / _cu_label_kernel_dists :453-490 / :586-629,
// numba_recompute_centroids :709-754; MyML/MyML/utils/sorting.py:9-47
// (arg_k_select); MyML/MyML/utils/partition.py:88-124 (generateEnsemble).
//
// Exactness: a label is argmin_k of sum_d float64(float32((x_d - c_kd)^2))
// with the first index winning ties, the stored distance is float32 of it,
// centroids are float32(float64(float32 sequential sum) / count), the
// inertia is numpy's float32 pairwise sum of the distances and a partition
// stops early when it changes by at most tol.  The float32 label pass below
// screens all centroids with an FMA-accumulated float32 distance and keeps
// the best two; when the runner-up is outside the screening error bound of
// the winner (|screen - exact| <= (D+3) 2^-23 |exact|), only the winner's
// exact distance is computed, otherwise the point is re-labelled by the
// exact reference loop.  The labels are therefore identical to the
// reference's for any input.
//
// Batching: all P partitions of an ensemble (each with its own k) advance
// together; every kernel takes the partition from its grid and partitions
// that stopped early are skipped on the device.
#include "eacb_common.cuh"
#include "scan_impl.cuh"
#include "members.cuh"
#include "kmeans_common.cuh"

#include <type_traits>

namespace eacb {

constexpr int kLT = 128;         // label threads per block
constexpr int kLPPT = 2;         // points per thread
constexpr int kLCH = 128;        // centroids per shared-memory chunk

template <int DM>
__global__ void __launch_bounds__(kLT)
k_label_f32(const float *__restrict__ X, int32_t n, int32_t D, const float *__restrict__ C,
            const int32_t *__restrict__ kk, int32_t kmax, const int32_t *__restrict__ active,
            double ratio, int32_t *__restrict__ labels, float *__restrict__ dists,
            int32_t *__restrict__ amb, int *__restrict__ namb)
{
    __shared__ float cs[kLCH * DM];
    const int p = blockIdx.y;
    if (!active[p]) return;
    const int K = kk[p];
    const float *Cp = C + (int64_t)p * kmax * D;
    float x[kLPPT][DM];
    float b1[kLPPT], b2[kLPPT];
    int i1[kLPPT];
    int64_t idx[kLPPT];
#pragma unroll
    for (int q = 0; q < kLPPT; ++q) {
        idx[q] = ((int64_t)blockIdx.x * kLPPT + q) * kLT + threadIdx.x;
#pragma unroll
        for (int d = 0; d < DM; ++d) x[q][d] = (idx[q] < n && d < D) ? X[idx[q] * D + d] : 0.f;
        b1[q] = b2[q] = __int_as_float(0x7f800000);
        i1[q] = 0;
    }
    for (int c0 = 0; c0 < K; c0 += kLCH) {
        const int cn = min(kLCH, K - c0);
        __syncthreads();
        for (int e = threadIdx.x; e < cn * D; e += kLT) {
            const int c = e / D, d = e - c * D;
            cs[c * DM + d] = Cp[(int64_t)(c0 + c) * D + d];
        }
        __syncthreads();
        for (int c = 0; c < cn; ++c) {
            float s[kLPPT];
#pragma unroll
            for (int q = 0; q < kLPPT; ++q) s[q] = 0.f;
#pragma unroll
            for (int d = 0; d < DM; ++d) {
                if (d < D) {
                    const float cv = cs[c * DM + d];
#pragma unroll
                    for (int q = 0; q < kLPPT; ++q) {
                        const float t = x[q][d] - cv;
                        s[q] = fmaf(t, t, s[q]);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < kLPPT; ++q) {
                if (s[q] < b1[q]) {
                    b2[q] = b1[q];
                    b1[q] = s[q];
                    i1[q] = c0 + c;
                } else if (s[q] < b2[q]) {
                    b2[q] = s[q];
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kLPPT; ++q) {
        if (idx[q] >= n) continue;
        const int64_t o = (int64_t)p * n + idx[q];
        if ((double)b2[q] > (double)b1[q] * ratio) {
            labels[o] = i1[q];
            dists[o] = (float)exact_dist<DM>(x[q], Cp + (int64_t)i1[q] * D, D);
        } else {
            const int slot = atomicAdd(namb, 1);
            amb[slot] = (int32_t)o;      // resolved by k_label_exact
        }
    }
}

// reference loop for the points the screen could not separate
__global__ void k_label_exact(const float *__restrict__ X, int32_t n, int32_t D,
                              const float *__restrict__ C, const int32_t *__restrict__ kk,
                              int32_t kmax, const int32_t *__restrict__ amb,
                              const int *__restrict__ namb, int32_t *labels, float *dists)
{
    const int m = *namb;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const int64_t o = amb[t];
        const int64_t p = o / n, i = o - p * n;
        const int K = kk[p];
        const float *x = X + i * D;
        const float *Cp = C + p * kmax * D;
        double best = 0.0;
        int bl = 0;
        for (int k = 0; k < K; ++k) {
            double dist = 0.0;
            for (int d = 0; d < D; ++d) {
                const float diff = __fsub_rn(x[d], Cp[(int64_t)k * D + d]);
                dist = __dadd_rn(dist, (double)__fmul_rn(diff, diff));
            }
            if (k == 0 || dist < best) {
                best = dist;
                bl = k;
            }
        }
        labels[o] = bl;
        dists[o] = (float)best;
    }
}

// numpy float32 add.reduce of a contiguous array: pairwise summation, blocks
// of at most 128 summed with 8 partial sums; a node longer than 128 splits at
// n/2 rounded down to a multiple of 8 and adds (left, right).
__device__ __forceinline__ float np_pairwise_leaf(const float *a, int64_t n)
{
    if (n < 8) {
        float r = -0.0f;
        for (int64_t i = 0; i < n; ++i) r = __fadd_rn(r, a[i]);
        return r;
    }
    float r[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) r[j] = a[j];
    int64_t i = 8;
    for (; i < n - (n % 8); i += 8)
#pragma unroll
        for (int j = 0; j < 8; ++j) r[j] = __fadd_rn(r[j], a[i + j]);
    float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                          __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
    for (; i < n; ++i) res = __fadd_rn(res, a[i]);
    return res;
}

// Iterative post-order walk of the split tree (depth < 48 for any int64 n),
// so no device stack is needed.
__device__ float np_pairwise(const float *a, int64_t n)
{
    int64_t off[48], len[48];
    float left[48];
    int stage[48];
    int sp = 0;
    off[0] = 0;
    len[0] = n;
    stage[0] = 0;
    float ret = 0.f;
    while (sp >= 0) {
        if (len[sp] <= 128) {
            ret = np_pairwise_leaf(a + off[sp], len[sp]);
            sp--;
            continue;
        }
        int64_t n2 = len[sp] / 2;
        n2 -= n2 % 8;
        if (stage[sp] == 0) {
            stage[sp] = 1;
            off[sp + 1] = off[sp];
            len[sp + 1] = n2;
            stage[sp + 1] = 0;
            sp++;
        } else if (stage[sp] == 1) {
            left[sp] = ret;
            stage[sp] = 2;
            off[sp + 1] = off[sp] + n2;
            len[sp + 1] = len[sp] - n2;
            stage[sp + 1] = 0;
            sp++;
        } else {
            ret = __fadd_rn(left[sp], ret);
            sp--;
        }
    }
    return ret;
}

// inertia and the convergence test of one iteration (KMeans.py:158-180).
// One block per partition.  The top levels of numpy's split tree are
// expanded while every node is still split (longer than 128) and there are
// at most kInertiaThreads nodes; each thread sums one node's subtree with the
// sequential walk, then the expanded levels are added back pairwise in the
// tree's own order, so the result is bit-identical to the sequential sum.
constexpr int kInertiaThreads = 256;
__global__ void __launch_bounds__(kInertiaThreads)
k_inertia(const float *dists, int32_t n, int32_t P, int32_t *active, float *inertia,
          int32_t *iters, float tol)
{
    __shared__ int64_t s_off[kInertiaThreads], s_len[kInertiaThreads];
    __shared__ float s_val[kInertiaThreads];
    __shared__ int s_cnt;
    const int p = blockIdx.x;
    if (p >= P || !active[p]) return;          // uniform across the block
    const float *a = dists + (int64_t)p * n;
    if (threadIdx.x == 0) {
        s_off[0] = 0;
        s_len[0] = n;
        int cnt = 1;
        while (cnt * 2 <= kInertiaThreads) {
            bool split_all = true;
            for (int q = 0; q < cnt; ++q)
                if (s_len[q] <= 128) split_all = false;
            if (!split_all) break;
            // children of node q go to 2q and 2q+1 (back to front, in place)
            for (int q = cnt - 1; q >= 0; --q) {
                const int64_t o = s_off[q], l = s_len[q];
                int64_t n2 = l / 2;
                n2 -= n2 % 8;
                s_off[2 * q] = o;
                s_len[2 * q] = n2;
                s_off[2 * q + 1] = o + n2;
                s_len[2 * q + 1] = l - n2;
            }
            cnt *= 2;
        }
        s_cnt = cnt;
    }
    __syncthreads();
    const int cnt = s_cnt;
    if ((int)threadIdx.x < cnt) s_val[threadIdx.x] = np_pairwise(a + s_off[threadIdx.x], s_len[threadIdx.x]);
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = cnt; c > 1; c >>= 1)
            for (int q = 0; q < c / 2; ++q) s_val[q] = __fadd_rn(s_val[2 * q], s_val[2 * q + 1]);
        const float I = s_val[0];
        const float err = fabsf(__fsub_rn(I, inertia[p]));
        inertia[p] = I;
        iters[p] += 1;
        if (err <= tol) active[p] = 0;
    }
}

// float32 (reference) or float64 sums of each cluster's members in point order
constexpr int kCentDepth = 16;       // members in flight per lane

template <bool F64>
__global__ void k_centroids(const float *__restrict__ X, int32_t n, int32_t D,
                            const int32_t *__restrict__ members, const int64_t *__restrict__ S,
                            int32_t K, int64_t ntiles, const int32_t *__restrict__ kk, int32_t kmax,
                            const int32_t *__restrict__ active, float *C, int32_t *nempty)
{
    const int p = blockIdx.y;
    if (!active[p]) return;
    const int Kp = kk[p];
    const int lane = threadIdx.x & 31;
    const int G = 32 / D;                       // clusters per warp
    const int g = lane / D, d = lane - g * D;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int c = warp * G + g;
    if (g >= G || c >= Kp) return;
    const int64_t s0 = S[((int64_t)p * K + c) * ntiles], s1 = S[((int64_t)p * K + c + 1) * ntiles];
    const int64_t cnt = s1 - s0;
    float *out = C + ((int64_t)p * kmax + c) * D + d;
    if (cnt == 0) {
        if (d == 0) atomicAdd(&nempty[p], 1);
        return;
    }
    // The sums are sequential in member order (the reference's order), so a
    // cluster's sum is a chain as long as the cluster; the largest cluster
    // sets the kernel's time.  Members go kCentDepth at a time: the next
    // batch's ids load while this batch's coordinates do, and the adds follow
    // in order, so a batch costs one memory latency.
    using Acc = typename std::conditional<F64, double, float>::type;
    Acc acc = 0;
    auto add = [&](float v) {
        if (F64) acc += (double)v;
        else acc = (Acc)__fadd_rn((float)acc, v);
    };
    int64_t m = s0;
    if (m + kCentDepth <= s1) {
        int32_t id[kCentDepth];
#pragma unroll
        for (int q = 0; q < kCentDepth; ++q) id[q] = members[m + q];
        for (; m + kCentDepth <= s1; m += kCentDepth) {
            float v[kCentDepth];
#pragma unroll
            for (int q = 0; q < kCentDepth; ++q) v[q] = X[(int64_t)id[q] * D + d];
            const bool more = m + 2 * kCentDepth <= s1;
#pragma unroll
            for (int q = 0; q < kCentDepth; ++q) id[q] = more ? members[m + kCentDepth + q] : 0;
#pragma unroll
            for (int q = 0; q < kCentDepth; ++q) add(v[q]);
        }
    }
    for (; m < s1; ++m) add(X[(int64_t)members[m] * D + d]);
    if (F64) *out = __double2float_rn((double)acc / (double)cnt);
    else *out = __double2float_rn(__ddiv_rn((double)acc, (double)cnt));
}

// Empty clusters take the points arg_k_select returns for their number
// (KMeans.py:727-750, MyML/MyML/utils/sorting.py:9-47): the reference's
// quickselect on (distance, index) pairs, one block per partition, with the
// distances permuted in place (key[r] is the reference's a[args[r]]; the
// distances are not needed again before the next label pass).
//
// One partition step of the reference on [lo, hi] with pivot mid moves the
// element at r to the back (swapping in the element at w) when it is >= mid,
// and otherwise advances r.  Its result has a closed form that a block can
// compute in parallel.  Read the range from the front (F[t] = position
// lo + t) and from the back (B[u] = position hi - u); "big" means >= mid.
// The step examines F up to its m-th big a_m, then B up to its m-th small
// b_m, then F again, and so on, until hi - lo + 1 elements are examined; the
// last one examined stays at r.  Every other examined element lands at:
//   a front small F[t]       -> position of F[t] (it stays),
//   the m-th front big       -> position of B[b_{m-1} + 1]   (b_0 = -1),
//   the m-th back small      -> position of F[a_m],
//   a back big B[u]          -> position of B[u + 1],
// and r = lo + (number of smalls that landed).  Ranges up to kFillSeqMax
// elements finish with the reference's loop on one thread: its dependent
// loads cost about as much per element as a parallel step costs per range,
// so the handover is at a few hundred elements.
constexpr int kFillThreads = 1024;
constexpr int kFillItems = 8;
constexpr int64_t kFillSeqMax = 256;
constexpr int64_t kFillInf = (int64_t)1 << 62;

// Walks [lo, hi] in ascending order, calling f(p, big, bigs_before) for every
// position (bigs_before = # bigs in [lo, p)); returns the number of bigs.
// Called by the whole block.
template <typename F>
__device__ int64_t fill_scan_bigs(const float *key, int64_t lo, int64_t hi, float mid, F f)
{
    int64_t base = 0;
    for (int64_t t0 = lo; t0 <= hi; t0 += (int64_t)kFillThreads * kFillItems) {
        const int64_t p0 = t0 + (int64_t)threadIdx.x * kFillItems;
        unsigned mask = 0;
        int c = 0;
#pragma unroll
        for (int q = 0; q < kFillItems; ++q) {
            const int64_t p = p0 + q;
            if (p <= hi && key[p] >= mid) {
                mask |= 1u << q;
                ++c;
            }
        }
        int64_t tot;
        int64_t before = base + block_excl_sum<kFillThreads>(c, tot);
#pragma unroll
        for (int q = 0; q < kFillItems; ++q) {
            const int64_t p = p0 + q;
            if (p <= hi) {
                const bool big = (mask >> q) & 1u;
                f(p, big, before);
                before += big;
            }
        }
        base += tot;
    }
    return base;
}

// number of entries <= v in the ascending array a[0, len)
__device__ __forceinline__ int64_t count_le(const int32_t *a, int64_t len, int64_t v)
{
    int64_t lo = 0, hi = len;
    while (lo < hi) {
        const int64_t m = (lo + hi) >> 1;
        if (a[m] <= v) lo = m + 1; else hi = m;
    }
    return lo;
}

__global__ void __launch_bounds__(kFillThreads, 1)
k_fill_empty(const float *X, int32_t n, int32_t D, float *dists, const int64_t *S, int32_t K,
             int64_t ntiles, const int32_t *kk, int32_t kmax, const int32_t *active,
             const int32_t *nempty, int32_t *args_all, int32_t *sel_all, float *okey_all,
             int32_t *oarg_all, float *C, int *err)
{
    __shared__ int64_t s_v[5];
    const int p = blockIdx.x;
    if (!active[p] || nempty[p] == 0) return;          // uniform across the block
    const int k = nempty[p];
    float *key = dists + (int64_t)p * n;
    int32_t *args = args_all + (int64_t)p * n;
    int32_t *sel = sel_all + (int64_t)p * n;           // front-big and back-small indices
    float *okey = okey_all + (int64_t)p * n;
    int32_t *oarg = oarg_all + (int64_t)p * n;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) args[i] = (int32_t)i;
    __syncthreads();
    int64_t lo = 0, hi = n - 1;
    int rounds = 0;
    while (hi - lo + 1 > kFillSeqMax) {
        if (++rounds > 4096) {                         // cannot happen: every step shrinks the range
            if (threadIdx.x == 0) set_err(err, DEV_CHASE_LIMIT);
            return;
        }
        const int64_t L = hi - lo + 1;
        const float mid = key[(lo + hi) / 2];
        // count the bigs, then list front bigs (sel[0, NB)) and back smalls
        // (sel[NB, L)) by rank
        int64_t nbig;
        {
            int64_t c = 0;
            for (int64_t q = lo + threadIdx.x; q <= hi; q += blockDim.x) c += key[q] >= mid;
            nbig = 0;
            block_excl_sum<kFillThreads>(c, nbig);
        }
        const int64_t NB = nbig, NS = L - NB;
        fill_scan_bigs(key, lo, hi, mid, [&](int64_t q, bool big, int64_t before) {
            const int64_t t = q - lo;
            if (big) sel[before] = (int32_t)t;
            else sel[NB + NS - 1 - (t - before)] = (int32_t)(hi - q);   // rank from the back
        });
        __syncthreads();
        if (threadIdx.x == 0) {
            const int32_t *A = sel, *Bs = sel + NB;
            auto a_of = [&](int64_t m) -> int64_t { return m <= NB ? A[m - 1] : kFillInf; };
            auto b_of = [&](int64_t m) -> int64_t {
                return m == 0 ? -1 : (m <= NS ? Bs[m - 1] : kFillInf);
            };
            // the segment m1 in which the examination ends: first m with
            // (a_m + 1) + (b_m + 1) >= L
            int64_t ml = 1, mh = (NB < NS ? NB : NS) + 1;
            while (ml < mh) {
                const int64_t m = (ml + mh) >> 1;
                const int64_t am = a_of(m), bm = b_of(m);
                const bool reach = am >= kFillInf || bm >= kFillInf || am + bm + 2 >= L;
                if (reach) mh = m; else ml = m + 1;
            }
            const int64_t m1 = ml, am1 = a_of(m1), bprev = b_of(m1 - 1);
            int64_t x, y, last_front;
            if (am1 >= kFillInf || am1 + 1 + bprev + 1 >= L) {   // ends in the front run
                y = bprev;
                x = L - 2 - y;
                last_front = 1;
            } else {                                              // ends in the back run
                x = am1;
                y = L - 2 - x;
                last_front = 0;
            }
            const int64_t front_smalls = (x + 1) - count_le(A, NB, x);
            const int64_t back_smalls = count_le(Bs, NS, y);
            const int64_t lp = last_front ? lo + x : hi - y;
            const int64_t settled_smalls = front_smalls + back_smalls - (key[lp] < mid ? 1 : 0);
            s_v[0] = x;
            s_v[1] = y;
            s_v[2] = last_front;
            s_v[3] = settled_smalls;
        }
        __syncthreads();
        const int64_t x = s_v[0], y = s_v[1], last_front = s_v[2], Sm = s_v[3];
        fill_scan_bigs(key, lo, hi, mid, [&](int64_t q, bool big, int64_t before) {
            const int64_t t = q - lo, u = hi - q;
            const bool front = t <= x;
            int64_t dst;
            if ((front && last_front && t == x) || (!front && !last_front && u == y)) {
                dst = Sm;
            } else if (front) {
                if (!big) {
                    dst = t;
                } else {                       // the m-th front big, m = before + 1
                    const int64_t bm = before == 0 ? -1 : sel[NB + before - 1];
                    dst = (L - 1) - (bm + 1);
                }
            } else {
                if (!big) {                    // back small of rank (from the back)
                    const int64_t rank = NS - 1 - (t - before);
                    dst = sel[rank];
                } else {
                    dst = (L - 1) - (u + 1);
                }
            }
            okey[lo + dst] = key[q];
            oarg[lo + dst] = args[q];
        });
        __syncthreads();
        for (int64_t q = lo + threadIdx.x; q <= hi; q += blockDim.x) {
            key[q] = okey[q];
            args[q] = oarg[q];
        }
        __syncthreads();
        int64_t r = lo + Sm;
        if (key[r] > mid) r--;
        if (k <= r) hi = r; else lo = r + 1;
    }
    if (threadIdx.x != 0) return;
    int64_t guard = 0;
    const int64_t limit = 64 * (int64_t)n + 4096;
    while (lo < hi) {
        int64_t r = lo, w = hi;
        const float mid = key[(r + w) / 2];
        float kr = key[r];
        while (r < w) {
            if (kr >= mid) {
                const float kw = key[w];
                const int32_t t = args[w];
                key[w] = kr;
                args[w] = args[r];
                key[r] = kw;
                args[r] = t;
                kr = kw;
                w--;
            } else {
                kr = key[++r];
            }
            ++guard;
        }
        if (key[r] > mid) r--;
        if (k <= r) hi = r; else lo = r + 1;
        if (++guard > limit) { set_err(err, DEV_CHASE_LIMIT); return; }
    }
    const int Kp = kk[p];
    int e = 0;
    for (int c = 0; c < Kp; ++c) {
        if (S[((int64_t)p * K + c + 1) * ntiles] != S[((int64_t)p * K + c) * ntiles]) continue;
        const int32_t src = args[e++];
        for (int d = 0; d < D; ++d) C[((int64_t)p * kmax + c) * D + d] = X[(int64_t)src * D + d];
    }
}

__global__ void k_init_centroids(const float *X, int32_t D, const int32_t *init, const int32_t *kk,
                                 int32_t kmax, int32_t P, float *C, int32_t *active, float *inertia,
                                 int32_t *iters, int32_t n, int *err)
{
    const int64_t total = (int64_t)P * kmax * D;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = e / ((int64_t)kmax * D);
        const int64_t r = e - p * kmax * D;
        const int c = (int)(r / D), d = (int)(r % D);
        if (c >= kk[p]) continue;
        const int32_t src = init[p * kmax + c];
        if (src < 0 || src >= n) { set_err(err, DEV_BAD_INPUT); continue; }
        C[e] = X[(int64_t)src * D + d];
        if (c == 0 && d == 0) {
            active[p] = 1;
            inertia[p] = __int_as_float(0x7f800000);
            iters[p] = 0;
        }
    }
}

struct KMWS {
    int *err;
    float *dists;
    int32_t *active, *iters, *nempty, *amb, *namb;
    float *inertia;
    int32_t *members, *mypos, *cnt, *args;
    int64_t *S;
    int32_t *ncl, *order;
    int *maxsize;
    ScanScratch scan;
    TcScratch tc;
    int64_t ntiles;
    static KMWS carve(Carver &c, int32_t n, int32_t D, int32_t P, int32_t kmax)
    {
        KMWS w;
        w.err = c.take<int>(1);
        const int64_t pn = (int64_t)P * n;
        w.ntiles = ((int64_t)n + kMLTile - 1) / kMLTile;
        const int64_t m = (int64_t)P * kmax * w.ntiles;
        w.dists = c.take<float>(pn);
        w.active = c.take<int32_t>(P);
        w.iters = c.take<int32_t>(P);
        w.nempty = c.take<int32_t>(P);
        w.namb = c.take<int32_t>(1);
        w.inertia = c.take<float>(P);
        w.amb = c.take<int32_t>(pn);
        w.members = c.take<int32_t>(pn);
        w.mypos = c.take<int32_t>(pn);
        w.args = c.take<int32_t>(pn);
        w.cnt = c.take<int32_t>(m + 1);
        w.S = c.take<int64_t>(m + 1);
        w.ncl = c.take<int32_t>(P);
        w.order = c.take<int32_t>(P);
        w.maxsize = c.take<int>(1);
        w.scan = ScanScratch::carve(c, m + 1, w.err);
        w.tc = TcScratch::carve(c, n, D, P, kmax);
        w.tc.err = w.err;         // tensor-core failures report through the same word
        return w;
    }
};

template <int DM>
static void launch_label(dim3 grid, cudaStream_t st, const float *X, int32_t n, int32_t D,
                         const float *C, const int32_t *kk, int32_t kmax, const int32_t *active,
                         double ratio, int32_t *labels, float *dists, int32_t *amb, int *namb)
{
    k_label_f32<DM><<<grid, kLT, 0, st>>>(X, n, D, C, kk, kmax, active, ratio, labels, dists, amb,
                                          namb);
}

int label_pass_f32(const float *X, int32_t n, int32_t D, int32_t P, const float *C,
                   const int32_t *kk, int32_t kmax, const int32_t *active, int32_t *labels,
                   float *dists, int32_t *amb, int *namb, cudaStream_t st)
{
    // |screen - exact| <= (D + 3) 2^-23 exact, so the winner is certain when
    // the runner-up's screened distance exceeds ratio * the winner's
    const double eps = (double)(D + 3) * ldexp(1.0, -23);
    const double ratio = (1.0 + eps) / (1.0 - eps);
    EACB_CUDA(cudaMemsetAsync(namb, 0, sizeof(int), st));
    dim3 grid((unsigned)((n + kLT * kLPPT - 1) / (kLT * kLPPT)), (unsigned)P);
    ProfScope ps(PROF_KMEANS, st);
    if (D <= 4) launch_label<4>(grid, st, X, n, D, C, kk, kmax, active, ratio, labels, dists, amb, namb);
    else if (D <= 8) launch_label<8>(grid, st, X, n, D, C, kk, kmax, active, ratio, labels, dists, amb, namb);
    else if (D <= 16) launch_label<16>(grid, st, X, n, D, C, kk, kmax, active, ratio, labels, dists, amb, namb);
    else launch_label<32>(grid, st, X, n, D, C, kk, kmax, active, ratio, labels, dists, amb, namb);
    EACB_CHECK_LAUNCH();
    ps.done(0.0);
    k_label_exact<<<148 * 4, 128, 0, st>>>(X, n, D, C, kk, kmax, amb, namb, labels, dists);
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

}  // namespace eacb

using namespace eacb;

extern "C" size_t eacb_kmeans_workspace_size(int32_t n, int32_t d, int32_t P, int32_t kmax)
{
    Carver c(nullptr, 0);
    KMWS::carve(c, n, d, P, kmax);
    (void)d;
    return c.off;
}

extern "C" int eacb_kmeans_ensemble(const float *X, int32_t n, int32_t d, int32_t P,
                                    const int32_t *k, int32_t kmax, const int32_t *init,
                                    int32_t max_iter, float tol, int32_t label_mode,
                                    int32_t centroid_mode, int32_t *labels, float *centroids,
                                    float *dists_out, int32_t *iters_out, float *inertia_out,
                                    void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (!X || n <= 0 || d <= 0 || P <= 0 || !k || kmax <= 0 || !init || max_iter <= 0 ||
        !labels || !centroids || !ws)
        return EACB_ERR_BAD_ARGUMENT;
    if (d > 32 || kmax > 8192) return EACB_ERR_UNSUPPORTED;
    if (label_mode != 0 && label_mode != 1) return EACB_ERR_BAD_ARGUMENT;
    if ((int64_t)P * n >= ((int64_t)1 << 31)) return EACB_ERR_UNSUPPORTED;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    KMWS w = KMWS::carve(c, n, d, P, kmax);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    k_init_centroids<<<grid_for((int64_t)P * kmax * d, 256), 256, 0, st>>>(
        X, d, init, k, kmax, P, centroids, w.active, w.inertia, w.iters, n, w.err);
    EACB_CHECK_LAUNCH();
    const int64_t nt = w.ntiles;
    const int64_t m = (int64_t)P * kmax * nt;
    for (int it = 0;; ++it) {
        int s;
        if (label_mode == 1)
            s = label_pass_tc(X, n, d, P, centroids, k, kmax, w.active, labels, w.dists, w.amb,
                              w.namb, w.tc, st);
        else
            s = label_pass_f32(X, n, d, P, centroids, k, kmax, w.active, labels, w.dists, w.amb,
                               w.namb, st);
        if (s) return s;
        k_inertia<<<P, kInertiaThreads, 0, st>>>(w.dists, n, P, w.active, w.inertia, w.iters,
                                                  tol);
        EACB_CHECK_LAUNCH();
        if (it + 1 >= max_iter) break;
        // centroids of the partitions still running
        k_ml_count<<<(unsigned)(P * nt), 256, kmax * sizeof(int), st>>>(labels, n, kmax, nt, w.cnt,
                                                                        w.err);
        EACB_CHECK_LAUNCH();
        if ((s = scan_launch<int32_t, int64_t>(w.cnt, w.S, m, 0, &w.S[m], w.scan, st))) return s;
        const size_t place_smem = (size_t)kmax * (sizeof(int64_t) + sizeof(int32_t));
        if (place_smem > 48 * 1024)
            EACB_CUDA(allow_max_dyn_smem(k_ml_place));
        k_ml_place<<<(unsigned)(P * nt), 32, place_smem, st>>>(labels, n, kmax, nt, w.S, w.members,
                                                               w.mypos);
        EACB_CHECK_LAUNCH();
        EACB_CUDA(cudaMemsetAsync(w.nempty, 0, sizeof(int32_t) * P, st));
        const int G = 32 / d;
        const int warps = (kmax + G - 1) / G;
        dim3 cg((unsigned)((warps * 32 + 255) / 256), (unsigned)P);
        if (centroid_mode == 1)
            k_centroids<true><<<cg, 256, 0, st>>>(X, n, d, w.members, w.S, kmax, nt, k, kmax,
                                                  w.active, centroids, w.nempty);
        else
            k_centroids<false><<<cg, 256, 0, st>>>(X, n, d, w.members, w.S, kmax, nt, k, kmax,
                                                   w.active, centroids, w.nempty);
        EACB_CHECK_LAUNCH();
        // amb, mypos and members are free here (the centroids are done) and
        // serve as the quickselect's scratch
        k_fill_empty<<<P, kFillThreads, 0, st>>>(X, n, d, w.dists, w.S, kmax, nt, k, kmax,
                                                 w.active, w.nempty, w.args, w.amb,
                                                 (float *)w.mypos, w.members, centroids, w.err);
        EACB_CHECK_LAUNCH();
    }
    if (dists_out)
        EACB_CUDA(cudaMemcpyAsync(dists_out, w.dists, sizeof(float) * (size_t)P * n,
                                  cudaMemcpyDeviceToDevice, st));
    if (iters_out)
        EACB_CUDA(cudaMemcpyAsync(iters_out, w.iters, sizeof(int32_t) * P, cudaMemcpyDeviceToDevice,
                                  st));
    if (inertia_out)
        EACB_CUDA(cudaMemcpyAsync(inertia_out, w.inertia, sizeof(float) * P,
                                  cudaMemcpyDeviceToDevice, st));
    int e = 0;
    EACB_CUDA(cudaMemcpyAsync(&e, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    return dev_err_to_status(e);
}

extern "C" int eacb_kmeans_label(const float *X, int32_t n, int32_t d, const float *C, int32_t k,
                                 int32_t label_mode, int32_t *labels, float *dists, void *ws,
                                 size_t ws_bytes, uintptr_t stream)
{
    if (!X || n <= 0 || d <= 0 || !C || k <= 0 || !labels || !dists || !ws)
        return EACB_ERR_BAD_ARGUMENT;
    if (d > 32) return EACB_ERR_UNSUPPORTED;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    int *err = c.take<int>(1);
    int32_t *kk = c.take<int32_t>(1);
    int32_t *active = c.take<int32_t>(1);
    int *namb = c.take<int>(1);
    int32_t *amb = c.take<int32_t>(n);
    TcScratch tc = TcScratch::carve(c, n, d, 1, k);
    tc.err = err;
    if (c.overflow) return EACB_ERR_WORKSPACE;
    EACB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    k_set2<<<1, 1, 0, st>>>(kk, active, k, 1);
    EACB_CHECK_LAUNCH();
    if (label_mode == 1)
        return label_pass_tc(X, n, d, 1, C, kk, k, active, labels, dists, amb, namb, tc, st);
    return label_pass_f32(X, n, d, 1, C, kk, k, active, labels, dists, amb, namb, st);
}

extern "C" size_t eacb_kmeans_label_workspace_size(int32_t n, int32_t d, int32_t k)
{
    Carver c(nullptr, 0);
    c.take<int>(1);
    c.take<int32_t>(1);
    c.take<int32_t>(1);
    c.take<int>(1);
    c.take<int32_t>(n);
    TcScratch::carve(c, n, d, 1, k);
    return c.off;
}

// The label step with its arithmetic path fixed by name.
extern "C" int eacb_kmeans_label_fp32(const float *X, int32_t n, int32_t d, const float *C,
                                      int32_t k, int32_t *labels, float *dists, void *ws,
                                      size_t ws_bytes, uintptr_t stream)
{
    return eacb_kmeans_label(X, n, d, C, k, 0, labels, dists, ws, ws_bytes, stream);
}

extern "C" int eacb_kmeans_label_bf16tc(const float *X, int32_t n, int32_t d, const float *C,
                                        int32_t k, int32_t *labels, float *dists, void *ws,
                                        size_t ws_bytes, uintptr_t stream)
{
    return eacb_kmeans_label(X, n, d, C, k, 1, labels, dists, ws, ws_bytes, stream);
}

// Workspace of one centroid update (the ensemble's second half for P = 1).
struct CentWS {
    int *err;
    int32_t *kk, *active, *nempty;
    int32_t *cnt, *members, *mypos, *args, *sel, *oarg;
    float *key, *okey;
    int64_t *S;
    ScanScratch scan;
    int64_t ntiles;
    static CentWS carve(Carver &c, int32_t n, int32_t k)
    {
        CentWS w;
        w.err = c.take<int>(1);
        w.kk = c.take<int32_t>(1);
        w.active = c.take<int32_t>(1);
        w.nempty = c.take<int32_t>(1);
        w.ntiles = ((int64_t)n + kMLTile - 1) / kMLTile;
        const int64_t m = (int64_t)k * w.ntiles;
        w.cnt = c.take<int32_t>(m + 1);
        w.S = c.take<int64_t>(m + 1);
        w.members = c.take<int32_t>(n);
        w.mypos = c.take<int32_t>(n);
        w.args = c.take<int32_t>(n);
        w.sel = c.take<int32_t>(n);
        w.oarg = c.take<int32_t>(n);
        w.key = c.take<float>(n);
        w.okey = c.take<float>(n);
        w.scan = ScanScratch::carve(c, m + 1, w.err);
        return w;
    }
};

extern "C" size_t eacb_kmeans_centroids_workspace_size(int32_t n, int32_t d, int32_t k)
{
    Carver c(nullptr, 0);
    CentWS::carve(c, n, k);
    (void)d;
    return c.off;
}

extern "C" int eacb_kmeans_centroids(const float *X, int32_t n, int32_t d, const int32_t *labels,
                                     const float *dists, int32_t k, int32_t centroid_mode,
                                     float *C, void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (!X || n <= 0 || d <= 0 || !labels || !dists || k <= 0 || !C || !ws)
        return EACB_ERR_BAD_ARGUMENT;
    if (centroid_mode != 0 && centroid_mode != 1) return EACB_ERR_BAD_ARGUMENT;
    if (d > 32 || k > 8192) return EACB_ERR_UNSUPPORTED;
    cudaStream_t st = as_stream(stream);
    Carver c(ws, ws_bytes);
    CentWS w = CentWS::carve(c, n, k);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    const int64_t nt = w.ntiles;
    const int64_t m = (int64_t)k * nt;
    EACB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    EACB_CUDA(cudaMemsetAsync(w.nempty, 0, sizeof(int32_t), st));
    k_set2<<<1, 1, 0, st>>>(w.kk, w.active, k, 1);
    EACB_CHECK_LAUNCH();
    k_ml_count<<<(unsigned)nt, 256, k * sizeof(int), st>>>(labels, n, k, nt, w.cnt, w.err);
    EACB_CHECK_LAUNCH();
    int s = scan_launch<int32_t, int64_t>(w.cnt, w.S, m, 0, &w.S[m], w.scan, st);
    if (s) return s;
    const size_t place_smem = (size_t)k * (sizeof(int64_t) + sizeof(int32_t));
    if (place_smem > 48 * 1024) EACB_CUDA(allow_max_dyn_smem(k_ml_place));
    k_ml_place<<<(unsigned)nt, 32, place_smem, st>>>(labels, n, k, nt, w.S, w.members, w.mypos);
    EACB_CHECK_LAUNCH();
    const int G = 32 / d;
    const int warps = (k + G - 1) / G;
    dim3 cg((unsigned)((warps * 32 + 255) / 256), 1u);
    if (centroid_mode == 1)
        k_centroids<true><<<cg, 256, 0, st>>>(X, n, d, w.members, w.S, k, nt, w.kk, k, w.active, C,
                                              w.nempty);
    else
        k_centroids<false><<<cg, 256, 0, st>>>(X, n, d, w.members, w.S, k, nt, w.kk, k, w.active, C,
                                               w.nempty);
    EACB_CHECK_LAUNCH();
    // the quickselect permutes its keys: it works on a copy of the distances
    EACB_CUDA(cudaMemcpyAsync(w.key, dists, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    k_fill_empty<<<1, kFillThreads, 0, st>>>(X, n, d, w.key, w.S, k, nt, w.kk, k, w.active,
                                             w.nempty, w.args, w.sel, w.okey, w.oarg, C, w.err);
    EACB_CHECK_LAUNCH();
    int e = 0;
    EACB_CUDA(cudaMemcpyAsync(&e, w.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    EACB_CUDA(cudaStreamSynchronize(st));
    return dev_err_to_status(e);
}
