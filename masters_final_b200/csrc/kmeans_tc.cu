// K-means label pass on tcgen05 tensor cores.
//
// dist(x, c) = |x|^2 - 2 x.c + |c|^2 on data centred at its mean.  The dot
// products run as ONE BF16 GEMM with FP32 accumulation in tensor memory:
// each float32 operand is split into three BF16 parts (h + m + l, ~24
// significant bits) and the K dimension holds the six products that matter
// (see put_row), the large h*h group last.  The epilogue (8 warps, one point
// row per thread, half the columns per warp) reads the accumulator tile
// from TMEM with tcgen05.ld, forms the screened distance and keeps the best
// two per point.  A point whose runner-up lies within the proven error bound
// E (|x|^2 + max|c|^2) of its winner (E from the split, the accumulation
// order and the epilogue arithmetic, times 2) is re-labelled by the
// reference's exact loop; every other point gets its winner's exact
// reference distance.  Labels therefore equal the reference's
// (MyML/MyML/cluster/KMeans.py:453-490) for any input.
//
// Shapes: M = 128 points per CTA, N <= 128 centroids per MMA tile, K = 6d
// padded to a multiple of 16 (<= 192).  Operands are pre-arranged in global
// memory in the UMMA K-major no-swizzle core-matrix layout (8 rows x 16
// bytes per core matrix, LBO = 128 B along K, SBO = 128 B * K/8 along M/N),
// so each tile is one contiguous cp.async.bulk copy into shared memory.
// One thread issues the MMAs; TMEM holds one 128 x 128 FP32 accumulator per
// CTA (128 columns), four CTAs per SM share the 512 columns and overlap each
// other's MMA and epilogue.  Every wait is bounded and reports an error.
#include "kmeans_common.cuh"
#include <cuda_bf16.h>

#include <algorithm>

namespace eacb {

constexpr int kTM = 128;           // points per CTA tile
constexpr int kTN = 128;           // centroids per MMA tile
constexpr int kTThreads = 256;     // 8 warps: 4 TMEM lane quarters x 2 column halves
constexpr int kTColGroups = kTThreads / kTM;
constexpr int kTColsPer = kTN / kTColGroups;
constexpr int kTmemCols = kTN;
constexpr int kWaitLimit = 1 << 26;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// bounded wait on a phase; returns false when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase)
{
    for (int i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// UMMA shared-memory descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t umma_desc(const void *p, uint32_t lbo, uint32_t sbo)
{
    const uint64_t a = smem_addr(p);
    uint64_t d = 0;
    d |= (a >> 4) & 0x3FFFull;
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;          // descriptor version (sm_100)
    return d;                         // base offset 0, layout type 0 (no swizzle)
}

// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N)
{
    return (1u << 4)                       // D format F32
           | (1u << 7)                     // A format BF16
           | (1u << 10)                    // B format BF16
           | ((uint32_t)(N >> 3) << 17)    // N
           | ((uint32_t)(M >> 4) << 24);   // M
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
            tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// 32 accumulator columns of the warp's 32 TMEM lanes (one per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,"
        "%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__host__ __device__ __forceinline__ uint32_t sbo_b(int Kp) { return 128u * (uint32_t)(Kp >> 3); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// byte offset of element (row, k) inside a blocked K-major tile with Kp columns
__host__ __device__ __forceinline__ uint32_t core_off(int row, int k, int Kp)
{
    const int g = row >> 3, rr = row & 7, q = k >> 3, kk = k & 7;
    return (uint32_t)((((g * (Kp >> 3) + q) << 3) + rr) * 16 + kk * 2);
}

// ------------------------------------------------------------ preparation --
// data mean, float64 partials per block then a fixed-order final sum
__global__ void k_colsum(const float *X, int32_t n, int32_t D, double *part)
{
    __shared__ double s[32][33];
    const int d = threadIdx.x & 31, r = threadIdx.x >> 5;   // 256 threads: 8 row lanes
    double acc = 0.0;
    if (d < D)
        for (int64_t i = (int64_t)blockIdx.x * 8 + r; i < n; i += (int64_t)gridDim.x * 8)
            acc += (double)X[i * D + d];
    s[r][d] = acc;
    __syncthreads();
    if (r == 0 && d < D) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q) t += s[q][d];
        part[(int64_t)blockIdx.x * 32 + d] = t;
    }
}

__global__ void k_mean(const double *part, int nblocks, int32_t n, int32_t D, float *mu)
{
    const int d = threadIdx.x;
    if (d >= D) return;
    double t = 0.0;
    for (int b = 0; b < nblocks; ++b) t += part[(int64_t)b * 32 + d];
    mu[d] = (float)(t / (double)n);
}

// Rows of one operand, centred and split into three BF16 parts
// v = h + m + l (each part the BF16 rounding of the remainder, so |m| <=
// 2^-8 |v|, |l| <= 2^-16 |v| and the rest is below 2^-24 |v|).  The K axis
// holds six groups of D products, smallest first so that the large h*h
// products are accumulated last:
//   group      0    1    2    3    4    5
//   point      l    m    h    m    h    h
//   centroid   h    m    l    h    m    h
// Their sum is x.c up to the dropped l*m, m*l, l*l terms (< 3 * 2^-24 |x||c|).
__device__ __forceinline__ void put_row(const float *v, const float *mu, int D, int Kp, int row,
                                       uint8_t *tile, bool point_side, float &norm)
{
    constexpr int kPointPart[6] = {2, 1, 0, 1, 0, 0};      // 0 = h, 1 = m, 2 = l
    constexpr int kCentPart[6] = {0, 1, 2, 0, 1, 0};
    float nrm = 0.f;
    for (int k = 0; k < Kp; ++k) {
        __nv_bfloat16 b = __float2bfloat16_rn(0.f);
        if (k < 6 * D) {
            const int d = k % D, grp = k / D;
            const float xc = __fsub_rn(v[d], mu[d]);
            const __nv_bfloat16 h = __float2bfloat16_rn(xc);
            const float r1 = __fsub_rn(xc, __bfloat162float(h));
            const __nv_bfloat16 m = __float2bfloat16_rn(r1);
            const __nv_bfloat16 l = __float2bfloat16_rn(__fsub_rn(r1, __bfloat162float(m)));
            const int part = point_side ? kPointPart[grp] : kCentPart[grp];
            b = part == 0 ? h : (part == 1 ? m : l);
            if (grp == 0) nrm = fmaf(xc, xc, nrm);
        }
        *reinterpret_cast<__nv_bfloat16 *>(tile + core_off(row, k, Kp)) = b;
    }
    norm = nrm;
}

__global__ void k_prep_points(const float *X, int32_t n, int32_t D, int32_t Kp, const float *mu,
                              uint8_t *A, float *nx, int64_t n_pad)
{
    const int64_t tile_bytes = (int64_t)kTM * Kp * 2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_pad;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint8_t *tile = A + (i / kTM) * tile_bytes;
        float v[32];
        for (int d = 0; d < D; ++d) v[d] = i < n ? X[i * D + d] : mu[d];
        float nrm;
        put_row(v, mu, D, Kp, (int)(i % kTM), tile, true, nrm);
        nx[i] = nrm;
    }
}

__global__ void k_prep_centroids(const float *C, const int32_t *kk, int32_t kmax, int32_t P,
                                 int32_t D, int32_t Kp, int32_t kt_max, const float *mu,
                                 const int32_t *active, uint8_t *B, float *nc, float *cmax2)
{
    const int64_t tile_bytes = (int64_t)kTN * Kp * 2;
    const int64_t per_p = (int64_t)kt_max * kTN;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < (int64_t)P * per_p;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(e / per_p);
        if (!active[p]) continue;
        const int c = (int)(e % per_p);
        uint8_t *tile = B + ((int64_t)p * kt_max + c / kTN) * tile_bytes;
        float v[32];
        const bool real = c < kk[p];
        for (int d = 0; d < D; ++d) v[d] = real ? C[((int64_t)p * kmax + c) * D + d] : mu[d];
        float nrm;
        put_row(v, mu, D, Kp, c % kTN, tile, false, nrm);
        nc[e] = real ? nrm : __int_as_float(0x7f800000);
        if (real) atomicMax(reinterpret_cast<int *>(&cmax2[p]), __float_as_int(nrm));
    }
}

// ---------------------------------------------------------------- labels --
__global__ void __launch_bounds__(kTThreads, 4)
k_label_tc(const float *__restrict__ X, int32_t n, int32_t D, int32_t Kp, const float *__restrict__ C,
           const int32_t *__restrict__ kk, int32_t kmax, int32_t kt_max, int32_t P, int32_t ppc,
           const int32_t *__restrict__ active, const uint8_t *__restrict__ A,
           const float *__restrict__ nx, const uint8_t *__restrict__ B,
           const float *__restrict__ nc, const float *__restrict__ cmax2, float E, int nbuf,
           int32_t *labels, float *dists, int32_t *amb, int *namb, int *err)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t bar_a, bar_b[2], bar_mma;
    __shared__ uint32_t tmem_slot;
    __shared__ float s_b1[kTColGroups - 1][kTM], s_b2[kTColGroups - 1][kTM];
    __shared__ int s_i1[kTColGroups - 1][kTM];
    __shared__ int s_fail;
    const uint32_t a_bytes = (uint32_t)kTM * Kp * 2, b_bytes = (uint32_t)kTN * Kp * 2;
    uint8_t *sA = smem;
    // two centroid-tile buffers when they fit (prefetch overlaps the MMA),
    // else one (prefetch overlaps the epilogue)
    uint8_t *sB[2] = {smem + a_bytes, nbuf == 2 ? smem + a_bytes + b_bytes : smem + a_bytes};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the MMA issuer: a thread of the last warp, which has no per-partition
    // tail, so the next MMA starts while the first warps finish a partition
    const bool issuer = threadIdx.x == kTThreads - 32;
    const int64_t tile0 = blockIdx.x;
    const uint8_t *Ap = A + tile0 * a_bytes;
    // the tiles in order: every centroid tile of every active partition of
    // this CTA's share [pb, pe) of the partitions
    const int pb = blockIdx.y * ppc, pe = min(P, pb + ppc);
    auto ntiles = [&](int q) -> int { return active[q] ? (kk[q] + kTN - 1) / kTN : 0; };
    auto first_from = [&](int q) -> int {
        while (q < pe && ntiles(q) == 0) ++q;
        return q < pe ? q : P;
    };
    auto btile = [&](int q, int t) -> const uint8_t * {
        return B + ((int64_t)q * kt_max + t) * b_bytes;
    };

    int p = first_from(pb);
    if (p >= P) return;                          // uniform: nothing to label
    if (threadIdx.x == 0) {
        s_fail = 0;
        mbar_init(&bar_a, 1);
        mbar_init(&bar_b[0], 1);
        mbar_init(&bar_b[1], 1);
        mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_slot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (issuer) {
        mbar_expect_tx(&bar_a, a_bytes);
        bulk_g2s(sA, Ap, a_bytes, &bar_a);
        mbar_expect_tx(&bar_b[0], b_bytes);
        bulk_g2s(sB[0], btile(p, 0), b_bytes, &bar_b[0]);
    }
    // epilogue ownership: row = 32*(warp%4) + lane (the TMEM lanes warp w may
    // read), columns [64*(warp/4), +64) of the 128-column tile
    const int row = 32 * (warp & 3) + lane;
    const int cgrp = warp >> 2, colh = kTColsPer * cgrp;
    const int64_t i = tile0 * kTM + row;
    const float xn = (i < n) ? nx[i] : 0.f;
    float b1 = __int_as_float(0x7f800000), b2 = b1;
    int i1 = 0;
    const uint32_t lbo = 128, sbo = 128u * (uint32_t)(Kp >> 3);
    uint32_t ph_b[2] = {0, 0}, ph_mma = 0;
    int pend = -1;                               // buffer with a copy in flight (issuer)
    int mma_ph = -1;                             // phase of an MMA not yet seen complete
    bool ok = true;
    int t = 0, tiles = ntiles(p);
    for (int64_t j = 0; p < P; ++j) {
        // the tile after (p, t): its copy is issued while this one is used
        int pn = p, tn = t + 1;
        if (tn == tiles) {
            pn = first_from(p + 1);
            tn = 0;
        }
        const int buf = nbuf == 2 ? (int)(j & 1) : 0;
        const int nvalid = min(kTN, kk[p] - t * kTN);
        const int N = (nvalid + 15) & ~15;
        if (issuer) {
            bool got = (j == 0 ? mbar_wait(&bar_a, 0) : true) && mbar_wait(&bar_b[buf], ph_b[buf]);
            if (!got) {
                set_err(err, DEV_SPIN_LIMIT);
                s_fail = 1;
            } else {
                pend = -1;
                tc_fence_after();
                const uint32_t idesc = umma_idesc(kTM, N);
                for (int s = 0; s < (Kp >> 4); ++s) {
                    const uint64_t ad = umma_desc(sA + s * 256, lbo, sbo);
                    const uint64_t bd = umma_desc(sB[buf] + s * 256, lbo, sbo_b(Kp));
                    mma_bf16(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
                }
                mma_commit(&bar_mma);
                mma_ph = (int)ph_mma;
                if (nbuf == 2 && pn < P) {
                    // the other buffer's last reader (the previous MMA) completed
                    mbar_expect_tx(&bar_b[buf ^ 1], b_bytes);
                    bulk_g2s(sB[buf ^ 1], btile(pn, tn), b_bytes, &bar_b[buf ^ 1]);
                    pend = buf ^ 1;
                }
            }
        }
        ph_b[buf] ^= 1;
        __syncthreads();
        if (s_fail) { ok = false; break; }
        if (!mbar_wait(&bar_mma, ph_mma)) {
            set_err(err, DEV_SPIN_LIMIT);
            s_fail = 1;
        } else if (issuer) {
            mma_ph = -1;
            if (nbuf == 1 && pn < P) {
                // single buffer: this tile's MMA has finished reading it
                mbar_expect_tx(&bar_b[0], b_bytes);
                bulk_g2s(sB[0], btile(pn, tn), b_bytes, &bar_b[0]);
                pend = 0;
            }
        }
        ph_mma ^= 1;
        tc_fence_after();
        const float *ncp = nc + ((int64_t)p * kt_max + t) * kTN;
        const int c_lo = colh, c_hi = min(colh + kTColsPer, nvalid);
        // 32 columns at a time (a 64-column share; past the tile's valid
        // columns the norms are +inf, so those columns never win)
        for (int c0 = c_lo; c0 < c_hi; c0 += 32) {
            float v[32], ncv[32];
            tmem_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)c0, v);
            // the 32 centroid norms, the same for every lane: eight 16-byte loads
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 f = __ldg(reinterpret_cast<const float4 *>(ncp + c0) + q);
                ncv[4 * q] = f.x;
                ncv[4 * q + 1] = f.y;
                ncv[4 * q + 2] = f.z;
                ncv[4 * q + 3] = f.w;
            }
            // the screened distance less the row's |x|^2 (the same for every
            // column, so the order and the gaps are those of the distance):
            // one rounding, where adding |x|^2 first would take two
            const int cb = t * kTN + c0;
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
                const float sv = fmaf(-2.f, v[jj], ncv[jj]);      // ncp[c] = +inf past K
                i1 = sv < b1 ? cb + jj : i1;
                b2 = fminf(b2, fmaxf(b1, sv));
                b1 = fminf(b1, sv);
            }
        }
        tc_fence_before();
        __syncthreads();                         // the accumulator is free again
        if (s_fail) { ok = false; break; }
        if (t + 1 == tiles) {
            // the partition is done: merge the column groups of each row, in
            // column order
            if (cgrp > 0) {
                s_b1[cgrp - 1][row] = b1;
                s_b2[cgrp - 1][row] = b2;
                s_i1[cgrp - 1][row] = i1;
            }
            __syncthreads();
            if (cgrp == 0 && i < n) {
                // the lower index wins equal screened values; equal values are
                // a near tie anyway and go to the exact re-check
                float w1 = b1, w2 = b2;
                int wi = i1;
#pragma unroll
                for (int q = 0; q < kTColGroups - 1; ++q) {
                    const float o1 = s_b1[q][row], o2 = s_b2[q][row];
                    if (o1 < w1) {
                        w2 = fminf(w1, o2);
                        w1 = o1;
                        wi = s_i1[q][row];
                    } else {
                        w2 = fminf(w2, o1);
                    }
                }
                // Column c's screened distance is within e(c) = E/2 (|x|^2 +
                // |c|^2) of the exact one.  A column c* that the exact
                // arithmetic could rank at or before the winner w has
                // |x - c*|^2 <= |x - c_w|^2 <= w1 + |x|^2 + e(w), so |c*| <=
                // |x| + sqrt(w1 + |x|^2 + e(w)) (capped by the largest norm).
                // The winner is certain when the runner-up is more than e(w) +
                // e(c*) above it (the bound taken 1% wide for the rounding of
                // this arithmetic).
                const float ew = 0.5f * E * (xn + nc[((int64_t)p * kt_max) * kTN + wi]);
                const float rc = sqrtf(xn) + sqrtf(fmaxf(0.f, w1 + xn + ew));
                const float cstar2 = fminf(rc * rc, cmax2[p]);
                const float bound = 1.01f * (ew + 0.5f * E * (xn + cstar2));
                const int64_t o = (int64_t)p * n + i;
                if (w2 - w1 > bound) {
                    float xv[32];
                    for (int d = 0; d < D; ++d) xv[d] = X[i * D + d];
                    labels[o] = wi;
                    dists[o] = (float)exact_dist<32>(xv, C + ((int64_t)p * kmax + wi) * D, D);
                } else {
                    amb[atomicAdd(namb, 1)] = (int32_t)o;
                }
            }
            b1 = b2 = __int_as_float(0x7f800000);
            i1 = 0;
        }
        p = pn;
        t = tn;
        if (tn == 0 && pn < P) tiles = ntiles(pn);
    }
    if (!ok && issuer) {
        // leave no copy or MMA writing into this CTA's memory (bounded waits)
        if (pend >= 0) mbar_wait(&bar_b[pend], ph_b[pend]);
        if (mma_ph >= 0) mbar_wait(&bar_mma, (uint32_t)mma_ph);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemCols));
}

__device__ __forceinline__ void exact_label_point(const float *__restrict__ X, int32_t n, int32_t D,
                                                  const float *__restrict__ C,
                                                  const int32_t *__restrict__ kk, int32_t kmax,
                                                  int64_t o, int32_t *labels, float *dists)
{
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

// if a tile gave up waiting, relabel every active point with the exact loop
// (never expected; keeps the result correct and the error reported)
__global__ void k_exact_all(const float *__restrict__ X, int32_t n, int32_t D,
                            const float *__restrict__ C, const int32_t *__restrict__ kk,
                            int32_t kmax, int32_t P, const int32_t *active, const int *err,
                            int32_t *labels, float *dists)
{
    if (*err == 0) return;
    for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < (int64_t)P * n;
         o += (int64_t)gridDim.x * blockDim.x)
        if (active[o / n]) exact_label_point(X, n, D, C, kk, kmax, o, labels, dists);
}

// The reference's distance sum_d (double) fl(fl(x_d - c_d)^2) and the FP32
// sum of the same squares by fused multiply-adds differ by at most (D + 2)
// 2^-24 of either (the squares round once, the chain once per term; the
// double sum adds < D 2^-53), plus subnormal rounding far below 1e-38.  So
// every centroid that can hold the reference's minimum -- and every one tied
// with it -- has an FP32 sum within (1 + 4 (D + 2) 2^-24) of the smallest
// FP32 sum, with a factor 2 to spare.
// a centroid row into registers: four floats at a time when D is a
// multiple of four (rows then start on 16-byte boundaries)
template <int DM, bool VEC>
__device__ __forceinline__ void load_row(const float *c, int D, float (&v)[DM])
{
    if (VEC) {
#pragma unroll
        for (int d = 0; d < DM; d += 4) {
            const float4 f = __ldg(reinterpret_cast<const float4 *>(c + d));
            v[d] = f.x;
            v[d + 1] = f.y;
            v[d + 2] = f.z;
            v[d + 3] = f.w;
        }
    } else {
#pragma unroll
        for (int d = 0; d < DM; ++d) v[d] = d < D ? __ldg(c + d) : 0.f;
    }
}

template <int DM>
__device__ __forceinline__ float screen_dist(const float (&x)[DM], const float (&c)[DM], int D)
{
    float acc = 0.f;
#pragma unroll
    for (int d = 0; d < DM; ++d)
        if (d < D) {
            const float diff = __fsub_rn(x[d], c[d]);
            acc = __fmaf_rn(diff, diff, acc);
        }
    return acc;
}

template <int DM>
__device__ __forceinline__ double exact_dist_reg(const float (&x)[DM], const float (&c)[DM], int D)
{
    double dist = 0.0;
#pragma unroll
    for (int d = 0; d < DM; ++d)
        if (d < D) {
            const float diff = __fsub_rn(x[d], c[d]);
            dist = __dadd_rn(dist, (double)__fmul_rn(diff, diff));
        }
    return dist;
}

constexpr int kExactThreads = 256;
constexpr int kExactCacheK = 2048;     // FP32 sums kept in shared memory up to this k

// One warp per ambiguous point, lane l over centroids l, l + 32, ...: an FP32
// pass finds the smallest sum (keeping each sum in shared memory when k is at
// most kExactCacheK), a second pass evaluates the reference's arithmetic only
// for the centroids within the bound above, and the warp keeps the smallest
// distance, the smallest index among equal ones (the reference loop's first
// minimum).
template <int DM, bool VEC>
__global__ void __launch_bounds__(kExactThreads)
k_label_exact_tc(const float *__restrict__ X, int32_t n, int32_t D, const float *__restrict__ C,
                 const int32_t *__restrict__ kk, int32_t kmax, int32_t P,
                 const int32_t *__restrict__ amb, const int *__restrict__ namb,
                 const int *__restrict__ err, int32_t *labels, float *dists)
{
    extern __shared__ float s_sum[];
    if (*err != 0) return;                      // k_exact_all did every point
    const int64_t cap = (int64_t)P * n;
    const int m = (int)min((int64_t)*namb, cap);
    const float grow = 1.f + 4.f * (float)(D + 2) * 5.9604645e-8f;     // 2^-24
    const bool cached = kmax <= kExactCacheK;
    float *mine = s_sum + (threadIdx.x >> 5) * (cached ? kmax : 0);
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < m; t += nw) {
        const int64_t o = amb[t];
        const int64_t p = o / n, i = o - p * n;
        const int K = kk[p];
        float xv[DM], cv[DM];
        load_row<DM, VEC>(X + i * D, D, xv);
        const float *Cp = C + p * kmax * D;
        float mn = __int_as_float(0x7f800000);
        for (int k = lane; k < K; k += 32) {
            load_row<DM, VEC>(Cp + (int64_t)k * D, D, cv);
            const float d32 = screen_dist<DM>(xv, cv, D);
            if (cached) mine[k] = d32;
            mn = fminf(mn, d32);
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, off));
        const float thr = __fadd_ru(__fmul_ru(mn, grow), 1e-38f);
        double best = 0.0;
        int bl = 0x7fffffff;
        for (int k = lane; k < K; k += 32) {
            float d32;
            if (cached) {
                d32 = mine[k];
            } else {
                load_row<DM, VEC>(Cp + (int64_t)k * D, D, cv);
                d32 = screen_dist<DM>(xv, cv, D);
            }
            if (d32 > thr) continue;
            load_row<DM, VEC>(Cp + (int64_t)k * D, D, cv);
            const double dist = exact_dist_reg<DM>(xv, cv, D);
            if (bl == 0x7fffffff || dist < best) {
                best = dist;
                bl = k;
            }
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, off);
            const int ok = __shfl_xor_sync(0xffffffffu, bl, off);
            if (ok != 0x7fffffff && (bl == 0x7fffffff || ob < best || (!(best < ob) && ok < bl))) {
                best = ob;
                bl = ok;
            }
        }
        if (lane == 0) {
            labels[o] = bl;
            dists[o] = (float)best;
        }
        __syncwarp();                           // the sums are rewritten by the next point
    }
}

size_t tc_scratch_bytes(int32_t n, int32_t D, int32_t P, int32_t kmax)
{
    Carver c(nullptr, 0);
    TcScratch::carve(c, n, D, P, kmax);
    return c.off;
}

TcScratch TcScratch::carve(Carver &c, int32_t n, int32_t D, int32_t P, int32_t kmax)
{
    TcScratch s;
    s.Kp = ((6 * D + 15) / 16) * 16;
    s.n_pad = ((int64_t)n + kTM - 1) / kTM * kTM;
    s.kt_max = (kmax + kTN - 1) / kTN;
    s.A = c.take<uint8_t>((size_t)s.n_pad * s.Kp * 2);
    s.nx = c.take<float>((size_t)s.n_pad);
    s.B = c.take<uint8_t>((size_t)P * s.kt_max * kTN * s.Kp * 2);
    s.nc = c.take<float>((size_t)P * s.kt_max * kTN);
    s.cmax2 = c.take<float>((size_t)P);
    s.mu = c.take<float>(32);
    s.part = c.take<double>((size_t)32 * 296);
    s.err = c.take<int>(1);
    s.points_ready = false;
    return s;
}

int label_pass_tc(const float *X, int32_t n, int32_t D, int32_t P, const float *C,
                  const int32_t *kk, int32_t kmax, const int32_t *active, int32_t *labels,
                  float *dists, int32_t *amb, int *namb, TcScratch &s, cudaStream_t st)
{
    if (!s.points_ready) {
        k_colsum<<<296, 256, 0, st>>>(X, n, D, s.part);
        EACB_CHECK_LAUNCH();
        k_mean<<<1, 32, 0, st>>>(s.part, 296, n, D, s.mu);
        EACB_CHECK_LAUNCH();
        k_prep_points<<<grid_for(s.n_pad, 128), 128, 0, st>>>(X, n, D, s.Kp, s.mu, s.A, s.nx,
                                                              s.n_pad);
        EACB_CHECK_LAUNCH();
        s.points_ready = true;
    }
    EACB_CUDA(cudaMemsetAsync(s.cmax2, 0, sizeof(float) * P, st));
    EACB_CUDA(cudaMemsetAsync(namb, 0, sizeof(int), st));
    k_prep_centroids<<<grid_for((int64_t)P * s.kt_max * kTN, 128), 128, 0, st>>>(
        C, kk, kmax, P, D, s.Kp, s.kt_max, s.mu, active, s.B, s.nc, s.cmax2);
    EACB_CHECK_LAUNCH();
    // Error model of the screened distance, doubled for margin.  The dot
    // product: the three-way split drops < 3 * 2^-24 |x||c|; the MMA adds
    // the h*h group last, so its accumulation error is at most
    // (16 ceil(D/16) + 3) 2^-23 of sum|x_d c_d| (<= |x||c|), the earlier,
    // 2^8-times smaller groups add less than one more 2^-23.  Norms and the
    // epilogue: (D + 6) 2^-24 of |x|^2 + |c|^2.  With 2|x||c| <= |x|^2 +
    // |c|^2 the screened distance is within E (|x|^2 + max|c|^2) / 2.
    const double dot_err = 3.0 * ldexp(1.0, -24) +
                           (16.0 * ((D + 15) / 16) + 4.0) * ldexp(1.0, -23);
    const float E = 2.f * (float)(dot_err + (D + 6) * ldexp(1.0, -24));
    const size_t a_bytes = (size_t)kTM * s.Kp * 2, b_bytes = (size_t)kTN * s.Kp * 2;
    // CTAs per SM (each holds 128 TMEM columns): four by default, fewer when
    // their operand tiles do not fit four to an SM
    int ctas = (int)tune_get(TUNE_TC_CTAS_PER_SM, D, n, 4);
    ctas = ctas >= 4 ? 4 : (ctas >= 2 ? 2 : 1);
    while (ctas > 1 && a_bytes + b_bytes > (size_t)(220 / ctas) * 1024) ctas /= 2;
    const size_t cap_bytes = (size_t)(220 / ctas) * 1024;
    int nbuf = (a_bytes + 2 * b_bytes <= cap_bytes) ? 2 : 1;
    nbuf = (int)std::min<int64_t>(nbuf, std::max<int64_t>(1, tune_get(TUNE_TC_BUFFERS, D, n, nbuf)));
    const size_t smem = a_bytes + nbuf * b_bytes;
    // a floor on the request so that no more CTAs than asked share an SM
    const size_t floor_bytes = (size_t)(228 / (ctas + 1) + 2) * 1024;
    const size_t smem_req = smem < floor_bytes ? floor_bytes : smem;
    EACB_CUDA(allow_max_dyn_smem(k_label_tc));
    // one CTA per 128-point tile and share of the partitions: all partitions
    // (the tile's operands load once) unless that leaves fewer than two
    // CTAs per SM slot in flight
    const int64_t ptiles = s.n_pad / kTM;
    const int64_t want = 2 * 148 * ctas;
    const int groups = (int)std::min<int64_t>(P, std::max<int64_t>(1, (want + ptiles - 1) / ptiles));
    const int ppc = (P + groups - 1) / groups;
    dim3 grid((unsigned)ptiles, (unsigned)((P + ppc - 1) / ppc));
    ProfScope ps(PROF_KMEANS, st);
    k_label_tc<<<grid, kTThreads, smem_req, st>>>(X, n, D, s.Kp, C, kk, kmax, s.kt_max, P, ppc, active,
                                                  s.A, s.nx, s.B, s.nc, s.cmax2, E, nbuf, labels, dists,
                                                  amb, namb, s.err);
    EACB_CHECK_LAUNCH();
    ps.done(0.0);
    k_exact_all<<<296, 256, 0, st>>>(X, n, D, C, kk, kmax, P, active, s.err, labels, dists);
    EACB_CHECK_LAUNCH();
    const size_t esmem = kmax <= kExactCacheK
                             ? (size_t)(kExactThreads / 32) * kmax * sizeof(float) : 0;
    int es = EACB_OK;
    auto exact = [&](auto kern) {
        if (esmem > 48 * 1024 && cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)esmem) != cudaSuccess)
            es = EACB_ERR_CUDA;
        else
            kern<<<148 * 8, kExactThreads, esmem, st>>>(X, n, D, C, kk, kmax, P, amb, namb, s.err,
                                                        labels, dists);
    };
    // 16-byte row loads when every row is exactly DM floats on a 16-byte boundary
    const bool al = ((uintptr_t)X % 16 == 0) && ((uintptr_t)C % 16 == 0);
    if (D == 4 && al) exact(k_label_exact_tc<4, true>);
    else if (D <= 4) exact(k_label_exact_tc<4, false>);
    else if (D == 8 && al) exact(k_label_exact_tc<8, true>);
    else if (D <= 8) exact(k_label_exact_tc<8, false>);
    else if (D == 16 && al) exact(k_label_exact_tc<16, true>);
    else if (D <= 16) exact(k_label_exact_tc<16, false>);
    else if (D == 32 && al) exact(k_label_exact_tc<32, true>);
    else exact(k_label_exact_tc<32, false>);
    if (es) return es;
    EACB_CHECK_LAUNCH();
    return EACB_OK;
}

}  // namespace eacb
