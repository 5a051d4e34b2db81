// Pieces shared by the float32 and the tensor-core k-means label passes.
#pragma once
#include "eacb_common.cuh"

namespace eacb {

// The reference's distance (MyML/MyML/cluster/KMeans.py:463-466): float32
// difference, float32 square, float64 running sum in dimension order.
template <int DM>
__device__ __forceinline__ double exact_dist(const float *x, const float *c, int D)
{
    double dist = 0.0;
#pragma unroll
    for (int d = 0; d < DM; ++d) {
        if (d < D) {
            const float diff = __fsub_rn(x[d], c[d]);
            dist = __dadd_rn(dist, (double)__fmul_rn(diff, diff));
        }
    }
    return dist;
}

static __global__ void k_set2(int32_t *a, int32_t *b, int32_t va, int32_t vb)
{
    *a = va;
    *b = vb;
}

// Scratch of the tensor-core label pass: operands in the UMMA layout.
struct TcScratch {
    int Kp;              // 3d rounded up to a multiple of 16
    int64_t n_pad;       // points rounded up to the 128-point tile
    int kt_max;          // 256-centroid tiles per partition
    uint8_t *A;          // point tiles (BF16 [hi, hi, lo])
    float *nx;           // |x - mu|^2
    uint8_t *B;          // centroid tiles (BF16 [hi, lo, hi])
    float *nc;           // |c - mu|^2 (+inf for padding)
    float *cmax2;        // per partition max |c - mu|^2
    float *mu;           // data mean
    double *part;        // column-sum partials
    int *err;
    bool points_ready;   // A / nx / mu depend on X only
    static TcScratch carve(Carver &c, int32_t n, int32_t D, int32_t P, int32_t kmax);
};

// Label pass on tcgen05 tensor cores (kmeans_tc.cu); same contract as the
// float32 pass: every point of every active partition gets the reference's
// label and distance.
int label_pass_tc(const float *X, int32_t n, int32_t D, int32_t P, const float *C,
                  const int32_t *kk, int32_t kmax, const int32_t *active, int32_t *labels,
                  float *dists, int32_t *amb, int *namb, TcScratch &s, cudaStream_t st);

}  // namespace eacb
