/*
 * eac_oracle.c -- CPU restatement of the reference EAC hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is compiled into
 * oracle/liboracle.so and loaded by tests/, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline leg.  The product path (masters_final_b200) never
 * links or calls it.
 *
 * Every function restates, in plain C, the algorithm of a reference function
 * (diogo-aos/masters_final, Python 2 + Numba).  Citations are file:line within
 * that project.  The restatements keep the reference's arithmetic (integer
 * widths, FP32/FP64 mix, comparison direction, processing order) because the
 * tests compare the CUDA path against these results bit for bit.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_OK 0
#define ORC_ERR_ARG -1
#define ORC_ERR_FIRST_OVERFLOW -7
#define ORC_ERR_ALLOC -9

/* ------------------------------------------------------------------------ */
/* Exclusive scans.  MyML/MyML/utils/scan.py:42-53 (exprefixsumNumba): the   */
/* carry is a 64-bit Numba integer, each store truncates to the output type, */
/* the return value is the full 64-bit total.                                */
/* ------------------------------------------------------------------------ */
int64_t orc_exscan_i32(const int32_t *in, int32_t *out, int64_t n, int64_t init)
{
    int64_t carry = init;
    for (int64_t i = 0; i < n; ++i) {
        int64_t v = in[i];           /* read before write: in may alias out */
        out[i] = (int32_t)(uint32_t)(uint64_t)carry;
        carry += v;
    }
    return carry;
}

int64_t orc_exscan_i32_to_i64(const int32_t *in, int64_t *out, int64_t n, int64_t init)
{
    int64_t carry = init;
    for (int64_t i = 0; i < n; ++i) {
        int64_t v = in[i];
        out[i] = carry;
        carry += v;
    }
    return carry;
}

int64_t orc_exscan_i64(const int64_t *in, int64_t *out, int64_t n, int64_t init)
{
    int64_t carry = init;
    for (int64_t i = 0; i < n; ++i) {
        int64_t v = in[i];
        out[i] = carry;
        carry += v;
    }
    return carry;
}

/* ------------------------------------------------------------------------ */
/* Boruvka on a CSR graph, the reference's sequential variant.               */
/* MyML/MyML/graph/mst.py:143-232 (boruvka_minho_seq) with its steps         */
/* findMinEdgeNumba :250-279, removeMirroredNumba :283-305,                  */
/* addEdgesToMSTNumba :309-317, initColorsNumba :321-330,                    */
/* propagateColorsNumba :334-351, buildFlag :236-243,                        */
/* countNewEdgesNumba :355-372, assignInsertNumba :379-407; and              */
/* MyML/MyML/graph/connected_components.py:46-137 (connected_comps_seq) with */
/* update_labels_single_pass :163-173.                                       */
/*                                                                           */
/* Weights are passed as double (exact for every integer type up to 32 bits */
/* and for float32), so the comparisons equal the reference's.               */
/* mst_out (size V-1, may be NULL) receives input edge ids in the order the  */
/* reference appends them; labels (size V, may be NULL) receives the         */
/* connected-component labels of connected_comps_seq.                       */
/* Returns the number of MST edges, or a negative error.                     */
/* ------------------------------------------------------------------------ */
int64_t orc_boruvka_seq(int32_t V, int64_t E, const int32_t *dest_in,
                        const double *w_in, const int32_t *first_in,
                        const int32_t *deg_in, int32_t *mst_out,
                        int32_t *labels)
{
    if (V <= 0) return ORC_ERR_ARG;
    int32_t nv = V;
    int64_t ne = E;
    int32_t *dest = malloc(sizeof(int32_t) * (ne > 0 ? ne : 1));
    double *w = malloc(sizeof(double) * (ne > 0 ? ne : 1));
    int32_t *eid = malloc(sizeof(int32_t) * (ne > 0 ? ne : 1));
    int32_t *first = malloc(sizeof(int32_t) * nv);
    int32_t *deg = malloc(sizeof(int32_t) * nv);
    int32_t *minedge = malloc(sizeof(int32_t) * nv);
    int32_t *color = malloc(sizeof(int32_t) * nv);
    int32_t *newid = malloc(sizeof(int32_t) * nv);
    int32_t *lab = malloc(sizeof(int32_t) * nv);
    if (!dest || !w || !eid || !first || !deg || !minedge || !color || !newid || !lab)
        return ORC_ERR_ALLOC;
    memcpy(dest, dest_in, sizeof(int32_t) * ne);
    memcpy(w, w_in, sizeof(double) * ne);
    for (int64_t e = 0; e < ne; ++e) eid[e] = (int32_t)e;
    memcpy(first, first_in, sizeof(int32_t) * nv);
    memcpy(deg, deg_in, sizeof(int32_t) * nv);

    int64_t n_mst = 0;
    int first_round = 1;
    for (;;) {
        /* minimum out-edge of each vertex by (weight, destination id); the
         * first edge in segment order wins among equal pairs */
        for (int32_t v = 0; v < nv; ++v) {
            if (deg[v] == 0) { minedge[v] = -1; continue; }
            int64_t s = first[v], best = s;
            for (int64_t e = s + 1; e < s + deg[v]; ++e) {
                if (w[e] < w[best] || (w[e] == w[best] && dest[e] < dest[best]))
                    best = e;
            }
            minedge[v] = (int32_t)best;
        }
        /* a 2-cycle keeps the edge of its larger endpoint */
        for (int32_t v = 0; v < nv; ++v) {
            int32_t me = minedge[v];
            if (me < 0) continue;
            int32_t succ = dest[me];
            int32_t se = minedge[succ];
            if (se < 0) continue;
            if (dest[se] == v && v < succ) minedge[v] = -1;
        }
        for (int32_t v = 0; v < nv; ++v)
            if (minedge[v] >= 0) {
                if (mst_out) mst_out[n_mst] = eid[minedge[v]];
                n_mst++;
            }
        for (int32_t v = 0; v < nv; ++v)
            color[v] = minedge[v] >= 0 ? dest[minedge[v]] : v;
        /* pointer jumping until every vertex holds its root */
        for (int changed = 1; changed;) {
            changed = 0;
            for (int32_t v = 0; v < nv; ++v) {
                int32_t c = color[v];
                if (c != v) {
                    int32_t nc = color[c];
                    if (nc != c) changed = 1;
                    color[v] = nc;
                }
            }
        }
        int32_t nnew = 0;
        for (int32_t v = 0; v < nv; ++v) {
            newid[v] = nnew;
            nnew += (color[v] == v);
        }
        if (first_round) {
            memcpy(lab, color, sizeof(int32_t) * nv);
            first_round = 0;
        }
        for (int64_t x = 0; x < V; ++x) lab[x] = newid[color[lab[x]]];
        if (nnew == 1) break;

        /* contracted graph: inter-supervertex edges, stable order */
        int32_t *ndeg = calloc(nnew, sizeof(int32_t));
        for (int32_t v = 0; v < nv; ++v) {
            int32_t cv = color[v];
            for (int64_t e = first[v]; e < first[v] + deg[v]; ++e)
                if (color[dest[e]] != cv) ndeg[newid[cv]]++;
        }
        int32_t *nfirst = malloc(sizeof(int32_t) * nnew);
        int64_t tot = 0;
        for (int32_t s = 0; s < nnew; ++s) { nfirst[s] = (int32_t)tot; tot += ndeg[s]; }
        if (tot == 0) { free(ndeg); free(nfirst); break; }
        int32_t *ndest = malloc(sizeof(int32_t) * tot);
        double *nw = malloc(sizeof(double) * tot);
        int32_t *neid = malloc(sizeof(int32_t) * tot);
        int32_t *top = malloc(sizeof(int32_t) * nnew);
        memcpy(top, nfirst, sizeof(int32_t) * nnew);
        for (int32_t v = 0; v < nv; ++v) {
            int32_t cv = color[v];
            for (int64_t e = first[v]; e < first[v] + deg[v]; ++e) {
                int32_t cd = color[dest[e]];
                if (cd != cv) {
                    int32_t s = newid[cv];
                    int32_t p = top[s]++;
                    ndest[p] = newid[cd];
                    nw[p] = w[e];
                    neid[p] = eid[e];
                }
            }
        }
        free(dest); free(w); free(eid); free(first); free(deg); free(top);
        dest = ndest; w = nw; eid = neid; first = nfirst; deg = ndeg;
        nv = nnew; ne = tot;
    }
    if (labels) memcpy(labels, lab, sizeof(int32_t) * V);
    free(dest); free(w); free(eid); free(first); free(deg);
    free(minedge); free(color); free(newid); free(lab);
    return n_mst;
}

/* ------------------------------------------------------------------------ */
/* Kruskal over undirected edges (a < b) with the strict total order         */
/* (w, a, b).  The reference's Kruskal (scipy_numba/scipy_numba/sparse/      */
/* csgraph/_min_spanning_tree.py:21-175) orders edges with an unstable       */
/* argsort; fixing the tie order makes the spanning forest unique, so the    */
/* GPU edge set can be compared exactly.  Keys are given pre-packed          */
/* (weight-order bits above a, above b) by the caller; in_forest[e] is set   */
/* to 1 for each chosen edge.  Returns the number of chosen edges.           */
/* ------------------------------------------------------------------------ */
static int cmp_u64(const void *x, const void *y)
{
    uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    return a < b ? -1 : a > b;
}

static int32_t uf_find(int32_t *par, int32_t x)
{
    while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; }
    return x;
}

int64_t orc_kruskal_keys(int32_t V, int64_t M, const uint64_t *keys,
                         const int32_t *a, const int32_t *b, uint8_t *in_forest)
{
    /* sort edge indices by key: pack (key, index) pairs */
    uint64_t *order = malloc(sizeof(uint64_t) * 2 * (M > 0 ? M : 1));
    if (!order) return ORC_ERR_ALLOC;
    for (int64_t e = 0; e < M; ++e) { order[2 * e] = keys[e]; order[2 * e + 1] = (uint64_t)e; }
    qsort(order, M, 2 * sizeof(uint64_t), cmp_u64);
    int32_t *par = malloc(sizeof(int32_t) * V);
    for (int32_t v = 0; v < V; ++v) par[v] = v;
    if (M > 0) memset(in_forest, 0, (size_t)M);
    int64_t cnt = 0;
    for (int64_t i = 0; i < M && cnt < V - 1; ++i) {
        int64_t e = (int64_t)order[2 * i + 1];
        int32_t ra = uf_find(par, a[e]), rb = uf_find(par, b[e]);
        if (ra != rb) { par[ra] = rb; in_forest[e] = 1; cnt++; }
    }
    free(order); free(par);
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* Sparse co-association build, condensed (upper triangle), with the         */
/* reference's per-row capacity and discard rule.                            */
/* MyML/MyML/EAC/sparse.py:154-166 (update_ensemble),                        */
/* :446-465 (update_cluster_fp_condensed, first partition: no capacity       */
/* check), :957-1040 (update_cluster_sorted_surgical_condensed: existing     */
/* associations are incremented, new ones are inserted in sorted position    */
/* while the row holds fewer than its capacity, later ones are discarded),   */
/* :1070-1099 (binary_search_interval), :212-226 + :336-349 (condense).      */
/*                                                                           */
/* Input: the ensemble as a label matrix labels[p*n + i] (cluster id of      */
/* point i in partition p, -1 = in no cluster); cluster ids of a partition   */
/* need not be contiguous.  order[q] = partition processed q-th (the caller  */
/* puts argmin(#clusters) first, then the rest by index).  cap_indptr (n+1,  */
/* int64) = the reference's capacity layout (indptr_linear).                 */
/* Output: indptr (n+1, int64), indices (int32) and counts (uint8) of the    */
/* condensed CSR (rows sorted by column), nnz and nnz_discarded.  Sizes of   */
/* indices/counts must be >= cap_indptr[n].                                  */
/* Returns 0, or ORC_ERR_FIRST_OVERFLOW when a first-partition row tail      */
/* exceeds that row's capacity (the reference then writes past the row).    */
/* ------------------------------------------------------------------------ */
typedef struct { int32_t lab; int32_t idx; } li_pair;

static int cmp_li(const void *x, const void *y)
{
    const li_pair *a = x, *b = y;
    if (a->lab != b->lab) return a->lab < b->lab ? -1 : 1;
    return a->idx < b->idx ? -1 : a->idx > b->idx;
}

int orc_coassoc_build(int32_t n, int32_t P, const int32_t *labels,
                      const int32_t *order, const int64_t *cap_indptr,
                      int64_t *indptr, int32_t *indices, uint8_t *counts,
                      int64_t *nnz_out, int64_t *discarded_out)
{
    int64_t cap_total = cap_indptr[n];
    int32_t *ind = malloc(sizeof(int32_t) * (cap_total > 0 ? cap_total : 1));
    uint8_t *dat = malloc(cap_total > 0 ? cap_total : 1);
    int32_t *degree = calloc(n + 1, sizeof(int32_t));
    li_pair *pairs = malloc(sizeof(li_pair) * n);
    int32_t *newj = malloc(sizeof(int32_t) * (n > 0 ? n : 1));
    int64_t *newpos = malloc(sizeof(int64_t) * (n > 0 ? n : 1));
    if (!ind || !dat || !degree || !pairs || !newj || !newpos) return ORC_ERR_ALLOC;
    int64_t nnz = 0, disc = 0;
    int status = ORC_OK;

    for (int32_t q = 0; q < P; ++q) {
        int32_t p = order[q];
        const int32_t *lp = labels + (int64_t)p * n;
        int32_t m = 0;
        for (int32_t i = 0; i < n; ++i)
            if (lp[i] >= 0) { pairs[m].lab = lp[i]; pairs[m].idx = i; m++; }
        qsort(pairs, m, sizeof(li_pair), cmp_li);
        for (int32_t s = 0; s < m;) {
            int32_t e = s;
            while (e < m && pairs[e].lab == pairs[s].lab) e++;
            /* cluster members pairs[s..e) in ascending index order */
            for (int32_t a = s; a < e; ++a) {
                int32_t i = pairs[a].idx;
                int64_t fa = cap_indptr[i];
                int64_t cap = cap_indptr[i + 1] - fa;
                if (q == 0) {
                    int64_t tail = e - a - 1;
                    if (tail > cap) status = ORC_ERR_FIRST_OVERFLOW;
                    int64_t k = 0;
                    for (int32_t b = a + 1; b < e && k < cap; ++b, ++k) {
                        ind[fa + k] = pairs[b].idx;
                        dat[fa + k] = 1;
                    }
                    degree[i] = (int32_t)(tail < cap ? tail : cap);
                    nnz += tail;
                    continue;
                }
                int64_t deg = degree[i];
                int64_t ndeg = deg;
                int32_t nn = 0;
                for (int32_t b = a + 1; b < e; ++b) {
                    int32_t j = pairs[b].idx;
                    /* binary search of j among the row's current columns */
                    int64_t lo = fa, hi = fa + deg;
                    while (lo < hi) {
                        int64_t mid = lo + (hi - lo) / 2;
                        if (ind[mid] < j) lo = mid + 1; else hi = mid;
                    }
                    if (lo < fa + deg && ind[lo] == j) { dat[lo]++; continue; }
                    if (ndeg >= cap) { disc++; continue; }
                    newj[nn] = j; newpos[nn] = lo; nn++; ndeg++;
                }
                if (nn == 0) continue;
                /* merge the new columns into the sorted row, from the back */
                int64_t src = fa + deg - 1, dst = fa + deg + nn - 1;
                for (int32_t t = nn - 1; t >= 0; --t) {
                    while (src >= newpos[t]) { ind[dst] = ind[src]; dat[dst] = dat[src]; dst--; src--; }
                    ind[dst] = newj[t]; dat[dst] = 1; dst--;
                }
                degree[i] = (int32_t)ndeg;
                nnz += nn;
            }
            s = e;
        }
    }
    /* condense: rows back to back */
    int64_t ptr = 0;
    for (int32_t i = 0; i < n; ++i) {
        indptr[i] = ptr;
        int64_t fa = cap_indptr[i];
        for (int32_t k = 0; k < degree[i]; ++k) {
            indices[ptr] = ind[fa + k];
            counts[ptr] = dat[fa + k];
            ptr++;
        }
    }
    indptr[n] = ptr;
    *nnz_out = nnz;
    *discarded_out = disc;
    free(ind); free(dat); free(degree); free(pairs); free(newj); free(newpos);
    return status;
}

/* ------------------------------------------------------------------------ */
/* K-Means label step.  MyML/MyML/cluster/KMeans.py:453-490 (py_label /      */
/* numba_label, and its GPU twin :586-629): the difference and its square    */
/* are float32, the running distance is float64, the lowest index wins ties  */
/* (strict <), the stored distance is float32(best).                         */
/* ------------------------------------------------------------------------ */
void orc_kmeans_label(int64_t N, int32_t D, int32_t K, const float *x,
                      const float *c, int32_t *labels, float *dists)
{
    for (int64_t i = 0; i < N; ++i) {
        const float *xi = x + i * D;
        double best = 0.0;
        int32_t bl = 0;
        for (int32_t k = 0; k < K; ++k) {
            double dist = 0.0;
            for (int32_t d = 0; d < D; ++d) {
                volatile float diff = xi[d] - c[(int64_t)k * D + d];
                volatile float sq = diff * diff;
                dist += (double)sq;
            }
            if (k == 0 || dist < best) { best = dist; bl = k; }
        }
        labels[i] = bl;
        dists[i] = (float)best;
    }
}

/* ------------------------------------------------------------------------ */
/* Quickselect of the k smallest distances, the reference's exact            */
/* partitioning sequence (MyML/MyML/utils/sorting.py:9-47, arg_k_select).    */
/* ------------------------------------------------------------------------ */
void orc_arg_k_select(const float *a, int64_t n, int32_t k, int32_t *out)
{
    int32_t *args = malloc(sizeof(int32_t) * n);
    for (int64_t i = 0; i < n; ++i) args[i] = (int32_t)i;
    int64_t lo = 0, hi = n - 1;
    while (lo < hi) {
        int64_t r = lo, w = hi;
        float mid = a[args[(r + w) / 2]];
        while (r < w) {
            if (a[args[r]] >= mid) {
                int32_t t = args[w]; args[w] = args[r]; args[r] = t;
                w--;
            } else {
                r++;
            }
        }
        if (a[args[r]] > mid) r--;
        if (k <= r) hi = r; else lo = r + 1;
    }
    for (int32_t i = 0; i < k; ++i) out[i] = args[i];
    free(args);
}

/* ------------------------------------------------------------------------ */
/* Centroid update.  MyML/MyML/cluster/KMeans.py:709-754                     */
/* (py_recompute_centroids / numba_recompute_centroids): float32 sums in     */
/* point order, centroid = float32(float64(sum) / count); empty clusters, in */
/* index order, take the points arg_k_select returns for the number of       */
/* empty clusters.  mode 1 = the float64-sum variant (sums in double).       */
/* ------------------------------------------------------------------------ */
void orc_kmeans_centroids(int64_t N, int32_t D, int32_t K, const float *x,
                          const int32_t *labels, const float *dists,
                          float *out, int mode)
{
    int32_t *cnt = calloc(K, sizeof(int32_t));
    float *s32 = calloc((int64_t)K * D, sizeof(float));
    double *s64 = calloc((int64_t)K * D, sizeof(double));
    for (int64_t i = 0; i < N; ++i) cnt[labels[i]]++;
    int32_t n_empty = 0;
    for (int32_t k = 0; k < K; ++k) n_empty += (cnt[k] == 0);
    int32_t *far = NULL;
    if (n_empty > 0) {
        far = malloc(sizeof(int32_t) * n_empty);
        orc_arg_k_select(dists, N, n_empty, far);
    }
    for (int64_t i = 0; i < N; ++i) {
        int32_t l = labels[i];
        for (int32_t d = 0; d < D; ++d) {
            volatile float acc = s32[(int64_t)l * D + d] + x[i * D + d];
            s32[(int64_t)l * D + d] = acc;
            s64[(int64_t)l * D + d] += (double)x[i * D + d];
        }
    }
    int32_t e = 0;
    for (int32_t k = 0; k < K; ++k) {
        if (cnt[k] != 0) {
            for (int32_t d = 0; d < D; ++d) {
                double s = mode == 1 ? s64[(int64_t)k * D + d] : (double)s32[(int64_t)k * D + d];
                out[(int64_t)k * D + d] = (float)(s / (double)cnt[k]);
            }
        } else {
            int32_t src = far[e++];
            for (int32_t d = 0; d < D; ++d) out[(int64_t)k * D + d] = x[(int64_t)src * D + d];
        }
    }
    free(cnt); free(s32); free(s64); free(far);
}

/* ------------------------------------------------------------------------ */
/* numpy's float32 add-reduction of a contiguous 1-D array (pairwise         */
/* summation with 8 partial sums in blocks of up to 128 elements), which the */
/* reference uses for the K-Means inertia (KMeans.py:164, self._dists.sum()).*/
/* ------------------------------------------------------------------------ */
static float pw_sum(const float *a, int64_t n)
{
    if (n < 8) {
        volatile float r = -0.0f;
        for (int64_t i = 0; i < n; ++i) r = r + a[i];
        return r;
    } else if (n <= 128) {
        volatile float r[8];
        for (int j = 0; j < 8; ++j) r[j] = a[j];
        int64_t i;
        for (i = 8; i < n - (n % 8); i += 8)
            for (int j = 0; j < 8; ++j) r[j] = r[j] + a[i + j];
        volatile float s01 = r[0] + r[1], s23 = r[2] + r[3];
        volatile float s45 = r[4] + r[5], s67 = r[6] + r[7];
        volatile float lo = s01 + s23, hi = s45 + s67;
        volatile float res = lo + hi;
        for (; i < n; ++i) res = res + a[i];
        return res;
    } else {
        int64_t n2 = n / 2;
        n2 -= n2 % 8;
        volatile float l = pw_sum(a, n2);
        volatile float r = pw_sum(a + n2, n - n2);
        volatile float s = l + r;
        return s;
    }
}

float orc_np_sum_f32(const float *a, int64_t n)
{
    return pw_sum(a, n);
}
