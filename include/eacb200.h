/*
 * eacb200.h -- C ABI of libeacb200.so, the B200 (sm_100a) evidence
 * accumulation clustering (EAC) hot path.
 *
 * The reference (diogo-aos/masters_final) is Python 2 + Numba and has no
 * native interface; each entry point below replaces one reference Python
 * function or kernel sequence, cited as path:line within that project.
 *
 * Conventions:
 *   - every pointer argument is a DEVICE pointer unless the name says host_;
 *   - `stream` is a cudaStream_t cast to uintptr_t (0 = legacy default stream);
 *   - scratch memory is a caller-owned device buffer `ws` of `ws_bytes` bytes,
 *     at least the size returned by the matching *_workspace_size() query,
 *     256-byte aligned (a misaligned one gives EACB_ERR_WORKSPACE); the
 *     library never allocates device memory;
 *   - functions return an eacb_status (0 = success, negative = error) and
 *     never throw; outputs are undefined after an error;
 *   - functions whose work has data-dependent sizes (Boruvka, connected
 *     components, co-association, k-means, final clustering) synchronize
 *     `stream` a few times per call to read counters (all Boruvka rounds of
 *     a weight phase run inside one persistent kernel); the scans are
 *     asynchronous on `stream`;
 *   - entry points may be called from several host threads at once on
 *     different streams and workspaces (eacb_scan_excl_i32_noalloc excepted).
 */
#ifndef EACB200_H
#define EACB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    EACB_OK = 0,
    EACB_ERR_BAD_ARGUMENT = -1,          /* null pointer, negative size, bad enum */
    EACB_ERR_WORKSPACE = -2,             /* ws too small or misaligned, or an internal capacity exceeded */
    EACB_ERR_CUDA = -3,                  /* a CUDA runtime call failed */
    EACB_ERR_UNSUPPORTED = -4,           /* valid input this build does not handle */
    EACB_ERR_DEVICE_WAIT = -5,           /* a bounded device-side wait gave up */
    EACB_ERR_NOT_CONVERGED = -6,         /* iteration cap hit (input not a valid graph) */
    EACB_ERR_FIRST_PARTITION_OVERFLOW = -7, /* reference would write past a row (sparse.py:446-465) */
    EACB_ERR_BAD_INPUT = -8,             /* input failed a device-side validity check */
    EACB_ERR_VALUE = -9,                 /* the reference raises ValueError here */
    EACB_ERR_INTERNAL = -10
} eacb_status;

/* Element type codes for weight arrays. */
typedef enum {
    EACB_U8 = 1,
    EACB_U16 = 2,
    EACB_I32 = 3,
    EACB_U32 = 4,
    EACB_F32 = 5
} eacb_dtype;

int eacb_version(void);
const char *eacb_status_string(int status);

/* After EACB_ERR_CUDA: the cudaError_t of the failed runtime call, on the
 * calling thread, and the library source file and line that made it. */
int eacb_last_cuda_error(const char **file, int *line);

/* Every workspace starts with a device error word that asynchronous entry
 * points set on a device-side failure.  Synchronizes `stream`, returns the
 * status that word encodes and clears it. */
int eacb_workspace_status(void *ws, uintptr_t stream);

/* Built-in profiling, off by default.  eacb_profile_enable(1) resets the
 * counters and turns on CUDA-event timing (on the launching stream) of the
 * tagged kernels; eacb_profile_read returns the number of kernels the
 * library launched since, and per tag (0 = Boruvka round kernel, 1 = scan,
 * 2 = co-association rows, 3 = k-means labels, 4 = Boruvka weight-phase
 * builds; arrays of 8) the total milliseconds, algorithmic bytes and
 * launches. */
void eacb_profile_enable(int on);
void eacb_profile_read(int64_t *launches, double *ms, double *bytes, int64_t *count);

/* Launch-shape tuning table (no counterpart in the reference, which has
 * fixed launch shapes: MyML/MyML/cluster/KMeans.py:286-291).  Knobs, each
 * with a built-in default and a shape (a, b): 0 tensor-core labeler CTAs
 * per SM (1 or 2; a = d, b = n), 1 its centroid tile buffers (1 or 2),
 * 2 co-association count pass CTAs per SM (a = P, b = n), 3 fill pass CTAs
 * per SM, 4 the graph MST's first weight phase as a share of the entries
 * in per mille (a = 0, b = vertices), 5 the Boruvka round kernel's
 * participants at most (a = 0 graph MST/CC, 1 EAC final clustering;
 * b = vertices), 6 the co-association pair tiles: the compare work a group
 * may take per member visit of the streaming kernels (0: streaming only;
 * a = P, b = n).  eacb_tune_set adds an entry for a <= .. <= a_hi and
 * b_lo <= .. <= b_hi (the first matching entry wins); eacb_tune_clear
 * removes all; eacb_tune_get returns the value a launch of shape (a, b)
 * would use (dflt when no entry matches).  Process-wide; set it between
 * calls (the Python binding loads masters_final_b200/tuning.json at start). */
int eacb_tune_set(int knob, int64_t a_lo, int64_t a_hi, int64_t b_lo, int64_t b_hi,
                  int64_t value);
void eacb_tune_clear(void);
int64_t eacb_tune_get(int knob, int64_t a, int64_t b, int64_t dflt);

/* Test hooks of the Boruvka round kernel, process-wide, to be set between
 * calls.  eacb_debug_set_round_cap: rounds a weight phase may run (0 = the
 * built-in cap of 96); a graph that needs more returns
 * EACB_ERR_NOT_CONVERGED, as an inconsistent one does at the built-in cap.
 * eacb_debug_set_round_team: participants of the round kernel (0 =
 * automatic, 1 = a single block, more = that many cooperative blocks, at
 * most the number that can be resident); results do not depend on it. */
void eacb_debug_set_round_cap(int rounds);
void eacb_debug_set_round_team(int blocks);

/* ------------------------------------------------------------------------
 * Exclusive prefix sum.
 * Replaces MyML/MyML/utils/scan.py:144-249 (scan_gpu, recursive Blelloch
 * scan) and the CPU scans :42-72 (exprefixsumNumba / exprefixsumNumbaSingle).
 * out[i] = init + sum(in[0..i)); `in` may equal `out` (in place).  The int32
 * variant stores each prefix truncated to 32 bits (wraps modulo 2^32 like the
 * reference's int64 carry stored into an int32 array); *d_total (device int64)
 * receives the exact 64-bit total.  Single pass (decoupled look-back).
 * ------------------------------------------------------------------------ */
size_t eacb_scan_workspace_size(int64_t n);
int eacb_scan_excl_i32(const int32_t *in, int32_t *out, int64_t n, int64_t init,
                       int64_t *d_total, void *ws, size_t ws_bytes, uintptr_t stream);
int eacb_scan_excl_i32_i64(const int32_t *in, int64_t *out, int64_t n, int64_t init,
                           int64_t *d_total, void *ws, size_t ws_bytes, uintptr_t stream);
int eacb_scan_excl_i64(const int64_t *in, int64_t *out, int64_t n, int64_t init,
                       int64_t *d_total, void *ws, size_t ws_bytes, uintptr_t stream);

/* Allocation-free variant of eacb_scan_excl_i32 (no counterpart in the
 * reference).  For callers that may not allocate device memory while they
 * run -- a host with pools fixed at start-up, a real-time path that forbids
 * allocation, a plugin handed raw buffers and no allocator -- and so cannot
 * supply the workspace eacb_scan_excl_i32 needs.  Same inputs, outputs and
 * wrap-around as eacb_scan_excl_i32, no workspace argument: the look-back
 * scratch is a fixed array of about 350 KiB in the library's device image,
 * held on every GPU that loads the library until the process exits.  n may
 * not exceed EACB_SCAN_NOALLOC_MAX_N (returns EACB_ERR_WORKSPACE beyond it).
 * The first call on each device looks up that array's address
 * (cudaGetSymbolAddress; make this first call before any stream capture)
 * and keeps it for the life of the process: do not call this entry point
 * on a device after resetting it (cudaDeviceReset).  Calls share the array:
 * calls that overlap on the GPU race, so serialise them.  Each call copies
 * its device-side status to the host, synchronizes `stream` (so it returns
 * only after the scan has finished) and returns that status. */
#define EACB_SCAN_NOALLOC_MAX_N (((int64_t)1) << 28)
int eacb_scan_excl_i32_noalloc(const int32_t *in, int32_t *out, int64_t n, int64_t init,
                               int64_t *d_total, uintptr_t stream);

/* ------------------------------------------------------------------------
 * Boruvka minimum spanning forest of a symmetric CSR graph.
 * Replaces MyML/MyML/graph/mst.py:417-564 (boruvka_minho_gpu) and its
 * kernels :574-809.  Graph: row r has the entries [first_edge[r],
 * first_edge[r] + out_degree[r]) of dest/weight; every undirected edge is
 * stored in both directions (a graph with unequal numbers of entries u -> v
 * with u < v and with u > v returns EACB_ERR_BAD_INPUT); self loops are
 * ignored.
 * Ties are broken by the strict order (weight, min(u,v), max(u,v)), so the
 * forest is unique.  mst_out (capacity n_vertices - 1) receives, per chosen
 * edge, the index of its entry in row min(u,v) (the smallest such index with
 * the chosen weight), in round order, supervertex order within a round;
 * *host_n_mst receives the number of forest edges.
 * Requires bits(weight) + 2*ceil(log2(n_vertices)) + 1 <= 64.
 * ------------------------------------------------------------------------ */
size_t eacb_boruvka_workspace_size(int32_t n_vertices, int64_t n_edges);
int eacb_boruvka_mst(const int32_t *dest, const void *weight, int weight_dtype,
                     const int32_t *first_edge, const int32_t *out_degree,
                     int32_t n_vertices, int64_t n_edges,
                     int32_t *mst_out, int64_t *host_n_mst,
                     void *ws, size_t ws_bytes, uintptr_t stream);

/* ------------------------------------------------------------------------
 * Connected components by Boruvka contraction, with the reference's own
 * label numbering: each round a vertex picks its minimum out-edge by
 * (weight, destination supervertex), the smaller endpoint of a mutual pick
 * becomes the root, and supervertices are renumbered in root order.
 * Replaces MyML/MyML/graph/connected_components.py:176-314
 * (connected_comps_gpu; same labels as connected_comps_seq :46-137).
 * labels (n_vertices, int32) receive the component labels; *host_n_comps the
 * number of components.
 * ------------------------------------------------------------------------ */
int eacb_connected_components(const int32_t *dest, const void *weight, int weight_dtype,
                              const int32_t *first_edge, const int32_t *out_degree,
                              int32_t n_vertices, int64_t n_edges,
                              int32_t *labels, int64_t *host_n_comps,
                              void *ws, size_t ws_bytes, uintptr_t stream);

/* ------------------------------------------------------------------------
 * K-Means ensemble (batched Lloyd iterations, all partitions at once).
 * Replaces MyML/MyML/utils/partition.py:88-124 (generateEnsemble) running
 * MyML/MyML/cluster/KMeans.py:117-189 (K_Means.fit) per partition, with the
 * label step :453-490 / :586-629 and the centroid step :709-754
 * (empty clusters take the points of MyML/MyML/utils/sorting.py:9-47).
 * X: n x d float32 row-major (d <= 32).  Partition p has k[p] <= kmax
 * clusters (device int32[P]) and starts from the points init[p*kmax + c],
 * c < k[p] (device int32; the host draws them like the reference, with
 * random.sample).  Each partition runs until max_iter label passes or until
 * its inertia (numpy float32 sum of the distances) changes by at most tol.
 * label_mode 0 = float32 screen + exact re-check (CUDA cores),
 *            1 = tcgen05 tensor cores + exact re-check;
 * both return the reference's labels exactly.  centroid_mode 0 = float32
 * sums in point order (the reference's arithmetic), 1 = float64 sums.
 * Outputs: labels (P*n int32), centroids (P*kmax*d float32, rows c < k[p]),
 * optional dists (P*n float32), iters (P int32), inertia (P float32).
 * ------------------------------------------------------------------------ */
size_t eacb_kmeans_workspace_size(int32_t n, int32_t d, int32_t P, int32_t kmax);
int eacb_kmeans_ensemble(const float *X, int32_t n, int32_t d, int32_t P,
                         const int32_t *k, int32_t kmax, const int32_t *init,
                         int32_t max_iter, float tol, int32_t label_mode,
                         int32_t centroid_mode, int32_t *labels, float *centroids,
                         float *dists, int32_t *iters, float *inertia,
                         void *ws, size_t ws_bytes, uintptr_t stream);

/* One label step for given centroids (k x d float32): the reference's
 * labels and float32 distances (KMeans.py:453-490). */
size_t eacb_kmeans_label_workspace_size(int32_t n, int32_t d, int32_t k);
int eacb_kmeans_label(const float *X, int32_t n, int32_t d, const float *C, int32_t k,
                      int32_t label_mode, int32_t *labels, float *dists,
                      void *ws, size_t ws_bytes, uintptr_t stream);

/* The label step with its arithmetic path fixed by name: float32 screen on
 * CUDA cores, or tcgen05 BF16 tensor cores; both with the exact re-check,
 * so both return the reference's labels and distances.  Workspace as for
 * eacb_kmeans_label. */
int eacb_kmeans_label_fp32(const float *X, int32_t n, int32_t d, const float *C, int32_t k,
                           int32_t *labels, float *dists, void *ws, size_t ws_bytes,
                           uintptr_t stream);
int eacb_kmeans_label_bf16tc(const float *X, int32_t n, int32_t d, const float *C, int32_t k,
                             int32_t *labels, float *dists, void *ws, size_t ws_bytes,
                             uintptr_t stream);

/* One centroid update, MyML/MyML/cluster/KMeans.py:709-754
 * (numba_recompute_centroids): C (k x d float32) receives, per cluster, the
 * float32 sum of its points in point order (centroid_mode 1: float64 sums)
 * divided as f32(f64(sum) / count); empty clusters take, in cluster order,
 * the points arg_k_select (MyML/MyML/utils/sorting.py:9-47) returns for
 * their number from `dists` (n float32, left unchanged).  labels in [0, k). */
size_t eacb_kmeans_centroids_workspace_size(int32_t n, int32_t d, int32_t k);
int eacb_kmeans_centroids(const float *X, int32_t n, int32_t d, const int32_t *labels,
                          const float *dists, int32_t k, int32_t centroid_mode, float *C,
                          void *ws, size_t ws_bytes, uintptr_t stream);

/* ------------------------------------------------------------------------
 * Sparse co-association matrix, condensed (row i holds columns j > i).
 * Replaces MyML/MyML/EAC/sparse.py:154-226 (EAC_CSR.update_ensemble with
 * update_cluster_fp_condensed :446-465 and
 * update_cluster_sorted_surgical_condensed :957-1040, then _condense).
 * The ensemble is a label matrix labels[p*n + i] (cluster id in [0, K) of
 * point i in partition p, -1 = in no cluster); P <= 255, K <= 8192.
 * cap_indptr (n+1, int64) is the reference's per-row capacity layout
 * (indptr_linear / indptr_constant): row i keeps at most cap_indptr[i+1] -
 * cap_indptr[i] columns -- the first ones met in processing order (the
 * partition with the fewest clusters, then the others by index; within a
 * partition by column) -- and the counts of the others are discarded.
 * Three calls sharing one workspace, in this order:
 *   eacb_coassoc_prepare: builds the cluster member lists (stable counting
 *     sort) and the processing order; *host_max_cluster receives the largest
 *     cluster size (MyML/MyML/EAC/sparse.py:1065, the base of max_assocs);
 *   eacb_coassoc_count: counts the kept columns of every row, writes indptr
 *     (n+1) and *host_nnz; returns EACB_ERR_FIRST_PARTITION_OVERFLOW where
 *     the reference would write a first-partition row past its capacity;
 *   eacb_coassoc_fill: writes indices (nnz, int32, ascending per row) and
 *     data (nnz, uint8 counts, or (max count + 1) - count when make_diassoc,
 *     MyML/MyML/EAC/sparse.py:295-311), *host_discarded (nnz_discarded) and
 *     *host_max_count.
 * ------------------------------------------------------------------------ */
size_t eacb_coassoc_workspace_size(int32_t n, int32_t P, int32_t K);
int eacb_coassoc_prepare(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                         int64_t *host_max_cluster, void *ws, size_t ws_bytes, uintptr_t stream);
int eacb_coassoc_count(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                       const int64_t *cap_indptr, int64_t *indptr, int64_t *host_nnz,
                       void *ws, size_t ws_bytes, uintptr_t stream);
int eacb_coassoc_fill(const int32_t *labels, int32_t n, int32_t P, int32_t K,
                      const int64_t *cap_indptr, const int64_t *indptr,
                      int32_t *indices, uint8_t *data, int32_t make_diassoc,
                      int64_t *host_discarded, int32_t *host_max_count,
                      void *ws, size_t ws_bytes, uintptr_t stream);

/* The whole build in one call, as EAC.buildMatrix runs it
 * (MyML/MyML/EAC/eac.py:115-140): member lists, then the capacity layout
 * (cap_mode 0 = indptr_linear with its default line, 1 = indptr_constant)
 * for max_assocs (0: factor x the largest cluster), then counts and rows.
 * indices/data have room for `capacity` entries (the reference preallocates
 * the layout's total; the kept count never exceeds it).  *host_nnz,
 * *host_discarded, *host_max_count and *host_max_assocs are set. */
size_t eacb_coassoc_build_workspace_size(int32_t n, int32_t P, int32_t K);
int eacb_coassoc_build(const int32_t *labels, int32_t n, int32_t P, int32_t K, int32_t cap_mode,
                       int64_t max_assocs, int32_t factor, int64_t *indptr, int32_t *indices,
                       uint8_t *data, int64_t capacity, int32_t make_diassoc, int64_t *host_nnz,
                       int64_t *host_discarded, int32_t *host_max_count,
                       int64_t *host_max_assocs, void *ws, size_t ws_bytes, uintptr_t stream);

/* Per-row capacity layouts of the co-association rows (exclusive scan of
 * the capacities, n+1 int64).  Replaces MyML/MyML/EAC/sparse.py:371-413
 * (indptr_linear: max_assocs for rows below n_s*n, then the line down to
 * val_e*max_assocs at n_e*n, in the reference's float64 arithmetic) and
 * :368-369 (indptr_constant). */
size_t eacb_capacity_workspace_size(int32_t n);
int eacb_capacity_linear(int32_t n, int64_t max_assocs, double n_s, double n_e,
                         double val_s, double val_e, int64_t *cap_indptr,
                         void *ws, size_t ws_bytes, uintptr_t stream);
int eacb_capacity_constant(int32_t n, int64_t max_assocs, int64_t *cap_indptr,
                           uintptr_t stream);

/* data[e] = max_val - data[e] (uint8), MyML/MyML/EAC/sparse.py:295-311
 * (make_diassoc; the reference passes max count + 1). */
int eacb_make_diassoc(uint8_t *data, int64_t nnz, int32_t max_val, uintptr_t stream);

/* ------------------------------------------------------------------------
 * EAC final clustering of a condensed co-association dissimilarity matrix.
 * Replaces MyML/MyML/EAC/eac.py:199-267 (sp_sl_lifetime) with
 * lifetime_n_clusters :366-391, whose MST is the Kruskal of
 * scipy_numba/scipy_numba/sparse/csgraph/_min_spanning_tree.py:21-175 and
 * whose labels come from scipy.sparse.csgraph.connected_components.
 * Input: upper-triangle CSR (row i holds columns j > i, sorted) with uint8
 * dissimilarities; max_dist = the number of partitions (the reference adds 1).
 * n_clusters = 0 uses the maximum-lifetime rule.
 * Outputs: labels (n, int32) numbered by each cluster's smallest member (the
 * numbering connected_components produces); *host_n_fclusts; *host_labels_valid
 * = 0 when the reference returns an empty label array (one cluster).
 * Returns EACB_ERR_VALUE where the reference raises ValueError (fewer than
 * two MST edges, or no two MST edges of equal weight).
 * ------------------------------------------------------------------------ */
size_t eacb_final_clustering_workspace_size(int32_t n, int64_t nnz);
int eacb_final_clustering(const int64_t *indptr, const int32_t *indices,
                          const uint8_t *diassoc, int32_t n, int64_t nnz,
                          int32_t max_dist, int32_t n_clusters,
                          int32_t *labels, int64_t *host_n_fclusts,
                          int32_t *host_labels_valid,
                          void *ws, size_t ws_bytes, uintptr_t stream);

/* The final clustering's two steps as separate calls.
 * eacb_lifetime_cut: lifetime_n_clusters (MyML/MyML/EAC/eac.py:366-391) and
 * the cut decision of sp_sl_lifetime (:220-265) on the uint8 weights of a
 * minimum spanning forest of n points (n_mst < n weights, any order);
 * *host_n_clusters receives the number of clusters and *host_threshold the
 * largest forest weight kept (-1 keeps none).  EACB_ERR_VALUE where the
 * reference raises ValueError.
 * eacb_relabel_canonical: numbers the groups of a labelling (n ids in
 * [0, n)) by their smallest member, the numbering of scipy's
 * connected_components that the final labels use; labels_out may equal
 * labels_in; *host_n_groups receives the number of groups. */
size_t eacb_lifetime_cut_workspace_size(void);
int eacb_lifetime_cut(const uint8_t *mst_weights, int64_t n_mst, int32_t n, int32_t max_dist,
                      int32_t n_clusters, int64_t *host_n_clusters, int32_t *host_threshold,
                      void *ws, size_t ws_bytes, uintptr_t stream);
size_t eacb_relabel_canonical_workspace_size(int32_t n);
int eacb_relabel_canonical(const int32_t *labels_in, int32_t n, int32_t *labels_out,
                           int64_t *host_n_groups, void *ws, size_t ws_bytes, uintptr_t stream);

/* ------------------------------------------------------------------------
 * Batched EAC: many independent instances, each the whole path above
 * (eacb_kmeans_ensemble -> eacb_coassoc_prepare/count/fill with the
 * dissimilarity transform -> eacb_final_clustering), in one call.
 * Replaces the reference's per-dataset loop over generateEnsemble
 * (MyML/MyML/utils/partition.py:88-124), EAC.buildMatrix
 * (MyML/MyML/EAC/eac.py:115-140) and EAC.finalClustering (:142-179), as its
 * experiment drivers run it (experiments/study_kmin.py:398-587).
 * Per instance the caller gives device X (n x d float32), k (P int32) and
 * init (P*kmax int32) drawn like the reference, and a device labels array
 * (n int32).  Results per instance: labels (numbered by smallest member;
 * all 0 when the lifetime rule yields one cluster, where the reference
 * returns an empty array), n_fclusts, labels_valid, nnz, nnz_discarded and
 * status.  The workspace holds n_workers fixed slices
 * (eacb_batched_workspace_size) and, after them, an arena for the
 * count-dependent arrays of the instances in flight (at least the largest
 * instance's co-association CSR plus its final-clustering workspace; more
 * lets more instances run at once).  ws must be 256-byte aligned.
 * n_workers host threads, each with its own stream, take the instances
 * largest first.  The call returns when every instance is done: EACB_OK, or
 * the status of the first failed instance in input order.
 * ------------------------------------------------------------------------ */
typedef struct eacb_instance {
    const float *X;           /* in: device, n x d row-major */
    const int32_t *k;         /* in: device, clusters per partition (P) */
    const int32_t *init;      /* in: device, initial sample indices (P x kmax) */
    int32_t *labels;          /* out: device, final labels (n) */
    int32_t n, d, P, kmax;    /* in: d <= 32, P <= 255, kmax <= 8192 */
    int64_t n_fclusts;        /* out */
    int64_t nnz;              /* out: co-association entries kept */
    int64_t nnz_discarded;    /* out */
    int32_t labels_valid;     /* out */
    int32_t status;           /* out: eacb status of this instance */
    float ms_ensemble;        /* out: host wall-clock ms of each stage on its worker */
    float ms_coassoc;
    float ms_final;
    int32_t worker;           /* out: the worker that ran the instance */
    int32_t cuda_error;       /* out: after EACB_ERR_CUDA, the cudaError_t ... */
    int32_t cuda_line;        /* ... and the source line of the failed call */
} eacb_instance;

typedef struct eacb_batch_options {
    int32_t max_iter;          /* Lloyd label passes (the reference's iters, 3) */
    float tol;                 /* inertia tolerance (1e-4) */
    int32_t label_mode;        /* 0 float32 cores, 1 tcgen05 (both exact) */
    int32_t centroid_mode;     /* 0 float32 point-order sums, 1 float64 */
    int32_t cap_mode;          /* 0 indptr_linear, 1 indptr_constant */
    int32_t max_assocs_factor; /* max_assocs = factor * largest cluster (3) */
    double n_s, n_e, val_s, val_e;  /* indptr_linear parameters (0.05, 1, 1, 0.05) */
    int32_t n_clusters;        /* 0 = lifetime rule */
    int32_t reserved;
} eacb_batch_options;

size_t eacb_batched_workspace_size(const eacb_instance *inst, int32_t n_inst, int32_t n_workers);
int eacb_batched_eac(eacb_instance *inst, int32_t n_inst, const eacb_batch_options *opt,
                     int32_t n_workers, void *ws, size_t ws_bytes, uintptr_t stream);

#ifdef __cplusplus
}
#endif

#endif /* EACB200_H */
