// Batched EAC: many independent instances (ensemble -> co-association ->
// Boruvka MST -> lifetime cut) in one call.
//
// The reference runs one EAC at a time from its experiment drivers
// (experiments/study_kmin.py:398-587 loops over datasets, each doing
// generateEnsemble MyML/MyML/utils/partition.py:88-124, EAC.buildMatrix
// MyML/MyML/EAC/eac.py:115-140 and EAC.finalClustering :142-179).  Here a
// pool of host workers, each with its own CUDA stream and its own slice of
// the caller's workspace, takes instances largest first; small instances
// (most of a batch) are launch- and latency-bound, so several of them in
// flight on separate streams fill the GPU that one alone leaves idle.
//
// Workspace: n_workers fixed slices (sized for the largest instance: label
// matrix, centroids, row pointers, and the union of the k-means and the
// co-association scratch) followed by an arena for the parts whose size
// depends on the co-association count (CSR columns + values and the final
// clustering's edge arrays).  The arena is shared: a worker reserves its
// instance's block after the count pass and returns it at the end, waiting
// while other workers hold the memory it needs.
#include "eacb_common.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <iterator>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace eacb {
namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// First-fit allocator over the arena.  A block is held only while one
// instance finishes (fill + final clustering), and a worker holds at most
// one block, so a waiting worker always sees memory come back.
class Arena {
  public:
    Arena(char *base, size_t size) : base_(base), size_(size)
    {
        if (size) free_[0] = size;
    }
    char *alloc(size_t bytes)
    {
        bytes = align_up(bytes ? bytes : 1);
        if (bytes > size_) return nullptr;
        std::unique_lock<std::mutex> lk(m_);
        for (;;) {
            for (auto it = free_.begin(); it != free_.end(); ++it) {
                if (it->second < bytes) continue;
                const size_t off = it->first, sz = it->second;
                free_.erase(it);
                if (sz > bytes) free_[off + bytes] = sz - bytes;
                ++live_;
                return base_ + off;
            }
            if (live_ == 0) return nullptr;   // unreachable: an empty arena holds `bytes`
            cv_.wait(lk);
        }
    }
    void release(char *p, size_t bytes)
    {
        bytes = align_up(bytes ? bytes : 1);
        std::lock_guard<std::mutex> lk(m_);
        auto it = free_.emplace((size_t)(p - base_), bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
        --live_;
        cv_.notify_all();
    }

  private:
    char *base_;
    size_t size_;
    std::map<size_t, size_t> free_;   // offset -> bytes
    int live_ = 0;
    std::mutex m_;
    std::condition_variable cv_;
};

// A block returns to the arena only once the stream that uses it is idle.
struct ArenaBlock {
    Arena &a;
    cudaStream_t st;
    char *p;
    size_t bytes;
    ArenaBlock(Arena &ar, cudaStream_t s, size_t b) : a(ar), st(s), p(ar.alloc(b)), bytes(b) {}
    ~ArenaBlock()
    {
        if (!p) return;
        cudaStreamSynchronize(st);
        a.release(p, bytes);
    }
};

struct Slice {
    int32_t *labels;       // P x n
    float *centroids;      // P x kmax x d
    int32_t *iters;
    float *inertia;
    int64_t *cap_indptr;   // n + 1
    int64_t *indptr;       // n + 1
    char *scratch;         // k-means scratch, later co-association + capacity scratch
    size_t kmeans_bytes, coassoc_bytes, capacity_bytes;
    char *capacity;        // inside scratch, after the co-association part

    static Slice carve(Carver &c, const eacb_instance &I)
    {
        Slice s;
        s.labels = c.take<int32_t>((size_t)I.P * I.n);
        s.centroids = c.take<float>((size_t)I.P * I.kmax * I.d);
        s.iters = c.take<int32_t>(I.P);
        s.inertia = c.take<float>(I.P);
        s.cap_indptr = c.take<int64_t>((size_t)I.n + 1);
        s.indptr = c.take<int64_t>((size_t)I.n + 1);
        s.kmeans_bytes = eacb_kmeans_workspace_size(I.n, I.d, I.P, I.kmax);
        s.coassoc_bytes = align_up(eacb_coassoc_workspace_size(I.n, I.P, I.kmax));
        s.capacity_bytes = eacb_capacity_workspace_size(I.n);
        const size_t co = s.coassoc_bytes + s.capacity_bytes;
        s.scratch = c.take<char>(std::max(s.kmeans_bytes, co));
        s.capacity = s.scratch ? s.scratch + s.coassoc_bytes : nullptr;
        return s;
    }
};

size_t slice_bytes(const eacb_instance &I)
{
    Carver c(nullptr, 0);
    Slice::carve(c, I);
    return align_up(c.off);
}

bool valid_instance(const eacb_instance &I)
{
    return I.X && I.n > 0 && I.d > 0 && I.d <= 32 && I.P > 0 && I.P <= 255 && I.kmax > 0 &&
           I.kmax <= 8192 && I.k && I.init && I.labels;
}

typedef std::chrono::steady_clock Clock;
inline float ms_since(Clock::time_point t0)
{
    return std::chrono::duration<float, std::milli>(Clock::now() - t0).count();
}

int run_instance(eacb_instance &I, const eacb_batch_options &o, char *slice, size_t bytes,
                 Arena &arena, cudaStream_t st)
{
    const uintptr_t hs = (uintptr_t)st;
    Clock::time_point t0 = Clock::now();
    Carver c(slice, bytes);
    Slice s = Slice::carve(c, I);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    int r = eacb_kmeans_ensemble(I.X, I.n, I.d, I.P, I.k, I.kmax, I.init, o.max_iter, o.tol,
                                 o.label_mode, o.centroid_mode, s.labels, s.centroids, nullptr,
                                 s.iters, s.inertia, s.scratch, s.kmeans_bytes, hs);
    if (r) return r;
    I.ms_ensemble = ms_since(t0);
    t0 = Clock::now();
    int64_t max_cluster = 0;
    r = eacb_coassoc_prepare(s.labels, I.n, I.P, I.kmax, &max_cluster, s.scratch, s.coassoc_bytes,
                             hs);
    if (r) return r;
    const int64_t max_assocs = max_cluster * (int64_t)o.max_assocs_factor;
    if (o.cap_mode == 0)
        r = eacb_capacity_linear(I.n, max_assocs, o.n_s, o.n_e, o.val_s, o.val_e, s.cap_indptr,
                                 s.capacity, s.capacity_bytes, hs);
    else
        r = eacb_capacity_constant(I.n, max_assocs, s.cap_indptr, hs);
    if (r) return r;
    int64_t nnz = 0;
    r = eacb_coassoc_count(s.labels, I.n, I.P, I.kmax, s.cap_indptr, s.indptr, &nnz, s.scratch,
                           s.coassoc_bytes, hs);
    if (r) return r;
    I.nnz = nnz;
    // the count-dependent part, from the shared arena
    const size_t b_ind = align_up((size_t)nnz * sizeof(int32_t));
    const size_t b_dat = align_up((size_t)nnz);
    const size_t b_fin = eacb_final_clustering_workspace_size(I.n, nnz);
    ArenaBlock blk(arena, st, b_ind + b_dat + b_fin);
    if (!blk.p) return EACB_ERR_WORKSPACE;
    int32_t *indices = (int32_t *)blk.p;
    uint8_t *data = (uint8_t *)(blk.p + b_ind);
    char *fws = blk.p + b_ind + b_dat;
    int64_t discarded = 0;
    int32_t max_count = 0;
    r = eacb_coassoc_fill(s.labels, I.n, I.P, I.kmax, s.cap_indptr, s.indptr, indices, data, 1,
                          &discarded, &max_count, s.scratch, s.coassoc_bytes, hs);
    if (r) return r;
    I.nnz_discarded = discarded;
    I.ms_coassoc = ms_since(t0);
    t0 = Clock::now();
    int64_t nf = 0;
    int32_t valid = 0;
    r = eacb_final_clustering(s.indptr, indices, data, I.n, nnz, I.P, o.n_clusters, I.labels, &nf,
                              &valid, fws, b_fin, hs);
    if (r) return r;
    if (!valid) {   // one cluster: the reference returns no labels; all points get 0
        EACB_CUDA(cudaMemsetAsync(I.labels, 0, sizeof(int32_t) * (size_t)I.n, st));
        EACB_CUDA(cudaStreamSynchronize(st));
    }
    I.n_fclusts = nf;
    I.labels_valid = valid;
    I.ms_final = ms_since(t0);
    return EACB_OK;
}

}  // namespace
}  // namespace eacb

using namespace eacb;

extern "C" size_t eacb_batched_workspace_size(const eacb_instance *inst, int32_t n_inst,
                                              int32_t n_workers)
{
    if (!inst || n_inst <= 0 || n_workers <= 0) return 0;
    size_t mx = 0;
    for (int32_t i = 0; i < n_inst; ++i)
        if (valid_instance(inst[i])) mx = std::max(mx, slice_bytes(inst[i]));
    return (size_t)n_workers * mx;
}

extern "C" int eacb_batched_eac(eacb_instance *inst, int32_t n_inst,
                                const eacb_batch_options *opt, int32_t n_workers, void *ws,
                                size_t ws_bytes, uintptr_t stream)
{
    if (!inst || n_inst <= 0 || !opt || n_workers <= 0 || !ws) return EACB_ERR_BAD_ARGUMENT;
    if (opt->max_iter <= 0 || opt->max_assocs_factor <= 0 || opt->n_clusters < 0 ||
        (opt->cap_mode != 0 && opt->cap_mode != 1) ||
        (opt->label_mode != 0 && opt->label_mode != 1))
        return EACB_ERR_BAD_ARGUMENT;
    for (int32_t i = 0; i < n_inst; ++i)
        if (!valid_instance(inst[i])) return EACB_ERR_BAD_ARGUMENT;
    const size_t fixed = eacb_batched_workspace_size(inst, n_inst, n_workers);
    if (ws_bytes < fixed) return EACB_ERR_WORKSPACE;
    const size_t slice = fixed / (size_t)n_workers;
    char *base = (char *)ws;
    if ((uintptr_t)base % kAlign) return EACB_ERR_BAD_ARGUMENT;
    Arena arena(base + fixed, ws_bytes - fixed);
    int dev = 0;
    EACB_CUDA(cudaGetDevice(&dev));
    // the caller's stream may still be producing the inputs
    EACB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    // largest instances first (their k-means + co-association work ~ P * n * n / k)
    std::vector<int32_t> order(n_inst);
    for (int32_t i = 0; i < n_inst; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        const double ca = (double)inst[a].P * inst[a].n * inst[a].n / inst[a].kmax;
        const double cb = (double)inst[b].P * inst[b].n * inst[b].n / inst[b].kmax;
        return ca > cb || (ca == cb && a < b);
    });
    for (int32_t i = 0; i < n_inst; ++i) {
        inst[i].status = EACB_ERR_INTERNAL;
        inst[i].ms_ensemble = inst[i].ms_coassoc = inst[i].ms_final = 0.f;
        inst[i].worker = -1;
        inst[i].cuda_error = inst[i].cuda_line = 0;
    }
    std::atomic<int32_t> next(0);
    const int32_t nw = std::min(n_workers, n_inst);
    auto worker = [&](int w) {
        if (cudaSetDevice(dev) != cudaSuccess) return;
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return;
        // instances run side by side: each one's Boruvka rounds take one
        // block (a plain launch) instead of a cooperative grid over the GPU
        if (nw > 1) eacb::set_thread_round_team(1);
        char *sl = base + (size_t)w * slice;
        for (;;) {
            const int32_t q = next.fetch_add(1);
            if (q >= n_inst) break;
            eacb_instance &I = inst[order[q]];
            I.worker = w;
            try {
                I.status = run_instance(I, *opt, sl, slice, arena, st);
            } catch (...) {                              // host allocation failure
                I.status = EACB_ERR_INTERNAL;
            }
            if (I.status == EACB_ERR_CUDA) I.cuda_error = eacb_last_cuda_error(nullptr, &I.cuda_line);
            if (I.status) cudaStreamSynchronize(st);   // nothing of it left in flight
        }
        eacb::set_thread_round_team(0);
        cudaStreamDestroy(st);
    };
    std::vector<std::thread> pool;
    try {
        for (int w = 1; w < nw; ++w) pool.emplace_back(worker, w);
    } catch (...) {
        // fewer threads than asked: the ones running take every instance
    }
    worker(0);
    for (auto &t : pool) t.join();
    for (int32_t i = 0; i < n_inst; ++i)
        if (inst[i].status) return inst[i].status;
    return EACB_OK;
}
