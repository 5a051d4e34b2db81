// Single-pass exclusive scan (decoupled look-back) for int32/int64 streams.
//
// Replaces MyML/MyML/utils/scan.py:144-249 (scan_gpu: a recursive Blelloch
// scan with one launch per level plus a fix-up pass, int only) and the CPU
// scans :42-72.  One launch: each CTA takes the next tile index from an
// atomic counter, reduces 16 elements per thread loaded with 128-bit loads,
// scans the thread sums across the CTA (warp shuffles + a Blelloch tree over
// warp totals), obtains its tile prefix by looking back over its
// predecessors' published aggregates, and writes its outputs.  HBM traffic is
// one read and one write of the stream.
#include "eacb_common.cuh"
#include "scan_impl.cuh"

using namespace eacb;

extern "C" size_t eacb_scan_workspace_size(int64_t n)
{
    Carver c(nullptr, 0);
    ScanScratch::carve(c, n);
    return c.off;
}

template <typename TIn, typename TOut>
static int scan_entry(const TIn *in, TOut *out, int64_t n, int64_t init, int64_t *d_total,
                      void *ws, size_t ws_bytes, uintptr_t stream)
{
    if (n < 0 || (n > 0 && (!in || !out)) || !d_total || (!ws && n > 0)) return EACB_ERR_BAD_ARGUMENT;
    Carver c(ws, ws_bytes);
    ScanScratch s = ScanScratch::carve(c, n);
    if (c.overflow) return EACB_ERR_WORKSPACE;
    if (n > 0) EACB_CUDA(cudaMemsetAsync(s.err, 0, sizeof(int), as_stream(stream)));
    ProfScope ps(PROF_SCAN, as_stream(stream));
    int st = scan_launch<TIn, TOut>(in, out, n, init, d_total, s, as_stream(stream));
    ps.done((double)n * (sizeof(TIn) + sizeof(TOut)));
    return st;
}

extern "C" int eacb_scan_excl_i32(const int32_t *in, int32_t *out, int64_t n, int64_t init,
                                  int64_t *d_total, void *ws, size_t ws_bytes, uintptr_t stream)
{
    return scan_entry<int32_t, int32_t>(in, out, n, init, d_total, ws, ws_bytes, stream);
}

extern "C" int eacb_scan_excl_i32_i64(const int32_t *in, int64_t *out, int64_t n, int64_t init,
                                      int64_t *d_total, void *ws, size_t ws_bytes, uintptr_t stream)
{
    return scan_entry<int32_t, int64_t>(in, out, n, init, d_total, ws, ws_bytes, stream);
}

extern "C" int eacb_scan_excl_i64(const int64_t *in, int64_t *out, int64_t n, int64_t init,
                                  int64_t *d_total, void *ws, size_t ws_bytes, uintptr_t stream)
{
    return scan_entry<int64_t, int64_t>(in, out, n, init, d_total, ws, ws_bytes, stream);
}
