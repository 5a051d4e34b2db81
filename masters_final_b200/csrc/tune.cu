// Launch-shape tuning table.
//
// A few launch shapes of the hot kernels are knobs with a built-in default:
// the tensor-core labeler's CTAs per SM and centroid tile buffers, the
// co-association row passes' CTAs per SM, the weight split of the graph
// MST's first phase and the Boruvka round kernel's participant cap.  The
// autotuner (masters_final_b200/tune.py) times the candidates on the
// workload shapes and writes a table; the Python binding loads it into this
// process-wide table at start-up (eacb_tune_set).  An entry applies to a
// knob for a shape (a, b) with a_lo <= a <= a_hi and b_lo <= b <= b_hi -- a
// is the dimension, the partition count or 0 and b the point or vertex
// count, as each knob's user states -- and the first matching entry wins.
// The table is the library's one global: it is written only between calls
// and read by every launch.
#include "eacb_common.cuh"

#include <mutex>

namespace {

struct TuneEntry {
    int knob;
    int64_t a_lo, a_hi, b_lo, b_hi;
    int64_t value;
};

constexpr int kMaxTuneEntries = 256;
TuneEntry g_tune[kMaxTuneEntries];
int g_tune_n = 0;
std::mutex g_tune_mutex;

}  // namespace

namespace eacb {

int64_t tune_get(int knob, int64_t a, int64_t b, int64_t dflt)
{
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    for (int i = 0; i < g_tune_n; ++i) {
        const TuneEntry &e = g_tune[i];
        if (e.knob == knob && a >= e.a_lo && a <= e.a_hi && b >= e.b_lo && b <= e.b_hi)
            return e.value;
    }
    return dflt;
}

}  // namespace eacb

extern "C" int eacb_tune_set(int knob, int64_t a_lo, int64_t a_hi, int64_t b_lo, int64_t b_hi,
                             int64_t value)
{
    if (knob < 0 || knob >= eacb::TUNE_NKNOBS || a_lo > a_hi || b_lo > b_hi)
        return EACB_ERR_BAD_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    if (g_tune_n >= kMaxTuneEntries) return EACB_ERR_WORKSPACE;
    g_tune[g_tune_n++] = TuneEntry{knob, a_lo, a_hi, b_lo, b_hi, value};
    return EACB_OK;
}

extern "C" void eacb_tune_clear(void)
{
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_n = 0;
}

extern "C" int64_t eacb_tune_get(int knob, int64_t a, int64_t b, int64_t dflt)
{
    if (knob < 0 || knob >= eacb::TUNE_NKNOBS) return dflt;
    return eacb::tune_get(knob, a, b, dflt);
}
