// Library-wide entry points: version, status strings, workspace error word.
#include "eacb_common.cuh"

namespace eacb {
__global__ void k_set_i64(int64_t *p, int64_t v) { *p = v; }
}  // namespace eacb

extern "C" int eacb_version(void) { return 1; }

extern "C" const char *eacb_status_string(int s)
{
    switch (s) {
    case EACB_OK: return "EACB_OK";
    case EACB_ERR_BAD_ARGUMENT: return "EACB_ERR_BAD_ARGUMENT";
    case EACB_ERR_WORKSPACE: return "EACB_ERR_WORKSPACE";
    case EACB_ERR_CUDA: return "EACB_ERR_CUDA";
    case EACB_ERR_UNSUPPORTED: return "EACB_ERR_UNSUPPORTED";
    case EACB_ERR_DEVICE_WAIT: return "EACB_ERR_DEVICE_WAIT";
    case EACB_ERR_NOT_CONVERGED: return "EACB_ERR_NOT_CONVERGED";
    case EACB_ERR_FIRST_PARTITION_OVERFLOW: return "EACB_ERR_FIRST_PARTITION_OVERFLOW";
    case EACB_ERR_BAD_INPUT: return "EACB_ERR_BAD_INPUT";
    case EACB_ERR_VALUE: return "EACB_ERR_VALUE";
    case EACB_ERR_INTERNAL: return "EACB_ERR_INTERNAL";
    default: return "EACB_ERR_UNKNOWN";
    }
}

// Every workspace layout starts with the device error word.  Asynchronous
// entry points leave device-side failures there; this reads and clears it.
extern "C" int eacb_workspace_status(void *ws, uintptr_t stream)
{
    if (!ws) return EACB_ERR_BAD_ARGUMENT;
    int e = 0;
    EACB_CUDA(cudaMemcpyAsync(&e, ws, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    EACB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (e != 0) {
        EACB_CUDA(cudaMemsetAsync(ws, 0, sizeof(int), (cudaStream_t)stream));
        EACB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    }
    return eacb::dev_err_to_status(e);
}

namespace eacb {
Prof &prof()
{
    static Prof p = {};
    return p;
}

struct CudaErrInfo {
    int code;
    const char *file;
    int line;
};
static thread_local CudaErrInfo t_cuda_err = {0, nullptr, 0};

void note_cuda_error(int code, const char *file, int line)
{
    t_cuda_err.code = code;
    t_cuda_err.file = file;
    t_cuda_err.line = line;
}
}  // namespace eacb

// The calling thread's last CUDA runtime error seen by the library (0 if
// none), with the source file and line of the failed call.
extern "C" int eacb_last_cuda_error(const char **file, int *line)
{
    if (file) *file = eacb::t_cuda_err.file ? eacb::t_cuda_err.file : "";
    if (line) *line = eacb::t_cuda_err.line;
    return eacb::t_cuda_err.code;
}

// Profiling: enable/disable and reset counters.
extern "C" void eacb_profile_enable(int on)
{
    eacb::prof() = eacb::Prof{};
    eacb::prof().enabled = on;
}

// Counters since the last eacb_profile_enable(): kernel launches issued by
// the library, and per tag (0 = edge tile, 1 = scan, 2 = coassoc rows,
// 3 = k-means labels) total ms, algorithmic bytes and launch count.
extern "C" void eacb_profile_read(int64_t *launches, double *ms, double *bytes, int64_t *count)
{
    if (launches) *launches = eacb::prof().launches;
    for (int i = 0; i < eacb::PROF_NTAGS; ++i) {
        if (ms) ms[i] = eacb::prof().ms[i];
        if (bytes) bytes[i] = eacb::prof().bytes[i];
        if (count) count[i] = eacb::prof().count[i];
    }
}

namespace eacb {
__global__ void k_clear_status(uint64_t *status, int64_t n, int *counter)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        status[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) *counter = 0;
}
}  // namespace eacb
