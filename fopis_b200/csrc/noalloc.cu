// noalloc.cu — electric-field energy of a caller-owned potential with no
// device allocation.
//
// Who needs it: callers that must not allocate device memory once their run
// loop has started — hosts that give the library only memory from their own
// pool allocator (a framework that owns all of the device's memory), and
// real-time loops that forbid allocator calls after start-up because
// cudaMalloc and cudaFree synchronise the device. They pass the potential and
// the one-double output in memory they already own; the reduction's scratch
// (per-block partial sums) lives in the file-scope array below instead of a
// cudaMalloc'd buffer.
//
// Limits and sharing:
//   * the scratch holds kMaxPartials partial sums, one per kNodesPerPartial
//     interior nodes, so the interior (nx)(ny)(nz) may hold at most
//     kMaxPartials * kNodesPerPartial = 33,554,432 nodes (e.g. 322^3); larger
//     grids are rejected with FOPIS_ERR_ARG;
//   * the array exists once per CUDA context that loads the library's module
//     and stays allocated until that context ends (32 KB);
//   * every call uses the same array: calls that overlap on the GPU (two
//     streams, or two host threads) race and may return wrong sums; serialise
//     them. Each call rewrites every partial it reads, so nothing carries over
//     from the previous call;
//   * the first call in a context looks up the array's device address with
//     cudaGetSymbolAddress while that context is current and keeps it, keyed
//     by the context's unique id (a context made after a device reset, or a
//     non-primary context, gets its own lookup).
#include "internal.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

namespace fopis {
namespace {

constexpr int kMaxPartials = 4096;
constexpr long long kNodesPerPartial = 8192;
constexpr int kThreadsNA = 256;
constexpr int kMaxContexts = 64;

static __device__ __align__(256) double g_energy_partials[kMaxPartials];

// The scratch address of each context met so far, by the context's unique id
// (cuCtxGetId never hands out an id twice in a process, so a context created
// after a device reset cannot pick up its predecessor's stale address).
struct ScratchEntry {
    unsigned long long ctx_id;
    double* addr;
};
ScratchEntry g_scratch[kMaxContexts];
int g_scratch_n = 0;
std::mutex g_setup_mutex;
PFN_cuCtxGetCurrent_v4000 g_get_current = nullptr;
PFN_cuCtxGetId_v12000 g_get_id = nullptr;
bool g_entry_points_tried = false;

// Id of the calling thread's current context; false when the driver entry
// points are unavailable or no context is current yet.
bool current_context_id(unsigned long long* id) {
    if (!g_entry_points_tried) {
        g_entry_points_tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
    }
    if (!g_get_current || !g_get_id) return false;
    CUcontext ctx = nullptr;
    if (g_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return g_get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of g_energy_partials in the current context (nullptr on
// failure). The runtime makes the device's primary context current on the
// first call below when no context is current yet, so the id is read after it.
double* scratch_address() {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long id = 0;
    if (current_context_id(&id))
        for (int t = 0; t < g_scratch_n; ++t)
            if (g_scratch[t].ctx_id == id) return g_scratch[t].addr;
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_energy_partials) != cudaSuccess || !p) return nullptr;
    if (current_context_id(&id) && g_scratch_n < kMaxContexts) g_scratch[g_scratch_n++] = {id, static_cast<double*>(p)};
    return static_cast<double*>(p);
}

__device__ __forceinline__ double block_reduce(double v) {
    __shared__ double red[32];
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Block b sums the squared edge differences of interior nodes
// [b * kNodesPerPartial, (b+1) * kNodesPerPartial), the same edges as
// Field::getEfieldEnergy (src/Grid/Field.cpp:194-213).
__global__ void energy_partials_kernel(const double* phi, int cx, int cy, int cz, double* partials) {
    const long long ny = cy - 2, nz = cz - 2;
    const long long M = (long long)(cx - 2) * ny * nz;
    const long long lo = (long long)blockIdx.x * kNodesPerPartial;
    const long long hi = min(M, lo + kNodesPerPartial);
    double e = 0.0;
    for (long long t = lo + threadIdx.x; t < hi; t += blockDim.x) {
        const int i = 1 + (int)(t / (ny * nz));
        const int j = 1 + (int)((t / nz) % ny);
        const int k = 1 + (int)(t % nz);
        const long long id = ((long long)i * cy + j) * cz + k;
        const double p = phi[id];
        if (i < cx - 2) { const double d = p - phi[id + (long long)cy * cz]; e += d * d; }
        if (j < cy - 2) { const double d = p - phi[id + cz]; e += d * d; }
        if (k < cz - 2) { const double d = p - phi[id + 1]; e += d * d; }
    }
    e = block_reduce(e);
    if (threadIdx.x == 0) partials[blockIdx.x] = e;
}

__global__ void energy_finish_kernel(const double* partials, int n, double half_eps0, double* out) {
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) v += partials[t];
    v = block_reduce(v);
    if (threadIdx.x == 0) *out = half_eps0 * v;
}

}  // namespace
}  // namespace fopis

extern "C" int fopis_efield_energy_noalloc(const double* phi, int nx, int ny, int nz, double eps0, double* energy,
                                           void* stream) {
    using namespace fopis;
    if (!phi || !energy || nx < 3 || ny < 3 || nz < 3) return FOPIS_ERR_ARG;
    const long long interior = (long long)nx * ny * nz;
    if (interior > (long long)kMaxPartials * kNodesPerPartial) return FOPIS_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FOPIS_ERR_NO_CUDA;
    double* partials = scratch_address();
    if (!partials) return FOPIS_ERR_CUDA;
    const int blocks = (int)((interior + kNodesPerPartial - 1) / kNodesPerPartial);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Each launch's own status is checked, so an earlier error of the caller's
    // is neither reported as this call's nor cleared.
    int cx = nx + 2, cy = ny + 2, cz = nz + 2;
    void* a1[] = {(void*)&phi, &cx, &cy, &cz, &partials};
    if (cudaLaunchKernel((const void*)energy_partials_kernel, dim3(blocks), dim3(kThreadsNA), a1, 0, st) != cudaSuccess) {
        cudaGetLastError();
        return FOPIS_ERR_CUDA;
    }
    int nb = blocks;
    double half_eps0 = 0.5 * eps0;
    void* a2[] = {&partials, &nb, &half_eps0, &energy};
    if (cudaLaunchKernel((const void*)energy_finish_kernel, dim3(1), dim3(1024), a2, 0, st) != cudaSuccess) {
        cudaGetLastError();
        return FOPIS_ERR_CUDA;
    }
    return FOPIS_OK;
}
