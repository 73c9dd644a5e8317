// noalloc.cu — electric-field energy of a caller-owned potential with no
// device allocation.
//
// Who needs it: callers that must not allocate device memory during their run
// loop — code recorded into a CUDA graph with stream capture (cudaMalloc is
// not a capturable call), hosts that hand the library only memory from their
// own pool allocator, and real-time loops that forbid allocator calls after
// start-up. They pass the potential and the one-double output in memory they
// already own; the reduction's scratch (per-block partial sums) lives in the
// file-scope array below instead of a cudaMalloc'd buffer.
//
// Limits and sharing:
//   * the scratch holds kMaxPartials partial sums, one per kNodesPerPartial
//     interior nodes, so the interior (nx)(ny)(nz) may hold at most
//     kMaxPartials * kNodesPerPartial = 33,554,432 nodes (e.g. 322^3); larger
//     grids are rejected with FOPIS_ERR_ARG;
//   * the array exists once per device that loads the library and stays
//     allocated until the process exits (32 KB);
//   * every call uses the same array: calls that overlap on the GPU (two
//     streams, or two host threads) race and may return wrong sums; serialise
//     them. Each call rewrites every partial it reads, so nothing carries over
//     from the previous call;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress while that device is current; make that first call
//     before any stream capture.
#include "internal.cuh"

#include <mutex>

namespace fopis {
namespace {

constexpr int kMaxPartials = 4096;
constexpr long long kNodesPerPartial = 8192;
constexpr int kThreadsNA = 256;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_energy_partials[kMaxPartials];

double* g_partials_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

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
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return FOPIS_ERR_NO_CUDA;
    double* partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_partials_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_energy_partials) != cudaSuccess || !p) return FOPIS_ERR_CUDA;
            g_partials_addr[dev] = static_cast<double*>(p);
        }
        partials = g_partials_addr[dev];
    }
    const int blocks = (int)((interior + kNodesPerPartial - 1) / kNodesPerPartial);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    energy_partials_kernel<<<blocks, kThreadsNA, 0, st>>>(phi, nx + 2, ny + 2, nz + 2, partials);
    energy_finish_kernel<<<1, 1024, 0, st>>>(partials, blocks, 0.5 * eps0, energy);
    return cudaGetLastError() == cudaSuccess ? FOPIS_OK : FOPIS_ERR_CUDA;
}
