// fields.cu — node-field kernels: charge fold and conversion, boundary
// conditions of phi, nodal electric field, field energy and exports.
#include "internal.cuh"

#include <algorithm>

namespace fopis {

namespace {

constexpr int kT = 256;

struct G {
    int cx, cy, cz;
    int n[3];
    int per[6];
};
G make_g(const Ctx& c) {
    G g;
    g.cx = c.cx; g.cy = c.cy; g.cz = c.cz;
    g.n[0] = c.nx; g.n[1] = c.ny; g.n[2] = c.nz;
    for (int t = 0; t < 6; ++t) g.per[t] = c.per[t];
    return g;
}
__device__ __forceinline__ long long L(const G& g, int i, int j, int k) {
    return ((long long)i * g.cy + j) * g.cz + k;
}
int blocks(long long n) {
    long long b = (n + kT - 1) / kT;
    return (int)(b < 148LL * 32 ? (b < 1 ? 1 : b) : 148LL * 32);
}

// Periodic fold of one axis for every species array (integer, exact):
// MPIw::Environment::sendRecvNodeScalar self-exchange, glue size 2
// (src/MPI/Communicator.cpp:497-574): node 0 and node n both become their sum,
// node 1 and node n+1 likewise.
// A fixed-point fold sum that passed 2^64 (unsigned wrap) is latched as
// FOPIS_DEV_RHO_OVERFLOW; FP64 sums have no such limit.
__device__ __forceinline__ bool fold_wrapped(unsigned long long sum, unsigned long long a) { return sum < a; }
__device__ __forceinline__ bool fold_wrapped(double, double) { return false; }

template <typename W>
__global__ void fold_kernel(W* rho, int nsp, long long N, G g, int axis, unsigned* status) {
    const int dims[3] = {g.cx, g.cy, g.cz};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const long long plane = (long long)dims[a1] * dims[a2];
    const long long total = plane * nsp;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(t / plane);
        const long long r = t % plane;
        int idx[3];
        idx[a1] = (int)(r / dims[a2]);
        idx[a2] = (int)(r % dims[a2]);
        W* a = rho + (long long)s * N;
        const int X = dims[axis];
        idx[axis] = 0; const long long p0 = L(g, idx[0], idx[1], idx[2]);
        idx[axis] = X - 2; const long long pn = L(g, idx[0], idx[1], idx[2]);
        idx[axis] = 1; const long long p1 = L(g, idx[0], idx[1], idx[2]);
        idx[axis] = X - 1; const long long pn1 = L(g, idx[0], idx[1], idx[2]);
        const W s0 = a[p0] + a[pn], s1 = a[p1] + a[pn1];
        if (fold_wrapped(s0, a[p0]) || fold_wrapped(s1, a[p1])) atomicOr(status, (unsigned)FOPIS_DEV_RHO_OVERFLOW);
        a[p0] = s0; a[pn] = s0; a[p1] = s1; a[pn1] = s1;
    }
}

struct Scales { double v[FOPIS_MAX_SPECIES]; };

// A species accumulator as a number: unsigned 64-bit fixed point (mixed mode;
// the weights are nonnegative and the deposit latches any wrap) or the FP64
// weight sum (FP64 mode).
__device__ __forceinline__ double weight_value(unsigned long long w) { return (double)w; }
__device__ __forceinline__ double weight_value(double w) { return w; }

// rho[0] = sum_s q_s size_s W_s (x 2^-51 in fixed point) (RootGridField.cpp:1206-1214).
template <typename W>
__global__ void convert_kernel(const W* rho, int nsp, long long N, Scales sc, double* rho0) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        double r = 0.0;
        for (int s = 0; s < nsp; ++s) r += sc.v[s] * weight_value(rho[(long long)s * N + t]);
        rho0[t] = r;
    }
}

template <typename W>
__global__ void convert_species_kernel(const W* rho, long long N, double scale, double* out) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        out[t] = scale * weight_value(rho[t]);
}

// Glue copy of one axis: node 0 <- node n, node n+1 <- node 1
// (Communicator::sendRecvFieldX/Y/Z self branch, Communicator.cpp:290-299).
__global__ void glue_kernel(double* a, G g, int axis) {
    const int dims[3] = {g.cx, g.cy, g.cz};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const long long plane = (long long)dims[a1] * dims[a2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < plane; t += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        idx[a1] = (int)(t / dims[a2]);
        idx[a2] = (int)(t % dims[a2]);
        const int X = dims[axis];
        idx[axis] = 1; const double lo = a[L(g, idx[0], idx[1], idx[2])];
        idx[axis] = X - 2; const double hi = a[L(g, idx[0], idx[1], idx[2])];
        idx[axis] = 0; a[L(g, idx[0], idx[1], idx[2])] = hi;
        idx[axis] = X - 1; a[L(g, idx[0], idx[1], idx[2])] = lo;
    }
}

// Field::setDirichletPhi / setNeumannPhi on one face (src/Grid/Field.cpp:34-96):
// the face plane over the interior of the other two axes.
__global__ void phi_face_kernel(double* phi, G g, int axis, int side, int neumann) {
    const int dims[3] = {g.cx, g.cy, g.cz};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const long long m1 = dims[a1] - 2, m2 = dims[a2] - 2;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < m1 * m2; t += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        idx[a1] = 1 + (int)(t / m2);
        idx[a2] = 1 + (int)(t % m2);
        const int X = dims[axis];
        const int bi = side == 0 ? 1 : X - 2, ni = side == 0 ? 2 : X - 3;
        idx[axis] = ni; const double nv = phi[L(g, idx[0], idx[1], idx[2])];
        idx[axis] = bi; phi[L(g, idx[0], idx[1], idx[2])] = neumann ? nv : 0.0;
    }
}

// Maps an index of a periodic axis onto its interior image.
__device__ __forceinline__ int wrapi(const G& g, int axis, int idx) {
    if (g.per[2 * axis]) {
        const int n = g.n[axis];
        if (idx == 0) return n;
        if (idx == n + 1) return 1;
    }
    return idx;
}

__device__ __forceinline__ void store_e(float4* o, const double e[3]) {
    *o = make_float4((float)e[0], (float)e[1], (float)e[2], 0.0f);
}
__device__ __forceinline__ void store_e(Vec4d* o, const double e[3]) { *o = Vec4d{e[0], e[1], e[2], 0.0}; }

// Nodal E of RootGrid::updateEfield + updateReferenceEfield
// (RootGridField.cpp:456-582): centred 0.5 (phi[i-1] - phi[i+1]) per axis,
// one-sided second order on Dirichlet/Neumann faces, zero glue on those axes,
// periodic images on periodic axes (sendRecvField self-copies).
template <typename Out>
__global__ void efield_kernel(const double* phi, G g, Out* out, double* outx, double* outy, double* outz) {
    const long long N = (long long)g.cx * g.cy * g.cz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i0 = (int)(t / ((long long)g.cy * g.cz));
        const int j0 = (int)((t / g.cz) % g.cy);
        const int k0 = (int)(t % g.cz);
        int id[3] = {wrapi(g, 0, i0), wrapi(g, 1, j0), wrapi(g, 2, k0)};
        const int dims[3] = {g.cx, g.cy, g.cz};
        bool outside = false;
        for (int a = 0; a < 3; ++a) if (id[a] == 0 || id[a] == dims[a] - 1) outside = true;
        double e[3] = {0.0, 0.0, 0.0};
        if (!outside) {
            for (int a = 0; a < 3; ++a) {
                int lo[3] = {id[0], id[1], id[2]}, hi[3] = {id[0], id[1], id[2]};
                const int X = dims[a];
                if (!g.per[2 * a] && id[a] == 1) {
                    int p2[3] = {id[0], id[1], id[2]}, p3[3] = {id[0], id[1], id[2]};
                    p2[a] = 2; p3[a] = 3;
                    e[a] = 0.5 * (phi[L(g, p3[0], p3[1], p3[2])] - 4.0 * phi[L(g, p2[0], p2[1], p2[2])] +
                                  3.0 * phi[L(g, id[0], id[1], id[2])]);
                } else if (!g.per[2 * a + 1] && id[a] == X - 2) {
                    int p2[3] = {id[0], id[1], id[2]}, p3[3] = {id[0], id[1], id[2]};
                    p2[a] = X - 3; p3[a] = X - 4;
                    e[a] = 0.5 * (-phi[L(g, p3[0], p3[1], p3[2])] + 4.0 * phi[L(g, p2[0], p2[1], p2[2])] -
                                  3.0 * phi[L(g, id[0], id[1], id[2])]);
                } else {
                    lo[a] = id[a] - 1; hi[a] = id[a] + 1;   // glue neighbours hold periodic images
                    e[a] = 0.5 * ((phi[L(g, lo[0], lo[1], lo[2])] - phi[L(g, id[0], id[1], id[2])]) +
                                  (phi[L(g, id[0], id[1], id[2])] - phi[L(g, hi[0], hi[1], hi[2])]));
                }
            }
        }
        if (out) store_e(out + t, e);
        if (outx) { outx[t] = e[0]; outy[t] = e[1]; outz[t] = e[2]; }
    }
}

__device__ __forceinline__ double bsum(double v) {
    __shared__ double red[32];
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Field::getEfieldEnergy (src/Grid/Field.cpp:194-213) from the edge fields
// ex[i] = phi[i] - phi[i+1] (RootGridField.cpp:470-478); per-block partials.
__global__ void field_energy_kernel(const double* phi, G g, double* partial) {
    const long long M = (long long)(g.cx - 2) * (g.cy - 2) * (g.cz - 2);
    double en = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < M; t += (long long)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(t / ((long long)(g.cy - 2) * (g.cz - 2)));
        const int j = 1 + (int)((t / (g.cz - 2)) % (g.cy - 2));
        const int k = 1 + (int)(t % (g.cz - 2));
        const double p = phi[L(g, i, j, k)];
        if (i < g.cx - 2) { const double d = p - phi[L(g, i + 1, j, k)]; en += d * d; }
        if (j < g.cy - 2) { const double d = p - phi[L(g, i, j + 1, k)]; en += d * d; }
        if (k < g.cz - 2) { const double d = p - phi[L(g, i, j, k + 1)]; en += d * d; }
    }
    en = bsum(en);
    if (threadIdx.x == 0) partial[blockIdx.x] = en;
}

__global__ void sum_partials_kernel(const double* partial, int n, double* out) {
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) v += partial[t];
    v = bsum(v);
    if (threadIdx.x == 0) *out = v;
}

}  // namespace

// Charge of one unit of a species' accumulator: q size 2^-51 for the
// fixed-point weights, q size for the FP64 weights.
double species_rho_scale(const Ctx& c, int s) {
    return c.p.species[s].charge * c.p.species[s].size * (c.fp64 ? 1.0 : kDepositUnit);
}

void rho_zero(Ctx& c) {
    FOPIS_CUDA(cudaMemsetAsync(c.rho_i64, 0, sizeof(unsigned long long) * c.N * c.nsp, c.st));
}

void glue_copy(Ctx& c, double* a) {
    const G g = make_g(c);
    const long long planes[3] = {(long long)c.cy * c.cz, (long long)c.cx * c.cz, (long long)c.cx * c.cy};
    for (int axis = 0; axis < 3; ++axis) {
        if (!c.per[2 * axis]) continue;
        ++c.launches;
        glue_kernel<<<blocks(planes[axis]), kT, 0, c.st>>>(a, g, axis);
        FOPIS_LAUNCH_CHECK();
    }
}

void rho_finalize(Ctx& c) {
    const G g = make_g(c);
    const long long planes[3] = {(long long)c.cy * c.cz, (long long)c.cx * c.cz, (long long)c.cx * c.cy};
    for (int axis = 0; axis < 3; ++axis) {
        if (!c.per[2 * axis]) continue;
        ++c.launches;
        if (c.fp64)
            fold_kernel<<<blocks(planes[axis] * c.nsp), kT, 0, c.st>>>(reinterpret_cast<double*>(c.rho_i64), c.nsp,
                                                                       (long long)c.N, g, axis, &c.d_sc->status);
        else
            fold_kernel<<<blocks(planes[axis] * c.nsp), kT, 0, c.st>>>(c.rho_i64, c.nsp, (long long)c.N, g, axis,
                                                                       &c.d_sc->status);
        FOPIS_LAUNCH_CHECK();
    }
    Scales sc{};
    for (int s = 0; s < c.nsp; ++s) sc.v[s] = species_rho_scale(c, s);
    ++c.launches;
    if (c.fp64)
        convert_kernel<<<blocks((long long)c.N), kT, 0, c.st>>>(reinterpret_cast<const double*>(c.rho_i64), c.nsp,
                                                                (long long)c.N, sc, c.rho0);
    else
        convert_kernel<<<blocks((long long)c.N), kT, 0, c.st>>>(c.rho_i64, c.nsp, (long long)c.N, sc, c.rho0);
    FOPIS_LAUNCH_CHECK();
}

// After a solve: the periodic glue copies first (the last halo exchange of the
// reference's doPSOR), then Field::setBoundaryConditionPhi on the D/N faces
// (RootGridField.cpp:65-103 calls it after the sweeps and exchanges nothing
// afterwards), so a glue node beside a Neumann face keeps the value it had
// before the face copy, as in the reference.
void phi_boundary(Ctx& c) {
    const G g = make_g(c);
    glue_copy(c, c.phi);
    for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side) {
            const char b = c.p.boundary[2 * axis + side];
            if (b == 'P') continue;
            const long long m = axis == 0 ? (long long)(c.cy - 2) * (c.cz - 2)
                                          : (axis == 1 ? (long long)(c.cx - 2) * (c.cz - 2) : (long long)(c.cx - 2) * (c.cy - 2));
            ++c.launches;
            phi_face_kernel<<<blocks(m), kT, 0, c.st>>>(c.phi, g, axis, side, b == 'N');
            FOPIS_LAUNCH_CHECK();
        }
}

void efield_update(Ctx& c) {
    const G g = make_g(c);
    ++c.launches;
    if (c.fp64) efield_kernel<Vec4d><<<blocks((long long)c.N), kT, 0, c.st>>>(c.phi, g, c.E64, nullptr, nullptr, nullptr);
    else efield_kernel<float4><<<blocks((long long)c.N), kT, 0, c.st>>>(c.phi, g, c.E, nullptr, nullptr, nullptr);
    FOPIS_LAUNCH_CHECK();
}

void field_export(Ctx& c, int which, double* host) {
    const G g = make_g(c);
    const size_t bytes = sizeof(double) * c.N;
    if (which == FOPIS_FIELD_PHI) {
        FOPIS_CUDA(cudaMemcpyAsync(host, c.phi, bytes, cudaMemcpyDeviceToHost, c.st));
    } else if (which == FOPIS_FIELD_RHO0) {
        FOPIS_CUDA(cudaMemcpyAsync(host, c.rho0, bytes, cudaMemcpyDeviceToHost, c.st));
    } else if (which >= FOPIS_FIELD_EXREF && which <= FOPIS_FIELD_EZREF) {
        double* tmp = nullptr;
        FOPIS_CUDA(cudaMallocAsync(&tmp, 3 * bytes, c.st));
        ++c.launches;
        efield_kernel<float4><<<blocks((long long)c.N), kT, 0, c.st>>>(c.phi, g, nullptr, tmp, tmp + c.N, tmp + 2 * c.N);
        FOPIS_LAUNCH_CHECK();
        FOPIS_CUDA(cudaMemcpyAsync(host, tmp + (which - FOPIS_FIELD_EXREF) * c.N, bytes, cudaMemcpyDeviceToHost, c.st));
        FOPIS_CUDA(cudaFreeAsync(tmp, c.st));
    } else if (which >= FOPIS_FIELD_RHO_SPECIES && which < FOPIS_FIELD_RHO_SPECIES + c.nsp) {
        const int s = which - FOPIS_FIELD_RHO_SPECIES;
        const double scale = species_rho_scale(c, s);
        ++c.launches;
        if (c.fp64)
            convert_species_kernel<<<blocks((long long)c.N), kT, 0, c.st>>>(
                reinterpret_cast<const double*>(c.rho_i64) + (size_t)s * c.N, (long long)c.N, scale, c.scratch64);
        else
            convert_species_kernel<<<blocks((long long)c.N), kT, 0, c.st>>>(c.rho_i64 + (size_t)s * c.N, (long long)c.N,
                                                                           scale, c.scratch64);
        FOPIS_LAUNCH_CHECK();
        FOPIS_CUDA(cudaMemcpyAsync(host, c.scratch64, bytes, cudaMemcpyDeviceToHost, c.st));
    } else {
        throw ApiError{FOPIS_ERR_ARG, "unknown field selector"};
    }
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
}

double efield_energy(Ctx& c) {
    const G g = make_g(c);
    const int nb = 148 * 4;
    double* part = c.red_partials;
    ++c.launches;
    field_energy_kernel<<<nb, kT, 0, c.st>>>(c.phi, g, part);
    ++c.launches;
    sum_partials_kernel<<<1, 1024, 0, c.st>>>(part, nb, &c.d_sc->red[15]);
    FOPIS_LAUNCH_CHECK();
    double v = 0.0;
    FOPIS_CUDA(cudaMemcpyAsync(&v, &c.d_sc->red[15], sizeof(double), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    return 0.5 * c.p.eps0 * v;
}

namespace {
__global__ void __launch_bounds__(256) axpy_kernel(double* dst, const double* a, const double* b, double sb, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = a[i] + sb * b[i];
}
}  // namespace

void phi_axpy(Ctx& c, double* dst, const double* a, const double* b, double sb) {
    const long long n = (long long)c.N;
    ++c.launches;
    axpy_kernel<<<(int)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0, c.st>>>(dst, a, b, sb, n);
    FOPIS_LAUNCH_CHECK();
}

}  // namespace fopis
