// multigrid.cu — the Poisson solve of RootGrid::solvePoisson
// (src/Grid/RootGrid/RootGridField.cpp:41-103) as geometric multigrid.
//
// The reference sweeps plane-parity PSOR up to 1000 times per solve. Here the
// FP64 outer loop computes r = f - A phi on the glue-layout node array
// (f = rho0/eps0, A = 6 - sum of the six neighbours, dx = 1), and each
// iteration solves A e = r approximately with one FP32 V-cycle (red-black
// Gauss-Seidel smoothing, full-weighting restriction, trilinear prolongation,
// rediscretised coarse operators, single-CTA FP64 coarsest solve), then adds
// e to phi in FP64. It stops when ||r||_2 <= tol ||f||_2.
//
// Unknowns are the nodes the reference's PSOR updates: glue indices 1..n on a
// periodic axis, 2..nx-1 on a Dirichlet/Neumann axis (Dirichlet and Neumann
// faces are held during the solve and set afterwards by Field::
// setBoundaryConditionPhi, src/Grid/Field.cpp:10-96). With every axis
// periodic the mean of f is removed and phi is kept at zero mean.
#include "internal.cuh"

#include <algorithm>
#include <cmath>

namespace fopis {

namespace {

constexpr int kT = 256;
constexpr int kRedBlocks = 148 * 2;
constexpr int kCoarseMax = 8192;    // unknowns the single-CTA coarsest solve holds (3 FP64 arrays, 192 KB)

struct Lv {
    int n0, n1, n2;
    int p0, p1, p2;
    float* u;
    float* f;
    float* r;
    float inv_scale;   // 1/scale: 4^level
};
Lv lv(const MGLevel& m) {
    return Lv{m.n[0], m.n[1], m.n[2], m.per[0], m.per[1], m.per[2], m.u, m.f, m.r, (float)(1.0 / m.scale)};
}

int nblocks(long long n) {
    long long b = (n + kT - 1) / kT;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

__device__ __forceinline__ float nb(const float* u, int n, int per, long long base, long long stride, int idx, int d) {
    int q = idx + d;
    if (q < 0) { if (!per) return 0.0f; q += n; }
    else if (q >= n) { if (!per) return 0.0f; q -= n; }
    return u[base + (long long)(q - idx) * stride];
}

// Six-neighbour sum at (a,b,c) with homogeneous Dirichlet or periodic closure.
__device__ __forceinline__ float nsum(const Lv& L, const float* u, int a, int b, int c) {
    const long long s1 = L.n2, s0 = (long long)L.n1 * L.n2;
    const long long id = a * s0 + b * s1 + c;
    return nb(u, L.n0, L.p0, id, s0, a, -1) + nb(u, L.n0, L.p0, id, s0, a, 1) +
           nb(u, L.n1, L.p1, id, s1, b, -1) + nb(u, L.n1, L.p1, id, s1, b, 1) +
           nb(u, L.n2, L.p2, id, 1, c, -1) + nb(u, L.n2, L.p2, id, 1, c, 1);
}

// One red-black half sweep: u <- (1-w) u + w (sum(nb) + f/scale) / 6 on the
// nodes with (a+b+c) % 2 == color; thread t owns every other node of a row.
__global__ void rb_smooth_kernel(Lv L, int color, float omega) {
    const int hn = (L.n2 + 1) / 2;
    const long long M = (long long)L.n0 * L.n1 * hn;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < M; t += (long long)gridDim.x * blockDim.x) {
        const int h = (int)(t % hn);
        const long long row = t / hn;
        const int b = (int)(row % L.n1), a = (int)(row / L.n1);
        const int c = 2 * h + ((a + b + color) & 1);
        if (c >= L.n2) continue;
        const long long id = ((long long)a * L.n1 + b) * L.n2 + c;
        const float s = nsum(L, L.u, a, b, c);
        const float v = (s + L.f[id] * L.inv_scale) * (1.0f / 6.0f);
        L.u[id] = (1.0f - omega) * L.u[id] + omega * v;
    }
}

// Weighted Jacobi sweep into r, for levels whose periodic axes are odd.
__global__ void jacobi_kernel(Lv L, float omega) {
    const long long M = (long long)L.n0 * L.n1 * L.n2;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)L.n1 * L.n2)), b = (int)((id / L.n2) % L.n1), c = (int)(id % L.n2);
        const float v = (nsum(L, L.u, a, b, c) + L.f[id] * L.inv_scale) * (1.0f / 6.0f);
        L.r[id] = (1.0f - omega) * L.u[id] + omega * v;
    }
}

__global__ void residual_kernel(Lv L) {
    const long long M = (long long)L.n0 * L.n1 * L.n2;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)L.n1 * L.n2)), b = (int)((id / L.n2) % L.n1), c = (int)(id % L.n2);
        L.r[id] = L.f[id] - (6.0f * L.u[id] - nsum(L, L.u, a, b, c)) / L.inv_scale;
    }
}

// fine index of coarse index I along an axis
__device__ __forceinline__ int fine_of(int I, int per) { return per ? 2 * I : 2 * I + 1; }

// Full weighting (1/4, 1/2, 1/4 per axis) of the fine residual.
__global__ void restrict_kernel(Lv F, Lv C) {
    const long long M = (long long)C.n0 * C.n1 * C.n2;
    const float w[3] = {0.25f, 0.5f, 0.25f};
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int A = (int)(id / ((long long)C.n1 * C.n2)), B = (int)((id / C.n2) % C.n1), Cc = (int)(id % C.n2);
        const int fa = fine_of(A, F.p0), fb = fine_of(B, F.p1), fc = fine_of(Cc, F.p2);
        float s = 0.0f;
        for (int da = -1; da <= 1; ++da) {
            int a = fa + da;
            if (a < 0) { if (!F.p0) continue; a += F.n0; } else if (a >= F.n0) { if (!F.p0) continue; a -= F.n0; }
            for (int db = -1; db <= 1; ++db) {
                int b = fb + db;
                if (b < 0) { if (!F.p1) continue; b += F.n1; } else if (b >= F.n1) { if (!F.p1) continue; b -= F.n1; }
                const float wab = w[da + 1] * w[db + 1];
                const long long rowb = ((long long)a * F.n1 + b) * F.n2;
                for (int dc = -1; dc <= 1; ++dc) {
                    int c = fc + dc;
                    if (c < 0) { if (!F.p2) continue; c += F.n2; } else if (c >= F.n2) { if (!F.p2) continue; c -= F.n2; }
                    s += wab * w[dc + 1] * F.r[rowb + c];
                }
            }
        }
        C.f[id] = s;
    }
}

// Coarse sources of a fine index: up to two (coarse index, weight) pairs.
__device__ __forceinline__ int coarse_src(int f, int per, int nc, int* I, float* w) {
    if (per) {
        if ((f & 1) == 0) { I[0] = f / 2; w[0] = 1.0f; return 1; }
        I[0] = f / 2; w[0] = 0.5f; I[1] = (f / 2 + 1) % nc; w[1] = 0.5f; return 2;
    }
    if (f & 1) { I[0] = (f - 1) / 2; w[0] = 1.0f; return I[0] < nc ? 1 : 0; }
    int k = 0;
    const int hi = f / 2, lo = hi - 1;
    if (lo >= 0) { I[k] = lo; w[k] = 0.5f; ++k; }
    if (hi < nc) { I[k] = hi; w[k] = 0.5f; ++k; }
    return k;
}

// Trilinear prolongation added into the fine correction.
__global__ void prolong_kernel(Lv C, Lv F) {
    const long long M = (long long)F.n0 * F.n1 * F.n2;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)F.n1 * F.n2)), b = (int)((id / F.n2) % F.n1), c = (int)(id % F.n2);
        int Ia[2], Ib[2], Ic[2];
        float wa[2], wb[2], wc[2];
        const int na = coarse_src(a, F.p0, C.n0, Ia, wa), nbv = coarse_src(b, F.p1, C.n1, Ib, wb),
                  nc = coarse_src(c, F.p2, C.n2, Ic, wc);
        float s = 0.0f;
        for (int x = 0; x < na; ++x)
            for (int y = 0; y < nbv; ++y) {
                const long long row = ((long long)Ia[x] * C.n1 + Ib[y]) * C.n2;
                for (int z = 0; z < nc; ++z) s += wa[x] * wb[y] * wc[z] * C.u[row + Ic[z]];
            }
        F.u[id] += s;
    }
}

// Coarsest level in one CTA, FP64 in shared memory: red-black Gauss-Seidel
// (or Jacobi when a periodic axis is odd) for `sweeps` sweeps; with every axis
// periodic the mean of f is removed first and the mean of u afterwards.
__global__ void coarse_kernel(Lv L, int sweeps, int allper, int rb) {
    extern __shared__ double sm[];
    const int M = L.n0 * L.n1 * L.n2;
    double* u = sm;
    double* f = sm + M;
    double* tmp = sm + 2 * M;
    __shared__ double red[32];
    __shared__ double mean;
    for (int t = threadIdx.x; t < M; t += blockDim.x) { u[t] = 0.0; f[t] = (double)L.f[t] * L.inv_scale; }
    __syncthreads();
    if (allper) {
        double s = 0.0;
        for (int t = threadIdx.x; t < M; t += blockDim.x) s += f[t];
        for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) { double q = 0; for (int w = 0; w < (int)(blockDim.x >> 5); ++w) q += red[w]; mean = q / M; }
        __syncthreads();
        for (int t = threadIdx.x; t < M; t += blockDim.x) f[t] -= mean;
        __syncthreads();
    }
    auto nsum_d = [&](const double* v, int a, int b, int c) {
        double s = 0.0;
        const int d0[6] = {-1, 1, 0, 0, 0, 0}, d1[6] = {0, 0, -1, 1, 0, 0}, d2[6] = {0, 0, 0, 0, -1, 1};
        for (int q = 0; q < 6; ++q) {
            int x = a + d0[q], y = b + d1[q], z = c + d2[q];
            if (x < 0) { if (!L.p0) continue; x += L.n0; } else if (x >= L.n0) { if (!L.p0) continue; x -= L.n0; }
            if (y < 0) { if (!L.p1) continue; y += L.n1; } else if (y >= L.n1) { if (!L.p1) continue; y -= L.n1; }
            if (z < 0) { if (!L.p2) continue; z += L.n2; } else if (z >= L.n2) { if (!L.p2) continue; z -= L.n2; }
            s += v[(x * L.n1 + y) * L.n2 + z];
        }
        return s;
    };
    for (int sw = 0; sw < sweeps; ++sw) {
        if (rb) {
            for (int color = 0; color < 2; ++color) {
                for (int t = threadIdx.x; t < M; t += blockDim.x) {
                    const int a = t / (L.n1 * L.n2), b = (t / L.n2) % L.n1, c = t % L.n2;
                    if (((a + b + c) & 1) != color) continue;
                    u[t] = (nsum_d(u, a, b, c) + f[t]) / 6.0;
                }
                __syncthreads();
            }
        } else {
            for (int t = threadIdx.x; t < M; t += blockDim.x) {
                const int a = t / (L.n1 * L.n2), b = (t / L.n2) % L.n1, c = t % L.n2;
                tmp[t] = 0.2 * u[t] + 0.8 * (nsum_d(u, a, b, c) + f[t]) / 6.0;
            }
            __syncthreads();
            for (int t = threadIdx.x; t < M; t += blockDim.x) u[t] = tmp[t];
            __syncthreads();
        }
    }
    if (allper) {
        double s = 0.0;
        for (int t = threadIdx.x; t < M; t += blockDim.x) s += u[t];
        for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) { double q = 0; for (int w = 0; w < (int)(blockDim.x >> 5); ++w) q += red[w]; mean = q / M; }
        __syncthreads();
        for (int t = threadIdx.x; t < M; t += blockDim.x) u[t] -= mean;
        __syncthreads();
    }
    for (int t = threadIdx.x; t < M; t += blockDim.x) L.u[t] = (float)u[t];
}

// ---- FP64 outer loop on the glue-layout arrays ----
struct Outer {
    int cx, cy, cz;
    int n0, n1, n2;       // unknowns per axis (= level 0)
    int o0, o1, o2;       // glue index of unknown 0
    int p0, p1, p2;       // periodic axes
    int nref0, nref1, nref2;
    double inv_eps0;
    double fmean;         // removed from f when every axis is periodic
};

__device__ __forceinline__ long long gl(const Outer& O, int i, int j, int k) {
    return ((long long)i * O.cy + j) * O.cz + k;
}
__device__ __forceinline__ int wrapn(int idx, int per, int nref) {
    if (per) { if (idx == 0) return nref; if (idx == nref + 1) return 1; }
    return idx;
}

__device__ __forceinline__ double bsum(double v, double* red) {
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

// Per-block partial sums of f and f^2 over the unknown nodes.
__global__ void fstats_kernel(Outer O, const double* rho0, double* partial) {
    __shared__ double red[32];
    const long long M = (long long)O.n0 * O.n1 * O.n2;
    double s = 0.0, s2 = 0.0;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)O.n1 * O.n2)), b = (int)((id / O.n2) % O.n1), c = (int)(id % O.n2);
        const double f = rho0[gl(O, a + O.o0, b + O.o1, c + O.o2)] * O.inv_eps0;
        s += f; s2 += f * f;
    }
    s = bsum(s, red);
    s2 = bsum(s2, red);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s; partial[2 * blockIdx.x + 1] = s2; }
}

// r = f - A phi in FP64; stores r to the level-0 right-hand side (FP32) and
// per-block partial sums of r^2.
__global__ void outer_residual_kernel(Outer O, const double* rho0, const double* phi, float* f0, double* partial) {
    __shared__ double red[32];
    const long long M = (long long)O.n0 * O.n1 * O.n2;
    double s2 = 0.0;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)O.n1 * O.n2)), b = (int)((id / O.n2) % O.n1), c = (int)(id % O.n2);
        const int i = a + O.o0, j = b + O.o1, k = c + O.o2;
        const double p = phi[gl(O, i, j, k)];
        const double s = phi[gl(O, wrapn(i - 1, O.p0, O.nref0), j, k)] + phi[gl(O, wrapn(i + 1, O.p0, O.nref0), j, k)] +
                         phi[gl(O, i, wrapn(j - 1, O.p1, O.nref1), k)] + phi[gl(O, i, wrapn(j + 1, O.p1, O.nref1), k)] +
                         phi[gl(O, i, j, wrapn(k - 1, O.p2, O.nref2))] + phi[gl(O, i, j, wrapn(k + 1, O.p2, O.nref2))];
        const double r = (rho0[gl(O, i, j, k)] * O.inv_eps0 - O.fmean) - (6.0 * p - s);
        f0[id] = (float)r;
        s2 += r * r;
    }
    s2 = bsum(s2, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s2;
}

__global__ void correct_kernel(Outer O, double* phi, const float* e) {
    const long long M = (long long)O.n0 * O.n1 * O.n2;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)O.n1 * O.n2)), b = (int)((id / O.n2) % O.n1), c = (int)(id % O.n2);
        phi[gl(O, a + O.o0, b + O.o1, c + O.o2)] += (double)e[id];
    }
}

__global__ void phi_mean_kernel(Outer O, const double* phi, double* partial) {
    __shared__ double red[32];
    const long long M = (long long)O.n0 * O.n1 * O.n2;
    double s = 0.0;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)O.n1 * O.n2)), b = (int)((id / O.n2) % O.n1), c = (int)(id % O.n2);
        s += phi[gl(O, a + O.o0, b + O.o1, c + O.o2)];
    }
    s = bsum(s, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void phi_shift_kernel(Outer O, double* phi, const double* sum) {
    const long long M = (long long)O.n0 * O.n1 * O.n2;
    const double m = *sum / (double)M;
    for (long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x; id < M; id += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(id / ((long long)O.n1 * O.n2)), b = (int)((id / O.n2) % O.n1), c = (int)(id % O.n2);
        phi[gl(O, a + O.o0, b + O.o1, c + O.o2)] -= m;
    }
}

// Deterministic sum of per-block partials (stride values apart) into out.
__global__ void reduce_partials_kernel(const double* partial, int n, int stride, int off, double* out) {
    __shared__ double red[32];
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) v += partial[t * stride + off];
    v = bsum(v, red);
    if (threadIdx.x == 0) *out = v;
}

Outer make_outer(const Ctx& c) {
    Outer O;
    O.cx = c.cx; O.cy = c.cy; O.cz = c.cz;
    const MGLevel& m = c.mg[0];
    O.n0 = m.n[0]; O.n1 = m.n[1]; O.n2 = m.n[2];
    O.p0 = m.per[0]; O.p1 = m.per[1]; O.p2 = m.per[2];
    O.o0 = O.p0 ? 1 : 2; O.o1 = O.p1 ? 1 : 2; O.o2 = O.p2 ? 1 : 2;
    O.nref0 = c.nx; O.nref1 = c.ny; O.nref2 = c.nz;
    O.inv_eps0 = 1.0 / c.p.eps0;
    O.fmean = 0.0;
    return O;
}

bool level_rb(const MGLevel& m) {
    for (int a = 0; a < 3; ++a) if (m.per[a] && (m.n[a] & 1)) return false;
    return true;
}

void smooth(Ctx& c, int l, int sweeps) {
    MGLevel& m = c.mg[l];
    const Lv L = lv(m);
    if (level_rb(m)) {
        const long long half = (long long)m.n[0] * m.n[1] * ((m.n[2] + 1) / 2);
        for (int s = 0; s < sweeps; ++s)
            for (int color = 0; color < 2; ++color) {
                ++c.launches;
                rb_smooth_kernel<<<nblocks(half), kT, 0, c.st>>>(L, color, 1.0f);
            }
    } else {
        for (int s = 0; s < sweeps; ++s) {
            ++c.launches;
            jacobi_kernel<<<nblocks((long long)m.size()), kT, 0, c.st>>>(L, 0.8f);
            FOPIS_CUDA(cudaMemcpyAsync(m.u, m.r, sizeof(float) * m.size(), cudaMemcpyDeviceToDevice, c.st));
        }
    }
    FOPIS_LAUNCH_CHECK();
}

void coarse_solve(Ctx& c, int l) {
    MGLevel& m = c.mg[l];
    const int M = (int)m.size();
    const bool allper = m.per[0] && m.per[1] && m.per[2];
    const int nmax = std::max({m.n[0], m.n[1], m.n[2]});
    const int sweeps = std::min(4000, std::max(30, 2 * nmax * nmax));
    if (M <= kCoarseMax) {
        const size_t smem = sizeof(double) * 3 * M;
        ++c.launches;
        coarse_kernel<<<1, 1024, smem, c.st>>>(lv(m), sweeps, allper ? 1 : 0, level_rb(m) ? 1 : 0);
        FOPIS_LAUNCH_CHECK();
    } else {
        FOPIS_CUDA(cudaMemsetAsync(m.u, 0, sizeof(float) * M, c.st));
        smooth(c, l, std::min(sweeps, 400));
    }
}

void vcycle(Ctx& c, int l) {
    const int L = (int)c.mg.size();
    if (l == L - 1) { coarse_solve(c, l); return; }
    MGLevel& m = c.mg[l];
    MGLevel& n = c.mg[l + 1];
    FOPIS_CUDA(cudaMemsetAsync(m.u, 0, sizeof(float) * m.size(), c.st));
    smooth(c, l, 2);
    ++c.launches;
    residual_kernel<<<nblocks((long long)m.size()), kT, 0, c.st>>>(lv(m));
    ++c.launches;
    restrict_kernel<<<nblocks((long long)n.size()), kT, 0, c.st>>>(lv(m), lv(n));
    FOPIS_LAUNCH_CHECK();
    vcycle(c, l + 1);
    ++c.launches;
    prolong_kernel<<<nblocks((long long)m.size()), kT, 0, c.st>>>(lv(n), lv(m));
    FOPIS_LAUNCH_CHECK();
    smooth(c, l, 2);
}

double read_red(Ctx& c, int slot) {
    double v = 0.0;
    FOPIS_CUDA(cudaMemcpyAsync(&v, &c.d_sc->red[slot], sizeof(double), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    return v;
}

}  // namespace

void mg_setup(Ctx& c) {
    mg_free(c);
    MGLevel m;
    const int nref[3] = {c.nx, c.ny, c.nz};
    for (int a = 0; a < 3; ++a) {
        const bool lo = c.per[2 * a], hi = c.per[2 * a + 1];
        if (lo != hi) throw ApiError{FOPIS_ERR_ARG, "an axis must be periodic on both sides or on neither"};
        m.per[a] = lo ? 1 : 0;
        m.n[a] = lo ? nref[a] : nref[a] - 2;
        if (m.n[a] < 1) throw ApiError{FOPIS_ERR_ARG, "grid too small for the Poisson solve"};
    }
    m.scale = 1.0;
    c.mg.push_back(m);
    for (;;) {
        const MGLevel& f = c.mg.back();
        bool ok = f.size() > 64;
        for (int a = 0; a < 3; ++a) {
            if (f.per[a]) ok = ok && (f.n[a] % 2 == 0) && f.n[a] >= 4;
            else ok = ok && f.n[a] >= 3;
        }
        if (!ok) break;
        MGLevel n;
        for (int a = 0; a < 3; ++a) { n.per[a] = f.per[a]; n.n[a] = f.n[a] / 2; }
        n.scale = f.scale * 0.25;
        c.mg.push_back(n);
    }
    for (auto& l : c.mg) {
        FOPIS_CUDA(cudaMalloc(&l.u, sizeof(float) * l.size()));
        FOPIS_CUDA(cudaMalloc(&l.f, sizeof(float) * l.size()));
        FOPIS_CUDA(cudaMalloc(&l.r, sizeof(float) * l.size()));
        FOPIS_CUDA(cudaMemset(l.u, 0, sizeof(float) * l.size()));
    }
    const MGLevel& last = c.mg.back();
    if ((int)last.size() <= kCoarseMax) {
        const size_t smem = sizeof(double) * 3 * last.size();
        if (smem > 48 * 1024)
            FOPIS_CUDA(cudaFuncSetAttribute(coarse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    c.red_blocks = kRedBlocks;
    FOPIS_CUDA(cudaMalloc(&c.red_partials, sizeof(double) * 2 * 148 * 8));
}

void mg_free(Ctx& c) {
    for (auto& l : c.mg) { cudaFree(l.u); cudaFree(l.f); cudaFree(l.r); }
    c.mg.clear();
    if (c.red_partials) { cudaFree(c.red_partials); c.red_partials = nullptr; }
}

int mg_solve(Ctx& c, double tol, int max_cycles) {
    Outer O = make_outer(c);
    const bool allper = O.p0 && O.p1 && O.p2;
    const long long M = (long long)O.n0 * O.n1 * O.n2;
    ++c.launches;
    fstats_kernel<<<kRedBlocks, kT, 0, c.st>>>(O, c.rho0, c.red_partials);
    ++c.launches;
    reduce_partials_kernel<<<1, 1024, 0, c.st>>>(c.red_partials, kRedBlocks, 2, 0, &c.d_sc->red[0]);
    ++c.launches;
    reduce_partials_kernel<<<1, 1024, 0, c.st>>>(c.red_partials, kRedBlocks, 2, 1, &c.d_sc->red[1]);
    FOPIS_LAUNCH_CHECK();
    FOPIS_CUDA(cudaMemcpyAsync(c.h_sc->red, c.d_sc->red, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    const double fsum = c.h_sc->red[0], fsq = c.h_sc->red[1];
    if (allper) O.fmean = fsum / (double)M;
    double fnorm = std::sqrt(std::max(0.0, fsq - (allper ? fsum * fsum / (double)M : 0.0)));
    if (!(fnorm > 0.0)) fnorm = 1.0;
    auto residual = [&]() {
        ++c.launches;
        outer_residual_kernel<<<kRedBlocks, kT, 0, c.st>>>(O, c.rho0, c.phi, c.mg[0].f, c.red_partials);
        ++c.launches;
        reduce_partials_kernel<<<1, 1024, 0, c.st>>>(c.red_partials, kRedBlocks, 1, 0, &c.d_sc->red[2]);
        FOPIS_LAUNCH_CHECK();
        return std::sqrt(read_red(c, 2));
    };
    double res = residual();
    c.first_res = res / fnorm;
    int cycles = 0;
    while (res > tol * fnorm && cycles < max_cycles) {
        vcycle(c, 0);
        ++c.launches;
        correct_kernel<<<nblocks(M), kT, 0, c.st>>>(O, c.phi, c.mg[0].u);
        FOPIS_LAUNCH_CHECK();
        res = residual();
        ++cycles;
        if (!std::isfinite(res)) break;
    }
    if (allper) {
        ++c.launches;
        phi_mean_kernel<<<kRedBlocks, kT, 0, c.st>>>(O, c.phi, c.red_partials);
        ++c.launches;
        reduce_partials_kernel<<<1, 1024, 0, c.st>>>(c.red_partials, kRedBlocks, 1, 0, &c.d_sc->red[3]);
        ++c.launches;
        phi_shift_kernel<<<nblocks(M), kT, 0, c.st>>>(O, c.phi, &c.d_sc->red[3]);
        FOPIS_LAUNCH_CHECK();
    }
    phi_boundary(c);
    c.last_vcycles = cycles;
    c.last_res = res / fnorm;
    c.last_converged = (res <= tol * fnorm) ? 1 : 0;
    c.step_vcycles += cycles;
    c.step_solves += 1;
    if (!std::isfinite(res)) return FOPIS_ERR_DEVICE;
    return c.last_converged ? FOPIS_OK : FOPIS_ERR_NOT_CONVERGED;
}

}  // namespace fopis
