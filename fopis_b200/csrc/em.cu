// em.cu — the field side of the EM mode (FOPIS_SOLVER_EM): the FDTD updates of
// E and B on a Yee grid with damping layers (RootGrid::updateEfieldFDTDDamping /
// updateBfieldDamping, src/Grid/RootGrid/RootGridField.cpp:594-820), the
// periodic glue copies and folds, the nodal reference fields the particle
// gather reads, the field energies and the exports.
//
// Layout. The six Yee arrays are boost::multi_arrays with index bases in the
// reference (RootGrid::initializeField, RootGridField.cpp:7-39): every axis
// that is not periodic on a side extends L = (that axis' node count) indices
// beyond it. Each is one FP64 array in C order over its own extent (YeeArr).
// At 128^3 with six non-periodic faces that is 389^3 cells per component,
// 2.8 GB for the six; the updates are streaming stencils (one thread per
// index, k fastest), bound by HBM.
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace fopis {

namespace {

constexpr int kT = 256;

struct Yee {
    double* v;
    int lo0, lo1, lo2, n1, n2;
    __device__ __forceinline__ double& at(int i, int j, int k) const {
        return v[((long long)(i - lo0) * n1 + (j - lo1)) * n2 + (k - lo2)];
    }
};
Yee view(const YeeArr& a) { return Yee{a.v, a.lo[0], a.lo[1], a.lo[2], a.n[1], a.n[2]}; }

struct Geo {
    int c[3];      // nodes with glue
    int L[3];      // damping lengths
    int lo[3];     // first index of the extended grid per axis
    int up[3];     // one past the last
    int per[3];    // axis periodic
    const double* mask[3];   // per-axis damping factor of index i at mask[a][i - lo[a]]
};
Geo make_geo(const Ctx& c) {
    Geo g;
    g.c[0] = c.cx; g.c[1] = c.cy; g.c[2] = c.cz;
    size_t off = 0;
    for (int a = 0; a < 3; ++a) {
        g.L[a] = c.em.L[a]; g.lo[a] = c.em.lo[a]; g.up[a] = c.em.up[a]; g.per[a] = c.per[2 * a];
        g.mask[a] = c.em.mask + off;
        off += (size_t)(g.up[a] - g.lo[a]);
    }
    return g;
}

int blocks(long long n) {
    const long long b = (n + kT - 1) / kT;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 32));
}

// The masking factor of the damping forms (RootGridField.cpp:628-642, 742-756):
// per axis 1 - (d / L)^2, d = the index's distance from the real grid [1, real-2]
// (masking_parameter 1), evaluated once per index into a table on the host
// (damp1), multiplied over the three axes on the device.
double damp1(int r, int L, int real) {
    const double d = (r <= 0) ? -(double)r + 1.0 : (r >= real - 1) ? (double)r - (double)real + 2.0 : 0.0;
    const double q = 1.0 * d / (double)L;
    return 1.0 - q * q;
}
__device__ __forceinline__ double damp(const Geo& g, int i, int j, int k) {
    return __ldg(g.mask[0] + (i - g.lo[0])) * __ldg(g.mask[1] + (j - g.lo[1])) * __ldg(g.mask[2] + (k - g.lo[2]));
}
__device__ __forceinline__ bool real_region(const Geo& g, int i, int j, int k) {
    return i > 0 && i < g.c[0] - 1 && j > 0 && j < g.c[1] - 1 && k > 0 && k < g.c[2] - 1;
}

// Index (i, j, k) of the interior [lo+1, up-1) of the extended grid.
__device__ __forceinline__ void interior_index(const Geo& g, long long t, int& i, int& j, int& k) {
    const int d1 = g.up[1] - g.lo[1] - 2, d2 = g.up[2] - g.lo[2] - 2;
    i = g.lo[0] + 1 + (int)(t / ((long long)d1 * d2));
    j = g.lo[1] + 1 + (int)((t / d2) % d1);
    k = g.lo[2] + 1 + (int)(t % d2);
}

// RootGrid::updateEfieldFDTDDamping's loop (RootGridField.cpp:643-701): on the
// real edges below the last one of their direction E += -J dt/eps0 + C curl B,
// elsewhere E = mask (E + C curl B); the last index of each direction in the
// damping layers is left alone. C = dt / (mu0 eps0 dx).
__global__ void fdtd_e_kernel(Yee ex, Yee ey, Yee ez, Yee bx, Yee by, Yee bz, const double* __restrict__ jx,
                              const double* __restrict__ jy, const double* __restrict__ jz, Geo g, double dte,
                              double C) {
    const long long M = (long long)(g.up[0] - g.lo[0] - 2) * (g.up[1] - g.lo[1] - 2) * (g.up[2] - g.lo[2] - 2);
    const int cx = g.c[0], cy = g.c[1], cz = g.c[2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < M; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        interior_index(g, t, i, j, k);
        const bool real = real_region(g, i, j, k);
        if (real ? true : i < g.up[0] - 2) {
            const double cv = bz.at(i, j, k) - bz.at(i, j - 1, k) - by.at(i, j, k) + by.at(i, j, k - 1);
            double& e = ex.at(i, j, k);
            if (real && i < cx - 2) e = e - jx[((long long)i * cy + j) * cz + k] * dte + C * cv;
            else e = 0.5 * (damp(g, i, j, k) + damp(g, i + 1, j, k)) * (e + C * cv);
        }
        if (real ? true : j < g.up[1] - 2) {
            const double cv = bx.at(i, j, k) - bx.at(i, j, k - 1) - bz.at(i, j, k) + bz.at(i - 1, j, k);
            double& e = ey.at(i, j, k);
            if (real && j < cy - 2) e = e - jy[((long long)i * (cy - 1) + j) * cz + k] * dte + C * cv;
            else e = 0.5 * (damp(g, i, j, k) + damp(g, i, j + 1, k)) * (e + C * cv);
        }
        if (real ? true : k < g.up[2] - 2) {
            const double cv = by.at(i, j, k) - by.at(i - 1, j, k) - bx.at(i, j, k) + bx.at(i, j - 1, k);
            double& e = ez.at(i, j, k);
            if (real && k < cz - 2) e = e - jz[((long long)i * cy + j) * (cz - 1) + k] * dte + C * cv;
            else e = 0.5 * (damp(g, i, j, k) + damp(g, i, j, k + 1)) * (e + C * cv);
        }
    }
}

// RootGrid::updateBfieldDamping's loop (RootGridField.cpp:758-816): B += dt/dx
// (dE/dz - dE/dy ...) on the real faces except the last of the two directions
// across them, masked there and in the damping layers (whose last index of
// those directions is left alone).
__global__ void fdtd_b_kernel(Yee bx, Yee by, Yee bz, Yee ex, Yee ey, Yee ez, Geo g, double d) {
    const long long M = (long long)(g.up[0] - g.lo[0] - 2) * (g.up[1] - g.lo[1] - 2) * (g.up[2] - g.lo[2] - 2);
    const int X = g.c[0], Y = g.c[1], Z = g.c[2];
    const int xm = g.up[0] - 2, ym = g.up[1] - 2, zm = g.up[2] - 2;   // max_x/y/z_index - 2
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < M; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        interior_index(g, t, i, j, k);
        const bool real = real_region(g, i, j, k);
        if (real || (j != ym && k != zm)) {
            const double gv = (ey.at(i, j, k + 1) - ey.at(i, j, k)) - (ez.at(i, j + 1, k) - ez.at(i, j, k));
            double& b = bx.at(i, j, k);
            if (real && j != Y - 2 && k != Z - 2) b = b + d * gv;
            else b = 0.25 * (damp(g, i, j, k) + damp(g, i, j + 1, k) + damp(g, i, j, k + 1) + damp(g, i, j + 1, k + 1)) *
                     (b + d * gv);
        }
        if (real || (i != xm && k != zm)) {
            const double gv = (ez.at(i + 1, j, k) - ez.at(i, j, k)) - (ex.at(i, j, k + 1) - ex.at(i, j, k));
            double& b = by.at(i, j, k);
            if (real && i != X - 2 && k != Z - 2) b = b + d * gv;
            else b = 0.25 * (damp(g, i, j, k) + damp(g, i + 1, j, k) + damp(g, i, j, k + 1) + damp(g, i + 1, j, k + 1)) *
                     (b + d * gv);
        }
        if (real || (i != xm && j != ym)) {
            const double gv = (ex.at(i, j + 1, k) - ex.at(i, j, k)) - (ey.at(i + 1, j, k) - ey.at(i, j, k));
            double& b = bz.at(i, j, k);
            if (real && i != X - 2 && j != Y - 2) b = b + d * gv;
            else b = 0.25 * (damp(g, i, j, k) + damp(g, i + 1, j, k) + damp(g, i, j + 1, k) + damp(g, i + 1, j + 1, k)) *
                     (b + d * gv);
        }
    }
}

// Communicator::sendRecvFieldX/Y/Z self branch (Communicator.cpp:265-343) on a
// Yee array along one periodic axis (index base 0 there): index 0 <- index
// m-2, index m-1 <- index 1, over the whole extent of the other two axes.
__global__ void yee_glue_kernel(Yee a, int n0, int axis) {
    const int n[3] = {n0, a.n1, a.n2};
    const int lo[3] = {a.lo0, a.lo1, a.lo2};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const long long plane = (long long)n[a1] * n[a2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < plane; t += (long long)gridDim.x * blockDim.x) {
        int p[3];
        p[a1] = lo[a1] + (int)(t / n[a2]);
        p[a2] = lo[a2] + (int)(t % n[a2]);
        const int m = n[axis];
        p[axis] = 1; const double v1 = a.at(p[0], p[1], p[2]);
        p[axis] = m - 2; const double vm2 = a.at(p[0], p[1], p[2]);
        p[axis] = 0; a.at(p[0], p[1], p[2]) = vm2;
        p[axis] = m - 1; a.at(p[0], p[1], p[2]) = v1;
    }
}

// Communicator::sendRecvScalarX/Y/Z self branch (Communicator.cpp:497-574)
// along one periodic axis of an edge current of dims d[3]: planes g-1-t and
// size-1-t (t < g) both become their sum (MPIw::Environment::sendRecvEdgeScalar,
// Environment.cpp:74-130: g = 2 along the current's direction, 1 across it).
__global__ void edge_fold_kernel(double* a, int d0, int d1, int d2, int axis, int glue) {
    const int d[3] = {d0, d1, d2};
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    const long long plane = (long long)d[a1] * d[a2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < plane; t += (long long)gridDim.x * blockDim.x) {
        int p[3];
        p[a1] = (int)(t / d[a2]);
        p[a2] = (int)(t % d[a2]);
        for (int q = 0; q < glue; ++q) {
            p[axis] = glue - 1 - q; const long long lo = ((long long)p[0] * d1 + p[1]) * d2 + p[2];
            p[axis] = d[axis] - 1 - q; const long long hi = ((long long)p[0] * d1 + p[1]) * d2 + p[2];
            const double s = a[lo] + a[hi];
            a[lo] = s;
            a[hi] = s;
        }
    }
}

// RootGrid::updateEfield (RootGridField.cpp:456-487) into the EM arrays: the
// edges of the glue grid from phi; the damping layers keep their values.
__global__ void e_from_phi_kernel(Yee ex, Yee ey, Yee ez, const double* __restrict__ phi, Geo g) {
    const int X = g.c[0], Y = g.c[1], Z = g.c[2];
    const long long N = (long long)X * Y * Z;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / ((long long)Y * Z)), j = (int)((t / Z) % Y), k = (int)(t % Z);
        const double p = phi[t];
        if (i < X - 1) ex.at(i, j, k) = p - phi[t + (long long)Y * Z];
        if (j < Y - 1) ey.at(i, j, k) = p - phi[t + Z];
        if (k < Z - 1) ez.at(i, j, k) = p - phi[t + 1];
    }
}

// A node index of a periodic axis mapped onto the interior image it receives
// from the glue copies; -1 for a glue node of a non-periodic axis (which the
// reference's nodal updates never write: zero).
__device__ __forceinline__ int node_image(const Geo& g, int axis, int idx) {
    const int c = g.c[axis];
    if (idx == 0) return g.per[axis] ? c - 2 : -1;
    if (idx == c - 1) return g.per[axis] ? 1 : -1;
    return idx;
}

__device__ __forceinline__ void store_node(float4* o, double x, double y, double z) {
    *o = make_float4((float)x, (float)y, (float)z, 0.0f);
}
__device__ __forceinline__ void store_node(Vec4d* o, double x, double y, double z) { *o = Vec4d{x, y, z, 0.0}; }

// RootGrid::updateReferenceEfield (RootGridField.cpp:489-582) on the Yee edges:
// nodal means of the two edges of each direction, on a non-periodic face's
// node 1 (and c-2) the one-sided second-order difference of phi, then the
// periodic glue copies (every glue node takes its image's value).
template <typename Out>
__global__ void eref_kernel(Yee ex, Yee ey, Yee ez, const double* __restrict__ phi, Geo g, Out* out,
                            double* eref, long long N) {
    const int X = g.c[0], Y = g.c[1], Z = g.c[2];
    const long long sx = (long long)Y * Z, sy = Z;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = node_image(g, 0, (int)(t / sx)), j = node_image(g, 1, (int)((t / Z) % Y)),
                  k = node_image(g, 2, (int)(t % Z));
        double e[3] = {0.0, 0.0, 0.0};
        if (i >= 0 && j >= 0 && k >= 0) {
            const long long q = i * sx + j * sy + k;
            if (!g.per[0] && i == 1) e[0] = 0.5 * (phi[q + 2 * sx] - 4.0 * phi[q + sx] + 3.0 * phi[q]);
            else if (!g.per[0] && i == X - 2) e[0] = 0.5 * (-phi[q - 2 * sx] + 4.0 * phi[q - sx] - 3.0 * phi[q]);
            else e[0] = 0.5 * (ex.at(i - 1, j, k) + ex.at(i, j, k));
            if (!g.per[1] && j == 1) e[1] = 0.5 * (phi[q + 2 * sy] - 4.0 * phi[q + sy] + 3.0 * phi[q]);
            else if (!g.per[1] && j == Y - 2) e[1] = 0.5 * (-phi[q - 2 * sy] + 4.0 * phi[q - sy] - 3.0 * phi[q]);
            else e[1] = 0.5 * (ey.at(i, j - 1, k) + ey.at(i, j, k));
            if (!g.per[2] && k == 1) e[2] = 0.5 * (phi[q + 2] - 4.0 * phi[q + 1] + 3.0 * phi[q]);
            else if (!g.per[2] && k == Z - 2) e[2] = 0.5 * (-phi[q - 2] + 4.0 * phi[q - 1] - 3.0 * phi[q]);
            else e[2] = 0.5 * (ez.at(i, j, k - 1) + ez.at(i, j, k));
        }
        store_node(out + t, e[0], e[1], e[2]);
        eref[t] = e[0]; eref[N + t] = e[1]; eref[2 * N + t] = e[2];
    }
}

// RootGrid::updateReferenceBfield (RootGridField.cpp:1102-1127): nodal means of
// the four faces around each node, then the periodic glue copies.
template <typename Out>
__global__ void bref_kernel(Yee bx, Yee by, Yee bz, Geo g, Out* out, double* bref, long long N) {
    const int Y = g.c[1], Z = g.c[2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = node_image(g, 0, (int)(t / ((long long)Y * Z))), j = node_image(g, 1, (int)((t / Z) % Y)),
                  k = node_image(g, 2, (int)(t % Z));
        double b[3] = {0.0, 0.0, 0.0};
        if (i >= 0 && j >= 0 && k >= 0) {
            b[0] = 0.25 * (bx.at(i, j, k) + bx.at(i, j - 1, k) + bx.at(i, j, k - 1) + bx.at(i, j - 1, k - 1));
            b[1] = 0.25 * (by.at(i, j, k) + by.at(i - 1, j, k) + by.at(i, j, k - 1) + by.at(i - 1, j, k - 1));
            b[2] = 0.25 * (bz.at(i, j, k) + bz.at(i - 1, j, k) + bz.at(i, j - 1, k) + bz.at(i - 1, j - 1, k));
        }
        store_node(out + t, b[0], b[1], b[2]);
        bref[t] = b[0]; bref[N + t] = b[1]; bref[2 * N + t] = b[2];
    }
}

// RootGrid::updateReferenceCurrent (RootGridField.cpp:1256-1285), one direction:
// nodal mean of the two edges, then the periodic glue copies.
__global__ void jref_kernel(const double* __restrict__ jd, int dir, Geo g, double* out, long long N) {
    const int X = g.c[0], Y = g.c[1], Z = g.c[2];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int i = node_image(g, 0, (int)(t / ((long long)Y * Z))), j = node_image(g, 1, (int)((t / Z) % Y)),
                  k = node_image(g, 2, (int)(t % Z));
        double v = 0.0;
        if (i >= 0 && j >= 0 && k >= 0) {
            if (dir == 0) v = 0.5 * (jd[((long long)(i - 1) * Y + j) * Z + k] + jd[((long long)i * Y + j) * Z + k]);
            else if (dir == 1) v = 0.5 * (jd[((long long)i * (Y - 1) + j - 1) * Z + k] + jd[((long long)i * (Y - 1) + j) * Z + k]);
            else v = 0.5 * (jd[((long long)i * Y + j) * (Z - 1) + k - 1] + jd[((long long)i * Y + j) * (Z - 1) + k]);
        }
        out[t] = v;
    }
    (void)X;
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

// Field::getEfieldEnergy (Field.cpp:194-213) and getBfieldEnergy (:215-234):
// sums of squares over the real grid's edges (faces); per-block partials.
__global__ void em_energy_kernel(Yee a0, Yee a1, Yee a2, Geo g, int bfield, double* partial) {
    const int X = g.c[0], Y = g.c[1], Z = g.c[2];
    const long long M = (long long)(X - 2) * (Y - 2) * (Z - 2);
    double en = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < M; t += (long long)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(t / ((long long)(Y - 2) * (Z - 2)));
        const int j = 1 + (int)((t / (Z - 2)) % (Y - 2));
        const int k = 1 + (int)(t % (Z - 2));
        if (!bfield) {
            if (i < X - 2) { const double v = a0.at(i, j, k); en += v * v; }
            if (j < Y - 2) { const double v = a1.at(i, j, k); en += v * v; }
            if (k < Z - 2) { const double v = a2.at(i, j, k); en += v * v; }
        } else {
            if (j < Y - 2 && k < Z - 2) { const double v = a0.at(i, j, k); en += v * v; }
            if (i < X - 2 && k < Z - 2) { const double v = a1.at(i, j, k); en += v * v; }
            if (i < X - 2 && j < Y - 2) { const double v = a2.at(i, j, k); en += v * v; }
        }
    }
    en = bsum(en);
    if (threadIdx.x == 0) partial[blockIdx.x] = en;
}

__global__ void em_sum_kernel(const double* partial, int n, double* out) {
    double v = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) v += partial[t];
    v = bsum(v);
    if (threadIdx.x == 0) *out = v;
}

void yee_glue(Ctx& c, const YeeArr& a) {
    for (int axis = 0; axis < 3; ++axis) {
        if (!c.per[2 * axis]) continue;
        const long long plane = axis == 0 ? (long long)a.n[1] * a.n[2]
                                          : (axis == 1 ? (long long)a.n[0] * a.n[2] : (long long)a.n[0] * a.n[1]);
        ++c.launches;
        yee_glue_kernel<<<blocks(plane), kT, 0, c.st>>>(view(a), a.n[0], axis);
        FOPIS_LAUNCH_CHECK();
    }
}

void reference_efield(Ctx& c) {
    const Geo g = make_geo(c);
    const YeeArr* f = c.em.f;
    ++c.launches;
    if (c.fp64)
        eref_kernel<Vec4d><<<blocks((long long)c.N), kT, 0, c.st>>>(view(f[0]), view(f[1]), view(f[2]), c.phi, g, c.E64,
                                                                   c.em.eref, (long long)c.N);
    else
        eref_kernel<float4><<<blocks((long long)c.N), kT, 0, c.st>>>(view(f[0]), view(f[1]), view(f[2]), c.phi, g, c.E,
                                                                    c.em.eref, (long long)c.N);
    FOPIS_LAUNCH_CHECK();
}

void reference_bfield(Ctx& c) {
    const Geo g = make_geo(c);
    const YeeArr* f = c.em.f;
    ++c.launches;
    if (c.fp64)
        bref_kernel<Vec4d><<<blocks((long long)c.N), kT, 0, c.st>>>(view(f[3]), view(f[4]), view(f[5]), g, c.em.B64,
                                                                   c.em.bref, (long long)c.N);
    else
        bref_kernel<float4><<<blocks((long long)c.N), kT, 0, c.st>>>(view(f[3]), view(f[4]), view(f[5]), g, c.em.B,
                                                                    c.em.bref, (long long)c.N);
    FOPIS_LAUNCH_CHECK();
}

long long interior_count(const Geo& g) {
    return (long long)(g.up[0] - g.lo[0] - 2) * (g.up[1] - g.lo[1] - 2) * (g.up[2] - g.lo[2] - 2);
}

double em_energy(Ctx& c, int bfield) {
    const Geo g = make_geo(c);
    const YeeArr* f = c.em.f + (bfield ? 3 : 0);
    const int nb = 148 * 4;
    ++c.launches;
    em_energy_kernel<<<nb, kT, 0, c.st>>>(view(f[0]), view(f[1]), view(f[2]), g, bfield, c.red_partials);
    ++c.launches;
    em_sum_kernel<<<1, 1024, 0, c.st>>>(c.red_partials, nb, &c.d_sc->red[14]);
    FOPIS_LAUNCH_CHECK();
    double v = 0.0;
    FOPIS_CUDA(cudaMemcpyAsync(&v, &c.d_sc->red[14], sizeof(double), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    return v;
}

}  // namespace

void em_alloc(Ctx& c) {
    EMState& e = c.em;
    e.on = true;
    e.L[0] = c.nx; e.L[1] = c.ny; e.L[2] = c.nz;   // RootGridField.cpp:17-20
    const int cc[3] = {c.cx, c.cy, c.cz};
    for (int a = 0; a < 3; ++a) {
        e.lo[a] = c.per[2 * a] ? 0 : -e.L[a];
        e.up[a] = c.per[2 * a + 1] ? cc[a] : cc[a] + e.L[a];
    }
    // ex [x_low, x_up-1) x [y_low, y_up) x [z_low, z_up), ... (RootGridField.cpp:31-37)
    const int shrink[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};
    for (int q = 0; q < 6; ++q) {
        YeeArr& y = e.f[q];
        for (int a = 0; a < 3; ++a) { y.lo[a] = e.lo[a]; y.n[a] = e.up[a] - shrink[q][a] - e.lo[a]; }
        FOPIS_CUDA(cudaMalloc(&y.v, sizeof(double) * y.size()));
        FOPIS_CUDA(cudaMemset(y.v, 0, sizeof(double) * y.size()));
    }
    const size_t nj[3] = {(size_t)(c.cx - 1) * c.cy * c.cz, (size_t)c.cx * (c.cy - 1) * c.cz,
                          (size_t)c.cx * c.cy * (c.cz - 1)};
    for (int a = 0; a < 3; ++a) {
        FOPIS_CUDA(cudaMalloc(&e.j[a], sizeof(double) * nj[a]));
        FOPIS_CUDA(cudaMemset(e.j[a], 0, sizeof(double) * nj[a]));
    }
    {   // damping factors per axis and index, [x extent][y extent][z extent] back to back
        std::vector<double> m;
        for (int a = 0; a < 3; ++a)
            for (int r = e.lo[a]; r < e.up[a]; ++r) m.push_back(damp1(r, e.L[a], cc[a]));
        FOPIS_CUDA(cudaMalloc(&e.mask, sizeof(double) * m.size()));
        FOPIS_CUDA(cudaMemcpy(e.mask, m.data(), sizeof(double) * m.size(), cudaMemcpyHostToDevice));
    }
    FOPIS_CUDA(cudaMalloc(&e.eref, sizeof(double) * 3 * c.N));
    FOPIS_CUDA(cudaMemset(e.eref, 0, sizeof(double) * 3 * c.N));
    FOPIS_CUDA(cudaMalloc(&e.bref, sizeof(double) * 3 * c.N));
    FOPIS_CUDA(cudaMemset(e.bref, 0, sizeof(double) * 3 * c.N));
    if (!c.fp64) {
        const size_t per = nj[0] + nj[1] + nj[2];
        FOPIS_CUDA(cudaMalloc(&e.jfix, sizeof(unsigned long long) * per * c.nsp));
        FOPIS_CUDA(cudaMemset(e.jfix, 0, sizeof(unsigned long long) * per * c.nsp));
    }
    if (c.fp64) {
        FOPIS_CUDA(cudaMalloc(&e.B64, sizeof(Vec4d) * c.N));
        FOPIS_CUDA(cudaMemset(e.B64, 0, sizeof(Vec4d) * c.N));
    } else {
        FOPIS_CUDA(cudaMalloc(&e.B, sizeof(float4) * c.N));
        FOPIS_CUDA(cudaMemset(e.B, 0, sizeof(float4) * c.N));
    }
}

void em_free(Ctx& c) {
    EMState& e = c.em;
    for (auto& y : e.f) { if (y.v) cudaFree(y.v); y.v = nullptr; }
    for (auto& p : e.j) { if (p) cudaFree(p); p = nullptr; }
    for (void* p : {(void*)e.eref, (void*)e.bref, (void*)e.B, (void*)e.B64, (void*)e.mask, (void*)e.jfix})
        if (p) cudaFree(p);
    e.eref = e.bref = e.mask = nullptr;
    e.jfix = nullptr;
    e.B = nullptr;
    e.B64 = nullptr;
    e.on = false;
}

void em_fold_currents(Ctx& c) {
    const int dims[3][3] = {{c.cx - 1, c.cy, c.cz}, {c.cx, c.cy - 1, c.cz}, {c.cx, c.cy, c.cz - 1}};
    for (int d = 0; d < 3; ++d)
        for (int axis = 0; axis < 3; ++axis) {
            if (!c.per[2 * axis]) continue;
            const int* n = dims[d];
            const long long plane = axis == 0 ? (long long)n[1] * n[2] : (axis == 1 ? (long long)n[0] * n[2] : (long long)n[0] * n[1]);
            ++c.launches;
            edge_fold_kernel<<<blocks(plane), kT, 0, c.st>>>(c.em.j[d], n[0], n[1], n[2], axis, axis == d ? 2 : 1);
            FOPIS_LAUNCH_CHECK();
        }
}

void em_efield_from_phi(Ctx& c) {
    const Geo g = make_geo(c);
    ++c.launches;
    e_from_phi_kernel<<<blocks((long long)c.N), kT, 0, c.st>>>(view(c.em.f[0]), view(c.em.f[1]), view(c.em.f[2]), c.phi, g);
    FOPIS_LAUNCH_CHECK();
    reference_efield(c);
}

void em_update_efield(Ctx& c) {
    const Geo g = make_geo(c);
    const YeeArr* f = c.em.f;
    const double dte = 1.0 / c.p.eps0;          // dt / eps0 (dt = 1)
    const double C = dte / (c.p.mu0 * 1.0);     // dt / (mu0 eps0 dx)
    ++c.launches;
    fdtd_e_kernel<<<blocks(interior_count(g)), kT, 0, c.st>>>(view(f[0]), view(f[1]), view(f[2]), view(f[3]), view(f[4]),
                                                              view(f[5]), c.em.j[0], c.em.j[1], c.em.j[2], g, dte, C);
    FOPIS_LAUNCH_CHECK();
    for (int q = 0; q < 3; ++q) yee_glue(c, f[q]);
    reference_efield(c);
}

void em_update_bfield(Ctx& c) {
    const Geo g = make_geo(c);
    const YeeArr* f = c.em.f;
    ++c.launches;
    fdtd_b_kernel<<<blocks(interior_count(g)), kT, 0, c.st>>>(view(f[3]), view(f[4]), view(f[5]), view(f[0]), view(f[1]),
                                                              view(f[2]), g, 1.0 /* dt / dx */);
    FOPIS_LAUNCH_CHECK();
    for (int q = 3; q < 6; ++q) yee_glue(c, f[q]);
    reference_bfield(c);
}

void em_reference_fields(Ctx& c) {
    reference_efield(c);
    reference_bfield(c);
}

double em_efield_energy(Ctx& c) { return 0.5 * c.p.eps0 * em_energy(c, 0); }
double em_bfield_energy(Ctx& c) { return 0.5 * em_energy(c, 1) / c.p.mu0; }

const YeeArr* em_array(const Ctx& c, int which) {
    if (!c.em.on || which < FOPIS_FIELD_EX || which > FOPIS_FIELD_BZ) return nullptr;
    return &c.em.f[which - FOPIS_FIELD_EX];
}

void em_field_export(Ctx& c, int which, double* host) {
    const size_t bytes = sizeof(double) * c.N;
    if (const YeeArr* y = em_array(c, which)) {
        FOPIS_CUDA(cudaMemcpyAsync(host, y->v, sizeof(double) * y->size(), cudaMemcpyDeviceToHost, c.st));
    } else if (which >= FOPIS_FIELD_JX && which <= FOPIS_FIELD_JZ) {
        const int d = which - FOPIS_FIELD_JX;
        const size_t n = (size_t)(c.cx - (d == 0)) * (c.cy - (d == 1)) * (c.cz - (d == 2));
        FOPIS_CUDA(cudaMemcpyAsync(host, c.em.j[d], sizeof(double) * n, cudaMemcpyDeviceToHost, c.st));
    } else if (which >= FOPIS_FIELD_EXREF && which <= FOPIS_FIELD_EZREF) {
        FOPIS_CUDA(cudaMemcpyAsync(host, c.em.eref + (size_t)(which - FOPIS_FIELD_EXREF) * c.N, bytes,
                                   cudaMemcpyDeviceToHost, c.st));
    } else if (which >= FOPIS_FIELD_BXREF && which <= FOPIS_FIELD_BZREF) {
        FOPIS_CUDA(cudaMemcpyAsync(host, c.em.bref + (size_t)(which - FOPIS_FIELD_BXREF) * c.N, bytes,
                                   cudaMemcpyDeviceToHost, c.st));
    } else if (which >= FOPIS_FIELD_JXREF && which <= FOPIS_FIELD_JZREF) {
        const int d = which - FOPIS_FIELD_JXREF;
        ++c.launches;
        jref_kernel<<<blocks((long long)c.N), kT, 0, c.st>>>(c.em.j[d], d, make_geo(c), c.scratch64, (long long)c.N);
        FOPIS_LAUNCH_CHECK();
        FOPIS_CUDA(cudaMemcpyAsync(host, c.scratch64, bytes, cudaMemcpyDeviceToHost, c.st));
    } else {
        throw ApiError{FOPIS_ERR_ARG, "unknown field selector"};
    }
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
}

}  // namespace fopis
