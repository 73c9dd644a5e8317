// particles.cu — particle kernels of the ES step on sm_100a.
//
// Particles are structure-of-arrays, split precision: a packed int32 node cell
// (i,j,k glue-layout indices, i = floor(x)+1 as include/position.hpp:59-69)
// plus FP32 in-cell offsets x-(i-1) and FP32 velocities: 28 bytes a particle.
// Charge is deposited as int64 fixed point (17 fractional bits per axis), so
// rho is bit-exact and independent of the order of the additions.
#include "internal.cuh"

#include <algorithm>
#include <cstring>

namespace fopis {

namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

struct Grid {
    int cx, cy, cz;      // nodes with glue
    int n[3];            // reference node counts
    int per[6];          // periodic sides
    long long sj, si;    // linear strides of j and i
    int nb[3];           // bricks per axis over the node cells 0..c-2
};

// Particles are counting-sorted by brick: 4 x 4 x 8 node cells (k fastest),
// then by cell inside the brick. One CTA of the fused push owns one brick.
constexpr int kBX = 4, kBY = 4, kBZ = 8, kBrickCells = kBX * kBY * kBZ;

__host__ Grid make_grid(const Ctx& c) {
    Grid g;
    g.cx = c.cx; g.cy = c.cy; g.cz = c.cz;
    g.n[0] = c.nx; g.n[1] = c.ny; g.n[2] = c.nz;
    for (int t = 0; t < 6; ++t) g.per[t] = c.per[t];
    g.sj = c.cz; g.si = (long long)c.cy * c.cz;
    g.nb[0] = (c.cx - 1 + kBX - 1) / kBX;
    g.nb[1] = (c.cy - 1 + kBY - 1) / kBY;
    g.nb[2] = (c.cz - 1 + kBZ - 1) / kBZ;
    return g;
}

// Brick of a node cell (i slowest, k fastest) and the cell's place inside it.
__device__ __forceinline__ int brick_index(const Grid& g, int i, int j, int k) {
    return ((i / kBX) * g.nb[1] + (j / kBY)) * g.nb[2] + (k / kBZ);
}
__device__ __forceinline__ int local_cell(int i, int j, int k) {
    return ((i % kBX) * kBY + (j % kBY)) * kBZ + (k % kBZ);
}

// Linear node index. fopis_create caps every axis at 1022 nodes with glue, so
// indices stay below 2^31 and are formed in 32-bit arithmetic.
__device__ __forceinline__ int lin(const Grid& g, int i, int j, int k) {
    return i * (int)g.si + j * (int)g.sj + k;
}

// Boundary rule of one axis on the split position (cell index ci, offset o):
// the coordinate is (ci-1)+o. Restates RootGrid::checkX/Y/ZBoundary
// (include/grid.hpp:309-395) plus the single-rank periodic migration
// (src/Grid/GridParticleTreatmentES.cpp:115-177). Returns false to invalidate.
template <typename T>
__device__ __forceinline__ bool axis_boundary(const Grid& g, int axis, int& ci, T o) {
    const int n = g.n[axis];
    if (ci <= 0) {                                 // x < 0
        if (g.per[2 * axis]) { if (ci <= -1) ci += n; }   // x < -1 -> x + sl
        else return false;
    } else if (ci > n || (ci == n && o > (T)0)) {  // x > sl - 1
        if (g.per[2 * axis + 1]) { if (ci >= n + 1) ci -= n; }  // x >= sl -> x - sl
        else return false;
    }
    return true;
}

// Same rule on an FP64 coordinate (sources created in double).
__device__ __forceinline__ bool axis_boundary_d(const Grid& g, int axis, double& x) {
    const double sl = g.n[axis];
    if (x < 0.0) {
        if (g.per[2 * axis]) { if (x < -1.0) x += sl; }
        else return false;
    } else if (x > sl - 1.0) {
        if (g.per[2 * axis + 1]) { if (x >= sl) x -= sl; }
        else return false;
    }
    return true;
}

// Split an FP64 coordinate into node cell index and in-cell offset (FP32 in
// the mixed mode, where rounding can reach 1 and carries into the cell).
template <typename T>
__device__ __forceinline__ void split(double x, int& ci, T& o) {
    const double f = floor(x);
    ci = (int)f + 1;
    o = (T)(x - f);
    if (o >= (T)1) { o = (T)0; ci += 1; }
}

// FP64 CIC deposit of the FP64 mode: the eight corner weights of a particle
// (corner order of corner_offset) added to the species' FP64 weight sums.
__device__ __forceinline__ void deposit_f64(double* rho, long long base, const long long off[8], double ox, double oy,
                                            double oz) {
    const double wx[2] = {1.0 - ox, ox}, wy[2] = {1.0 - oy, oy}, wz[2] = {1.0 - oz, oz};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const double w = wx[t >> 2] * wy[(t >> 1) & 1] * wz[t & 1];
        if (w != 0.0) atomicAdd(rho + base + off[t], w);
    }
}

__device__ __forceinline__ bool cell_in_range(const Grid& g, int i, int j, int k) {
    return i >= 0 && j >= 0 && k >= 0 && i <= g.cx - 2 && j <= g.cy - 2 && k <= g.cz - 2;
}

// Eight integer CIC corner weights (sum 2^51) in the corner order
// (di,dj,dk) = 000,001,010,011,100,101,110,111.
__device__ __forceinline__ void corner_weights(float ox, float oy, float oz, unsigned long long w[8]) {
    const long long a = __float2int_rn(ox * kDepositScale);
    const long long b = __float2int_rn(oy * kDepositScale);
    const long long d = __float2int_rn(oz * kDepositScale);
    const long long wx[2] = {kDepositOne - a, a}, wy[2] = {kDepositOne - b, b}, wz[2] = {kDepositOne - d, d};
#pragma unroll
    for (int t = 0; t < 8; ++t) w[t] = (unsigned long long)(wx[t >> 2] * wy[(t >> 1) & 1] * wz[t & 1]);
}

__device__ __forceinline__ long long corner_offset(const Grid& g, int t) {
    return ((t >> 2) ? g.si : 0) + (((t >> 1) & 1) ? g.sj : 0) + (t & 1);
}

// Warp-aggregated int64 deposit. Lanes whose cell is unique in the warp add
// their eight weights directly; lanes sharing a cell are reduced first with
// three 17-bit-chunk redux.sync sums per corner (exact), then their leader adds.
// Every lane of the warp must call this (dep selects the depositing ones).
// Returns true when one of this lane's additions wrapped a node past 2^64.
__device__ __forceinline__ bool warp_deposit(unsigned long long* rho, const Grid& g, bool dep, long long base,
                                             float ox, float oy, float oz) {
    const int lane = threadIdx.x & 31;
    unsigned long long w[8];
    if (dep) corner_weights(ox, oy, oz, w);
    else {
#pragma unroll
        for (int t = 0; t < 8; ++t) w[t] = 0ull;
    }
    const long long key = dep ? base : -1ll - lane;
    const unsigned grp = __match_any_sync(kFull, key);
    const bool single = __popc(grp) == 1;
    bool wrap = false;
    if (dep && single) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if (w[t]) {
                const unsigned long long old = atomicAdd(rho + base + corner_offset(g, t), w[t]);
                wrap |= old + w[t] < old;
            }
    }
    unsigned multi = __ballot_sync(kFull, dep && !single);
    while (multi) {
        const int leader = __ffs(multi) - 1;
        const unsigned members = __shfl_sync(kFull, grp, leader);
        const bool in = (members >> lane) & 1u;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const unsigned long long v = in ? w[t] : 0ull;
            const unsigned s0 = __reduce_add_sync(kFull, (unsigned)(v & 0x1FFFFull));
            const unsigned s1 = __reduce_add_sync(kFull, (unsigned)((v >> 17) & 0x1FFFFull));
            const unsigned s2 = __reduce_add_sync(kFull, (unsigned)(v >> 34));
            if (lane == leader) {
                const unsigned long long tot = (unsigned long long)s0 + ((unsigned long long)s1 << 17) +
                                               ((unsigned long long)s2 << 34);
                if (tot) {
                    const unsigned long long old = atomicAdd(rho + base + corner_offset(g, t), tot);
                    wrap |= old + tot < old;
                }
            }
        }
        multi &= ~members;
    }
    return wrap;
}

// Warp-aggregated slot reservation on a 64-bit counter.
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long* counter, bool want) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(kFull, want);
    unsigned long long base = 0;
    if (m) {
        const int leader = __ffs(m) - 1;
        if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(m));
        base = __shfl_sync(kFull, base, leader);
    }
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[32];
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    }
    return v;
}

template <typename T> struct NodeE;
template <> struct NodeE<float> { using type = float4; };
template <> struct NodeE<double> { using type = Vec4d; };
__device__ __forceinline__ float4 load_e(const float4* p) { return __ldg(p); }
__device__ __forceinline__ Vec4d load_e(const Vec4d* p) { return *p; }

template <typename T>
struct PushArgsT {
    SoaT<T> p;
    int s;
    long long cap;
    long long lo;             // first slot of the pass (the unsorted tail in the fused step)
    const unsigned long long* count;
    const typename NodeE<T>::type* E;
    Grid g;
    T qm;                     // 0.5 q/m
    T bx, by, bz, boris;      // static B as the reference uses it, 2/(1+|b|^2)
    int bzero;                // B = 0: the rotation adds exact zeros and is skipped
    const uint8_t* cellmap;   // nullptr without objects
    unsigned long long* rho;  // species accumulator: int64 fixed point, or FP64 weights in the FP64 mode
    AbsorbList ab;
    DevScalars* sc;
};
using PushArgs = PushArgsT<float>;

template <typename T>
struct PStateT {
    int i, j, k;
    T ox, oy, oz, vx, vy, vz;
};
using PState = PStateT<float>;

__device__ __forceinline__ float floor_of(float x) { return floorf(x); }
__device__ __forceinline__ double floor_of(double x) { return floor(x); }
__device__ __forceinline__ int int_of(float x) { return __float2int_rd(x); }
__device__ __forceinline__ int int_of(double x) { return __double2int_rd(x); }

// CIC gather of nodal E and the Boris kick/rotate/kick of
// Grid::updateParticleVelocityES (GridParticleTreatmentES.cpp:13-88): weights
// qm dx2 dy2 dz2 ... on the eight nodes, B used as given.
template <typename T>
__device__ __forceinline__ void gather_boris(const PushArgsT<T>& a, PStateT<T>& s) {
    const int b = lin(a.g, s.i, s.j, s.k);
    const int sj = (int)a.g.sj, si = (int)a.g.si;
    const T x1 = s.ox, x2 = (T)1 - s.ox, y1 = s.oy, y2 = (T)1 - s.oy, z1 = s.oz, z2 = (T)1 - s.oz;
    const auto* e = a.E + b;
    const auto e000 = load_e(e), e001 = load_e(e + 1);
    const auto e010 = load_e(e + sj), e011 = load_e(e + sj + 1);
    const auto e100 = load_e(e + si), e101 = load_e(e + si + 1);
    const auto e110 = load_e(e + si + sj), e111 = load_e(e + si + sj + 1);
    const T w000 = x2 * y2 * z2, w100 = x1 * y2 * z2, w010 = x2 * y1 * z2, w110 = x1 * y1 * z2;
    const T w001 = x2 * y2 * z1, w101 = x1 * y2 * z1, w011 = x2 * y1 * z1, w111 = x1 * y1 * z1;
    const T ex = a.qm * (w000 * e000.x + w100 * e100.x + w010 * e010.x + w110 * e110.x +
                         w001 * e001.x + w101 * e101.x + w011 * e011.x + w111 * e111.x);
    const T ey = a.qm * (w000 * e000.y + w100 * e100.y + w010 * e010.y + w110 * e110.y +
                         w001 * e001.y + w101 * e101.y + w011 * e011.y + w111 * e111.y);
    const T ez = a.qm * (w000 * e000.z + w100 * e100.z + w010 * e010.z + w110 * e110.z +
                         w001 * e001.z + w101 * e101.z + w011 * e011.z + w111 * e111.z);
    const T vx1 = s.vx + ex, vy1 = s.vy + ey, vz1 = s.vz + ez;
    if (a.bzero) {
        s.vx = vx1 + ex; s.vy = vy1 + ey; s.vz = vz1 + ez;
        return;
    }
    const T vxt = vx1 + vy1 * a.bz - vz1 * a.by;
    const T vyt = vy1 + vz1 * a.bx - vx1 * a.bz;
    const T vzt = vz1 + vx1 * a.by - vy1 * a.bx;
    s.vx = vx1 + (ex + a.boris * (vyt * a.bz - vzt * a.by));
    s.vy = vy1 + (ey + a.boris * (vzt * a.bx - vxt * a.bz));
    s.vz = vz1 + (ez + a.boris * (vxt * a.by - vyt * a.bx));
}

// x += v with the cell carry, then the boundary rules; false invalidates.
// Cells 1..n-1 of every axis are away from both faces (the rules only act on
// cells <= 0 and >= n), so most particles skip them.
template <typename T>
__device__ __forceinline__ bool move_boundary(const PushArgsT<T>& a, PStateT<T>& s) {
    s.ox += s.vx; s.oy += s.vy; s.oz += s.vz;
    const T fx = floor_of(s.ox), fy = floor_of(s.oy), fz = floor_of(s.oz);
    s.ox -= fx; s.oy -= fy; s.oz -= fz;
    s.i += int_of(fx); s.j += int_of(fy); s.k += int_of(fz);
    if ((unsigned)(s.i - 1) < (unsigned)(a.g.n[0] - 1) && (unsigned)(s.j - 1) < (unsigned)(a.g.n[1] - 1) &&
        (unsigned)(s.k - 1) < (unsigned)(a.g.n[2] - 1))
        return true;
    bool live = axis_boundary(a.g, 0, s.i, s.ox) && axis_boundary(a.g, 1, s.j, s.oy) &&
                axis_boundary(a.g, 2, s.k, s.oz);
    if (live && !cell_in_range(a.g, s.i, s.j, s.k)) {  // non-finite or runaway velocity
        live = false;
        atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_NONFINITE);
    }
    return live;
}

// Body test and absorbed-list append of RootGrid::updateRho's per-particle
// part (RootGridField.cpp:1173-1178); every lane of the warp calls it.
template <typename T>
__device__ __forceinline__ bool absorb_check(const PushArgsT<T>& a, const PStateT<T>& s, bool live) {
    uint8_t ob = 0;
    if (live && a.cellmap) ob = a.cellmap[lin(a.g, s.i, s.j, s.k)];
    const bool absorbed = ob != 0;
    const unsigned long long slot = warp_reserve(&a.sc->absorbed_n, absorbed);
    if (absorbed) {
        if ((long long)slot < a.ab.cap) {
            a.ab.cell[slot] = pack_cell(s.i, s.j, s.k);
            a.ab.ox[slot] = s.ox; a.ab.oy[slot] = s.oy; a.ab.oz[slot] = s.oz;
            a.ab.vx[slot] = s.vx; a.ab.vy[slot] = s.vy; a.ab.vz[slot] = s.vz;
            a.ab.species[slot] = (uint8_t)a.s;
            a.ab.object[slot] = (uint8_t)(ob - 1);
        } else {
            atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_ABSORB_OVERFLOW);
        }
    }
    return absorbed;
}

// The fused particle pass over slots [lo, count). VEL: CIC gather of nodal E
// and Boris kick/rotate (Grid::updateParticleVelocityES,
// GridParticleTreatmentES.cpp:13-88). POS: x += v and boundaries
// (RootGrid::updateParticlePositionES, :90-181). DEP: the per-particle part of
// RootGrid::updateRho (RootGridField.cpp:1168-1196): particles inside a body go
// to the absorbed list (Spacecraft::distributeInnerParticleCharge,
// Spacecraft.cpp:512-592, finished by absorb_kernel); the rest deposit their CIC
// weights with warp-aggregated atomics. The fused step runs it only on the
// unsorted tail; push_brick_kernel takes the sorted bricks.
template <typename T, bool VEL, bool POS, bool DEP>
__global__ void __launch_bounds__(kThreads) push_kernel(PushArgsT<T> a) {
    const long long n = (long long)min(*a.count, (unsigned long long)a.cap);
    const long long stride = (long long)gridDim.x * blockDim.x;
    double e2 = 0.0, npushed = 0.0, nkept = 0.0;
    for (long long base = a.lo + (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const long long idx = base + (threadIdx.x & 31);
        const bool inb = idx < n;
        const int32_t cell = inb ? a.p.cell[idx] : -1;
        bool live = cell >= 0;
        PStateT<T> st{0, 0, 0, (T)0, (T)0, (T)0, (T)0, (T)0, (T)0};
        if (live) {
            unpack_cell(cell, st.i, st.j, st.k);
            st.ox = a.p.ox[idx]; st.oy = a.p.oy[idx]; st.oz = a.p.oz[idx];
            st.vx = a.p.vx[idx]; st.vy = a.p.vy[idx]; st.vz = a.p.vz[idx];
        }
        if (VEL && live) gather_boris(a, st);
        if (POS && live) live = move_boundary(a, st);
        if (DEP) {
            if (absorb_check(a, st, live)) live = false;
            if constexpr (sizeof(T) == 4) {
                if (warp_deposit(a.rho, a.g, live, live ? lin(a.g, st.i, st.j, st.k) : 0, st.ox, st.oy, st.oz))
                    atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_RHO_OVERFLOW);
            } else if (live) {
                long long off[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) off[t] = corner_offset(a.g, t);
                deposit_f64(reinterpret_cast<double*>(a.rho), lin(a.g, st.i, st.j, st.k), off, st.ox, st.oy, st.oz);
            }
            if (live && VEL) e2 += (double)st.vx * st.vx + (double)st.vy * st.vy + (double)st.vz * st.vz;
            if (VEL && POS) { npushed += cell >= 0 ? 1.0 : 0.0; nkept += live ? 1.0 : 0.0; }
        }
        if (inb && cell >= 0) {
            if (POS || DEP) a.p.cell[idx] = live ? pack_cell(st.i, st.j, st.k) : -1;
            if (POS) { a.p.ox[idx] = st.ox; a.p.oy[idx] = st.oy; a.p.oz[idx] = st.oz; }
            if (VEL) { a.p.vx[idx] = st.vx; a.p.vy[idx] = st.vy; a.p.vz[idx] = st.vz; }
        }
    }
    if (DEP && VEL) {
        const double t = block_sum(e2);
        if (threadIdx.x == 0 && t != 0.0) atomicAdd(&a.sc->energy[a.s], t);
    }
    if (DEP && VEL && POS) {   // the fused pass: counts of the step (exact in FP64 below 2^53)
        const double np = block_sum(npushed), nk = block_sum(nkept);
        if (threadIdx.x == 0) {
            if (np > 0.0) atomicAdd(&a.sc->pushed[a.s], (unsigned long long)np);
            if (nk > 0.0) atomicAdd(&a.sc->survived[a.s], (unsigned long long)nk);
        }
    }
}

// ------------------------------------------------------------------ EM particle phases
// Grid::updateParticleVelocityEM (src/Grid/GridParticleTreatmentEM.cpp:13-105):
// the CIC gather of the nodal E and B, both scaled by 0.5 q/m, then Boris with
// the gathered b, boris = 2 / (1 + |b|^2). One particle per thread.
template <typename T>
__device__ __forceinline__ void em_kick(const PushArgsT<T>& a, const typename NodeE<T>::type* B, PStateT<T>& st) {
    const T x1 = st.ox, y1 = st.oy, z1 = st.oz;
    const T x2 = (T)1 - x1, y2 = (T)1 - y1, z2 = (T)1 - z1;
    const T w[8] = {a.qm * x2 * y2 * z2, a.qm * x1 * y2 * z2, a.qm * x2 * y1 * z2, a.qm * x1 * y1 * z2,
                    a.qm * x2 * y2 * z1, a.qm * x1 * y2 * z1, a.qm * x2 * y1 * z1, a.qm * x1 * y1 * z1};
    const int b = lin(a.g, st.i, st.j, st.k), sj = (int)a.g.sj, si = (int)a.g.si;
    const int off[8] = {0, si, sj, si + sj, 1, si + 1, sj + 1, si + sj + 1};
    T e[3] = {(T)0, (T)0, (T)0}, m[3] = {(T)0, (T)0, (T)0};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const auto ev = load_e(a.E + b + off[t]);
        const auto bv = load_e(B + b + off[t]);
        e[0] += w[t] * ev.x; e[1] += w[t] * ev.y; e[2] += w[t] * ev.z;
        m[0] += w[t] * bv.x; m[1] += w[t] * bv.y; m[2] += w[t] * bv.z;
    }
    const T boris = (T)2 / ((T)1 + (m[0] * m[0] + m[1] * m[1] + m[2] * m[2]));
    const T vx1 = st.vx + e[0], vy1 = st.vy + e[1], vz1 = st.vz + e[2];
    const T vxt = vx1 + vy1 * m[2] - vz1 * m[1];
    const T vyt = vy1 + vz1 * m[0] - vx1 * m[2];
    const T vzt = vz1 + vx1 * m[1] - vy1 * m[0];
    st.vx = vx1 + e[0] + boris * (vyt * m[2] - vzt * m[1]);
    st.vy = vy1 + e[1] + boris * (vzt * m[0] - vxt * m[2]);
    st.vz = vz1 + e[2] + boris * (vxt * m[1] - vyt * m[0]);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) em_velocity_kernel(PushArgsT<T> a, const typename NodeE<T>::type* B) {
    const long long n = (long long)min(*a.count, (unsigned long long)a.cap);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int32_t cell = a.p.cell[idx];
        if (cell < 0) continue;
        PStateT<T> st;
        unpack_cell(cell, st.i, st.j, st.k);
        st.ox = a.p.ox[idx]; st.oy = a.p.oy[idx]; st.oz = a.p.oz[idx];
        st.vx = a.p.vx[idx]; st.vy = a.p.vy[idx]; st.vz = a.p.vz[idx];
        em_kick(a, B, st);
        a.p.vx[idx] = st.vx; a.p.vy[idx] = st.vy; a.p.vz[idx] = st.vz;
    }
}

// Edge currents of the EM mode, FP64, glue-layout edges of the node grid.
struct EdgeJ {
    double *x, *y, *z;     // jx [cx-1][cy][cz], jy [cx][cy-1][cz], jz [cx][cy][cz-1]
    int cx, cy, cz;
};

// The zigzag relay point of Position::getReferencePosition
// (include/position.hpp:88-96) on one axis, in a frame whose cell index is
// floor(x) + 1: the shared face when the two cells differ, else the midpoint.
__device__ __forceinline__ double em_relay(int i_new, int i_old, double x_new, double x_old) {
    return fmin((double)min(i_new, i_old), fmax((double)max(i_new, i_old) - 1.0, 0.5 * (x_new + x_old)));
}

// One half of Particle::distributeCurrentAtOldPosition / AtNewPosition
// (src/Particle/particle.cpp:258-338) on the edges of cell (i, j, k): flux f
// and in-cell weights w (the mean of the half's two points in the cell's frame).
__device__ __forceinline__ void em_current_half(const EdgeJ& J, int i, int j, int k, const double f[3],
                                                const double w[3]) {
    const long long ax = ((long long)i * J.cy + j) * J.cz + k;                 // jx [cx-1][cy][cz]
    atomicAdd(J.x + ax, f[0] * (1.0 - w[1]) * (1.0 - w[2]));
    atomicAdd(J.x + ax + J.cz, f[0] * w[1] * (1.0 - w[2]));
    atomicAdd(J.x + ax + 1, f[0] * (1.0 - w[1]) * w[2]);
    atomicAdd(J.x + ax + J.cz + 1, f[0] * w[1] * w[2]);
    const long long ay = ((long long)i * (J.cy - 1) + j) * J.cz + k;           // jy [cx][cy-1][cz]
    const long long syi = (long long)(J.cy - 1) * J.cz;
    atomicAdd(J.y + ay, f[1] * (1.0 - w[0]) * (1.0 - w[2]));
    atomicAdd(J.y + ay + syi, f[1] * w[0] * (1.0 - w[2]));
    atomicAdd(J.y + ay + 1, f[1] * (1.0 - w[0]) * w[2]);
    atomicAdd(J.y + ay + syi + 1, f[1] * w[0] * w[2]);
    const long long az = ((long long)i * J.cy + j) * (J.cz - 1) + k;           // jz [cx][cy][cz-1]
    const long long szi = (long long)J.cy * (J.cz - 1);
    atomicAdd(J.z + az, f[2] * (1.0 - w[0]) * (1.0 - w[1]));
    atomicAdd(J.z + az + szi, f[2] * w[0] * (1.0 - w[1]));
    atomicAdd(J.z + az + (J.cz - 1), f[2] * (1.0 - w[0]) * w[1]);
    atomicAdd(J.z + az + szi + (J.cz - 1), f[2] * w[0] * w[1]);
}

// RootGrid::updateParticlePositionEM's per-particle part
// (src/Grid/GridParticleTreatmentEM.cpp:107-139): the old-cell half of the
// charge-conserving current (from x to x + v), the move with the boundary rules
// and, while still valid, the new-cell half (from x - v to x in the frame of
// the cell the particle lands in, a periodic crossing included). Positions
// enter the current in the cell's frame (offset in [0, 1)), the reference's
// global coordinates shifted by the cell's lower node. q is the super-particle
// charge per step.
template <typename T>
__global__ void __launch_bounds__(kThreads) em_position_kernel(PushArgsT<T> a, EdgeJ J, double q) {
    const long long n = (long long)min(*a.count, (unsigned long long)a.cap);
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int32_t cell = a.p.cell[idx];
        if (cell < 0) continue;
        PStateT<T> st;
        unpack_cell(cell, st.i, st.j, st.k);
        st.ox = a.p.ox[idx]; st.oy = a.p.oy[idx]; st.oz = a.p.oz[idx];
        st.vx = a.p.vx[idx]; st.vy = a.p.vy[idx]; st.vz = a.p.vz[idx];
        {
            const T o[3] = {st.ox, st.oy, st.oz}, v[3] = {st.vx, st.vy, st.vz};
            double f[3], w[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double x1 = (double)o[d], x2 = (double)(T)(o[d] + v[d]);   // the move's own sum
                const int i2 = (int)floor(x2) + 1;
                const double r = em_relay(i2, 1, x2, x1);
                f[d] = q * (r - x1);
                w[d] = 0.5 * (r + x1);
            }
            em_current_half(J, st.i, st.j, st.k, f, w);
        }
        const bool live = move_boundary(a, st);
        if (live) {
            const T o[3] = {st.ox, st.oy, st.oz}, v[3] = {st.vx, st.vy, st.vz};
            double f[3], w[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double x2 = (double)o[d], x1 = x2 - (double)v[d];
                const int i1 = (int)floor(x1) + 1;
                const double r = em_relay(1, i1, x2, x1);
                f[d] = q * (x2 - r);
                w[d] = 0.5 * (r + x2);
            }
            em_current_half(J, st.i, st.j, st.k, f, w);
        }
        a.p.cell[idx] = live ? pack_cell(st.i, st.j, st.k) : -1;
        a.p.ox[idx] = st.ox; a.p.oy[idx] = st.oy; a.p.oz[idx] = st.oz;
    }
}

// Edge currents of the mixed mode in fixed point: per species the sum of
// J / (q size) in units of 2^-24 of one particle crossing a cell (the FP32
// resolution of the particle offsets), int64 two's complement sums (exact,
// independent of the order of the additions), converted to the FP64 J of
// Field::jx.. once per step.
constexpr float kCurrentScale = 16777216.0f;   // 2^24
struct EdgeFix {
    unsigned long long *x = nullptr, *y = nullptr, *z = nullptr;   // this species' jx, jy, jz sums
    int cx = 0, cy = 0, cz = 0;
    const float4* B = nullptr;   // nodal B: the pass also gives the velocity update first (em_kick)
};

__device__ __forceinline__ float em_relay_f(int i_new, int i_old, float x_new, float x_old) {
    return fminf((float)min(i_new, i_old), fmaxf((float)max(i_new, i_old) - 1.0f, 0.5f * (x_new + x_old)));
}

// The old-cell half of the zigzag (the move from x to x + v) in the cell's frame,
// unit charge: flux f and weights w (src/Particle/particle.cpp:258-298), FP32.
__device__ __forceinline__ void em_half_old(const PState& st, float f[3], float w[3]) {
    const float o[3] = {st.ox, st.oy, st.oz}, v[3] = {st.vx, st.vy, st.vz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float x1 = o[d], x2 = o[d] + v[d];   // the move's own sum
        const float r = em_relay_f((int)floorf(x2) + 1, 1, x2, x1);
        f[d] = r - x1;
        w[d] = 0.5f * (r + x1);
    }
}
// The new-cell half (from x - v to x) in the frame of the cell the particle
// landed in (particle.cpp:300-338).
__device__ __forceinline__ void em_half_new(const PState& st, float f[3], float w[3]) {
    const float o[3] = {st.ox, st.oy, st.oz}, v[3] = {st.vx, st.vy, st.vz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float x2 = o[d], x1 = x2 - v[d];
        const float r = em_relay_f(1, (int)floorf(x1) + 1, x2, x1);
        f[d] = x2 - r;
        w[d] = 0.5f * (r + x2);
    }
}

// The twelve edge terms of one half in fixed point (|term| <= 2^24), in the edge
// order of em_current_half, and the address of term q of cell (i, j, k).
__device__ __forceinline__ void em_terms(const float f[3], const float w[3], int t[12]) {
    const float s0 = kCurrentScale * f[0], s1 = kCurrentScale * f[1], s2 = kCurrentScale * f[2];
    t[0] = __float2int_rn(s0 * (1.0f - w[1]) * (1.0f - w[2]));
    t[1] = __float2int_rn(s0 * w[1] * (1.0f - w[2]));
    t[2] = __float2int_rn(s0 * (1.0f - w[1]) * w[2]);
    t[3] = __float2int_rn(s0 * w[1] * w[2]);
    t[4] = __float2int_rn(s1 * (1.0f - w[0]) * (1.0f - w[2]));
    t[5] = __float2int_rn(s1 * w[0] * (1.0f - w[2]));
    t[6] = __float2int_rn(s1 * (1.0f - w[0]) * w[2]);
    t[7] = __float2int_rn(s1 * w[0] * w[2]);
    t[8] = __float2int_rn(s2 * (1.0f - w[0]) * (1.0f - w[1]));
    t[9] = __float2int_rn(s2 * w[0] * (1.0f - w[1]));
    t[10] = __float2int_rn(s2 * (1.0f - w[0]) * w[1]);
    t[11] = __float2int_rn(s2 * w[0] * w[1]);
}
__device__ __forceinline__ unsigned long long* em_term_ptr(const EdgeFix& J, int i, int j, int k, int q) {
    const int e = q & 3;
    if (q < 4) return J.x + ((long long)i * J.cy + j) * J.cz + k + ((e & 1) ? J.cz : 0) + ((e >> 1) ? 1 : 0);
    if (q < 8) return J.y + ((long long)i * (J.cy - 1) + j) * J.cz + k + ((e & 1) ? (long long)(J.cy - 1) * J.cz : 0) +
                      ((e >> 1) ? 1 : 0);
    return J.z + ((long long)i * J.cy + j) * (J.cz - 1) + k + ((e & 1) ? (long long)J.cy * (J.cz - 1) : 0) +
           ((e >> 1) ? (J.cz - 1) : 0);
}

// Warp-aggregated fixed-point current terms t[12] of cell (i, j, k). When every
// depositing lane shares one cell the warp sums each term with one redux.sync
// (32 terms of at most 2^25 stay below 2^30) and lane 0 adds; otherwise lanes
// whose cell is unique add their terms directly and lanes sharing a cell are
// summed per cell, their leader adding. Every lane of the warp calls it.
__device__ __forceinline__ void em_warp_add(const EdgeFix& J, bool dep, int i, int j, int k, const int t[12]) {
    const int lane = threadIdx.x & 31;
    const int key = dep ? (i * J.cy + j) * J.cz + k : -1;   // node cells stay below 2^31
    const unsigned deps = __ballot_sync(kFull, dep);
    if (!deps) return;
    const int key0 = __shfl_sync(kFull, key, __ffs(deps) - 1);
    if (__all_sync(kFull, !dep || key == key0)) {
        const int first = __ffs(deps) - 1;
#pragma unroll
        for (int q = 0; q < 12; ++q) {
            const int sum = __reduce_add_sync(kFull, dep ? t[q] : 0);
            if (lane == first && sum) atomicAdd(em_term_ptr(J, i, j, k, q), (unsigned long long)(long long)sum);
        }
        return;
    }
    const unsigned grp = __match_any_sync(kFull, dep ? key : -1 - lane);
    const bool single = __popc(grp) == 1;
    if (dep && single) {
#pragma unroll
        for (int q = 0; q < 12; ++q)
            if (t[q]) atomicAdd(em_term_ptr(J, i, j, k, q), (unsigned long long)(long long)t[q]);
    }
    unsigned multi = __ballot_sync(kFull, dep && !single);
    while (multi) {
        const int leader = __ffs(multi) - 1;
        const unsigned members = __shfl_sync(kFull, grp, leader);
        const bool in = (members >> lane) & 1u;
#pragma unroll
        for (int q = 0; q < 12; ++q) {
            const int sum = __reduce_add_sync(kFull, in ? t[q] : 0);
            if (lane == leader && sum) atomicAdd(em_term_ptr(J, i, j, k, q), (unsigned long long)(long long)sum);
        }
        multi &= ~members;
    }
}

// Both halves of a move that stays in its cell, summed in closed form: with the
// midpoint m = x + v/2 and d = v/4 per axis, the two halves' x-edge terms
// (v/2)[(1 - m_y - d_y)(1 - m_z - d_z) + (1 - m_y + d_y)(1 - m_z + d_z)] ... are
// v_x [(1 - m_y)(1 - m_z) + d_y d_z], v_x [m_y (1 - m_z) - d_y d_z], ... (the
// relay point of both halves is the midpoint, include/position.hpp:88-96).
__device__ __forceinline__ void em_terms_same(const float o[3], const float v[3], int t[12]) {
    float m[3], d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) { m[a] = o[a] + 0.5f * v[a]; d[a] = 0.25f * v[a]; }
    const float s0 = kCurrentScale * v[0], s1 = kCurrentScale * v[1], s2 = kCurrentScale * v[2];
    const float dyz = d[1] * d[2], dxz = d[0] * d[2], dxy = d[0] * d[1];
    t[0] = __float2int_rn(s0 * ((1.0f - m[1]) * (1.0f - m[2]) + dyz));
    t[1] = __float2int_rn(s0 * (m[1] * (1.0f - m[2]) - dyz));
    t[2] = __float2int_rn(s0 * ((1.0f - m[1]) * m[2] - dyz));
    t[3] = __float2int_rn(s0 * (m[1] * m[2] + dyz));
    t[4] = __float2int_rn(s1 * ((1.0f - m[0]) * (1.0f - m[2]) + dxz));
    t[5] = __float2int_rn(s1 * (m[0] * (1.0f - m[2]) - dxz));
    t[6] = __float2int_rn(s1 * ((1.0f - m[0]) * m[2] - dxz));
    t[7] = __float2int_rn(s1 * (m[0] * m[2] + dxz));
    t[8] = __float2int_rn(s2 * ((1.0f - m[0]) * (1.0f - m[1]) + dxy));
    t[9] = __float2int_rn(s2 * (m[0] * (1.0f - m[1]) - dxy));
    t[10] = __float2int_rn(s2 * ((1.0f - m[0]) * m[1] - dxy));
    t[11] = __float2int_rn(s2 * (m[0] * m[1] + dxy));
}

// The current of one particle move, from the start offsets o0 and velocity of
// the particle in cell (oi, oj, ok) and its state after the move (st, live):
// a move that stays in its cell adds both halves at once (em_terms_same);
// otherwise the old-cell half goes to the old cell and, while the particle is
// still valid, the new-cell half to the new one. Every lane of the warp calls it.
__device__ __forceinline__ void em_warp_move_current(const EdgeFix& J, bool had, int oi, int oj, int ok,
                                                     const float o0[3], const PState& st, bool live) {
    const float v[3] = {st.vx, st.vy, st.vz};
    int t[12];
    const bool same = live && st.i == oi && st.j == oj && st.k == ok;
    if (same) {
        em_terms_same(o0, v, t);
    } else if (had) {
        PState s0 = st;
        s0.ox = o0[0]; s0.oy = o0[1]; s0.oz = o0[2];
        float f[3], w[3];
        em_half_old(s0, f, w);
        em_terms(f, w, t);
    } else {
#pragma unroll
        for (int q = 0; q < 12; ++q) t[q] = 0;
    }
    em_warp_add(J, had, oi, oj, ok, t);
    const bool cross = live && !same;
    if (__any_sync(kFull, cross)) {
        if (cross) {
            float f[3], w[3];
            em_half_new(st, f, w);
            em_terms(f, w, t);
        } else {
#pragma unroll
            for (int q = 0; q < 12; ++q) t[q] = 0;
        }
        em_warp_add(J, cross, st.i, st.j, st.k, t);
    }
}

// The mixed mode's particle pass of the EM step over the unsorted slots
// [a.lo, count): the old-cell half of the current, the move with the boundary
// rules, the new-cell half, the body test and the rho deposit
// (updateParticlePositionEM, then updateRho's per-particle part,
// RootGridField.cpp:1168-1196). push_brick_kernel<.., true> takes the sorted bricks.
__global__ void __launch_bounds__(kThreads) em_tail_kernel(PushArgs a, EdgeFix J) {
    const long long n = (long long)min(*a.count, (unsigned long long)a.cap);
    const long long stride = (long long)gridDim.x * blockDim.x;
    double npushed = 0.0, nkept = 0.0;
    for (long long base = a.lo + (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const long long idx = base + (threadIdx.x & 31);
        const int32_t cell = idx < n ? a.p.cell[idx] : -1;
        bool live = cell >= 0;
        PState st{0, 0, 0, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (live) {
            unpack_cell(cell, st.i, st.j, st.k);
            st.ox = a.p.ox[idx]; st.oy = a.p.oy[idx]; st.oz = a.p.oz[idx];
            st.vx = a.p.vx[idx]; st.vy = a.p.vy[idx]; st.vz = a.p.vz[idx];
            if (J.B) em_kick(a, J.B, st);
        }
        const int oi = st.i, oj = st.j, ok = st.k;
        const float o0[3] = {st.ox, st.oy, st.oz};
        if (live) live = move_boundary(a, st);
        em_warp_move_current(J, cell >= 0, oi, oj, ok, o0, st, live);
        if (absorb_check(a, st, live)) live = false;
        if (warp_deposit(a.rho, a.g, live, live ? lin(a.g, st.i, st.j, st.k) : 0, st.ox, st.oy, st.oz))
            atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_RHO_OVERFLOW);
        npushed += cell >= 0 ? 1.0 : 0.0;
        nkept += live ? 1.0 : 0.0;
        if (cell >= 0) {
            a.p.cell[idx] = live ? pack_cell(st.i, st.j, st.k) : -1;
            a.p.ox[idx] = st.ox; a.p.oy[idx] = st.oy; a.p.oz[idx] = st.oz;
            if (J.B) { a.p.vx[idx] = st.vx; a.p.vy[idx] = st.vy; a.p.vz[idx] = st.vz; }
        }
    }
    const double np = block_sum(npushed), nk = block_sum(nkept);
    if (threadIdx.x == 0) {
        if (np > 0.0) atomicAdd(&a.sc->pushed[a.s], (unsigned long long)np);
        if (nk > 0.0) atomicAdd(&a.sc->survived[a.s], (unsigned long long)nk);
    }
}

// J_d = sum_s q_s size_s 2^-40 (fixed-point sums), FP64, for the three edge arrays.
struct FixScales { double v[FOPIS_MAX_SPECIES]; };
__global__ void em_j_convert_kernel(const unsigned long long* fix, long long per_species, int nsp, FixScales sc,
                                    double* jx, long long nx, double* jy, long long ny, double* jz) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < per_species;
         t += (long long)gridDim.x * blockDim.x) {   // the three arrays back to back
        double v = 0.0;
        for (int s = 0; s < nsp; ++s) v += sc.v[s] * (double)(long long)fix[(long long)s * per_species + t];
        if (t < nx) jx[t] = v;
        else if (t < nx + ny) jy[t - nx] = v;
        else jz[t - nx - ny] = v;
    }
}

// ------------------------------------------------------------------ brick push
// push_brick_kernel: the fused push (gather + Boris + move + boundaries +
// absorption flag + deposit + kinetic energy) over the brick-sorted particles,
// one brick per CTA.
//
// Push. Lanes hold consecutive particles. Between sorts a warp's 32 particles
// start in one or two cells, so the eight corner loads of the field gather are
// broadcasts (measured on B200: eight float4 loads cost ~1.9 SM cycles per warp
// instruction when lanes share a node, ~12 when all 32 lanes read different
// nodes), and the state loads and stores are coalesced 128-byte rows.
//
// Deposit. The charge of a cell's particles reaches the cell's eight corner
// nodes as sums of the in-cell moments 1, a, b, d, ab, ad, bd, abd (a, b, d the
// offsets in 17-bit fixed point): the corner (ex,ey,ez) weight of one particle
// is prod(e ? q : 2^17 - q), a polynomial in those moments. Each lane packs its
// particle's new window cell and offsets into one 64-bit word of a batch buffer
// (kBatch particles, sorted order); the buffer is then read with lanes
// kBatch/32 particles apart, i.e. in different cells, each thread summing the
// moments of its run of consecutive entries in registers and adding them,
// cut into 17-bit pieces, to the CTA's moment tile over the brick's cells plus
// a two-cell halo (13 planes of 32-bit words, no-return shared atomics; lanes
// on the same word would serialise, lanes on distinct words cost ~1.4 SM
// cycles per instruction). After each segment of at most
// kSegment particles the occupied cells turn their moments into corner weights
// (exact modulo 2^64), summed per node in a tile (low/high 32-bit planes with
// carry, in the batch buffer's memory) that is then added to the species'
// int64 accumulator. A segment holds fewer than 2^13 particles, so no corner
// sum of one cell reaches 2^64 and no moment plane reaches 2^32; a wrap of a
// node sum (more than 2^13 full weights on one node) is detected and latched
// as FOPIS_DEV_RHO_OVERFLOW. Particles that leave the halo add their eight
// corner weights straight to the global accumulator.
constexpr int kBrickThreads = 256;
constexpr int kPer = 2;                                  // particles per thread per compute pass (64 registers)
constexpr int kPass = kBrickThreads * kPer;              // 512
constexpr int kBatch = 1024;                             // particles per deposit batch (two passes)
constexpr int kBatchPad = kBatch + kBatch / 32;          // one pad word per 32 entries: conflict-free reads
constexpr int kHalo = 2;                                 // cells a particle may drift out of its brick
constexpr int kCX = kBX + 2 * kHalo, kCY = kBY + 2 * kHalo, kCZ = kBZ + 2 * kHalo;   // window cells
constexpr int kWinCells = kCX * kCY * kCZ;               // 8 x 8 x 12 = 768
constexpr int kNX = kCX + 1, kNY = kCY + 1, kNZ = kCZ + 1;                           // window nodes
constexpr int kWinNodes = kNX * kNY * kNZ;               // 9 x 9 x 13 = 1053
constexpr int kPlanes = 13;                              // N, A, B, D, AB lo/hi, AD lo/hi, BD lo/hi, ABD x3
constexpr int kSegment = 7 * kBatch;                     // 7168 < 2^13 particles per moment segment
constexpr unsigned kChunk17 = 0x1FFFFu;
constexpr unsigned long long kNoDeposit = 0x3FFull;      // batch entry without a deposit (cell field all ones)
static_assert(kBatch == 2 * kPass, "a batch is two compute passes");
static_assert(kWinCells < 0x3FF, "window cell fits the 10-bit field of a batch entry");
static_assert(2 * kWinNodes <= 2 * kBatchPad, "the node tile fits in the batch buffer");
__device__ __forceinline__ int bpad(int q) { return q + (q >> 5); }

// Adds one corner weight (a value below 2^64) to the node tile held as a low
// and a high 32-bit plane; returns true when the node's sum wrapped past 2^64.
__device__ __forceinline__ bool tile_add_checked(unsigned* lo, unsigned* hi, int idx, unsigned long long w) {
    const unsigned wl = (unsigned)w, wh = (unsigned)(w >> 32);
    const unsigned old = atomicAdd(lo + idx, wl);
    const unsigned add = wh + ((old + wl < old) ? 1u : 0u);
    const unsigned oldh = atomicAdd(hi + idx, add);
    return add < wh || oldh + add < oldh;
}

// Adds a particle's eight corner weights straight to the global accumulator.
__device__ __forceinline__ bool global_deposit(unsigned long long* rho, const Grid& g, int base, unsigned qa,
                                               unsigned qb, unsigned qd) {
    const unsigned wx[2] = {(unsigned)kDepositOne - qa, qa}, wy[2] = {(unsigned)kDepositOne - qb, qb};
    const unsigned wz[2] = {(unsigned)kDepositOne - qd, qd};
    bool wrap = false;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const unsigned long long w = (unsigned long long)wx[t >> 2] * wy[(t >> 1) & 1] * wz[t & 1];
        if (w) {
            const unsigned long long old = atomicAdd(rho + base + corner_offset(g, t), w);
            wrap |= old + w < old;
        }
    }
    return wrap;
}

// Moment sums of a few particles of one cell; flush() adds them to the cell's
// words of the moment tile (13 no-return 32-bit shared atomics). Each 64-bit
// moment is cut into 17-bit pieces; every piece a flush adds stays below 2^20,
// so a plane word, summed over one segment, stays below 2^32.
struct MomentSum {
    unsigned n = 0, a = 0, b = 0, d = 0;
    unsigned long long ab = 0, ad = 0, bd = 0, abd = 0;
    __device__ __forceinline__ void add(unsigned qa, unsigned qb, unsigned qd) {
        const unsigned long long pab = (unsigned long long)qa * qb;
        n += 1u; a += qa; b += qb; d += qd;
        ab += pab; ad += (unsigned long long)qa * qd; bd += (unsigned long long)qb * qd; abd += pab * qd;
    }
    __device__ __forceinline__ void flush(unsigned* mom, int wc) const {
        unsigned* m = mom + wc;
        atomicAdd(m, n);
        atomicAdd(m + 1 * kWinCells, a);
        atomicAdd(m + 2 * kWinCells, b);
        atomicAdd(m + 3 * kWinCells, d);
        atomicAdd(m + 4 * kWinCells, (unsigned)ab & kChunk17);
        atomicAdd(m + 5 * kWinCells, (unsigned)(ab >> 17));
        atomicAdd(m + 6 * kWinCells, (unsigned)ad & kChunk17);
        atomicAdd(m + 7 * kWinCells, (unsigned)(ad >> 17));
        atomicAdd(m + 8 * kWinCells, (unsigned)bd & kChunk17);
        atomicAdd(m + 9 * kWinCells, (unsigned)(bd >> 17));
        atomicAdd(m + 10 * kWinCells, (unsigned)abd & kChunk17);
        atomicAdd(m + 11 * kWinCells, (unsigned)(abd >> 17) & kChunk17);
        atomicAdd(m + 12 * kWinCells, (unsigned)(abd >> 34));
    }
};

// The eight corner weight sums of a cell from its moments M[T] (T bits: 4 = x,
// 2 = y, 1 = z; M[T] = sum over the particles of the product of the offsets
// of the axes in T). Per axis, a set T without the axis becomes the "0" corner
// side O M_T - M_{T+axis} and the set with it the "1" side: after the three
// axes M[t] holds the corner t = (ex,ey,ez) sum of prod(e ? q : O - q).
// Modulo 2^64 and exact: every true corner sum lies in [0, 2^64).
__device__ __forceinline__ void corners_from_moments(unsigned long long M[8]) {
#pragma unroll
    for (int axis = 4; axis >= 1; axis >>= 1)
#pragma unroll
        for (int T = 0; T < 8; ++T)
            if (!(T & axis)) M[T] = (M[T] << kDepositBits) - M[T | axis];
}

template <int MINB, bool EM>
__global__ void __launch_bounds__(kBrickThreads, MINB) push_brick_kernel(PushArgs a, const int32_t* brick_start,
                                                                         EdgeFix J) {
    __shared__ __align__(16) unsigned s_mom[kPlanes * kWinCells];
    __shared__ __align__(16) unsigned long long s_batch[kBatchPad];    // batch entries; node tile in the epilogue
    unsigned* const t_lo = reinterpret_cast<unsigned*>(s_batch);
    unsigned* const t_hi = t_lo + kWinNodes;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x;
    const int bi = b / (a.g.nb[1] * a.g.nb[2]), bj = (b / a.g.nb[2]) % a.g.nb[1], bk = b % a.g.nb[2];
    const int wx0 = bi * kBX - kHalo, wy0 = bj * kBY - kHalo, wz0 = bk * kBZ - kHalo;
    int body = 0;
    for (int t = tid; t < kWinCells; t += kBrickThreads) {
        // a body cell anywhere in the window?
        const int x = wx0 + t / (kCY * kCZ), y = wy0 + (t / kCZ) % kCY, z = wz0 + t % kCZ;
        if (a.cellmap && x >= 0 && y >= 0 && z >= 0 && x < a.g.cx - 1 && y < a.g.cy - 1 && z < a.g.cz - 1 &&
            a.cellmap[lin(a.g, x, y, z)] != 0)
            body = 1;
    }
    // particles that stay inside a body-free window need no body test
    const bool window_body = __syncthreads_or(body) != 0;
    const long long p0 = brick_start[b], p1 = brick_start[b + 1];
    double e2 = 0.0, npushed = 0.0, nkept = 0.0;
    bool wrap = false;
    for (long long s0 = p0; s0 < p1; s0 += kSegment) {
        const long long s1 = min(p1, s0 + (long long)kSegment);
        static_assert((kPlanes * kWinCells) % 4 == 0, "moment tile cleared in 16-byte stores");
        for (int t = tid; t < kPlanes * kWinCells / 4; t += kBrickThreads)
            reinterpret_cast<uint4*>(s_mom)[t] = make_uint4(0u, 0u, 0u, 0u);
        for (long long c0 = s0; c0 < s1; c0 += kBatch) {
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const long long cp = c0 + h * kPass;
                int32_t cell[kPer];
                float f[kPer][6];
#pragma unroll
                for (int r = 0; r < kPer; ++r) {
                    const long long idx = cp + (r * (kBrickThreads / 32) + warp) * 32 + lane;
                    cell[r] = idx < s1 ? a.p.cell[idx] : -1;
                    if (cell[r] >= 0) {
                        f[r][0] = a.p.ox[idx]; f[r][1] = a.p.oy[idx]; f[r][2] = a.p.oz[idx];
                        f[r][3] = a.p.vx[idx]; f[r][4] = a.p.vy[idx]; f[r][5] = a.p.vz[idx];
                    }
                }
#pragma unroll
                for (int r = 0; r < kPer; ++r) {
                    const int q = h * kPass + (r * (kBrickThreads / 32) + warp) * 32 + lane;   // place in the batch
                    const long long idx = c0 + q;
                    bool live = cell[r] >= 0;
                    PState st{0, 0, 0, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                    if constexpr (EM) {
                        // the EM step: velocities were updated by em_velocity_kernel; the move
                        // carries the two halves of the charge-conserving current
                        const bool had = live;
                        if (live) {
                            unpack_cell(cell[r], st.i, st.j, st.k);
                            st.ox = f[r][0]; st.oy = f[r][1]; st.oz = f[r][2];
                            st.vx = f[r][3]; st.vy = f[r][4]; st.vz = f[r][5];
                            if (J.B) em_kick(a, J.B, st);
                        }
                        const int oi = st.i, oj = st.j, ok = st.k;
                        const float o0[3] = {st.ox, st.oy, st.oz};
                        if (live) live = move_boundary(a, st);
                        em_warp_move_current(J, had, oi, oj, ok, o0, st, live);
                    } else if (live) {
                        unpack_cell(cell[r], st.i, st.j, st.k);
                        st.ox = f[r][0]; st.oy = f[r][1]; st.oz = f[r][2];
                        st.vx = f[r][3]; st.vy = f[r][4]; st.vz = f[r][5];
                        gather_boris(a, st);
                        live = move_boundary(a, st);
                    }
                    const int li = st.i - wx0, lj = st.j - wy0, lk = st.k - wz0;
                    const bool inwin = (unsigned)li < (unsigned)kCX && (unsigned)lj < (unsigned)kCY &&
                                       (unsigned)lk < (unsigned)kCZ;
                    const bool test = live && (window_body || !inwin);
                    if (__any_sync(kFull, test) && absorb_check(a, st, test)) live = false;
                    const unsigned qa = (unsigned)__float2int_rn(st.ox * kDepositScale);
                    const unsigned qb = (unsigned)__float2int_rn(st.oy * kDepositScale);
                    const unsigned qd = (unsigned)__float2int_rn(st.oz * kDepositScale);
                    s_batch[bpad(q)] = (live && inwin)
                                           ? ((unsigned long long)((li * kCY + lj) * kCZ + lk) |
                                              ((unsigned long long)qa << 10) | ((unsigned long long)qb << 28) |
                                              ((unsigned long long)qd << 46))
                                           : kNoDeposit;
                    if (live && !inwin) wrap |= global_deposit(a.rho, a.g, lin(a.g, st.i, st.j, st.k), qa, qb, qd);
                    if (live) e2 += (double)(st.vx * st.vx + st.vy * st.vy + st.vz * st.vz);
                    npushed += cell[r] >= 0 ? 1.0 : 0.0;
                    nkept += live ? 1.0 : 0.0;
                    if (cell[r] >= 0) {
                        a.p.cell[idx] = live ? pack_cell(st.i, st.j, st.k) : -1;
                        a.p.ox[idx] = st.ox; a.p.oy[idx] = st.oy; a.p.oz[idx] = st.oz;
                        a.p.vx[idx] = st.vx; a.p.vy[idx] = st.vy; a.p.vz[idx] = st.vz;
                    }
                }
            }
            __syncthreads();
            // deposit: lane l takes the run of entries l*32 + warp*4 + r (r = 0..3), runs of
            // different lanes 32 sorted places (about one cell) apart; a run's particles
            // mostly share a cell and are summed in registers, two cells at a time
            {
                MomentSum ma, mb;
                int ca = -1, cb = -1;
#pragma unroll
                for (int r = 0; r < kBatch / kBrickThreads; ++r) {
                    const unsigned long long e =
                        s_batch[bpad(lane * (kBatch / 32) + warp * (kBatch / kBrickThreads) + r)];
                    const int wc = (int)(e & 0x3FFull);
                    if (wc == (int)kNoDeposit) continue;
                    const unsigned qa = (unsigned)(e >> 10) & 0x3FFFFu, qb = (unsigned)(e >> 28) & 0x3FFFFu;
                    const unsigned qd = (unsigned)(e >> 46);
                    if (ca < 0 || wc == ca) { ca = wc; ma.add(qa, qb, qd); }
                    else if (cb < 0 || wc == cb) { cb = wc; mb.add(qa, qb, qd); }
                    else { MomentSum one; one.add(qa, qb, qd); one.flush(s_mom, wc); }
                }
                if (ca >= 0) ma.flush(s_mom, ca);
                if (cb >= 0) mb.flush(s_mom, cb);
            }
            __syncthreads();
        }
        // occupied cells: moments -> corner weights -> node tile (in the batch buffer)
        for (int t = tid; t < 2 * kWinNodes; t += kBrickThreads) t_lo[t] = 0u;
        __syncthreads();
        for (int t = tid; t < kWinCells; t += kBrickThreads) {
            const unsigned n = s_mom[t];
            if (!n) continue;
            const unsigned* m = s_mom + t;
            unsigned long long M[8];
            M[0] = n;                                                      // {}
            M[4] = m[1 * kWinCells];                                       // {x}: A
            M[2] = m[2 * kWinCells];                                       // {y}: B
            M[1] = m[3 * kWinCells];                                       // {z}: D
            M[6] = m[4 * kWinCells] + ((unsigned long long)m[5 * kWinCells] << 17);    // {x,y}: AB
            M[5] = m[6 * kWinCells] + ((unsigned long long)m[7 * kWinCells] << 17);    // {x,z}: AD
            M[3] = m[8 * kWinCells] + ((unsigned long long)m[9 * kWinCells] << 17);    // {y,z}: BD
            M[7] = m[10 * kWinCells] + ((unsigned long long)m[11 * kWinCells] << 17) +
                   ((unsigned long long)m[12 * kWinCells] << 34);                      // {x,y,z}: ABD
            corners_from_moments(M);
            const int x = t / (kCY * kCZ), y = (t / kCZ) % kCY, z = t % kCZ;
            const int nb = (x * kNY + y) * kNZ + z;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int off = ((c >> 2) ? kNY * kNZ : 0) + (((c >> 1) & 1) ? kNZ : 0) + (c & 1);
                wrap |= tile_add_checked(t_lo, t_hi, nb + off, M[c]);
            }
        }
        __syncthreads();
        for (int t = tid; t < kWinNodes; t += kBrickThreads) {
            const unsigned long long v = (unsigned long long)t_lo[t] | ((unsigned long long)t_hi[t] << 32);
            if (!v) continue;
            const int x = wx0 + t / (kNY * kNZ), y = wy0 + (t / kNZ) % kNY, z = wz0 + t % kNZ;
            const unsigned long long old = atomicAdd(a.rho + lin(a.g, x, y, z), v);
            wrap |= old + v < old;
        }
        __syncthreads();
    }
    if (wrap) atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_RHO_OVERFLOW);
    const double tot = block_sum(e2);
    if (tid == 0 && tot != 0.0) atomicAdd(&a.sc->energy[a.s], tot);
    const double np = block_sum(npushed), nk = block_sum(nkept);
    if (tid == 0) {
        if (np > 0.0) atomicAdd(&a.sc->pushed[a.s], (unsigned long long)np);
        if (nk > 0.0) atomicAdd(&a.sc->survived[a.s], (unsigned long long)nk);
    }
}

// Writes a particle created in FP64 into a species slot (split precision).
template <typename T>
__device__ __forceinline__ void store_split(SoaT<T> p, long long slot, int i, int j, int k, T ox, T oy, T oz,
                                            double vx, double vy, double vz) {
    p.cell[slot] = pack_cell(i, j, k);
    p.ox[slot] = ox; p.oy[slot] = oy; p.oz[slot] = oz;
    p.vx[slot] = (T)vx; p.vy[slot] = (T)vy; p.vz[slot] = (T)vz;
}

template <typename T>
struct SourceArgsT {
    SoaT<T> p[FOPIS_MAX_SPECIES];
    long long cap[FOPIS_MAX_SPECIES];
    Grid g;
    const uint8_t* cellmap;
    unsigned long long* rho;       // base of [nsp][N]
    long long N;
    AbsorbList ab;
    DevScalars* sc;
    uint64_t seed;
    int fused;                     // 1: move, absorb-check and deposit now
};

// Finishes a newly created particle: in the fused step it is moved (emission
// only), checked against the bodies and deposited; it is then appended. Every
// active lane of the warp calls it: slots are reserved with one atomic per
// species per warp, and the kinetic energy goes to the block's accumulator
// s_energy (flushed once per block by the caller).
template <typename T>
__device__ void finish_source(const SourceArgsT<T>& a, int s, double x, double y, double z, double vx, double vy,
                              double vz, bool move, bool want, double* s_energy) {
    bool live = want;
    int i = 0, j = 0, k = 0;
    T ox = (T)0, oy = (T)0, oz = (T)0;
    if (live && a.fused && move) {
        x += vx; y += vy; z += vz;
        live = axis_boundary_d(a.g, 0, x) && axis_boundary_d(a.g, 1, y) && axis_boundary_d(a.g, 2, z);
    }
    if (live) {
        split(x, i, ox); split(y, j, oy); split(z, k, oz);
        if (!cell_in_range(a.g, i, j, k)) { live = false; atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_NONFINITE); }
    }
    bool absorbed = false;
    if (live && a.fused && a.cellmap) absorbed = a.cellmap[lin(a.g, i, j, k)] != 0;
    if (absorbed) {
        const unsigned long long slot = atomicAdd(&a.sc->absorbed_n, 1ull);
        if ((long long)slot < a.ab.cap) {
            a.ab.cell[slot] = pack_cell(i, j, k);
            a.ab.ox[slot] = ox; a.ab.oy[slot] = oy; a.ab.oz[slot] = oz;
            a.ab.vx[slot] = (T)vx; a.ab.vy[slot] = (T)vy; a.ab.vz[slot] = (T)vz;
            a.ab.species[slot] = (uint8_t)s;
            a.ab.object[slot] = (uint8_t)(a.cellmap[lin(a.g, i, j, k)] - 1);
        } else {
            atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_ABSORB_OVERFLOW);
        }
        live = false;
    }
    if (live && a.fused) {
        const long long b = lin(a.g, i, j, k);
        if constexpr (sizeof(T) == 4) {
            unsigned long long w[8];
            corner_weights(ox, oy, oz, w);
            unsigned long long* rho = a.rho + (long long)s * a.N;
            bool wrap = false;
#pragma unroll
            for (int t = 0; t < 8; ++t)
                if (w[t]) {
                    const unsigned long long old = atomicAdd(rho + b + corner_offset(a.g, t), w[t]);
                    wrap |= old + w[t] < old;
                }
            if (wrap) atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_RHO_OVERFLOW);
        } else {
            long long off[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) off[t] = corner_offset(a.g, t);
            deposit_f64(reinterpret_cast<double*>(a.rho) + (long long)s * a.N, b, off, ox, oy, oz);
        }
        const T fx = (T)vx, fy = (T)vy, fz = (T)vz;
        atomicAdd(&s_energy[s], (double)fx * fx + (double)fy * fy + (double)fz * fz);
    }
    const unsigned act = __activemask();
    const unsigned grp = __match_any_sync(act, live ? s : -1);
    if (!live) return;
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    unsigned long long base = 0;
    if (lane == leader) {
        base = atomicAdd(&a.sc->count[s], (unsigned long long)__popc(grp));
        atomicAdd(&a.sc->added[s], (unsigned long long)__popc(grp));
    }
    base = __shfl_sync(grp, base, leader);
    const unsigned long long slot = base + __popc(grp & ((1u << lane) - 1u));
    if ((long long)slot < a.cap[s]) store_split(a.p[s], (long long)slot, i, j, k, ox, oy, oz, vx, vy, vz);
    else atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_PARTICLE_OVERFLOW);
}

__device__ __forceinline__ void energy_init(double* s_energy) {
    for (int t = threadIdx.x; t < FOPIS_MAX_SPECIES; t += blockDim.x) s_energy[t] = 0.0;
    __syncthreads();
}
template <typename T>
__device__ __forceinline__ void energy_flush(const SourceArgsT<T>& a, const double* s_energy) {
    __syncthreads();
    for (int t = threadIdx.x; t < FOPIS_MAX_SPECIES; t += blockDim.x)
        if (s_energy[t] != 0.0) atomicAdd(&a.sc->energy[t], s_energy[t]);
}

// ------------------------------------------------------------------ injection
struct InjectTable {
    int n;                         // batches
    int species[FOPIS_MAX_SPECIES * 6];
    int face[FOPIS_MAX_SPECIES * 6];
    long long start[FOPIS_MAX_SPECIES * 6 + 1];
    double vth[FOPIS_MAX_SPECIES * 6], dev[FOPIS_MAX_SPECIES * 6];
    double drift[FOPIS_MAX_SPECIES * 6][3];
    double maxe[3];                // RootGrid max_x/y/z (RootGridParticle.cpp:196-203)
    long long step;
};

// One injected particle: AmbientParticleType::generateNewInjectionVelocity
// (AmbientParticleType.cpp:101-157, rejection redrawing all three components)
// and generateNewParticle with the slab ranges of
// RootGrid::injectParticlesFromBoundary (RootGridParticle.cpp:212-302).
template <typename T>
__global__ void inject_kernel(SourceArgsT<T> a, InjectTable tb) {
    __shared__ double s_energy[FOPIS_MAX_SPECIES];
    energy_init(s_energy);
    const long long total = tb.start[tb.n];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int b = 0;
        while (b + 1 < tb.n && tb.start[b + 1] <= t) ++b;
        const uint32_t idx = (uint32_t)(t - tb.start[b]);
        const int s = tb.species[b], face = tb.face[b], axis = face >> 1;
        const double sign = (face & 1) ? -1.0 : 1.0;
        const uint32_t cc = (uint32_t)s | ((uint32_t)face << 8), dtag = TAG_INJECT << 24;
        double v[3] = {0, 0, 0};
        int attempt = 0;
        for (; attempt < 256; ++attempt) {
            const U2 r0 = draw2(a.seed, idx, (uint32_t)tb.step, cc, dtag | (uint32_t)(2 * attempt));
            const U2 r1 = draw2(a.seed, idx, (uint32_t)tb.step, cc, dtag | (uint32_t)(2 * attempt + 1));
            double n0, n1, n2, n3;
            box_muller(r0.a, r0.b, n0, n1);
            box_muller(r1.a, r1.b, n2, n3);
            const double nn[3] = {n0, n1, n2};
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] = tb.drift[b][c] + (c == axis ? tb.vth[b] : tb.dev[b]) * nn[c];
            if (!((v[axis] * sign) < 0.0)) break;
        }
        if (attempt == 256) atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_INJECT_REJECTS);
        const U2 q0 = draw2(a.seed, idx, (uint32_t)tb.step, cc, dtag | 0xFFF0u);
        const U2 q1 = draw2(a.seed, idx, (uint32_t)tb.step, cc, dtag | 0xFFF1u);
        const double u[3] = {q0.a, q0.b, q1.a};
        double lo[3] = {0, 0, 0}, hi[3] = {tb.maxe[0], tb.maxe[1], tb.maxe[2]};
        if ((face & 1) == 0) hi[axis] = v[axis];
        else lo[axis] = tb.maxe[axis] + v[axis];
        double x[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) x[c] = lo[c] + (hi[c] - lo[c]) * u[c];
        finish_source(a, s, x[0], x[1], x[2], v[0], v[1], v[2], false, true, s_energy);
    }
    energy_flush(a, s_energy);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.sc->injected, (unsigned long long)total);
}

// ------------------------------------------------------------------ emission
struct EmitArgs {
    int obj, s, K, eaxis;
    double ev[3];
    double vth;
    int n_lit;
    const int32_t* lit;          // cmat numbers
    const int32_t* lit_ijk;      // packed node of each lit cmat
    const int32_t* node_cmat;
    long long* charge_tmp;       // this object's [nsp][n_cmat]
    int n_cmat;
    long long step;
};

__device__ __forceinline__ long long qsurf(double d) {
    long long q = __double2ll_rn(d * kSurfaceScale);
    return q < 0 ? 0 : (q > kSurfaceOne ? kSurfaceOne : q);
}

// Looks up the cmat number of node (i,j,k) for object obj; -1 when absent.
__device__ __forceinline__ int cmat_of(const Grid& g, const int32_t* node_cmat, int obj, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= g.cx || j >= g.cy || k >= g.cz) return -1;
    const int32_t v = node_cmat[lin(g, i, j, k)];
    if (v < 0 || (v >> 24) != obj) return -1;
    return v & 0xFFFFFF;
}

// Fixed-point bilinear surface charge of Spacecraft::distributeInnerParticle
// ChargeTo{X,Y,Z}surface / subtractChargeOfParticleFrom{X,Y,Z}surface
// (Spacecraft.cpp:594-613, :945-970): in-face coordinates rounded to 20 bits,
// four weights summing to 2^40, signed by add (+1 absorb, -1 emit).
__device__ bool surface_charge(const Grid& g, const int32_t* node_cmat, int obj, long long* tmp, int axis, int pi,
                               int pj, int pk, double d1a, double d1b, long long sign) {
    const long long qa = qsurf(d1a), qb = qsurf(d1b);
    const long long wa[2] = {kSurfaceOne - qa, qa}, wb[2] = {kSurfaceOne - qb, qb};
    int nodes[4];
    // corner order (a,b) = 00, 10, 01, 11 as the reference lists them
    const int da[4] = {0, 1, 0, 1}, db[4] = {0, 0, 1, 1};
    for (int t = 0; t < 4; ++t) {
        int ii = pi, jj = pj, kk = pk;
        if (axis == 0) { jj += da[t]; kk += db[t]; }
        else if (axis == 1) { ii += da[t]; kk += db[t]; }
        else { ii += da[t]; jj += db[t]; }
        nodes[t] = cmat_of(g, node_cmat, obj, ii, jj, kk);
        if (nodes[t] < 0) return false;
    }
    for (int t = 0; t < 4; ++t) {
        const long long w = wa[da[t]] * wb[db[t]] * sign;
        if (w) atomicAdd((unsigned long long*)(tmp + nodes[t]), (unsigned long long)w);
    }
    return true;
}

// One photoelectron per thread: PhotoElectronParticleType::generateNewParticle
// (PhotoElectronParticleType.cpp:9-101) at a lit node of the emitting face,
// its charge taken off the surface at its next crossing point
// (Spacecraft::emitParticles, Spacecraft.cpp:882-899).
template <typename T>
__global__ void emit_kernel(SourceArgsT<T> a, EmitArgs e) {
    __shared__ double s_energy[FOPIS_MAX_SPECIES];
    energy_init(s_energy);
    const long long total = (long long)e.n_lit * e.K;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int node = (int)(t / e.K);
        const uint32_t m = (uint32_t)(t % e.K);
        const int cm = e.lit[node];
        int ni, nj, nk;
        unpack_cell(e.lit_ijk[node], ni, nj, nk);
        const double rel[3] = {(double)(ni - 1), (double)(nj - 1), (double)(nk - 1)};
        const uint32_t cc = (uint32_t)e.s | ((uint32_t)cm << 8), dtag = TAG_EMIT << 24;
        const U2 r0 = draw2(a.seed, m, (uint32_t)e.step, cc, dtag | 0);
        const U2 r1 = draw2(a.seed, m, (uint32_t)e.step, cc, dtag | 1);
        const U2 r2 = draw2(a.seed, m, (uint32_t)e.step, cc, dtag | 2);
        const double dep = asin(2.0 * r0.a - 1.0);
        const double az = 2.0 * 3.14159265358979323846 * r0.b;
        const double cd = cos(dep), sd = sin(dep), ca = cos(az), sa = sin(az);
        double v[3];
        if (e.eaxis == 0) { v[0] = e.vth * cd * e.ev[0]; v[1] = e.vth * sd * ca; v[2] = e.vth * sd * sa; }
        else if (e.eaxis == 1) { v[0] = e.vth * sd * sa; v[1] = e.vth * cd * e.ev[1]; v[2] = e.vth * sd * ca; }
        else { v[0] = e.vth * sd * ca; v[1] = e.vth * sd * sa; v[2] = e.vth * cd * e.ev[2]; }
        const double tw = r1.a;
        double x[3] = {rel[0] + (tw - 1.0) * v[0], rel[1] + (tw - 1.0) * v[1], rel[2] + (tw - 1.0) * v[2]};
        if (e.eaxis == 0) { x[1] += r1.b; x[2] += r2.a; }
        else if (e.eaxis == 1) { x[0] += r1.b; x[2] += r2.a; }
        else { x[0] += r1.b; x[1] += r2.a; }
        // Particle::getNext{X,Y,Z}CrossPoint (src/Particle/particle.cpp:206-255)
        double cp[3] = {x[0], x[1], x[2]};
        const int ax = e.eaxis;
        const double fl = floor(x[ax]);
        const double d1 = x[ax] - fl, d2 = 1.0 - d1;
        if (v[ax] > 0.0) {
            const double mv = d2 / v[ax];
            for (int c = 0; c < 3; ++c) cp[c] = (c == ax) ? ceil(x[c]) : x[c] + v[c] * mv;
        } else if (v[ax] < 0.0) {
            const double mv = d1 / (-v[ax]);
            for (int c = 0; c < 3; ++c) cp[c] = (c == ax) ? floor(x[c]) : x[c] + v[c] * mv;
        }
        const double f0 = floor(cp[0]), f1 = floor(cp[1]), f2 = floor(cp[2]);
        const int pi = (int)f0 + 1, pj = (int)f1 + 1, pk = (int)f2 + 1;
        const double dd[3] = {cp[0] - f0, cp[1] - f1, cp[2] - f2};
        const int oa = ax == 0 ? 1 : 0, ob = ax == 2 ? 1 : 2;
        long long* tmp = e.charge_tmp + (long long)e.s * e.n_cmat;
        if (!surface_charge(a.g, e.node_cmat, e.obj, tmp, ax, pi, pj, pk, dd[oa], dd[ob], -1))
            atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_BAD_CMAT_NODE);
        finish_source(a, e.s, x[0], x[1], x[2], v[0], v[1], v[2], true, true, s_energy);
    }
    energy_flush(a, s_energy);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.sc->emitted_by[e.obj][e.s], (unsigned long long)total);
}

// ------------------------------------------------------------------ absorption
struct AbsorbArgs {
    AbsorbList ab;
    Grid g;
    const uint8_t* cellmap;
    const int32_t* node_cmat;
    long long* charge_tmp[FOPIS_MAX_OBJECTS];
    int n_cmat[FOPIS_MAX_OBJECTS];
    int secondary[FOPIS_MAX_OBJECTS];   // the body emits secondaries: record its hits
    IncidentList inc;
    DevScalars* sc;
};

struct DPos {  // Position in FP64 (include/position.hpp)
    int i, j, k;
    double d1[3];
    __device__ void set(double x, double y, double z) {
        const double f0 = floor(x), f1 = floor(y), f2 = floor(z);
        i = (int)f0 + 1; j = (int)f1 + 1; k = (int)f2 + 1;
        d1[0] = x - f0; d1[1] = y - f1; d1[2] = z - f2;
    }
};

__device__ __forceinline__ bool valid_cell(const Grid& g, int i, int j, int k) {
    return i >= 0 && i < g.n[0] + 1 && j >= 0 && j < g.n[1] + 1 && k >= 0 && k < g.n[2] + 1;
}
__device__ __forceinline__ bool cell_in(const AbsorbArgs& a, int obj, int i, int j, int k) {
    if (!valid_cell(a.g, i, j, k)) return false;
    return a.cellmap[lin(a.g, i, j, k)] == obj + 1;
}

// Spacecraft::is{X,Y,Z}surfacePoint (Spacecraft.cpp:462-506) for axis ax.
__device__ bool surface_point(const AbsorbArgs& a, int obj, const DPos& p, int ax, int sign) {
    if (p.d1[ax] >= 1e-10) return false;
    int di = 0, dj = 0, dk = 0;
    if (ax == 0) di = 1; else if (ax == 1) dj = 1; else dk = 1;
    if (valid_cell(a.g, p.i, p.j, p.k) && valid_cell(a.g, p.i - di, p.j - dj, p.k - dk)) {
        const bool here = cell_in(a, obj, p.i, p.j, p.k), below = cell_in(a, obj, p.i - di, p.j - dj, p.k - dk);
        return sign > 0 ? (here && !below) : (!here && below);
    }
    const int oa[3][3] = {{0, 1, 0}, {1, 0, 0}, {1, 0, 0}};
    const int ob[3][3] = {{0, 0, 1}, {0, 0, 1}, {0, 1, 0}};
    for (int t = 0; t < 4; ++t) {
        const int ii = p.i + ((t & 1) ? oa[ax][0] : 0) + ((t & 2) ? ob[ax][0] : 0);
        const int jj = p.j + ((t & 1) ? oa[ax][1] : 0) + ((t & 2) ? ob[ax][1] : 0);
        const int kk = p.k + ((t & 1) ? oa[ax][2] : 0) + ((t & 2) ? ob[ax][2] : 0);
        if (cmat_of(a.g, a.node_cmat, obj, ii, jj, kk) < 0) return false;
    }
    return true;
}

// Particle::get{X,Y,Z}MoveRatio (src/Particle/particle.cpp:46-80).
__device__ __forceinline__ double move_ratio(double d1, double v) {
    if (v == 0.0) return 0.0;
    return v > 0.0 ? d1 / fabs(v) : (1.0 - d1) / fabs(v);
}

// Particle::computeCrossPoints (particle.cpp:82-204, with the xz-case
// comparison `mvx <= mvx` that always puts x first) for the particle at
// (x, y, z) that moved by v this step, and the first crossing that is a body
// face whose axis is not `skip` (Spacecraft::distributeInnerParticleCharge,
// Spacecraft.cpp:556-591; distributeInnerParticleChargeForSecondary skips the
// axis it was emitted from, SecondaryEmission.cpp:35-110). Returns the face
// axis (-1: none) with the crossing as a position and as coordinates.
__device__ int find_body_face(const AbsorbArgs& a, int obj, double x, double y, double z, double vx, double vy,
                              double vz, int skip, DPos& hit, double hitc[3]) {
    DPos pos, old;
    pos.set(x, y, z);
    old.set(x - vx, y - vy, z - vz);
    const double ox_[3] = {x - vx, y - vy, z - vz};
    const double v[3] = {vx, vy, vz};
    const double mv[3] = {1.0 - move_ratio(pos.d1[0], vx), 1.0 - move_ratio(pos.d1[1], vy), 1.0 - move_ratio(pos.d1[2], vz)};
    const bool mvd[3] = {pos.i != old.i, pos.j != old.j, pos.k != old.k};
    int order[3], cnt = 0;
    const int count = (int)mvd[0] + (int)mvd[1] + (int)mvd[2];
    const double mvx = mv[0], mvy = mv[1], mvz = mv[2];
    if (count == 3) {
        if (mvx <= mvy) {
            if (mvx <= mvz) { order[0] = 0; if (mvy <= mvz) { order[1] = 1; order[2] = 2; } else { order[1] = 2; order[2] = 1; } }
            else { order[0] = 2; order[1] = 0; order[2] = 1; }
        } else {
            if (mvy <= mvz) { order[0] = 1; if (mvx <= mvz) { order[1] = 0; order[2] = 2; } else { order[1] = 2; order[2] = 0; } }
            else { order[0] = 2; order[1] = 1; order[2] = 0; }
        }
        cnt = 3;
    } else if (count == 2) {
        if (mvd[0] && mvd[1]) { if (mvx <= mvy) { order[0] = 0; order[1] = 1; } else { order[0] = 1; order[1] = 0; } }
        else if (mvd[0]) { order[0] = 0; order[1] = 2; }
        else { if (mvy <= mvz) { order[0] = 1; order[1] = 2; } else { order[0] = 2; order[1] = 1; } }
        cnt = 2;
    } else if (count == 1) {
        order[0] = mvd[0] ? 0 : (mvd[1] ? 1 : 2);
        cnt = 1;
    }
    const int sgn[3] = {vx > 0.0 ? 1 : -1, vy > 0.0 ? 1 : -1, vz > 0.0 ? 1 : -1};
    for (int q = 0; q < cnt; ++q) {
        const int ax0 = order[q];
        double c[3];
        for (int r = 0; r < 3; ++r)
            c[r] = (r == ax0) ? (v[ax0] > 0.0 ? ceil(ox_[r]) : floor(ox_[r])) : ox_[r] + v[r] * mv[ax0];
        DPos cp;
        cp.set(c[0], c[1], c[2]);
        for (int ax = 0; ax < 3; ++ax) {
            if (ax == skip) continue;
            if (surface_point(a, obj, cp, ax, sgn[ax])) {
                hit = cp;
                hitc[0] = c[0]; hitc[1] = c[1]; hitc[2] = c[2];
                return ax;
            }
        }
    }
    return -1;
}

// Absorbed particle: the charge goes to the first body face it crossed
// (bilinear, fixed point); for a body that emits secondaries the hit is kept
// as an incident event (Spacecraft::addIncidentEvent with the move ratio along
// the face axis as the remaining time, SecondaryEmission.cpp:14-33).
__global__ void absorb_kernel(AbsorbArgs a) {
    const long long n = (long long)min(a.sc->absorbed_n, (unsigned long long)a.ab.cap);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int s = a.ab.species[t], obj = a.ab.object[t];
        int ci, cj, ck;
        unpack_cell(a.ab.cell[t], ci, cj, ck);
        const double x = (ci - 1) + (double)a.ab.ox[t], y = (cj - 1) + (double)a.ab.oy[t], z = (ck - 1) + (double)a.ab.oz[t];
        const double vx = a.ab.vx[t], vy = a.ab.vy[t], vz = a.ab.vz[t];
        DPos cp;
        double cc[3];
        const int ax = find_body_face(a, obj, x, y, z, vx, vy, vz, -1, cp, cc);
        if (ax >= 0) {
            long long* tmp = a.charge_tmp[obj] + (long long)s * a.n_cmat[obj];
            const int oa = ax == 0 ? 1 : 0, ob = ax == 2 ? 1 : 2;
            if (!surface_charge(a.g, a.node_cmat, obj, tmp, ax, cp.i, cp.j, cp.k, cp.d1[oa], cp.d1[ob], 1))
                atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_BAD_CMAT_NODE);
            if (a.secondary[obj]) {
                const unsigned long long slot = atomicAdd(&a.sc->incident_n, 1ull);
                if ((long long)slot < a.inc.cap) {
                    DPos pos;
                    pos.set(x, y, z);
                    const double v[3] = {vx, vy, vz};
                    a.inc.x[slot] = cc[0]; a.inc.y[slot] = cc[1]; a.inc.z[slot] = cc[2];
                    a.inc.vx[slot] = vx; a.inc.vy[slot] = vy; a.inc.vz[slot] = vz;
                    a.inc.trem[slot] = move_ratio(pos.d1[ax], v[ax]);
                    a.inc.species[slot] = (uint8_t)s;
                    a.inc.object[slot] = (uint8_t)obj;
                    a.inc.axis[slot] = (uint8_t)ax;
                } else {
                    atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_ABSORB_OVERFLOW);
                }
            }
        } else {
            atomicAdd(&a.sc->not_found, 1ull);
            atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_SURFACE_NOT_FOUND);
        }
        atomicAdd(&a.sc->absorbed_by[obj][s], 1ull);
    }
}

// ------------------------------------------------------------------ secondary electrons
// Spacecraft::emitParticles' secondary branch (Spacecraft.cpp:901-937) with
// SecondaryParticleType::generateNewParticles (SecondaryParticleType.cpp:16-51)
// on the test material the reference hard-codes (Fermi energy 9.1 eV, delta_max
// 3.0 at 420 eV, Z = 13). Per incident: elastic backscatter with probability r,
// inelastic backscatter with eta, else floor(delta') + (u < frac) true
// secondaries, delta' = delta / (1 - r - eta) (Whipple's coefficients,
// :162-194). The draws are Philox keyed by the incident's own content (its
// crossing point and velocity rounded to 2^-24, species, axis and object) and
// the step, so an incident gives the same secondaries wherever it is listed,
// and runs whose trajectories agree to far below 2^-24 draw the same ones.
constexpr int kMaxSecondaries = 64;   // per incident; more latch FOPIS_DEV_PARTICLE_OVERFLOW
struct SeeMaterial {
    static constexpr double fermi = 9.1, delta_max = 3.0, eps_max = 420.0, z = 13.0;
};

__device__ inline uint64_t see_mix(uint64_t h, uint64_t w) {
    h ^= w;
    h *= 0x100000001B3ull;
    h ^= h >> 29;
    return h;
}
__device__ inline uint64_t incident_key(double x, double y, double z, double vx, double vy, double vz, int species,
                                                 int axis, int object) {
    const double d[6] = {x, y, z, vx, vy, vz};
    uint64_t h = 0xCBF29CE484222325ull;
    for (int q = 0; q < 6; ++q) h = see_mix(h, (uint64_t)__double2ll_rn(d[q] * 16777216.0));
    return see_mix(h, (uint64_t)species | ((uint64_t)axis << 8) | ((uint64_t)object << 16));
}

struct SecondaryArgs {
    IncidentList inc;
    long long n;                           // incidents
    int sec[FOPIS_MAX_OBJECTS];            // secondary species of each object
    double mass[FOPIS_MAX_SPECIES], charge[FOPIS_MAX_SPECIES], vth[FOPIS_MAX_SPECIES];
    double energy_ev;
    uint64_t seed;
    long long step;
};

// What one incident emits: kind (0 none, 1 elastic, 2 inelastic, 3 true) and count.
struct SeePlan { int kind, count; };
__device__ SeePlan see_plan(const SecondaryArgs& e, long long t, uint64_t key) {
    const int s = e.inc.species[t], ax = e.inc.axis[t];
    const double v[3] = {e.inc.vx[t], e.inc.vy[t], e.inc.vz[t]};
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double E = 0.5 * e.mass[s] * v2 * e.energy_ev;                 // IncidentInfo_t energy in eV
    const double th = acos(fabs(v[ax]) / sqrt(v2));                       // angle from the normal
    const double ct = cos(th);
    using M = SeeMaterial;
    double r = 0.0, eta = 0.0;
    if (e.charge[s] < 0.0) {
        const double f3 = M::fermi * M::fermi * M::fermi;
        r = (1.0 / 13.54) * (f3 * M::fermi) / (16.0 * ((E + M::fermi) * (E + M::fermi) * (E + M::fermi) + f3));
        const double eta1 = 1.0 - pow(2.0 / E, 0.037 * M::z);
        const double eta2 = 0.1 * exp(-E / 5000.0);
        double eta0 = 0.0;
        if (E > 50.0 && E < 1000.0) eta0 = log(E / 50.0) / log(20.0);
        else if (E > 1000.0) eta0 = 1.0;
        eta = eta0 * (eta1 + eta2) * (7.37 * pow(M::z, -0.56875)) * (1.0 - ct);
    }
    const double delta = (1.114 * M::delta_max / ct) * pow(M::eps_max / E, 0.35) *
                         (1.0 - exp(-2.28 * ct * pow(E / M::eps_max, 1.35)));
    const U2 u = draw2(e.seed, (uint32_t)key, (uint32_t)(key >> 32), (uint32_t)e.step, TAG_SECONDARY << 24);
    if (u.a < r) return {1, 1};
    if (u.a < r + eta) return {2, 1};
    const double d = delta / (1.0 - r - eta);
    const double fl = floor(d);
    int cnt = (int)fl + ((u.b < d - fl) ? 1 : 0);
    return {3, cnt};
}

__device__ __forceinline__ uint64_t incident_key_at(const SecondaryArgs& e, long long t) {
    return incident_key(e.inc.x[t], e.inc.y[t], e.inc.z[t], e.inc.vx[t], e.inc.vy[t], e.inc.vz[t], e.inc.species[t],
                        e.inc.axis[t], e.inc.object[t]);
}

// Count pass: the secondaries of every incident, and their total.
__global__ void see_count_kernel(SecondaryArgs e, DevScalars* sc) {
    unsigned long long tot = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < e.n; t += (long long)gridDim.x * blockDim.x) {
        int c = 0;
        if (e.sec[e.inc.object[t]] >= 0) c = min(see_plan(e, t, incident_key_at(e, t)).count, kMaxSecondaries);
        e.inc.count[t] = c;
        tot += (unsigned long long)c;
    }
    for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(kFull, tot, o);
    if ((threadIdx.x & 31) == 0 && tot) atomicAdd(&sc->secondary_n, tot);
}

// Emission pass: each secondary leaves the crossing point for the remaining
// time with its new velocity. Outside the body its charge comes off the face
// it left, at the next crossing of its back-dated position along the incident
// axis (Spacecraft::subtractChargeOfParticleFrom{X,Y,Z}surface, :945-970), and
// it is appended; inside the body it is absorbed at once on a face of another
// axis (distributeInnerParticleChargeForSecondary). The reference records that
// re-absorption as an incident too, in the list it is iterating and clears
// right after, so it emits nothing here.
template <typename T>
__global__ void see_emit_kernel(SourceArgsT<T> a, SecondaryArgs e, AbsorbArgs b) {
    __shared__ double s_energy[FOPIS_MAX_SPECIES];
    energy_init(s_energy);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < e.n; t += (long long)gridDim.x * blockDim.x) {
        const int obj = e.inc.object[t], sec = e.sec[obj];
        if (sec < 0) continue;
        const uint64_t key = incident_key_at(e, t);
        const SeePlan plan = see_plan(e, t, key);
        if (plan.count > kMaxSecondaries) atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_PARTICLE_OVERFLOW);
        const int n = min(plan.count, kMaxSecondaries);
        const int s = e.inc.species[t], ax = e.inc.axis[t];
        const double vin[3] = {e.inc.vx[t], e.inc.vy[t], e.inc.vz[t]};
        const double cp[3] = {e.inc.x[t], e.inc.y[t], e.inc.z[t]};
        const double trem = e.inc.trem[t];
        double speed = e.vth[sec];                                          // true secondaries: sqrt(2 T / m)
        if (plan.kind == 2) {
            const U2 ue = draw2(e.seed, (uint32_t)key, (uint32_t)(key >> 32), (uint32_t)e.step, (TAG_SECONDARY << 24) | 1u);
            const double v2 = vin[0] * vin[0] + vin[1] * vin[1] + vin[2] * vin[2];
            speed = sqrt(2.0 * (ue.a * 0.5 * e.mass[s] * v2) / e.mass[sec]);   // uniform share of the incident energy
        }
        for (int m = 0; m < n; ++m) {
            double v[3];
            if (plan.kind == 1) {
                v[0] = vin[0]; v[1] = vin[1]; v[2] = vin[2];
                v[ax] = -v[ax];
            } else {
                const U2 ua = draw2(e.seed, (uint32_t)key, (uint32_t)(key >> 32), (uint32_t)e.step,
                                    (TAG_SECONDARY << 24) | (uint32_t)(2 + m));
                const double dep = asin(2.0 * ua.a - 1.0), az = 2.0 * 3.14159265358979323846 * ua.b;
                const double sgn = vin[ax] > 0.0 ? -1.0 : 1.0;
                const double cn = speed * cos(dep) * sgn, sa = speed * sin(dep) * cos(az), sb = speed * sin(dep) * sin(az);
                if (ax == 0) { v[0] = cn; v[1] = sa; v[2] = sb; }
                else if (ax == 1) { v[0] = sb; v[1] = cn; v[2] = sa; }
                else { v[0] = sa; v[1] = sb; v[2] = cn; }
            }
            const double x[3] = {cp[0] + trem * v[0], cp[1] + trem * v[1], cp[2] + trem * v[2]};
            DPos pos;
            pos.set(x[0], x[1], x[2]);
            long long* tmp = b.charge_tmp[obj] + (long long)sec * b.n_cmat[obj];
            if (cell_in(b, obj, pos.i, pos.j, pos.k)) {
                DPos hp;
                double hc[3];
                const int hax = find_body_face(b, obj, x[0], x[1], x[2], v[0], v[1], v[2], ax, hp, hc);
                if (hax >= 0) {
                    const int oa = hax == 0 ? 1 : 0, ob = hax == 2 ? 1 : 2;
                    if (!surface_charge(b.g, b.node_cmat, obj, tmp, hax, hp.i, hp.j, hp.k, hp.d1[oa], hp.d1[ob], 1))
                        atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_BAD_CMAT_NODE);
                } else {
                    atomicAdd(&a.sc->not_found, 1ull);
                    atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_SURFACE_NOT_FOUND);
                }
                atomicAdd(&a.sc->absorbed_by[obj][sec], 1ull);
                continue;
            }
            // Particle::getNext{X,Y,Z}CrossPoint (particle.cpp:206-255) of the position one step back
            double o[3] = {x[0] - v[0], x[1] - v[1], x[2] - v[2]}, c[3] = {o[0], o[1], o[2]};
            const double fo = floor(o[ax]), d1 = o[ax] - fo, d2 = 1.0 - d1;
            if (v[ax] > 0.0) {
                const double mv = d2 / v[ax];
                for (int r = 0; r < 3; ++r) c[r] = (r == ax) ? ceil(o[r]) : o[r] + v[r] * mv;
            } else if (v[ax] < 0.0) {
                const double mv = d1 / (-v[ax]);
                for (int r = 0; r < 3; ++r) c[r] = (r == ax) ? floor(o[r]) : o[r] + v[r] * mv;
            }
            DPos np;
            np.set(c[0], c[1], c[2]);
            const int oa = ax == 0 ? 1 : 0, ob = ax == 2 ? 1 : 2;
            if (!surface_charge(b.g, b.node_cmat, obj, tmp, ax, np.i, np.j, np.k, np.d1[oa], np.d1[ob], -1))
                atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_BAD_CMAT_NODE);
            atomicAdd(&a.sc->emitted_by[obj][sec], 1ull);
            finish_source(a, sec, x[0], x[1], x[2], v[0], v[1], v[2], true, true, s_energy);
        }
    }
    energy_flush(a, s_energy);
}

// ------------------------------------------------------------------ loading
template <typename T>
struct AmbientArgs {
    SoaT<T> p;
    long long cap;
    int s;
    long long total;
    double maxe[3];
    double drift[3], dev;
    uint64_t seed;
    Grid g;
    const uint8_t* cellmap;
    DevScalars* sc;
};

// RootGrid::RootGrid uniform loading (RootGrid.cpp:59-79): positions uniform in
// [0,max), velocities Maxwellian about the drift, particles inside a body
// dropped (Spacecraft::removeInnerParticle, Spacecraft.cpp:508-510).
template <typename T>
__global__ void ambient_kernel(AmbientArgs<T> a) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < a.total; base += stride) {
        const long long t = base + (threadIdx.x & 31);
        bool keep = t < a.total;
        int i = 0, j = 0, k = 0;
        T ox = 0, oy = 0, oz = 0;
        double vx = 0, vy = 0, vz = 0;
        if (keep) {
            const uint32_t c0 = (uint32_t)t, c1 = (uint32_t)(t >> 32), c2 = (uint32_t)a.s, dt = TAG_LOAD << 24;
            const U2 r0 = draw2(a.seed, c0, c1, c2, dt | 0), r1 = draw2(a.seed, c0, c1, c2, dt | 1);
            const U2 r2 = draw2(a.seed, c0, c1, c2, dt | 2), r3 = draw2(a.seed, c0, c1, c2, dt | 3);
            const double x = a.maxe[0] * r0.a, y = a.maxe[1] * r0.b, z = a.maxe[2] * r1.a;
            double n0, n1, n2, n3;
            box_muller(r1.b, r2.a, n0, n1);
            box_muller(r2.b, r3.a, n2, n3);
            vx = a.drift[0] + a.dev * n0; vy = a.drift[1] + a.dev * n1; vz = a.drift[2] + a.dev * n2;
            split(x, i, ox); split(y, j, oy); split(z, k, oz);
            if (a.cellmap && valid_cell(a.g, i, j, k) && a.cellmap[lin(a.g, i, j, k)]) keep = false;
        }
        const unsigned long long slot = warp_reserve(&a.sc->count[a.s], keep);
        if (keep) {
            if ((long long)slot < a.cap) store_split(a.p, (long long)slot, i, j, k, ox, oy, oz, vx, vy, vz);
            else atomicOr(&a.sc->status, (unsigned)FOPIS_DEV_PARTICLE_OVERFLOW);
        }
    }
}

struct Rec56 { double x, y, z, vx, vy, vz; int typeId, isValid; };

template <typename T>
__global__ void load56_kernel(SoaT<T> p, long long cap, unsigned long long* count, const Rec56* in, long long n, Grid g,
                              DevScalars* sc) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const long long t = base + (threadIdx.x & 31);
        bool keep = t < n && in[t].isValid;
        int i = 0, j = 0, k = 0;
        T ox = 0, oy = 0, oz = 0;
        if (keep) {
            split(in[t].x, i, ox); split(in[t].y, j, oy); split(in[t].z, k, oz);
            if (!cell_in_range(g, i, j, k)) { keep = false; atomicOr(&sc->status, (unsigned)FOPIS_DEV_NONFINITE); }
        }
        const unsigned long long slot = warp_reserve(count, keep);
        if (keep) {
            if ((long long)slot < cap) store_split(p, (long long)slot, i, j, k, ox, oy, oz, in[t].vx, in[t].vy, in[t].vz);
            else atomicOr(&sc->status, (unsigned)FOPIS_DEV_PARTICLE_OVERFLOW);
        }
    }
}

// Sum of v^2 over the valid particles of a species.
template <typename T>
__global__ void energy_kernel(SoaT<T> p, long long cap, const unsigned long long* count, double* out) {
    const long long n = (long long)min(*count, (unsigned long long)cap);
    double e = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        if (p.cell[t] >= 0) e += (double)p.vx[t] * p.vx[t] + (double)p.vy[t] * p.vy[t] + (double)p.vz[t] * p.vz[t];
    e = block_sum(e);
    if (threadIdx.x == 0 && e != 0.0) atomicAdd(out, e);
}

// ------------------------------------------------------------------ sort
// Two passes per species. Pass 1 moves every particle into its brick's slot
// range; pass 2 orders each brick's range by cell. Both write whole runs of
// consecutive slots (pass 1 groups a chunk by brick before it writes, pass 2
// gathers inside one brick), so every 32-byte sector of the destination is
// filled by one CTA within one chunk or brick: scattered 4-byte stores that
// leave sectors partial cost a DRAM fill and a write-back each.

// cnt[b] += particles of brick b (valid slots only), one atomic per warp and brick.
template <typename T>
__global__ void sort_count_kernel(SoaT<T> p, long long cap, const unsigned long long* count, Grid g, int32_t* cnt) {
    const long long n = (long long)min(*count, (unsigned long long)cap);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n; base += stride) {
        const long long t = base + (threadIdx.x & 31);
        const int32_t c = t < n ? p.cell[t] : -1;
        int key = -1 - (int)(threadIdx.x & 31);
        if (c >= 0) { int i, j, k; unpack_cell(c, i, j, k); key = brick_index(g, i, j, k); }
        const unsigned grp = __match_any_sync(kFull, key);
        const int lane = threadIdx.x & 31;
        if (c >= 0 && (__ffs(grp) - 1) == lane) atomicAdd(cnt + key, __popc(grp));
    }
}

// Exclusive scan of n int32 values in three passes (block sums, a single-block
// scan of the sums, block rescans).
constexpr int kScanThreads = 1024, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int ws[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(kFull, x, o); if (lane >= o) x += y; }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(kFull, s, o); if (lane >= o) s += y; }
        ws[lane] = s;
    }
    __syncthreads();
    const int pre = (w ? ws[w - 1] : 0) + x - v;
    *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return pre;
}

__global__ void scan_tiles_kernel(const int32_t* in, long long n, int32_t* partial) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int s = 0;
    for (int q = 0; q < kScanItems; ++q) if (base + q < n) s += in[base + q];
    int tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}
__global__ void scan_partials_kernel(int32_t* partial, int np) {
    int carry = 0;
    for (int b0 = 0; b0 < np; b0 += blockDim.x) {
        const int t = b0 + threadIdx.x;
        const int v = t < np ? partial[t] : 0;
        int tot;
        const int pre = block_exclusive_scan(v, &tot);
        if (t < np) partial[t] = carry + pre;
        carry += tot;
    }
    if (threadIdx.x == 0) partial[np] = carry;
}
__global__ void scan_apply_kernel(const int32_t* in, long long n, const int32_t* partial, int32_t* out) {
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems], s = 0;
    for (int q = 0; q < kScanItems; ++q) { v[q] = (base + q < n) ? in[base + q] : 0; s += v[q]; }
    int tot;
    int pre = block_exclusive_scan(s, &tot) + partial[blockIdx.x];
    for (int q = 0; q < kScanItems; ++q) { if (base + q < n) out[base + q] = pre; pre += v[q]; }
}

// Order-preserving export of slots [lo, hi): each tile of kScanTile slots
// counts its valid particles, the tile totals are scanned, and each tile
// writes its particles at its offset plus their rank inside the tile, so the
// records come out in slot order.
template <typename T>
__global__ void export_count_kernel(SoaT<T> p, long long lo, long long hi, int32_t* partial) {
    const long long base = lo + (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int n = 0;
    for (int q = 0; q < kScanItems; ++q) if (base + q < hi && p.cell[base + q] >= 0) ++n;
    int tot;
    block_exclusive_scan(n, &tot);
    if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

template <typename T>
__global__ void export_kernel(SoaT<T> p, long long lo, long long hi, int s, Rec56* out56, SoaT<T> raw,
                              const int32_t* partial) {
    const long long base = lo + (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int32_t cell[kScanItems];
    int n = 0;
    for (int q = 0; q < kScanItems; ++q) {
        cell[q] = base + q < hi ? p.cell[base + q] : -1;
        n += cell[q] >= 0;
    }
    int tot;
    long long slot = (long long)block_exclusive_scan(n, &tot) + partial[blockIdx.x];
    for (int q = 0; q < kScanItems; ++q) {
        if (cell[q] < 0) continue;
        const long long t = base + q;
        if (out56) {
            int i, j, k;
            unpack_cell(cell[q], i, j, k);
            Rec56 r;
            r.x = (i - 1) + (double)p.ox[t]; r.y = (j - 1) + (double)p.oy[t]; r.z = (k - 1) + (double)p.oz[t];
            r.vx = p.vx[t]; r.vy = p.vy[t]; r.vz = p.vz[t];
            r.typeId = s; r.isValid = 1;
            out56[slot] = r;
        } else {
            raw.cell[slot] = cell[q];
            raw.ox[slot] = p.ox[t]; raw.oy[slot] = p.oy[t]; raw.oz[slot] = p.oz[t];
            raw.vx[slot] = p.vx[t]; raw.vy[slot] = p.vy[t]; raw.vz[slot] = p.vz[t];
        }
        ++slot;
    }
}

// Pass 1. A CTA takes chunks of kSortChunk slots; a shared hash table maps
// each brick met in the chunk to a slot that counts its particles (ranks in
// lane order, so equal-brick lanes of a warp get consecutive places); one
// atomic per brick and chunk then reserves the brick's run in the cursor.
constexpr int kSortThreads = 256, kSortItems = 4, kSortChunk = kSortThreads * kSortItems;
constexpr int kSortSlots = 2 * kSortChunk;   // more slots than distinct bricks a chunk can hold

__device__ __forceinline__ int sort_slot(int* keys, int b) {
    const unsigned h = ((unsigned)b * 2654435761u) >> 21;   // 11 bits: kSortSlots = 2048
    for (int q = 0; q < kSortSlots; ++q) {
        const int s = (int)((h + q) & (kSortSlots - 1));
        const int k = keys[s];
        if (k == b) return s;
        if (k == -1) {
            const int old = atomicCAS(&keys[s], -1, b);
            if (old == -1 || old == b) return s;
        }
    }
    return -1;   // unreachable: at most kSortChunk distinct bricks in kSortSlots slots
}

template <typename T>
__global__ void __launch_bounds__(kSortThreads) sort_brick_scatter_kernel(SoaT<T> src, SoaT<T> dst, long long cap,
                                                                          const unsigned long long* count, Grid g,
                                                                          int32_t* cursor) {
    static_assert(kSortSlots == 2048, "sort_slot hashes to 11 bits");
    __shared__ int s_key[kSortSlots];   // brick of a slot, -1 while free
    __shared__ int s_cnt[kSortSlots];
    __shared__ int s_base[kSortSlots];
    const long long n = (long long)min(*count, (unsigned long long)cap);
    const int tid = threadIdx.x, lane = tid & 31;
    for (int q = tid; q < kSortSlots; q += kSortThreads) { s_key[q] = -1; s_cnt[q] = 0; }
    __syncthreads();
    for (long long c0 = (long long)blockIdx.x * kSortChunk; c0 < n; c0 += (long long)gridDim.x * kSortChunk) {
        int32_t cell[kSortItems];
        T f[kSortItems][6];
        int slot[kSortItems], rank[kSortItems];
#pragma unroll
        for (int e = 0; e < kSortItems; ++e) {
            const long long t = c0 + e * kSortThreads + tid;
            cell[e] = t < n ? src.cell[t] : -1;
            if (cell[e] >= 0) {
                f[e][0] = src.ox[t]; f[e][1] = src.oy[t]; f[e][2] = src.oz[t];
                f[e][3] = src.vx[t]; f[e][4] = src.vy[t]; f[e][5] = src.vz[t];
            }
        }
#pragma unroll
        for (int e = 0; e < kSortItems; ++e) {
            int b = -1 - lane;   // distinct per lane for empty slots
            if (cell[e] >= 0) { int i, j, k; unpack_cell(cell[e], i, j, k); b = brick_index(g, i, j, k); }
            const unsigned grp = __match_any_sync(kFull, b);
            const int leader = __ffs(grp) - 1;
            int sl = -1, r0 = 0;
            if (cell[e] >= 0 && lane == leader) {
                sl = sort_slot(s_key, b);
                if (sl >= 0) r0 = atomicAdd(&s_cnt[sl], __popc(grp));
            }
            slot[e] = __shfl_sync(kFull, sl, leader);
            rank[e] = __shfl_sync(kFull, r0, leader) + __popc(grp & ((1u << lane) - 1u));
        }
        __syncthreads();
        for (int q = tid; q < kSortSlots; q += kSortThreads)
            if (s_key[q] >= 0) s_base[q] = atomicAdd(cursor + s_key[q], s_cnt[q]);
        __syncthreads();
#pragma unroll
        for (int e = 0; e < kSortItems; ++e) {
            if (cell[e] < 0 || slot[e] < 0) continue;
            const long long d = (long long)s_base[slot[e]] + rank[e];
            dst.cell[d] = cell[e];
            dst.ox[d] = f[e][0]; dst.oy[d] = f[e][1]; dst.oz[d] = f[e][2];
            dst.vx[d] = f[e][3]; dst.vy[d] = f[e][4]; dst.vz[d] = f[e][5];
        }
        for (int q = tid; q < kSortSlots; q += kSortThreads) { s_key[q] = -1; s_cnt[q] = 0; }
        __syncthreads();
    }
}

// Pass 2. One CTA per brick (grid-stride): a shared histogram of the brick's
// 128 cells, its exclusive scan, then the inverse permutation and a gather
// inside the brick's range, so the stores run over consecutive slots. Bricks
// above kCellCap particles place each particle straight at its cell cursor.
// Loads are issued kCellBatch particles per thread at a time so their
// latencies overlap; shared counters take one atomic per warp and cell.
constexpr int kCellThreads = 256, kCellCap = 8192, kCellBatch = 4;

__device__ __forceinline__ int cell_rank(int* counter, int lc, bool valid) {
    const unsigned grp = __match_any_sync(kFull, valid ? lc : -1 - (int)(threadIdx.x & 31));
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    int r0 = 0;
    if (valid && lane == leader) r0 = atomicAdd(counter + lc, __popc(grp));
    return __shfl_sync(kFull, r0, leader) + __popc(grp & ((1u << lane) - 1u));
}

template <typename T>
__global__ void __launch_bounds__(kCellThreads) sort_cell_kernel(SoaT<T> src, SoaT<T> dst, const int32_t* brick_start,
                                                                 int nbricks) {
    __shared__ uint8_t s_lc[kCellCap];
    __shared__ uint16_t s_perm[kCellCap];
    __shared__ int s_off[kBrickCells];
    const int tid = threadIdx.x, lane = tid & 31;
    constexpr int kStep = kCellThreads * kCellBatch;
    for (int b = blockIdx.x; b < nbricks; b += gridDim.x) {
        const long long base = brick_start[b];
        const int n = brick_start[b + 1] - (int)base;
        if (n <= 0) continue;
        const bool fits = n <= kCellCap;
        if (tid < kBrickCells) s_off[tid] = 0;
        __syncthreads();
        for (int q0 = 0; q0 < n; q0 += kStep) {
            int lc[kCellBatch];
#pragma unroll
            for (int e = 0; e < kCellBatch; ++e) {
                const int q = q0 + e * kCellThreads + tid;
                lc[e] = -1;
                if (q < n) { int i, j, k; unpack_cell(src.cell[base + q], i, j, k); lc[e] = local_cell(i, j, k); }
            }
#pragma unroll
            for (int e = 0; e < kCellBatch; ++e) {
                const int q = q0 + e * kCellThreads + tid;
                if (fits && q < n) s_lc[q] = (uint8_t)lc[e];
                cell_rank(s_off, lc[e], q < n);
            }
        }
        __syncthreads();
        if (tid < 32) {   // exclusive scan of 128 counts, 4 per lane
            static_assert(kBrickCells == 128, "one warp scans 4 counts per lane");
            int v[4], sum = 0;
#pragma unroll
            for (int e = 0; e < 4; ++e) { v[e] = s_off[lane * 4 + e]; sum += v[e]; }
            int x = sum;
            for (int o = 1; o < 32; o <<= 1) { const int y = __shfl_up_sync(kFull, x, o); if (lane >= o) x += y; }
            int pre = x - sum;
#pragma unroll
            for (int e = 0; e < 4; ++e) { s_off[lane * 4 + e] = pre; pre += v[e]; }
        }
        __syncthreads();
        if (fits) {
            for (int q0 = 0; q0 < n; q0 += kCellThreads) {
                const int q = q0 + tid;
                const bool ok = q < n;
                const int lc = ok ? s_lc[q] : 0;
                const int r = cell_rank(s_off, lc, ok);
                if (ok) s_perm[r] = (uint16_t)q;
            }
            __syncthreads();
            for (int r0 = 0; r0 < n; r0 += kStep) {
                int32_t c[kCellBatch];
                T v[kCellBatch][6];
#pragma unroll
                for (int e = 0; e < kCellBatch; ++e) {
                    const int r = r0 + e * kCellThreads + tid;
                    if (r < n) {
                        const long long sidx = base + s_perm[r];
                        c[e] = src.cell[sidx];
                        v[e][0] = src.ox[sidx]; v[e][1] = src.oy[sidx]; v[e][2] = src.oz[sidx];
                        v[e][3] = src.vx[sidx]; v[e][4] = src.vy[sidx]; v[e][5] = src.vz[sidx];
                    }
                }
#pragma unroll
                for (int e = 0; e < kCellBatch; ++e) {
                    const int r = r0 + e * kCellThreads + tid;
                    if (r < n) {
                        const long long d = base + r;
                        dst.cell[d] = c[e];
                        dst.ox[d] = v[e][0]; dst.oy[d] = v[e][1]; dst.oz[d] = v[e][2];
                        dst.vx[d] = v[e][3]; dst.vy[d] = v[e][4]; dst.vz[d] = v[e][5];
                    }
                }
            }
        } else {
            for (int q0 = 0; q0 < n; q0 += kCellThreads) {
                const int q = q0 + tid;
                const bool ok = q < n;
                const long long sidx = base + (ok ? q : 0);
                const int32_t c = src.cell[sidx];
                int i, j, k;
                unpack_cell(c, i, j, k);
                const int r = cell_rank(s_off, local_cell(i, j, k), ok);
                if (!ok) continue;
                const long long d = base + r;
                dst.cell[d] = c;
                dst.ox[d] = src.ox[sidx]; dst.oy[d] = src.oy[sidx]; dst.oz[d] = src.oz[sidx];
                dst.vx[d] = src.vx[sidx]; dst.vy[d] = src.vy[sidx]; dst.vz[d] = src.vz[sidx];
            }
        }
        __syncthreads();
    }
}

int grid_for(long long n, int threads = kThreads) {
    const long long b = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}

// Particle arrays come from the device's stream-ordered pool, so growing them
// mid-run neither synchronises the device nor returns memory to the driver.
template <typename T>
void alloc_soa(SoaT<T>& s, int64_t cap, cudaStream_t st) {
    FOPIS_CUDA(cudaMallocAsync((void**)&s.cell, sizeof(int32_t) * cap, st));
    T** f[6] = {&s.ox, &s.oy, &s.oz, &s.vx, &s.vy, &s.vz};
    for (auto* q : f) FOPIS_CUDA(cudaMallocAsync((void**)q, sizeof(T) * cap, st));
}
template <typename T>
void free_soa(SoaT<T>& s, cudaStream_t st) {
    if (s.cell) cudaFreeAsync(s.cell, st);
    T* f[6] = {s.ox, s.oy, s.oz, s.vx, s.vy, s.vz};
    for (auto* q : f) if (q) cudaFreeAsync(q, st);
    s = SoaT<T>{};
}
template <typename T>
void copy_soa(SoaT<T>& d, const SoaT<T>& s, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    FOPIS_CUDA(cudaMemcpyAsync(d.cell, s.cell, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, st));
    T* df[6] = {d.ox, d.oy, d.oz, d.vx, d.vy, d.vz};
    T* sf[6] = {s.ox, s.oy, s.oz, s.vx, s.vy, s.vz};
    for (int t = 0; t < 6; ++t) FOPIS_CUDA(cudaMemcpyAsync(df[t], sf[t], sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
}

// The particle arrays of a precision: the live set and the sort target.
template <typename T> SoaT<T>* parts(Ctx& c);
template <> Soa* parts<float>(Ctx& c) { return c.sp; }
template <> Soa64* parts<double>(Ctx& c) { return c.dp; }
template <typename T> SoaT<T>* parts2(Ctx& c);
template <> Soa* parts2<float>(Ctx& c) { return c.sp2; }
template <> Soa64* parts2<double>(Ctx& c) { return c.dp2; }

template <typename T>
void alloc_species(Ctx& c, int s, int64_t cap) {
    SoaT<T> a{}, b{};
    alloc_soa(a, cap, c.st);
    alloc_soa(b, cap, c.st);
    FOPIS_CUDA(cudaMemsetAsync(a.cell, 0xff, sizeof(int32_t) * cap, c.st));
    if (c.cap[s] > 0) {
        sync_scalars(c);
        copy_soa(a, parts<T>(c)[s], std::min<int64_t>(c.nslots[s], c.cap[s]), c.st);
        free_soa(parts<T>(c)[s], c.st);
        free_soa(parts2<T>(c)[s], c.st);
    }
    parts<T>(c)[s] = a;
    parts2<T>(c)[s] = b;
}

}  // namespace

// Makes sure species s can hold at least `need` slots (grows both buffers).
void particles_alloc(Ctx& c, int s, int64_t need) {
    if (need <= c.cap[s]) return;
    const int64_t cap = std::max<int64_t>(need, 1024);
    if (c.fp64) alloc_species<double>(c, s, cap);
    else alloc_species<float>(c, s, cap);
    c.cap[s] = cap;
}

void sync_scalars(Ctx& c) {
    FOPIS_CUDA(cudaMemcpyAsync(c.h_sc, c.d_sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    for (int s = 0; s < c.nsp; ++s) c.nslots[s] = (int64_t)std::min<unsigned long long>(c.h_sc->count[s], (unsigned long long)c.cap[s]);
}

template <typename T>
static void append_aos(Ctx& c, int s, const void* host56, int64_t n) {
    sync_scalars(c);
    particles_alloc(c, s, (int64_t)((c.nslots[s] + n) * std::max(1.0, c.p.capacity_factor)) + 4096);
    const int64_t chunk = 1 << 20;
    Rec56* d = nullptr;
    FOPIS_CUDA(cudaMalloc(&d, sizeof(Rec56) * chunk));
    const Grid g = make_grid(c);
    for (int64_t off = 0; off < n; off += chunk) {
        const int64_t m = std::min(chunk, n - off);
        FOPIS_CUDA(cudaMemcpyAsync(d, (const char*)host56 + 56 * off, 56 * m, cudaMemcpyHostToDevice, c.st));
        ++c.launches;
        load56_kernel<<<grid_for(m), kThreads, 0, c.st>>>(parts<T>(c)[s], c.cap[s], &c.d_sc->count[s], d, m, g, c.d_sc);
        FOPIS_LAUNCH_CHECK();
    }
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    cudaFree(d);
    sync_scalars(c);
}

void particles_append_aos(Ctx& c, int s, const void* host56, int64_t n) {
    if (c.fp64) append_aos<double>(c, s, host56, n);
    else append_aos<float>(c, s, host56, n);
}

// Export chunks hold kExportChunk slots; `partial` has kExportTiles + 1 entries.
constexpr int64_t kExportChunk = 1 << 20;
constexpr int kExportTiles = (int)((kExportChunk + kScanTile - 1) / kScanTile);

template <typename T>
static int64_t export_range(Ctx& c, int s, Rec56* d56, SoaT<T>* raw, int64_t lo, int64_t hi, int32_t* partial) {
    const int tiles = (int)((hi - lo + kScanTile - 1) / kScanTile);
    ++c.launches;
    export_count_kernel<<<tiles, kScanThreads, 0, c.st>>>(parts<T>(c)[s], lo, hi, partial);
    ++c.launches;
    scan_partials_kernel<<<1, kScanThreads, 0, c.st>>>(partial, tiles);
    ++c.launches;
    export_kernel<<<tiles, kScanThreads, 0, c.st>>>(parts<T>(c)[s], lo, hi, s, d56, raw ? *raw : SoaT<T>{}, partial);
    FOPIS_LAUNCH_CHECK();
    int32_t k = 0;
    FOPIS_CUDA(cudaMemcpyAsync(&k, partial + tiles, sizeof(k), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    return (int64_t)k;
}

int64_t particles_export_aos(Ctx& c, int s, void* host56, int64_t cap) {
    sync_scalars(c);
    const int64_t n = c.nslots[s];
    const int64_t chunk = kExportChunk;
    Rec56* d = nullptr;
    int32_t* dc = nullptr;
    FOPIS_CUDA(cudaMalloc(&d, sizeof(Rec56) * chunk));
    FOPIS_CUDA(cudaMalloc(&dc, sizeof(int32_t) * (kExportTiles + 1)));
    int64_t total = 0;
    for (int64_t lo = 0; lo < n; lo += chunk) {
        const int64_t hi = std::min(n, lo + chunk);
        const int64_t k = c.fp64 ? export_range<double>(c, s, d, nullptr, lo, hi, dc)
                                 : export_range<float>(c, s, d, nullptr, lo, hi, dc);
        const int64_t w = std::max<int64_t>(0, std::min(k, cap - total));
        if (w > 0) FOPIS_CUDA(cudaMemcpy((char*)host56 + 56 * total, d, 56 * w, cudaMemcpyDeviceToHost));
        total += k;
    }
    cudaFree(d);
    cudaFree(dc);
    return total;
}

int64_t particles_export_raw(Ctx& c, int s, int32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                             float* vz, int64_t cap) {
    sync_scalars(c);
    const int64_t n = c.nslots[s];
    const int64_t chunk = kExportChunk;
    Soa raw{};
    alloc_soa(raw, chunk, c.st);
    int32_t* dc = nullptr;
    FOPIS_CUDA(cudaMalloc(&dc, sizeof(int32_t) * (kExportTiles + 1)));
    int64_t total = 0;
    for (int64_t lo = 0; lo < n; lo += chunk) {
        const int64_t hi = std::min(n, lo + chunk);
        const int64_t k = export_range(c, s, nullptr, &raw, lo, hi, dc);
        const int64_t w = std::max<int64_t>(0, std::min(k, cap - total));
        if (w > 0) {
            FOPIS_CUDA(cudaMemcpy(cell + total, raw.cell, 4 * w, cudaMemcpyDeviceToHost));
            float* dst[6] = {ox, oy, oz, vx, vy, vz};
            float* src[6] = {raw.ox, raw.oy, raw.oz, raw.vx, raw.vy, raw.vz};
            for (int t = 0; t < 6; ++t) FOPIS_CUDA(cudaMemcpy(dst[t] + total, src[t], 4 * w, cudaMemcpyDeviceToHost));
        }
        total += k;
    }
    free_soa(raw, c.st);
    cudaFree(dc);
    return total;
}

static double max_extent(const Ctx& c, int axis) {
    const int n = axis == 0 ? c.nx : (axis == 1 ? c.ny : c.nz);
    return c.per[2 * axis + 1] ? (double)n : n - 1.0;
}

template <typename T>
static void generate_ambient(Ctx& c) {
    const Grid g = make_grid(c);
    for (int s = 0; s < c.nsp; ++s) {
        const fopis_species& sp = c.p.species[s];
        if (sp.kind != FOPIS_SPECIES_AMBIENT) continue;
        // ParticleType::getTotalNumber (ParticleType.cpp:39-47)
        const int64_t cxn = c.per[1] ? c.nx : c.nx - 1, cyn = c.per[3] ? c.ny : c.ny - 1, czn = c.per[5] ? c.nz : c.nz - 1;
        const int64_t total = cxn * cyn * czn * (int64_t)sp.particle_per_cell;
        sync_scalars(c);
        particles_alloc(c, s, (int64_t)((c.nslots[s] + total) * std::max(1.0, c.p.capacity_factor)) + 4096);
        AmbientArgs<T> a;
        a.p = parts<T>(c)[s]; a.cap = c.cap[s]; a.s = s; a.total = total;
        for (int q = 0; q < 3; ++q) { a.maxe[q] = max_extent(c, q); a.drift[q] = sp.drift[q]; }
        a.dev = sp.deviation; a.seed = c.p.seed; a.g = g;
        a.cellmap = c.objs.empty() ? nullptr : c.cellmap;
        a.sc = c.d_sc;
        ++c.launches;
        ambient_kernel<<<grid_for(total), kThreads, 0, c.st>>>(a);
        FOPIS_LAUNCH_CHECK();
    }
    sync_scalars(c);
}

void particles_generate_ambient(Ctx& c) {
    if (c.fp64) generate_ambient<double>(c);
    else generate_ambient<float>(c);
}

int64_t brick_keys(const Ctx& c) {
    const Grid g = make_grid(c);
    return (int64_t)g.nb[0] * g.nb[1] * g.nb[2] * kBrickCells;
}

int brick_count(const Ctx& c) {
    const Grid g = make_grid(c);
    return g.nb[0] * g.nb[1] * g.nb[2];
}

// Sort of every species by brick (brick_index), then by cell inside the
// brick (local_cell); invalid slots are dropped. Records each brick's first slot
// for push_brick_kernel. The particles end in the live arrays; the sort
// targets hold the brick-grouped intermediate.
template <typename T>
static void sort_all(Ctx& c) {
    sync_scalars(c);
    const Grid g = make_grid(c);
    const int nbricks = brick_count(c);
    const int tiles = (int)((nbricks + 1 + kScanTile - 1) / kScanTile);
    for (int s = 0; s < c.nsp; ++s) {
        if (c.cap[s] == 0) continue;
        if (!c.brick_start[s]) FOPIS_CUDA(cudaMalloc(&c.brick_start[s], sizeof(int32_t) * (nbricks + 1)));
        FOPIS_CUDA(cudaMemsetAsync(c.sort_count, 0, sizeof(int32_t) * (nbricks + 1), c.st));
        ++c.launches;
        sort_count_kernel<<<grid_for(std::max<int64_t>(c.nslots[s], 1)), kThreads, 0, c.st>>>(
            parts<T>(c)[s], c.cap[s], &c.d_sc->count[s], g, c.sort_count);
        FOPIS_LAUNCH_CHECK();
        ++c.launches;
        scan_tiles_kernel<<<tiles, kScanThreads, 0, c.st>>>(c.sort_count, nbricks + 1, c.scan_partials);
        ++c.launches;
        scan_partials_kernel<<<1, kScanThreads, 0, c.st>>>(c.scan_partials, tiles);
        ++c.launches;
        scan_apply_kernel<<<tiles, kScanThreads, 0, c.st>>>(c.sort_count, nbricks + 1, c.scan_partials,
                                                            c.brick_start[s]);
        FOPIS_LAUNCH_CHECK();
        FOPIS_CUDA(cudaMemcpyAsync(c.sort_offset, c.brick_start[s], sizeof(int32_t) * (nbricks + 1),
                                   cudaMemcpyDeviceToDevice, c.st));
        ++c.launches;
        {
            const long long chunks = (std::max<int64_t>(c.nslots[s], 1) + kSortChunk - 1) / kSortChunk;
            const int grid = (int)std::max<long long>(1, std::min<long long>(chunks, 148LL * 8));
            sort_brick_scatter_kernel<<<grid, kSortThreads, 0, c.st>>>(parts<T>(c)[s], parts2<T>(c)[s], c.cap[s],
                                                                      &c.d_sc->count[s], g, c.sort_offset);
        }
        FOPIS_LAUNCH_CHECK();
        ++c.launches;
        sort_cell_kernel<<<std::min(nbricks, 148 * 8), kCellThreads, 0, c.st>>>(parts2<T>(c)[s], parts<T>(c)[s],
                                                                                c.brick_start[s], nbricks);
        FOPIS_LAUNCH_CHECK();
        // the new count is the total of valid particles: the scan's grand total
        FOPIS_CUDA(cudaMemcpyAsync(&c.d_sc->count[s], c.scan_partials + tiles, sizeof(int32_t), cudaMemcpyDeviceToDevice, c.st));
        FOPIS_CUDA(cudaMemsetAsync(((char*)&c.d_sc->count[s]) + 4, 0, 4, c.st));
    }
    sync_scalars(c);
    for (int s = 0; s < c.nsp; ++s) {
        if (c.cap[s] == 0) continue;
        const int64_t n = c.nslots[s];
        c.sorted_n[s] = n;
        c.valid[s] = n;             // the sort keeps exactly the valid particles
        if (n < c.cap[s]) FOPIS_CUDA(cudaMemsetAsync(parts<T>(c)[s].cell + n, 0xff, sizeof(int32_t) * (c.cap[s] - n), c.st));
        // keep head room for the appends of the coming steps
        const int64_t want = (int64_t)(n * 1.25) + 65536;
        if (want > c.cap[s]) particles_alloc(c, s, (int64_t)(n * std::max(1.5, c.p.capacity_factor)) + 65536);
    }
}

void particles_sort(Ctx& c) {
    if (c.fp64) sort_all<double>(c);
    else sort_all<float>(c);
}

template <typename T> const typename NodeE<T>::type* node_e(const Ctx& c);
template <> const float4* node_e<float>(const Ctx& c) { return c.E; }
template <> const Vec4d* node_e<double>(const Ctx& c) { return c.E64; }
template <typename T> const typename NodeE<T>::type* node_b(const Ctx& c);
template <> const float4* node_b<float>(const Ctx& c) { return c.em.B; }
template <> const Vec4d* node_b<double>(const Ctx& c) { return c.em.B64; }

template <typename T>
static PushArgsT<T> push_args(Ctx& c, int s) {
    PushArgsT<T> a;
    a.p = parts<T>(c)[s]; a.s = s; a.cap = c.cap[s]; a.lo = 0; a.count = &c.d_sc->count[s];
    a.E = node_e<T>(c); a.g = make_grid(c);
    a.qm = (T)(0.5 * c.p.species[s].charge / c.p.species[s].mass);
    a.bx = (T)c.p.static_bfield[0]; a.by = (T)c.p.static_bfield[1]; a.bz = (T)c.p.static_bfield[2];
    const double b2 = c.p.static_bfield[0] * c.p.static_bfield[0] + c.p.static_bfield[1] * c.p.static_bfield[1] +
                      c.p.static_bfield[2] * c.p.static_bfield[2];
    a.boris = (T)(2.0 / (1.0 + b2));
    a.bzero = b2 == 0.0 ? 1 : 0;
    a.cellmap = c.objs.empty() ? nullptr : c.cellmap;
    a.rho = c.rho_i64 + (size_t)s * c.N;
    a.ab = c.ab; a.sc = c.d_sc;
    return a;
}

template <typename T>
static void push_generic(Ctx& c, const PushArgsT<T>& a, int grid, bool vel, bool pos, bool dep) {
    if (vel && pos && dep) push_kernel<T, true, true, true><<<grid, kThreads, 0, c.st>>>(a);
    else if (vel && !pos && !dep) push_kernel<T, true, false, false><<<grid, kThreads, 0, c.st>>>(a);
    else if (!vel && pos && !dep) push_kernel<T, false, true, false><<<grid, kThreads, 0, c.st>>>(a);
    else if (!vel && !pos && dep) push_kernel<T, false, false, true><<<grid, kThreads, 0, c.st>>>(a);
    else throw ApiError{FOPIS_ERR_ARG, "unsupported push combination"};
}

// The fused step takes the brick-sorted slots with push_brick_kernel and the
// appended tail with push_kernel (mixed mode); the FP64 mode and the single
// phases run push_kernel over every slot.
void launch_push(Ctx& c, bool vel, bool pos, bool dep) {
    for (int s = 0; s < c.nsp; ++s) {
        if (c.cap[s] == 0) continue;
        const int grid = grid_for(c.cap[s]);
        if (c.fp64) {
            ++c.launches;
            push_generic<double>(c, push_args<double>(c, s), grid, vel, pos, dep);
        } else if (vel && pos && dep && c.sorted_n[s] > 0 && c.brick_start[s]) {
            PushArgs a = push_args<float>(c, s);
            ++c.launches;
            push_brick_kernel<4, false><<<brick_count(c), kBrickThreads, 0, c.st>>>(a, c.brick_start[s], EdgeFix{});
            a.lo = c.sorted_n[s];
            ++c.launches;
            push_kernel<float, true, true, true><<<grid_for(std::max<int64_t>(c.cap[s] - a.lo, 1)), kThreads, 0, c.st>>>(a);
        } else {
            ++c.launches;
            push_generic<float>(c, push_args<float>(c, s), grid, vel, pos, dep);
        }
        FOPIS_LAUNCH_CHECK();
    }
}

void launch_deposit_all(Ctx& c) { launch_push(c, false, false, true); }

// Grid::updateParticleVelocityEM for every species.
void launch_em_velocity(Ctx& c) {
    for (int s = 0; s < c.nsp; ++s) {
        if (c.cap[s] == 0) continue;
        ++c.launches;
        if (c.fp64) em_velocity_kernel<double><<<grid_for(c.cap[s]), kThreads, 0, c.st>>>(push_args<double>(c, s), node_b<double>(c));
        else em_velocity_kernel<float><<<grid_for(c.cap[s]), kThreads, 0, c.st>>>(push_args<float>(c, s), node_b<float>(c));
        FOPIS_LAUNCH_CHECK();
    }
}

// The mixed mode's EM particle pass: per species the brick-sorted slots with
// push_brick_kernel<.., true> and the appended tail with em_tail_kernel (move,
// fixed-point current halves, body test, rho deposit), then J in FP64 and its
// periodic folds. With kick the same pass gives the velocity update first
// (the caller's choice when no particle is emitted between the two updates).
// The caller zeroes rho and the fixed-point sums.
void launch_em_move(Ctx& c, bool kick) {
    const long long nxe = (long long)(c.cx - 1) * c.cy * c.cz, nye = (long long)c.cx * (c.cy - 1) * c.cz;
    const long long per = nxe + nye + (long long)c.cx * c.cy * (c.cz - 1);
    FixScales sc{};
    for (int s = 0; s < c.nsp; ++s) {
        sc.v[s] = c.p.species[s].charge * c.p.species[s].size / (double)kCurrentScale;
        if (c.cap[s] == 0) continue;
        unsigned long long* base = c.em.jfix + (size_t)s * per;
        const EdgeFix J{base, base + nxe, base + nxe + nye, c.cx, c.cy, c.cz, kick ? c.em.B : nullptr};
        PushArgs a = push_args<float>(c, s);
        if (c.sorted_n[s] > 0 && c.brick_start[s]) {
            ++c.launches;
            push_brick_kernel<3, true><<<brick_count(c), kBrickThreads, 0, c.st>>>(a, c.brick_start[s], J);
            a.lo = c.sorted_n[s];
        }
        ++c.launches;
        em_tail_kernel<<<grid_for(std::max<int64_t>(c.cap[s] - a.lo, 1)), kThreads, 0, c.st>>>(a, J);
        FOPIS_LAUNCH_CHECK();
    }
    ++c.launches;
    em_j_convert_kernel<<<grid_for(per), kThreads, 0, c.st>>>(c.em.jfix, per, c.nsp, sc, c.em.j[0], nxe, c.em.j[1], nye,
                                                              c.em.j[2]);
    FOPIS_LAUNCH_CHECK();
    em_fold_currents(c);
}

// RootGrid::updateParticlePositionEM: J = 0 (Field::initializeCurrent), the
// moves with their edge currents, then the periodic folds of the currents.
void launch_em_position(Ctx& c) {
    const size_t nx = (size_t)(c.cx - 1) * c.cy * c.cz, ny = (size_t)c.cx * (c.cy - 1) * c.cz,
                 nz = (size_t)c.cx * c.cy * (c.cz - 1);
    FOPIS_CUDA(cudaMemsetAsync(c.em.j[0], 0, sizeof(double) * nx, c.st));
    FOPIS_CUDA(cudaMemsetAsync(c.em.j[1], 0, sizeof(double) * ny, c.st));
    FOPIS_CUDA(cudaMemsetAsync(c.em.j[2], 0, sizeof(double) * nz, c.st));
    const EdgeJ J{c.em.j[0], c.em.j[1], c.em.j[2], c.cx, c.cy, c.cz};
    for (int s = 0; s < c.nsp; ++s) {
        if (c.cap[s] == 0) continue;
        const double q = c.p.species[s].charge * c.p.species[s].size;   // getChargeOfSuperParticle() / dt
        ++c.launches;
        if (c.fp64) em_position_kernel<double><<<grid_for(c.cap[s]), kThreads, 0, c.st>>>(push_args<double>(c, s), J, q);
        else em_position_kernel<float><<<grid_for(c.cap[s]), kThreads, 0, c.st>>>(push_args<float>(c, s), J, q);
        FOPIS_LAUNCH_CHECK();
    }
    em_fold_currents(c);
}

template <typename T>
static SourceArgsT<T> source_args(Ctx& c, bool fused) {
    SourceArgsT<T> a;
    for (int s = 0; s < FOPIS_MAX_SPECIES; ++s) { a.p[s] = parts<T>(c)[s]; a.cap[s] = c.cap[s]; }
    a.g = make_grid(c);
    a.cellmap = c.objs.empty() ? nullptr : c.cellmap;
    a.rho = c.rho_i64; a.N = (long long)c.N; a.ab = c.ab; a.sc = c.d_sc; a.seed = c.p.seed;
    a.fused = fused ? 1 : 0;
    return a;
}

void launch_emit(Ctx& c, bool fused) {
    int eaxis = -1;
    for (int q = 0; q < 3; ++q) if (std::fabs(c.p.shine_vector[q]) == 1.0) { eaxis = q; break; }
    for (size_t o = 0; o < c.objs.size(); ++o) {
        ObjectDev& ob = c.objs[o];
        const int s = ob.emit_species;
        if (s < 0 || c.p.species[s].kind != FOPIS_SPECIES_PHOTOELECTRON || ob.n_lit == 0) continue;
        if (eaxis < 0) throw ApiError{FOPIS_ERR_ARG, "shine_vector must be [+-1,0,0], [0,+-1,0] or [0,0,+-1]"};
        const int K = (int)std::ceil(c.p.species[s].emission_amount);
        if (K <= 0) continue;
        const int64_t add = (int64_t)ob.n_lit * K;
        sync_scalars(c);
        if (c.nslots[s] + add > c.cap[s])
            particles_alloc(c, s, std::max<int64_t>((int64_t)((c.nslots[s] + add) * 1.5), add * 2048) + 65536);
        EmitArgs e;
        e.obj = (int)o; e.s = s; e.K = K; e.eaxis = eaxis;
        for (int q = 0; q < 3; ++q) e.ev[q] = -c.p.shine_vector[q];
        e.vth = c.p.species[s].thermal_velocity;
        e.n_lit = ob.n_lit; e.lit = ob.lit; e.lit_ijk = ob.lit + ob.n_lit;
        e.node_cmat = c.node_cmat; e.charge_tmp = ob.charge_tmp; e.n_cmat = ob.n; e.step = c.timestep;
        ++c.launches;
        if (c.fp64) emit_kernel<<<grid_for(add), kThreads, 0, c.st>>>(source_args<double>(c, fused), e);
        else emit_kernel<<<grid_for(add), kThreads, 0, c.st>>>(source_args<float>(c, fused), e);
        FOPIS_LAUNCH_CHECK();
    }
    launch_secondary(c, fused);
}

static int node_size(const Ctx& c, int axis) {
    const int n = axis == 0 ? c.nx : (axis == 1 ? c.ny : c.nz);
    return c.per[2 * axis + 1] ? n + 1 : n;
}

void launch_inject(Ctx& c, bool fused) {
    InjectTable tb{};
    tb.n = 0;
    tb.start[0] = 0;
    for (int q = 0; q < 3; ++q) tb.maxe[q] = max_extent(c, q);
    tb.step = c.timestep;
    int64_t need[FOPIS_MAX_SPECIES] = {0};
    for (int s = 0; s < c.nsp; ++s) {
        const fopis_species& sp = c.p.species[s];
        if (sp.kind != FOPIS_SPECIES_AMBIENT) continue;
        for (int face = 0; face < 6; ++face) {
            const int axis = face / 2, side = face % 2;
            if (c.per[2 * axis + side]) continue;
            const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
            const double area = (double)(node_size(c, a2) - 1) * (node_size(c, a1) - 1);
            const double flux = sp.injection_axis[face] ? sp.flux[face] : 0.0;
            const double nd = 1.0 * area * flux;
            const int num = (int)std::floor(nd + c.inject_residual[s][face]);
            c.inject_residual[s][face] += nd - num;
            if (num <= 0) continue;
            tb.species[tb.n] = s; tb.face[tb.n] = face;
            tb.vth[tb.n] = sp.thermal_velocity; tb.dev[tb.n] = sp.deviation;
            for (int q = 0; q < 3; ++q) tb.drift[tb.n][q] = sp.drift[q];
            tb.start[tb.n + 1] = tb.start[tb.n] + num;
            need[s] += num;
            ++tb.n;
        }
    }
    c.injected_step = tb.n ? tb.start[tb.n] : 0;
    if (tb.n == 0) return;
    bool grow = false;
    for (int s = 0; s < c.nsp; ++s) if (need[s] && c.nslots[s] + need[s] > c.cap[s]) grow = true;
    if (grow) {
        sync_scalars(c);
        for (int s = 0; s < c.nsp; ++s)
            if (need[s] && c.nslots[s] + need[s] > c.cap[s]) particles_alloc(c, s, (int64_t)((c.nslots[s] + need[s]) * 1.5) + 65536);
    }
    ++c.launches;
    if (c.fp64) inject_kernel<<<grid_for(tb.start[tb.n]), kThreads, 0, c.st>>>(source_args<double>(c, fused), tb);
    else inject_kernel<<<grid_for(tb.start[tb.n]), kThreads, 0, c.st>>>(source_args<float>(c, fused), tb);
    FOPIS_LAUNCH_CHECK();
}

static AbsorbArgs absorb_args(const Ctx& c) {
    AbsorbArgs a;
    a.ab = c.ab; a.g = make_grid(c); a.cellmap = c.cellmap; a.node_cmat = c.node_cmat; a.sc = c.d_sc;
    a.inc = c.inc;
    for (int o = 0; o < FOPIS_MAX_OBJECTS; ++o) { a.charge_tmp[o] = nullptr; a.n_cmat[o] = 0; a.secondary[o] = 0; }
    for (size_t o = 0; o < c.objs.size(); ++o) {
        a.charge_tmp[o] = c.objs[o].charge_tmp;
        a.n_cmat[o] = c.objs[o].n;
        a.secondary[o] = c.objs[o].secondary_species >= 0 && c.inc.cap > 0 ? 1 : 0;
    }
    return a;
}

void launch_absorb(Ctx& c) {
    if (c.objs.empty()) return;
    ++c.launches;
    absorb_kernel<<<148 * 4, kThreads, 0, c.st>>>(absorb_args(c));
    FOPIS_LAUNCH_CHECK();
}

// The secondaries of the incidents the last absorption recorded, then the
// list is cleared (Spacecraft::clearIncidentEvents, SecondaryEmission.cpp:31-33).
void launch_secondary(Ctx& c, bool fused) {
    if (c.inc.cap == 0) return;
    sync_scalars(c);
    const long long n = (long long)std::min<unsigned long long>(c.h_sc->incident_n, (unsigned long long)c.inc.cap);
    if (n > 0) {
        SecondaryArgs e;
        e.inc = c.inc; e.n = n; e.energy_ev = c.p.energy_ev; e.seed = c.p.seed; e.step = c.timestep;
        for (int o = 0; o < FOPIS_MAX_OBJECTS; ++o) e.sec[o] = -1;
        for (size_t o = 0; o < c.objs.size(); ++o) e.sec[o] = c.objs[o].secondary_species;
        for (int s = 0; s < FOPIS_MAX_SPECIES; ++s) {
            e.mass[s] = s < c.nsp ? c.p.species[s].mass : 1.0;
            e.charge[s] = s < c.nsp ? c.p.species[s].charge * c.p.species[s].size : 0.0;
            e.vth[s] = s < c.nsp ? c.p.species[s].thermal_velocity : 0.0;
        }
        FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->secondary_n, 0, sizeof(unsigned long long), c.st));
        ++c.launches;
        see_count_kernel<<<grid_for(n), kThreads, 0, c.st>>>(e, c.d_sc);
        FOPIS_LAUNCH_CHECK();
        sync_scalars(c);
        const int64_t add = (int64_t)c.h_sc->secondary_n;
        for (size_t o = 0; o < c.objs.size(); ++o) {
            const int s = c.objs[o].secondary_species;
            if (s >= 0 && c.nslots[s] + add > c.cap[s])
                particles_alloc(c, s, (int64_t)((c.nslots[s] + add) * 1.5) + 65536);
        }
        ++c.launches;
        if (c.fp64) see_emit_kernel<<<grid_for(n), kThreads, 0, c.st>>>(source_args<double>(c, fused), e, absorb_args(c));
        else see_emit_kernel<<<grid_for(n), kThreads, 0, c.st>>>(source_args<float>(c, fused), e, absorb_args(c));
        FOPIS_LAUNCH_CHECK();
    }
    FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->incident_n, 0, sizeof(unsigned long long), c.st));
}

void launch_energy(Ctx& c) {
    FOPIS_CUDA(cudaMemsetAsync(c.d_sc->energy, 0, sizeof(double) * FOPIS_MAX_SPECIES, c.st));
    for (int s = 0; s < c.nsp; ++s) {
        if (c.cap[s] == 0) continue;
        ++c.launches;
        if (c.fp64)
            energy_kernel<<<grid_for(c.cap[s]), kThreads, 0, c.st>>>(c.dp[s], c.cap[s], &c.d_sc->count[s],
                                                                      &c.d_sc->energy[s]);
        else
            energy_kernel<<<grid_for(c.cap[s]), kThreads, 0, c.st>>>(c.sp[s], c.cap[s], &c.d_sc->count[s],
                                                                      &c.d_sc->energy[s]);
        FOPIS_LAUNCH_CHECK();
    }
}

}  // namespace fopis
