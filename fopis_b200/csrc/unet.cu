// unet.cu — learned initial guess for the first Poisson solve of a step.
//
// A 3-level 3D U-Net (16/32/64 channels, 3x3x3 convolutions, BF16 weights and
// activations, FP32 accumulation) maps features of (rho^n, phi^{n-1},
// phi^{n-2}) on the multigrid unknowns to the increment phi^n - phi^{n-1},
// where phi^k is the first-solve potential of step k. It is trained online,
// one Adam step per solve, on the pairs the multigrid solver itself produces;
// its prediction only seeds the solve, which still iterates to the same
// residual tolerance. A guess that does not lower the initial residual is
// dropped for that solve, and a policy compares the V-cycles of learned and
// history starts and falls back to the history start when the network does
// not save cycles.
//
// Layout. Each level is the multigrid level grid (n0 x n1 x n2 unknowns) with
// one zero halo layer: m = n + 2 per axis, positions p = (i*m1 + j)*m2 + k.
// A tensor of C channels is C/8 planes; a plane holds 8 BF16 channels (16 B)
// per position, with zero slack before and after so that every shifted read
// of a tile stays inside the allocation. Halo and slack are zero and stay zero.
//
// Convolution (forward and input gradient): implicit GEMM on tcgen05. A CTA
// computes 128 consecutive positions (M = 128) x COUT channels (N) in TMEM.
// The 27 taps are grouped by (di, dj) into 9 stages; a stage stages the 130
// positions of each input plane that the three dk taps read, plus the three
// taps' weights, with cp.async into shared memory. The A operand of tap dk is
// the staged segment started dk rows later (K-major, rows 16 B apart), so no
// im2col copy is made. Weight gradient: tcgen05 with both operands MN-major,
// positions as K: A rows are (tap, input channel) built by 16-byte shifted
// copies, B is the output gradient; partial sums leave TMEM through FP32
// atomics.
#include "internal.cuh"
#include "tc.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>

namespace fopis {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kLevels = 3;
constexpr int kLayers = 6;
constexpr int kHead = 16;       // channels entering the 1x1 output head

// ------------------------------------------------------------------ grids
struct NGrid {
    int n[3] = {0, 0, 0};
    int per[3] = {0, 0, 0};
    long long Sj = 0, Si = 0, P = 0;
    long long front = 0, stride = 0;
    int tiles = 0;
};

NGrid make_grid(const MGLevel& l) {
    NGrid g;
    for (int a = 0; a < 3; ++a) { g.n[a] = l.n[a]; g.per[a] = l.per[a]; }
    g.Sj = g.n[2] + 2;
    g.Si = (long long)(g.n[1] + 2) * g.Sj;
    g.P = (long long)(g.n[0] + 2) * g.Si;
    g.tiles = (int)((g.P + 127) / 128);
    g.front = ((g.Si + g.Sj + 16 + 7) / 8) * 8;
    const long long back = ((128 + g.Si + g.Sj + 16 + 7) / 8) * 8;
    g.stride = g.front + g.P + back;
    return g;
}

// Device view of a tensor: plane pl, position pos lives at p + 8 * (pl*stride + pos).
struct TV {
    bf16* p = nullptr;
    long long stride = 0;
};
__device__ __forceinline__ uint4* vat(TV t, int pl, long long pos) {
    return reinterpret_cast<uint4*>(t.p + ((long long)pl * t.stride + pos) * 8);
}

struct Tensor {
    bf16* base = nullptr;
    int C = 0;
    int level = 0;
    const NGrid* g = nullptr;
    TV view() const { return TV{base + g->front * 8, g->stride}; }
    size_t bytes() const { return (size_t)(C / 8) * g->stride * 16; }
};

struct GV {  // grid view for the elementwise kernels
    int n0, n1, n2, p0, p1, p2;
    long long Sj, Si;
};
GV gv(const NGrid& g) { return GV{g.n[0], g.n[1], g.n[2], g.per[0], g.per[1], g.per[2], g.Sj, g.Si}; }
__device__ __forceinline__ long long pos_of(const GV& g, int a, int b, int c) {
    return (long long)(a + 1) * g.Si + (long long)(b + 1) * g.Sj + (c + 1);
}

__device__ __forceinline__ void report(unsigned int* err, unsigned int code) {
    if (err) atomicOr(err, code);
}

// The bounded mbarrier wait of the tensor-core kernels, run on its own: one
// thread initialises an mbarrier that expects one arrival and, when `arrive`
// is 0, waits for a phase that nothing completes. With nothing asynchronous
// in flight the wait can only run out: it gives up after `polls` polls and
// reports code 1 through the same path the convolution kernels use.
__global__ void bounded_wait_check_kernel(uint32_t polls, int arrive, unsigned int* err) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    const uint32_t b = tc::saddr(&bar);
    tc::mbar_init(b, 1);
    tc::fence_mbar_init();
    if (arrive) tc::mbar_arrive(b);
    if (!tc::mbar_wait(b, 0u, polls)) report(err, 1u);
}

__device__ __forceinline__ void unpack8(uint4 u, float* f) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
    uint4 u;
    __nv_bfloat162* h = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    return u;
}

// ------------------------------------------------------------------ convolution
enum { EPI_FWD = 0, EPI_HEAD = 1, EPI_BWD = 2 };

struct ConvArgs {
    TV x, y;
    const bf16* w;        // B image: [27][CIN/16][2][COUT][8]
    const float* bias;    // forward bias [COUT]
    TV mask;              // backward: keep where mask > 0 (mask.p may be null)
    TV skip;              // head: skip tensor added before the 1x1 head
    const float* head;    // head: w[16], b
    float* out;           // head: prediction per position
    long long Sj, Si, P;
    int n0, n1, n2;
    int tiles;
    unsigned int* err;
};

__device__ __forceinline__ bool interior(long long p, long long Si, long long Sj, int n0, int n1, int n2) {
    const int i = (int)(p / Si);
    const long long r = p - (long long)i * Si;
    const int j = (int)(r / Sj);
    const int k = (int)(r - (long long)j * Sj);
    return i >= 1 && i <= n0 && j >= 1 && j <= n1 && k >= 1 && k <= n2;
}

template <int COUT, int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, uint32_t tmem, long long p0, int warp, int lane) {
    uint32_t r[COUT];
    const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c = 0; c < COUT; c += 16) tc::tmem_ld16(ta + c, r + c);
    tc::tmem_wait<COUT>(r);
    const long long p = p0 + warp * 32 + lane;
    if (p >= a.P) return;
    const bool in = interior(p, a.Si, a.Sj, a.n0, a.n1, a.n2);
    float v[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) v[c] = __uint_as_float(r[c]);
    if (EPI == EPI_BWD) {
#pragma unroll
        for (int pl = 0; pl < COUT / 8; ++pl) {
            float m[8] = {1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f};
            if (in && a.mask.p) unpack8(*vat(a.mask, pl, p), m);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int c = pl * 8 + e;
                v[c] = (in && m[e] > 0.0f) ? v[c] : 0.0f;
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < COUT; ++c) v[c] = in ? fmaxf(v[c] + a.bias[c], 0.0f) : 0.0f;
    }
#pragma unroll
    for (int pl = 0; pl < COUT / 8; ++pl) {
        const uint4 u = pack8(v + pl * 8);
        *vat(a.y, pl, p) = u;
        if (EPI == EPI_HEAD) unpack8(u, v + pl * 8);   // the head sees the stored (rounded) activation
    }
    if (EPI == EPI_HEAD) {
        float o = 0.0f;
        if (in) {
            o = a.head[kHead];
#pragma unroll
            for (int pl = 0; pl < COUT / 8; ++pl) {
                float s[8];
                unpack8(*vat(a.skip, pl, p), s);
#pragma unroll
                for (int e = 0; e < 8; ++e) o += a.head[pl * 8 + e] * (v[pl * 8 + e] + s[e]);
            }
        }
        a.out[p] = o;
    }
}

template <int CIN, int COUT>
struct ConvShape {
    static constexpr int KB = CIN / 16;
    static constexpr int A_PL = 130 * 16;
    static constexpr int A_BYTES = (CIN / 8) * A_PL;
    static constexpr int W_TAP = CIN * COUT * 2;
    static constexpr int B_BYTES = 3 * W_TAP;
    static constexpr int ST = A_BYTES + B_BYTES;
    // stages in the ring (about 48 KB of it, 2 to 8), and the copies kept in flight ahead of the MMAs
    static constexpr int NST = ST * 8 <= 49152 ? 8 : (ST * 2 >= 49152 ? 2 : 49152 / ST);
    static constexpr int LA = NST > 2 ? NST - 2 : 1;   // one stage of slack for the MMAs to release a buffer
    static constexpr int COLS = COUT < 32 ? 32 : COUT;
    static constexpr int SMEM = NST * ST + (2 * NST + 1) * 8 + 16;
    static constexpr uint32_t STAGE_TX = (CIN / 8) * A_PL + B_BYTES;   // bytes one stage's bulk copies bring
};

// One implicit-GEMM convolution tile loop. Thread 0 produces and issues: for
// stage q it waits until the MMAs of stage q - NST have released the buffer,
// then brings the CIN/8 contiguous 2,080-byte plane segments of the shifted
// positions and the three taps' weight block in with bulk copies (TMA engine,
// completion counted on the stage's full barrier); for stage q - LA it waits on
// that full barrier and issues the tcgen05 MMAs into the TMEM accumulator. The
// four warps run the epilogue once a tile's nine stages are committed.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(128) conv_kernel(ConvArgs a) {
    using S = ConvShape<CIN, COUT>;
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 64, "channel counts");
    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, false, false);
    extern __shared__ __align__(128) uint8_t sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::NST * S::ST);   // [NST] MMAs done, [NST] tile done
    uint64_t* full = bar + S::NST + 1;                                   // [NST] stage data landed
    uint32_t* tslot = reinterpret_cast<uint32_t*>(full + S::NST);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(tc::saddr(tslot), S::COLS);
    if (tid == 0) {
        for (int b = 0; b <= S::NST; ++b) tc::mbar_init(tc::saddr(bar + b), 1);
        for (int b = 0; b < S::NST; ++b) tc::mbar_init(tc::saddr(full + b), 1);
        tc::fence_mbar_init();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t sbase = tc::saddr(sm);
    const int ntl = (int)blockIdx.x < a.tiles ? (a.tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int total = ntl * 9;
    for (int q = 0; q < total + S::LA; ++q) {
        const int cq = q - S::LA;
        if (tid == 0) {
            if (q < total) {
                const int b = q % S::NST;
                if (q >= S::NST && !tc::mbar_wait(tc::saddr(bar + b), (uint32_t)((q / S::NST) - 1) & 1u)) report(a.err, 1u);
                const int tl = q / 9, s = q - tl * 9;
                const long long p0 = ((long long)blockIdx.x + (long long)tl * gridDim.x) * 128;
                const int di = s / 3 - 1, dj = s % 3 - 1;
                const long long pb = p0 + di * a.Si + dj * a.Sj - 1;
                const uint32_t sA = sbase + b * S::ST, sB = sA + S::A_BYTES, fb = tc::saddr(full + b);
                tc::mbar_arrive_expect_tx(fb, S::STAGE_TX);
#pragma unroll
                for (int pl = 0; pl < CIN / 8; ++pl)
                    tc::bulk_g2s(sA + pl * S::A_PL, a.x.p + ((long long)pl * a.x.stride + pb) * 8, S::A_PL, fb);
                tc::bulk_g2s(sB, reinterpret_cast<const uint8_t*>(a.w) + (size_t)(s * 3) * S::W_TAP, S::B_BYTES, fb);
            }
            if (cq >= 0) {
                const int b = cq % S::NST, s = cq % 9;
                if (!tc::mbar_wait(tc::saddr(full + b), (uint32_t)(cq / S::NST) & 1u)) report(a.err, 4u);
                tc::fence_after();
                const uint32_t sA = sbase + b * S::ST, sB = sA + S::A_BYTES;
#pragma unroll
                for (int dk = 0; dk < 3; ++dk)
#pragma unroll
                    for (int kb = 0; kb < S::KB; ++kb) {
                        const uint64_t ad = tc::sdesc(sA + (2 * kb) * S::A_PL + dk * 16, S::A_PL, 128);
                        const uint64_t bd = tc::sdesc(sB + dk * S::W_TAP + kb * COUT * 32, COUT * 16, 128);
                        tc::mma(tmem, ad, bd, IDESC, (s | dk | kb) != 0 ? 1u : 0u);
                    }
                tc::commit(tc::saddr(bar + b));
                if (s == 8) tc::commit(tc::saddr(bar + S::NST));
            }
        }
        if (cq >= 0 && cq % 9 == 8) {
            const int tl = cq / 9;
            if (!tc::mbar_wait(tc::saddr(bar + S::NST), (uint32_t)tl & 1u)) report(a.err, 2u);
            tc::fence_after();
            conv_epilogue<COUT, EPI>(a, tmem, ((long long)blockIdx.x + (long long)tl * gridDim.x) * 128, warp, lane);
            tc::fence_before();
            __syncthreads();   // every warp's TMEM reads done before the next tile's MMAs overwrite it
            tc::fence_after();
        }
    }
    __syncthreads();   // every issued stage was consumed: no copy is in flight
    tc::fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, S::COLS);
}

// ------------------------------------------------------------------ weight gradient
struct WgArgs {
    TV x, g;
    float* dw;            // [27][COUT][CIN]
    float* db;            // [COUT]
    long long Sj, Si;
    long long chunks;     // KC-position chunks covering the tiles
    unsigned int* err;
};

__host__ __device__ constexpr int wg_taps_per_mtile(int cin) { return 128 / cin; }
__host__ __device__ constexpr int wg_mtiles(int cin) { return (27 + 128 / cin - 1) / (128 / cin); }
__host__ __device__ constexpr int wg_mt_per_cta(int cin, int cout) {
    return wg_mtiles(cin) < 4 ? (wg_mtiles(cin) < 128 / cout ? wg_mtiles(cin) : 128 / cout)
                              : (4 < 128 / cout ? 4 : 128 / cout);
}
__host__ __device__ constexpr int pow2_cols(int c) { return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : 256; }

template <int CIN, int COUT>
struct WgShape {
    static constexpr int KC = 32, NST = 3, LA = 1;
    static constexpr int PLI = CIN / 8;
    static constexpr int TPM = wg_taps_per_mtile(CIN);
    static constexpr int MTILES = wg_mtiles(CIN);
    static constexpr int MTC = wg_mt_per_cta(CIN, COUT);
    static constexpr int GRP = KC * 16;
    static constexpr int A_MT = 16 * GRP;
    static constexpr int A_BYTES = MTC * A_MT;
    static constexpr int B_BYTES = (COUT / 8) * GRP;
    static constexpr int ST = A_BYTES + B_BYTES;
    static constexpr int COLS = pow2_cols(MTC * COUT);
    static constexpr int SMEM = NST * ST + (NST + 1) * 8 + 16;
    static constexpr int YSPLIT = (MTILES + MTC - 1) / MTC;
};

__device__ __forceinline__ long long tap_offset(int t, long long Si, long long Sj) {
    return (long long)(t / 9 - 1) * Si + (long long)((t / 3) % 3 - 1) * Sj + (t % 3 - 1);
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(128) wgrad_kernel(WgArgs a) {
    using S = WgShape<CIN, COUT>;
    constexpr uint32_t IDESC = tc::idesc_bf16(128, COUT, true, true);
    extern __shared__ __align__(128) uint8_t sm[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::NST * S::ST);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + S::NST + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt0 = blockIdx.y * S::MTC;
    const int nmt = min(S::MTC, S::MTILES - mt0);
    // A groups of taps beyond 26 (last M-tile only) are never loaded: zero them once
    for (int bb = 0; bb < S::NST; ++bb)
        for (int mt = 0; mt < nmt; ++mt)
            for (int gq = 0; gq < 16; ++gq) {
                const int t = (mt0 + mt) * S::TPM + gq / S::PLI;
                if (t < 27) continue;
                uint4* d = reinterpret_cast<uint4*>(sm + bb * S::ST + mt * S::A_MT + gq * S::GRP);
                for (int e = tid; e < S::GRP / 16; e += 128) d[e] = make_uint4(0, 0, 0, 0);
            }
    if (warp == 0) tc::tmem_alloc(tc::saddr(tslot), S::COLS);
    if (tid == 0) {
        for (int b = 0; b <= S::NST; ++b) tc::mbar_init(tc::saddr(bar + b), 1);
        tc::fence_mbar_init();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t sbase = tc::saddr(sm);
    const long long nloc = (long long)blockIdx.x < a.chunks ? (a.chunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    float bsum = 0.0f;
    for (long long q = 0; q < nloc + S::LA; ++q) {
        if (q < nloc) {
            const int b = (int)(q % S::NST);
            if (q >= S::NST && !tc::mbar_wait(tc::saddr(bar + b), (uint32_t)((q / S::NST) - 1) & 1u)) report(a.err, 4u);
            const long long p0 = ((long long)blockIdx.x + q * gridDim.x) * S::KC;
            const uint32_t sA = sbase + b * S::ST, sB = sA + S::A_BYTES;
            for (int e = tid; e < nmt * 16 * S::KC; e += 128) {
                const int mt = e / (16 * S::KC), rem = e - mt * 16 * S::KC;
                const int gq = rem / S::KC, k = rem - gq * S::KC;
                const int t = (mt0 + mt) * S::TPM + gq / S::PLI, pl = gq % S::PLI;
                if (t >= 27) continue;
                const long long src = p0 + k + tap_offset(t, a.Si, a.Sj);
                tc::cp16(sA + mt * S::A_MT + gq * S::GRP + k * 16, a.x.p + ((long long)pl * a.x.stride + src) * 8);
            }
            for (int e = tid; e < (COUT / 8) * S::KC; e += 128) {
                const int pl = e / S::KC, k = e - pl * S::KC;
                tc::cp16(sB + pl * S::GRP + k * 16, a.g.p + ((long long)pl * a.g.stride + p0 + k) * 8);
            }
        }
        tc::cp_commit();
        const long long cq = q - S::LA;
        if (cq < 0) continue;
        tc::cp_wait<S::LA>();
        tc::fence_async_smem();
        __syncthreads();
        const int b = (int)(cq % S::NST);
        const uint32_t sA = sbase + b * S::ST, sB = sA + S::A_BYTES;
        if (tid == 0) {
            tc::fence_after();
            for (int mt = 0; mt < nmt; ++mt)
#pragma unroll
                for (int j = 0; j < S::KC / 16; ++j) {
                    const uint64_t ad = tc::sdesc(sA + mt * S::A_MT + j * 256, 128, S::GRP);
                    const uint64_t bd = tc::sdesc(sB + j * 256, 128, S::GRP);
                    tc::mma(tmem + mt * COUT, ad, bd, IDESC, (cq | j) != 0 ? 1u : 0u);
                }
            tc::commit(tc::saddr(bar + b));
        }
        if (blockIdx.y == 0 && tid < COUT) {
            const bf16* gb = reinterpret_cast<const bf16*>(sm + b * S::ST + S::A_BYTES + (tid / 8) * S::GRP) + (tid % 8);
#pragma unroll 8
            for (int k = 0; k < S::KC; ++k) bsum += __bfloat162float(gb[k * 8]);
        }
    }
    if (nloc > 0) {
        if (tid == 0) tc::commit(tc::saddr(bar + S::NST));
        if (!tc::mbar_wait(tc::saddr(bar + S::NST), 0u)) report(a.err, 8u);
        tc::fence_after();
        const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16);
        const int m = warp * 32 + lane;
        for (int mt = 0; mt < nmt; ++mt) {
            uint32_t r[COUT];
#pragma unroll
            for (int c = 0; c < COUT; c += 16) tc::tmem_ld16(ta + mt * COUT + c, r + c);
            tc::tmem_wait<COUT>(r);
            const int t = (mt0 + mt) * S::TPM + m / CIN, ci = m % CIN;
            if (t < 27) {
                float* dst = a.dw + (size_t)t * COUT * CIN + ci;
#pragma unroll
                for (int co = 0; co < COUT; ++co) atomicAdd(dst + (size_t)co * CIN, __uint_as_float(r[co]));
            }
        }
        if (blockIdx.y == 0 && tid < COUT) atomicAdd(a.db + tid, bsum);
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0) tc::tmem_dealloc(tmem, S::COLS);
}

// ------------------------------------------------------------------ features and targets
struct FeatArgs {
    int cy, cz;                 // glue dims (x extent not needed for indexing)
    int n0, n1, n2;             // unknowns
    int o0, o1, o2;             // glue index of unknown 0
    int p0, p1, p2;             // periodic axes
    int nref0, nref1, nref2;    // reference node counts
    double inv_eps0;
    int allper;
    GV g;
};
__device__ __forceinline__ long long glue(const FeatArgs& F, int i, int j, int k) {
    return ((long long)i * F.cy + j) * F.cz + k;
}
__device__ __forceinline__ int wrapg(int idx, int per, int nref) {
    if (per) { if (idx == 0) return nref; if (idx == nref + 1) return 1; }
    return idx;
}

// stats: [0] sum f, [1] sum f^2, [2] sum d^2, [3] sum phi1^2, [4] sum g, [5] sum g^2
// with g = f - A phi1; derived [6] sigma_f, [7] sigma_d, [8] sigma_phi, [9] mean f
// (all-periodic only), [10] sigma_r (r1 = g - mean f); [11] loss sum; [12] sum of
// the squared residual of the guess.
__device__ __forceinline__ double block_sum(double v, double* red) {
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// Rows of the level-0 unknowns with phi's six neighbours (periodic images wrapped).
struct RowPtrs {
    const double *p0, *im, *ip, *jm, *jp;
};
__device__ __forceinline__ RowPtrs row_ptrs(const FeatArgs& F, const double* phi, int a, int b) {
    const int i = a + F.o0, j = b + F.o1;
    return RowPtrs{phi + glue(F, i, j, 0), phi + glue(F, wrapg(i - 1, F.p0, F.nref0), j, 0),
                   phi + glue(F, wrapg(i + 1, F.p0, F.nref0), j, 0), phi + glue(F, i, wrapg(j - 1, F.p1, F.nref1), 0),
                   phi + glue(F, i, wrapg(j + 1, F.p1, F.nref1), 0)};
}
__device__ __forceinline__ double aphi(const FeatArgs& F, const RowPtrs& R, int k) {
    const double nb = R.im[k] + R.ip[k] + R.jm[k] + R.jp[k] + R.p0[wrapg(k - 1, F.p2, F.nref2)] +
                      R.p0[wrapg(k + 1, F.p2, F.nref2)];
    return 6.0 * R.p0[k] - nb;
}

__global__ void __launch_bounds__(256) feat_stats_kernel(FeatArgs F, const double* rho0, const double* phi1,
                                                         const double* phi2, double* stats) {
    __shared__ double red[32];
    double s[6] = {0, 0, 0, 0, 0, 0};
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        const RowPtrs R = row_ptrs(F, phi1, a, b);
        const long long base = glue(F, a + F.o0, b + F.o1, 0);
        for (int c = threadIdx.x; c < F.n2; c += blockDim.x) {
            const int k = c + F.o2;
            const double f = rho0[base + k] * F.inv_eps0, p1 = R.p0[k], d = p1 - phi2[base + k];
            const double g = f - aphi(F, R, k);
            s[0] += f; s[1] += f * f; s[2] += d * d; s[3] += p1 * p1; s[4] += g; s[5] += g * g;
        }
    }
    for (int q = 0; q < 6; ++q) {
        const double v = block_sum(s[q], red);
        if (threadIdx.x == 0) atomicAdd(stats + q, v);
    }
}

__global__ void feat_sigma_kernel(double* stats, double M, int allper) {
    const double fm = allper ? stats[0] / M : 0.0;
    const double sf = sqrt(fmax(stats[1] / M - fm * fm, 0.0));
    const double sd = sqrt(fmax(stats[2] / M, 0.0));
    const double sp = sqrt(fmax(stats[3] / M, 0.0));
    const double sr = sqrt(fmax((stats[5] - 2.0 * fm * stats[4]) / M + fm * fm, 0.0));
    stats[6] = sf > 0.0 ? sf : 1.0;
    stats[7] = sd;
    stats[8] = sp > 0.0 ? sp : 1.0;
    stats[9] = fm;
    stats[10] = sr > 0.0 ? sr : 1.0;
}

// Channels: r1 / sigma_r (residual of the history start), (f - mean) / sigma_f,
// (phi1 - phi2) / sigma_d, phi1 / sigma_phi; channels 4..15 stay zero.
__global__ void __launch_bounds__(256) feat_write_kernel(FeatArgs F, const double* rho0, const double* phi1,
                                                         const double* phi2, const double* stats, TV x0) {
    const double isf = 1.0 / stats[6], sd = stats[7], isd = sd > 0.0 ? 1.0 / sd : 0.0, isp = 1.0 / stats[8];
    const double fm = stats[9], isr = 1.0 / stats[10];
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        const RowPtrs R = row_ptrs(F, phi1, a, b);
        const long long base = glue(F, a + F.o0, b + F.o1, 0);
        for (int c = threadIdx.x; c < F.n2; c += blockDim.x) {
            const int k = c + F.o2;
            const double f = rho0[base + k] * F.inv_eps0 - fm;
            const double r1 = f - aphi(F, R, k);
            const double p1 = R.p0[k];
            float v[8] = {(float)(r1 * isr), (float)(f * isf), (float)((p1 - phi2[base + k]) * isd), (float)(p1 * isp),
                          0.f, 0.f, 0.f, 0.f};
            *vat(x0, 0, pos_of(F.g, a, b, c)) = pack8(v);
        }
    }
}

// phi += sigma_d * prediction on the unknowns.
__global__ void __launch_bounds__(256) apply_guess_kernel(FeatArgs F, const float* out, const double* stats,
                                                          double* phi) {
    const double sd = stats[7];
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        double* pr = phi + glue(F, a + F.o0, b + F.o1, F.o2);
        for (int c = threadIdx.x; c < F.n2; c += blockDim.x) pr[c] += sd * (double)out[pos_of(F.g, a, b, c)];
    }
}

// Squared residual of phi on the unknowns: sum (f - mean f - A phi)^2 -> stats[12].
__global__ void __launch_bounds__(256) guess_residual_kernel(FeatArgs F, const double* rho0, const double* phi,
                                                             double* stats) {
    __shared__ double red[32];
    const double fm = stats[9];
    double s2 = 0.0;
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        const RowPtrs R = row_ptrs(F, phi, a, b);
        const long long base = glue(F, a + F.o0, b + F.o1, 0);
        for (int c = threadIdx.x; c < F.n2; c += blockDim.x) {
            const int k = c + F.o2;
            const double r = rho0[base + k] * F.inv_eps0 - fm - aphi(F, R, k);
            s2 += r * r;
        }
    }
    const double v = block_sum(s2, red);
    if (threadIdx.x == 0) atomicAdd(stats + 12, v);
}

// Loss mean((out - t)^2) with t = (phi_new - phi1) / sigma_d, and the head's
// backward: gradients of the head weights, g5 = dL/dz5 (ReLU mask of a5) and
// ge0 = dL/de0 through the skip connection.
__global__ void __launch_bounds__(256) loss_kernel(FeatArgs F, const float* out, const double* phi_new,
                                                   const double* phi1, double* stats, TV a5, TV e0,
                                                   const float* head, float* dhead, TV g5, TV ge0, double inv_count) {
    __shared__ double red[32];
    const double sd = stats[7];
    const double isd = sd > 0.0 ? 1.0 / sd : 0.0;
    double loss = 0.0;
    float dh[kHead + 1];
#pragma unroll
    for (int c = 0; c <= kHead; ++c) dh[c] = 0.0f;
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        const long long gb = glue(F, a + F.o0, b + F.o1, F.o2);
        for (int c = threadIdx.x; c < F.n2; c += blockDim.x) {
            const long long p = pos_of(F.g, a, b, c);
            const double t = (phi_new[gb + c] - phi1[gb + c]) * isd;
            const double e = (double)out[p] - t;
            loss += e * e;
            const float dout = (float)(2.0 * e * inv_count);
            dh[kHead] += dout;
#pragma unroll
            for (int pl = 0; pl < kHead / 8; ++pl) {
                float av[8], ev[8], gv5[8], gve[8];
                unpack8(*vat(a5, pl, p), av);
                unpack8(*vat(e0, pl, p), ev);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int ch = pl * 8 + q;
                    dh[ch] += dout * (av[q] + ev[q]);
                    const float d = dout * head[ch];
                    gve[q] = d;
                    gv5[q] = av[q] > 0.0f ? d : 0.0f;
                }
                *vat(g5, pl, p) = pack8(gv5);
                *vat(ge0, pl, p) = pack8(gve);
            }
        }
    }
    const double l = block_sum(loss, red);
    if (threadIdx.x == 0) atomicAdd(stats + 11, l);
    for (int ch = 0; ch <= kHead; ++ch) {
        const double v = block_sum((double)dh[ch], red);
        if (threadIdx.x == 0) atomicAdd(dhead + ch, (float)v);
    }
}

// ------------------------------------------------------------------ resampling between levels
__device__ __forceinline__ int fine_of(int I, int per) { return per ? 2 * I : 2 * I + 1; }
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
// Fine indices that take coarse index I as a source, with their weights (adjoint of coarse_src).
__device__ __forceinline__ int fine_dst(int I, int per, int nf, int* f, float* w) {
    int k = 0;
    if (per) {
        f[k] = 2 * I; w[k++] = 1.0f;
        f[k] = 2 * I + 1; w[k++] = 0.5f;
        f[k] = 2 * I - 1 < 0 ? nf - 1 : 2 * I - 1; w[k++] = 0.5f;
        return k;
    }
    if (2 * I < nf) { f[k] = 2 * I; w[k++] = 0.5f; }
    if (2 * I + 1 < nf) { f[k] = 2 * I + 1; w[k++] = 1.0f; }
    if (2 * I + 2 < nf) { f[k] = 2 * I + 2; w[k++] = 0.5f; }
    return k;
}

// Injection at the coarse points: dst[I] = src[fine_of(I)].
__global__ void __launch_bounds__(128) down_kernel(GV F, GV Cg, TV src, TV dst, int planes) {
    const int rows = Cg.n0 * Cg.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int A = row / Cg.n1, B = row - A * Cg.n1;
        const int fa = fine_of(A, Cg.p0), fb = fine_of(B, Cg.p1);
        for (int e = threadIdx.x; e < Cg.n2 * planes; e += blockDim.x) {
            const int C = e / planes, pl = e - C * planes;
            *vat(dst, pl, pos_of(Cg, A, B, C)) = *vat(src, pl, pos_of(F, fa, fb, fine_of(C, Cg.p2)));
        }
    }
}

// Trilinear prolongation of (src + src2) to the fine level (the multigrid's).
__global__ void __launch_bounds__(128) up_kernel(GV Cg, GV F, TV src, TV src2, TV dst, int planes) {
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        int Ia[2], Ib[2];
        float wa[2], wb[2];
        const int na = coarse_src(a, F.p0, Cg.n0, Ia, wa), nb = coarse_src(b, F.p1, Cg.n1, Ib, wb);
        for (int e = threadIdx.x; e < F.n2 * planes; e += blockDim.x) {
            const int c = e / planes, pl = e - c * planes;
            int Ic[2];
            float wc[2];
            const int nc = coarse_src(c, F.p2, Cg.n2, Ic, wc);
            float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int x = 0; x < na; ++x)
                for (int y = 0; y < nb; ++y)
                    for (int z = 0; z < nc; ++z) {
                        const float w = wa[x] * wb[y] * wc[z];
                        const long long q = pos_of(Cg, Ia[x], Ib[y], Ic[z]);
                        float v[8];
                        unpack8(*vat(src, pl, q), v);
#pragma unroll
                        for (int t = 0; t < 8; ++t) acc[t] += w * v[t];
                        if (src2.p) {
                            unpack8(*vat(src2, pl, q), v);
#pragma unroll
                            for (int t = 0; t < 8; ++t) acc[t] += w * v[t];
                        }
                    }
            *vat(dst, pl, pos_of(F, a, b, c)) = pack8(acc);
        }
    }
}

// Adjoint of up_kernel: coarse gradient from the fine gradient.
__global__ void __launch_bounds__(128) up_adjoint_kernel(GV F, GV Cg, TV src, TV dst, int planes) {
    const int rows = Cg.n0 * Cg.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int A = row / Cg.n1, B = row - A * Cg.n1;
        int fa[3], fb[3];
        float wa[3], wb[3];
        const int na = fine_dst(A, F.p0, F.n0, fa, wa), nb = fine_dst(B, F.p1, F.n1, fb, wb);
        for (int e = threadIdx.x; e < Cg.n2 * planes; e += blockDim.x) {
            const int C = e / planes, pl = e - C * planes;
            int fc[3];
            float wc[3];
            const int nc = fine_dst(C, F.p2, F.n2, fc, wc);
            float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            for (int x = 0; x < na; ++x)
                for (int y = 0; y < nb; ++y)
                    for (int z = 0; z < nc; ++z) {
                        const float w = wa[x] * wb[y] * wc[z];
                        float v[8];
                        unpack8(*vat(src, pl, pos_of(F, fa[x], fb[y], fc[z])), v);
#pragma unroll
                        for (int t = 0; t < 8; ++t) acc[t] += w * v[t];
                    }
            *vat(dst, pl, pos_of(Cg, A, B, C)) = pack8(acc);
        }
    }
}

// out = (add + injection-adjoint of coarse) masked by act > 0, on the fine level.
__global__ void __launch_bounds__(128) gmask_kernel(GV F, GV Cg, TV add, TV coarse, TV act, TV out, int planes) {
    const int rows = F.n0 * F.n1;
    for (int row = blockIdx.x; row < rows; row += gridDim.x) {
        const int a = row / F.n1, b = row - a * F.n1;
        const bool ca = F.p0 ? (a % 2 == 0) : (a % 2 == 1 && (a - 1) / 2 < Cg.n0);
        const bool cb = F.p1 ? (b % 2 == 0) : (b % 2 == 1 && (b - 1) / 2 < Cg.n1);
        for (int e = threadIdx.x; e < F.n2 * planes; e += blockDim.x) {
            const int c = e / planes, pl = e - c * planes;
            const long long p = pos_of(F, a, b, c);
            float v[8] = {0, 0, 0, 0, 0, 0, 0, 0}, t[8], m[8];
            if (add.p) unpack8(*vat(add, pl, p), v);
            const bool cc = F.p2 ? (c % 2 == 0) : (c % 2 == 1 && (c - 1) / 2 < Cg.n2);
            if (coarse.p && ca && cb && cc) {
                const int A = F.p0 ? a / 2 : (a - 1) / 2, B = F.p1 ? b / 2 : (b - 1) / 2, C = F.p2 ? c / 2 : (c - 1) / 2;
                unpack8(*vat(coarse, pl, pos_of(Cg, A, B, C)), t);
#pragma unroll
                for (int q = 0; q < 8; ++q) v[q] += t[q];
            }
            unpack8(*vat(act, pl, p), m);
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = m[q] > 0.0f ? v[q] : 0.0f;
            *vat(out, pl, p) = pack8(v);
        }
    }
}

// ------------------------------------------------------------------ parameters and Adam
struct LayerDesc {
    long long w_off, b_off, img, imgT;   // imgT < 0: no input-gradient image
    int cin, cout;
};
struct LayerTable {
    LayerDesc l[kLayers];
    long long head_off;
};

// Adam step (beta 0.9 / 0.999, eps 1e-8) on the FP32 master parameters, then
// the BF16 operand images of the forward and input-gradient convolutions.
__global__ void __launch_bounds__(256) adam_kernel(LayerTable T, long long n, float* prm, const float* grad, float* m1,
                                                   float* m2, bf16* img, float lr, float bc1, float bc2, int do_step) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float w = prm[i];
        if (do_step) {
            const float g = grad[i];
            const float a = 0.9f * m1[i] + 0.1f * g;
            const float b = 0.999f * m2[i] + 0.001f * g * g;
            m1[i] = a;
            m2[i] = b;
            w -= lr * (a / bc1) / (sqrtf(b / bc2) + 1e-8f);
            prm[i] = w;
        }
        for (int l = 0; l < kLayers; ++l) {
            const LayerDesc& d = T.l[l];
            const long long nw = 27LL * d.cout * d.cin;
            if (i < d.w_off || i >= d.w_off + nw) continue;
            const long long r = i - d.w_off;
            const int t = (int)(r / ((long long)d.cout * d.cin));
            const int co = (int)((r / d.cin) % d.cout), ci = (int)(r % d.cin);
            const bf16 h = __float2bfloat16_rn(w);
            img[d.img + (((long long)t * (d.cin / 16) + ci / 16) * 2 + (ci % 16) / 8) * d.cout * 8 + co * 8 + ci % 8] = h;
            if (d.imgT >= 0) {
                const int tt = 26 - t;
                img[d.imgT + (((long long)tt * (d.cout / 16) + co / 16) * 2 + (co % 16) / 8) * d.cin * 8 + ci * 8 + co % 8] = h;
            }
        }
    }
}

// ------------------------------------------------------------------ host side
// Tensor slots (fopis_unet_tensor indices).
enum Slot {
    S_X0, S_E0, S_D1, S_E1, S_D2, S_E2, S_E3, S_U1, S_A4, S_U0, S_A5,
    S_G5, S_DU0, S_DA1, S_G4, S_DU1, S_DE3, S_G3, S_G2, S_DD2, S_G1, S_DD1, S_G0, S_GE0, S_COUNT
};
struct SlotDesc { int level, ch; };
constexpr SlotDesc kSlot[S_COUNT] = {
    {0, 16}, {0, 16}, {1, 16}, {1, 32}, {2, 32}, {2, 64}, {2, 64}, {1, 64}, {1, 32}, {0, 32}, {0, 16},
    {0, 16}, {0, 32}, {1, 32}, {1, 32}, {1, 64}, {2, 64}, {2, 64}, {2, 64}, {2, 32}, {1, 32}, {1, 16}, {0, 16}, {0, 16}};
// cin, cout, level of the six convolutions
constexpr int kConv[kLayers][3] = {{16, 16, 0}, {16, 32, 1}, {32, 64, 2}, {64, 64, 2}, {64, 32, 1}, {32, 16, 0}};

struct Net {
    NGrid G[kLevels];
    Tensor t[S_COUNT];
    float* out = nullptr;        // prediction per level-0 position
    float* prm = nullptr;
    float* grad = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    bf16* img = nullptr;
    long long nprm = 0, nimg = 0;
    LayerTable T{};
    double* stats = nullptr;     // device [16]
    double* h_stats = nullptr;   // pinned mirror
    unsigned int* err = nullptr;
    int sms = 148;
    // training state
    bool training = false;
    bool loaded = false;         // parameters were set by the caller
    float lr = 1e-3f;
    int64_t steps = 0;
    double last_loss = 0.0;
    bool fwd_valid = false;      // the forward of this step's first solve is in the buffers
    int rejected_run = 0;        // consecutive steps whose guess did not lower the initial residual
    double warm_res = 0.0, guess_res = 0.0;   // last initial residuals relative to ||f||
    double ms_forward = 0.0, ms_train = 0.0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // policy: exponential averages of first-solve V-cycles
    double plain_avg = 0.0, learned_avg = 0.0;
    int plain_n = 0, learned_n = 0, cooldown = 0;
};

Net& net(Ctx& c) { return *static_cast<Net*>(c.unet); }

FeatArgs feat_args(const Ctx& c, const Net& n) {
    FeatArgs F{};
    F.cy = c.cy; F.cz = c.cz;
    const MGLevel& m = c.mg[0];
    F.n0 = m.n[0]; F.n1 = m.n[1]; F.n2 = m.n[2];
    F.p0 = m.per[0]; F.p1 = m.per[1]; F.p2 = m.per[2];
    F.o0 = m.per[0] ? 1 : 2; F.o1 = m.per[1] ? 1 : 2; F.o2 = m.per[2] ? 1 : 2;
    F.nref0 = c.nx; F.nref1 = c.ny; F.nref2 = c.nz;
    F.inv_eps0 = 1.0 / c.p.eps0;
    F.allper = m.per[0] && m.per[1] && m.per[2];
    F.g = gv(n.G[0]);
    return F;
}

int row_grid(long long rows) { return (int)std::max<long long>(1, std::min<long long>(rows, 1LL << 20)); }

template <int CIN, int COUT, int EPI>
void conv(Ctx& c, Net& n, const Tensor& x, const Tensor& y, const bf16* w, const float* bias, const Tensor* mask,
          const Tensor* skip, const float* head, float* out) {
    using S = ConvShape<CIN, COUT>;
    // shared memory at least 1/16 of the SM so that resident CTAs never ask for more than 512 TMEM columns
    const int smem = std::max(S::SMEM, 15 * 1024);
    FOPIS_CUDA(cudaFuncSetAttribute(conv_kernel<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const NGrid& g = *x.g;
    ConvArgs a{};
    a.x = x.view(); a.y = y.view(); a.w = w; a.bias = bias;
    a.mask = mask ? mask->view() : TV{};
    a.skip = skip ? skip->view() : TV{};
    a.head = head; a.out = out;
    a.Sj = g.Sj; a.Si = g.Si; a.P = g.P;
    a.n0 = g.n[0]; a.n1 = g.n[1]; a.n2 = g.n[2];
    a.tiles = g.tiles;
    a.err = n.err;
    const int per_sm = std::max(1, std::min(8, (227 * 1024) / smem));
    const int grid = std::max(1, std::min(g.tiles, n.sms * per_sm));
    ++c.launches;
    conv_kernel<CIN, COUT, EPI><<<grid, 128, smem, c.st>>>(a);
    FOPIS_LAUNCH_CHECK();
}

template <int CIN, int COUT>
void wgrad(Ctx& c, Net& n, const Tensor& x, const Tensor& g, float* dw, float* db) {
    using S = WgShape<CIN, COUT>;
    // shared memory sized so that resident CTAs never ask for more than 512 TMEM columns
    const int smem = std::max(S::SMEM, (S::COLS * 228 * 1024) / 512 + 1024);
    FOPIS_CUDA(cudaFuncSetAttribute(wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const NGrid& G = *x.g;
    WgArgs a{};
    a.x = x.view(); a.g = g.view(); a.dw = dw; a.db = db;
    a.Sj = G.Sj; a.Si = G.Si;
    a.chunks = ((long long)G.tiles * 128) / S::KC;
    a.err = n.err;
    const int per_sm = std::max(1, (227 * 1024) / smem);
    const long long want = std::max<long long>(1, (long long)n.sms * per_sm / S::YSPLIT);
    const int gx = (int)std::max<long long>(1, std::min<long long>(a.chunks, want));
    ++c.launches;
    wgrad_kernel<CIN, COUT><<<dim3(gx, S::YSPLIT), 128, smem, c.st>>>(a);
    FOPIS_LAUNCH_CHECK();
}

void down(Ctx& c, Net& n, const Tensor& src, const Tensor& dst) {
    const NGrid& F = n.G[src.level];
    const NGrid& C = n.G[dst.level];
    ++c.launches;
    down_kernel<<<row_grid((long long)C.n[0] * C.n[1]), 128, 0, c.st>>>(gv(F), gv(C), src.view(), dst.view(), src.C / 8);
    FOPIS_LAUNCH_CHECK();
}
void up(Ctx& c, Net& n, const Tensor& src, const Tensor* src2, const Tensor& dst) {
    const NGrid& C = n.G[src.level];
    const NGrid& F = n.G[dst.level];
    ++c.launches;
    up_kernel<<<row_grid((long long)F.n[0] * F.n[1]), 128, 0, c.st>>>(gv(C), gv(F), src.view(),
                                                                      src2 ? src2->view() : TV{}, dst.view(), src.C / 8);
    FOPIS_LAUNCH_CHECK();
}
void up_adjoint(Ctx& c, Net& n, const Tensor& src, const Tensor& dst) {
    const NGrid& F = n.G[src.level];
    const NGrid& C = n.G[dst.level];
    ++c.launches;
    up_adjoint_kernel<<<row_grid((long long)C.n[0] * C.n[1]), 128, 0, c.st>>>(gv(F), gv(C), src.view(), dst.view(),
                                                                              src.C / 8);
    FOPIS_LAUNCH_CHECK();
}
void gmask(Ctx& c, Net& n, const Tensor* add, const Tensor* coarse, const Tensor& act, const Tensor& out) {
    const NGrid& F = n.G[act.level];
    const NGrid& C = n.G[std::min(act.level + 1, kLevels - 1)];
    ++c.launches;
    gmask_kernel<<<row_grid((long long)F.n[0] * F.n[1]), 128, 0, c.st>>>(
        gv(F), gv(C), add ? add->view() : TV{}, coarse ? coarse->view() : TV{}, act.view(), out.view(), act.C / 8);
    FOPIS_LAUNCH_CHECK();
}

const bf16* wimg(const Net& n, int l) { return n.img + n.T.l[l].img; }
const bf16* wimgT(const Net& n, int l) { return n.img + n.T.l[l].imgT; }
const float* bias_of(const Net& n, int l) { return n.prm + n.T.l[l].b_off; }

// Features of (rho0, phi1, phi2) and the forward pass; the prediction lands in n.out.
void forward(Ctx& c, Net& n, const double* rho0, const double* phi1, const double* phi2) {
    const FeatArgs F = feat_args(c, n);
    FOPIS_CUDA(cudaMemsetAsync(n.stats, 0, 16 * sizeof(double), c.st));
    const long long rows = (long long)F.n0 * F.n1;
    ++c.launches;
    feat_stats_kernel<<<row_grid(std::min<long long>(rows, n.sms * 8)), 256, 0, c.st>>>(F, rho0, phi1, phi2, n.stats);
    ++c.launches;
    feat_sigma_kernel<<<1, 1, 0, c.st>>>(n.stats, (double)F.n0 * F.n1 * F.n2, F.allper);
    ++c.launches;
    feat_write_kernel<<<row_grid(rows), 256, 0, c.st>>>(F, rho0, phi1, phi2, n.stats, n.t[S_X0].view());
    FOPIS_LAUNCH_CHECK();
    Tensor* t = n.t;
    conv<16, 16, EPI_FWD>(c, n, t[S_X0], t[S_E0], wimg(n, 0), bias_of(n, 0), nullptr, nullptr, nullptr, nullptr);
    down(c, n, t[S_E0], t[S_D1]);
    conv<16, 32, EPI_FWD>(c, n, t[S_D1], t[S_E1], wimg(n, 1), bias_of(n, 1), nullptr, nullptr, nullptr, nullptr);
    down(c, n, t[S_E1], t[S_D2]);
    conv<32, 64, EPI_FWD>(c, n, t[S_D2], t[S_E2], wimg(n, 2), bias_of(n, 2), nullptr, nullptr, nullptr, nullptr);
    conv<64, 64, EPI_FWD>(c, n, t[S_E2], t[S_E3], wimg(n, 3), bias_of(n, 3), nullptr, nullptr, nullptr, nullptr);
    up(c, n, t[S_E3], nullptr, t[S_U1]);
    conv<64, 32, EPI_FWD>(c, n, t[S_U1], t[S_A4], wimg(n, 4), bias_of(n, 4), nullptr, nullptr, nullptr, nullptr);
    up(c, n, t[S_A4], &t[S_E1], t[S_U0]);
    conv<32, 16, EPI_HEAD>(c, n, t[S_U0], t[S_A5], wimg(n, 5), bias_of(n, 5), nullptr, &t[S_E0],
                           n.prm + n.T.head_off, n.out);
}

// Loss against phi_new - phi1 and the gradients of every parameter into n.grad.
void backward(Ctx& c, Net& n, const double* phi_new, const double* phi1) {
    const FeatArgs F = feat_args(c, n);
    Tensor* t = n.t;
    FOPIS_CUDA(cudaMemsetAsync(n.grad, 0, sizeof(float) * n.nprm, c.st));
    const long long rows = (long long)F.n0 * F.n1;
    ++c.launches;
    loss_kernel<<<row_grid(std::min<long long>(rows, n.sms * 8)), 256, 0, c.st>>>(
        F, n.out, phi_new, phi1, n.stats, t[S_A5].view(), t[S_E0].view(), n.prm + n.T.head_off,
        n.grad + n.T.head_off, t[S_G5].view(), t[S_GE0].view(), 1.0 / ((double)F.n0 * F.n1 * F.n2));
    FOPIS_LAUNCH_CHECK();
    auto dw = [&](int l) { return n.grad + n.T.l[l].w_off; };
    auto db = [&](int l) { return n.grad + n.T.l[l].b_off; };
    wgrad<32, 16>(c, n, t[S_U0], t[S_G5], dw(5), db(5));
    conv<16, 32, EPI_BWD>(c, n, t[S_G5], t[S_DU0], wimgT(n, 5), nullptr, nullptr, nullptr, nullptr, nullptr);
    up_adjoint(c, n, t[S_DU0], t[S_DA1]);
    gmask(c, n, &t[S_DA1], nullptr, t[S_A4], t[S_G4]);
    wgrad<64, 32>(c, n, t[S_U1], t[S_G4], dw(4), db(4));
    conv<32, 64, EPI_BWD>(c, n, t[S_G4], t[S_DU1], wimgT(n, 4), nullptr, nullptr, nullptr, nullptr, nullptr);
    up_adjoint(c, n, t[S_DU1], t[S_DE3]);
    gmask(c, n, &t[S_DE3], nullptr, t[S_E3], t[S_G3]);
    wgrad<64, 64>(c, n, t[S_E2], t[S_G3], dw(3), db(3));
    conv<64, 64, EPI_BWD>(c, n, t[S_G3], t[S_G2], wimgT(n, 3), nullptr, &t[S_E2], nullptr, nullptr, nullptr);
    wgrad<32, 64>(c, n, t[S_D2], t[S_G2], dw(2), db(2));
    conv<64, 32, EPI_BWD>(c, n, t[S_G2], t[S_DD2], wimgT(n, 2), nullptr, nullptr, nullptr, nullptr, nullptr);
    gmask(c, n, &t[S_DA1], &t[S_DD2], t[S_E1], t[S_G1]);
    wgrad<16, 32>(c, n, t[S_D1], t[S_G1], dw(1), db(1));
    conv<32, 16, EPI_BWD>(c, n, t[S_G1], t[S_DD1], wimgT(n, 1), nullptr, nullptr, nullptr, nullptr, nullptr);
    gmask(c, n, &t[S_GE0], &t[S_DD1], t[S_E0], t[S_G0]);
    wgrad<16, 16>(c, n, t[S_X0], t[S_G0], dw(0), db(0));
}

void adam(Ctx& c, Net& n, bool step) {
    float bc1 = 1.0f, bc2 = 1.0f;
    if (step) {
        const double k = (double)(n.steps + 1);
        bc1 = (float)(1.0 - std::pow(0.9, k));
        bc2 = (float)(1.0 - std::pow(0.999, k));
    }
    ++c.launches;
    adam_kernel<<<std::max<long long>(1, std::min<long long>((n.nprm + 255) / 256, 4096)), 256, 0, c.st>>>(
        n.T, n.nprm, n.prm, n.grad, n.m1, n.m2, n.img, n.lr, bc1, bc2, step ? 1 : 0);
    FOPIS_LAUNCH_CHECK();
}

void check_err(Ctx& c, Net& n) {
    unsigned int e = 0;
    FOPIS_CUDA(cudaMemcpyAsync(&e, n.err, sizeof(e), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    if (e) throw ApiError{FOPIS_ERR_DEVICE, "learned guess: tensor-core pipeline wait timed out (code " +
                                                std::to_string(e) + ")"};
}

void init_params(const Ctx& c, Net& n) {
    std::vector<float> h(n.nprm, 0.0f);
    const uint64_t seed = c.p.seed ^ 0x5eedu;
    uint32_t ctr = 0;
    auto normal = [&]() {
        const U2 u = draw2(seed, 0x4E4554u, ctr++, 0, 0);
        return std::sqrt(-2.0 * std::log(1.0 - u.a)) * std::cos(2.0 * M_PI * u.b);
    };
    for (int l = 0; l < kLayers; ++l) {
        const LayerDesc& d = n.T.l[l];
        const double sd = std::sqrt(2.0 / (27.0 * d.cin));
        for (long long i = 0; i < 27LL * d.cout * d.cin; ++i) h[d.w_off + i] = (float)(sd * normal());
    }
    for (int ch = 0; ch < kHead; ++ch) h[n.T.head_off + ch] = (float)(0.05 * normal());
    FOPIS_CUDA(cudaMemcpy(n.prm, h.data(), sizeof(float) * n.nprm, cudaMemcpyHostToDevice));
}

}  // namespace

void unet_free(Ctx& c) {
    if (!c.unet) return;
    Net* n = static_cast<Net*>(c.unet);
    for (auto& t : n->t) if (t.base) cudaFree(t.base);
    void* p[] = {n->out, n->prm, n->grad, n->m1, n->m2, n->img, n->stats, n->err};
    for (void* q : p) if (q) cudaFree(q);
    if (n->h_stats) cudaFreeHost(n->h_stats);
    for (auto& e : n->ev) if (e) cudaEventDestroy(e);
    delete n;
    c.unet = nullptr;
}

namespace {

Net* create(Ctx& c) {
    if (c.mg.size() < (size_t)kLevels) throw ApiError{FOPIS_ERR_STATE, "learned guess needs three multigrid levels"};
    auto* n = new Net();
    c.unet = n;
    try {
        int dev = 0;
        FOPIS_CUDA(cudaGetDevice(&dev));
        FOPIS_CUDA(cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, dev));
        for (int l = 0; l < kLevels; ++l) n->G[l] = make_grid(c.mg[l]);
        for (int s = 0; s < S_COUNT; ++s) {
            Tensor& t = n->t[s];
            t.C = kSlot[s].ch;
            t.level = kSlot[s].level;
            t.g = &n->G[t.level];
            FOPIS_CUDA(cudaMalloc(&t.base, t.bytes()));
            FOPIS_CUDA(cudaMemset(t.base, 0, t.bytes()));
        }
        FOPIS_CUDA(cudaMalloc(&n->out, sizeof(float) * n->G[0].P));
        FOPIS_CUDA(cudaMemset(n->out, 0, sizeof(float) * n->G[0].P));
        long long off = 0, img = 0;
        for (int l = 0; l < kLayers; ++l) {
            LayerDesc& d = n->T.l[l];
            d.cin = kConv[l][0];
            d.cout = kConv[l][1];
            d.w_off = off;
            off += 27LL * d.cin * d.cout;
            d.b_off = off;
            off += d.cout;
            d.img = img;
            img += 27LL * d.cin * d.cout;
            if (l > 0) { d.imgT = img; img += 27LL * d.cin * d.cout; } else d.imgT = -1;
        }
        n->T.head_off = off;
        off += kHead + 1;
        n->nprm = off;
        n->nimg = img;
        FOPIS_CUDA(cudaMalloc(&n->prm, sizeof(float) * off));
        FOPIS_CUDA(cudaMalloc(&n->grad, sizeof(float) * off));
        FOPIS_CUDA(cudaMalloc(&n->m1, sizeof(float) * off));
        FOPIS_CUDA(cudaMalloc(&n->m2, sizeof(float) * off));
        FOPIS_CUDA(cudaMemset(n->grad, 0, sizeof(float) * off));
        FOPIS_CUDA(cudaMemset(n->m1, 0, sizeof(float) * off));
        FOPIS_CUDA(cudaMemset(n->m2, 0, sizeof(float) * off));
        FOPIS_CUDA(cudaMalloc(&n->img, sizeof(bf16) * img));
        FOPIS_CUDA(cudaMalloc(&n->stats, 16 * sizeof(double)));
        FOPIS_CUDA(cudaMemset(n->stats, 0, 16 * sizeof(double)));
        FOPIS_CUDA(cudaMallocHost(&n->h_stats, 16 * sizeof(double)));
        std::memset(n->h_stats, 0, 16 * sizeof(double));
        for (auto& e : n->ev) FOPIS_CUDA(cudaEventCreate(&e));
        FOPIS_CUDA(cudaMalloc(&n->err, sizeof(unsigned int)));
        FOPIS_CUDA(cudaMemset(n->err, 0, sizeof(unsigned int)));
        init_params(c, *n);
    } catch (...) {
        unet_free(c);
        throw;
    }
    return n;
}

Net& ensure(Ctx& c) {
    if (!c.unet) {
        create(c);
        adam(c, net(c), false);   // operand images of the initial weights
    }
    return net(c);
}

void train_step(Ctx& c, Net& n, const double* phi_new, const double* phi1) {
    FOPIS_CUDA(cudaEventRecord(n.ev[2], c.st));
    backward(c, n, phi_new, phi1);
    adam(c, n, true);
    FOPIS_CUDA(cudaEventRecord(n.ev[3], c.st));
    FOPIS_CUDA(cudaMemcpyAsync(n.h_stats, n.stats, 16 * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    check_err(c, n);
    float ms = 0.0f;
    FOPIS_CUDA(cudaEventElapsedTime(&ms, n.ev[2], n.ev[3]));
    n.ms_train = ms;
    n.last_loss = n.h_stats[11] / ((double)c.mg[0].n[0] * c.mg[0].n[1] * c.mg[0].n[2]);
    n.steps += 1;
}

}  // namespace

int unet_set_training(Ctx& c, int enable, double lr) {
    Net& n = ensure(c);
    n.training = enable != 0;
    if (lr > 0.0) n.lr = (float)lr;
    return FOPIS_OK;
}

int unet_get_state(Ctx& c, double* loss, int64_t* steps) {
    if (loss) *loss = c.unet ? net(c).last_loss : 0.0;
    if (steps) *steps = c.unet ? net(c).steps : 0;
    return FOPIS_OK;
}

int unet_get_policy(Ctx& c, double* plain, double* learned, int* active) {
    if (plain) *plain = c.unet ? net(c).plain_avg : 0.0;
    if (learned) *learned = c.unet ? net(c).learned_avg : 0.0;
    if (active) *active = c.unet ? (net(c).cooldown == 0 ? 1 : 0) : 0;
    return FOPIS_OK;
}

int unet_get_last(Ctx& c, double* warm_res, double* guess_res, double* ms_forward, double* ms_train) {
    const Net* n = c.unet ? static_cast<const Net*>(c.unet) : nullptr;
    if (warm_res) *warm_res = n ? n->warm_res : 0.0;
    if (guess_res) *guess_res = n ? n->guess_res : 0.0;
    if (ms_forward) *ms_forward = n ? n->ms_forward : 0.0;
    if (ms_train) *ms_train = n ? n->ms_train : 0.0;
    return FOPIS_OK;
}

bool unet_training(const Ctx& c) { return c.unet && static_cast<const Net*>(c.unet)->training; }

bool unet_active(const Ctx& c) {
    return c.unet && (static_cast<const Net*>(c.unet)->training || c.p.guess_mode == FOPIS_GUESS_LEARNED);
}

// Before the first solve of a step, with a valid solve history (phi_prev =
// previous first solve = the start in FOPIS_GUESS_LEARNED, phi_prev2 = the one
// before): runs the network on (rho0, phi_prev, phi_prev2) and, when the policy
// allows, adds sigma_d * prediction to phi; a guess that does not lower the
// initial residual is taken back. Returns 1 when phi keeps the guess.
int unet_before_solve(Ctx& c) {
    if (c.p.guess_mode == FOPIS_GUESS_LEARNED) ensure(c);
    if (!unet_active(c) || !c.hist_ok) return 0;
    Net& n = net(c);
    FOPIS_CUDA(cudaEventRecord(n.ev[0], c.st));
    forward(c, n, c.rho0, c.phi_prev, c.phi_prev2);
    n.fwd_valid = true;
    bool use = c.p.guess_mode == FOPIS_GUESS_LEARNED && (n.steps > 0 || n.loaded) && n.cooldown == 0;
    const FeatArgs F = feat_args(c, n);
    if (use) {
        ++c.launches;
        apply_guess_kernel<<<row_grid((long long)F.n0 * F.n1), 256, 0, c.st>>>(F, n.out, n.stats, c.phi);
        ++c.launches;
        guess_residual_kernel<<<row_grid(std::min<long long>((long long)F.n0 * F.n1, n.sms * 8)), 256, 0, c.st>>>(
            F, c.rho0, c.phi, n.stats);
        FOPIS_LAUNCH_CHECK();
    }
    FOPIS_CUDA(cudaEventRecord(n.ev[1], c.st));
    FOPIS_CUDA(cudaMemcpyAsync(n.h_stats, n.stats, 16 * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    check_err(c, n);
    float ms = 0.0f;
    FOPIS_CUDA(cudaEventElapsedTime(&ms, n.ev[0], n.ev[1]));
    n.ms_forward = ms;
    const double M = (double)F.n0 * F.n1 * F.n2, fm = n.h_stats[9];
    const double fnorm = std::sqrt(M) * n.h_stats[6];
    const double warm2 = std::max(0.0, n.h_stats[5] - 2.0 * fm * n.h_stats[4] + M * fm * fm);
    n.warm_res = std::sqrt(warm2) / fnorm;
    n.guess_res = use ? std::sqrt(n.h_stats[12]) / fnorm : n.warm_res;
    if (use && !(n.h_stats[12] < warm2)) {
        FOPIS_CUDA(cudaMemcpyAsync(c.phi, c.phi_prev, sizeof(double) * c.N, cudaMemcpyDeviceToDevice, c.st));
        use = false;
        if (++n.rejected_run >= 8) { n.cooldown = 32; n.rejected_run = 0; }
    } else if (use) {
        n.rejected_run = 0;
    }
    return use ? 1 : 0;
}

// After the first solve (before the history moves on): trains on the pair
// (features, phi^n - phi_prev) and updates the V-cycle policy.
void unet_after_solve(Ctx& c, bool used, int cycles, bool converged) {
    if (!c.unet || !net(c).fwd_valid) return;
    Net& n = net(c);
    n.fwd_valid = false;
    // no target scale on the first step of a history (phi^{n-1} = phi^{n-2})
    if (n.training && converged && n.h_stats[7] > 0.0) train_step(c, n, c.phi, c.phi_prev);
    if (c.p.guess_mode == FOPIS_GUESS_LEARNED || n.training) {
        const double a = 0.125;
        if (used) {
            n.learned_avg = n.learned_n ? (1 - a) * n.learned_avg + a * cycles : cycles;
            n.learned_n += 1;
            // fall back when the learned start stops saving V-cycles over the history start
            if (n.learned_n >= 8 && (n.plain_n == 0 || n.learned_avg >= n.plain_avg - 0.05)) {
                n.cooldown = 32;
                n.learned_n = 0;
            }
        } else {
            n.plain_avg = n.plain_n ? (1 - a) * n.plain_avg + a * cycles : cycles;
            n.plain_n += 1;
            if (n.cooldown > 0) n.cooldown -= 1;
        }
    }
}

// ---------------------------------------------------------------- ABI helpers
int unet_eval(Ctx& c, const double* rho0, const double* phi1, const double* phi2, const double* phi_target,
              double* pred, float* grads, double* loss) {
    Net& n = ensure(c);
    const size_t bytes = sizeof(double) * c.N;
    double* d = nullptr;
    FOPIS_CUDA(cudaMallocAsync(&d, 4 * bytes, c.st));
    struct Free {
        Ctx& c;
        double* d;
        ~Free() { cudaFreeAsync(d, c.st); }
    } guard{c, d};
    FOPIS_CUDA(cudaMemcpyAsync(d, rho0, bytes, cudaMemcpyHostToDevice, c.st));
    FOPIS_CUDA(cudaMemcpyAsync(d + c.N, phi1, bytes, cudaMemcpyHostToDevice, c.st));
    FOPIS_CUDA(cudaMemcpyAsync(d + 2 * c.N, phi2, bytes, cudaMemcpyHostToDevice, c.st));
    forward(c, n, d, d + c.N, d + 2 * c.N);
    n.fwd_valid = false;
    if (phi_target) {
        FOPIS_CUDA(cudaMemcpyAsync(d + 3 * c.N, phi_target, bytes, cudaMemcpyHostToDevice, c.st));
        backward(c, n, d + 3 * c.N, d + c.N);
    }
    FOPIS_CUDA(cudaMemcpyAsync(n.h_stats, n.stats, 16 * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    std::vector<float> out(n.G[0].P);
    FOPIS_CUDA(cudaMemcpyAsync(out.data(), n.out, sizeof(float) * out.size(), cudaMemcpyDeviceToHost, c.st));
    if (grads && phi_target)
        FOPIS_CUDA(cudaMemcpyAsync(grads, n.grad, sizeof(float) * n.nprm, cudaMemcpyDeviceToHost, c.st));
    check_err(c, n);
    const double sd = n.h_stats[7];
    if (loss) *loss = phi_target ? n.h_stats[11] / ((double)c.mg[0].n[0] * c.mg[0].n[1] * c.mg[0].n[2]) : 0.0;
    if (pred) {
        std::fill(pred, pred + c.N, 0.0);
        const MGLevel& m = c.mg[0];
        const int o[3] = {m.per[0] ? 1 : 2, m.per[1] ? 1 : 2, m.per[2] ? 1 : 2};
        const NGrid& g = n.G[0];
        for (int a = 0; a < m.n[0]; ++a)
            for (int b = 0; b < m.n[1]; ++b)
                for (int k = 0; k < m.n[2]; ++k) {
                    const long long p = (long long)(a + 1) * g.Si + (long long)(b + 1) * g.Sj + (k + 1);
                    pred[((size_t)(a + o[0]) * c.cy + (b + o[1])) * c.cz + (k + o[2])] = sd * (double)out[p];
                }
    }
    return FOPIS_OK;
}

int unet_params(Ctx& c, float* get, const float* set, int64_t* count) {
    Net& n = ensure(c);
    if (count) *count = n.nprm;
    if (set) {
        FOPIS_CUDA(cudaMemcpyAsync(n.prm, set, sizeof(float) * n.nprm, cudaMemcpyHostToDevice, c.st));
        adam(c, n, false);
        n.loaded = true;
    }
    if (get) FOPIS_CUDA(cudaMemcpyAsync(get, n.prm, sizeof(float) * n.nprm, cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    return FOPIS_OK;
}

int unet_tensor(Ctx& c, int which, float* host, int64_t cap, int64_t* count) {
    Net& n = ensure(c);
    if (which < 0 || which > S_COUNT) throw ApiError{FOPIS_ERR_ARG, "tensor index"};
    const int level = which == S_COUNT ? 0 : kSlot[which].level;
    const int ch = which == S_COUNT ? 1 : kSlot[which].ch;
    const NGrid& g = n.G[level];
    const int64_t total = (int64_t)g.n[0] * g.n[1] * g.n[2] * ch;
    if (count) *count = total;
    if (!host) return FOPIS_OK;
    if (cap < total) throw ApiError{FOPIS_ERR_ARG, "tensor buffer too small"};
    std::vector<float> raw;
    std::vector<uint16_t> bits;
    if (which == S_COUNT) {
        raw.resize(g.P);
        FOPIS_CUDA(cudaMemcpyAsync(raw.data(), n.out, sizeof(float) * g.P, cudaMemcpyDeviceToHost, c.st));
    } else {
        bits.resize((size_t)(ch / 8) * g.stride * 8);
        FOPIS_CUDA(cudaMemcpyAsync(bits.data(), n.t[which].base, bits.size() * 2, cudaMemcpyDeviceToHost, c.st));
    }
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    int64_t o = 0;
    for (int a = 0; a < g.n[0]; ++a)
        for (int b = 0; b < g.n[1]; ++b)
            for (int k = 0; k < g.n[2]; ++k) {
                const long long p = (long long)(a + 1) * g.Si + (long long)(b + 1) * g.Sj + (k + 1);
                for (int q = 0; q < ch; ++q) {
                    if (which == S_COUNT) { host[o++] = raw[p]; continue; }
                    const uint32_t u = (uint32_t)bits[((size_t)(q / 8) * g.stride + g.front + p) * 8 + q % 8] << 16;
                    float f;
                    std::memcpy(&f, &u, 4);
                    host[o++] = f;
                }
            }
    return FOPIS_OK;
}

}  // namespace fopis

// Device self-check of the bounded wait (include/fopis_gpu.h).
extern "C" int fopis_check_bounded_wait(int device, uint32_t polls, int arrive, uint32_t* status) {
    using namespace fopis;
    if (!status) return FOPIS_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FOPIS_ERR_NO_CUDA;
    if (device < 0 || device >= ndev || cudaSetDevice(device) != cudaSuccess) return FOPIS_ERR_ARG;
    unsigned int* d = nullptr;
    if (cudaMalloc(&d, sizeof(unsigned int)) != cudaSuccess) return FOPIS_ERR_NOMEM;
    int rc = FOPIS_OK;
    unsigned int h = 0;
    if (cudaMemset(d, 0, sizeof(unsigned int)) != cudaSuccess) rc = FOPIS_ERR_CUDA;
    if (rc == FOPIS_OK) {
        bounded_wait_check_kernel<<<1, 32>>>(polls, arrive, d);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = FOPIS_ERR_CUDA;
    }
    cudaFree(d);
    *status = h;
    return rc;
}
