// internal.cuh — device data layout and helpers shared by the libfopis_gpu.so
// translation units. Not part of the public ABI (include/fopis_gpu.h).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fopis_gpu.h"

namespace fopis {

// ------------------------------------------------------------------ errors
struct CudaError {
    cudaError_t code;
    const char* where;
};
#define FOPIS_CUDA(call)                                                  \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) throw ::fopis::CudaError{e_, #call};      \
    } while (0)
#define FOPIS_LAUNCH_CHECK() FOPIS_CUDA(cudaGetLastError())

struct ApiError {
    int code;
    std::string msg;
};

// ------------------------------------------------------------------ packed cells
// A particle's node cell (glue-layout indices i = floor(x)+1 ...) packed into
// one int32: (i << 20) | (j << 10) | k. Invalid particles hold -1.
constexpr int kCellBits = 10;
constexpr int kCellMask = (1 << kCellBits) - 1;
__host__ __device__ __forceinline__ int32_t pack_cell(int i, int j, int k) {
    return (i << 20) | (j << 10) | k;
}
__host__ __device__ __forceinline__ void unpack_cell(int32_t c, int& i, int& j, int& k) {
    i = (c >> 20) & kCellMask;
    j = (c >> 10) & kCellMask;
    k = c & kCellMask;
}

// Fixed-point scales. Deposit: each in-cell offset is rounded to 17 fractional
// bits; a particle's eight corner weights sum to 2^51. Surface charge: each
// in-face coordinate to 20 bits; four corner weights sum to 2^40.
constexpr int kDepositBits = 17;
constexpr float kDepositScale = 131072.0f;  // 2^17
constexpr int64_t kDepositOne = 131072;     // 2^17
constexpr double kDepositUnit = 0x1p-51;
constexpr double kSurfaceScale = 1048576.0;  // 2^20
constexpr int64_t kSurfaceOne = 1048576;
constexpr double kSurfaceUnit = 0x1p-40;

// ------------------------------------------------------------------ Philox
// Philox4x32-10 (Salmon et al., SC'11). Identical keying to the oracle so the
// GPU and CPU draw the same particle sets.
enum : uint32_t { TAG_LOAD = 1u, TAG_INJECT = 2u, TAG_EMIT = 3u, TAG_SECONDARY = 4u };

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    }
}
struct U2 { double a, b; };
__host__ __device__ __forceinline__ U2 draw2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    uint32_t c[4] = {c0, c1, c2, c3};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t x = ((uint64_t)c[0] << 32) | c[1];
    const uint64_t y = ((uint64_t)c[2] << 32) | c[3];
    return {(double)(x >> 11) * 0x1p-53, (double)(y >> 11) * 0x1p-53};
}
__device__ __forceinline__ void box_muller(double u1, double u2, double& n0, double& n1) {
    const double r = sqrt(-2.0 * log(1.0 - u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    n0 = r * c;
    n1 = r * s;
}

// ------------------------------------------------------------------ device data
// Particles of one species as structure of arrays: packed node cell plus
// in-cell offsets and velocities, FP32 in the mixed mode, FP64 in FOPIS_FP64.
template <typename T>
struct SoaT {
    int32_t* cell = nullptr;
    T *ox = nullptr, *oy = nullptr, *oz = nullptr;
    T *vx = nullptr, *vy = nullptr, *vz = nullptr;
};
using Soa = SoaT<float>;
using Soa64 = SoaT<double>;

// Nodal E of the FP64 mode (one 32-byte record per node; w unused).
struct alignas(32) Vec4d { double x, y, z, w; };

// Scalars the kernels update; one copy lives on the device and is mirrored to
// pinned host memory after each API call.
struct DevScalars {
    unsigned long long count[FOPIS_MAX_SPECIES];        // slots in use per species
    unsigned long long absorbed_n;                      // entries in the absorbed list
    unsigned long long absorbed_by[FOPIS_MAX_OBJECTS][FOPIS_MAX_SPECIES];
    unsigned long long emitted_by[FOPIS_MAX_OBJECTS][FOPIS_MAX_SPECIES];
    unsigned long long injected;
    unsigned long long not_found;
    unsigned int status;                                // FOPIS_DEV_* bits
    unsigned int pad;
    unsigned long long pointwise_bits;                  // last solve's pointwise residual (double bits)
    // per species in the current fused step: valid particles the push moved, those that
    // stayed valid (in the domain, not absorbed), and particles injected or emitted
    unsigned long long pushed[FOPIS_MAX_SPECIES], survived[FOPIS_MAX_SPECIES], added[FOPIS_MAX_SPECIES];
    unsigned long long incident_n;                      // entries in the incident list
    unsigned long long secondary_n;                     // secondaries the pending incidents will emit
    double energy[FOPIS_MAX_SPECIES];                   // sum of v^2 of live particles
    double red[16];                                     // scratch reduction slots
};

// Absorbed-particle list, written by the deposit paths, read by absorb_kernel
// (FP64 so that both particle precisions store their state exactly).
struct AbsorbList {
    int32_t* cell = nullptr;
    double *ox = nullptr, *oy = nullptr, *oz = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    uint8_t* species = nullptr;
    uint8_t* object = nullptr;
    int64_t cap = 0;
};

// Incident events of Spacecraft::addIncidentEvent (SecondaryEmission.cpp:14-33):
// recorded by absorb_kernel for objects that emit secondaries, consumed by the
// next step's emission.
struct IncidentList {
    double *x = nullptr, *y = nullptr, *z = nullptr;      // crossing point
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;   // incident velocity
    double* trem = nullptr;                               // remaining time (move ratio since the crossing)
    uint8_t *species = nullptr, *object = nullptr, *axis = nullptr;
    int32_t* count = nullptr;                             // secondaries per incident (count pass)
    int64_t cap = 0;
};

struct ObjectDev {
    int n = 0;
    std::vector<int32_t> nodes_ijk;    // host copy, [n][3]
    int32_t* nodes = nullptr;          // linear node indices [n]
    double* C = nullptr;               // [n][n] row-major C(i,j)
    double* colsum = nullptr;          // sum_i C(i,j)
    double total = 0.0;                // Cmatrix::total
    long long* charge_tmp = nullptr;   // [nsp][n] fixed point (2^-40)
    double* charge_map = nullptr;      // [nsp][n]
    double* phis = nullptr;            // phi at the surface nodes
    double* drho_buf = nullptr;        // [3][n] redistributed surface charge of the last three steps
    double* drho[3] = {nullptr, nullptr, nullptr};   // this step, one and two steps back
    double* scal = nullptr;            // [4]: potential, total charge, sum C phi
    int is_fixed = 0;
    double fixed_potential = 0.0, offset = 0.0;
    int emit_species = -1;
    int secondary_species = -1;        // SecondaryParticleType emitted by this body, -1 = none
    int dielectric = 0;                // surface_type "dielectric"
    double* capacitance = nullptr;     // [n] node capacitance (dielectric)
    int n_lit = 0;
    int32_t* lit = nullptr;            // cmat numbers of the lit nodes
    bool has_C = false;
    double potential = 0.0, total_charge = 0.0;
    double current[FOPIS_MAX_SPECIES] = {0};
};

struct MGLevel {
    int n[3];            // unknowns per axis
    int per[3];          // axis periodic
    float* u = nullptr;  // correction
    float* f = nullptr;  // right-hand side
    float* r = nullptr;  // residual scratch
    double scale = 1.0;  // operator scale 1/4^level relative to the fine level
    size_t size() const { return (size_t)n[0] * n[1] * n[2]; }
};

// A Yee array of the EM mode: boost::multi_array with index bases, C order,
// element (i, j, k) at ((i - lo0) n1 + (j - lo1)) n2 + (k - lo2).
struct YeeArr {
    double* v = nullptr;
    int lo[3] = {0, 0, 0};
    int n[3] = {0, 0, 0};
    size_t size() const { return (size_t)n[0] * n[1] * n[2]; }
};

// Device state of the EM solver (FOPIS_SOLVER_EM).
struct EMState {
    bool on = false;
    int L[3] = {1, 1, 1};            // Environment::damping_length: the node counts
    int lo[3] = {0, 0, 0};           // x_low.. of RootGrid::initializeField
    int up[3] = {0, 0, 0};           // x_up..
    YeeArr f[6];                     // ex, ey, ez, bx, by, bz
    double* j[3] = {nullptr, nullptr, nullptr};   // jx [cx-1][cy][cz], jy [cx][cy-1][cz], jz [cx][cy][cz-1]
    double* eref = nullptr;          // [3][N] nodal E (FP64, the export copy)
    double* bref = nullptr;          // [3][N] nodal B (FP64)
    float4* B = nullptr;             // nodal B (FP32) for the gather of the mixed mode
    Vec4d* B64 = nullptr;            // nodal B (FP64) for the FP64 mode
    double* mask = nullptr;          // damping factor per axis and index (x, y, z extents back to back)
    unsigned long long* jfix = nullptr;   // mixed mode: [nsp][jx | jy | jz] fixed-point current sums (2^-40)
};

struct Ctx {
    fopis_params p{};
    int device = 0;
    cudaStream_t st = nullptr;
    int nx = 0, ny = 0, nz = 0;   // reference node counts
    int cx = 0, cy = 0, cz = 0;   // with glue
    size_t N = 0;                 // nodes with glue
    int per[6] = {0};             // isNotBoundary per side
    int nsp = 0;
    // particles
    bool fp64 = false;            // FOPIS_FP64: particles in dp/dp2, E in E64
    Soa sp[FOPIS_MAX_SPECIES];
    Soa sp2[FOPIS_MAX_SPECIES];   // sort targets
    Soa64 dp[FOPIS_MAX_SPECIES];
    Soa64 dp2[FOPIS_MAX_SPECIES];
    int64_t cap[FOPIS_MAX_SPECIES] = {0};
    int64_t nslots[FOPIS_MAX_SPECIES] = {0};   // host mirror of DevScalars::count
    int64_t sorted_n[FOPIS_MAX_SPECIES] = {0}; // slots [0, sorted_n) are brick-sorted
    int64_t valid[FOPIS_MAX_SPECIES] = {0};    // valid particles after the last fused step or sort
    int64_t pushed_step[FOPIS_MAX_SPECIES] = {0};   // valid particles the last fused step pushed
    int32_t* brick_start[FOPIS_MAX_SPECIES] = {nullptr};  // first slot of each brick
    // fields
    unsigned long long* rho_i64 = nullptr;  // [nsp][N] two's complement fixed point (FP64 mode: double weights)
    double* rho0 = nullptr;
    double* phi = nullptr;
    double* phi_prev = nullptr;      // first-solve phi of the previous step
    double* phi_prev2 = nullptr;     // first-solve phi two steps back
    double* phi_obj = nullptr;       // previous step's conductor response
    double* phi_obj2 = nullptr;      // the one before it
    int obj_hist = 0;                // conductor responses recorded (0..2)
    double* scratch64 = nullptr;     // [N] residual / field export
    float4* E = nullptr;             // nodal E (FP32) for the gather
    Vec4d* E64 = nullptr;            // nodal E (FP64) for the gather of the FP64 mode
    uint8_t* cellmap = nullptr;      // [N] object id + 1 of the node cell, 0 outside
    int32_t* node_cmat = nullptr;    // [N] (object << 24) | cmat, -1 elsewhere
    // sort
    int32_t* sort_count = nullptr;   // [N + 1]
    int32_t* sort_offset = nullptr;  // [N + 1]
    int32_t* scan_partials = nullptr;
    // absorbed list
    AbsorbList ab;
    IncidentList inc;
    // multigrid
    std::vector<MGLevel> mg;
    double* coarse64 = nullptr;
    cudaGraph_t mg_graph = nullptr;  // one refinement iteration, recorded once
    cudaGraphExec_t mg_exec = nullptr;
    // the whole solve as one graph with a device-side while loop over refinement
    // iterations (state: 0 not built, 1 built, -1 unavailable -> host loop)
    cudaGraph_t solve_graph = nullptr;
    cudaGraphExec_t solve_exec = nullptr;
    cudaStream_t body_st = nullptr;
    int solve_state = 0;
    bool pdl = true;                 // solver kernels launched with programmatic dependent launch
    int64_t solve_pre_launches = 0, solve_post_launches = 0;
    int64_t cycle_launches = 0;      // kernels in that graph
    int mg_cta_start = -1;           // first level whose V-cycle runs inside one CTA
    double* red_partials = nullptr;  // block partial sums
    int red_blocks = 0;
    // objects
    std::vector<ObjectDev> objs;
    // scalars
    DevScalars* d_sc = nullptr;
    DevScalars* h_sc = nullptr;
    double inject_residual[FOPIS_MAX_SPECIES][6] = {{0}};
    int64_t timestep = 1;            // Environment::timestep
    bool energy_valid = false;
    // solver state
    int last_vcycles = 0;
    double last_res = 0.0, first_res = 0.0;
    int last_converged = 1;
    int step_vcycles = 0, step_solves = 0;
    int64_t injected_step = 0, emitted_step = 0, absorbed_step = 0;
    int learned_used = 0;
    double ms_phase[8] = {0};
    cudaEvent_t ev[9] = {nullptr};
    std::string err;
    int64_t launches = 0;            // kernels launched by this context
    // solve history valid (phi_prev, phi_prev2, phi_obj)
    bool hist_ok = false;
    // learned guess (allocated on demand)
    void* unet = nullptr;
    // EM mode
    EMState em;
};

// ------------------------------------------------------------------ launchers
// particles.cu
void particles_alloc(Ctx& c, int s, int64_t cap);
void particles_append_aos(Ctx& c, int s, const void* host56, int64_t n);
int64_t particles_export_aos(Ctx& c, int s, void* host56, int64_t cap);
int64_t particles_export_raw(Ctx& c, int s, int32_t* cell, float* ox, float* oy, float* oz,
                             float* vx, float* vy, float* vz, int64_t cap);
void particles_generate_ambient(Ctx& c);
void particles_sort(Ctx& c);
int64_t brick_keys(const Ctx& c);
void launch_push(Ctx& c, bool vel, bool pos, bool dep);
void launch_deposit_all(Ctx& c);
void launch_em_velocity(Ctx& c);
void launch_em_position(Ctx& c);
void launch_em_move(Ctx& c, bool kick);
void launch_emit(Ctx& c, bool fused);
void launch_inject(Ctx& c, bool fused);
void launch_absorb(Ctx& c);
void launch_secondary(Ctx& c, bool fused);   // emission of the pending incidents' secondaries
void launch_energy(Ctx& c);
void sync_scalars(Ctx& c);
// fields.cu
void rho_zero(Ctx& c);
void rho_finalize(Ctx& c);
double species_rho_scale(const Ctx& c, int s);
void efield_update(Ctx& c);
void field_export(Ctx& c, int which, double* host);
double efield_energy(Ctx& c);
void phi_boundary(Ctx& c);
void phi_axpy(Ctx& c, double* dst, const double* a, const double* b, double sb);   // dst = a + sb * b over all nodes
void glue_copy(Ctx& c, double* a);
// em.cu (FDTD solver of the EM mode)
void em_alloc(Ctx& c);
void em_free(Ctx& c);
void em_fold_currents(Ctx& c);
void em_efield_from_phi(Ctx& c);   // RootGrid::updateEfield in the EM mode (start-up)
void em_update_efield(Ctx& c);     // RootGrid::updateEfieldFDTD
void em_update_bfield(Ctx& c);     // RootGrid::updateBfield
void em_reference_fields(Ctx& c);  // updateReferenceEfield + updateReferenceBfield
double em_efield_energy(Ctx& c);
double em_bfield_energy(Ctx& c);
const YeeArr* em_array(const Ctx& c, int which);   // FOPIS_FIELD_EX..BZ, or null
void em_field_export(Ctx& c, int which, double* host);
// multigrid.cu
void mg_setup(Ctx& c);
void mg_free(Ctx& c);
int mg_solve(Ctx& c, double tol, int max_cycles);
void mg_prepare(Ctx& c);   // records the solve graph (once the context's arrays exist)
// cmatrix.cu
void object_upload(Ctx& c, ObjectDev& o, const fopis_object_desc* d, int id);
void cmatrix_build(Ctx& c, int id);
void cmatrix_set(Ctx& c, int id, const double* hostC);
void redistribute(Ctx& c);
void conductor_start(Ctx& c);
void conductor_record(Ctx& c, const double* phi_first);
void objects_step_begin(Ctx& c);
void objects_step_end(Ctx& c);
// unet.cu (learned initial guess)
enum SolveKind { SOLVE_ONLY = 0, SOLVE_FIRST = 1, SOLVE_SECOND = 2 };
void unet_free(Ctx& c);
int unet_set_training(Ctx& c, int enable, double lr);
int unet_get_state(Ctx& c, double* loss, int64_t* steps);
int unet_get_policy(Ctx& c, double* plain, double* learned, int* active);
int unet_get_last(Ctx& c, double* warm_res, double* guess_res, double* ms_forward, double* ms_train);
bool unet_training(const Ctx& c);
int unet_before_solve(Ctx& c);       // 1 when phi keeps the learned guess
void unet_after_solve(Ctx& c, bool used, int cycles, bool converged);
int unet_eval(Ctx& c, const double* rho0, const double* phi1, const double* phi2, const double* phi_target,
              double* pred, float* grads, double* loss);
int unet_params(Ctx& c, float* get, const float* set, int64_t* count);
int unet_tensor(Ctx& c, int which, float* host, int64_t cap, int64_t* count);

}  // namespace fopis
