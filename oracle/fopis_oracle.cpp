// fopis_oracle.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// A CPU, FP64, OpenMP restatement of the FOPIS (TDPIC) electrostatic timestep for
// one MPI rank. It is the correctness oracle for libfopis_gpu.so and the timed
// CPU baseline ("port" kind). Only tests, the smoke check and the benchmark's CPU
// leg load it; nothing in the product links it.
//
// It keeps the reference's data layout and order of operations:
//   * the 56-byte array-of-structs Particle (include/particle.hpp:14-20);
//   * boost::multi_array<double,3> node fields with one glue layer, C order;
//   * RootGrid::mainLoopES phase order (src/Grid/RootGrid/RootGrid.cpp:82-143);
//   * the reference PSOR with its partial-sweep order, omega and pointwise
//     residual check (src/Grid/RootGrid/RootGridField.cpp:65-317);
//   * the single-rank periodic self-exchange semantics of src/MPI/Communicator.cpp
//     (node fold :497-574, field copy :265-343, partial phi :193-263).
// Deviations (each one also noted at its site):
//   * random numbers come from Philox4x32-10 (Salmon et al., SC'11) keyed by
//     (seed, species, step, face/node, index) instead of std::mt19937 +
//     std::normal_distribution, whose output is implementation-defined; the GPU
//     path uses the same keys, so both sides draw identical particle sets;
//   * migrated (wrapped) particles stay in place instead of being appended;
//     order only changes FP64 summation order in the deposit;
//   * a particle landing exactly on x == nx on a periodic axis wraps to 0 (the
//     reference keeps it and reads one node past the array);
//   * Eigen's MatrixXd::inverse (include/Spacecraft/Cmatrix.hpp:31-34) is replaced
//     by Gauss-Jordan elimination with partial pivoting;
//   * an extra "exact" Poisson solve (conjugate gradients to a tight tolerance)
//     serves as the converged FP64 reference for phi.
// Parity pins: Philox known-answer vectors, the reference's own Position header
// compiled by oracle/Makefile into oracle/_ref/pin_position, analytic checks
// (charge conservation, point-charge potential, Langmuir oscillation). The
// reference ships no golden vectors for this path (its test/ tree pins only AMR
// ID maps and does not compile).

#include "../include/fopis_gpu.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- Philox RNG
// Philox4x32-10 as published by Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of a 32x32->64 multiply
// bijection with a Weyl-sequence key schedule.
static inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
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

// Two uniforms in [0,1) with 53 random bits each from one Philox call.
struct U2 { double a, b; };
static inline U2 draw2(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    uint32_t c[4] = {c0, c1, c2, c3};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const uint64_t x = ((uint64_t)c[0] << 32) | c[1];
    const uint64_t y = ((uint64_t)c[2] << 32) | c[3];
    return {(double)(x >> 11) * 0x1p-53, (double)(y >> 11) * 0x1p-53};
}

// Box-Muller pair; 1-u keeps the logarithm's argument in (0,1].
static inline void box_muller(double u1, double u2, double& n0, double& n1) {
    const double r = std::sqrt(-2.0 * std::log(1.0 - u1));
    const double t = 2.0 * M_PI * u2;
    n0 = r * std::cos(t);
    n1 = r * std::sin(t);
}

enum : uint32_t { TAG_LOAD = 1u, TAG_INJECT = 2u, TAG_EMIT = 3u, TAG_SECONDARY = 4u };

// ---------------------------------------------------------------- containers
struct Arr3 {
    int cx = 0, cy = 0, cz = 0;
    std::vector<double> v;
    void resize(int a, int b, int c) { cx = a; cy = b; cz = c; v.assign((size_t)a * b * c, 0.0); }
    inline double& operator()(int i, int j, int k) { return v[((size_t)i * cy + j) * cz + k]; }
    inline double operator()(int i, int j, int k) const { return v[((size_t)i * cy + j) * cz + k]; }
    void zero() { std::fill(v.begin(), v.end(), 0.0); }
};

// boost::multi_array with index bases: the EM Yee arrays extended by the damping
// layers (RootGrid::initializeField, src/Grid/RootGrid/RootGridField.cpp:7-39).
struct ArrB {
    int lo[3] = {0, 0, 0}, n[3] = {0, 0, 0};
    std::vector<double> v;
    void resize(int l0, int u0, int l1, int u1, int l2, int u2) {   // half-open [l, u)
        lo[0] = l0; lo[1] = l1; lo[2] = l2;
        n[0] = u0 - l0; n[1] = u1 - l1; n[2] = u2 - l2;
        v.assign((size_t)n[0] * n[1] * n[2], 0.0);
    }
    inline double& operator()(int i, int j, int k) {
        return v[((size_t)(i - lo[0]) * n[1] + (j - lo[1])) * n[2] + (k - lo[2])];
    }
    inline double operator()(int i, int j, int k) const {
        return v[((size_t)(i - lo[0]) * n[1] + (j - lo[1])) * n[2] + (k - lo[2])];
    }
    int up(int a) const { return lo[a] + n[a]; }   // one past the last index
};

// include/particle.hpp:14-20 — 56 bytes.
struct Particle {
    double x, y, z;
    double vx, vy, vz;
    int typeId;
    int isValid;
};
static_assert(sizeof(Particle) == 56, "reference Particle is 56 bytes");

// include/position.hpp:13-69 — Position::setXYZ / setIJK / updateDelta.
struct Pos {
    int i, j, k;
    double x, y, z, dx1, dy1, dz1, dx2, dy2, dz2;
    void delta() {
        dx1 = x - (i - 1); dy1 = y - (j - 1); dz1 = z - (k - 1);
        dx2 = 1.0 - dx1; dy2 = 1.0 - dy1; dz2 = 1.0 - dz1;
    }
    void setXYZ(double a, double b, double c) {
        x = a; y = b; z = c;
        i = (int)std::floor(x) + 1; j = (int)std::floor(y) + 1; k = (int)std::floor(z) + 1;
        delta();
    }
    void setIJK(int a, int b, int c) {
        i = a; j = b; k = c;
        x = (double)(i - 1); y = (double)(j - 1); z = (double)(k - 1);
        delta();
    }
};
static inline Pos posXYZ(double x, double y, double z) { Pos p; p.setXYZ(x, y, z); return p; }

struct Object {
    int n_cmat = 0;
    std::vector<std::array<int, 3>> cmat;      // capacity_matrix_relation (cmat number -> glue node)
    std::vector<int> node_to_cmat;             // dense replacement of getCmatNumber's map scan
    std::vector<unsigned char> cell_map;       // object_cell_map [nx+1][ny+1][nz+1]
    std::vector<double> C;                     // capacity_matrix, row-major C(i,j) = C[i*n+j]
    double total_cmat_value = 0.0;
    std::vector<double> charge_map;            // [nsp][n]
    std::vector<double> tmp_charge_map;        // [nsp][n]
    std::vector<double> current;               // [nsp]
    double potential = 0.0, total_charge = 0.0;
    int is_potential_fixed = 0;
    double fixed_potential = 0.0, initial_potential_offset = 0.0;
    int emit_species = -1;
    int secondary_species = -1;                // SecondaryParticleType emitted by this body
    int dielectric = 0;                        // surface_type "dielectric"
    std::vector<double> capacitance;           // capacitance_map [n]
    bool has_C = false;
};

// IncidentInfo_t (src/Spacecraft/Incident.cpp) plus the object it hit.
struct Incident {
    int obj, s, axis;
    double trem, x, y, z, vx, vy, vz;
};

struct Ctx {
    fopis_params p;
    int nx, ny, nz;              // cell_x.. (single rank: equal to Environment::nx)
    int cx, cy, cz;              // nx+2 ..
    bool notb[6];                // Environment::isNotBoundary(axis, side) for x-,x+,y-,y+,z-,z+
    int nsp;
    std::vector<std::vector<Particle>> particles;
    std::vector<Arr3> rho;       // rho[0] total, rho[1+s]
    Arr3 phi, poisson_error, ex, ey, ez, exref, eyref, ezref;
    std::vector<Object> objects;
    std::vector<Incident> incidents;            // Spacecraft::incident_events of all objects
    std::vector<std::vector<Incident>> incidents_by_species;   // filled per species in update_rho
    std::vector<std::array<double, 6>> inject_residual;
    int64_t timestep = 1;        // Environment::timestep starts at 1 (Initialize.cpp:161)
    // solver
    int solver_mode = 0;         // 0 reference PSOR, 1 exact CG
    int max_post_loop = 1000;    // Options::maximum_poisson_post_loop
    double exact_tol = 1e-13;
    int last_iterations = 0;
    double last_residual = 0.0;
    int64_t injected_step = 0, emitted_step = 0, absorbed_step = 0;
    // EM mode (Environment::solver_type == "EM"): Yee E and B with damping layers,
    // edge currents, nodal B
    bool em = false;
    int L[3] = {1, 1, 1};        // Environment::damping_length (L_dx, L_dy, L_dz)
    ArrB fex, fey, fez, fbx, fby, fbz;
    Arr3 jx, jy, jz, bxref, byref, bzref;
    char err[256] = {0};
};

static inline bool isBoundary(const Ctx& c, int axis, int side) { return !c.notb[2 * axis + side]; }

// Environment::isValidCellPosition (src/Misc/Environment.cpp:287-293).
static inline bool validCell(const Ctx& c, int i, int j, int k) {
    return i >= 0 && i < c.nx + 1 && j >= 0 && j < c.ny + 1 && k >= 0 && k < c.nz + 1;
}
static inline size_t cellIndex(const Ctx& c, int i, int j, int k) {
    return ((size_t)i * (c.ny + 1) + j) * (c.nz + 1) + k;
}
static inline size_t nodeIndex(const Ctx& c, int i, int j, int k) {
    return ((size_t)i * c.cy + j) * c.cz + k;
}

// ---------------------------------------------------------------- set-up
static void init_ctx(Ctx& c, const fopis_params* p) {
    c.p = *p;
    c.nx = p->nx; c.ny = p->ny; c.nz = p->nz;
    c.cx = c.nx + 2; c.cy = c.ny + 2; c.cz = c.nz + 2;
    for (int s = 0; s < 6; ++s) c.notb[s] = (p->boundary[s] == 'P');
    c.nsp = p->nspecies;
    c.particles.assign(c.nsp, {});
    c.rho.resize(c.nsp + 1);
    for (auto& r : c.rho) r.resize(c.cx, c.cy, c.cz);
    c.phi.resize(c.cx, c.cy, c.cz);
    c.poisson_error.resize(c.cx, c.cy, c.cz);
    c.ex.resize(c.cx - 1, c.cy, c.cz);
    c.ey.resize(c.cx, c.cy - 1, c.cz);
    c.ez.resize(c.cx, c.cy, c.cz - 1);
    c.exref.resize(c.cx, c.cy, c.cz);
    c.eyref.resize(c.cx, c.cy, c.cz);
    c.ezref.resize(c.cx, c.cy, c.cz);
    c.inject_residual.assign(c.nsp, {0, 0, 0, 0, 0, 0});
    c.em = p->solver == FOPIS_SOLVER_EM;
    if (c.em) {
        // RootGrid::initializeField (RootGridField.cpp:7-39): damping length = node count per
        // axis, the arrays reach that far beyond every non-periodic face.
        c.L[0] = c.nx; c.L[1] = c.ny; c.L[2] = c.nz;
        const int cc[3] = {c.cx, c.cy, c.cz};
        int lo[3], up[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = isBoundary(c, a, 0) ? -c.L[a] : 0;
            up[a] = isBoundary(c, a, 1) ? cc[a] + c.L[a] : cc[a];
        }
        c.fex.resize(lo[0], up[0] - 1, lo[1], up[1], lo[2], up[2]);
        c.fey.resize(lo[0], up[0], lo[1], up[1] - 1, lo[2], up[2]);
        c.fez.resize(lo[0], up[0], lo[1], up[1], lo[2], up[2] - 1);
        c.fbx.resize(lo[0], up[0], lo[1], up[1] - 1, lo[2], up[2] - 1);
        c.fby.resize(lo[0], up[0] - 1, lo[1], up[1], lo[2], up[2] - 1);
        c.fbz.resize(lo[0], up[0] - 1, lo[1], up[1] - 1, lo[2], up[2]);
        // Grid::initializeField (src/Grid/Grid.cpp:170-194): edge currents, nodal B
        c.jx.resize(c.cx - 1, c.cy, c.cz);
        c.jy.resize(c.cx, c.cy - 1, c.cz);
        c.jz.resize(c.cx, c.cy, c.cz - 1);
        c.bxref.resize(c.cx, c.cy, c.cz);
        c.byref.resize(c.cx, c.cy, c.cz);
        c.bzref.resize(c.cx, c.cy, c.cz);
    }
}

// ---------------------------------------------------------------- halo semantics
// Communicator::sendRecvScalarX/Y/Z with prev == next == self and glue size 2
// (src/MPI/Communicator.cpp:497-574): node 0 and node n become the sum of both,
// node 1 and node n+1 likewise. Applied only on periodic axes
// (MPIw::Environment::sendRecvNodeScalar, src/MPI/Environment.cpp:53-72).
static void fold_node_scalar(const Ctx& c, Arr3& a) {
    const int X = a.cx, Y = a.cy, Z = a.cz;
    if (c.notb[0]) {
        for (int j = 0; j < Y; ++j) for (int k = 0; k < Z; ++k) {
            double s0 = a(0, j, k) + a(X - 2, j, k), s1 = a(1, j, k) + a(X - 1, j, k);
            a(0, j, k) = s0; a(X - 2, j, k) = s0; a(1, j, k) = s1; a(X - 1, j, k) = s1;
        }
    }
    if (c.notb[2]) {
        for (int i = 0; i < X; ++i) for (int k = 0; k < Z; ++k) {
            double s0 = a(i, 0, k) + a(i, Y - 2, k), s1 = a(i, 1, k) + a(i, Y - 1, k);
            a(i, 0, k) = s0; a(i, Y - 2, k) = s0; a(i, 1, k) = s1; a(i, Y - 1, k) = s1;
        }
    }
    if (c.notb[4]) {
        for (int i = 0; i < X; ++i) for (int j = 0; j < Y; ++j) {
            double s0 = a(i, j, 0) + a(i, j, Z - 2), s1 = a(i, j, 1) + a(i, j, Z - 1);
            a(i, j, 0) = s0; a(i, j, Z - 2) = s0; a(i, j, 1) = s1; a(i, j, Z - 1) = s1;
        }
    }
}

// Communicator::sendRecvFieldX/Y/Z self branch (src/MPI/Communicator.cpp:290-299):
// node 0 <- node n, node n+1 <- node 1, per periodic axis, x then y then z.
static void copy_field_glue(const Ctx& c, Arr3& a) {
    const int X = a.cx, Y = a.cy, Z = a.cz;
    if (c.notb[0])
        for (int j = 0; j < Y; ++j) for (int k = 0; k < Z; ++k) {
            double lo = a(1, j, k);
            a(0, j, k) = a(X - 2, j, k); a(X - 1, j, k) = lo;
        }
    if (c.notb[2])
        for (int i = 0; i < X; ++i) for (int k = 0; k < Z; ++k) {
            double lo = a(i, 1, k);
            a(i, 0, k) = a(i, Y - 2, k); a(i, Y - 1, k) = lo;
        }
    if (c.notb[4])
        for (int i = 0; i < X; ++i) for (int j = 0; j < Y; ++j) {
            double lo = a(i, j, 1);
            a(i, j, 0) = a(i, j, Z - 2); a(i, j, Z - 1) = lo;
        }
}

// MPIw::Environment::sendRecvPartialPhi self branch (src/MPI/Environment.cpp:174-208,
// Communicator.cpp:193-263): a plane segment at index 1 is copied to index n+1,
// one at index n to index 0, only when that side is periodic.
static void partial_phi(Ctx& c, int ib, int ie, int jb, int je, int kb, int ke) {
    Arr3& phi = c.phi;
    if (ib == ie) {
        const bool low = (ib == 1);
        if (low ? c.notb[0] : c.notb[1]) {
            const int dst = low ? c.cx - 1 : 0;
            for (int j = jb; j <= je; ++j) for (int k = kb; k <= ke; ++k) phi(dst, j, k) = phi(ib, j, k);
        }
    } else if (jb == je) {
        const bool low = (jb == 1);
        if (low ? c.notb[2] : c.notb[3]) {
            const int dst = low ? c.cy - 1 : 0;
            for (int i = ib; i <= ie; ++i) for (int k = kb; k <= ke; ++k) phi(i, dst, k) = phi(i, jb, k);
        }
    } else if (kb == ke) {
        const bool low = (kb == 1);
        if (low ? c.notb[4] : c.notb[5]) {
            const int dst = low ? c.cz - 1 : 0;
            for (int i = ib; i <= ie; ++i) for (int j = jb; j <= je; ++j) phi(i, j, dst) = phi(i, j, kb);
        }
    }
}

// ---------------------------------------------------------------- particle phases
// Grid::updateParticleVelocityES (src/Grid/GridParticleTreatmentES.cpp:13-88).
static void update_velocity(Ctx& c) {
    const double bx = c.p.static_bfield[0], by = c.p.static_bfield[1], bz = c.p.static_bfield[2];
    const double time_factor = 1.0;  // 1 / 2^level, level 0
    for (int pid = 0; pid < c.nsp; ++pid) {
        const double qm = 0.5 * c.p.species[pid].charge / c.p.species[pid].mass;
        auto& parray = c.particles[pid];
        const long n = (long)parray.size();
        const Arr3& exr = c.exref; const Arr3& eyr = c.eyref; const Arr3& ezr = c.ezref;
#pragma omp parallel for schedule(static)
        for (long pn = 0; pn < n; ++pn) {
            Particle& p = parray[pn];
            if (!p.isValid) continue;
            Pos pos = posXYZ(p.x, p.y, p.z);
            const int i = pos.i, j = pos.j, k = pos.k;
            const double v1 = qm * pos.dx2 * pos.dy2 * pos.dz2, v2 = qm * pos.dx1 * pos.dy2 * pos.dz2;
            const double v3 = qm * pos.dx2 * pos.dy1 * pos.dz2, v4 = qm * pos.dx1 * pos.dy1 * pos.dz2;
            const double v5 = qm * pos.dx2 * pos.dy2 * pos.dz1, v6 = qm * pos.dx1 * pos.dy2 * pos.dz1;
            const double v7 = qm * pos.dx2 * pos.dy1 * pos.dz1, v8 = qm * pos.dx1 * pos.dy1 * pos.dz1;
            auto g = [&](const Arr3& e) {
                return v1 * e(i, j, k) + v2 * e(i + 1, j, k) + v3 * e(i, j + 1, k) + v4 * e(i + 1, j + 1, k) +
                       v5 * e(i, j, k + 1) + v6 * e(i + 1, j, k + 1) + v7 * e(i, j + 1, k + 1) +
                       v8 * e(i + 1, j + 1, k + 1);
            };
            const double exv = g(exr), eyv = g(eyr), ezv = g(ezr);
            const double boris = 2.0 / (1.0 + (bx * bx + by * by + bz * bz));
            const double vx1 = p.vx + exv, vy1 = p.vy + eyv, vz1 = p.vz + ezv;
            const double vxt = vx1 + vy1 * bz - vz1 * by;
            const double vyt = vy1 + vz1 * bx - vx1 * bz;
            const double vzt = vz1 + vx1 * by - vy1 * bx;
            p.vx = vx1 + (exv + boris * (vyt * bz - vzt * by)) * time_factor;
            p.vy = vy1 + (eyv + boris * (vzt * bx - vxt * bz)) * time_factor;
            p.vz = vz1 + (ezv + boris * (vxt * by - vyt * bx)) * time_factor;
        }
    }
}

// RootGrid::checkX/Y/ZBoundary (include/grid.hpp:309-395) followed by the
// single-rank migration of updateParticlePositionES (:115-177): on a periodic
// axis a coordinate beyond -1 gains sl, one beyond sl loses sl (here also one
// exactly at sl, see the header); on a D/N axis x < 0 or x > sl-1 invalidates.
static inline void boundary_axis(const Ctx& c, double& x, int& valid, int axis, double sl) {
    if (x < 0.0) {
        if (c.notb[2 * axis]) { if (x < -1.0) x += sl; }
        else valid = 0;
    } else if (x > sl - 1.0) {
        if (c.notb[2 * axis + 1]) { if (x >= sl) x -= sl; }
        else valid = 0;
    }
}

// RootGrid::updateParticlePositionES (src/Grid/GridParticleTreatmentES.cpp:90-181).
static void update_position(Ctx& c) {
    const double slx = c.nx, sly = c.ny, slz = c.nz;
    for (int pid = 0; pid < c.nsp; ++pid) {
        auto& parray = c.particles[pid];
        const long n = (long)parray.size();
#pragma omp parallel for schedule(static)
        for (long pn = 0; pn < n; ++pn) {
            Particle& p = parray[pn];
            if (!p.isValid) continue;
            p.x += p.vx; p.y += p.vy; p.z += p.vz;  // Particle::updatePosition
            boundary_axis(c, p.x, p.isValid, 0, slx);
            boundary_axis(c, p.y, p.isValid, 1, sly);
            boundary_axis(c, p.z, p.isValid, 2, slz);
        }
    }
}

// ---------------------------------------------------------------- conductors
static inline bool cell_in(const Ctx& c, const Object& o, int i, int j, int k) {
    return o.cell_map[cellIndex(c, i, j, k)] != 0;
}
// Spacecraft::isContaining (Spacecraft.cpp:320-332).
static inline bool isContaining(const Ctx& c, const Object& o, const Pos& pos) {
    if (!validCell(c, pos.i, pos.j, pos.k)) return false;
    return cell_in(c, o, pos.i, pos.j, pos.k);
}
// Spacecraft::getCmatNumber (Spacecraft.cpp:210-235); -1 where the reference throws.
static inline int cmatNumber(const Ctx& c, const Object& o, int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= c.cx || j >= c.cy || k >= c.cz) return -1;
    return o.node_to_cmat[nodeIndex(c, i, j, k)];
}
static inline bool isCmatNode(const Ctx& c, const Object& o, int i, int j, int k) {
    return cmatNumber(c, o, i, j, k) >= 0;
}
// Spacecraft::isX/Y/Zsurface{Minus,Plus} (Spacecraft.cpp:334-356).
static inline bool xMinus(const Ctx& c, const Object& o, int i, int j, int k) { return cell_in(c, o, i, j, k) && !cell_in(c, o, i - 1, j, k); }
static inline bool xPlus(const Ctx& c, const Object& o, int i, int j, int k) { return !cell_in(c, o, i, j, k) && cell_in(c, o, i - 1, j, k); }
static inline bool yMinus(const Ctx& c, const Object& o, int i, int j, int k) { return cell_in(c, o, i, j, k) && !cell_in(c, o, i, j - 1, k); }
static inline bool yPlus(const Ctx& c, const Object& o, int i, int j, int k) { return !cell_in(c, o, i, j, k) && cell_in(c, o, i, j - 1, k); }
static inline bool zMinus(const Ctx& c, const Object& o, int i, int j, int k) { return cell_in(c, o, i, j, k) && !cell_in(c, o, i, j, k - 1); }
static inline bool zPlus(const Ctx& c, const Object& o, int i, int j, int k) { return !cell_in(c, o, i, j, k) && cell_in(c, o, i, j, k - 1); }

// Spacecraft::isX/Y/ZsurfacePoint (Spacecraft.cpp:462-506).
static bool isXsurfacePoint(const Ctx& c, const Object& o, const Pos& pos, int sign) {
    if (pos.dx1 >= 1e-10) return false;
    if (validCell(c, pos.i, pos.j, pos.k) && validCell(c, pos.i - 1, pos.j, pos.k))
        return sign > 0 ? xMinus(c, o, pos.i, pos.j, pos.k) : xPlus(c, o, pos.i, pos.j, pos.k);
    return isCmatNode(c, o, pos.i, pos.j, pos.k) && isCmatNode(c, o, pos.i, pos.j + 1, pos.k) &&
           isCmatNode(c, o, pos.i, pos.j, pos.k + 1) && isCmatNode(c, o, pos.i, pos.j + 1, pos.k + 1);
}
static bool isYsurfacePoint(const Ctx& c, const Object& o, const Pos& pos, int sign) {
    if (pos.dy1 >= 1e-10) return false;
    if (validCell(c, pos.i, pos.j, pos.k) && validCell(c, pos.i, pos.j - 1, pos.k))
        return sign > 0 ? yMinus(c, o, pos.i, pos.j, pos.k) : yPlus(c, o, pos.i, pos.j, pos.k);
    return isCmatNode(c, o, pos.i, pos.j, pos.k) && isCmatNode(c, o, pos.i + 1, pos.j, pos.k) &&
           isCmatNode(c, o, pos.i, pos.j, pos.k + 1) && isCmatNode(c, o, pos.i + 1, pos.j, pos.k + 1);
}
static bool isZsurfacePoint(const Ctx& c, const Object& o, const Pos& pos, int sign) {
    if (pos.dz1 >= 1e-10) return false;
    if (validCell(c, pos.i, pos.j, pos.k) && validCell(c, pos.i, pos.j, pos.k - 1))
        return sign > 0 ? zMinus(c, o, pos.i, pos.j, pos.k) : zPlus(c, o, pos.i, pos.j, pos.k);
    return isCmatNode(c, o, pos.i, pos.j, pos.k) && isCmatNode(c, o, pos.i + 1, pos.j, pos.k) &&
           isCmatNode(c, o, pos.i, pos.j + 1, pos.k) && isCmatNode(c, o, pos.i + 1, pos.j + 1, pos.k);
}

// Particle::get{X,Y,Z}MoveRatio (src/Particle/particle.cpp:46-80).
static inline double moveRatio(double d1, double d2, double v) {
    if (v == 0.0) return 0.0;
    return v > 0.0 ? d1 / std::fabs(v) : d2 / std::fabs(v);
}

// Particle::computeCrossPoints (src/Particle/particle.cpp:82-204), including the
// `mvx <= mvx` comparison of the xz case (:175), which always puts x first.
static int computeCrossPoints(const Particle& p, Pos out[3]) {
    const Pos pos = posXYZ(p.x, p.y, p.z);
    const Pos old = posXYZ(p.x - p.vx, p.y - p.vy, p.z - p.vz);
    const double mvx = 1.0 - moveRatio(pos.dx1, pos.dx2, p.vx);
    const double mvy = 1.0 - moveRatio(pos.dy1, pos.dy2, p.vy);
    const double mvz = 1.0 - moveRatio(pos.dz1, pos.dz2, p.vz);
    int count = 0;
    Pos xc, yc, zc;
    const bool mx = (pos.i != old.i), my = (pos.j != old.j), mz = (pos.k != old.k);
    if (mx) { xc.setXYZ(p.vx > 0.0 ? std::ceil(old.x) : std::floor(old.x), old.y + p.vy * mvx, old.z + p.vz * mvx); ++count; }
    if (my) { yc.setXYZ(old.x + p.vx * mvy, p.vy > 0.0 ? std::ceil(old.y) : std::floor(old.y), old.z + p.vz * mvy); ++count; }
    if (mz) { zc.setXYZ(old.x + p.vx * mvz, old.y + p.vy * mvz, p.vz > 0.0 ? std::ceil(old.z) : std::floor(old.z)); ++count; }
    int n = 0;
    if (count == 3) {
        if (mvx <= mvy) {
            if (mvx <= mvz) {
                out[n++] = xc;
                if (mvy <= mvz) { out[n++] = yc; out[n++] = zc; } else { out[n++] = zc; out[n++] = yc; }
            } else { out[n++] = zc; out[n++] = xc; out[n++] = yc; }
        } else {
            if (mvy <= mvz) {
                out[n++] = yc;
                if (mvx <= mvz) { out[n++] = xc; out[n++] = zc; } else { out[n++] = zc; out[n++] = xc; }
            } else { out[n++] = zc; out[n++] = yc; out[n++] = xc; }
        }
    } else if (count == 2) {
        if (mx) {
            if (my) { if (mvx <= mvy) { out[n++] = xc; out[n++] = yc; } else { out[n++] = yc; out[n++] = xc; } }
            else { out[n++] = xc; out[n++] = zc; }  // reference compares mvx <= mvx here
        } else {
            if (mvy <= mvz) { out[n++] = yc; out[n++] = zc; } else { out[n++] = zc; out[n++] = yc; }
        }
    } else if (count == 1) {
        out[n++] = mx ? xc : (my ? yc : zc);
    }
    return n;
}

// Spacecraft::distributeInnerParticleChargeTo{X,Y,Z}surface (Spacecraft.cpp:594-613)
// and subtractChargeOfParticleFrom{X,Y,Z}surface (:945-970); sign = +1 or -1.
// Returns false where getCmatNumber would throw.
static bool surface_charge(const Ctx& c, Object& o, int axis, const Pos& pos, int id, double q) {
    int n[4]; double w[4];
    if (axis == 0) {
        n[0] = cmatNumber(c, o, pos.i, pos.j, pos.k);         w[0] = pos.dy2 * pos.dz2;
        n[1] = cmatNumber(c, o, pos.i, pos.j + 1, pos.k);     w[1] = pos.dy1 * pos.dz2;
        n[2] = cmatNumber(c, o, pos.i, pos.j, pos.k + 1);     w[2] = pos.dy2 * pos.dz1;
        n[3] = cmatNumber(c, o, pos.i, pos.j + 1, pos.k + 1); w[3] = pos.dy1 * pos.dz1;
    } else if (axis == 1) {
        n[0] = cmatNumber(c, o, pos.i, pos.j, pos.k);         w[0] = pos.dx2 * pos.dz2;
        n[1] = cmatNumber(c, o, pos.i + 1, pos.j, pos.k);     w[1] = pos.dx1 * pos.dz2;
        n[2] = cmatNumber(c, o, pos.i, pos.j, pos.k + 1);     w[2] = pos.dx2 * pos.dz1;
        n[3] = cmatNumber(c, o, pos.i + 1, pos.j, pos.k + 1); w[3] = pos.dx1 * pos.dz1;
    } else {
        n[0] = cmatNumber(c, o, pos.i, pos.j, pos.k);         w[0] = pos.dx2 * pos.dy2;
        n[1] = cmatNumber(c, o, pos.i + 1, pos.j, pos.k);     w[1] = pos.dx1 * pos.dy2;
        n[2] = cmatNumber(c, o, pos.i, pos.j + 1, pos.k);     w[2] = pos.dx2 * pos.dy1;
        n[3] = cmatNumber(c, o, pos.i + 1, pos.j + 1, pos.k); w[3] = pos.dx1 * pos.dy1;
    }
    for (int t = 0; t < 4; ++t) if (n[t] < 0) return false;
    for (int t = 0; t < 4; ++t) o.tmp_charge_map[(size_t)id * o.n_cmat + n[t]] += q * w[t];
    return true;
}

// The first of a particle's crossing points that is a body face on an axis
// other than `skip` (-1: any), in the order of Spacecraft::distribute
// InnerParticleCharge (Spacecraft.cpp:512-592) and, with skip, of
// distributeInnerParticleChargeForSecondary (SecondaryEmission.cpp:35-110).
static int first_face(const Ctx& c, const Object& o, const Particle& p, int skip, Pos& hit) {
    const int isign = (p.vx > 0.0) ? 1 : -1, jsign = (p.vy > 0.0) ? 1 : -1, ksign = (p.vz > 0.0) ? 1 : -1;
    Pos cps[3];
    const int ncp = computeCrossPoints(p, cps);
    for (int t = 0; t < ncp; ++t) {
        const Pos& cp = cps[t];
        if (skip != 0 && isXsurfacePoint(c, o, cp, isign)) { hit = cp; return 0; }
        if (skip != 1 && isYsurfacePoint(c, o, cp, jsign)) { hit = cp; return 1; }
        if (skip != 2 && isZsurfacePoint(c, o, cp, ksign)) { hit = cp; return 2; }
    }
    return -1;
}

// Spacecraft::distributeInnerParticleCharge (Spacecraft.cpp:512-592). A body that
// emits secondaries keeps the hit as an incident event (its move ratio along the
// face axis is the remaining time, SecondaryEmission.cpp:14-33). Returns 1 if
// absorbed.
static int absorb(Ctx& c, int oi, Particle& p, int& bad, std::vector<Incident>* inc) {
    Object& o = c.objects[oi];
    const Pos pos = posXYZ(p.x, p.y, p.z);
    if (!isContaining(c, o, pos)) return 0;
    const int id = p.typeId;
    const double q = c.p.species[id].charge * c.p.species[id].size;
    Pos cp;
    const int ax = first_face(c, o, p, -1, cp);
    if (ax >= 0) {
        if (!surface_charge(c, o, ax, cp, id, q)) bad = 1;
        if (o.secondary_species >= 0 && inc) {
            const double d1[3] = {pos.dx1, pos.dy1, pos.dz1}, d2[3] = {pos.dx2, pos.dy2, pos.dz2};
            const double v[3] = {p.vx, p.vy, p.vz};
            inc->push_back(Incident{oi, id, ax, moveRatio(d1[ax], d2[ax], v[ax]), cp.x, cp.y, cp.z, p.vx, p.vy, p.vz});
        }
    }
    o.current[id] += q;
    p.isValid = 0;
    return 1;
}

// Spacecraft::sumWholeCharge (Spacecraft.cpp:615-626).
static void sum_whole_charge(Ctx& c, Object& o) {
    for (size_t t = 0; t < o.charge_map.size(); ++t) { o.charge_map[t] += o.tmp_charge_map[t]; o.tmp_charge_map[t] = 0.0; }
}

// Spacecraft::getTotalCharge (Spacecraft.cpp:248-259).
static double total_charge(const Ctx& c, const Object& o) {
    double q = 0.0;
    for (int m = 0; m < o.n_cmat; ++m)
        for (int s = 0; s < c.nsp; ++s) q += o.charge_map[(size_t)s * o.n_cmat + m];
    return q;
}

// Spacecraft::redistributeChargeForDielectric (Spacecraft.cpp:641-706): a node j
// with capacitance c_j > 0 enters with phi_j - Q_j / c_j, Q_j its charge summed
// over the species, in both the potential and delta rho. d holds V - phi_j on
// entry; the potential and d are recomputed here.
static void redistribute_dielectric(Ctx& c, Object& o, std::vector<double>& d) {
    const int n = o.n_cmat;
    std::vector<double> pe(n);
    for (int j = 0; j < n; ++j) {
        const auto& nd = o.cmat[j];
        pe[j] = c.phi(nd[0], nd[1], nd[2]);
        if (o.capacitance[j] > 0.0) {
            double qn = 0.0;
            for (int pid = 0; pid < c.nsp; ++pid) qn += o.charge_map[(size_t)pid * n + j];
            pe[j] -= qn / o.capacitance[j];
        }
    }
    double ctp = 0.0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) ctp += o.C[(size_t)i * n + j] * pe[j];
    o.potential = o.is_potential_fixed ? o.fixed_potential : (ctp + o.total_charge) / o.total_cmat_value;
    for (int j = 0; j < n; ++j) d[j] = o.potential - pe[j];
}

// Spacecraft::redistributeChargeForPerfectConductor (Spacecraft.cpp:708-758).
static void redistribute(Ctx& c, Object& o) {
    o.total_charge = total_charge(c, o);
    const int n = o.n_cmat;
    double ctp = 0.0;
    for (int j = 0; j < n; ++j) {
        const auto& nd = o.cmat[j];
        const double ph = c.phi(nd[0], nd[1], nd[2]);
        for (int i = 0; i < n; ++i) ctp += o.C[(size_t)i * n + j] * ph;
    }
    o.potential = o.is_potential_fixed ? o.fixed_potential : (ctp + o.total_charge) / o.total_cmat_value;
    std::vector<double> d(n);
    for (int j = 0; j < n; ++j) { const auto& nd = o.cmat[j]; d[j] = o.potential - c.phi(nd[0], nd[1], nd[2]); }
    if (o.dielectric) redistribute_dielectric(c, o, d);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double dr = 0.0;
        for (int j = 0; j < n; ++j) dr += o.C[(size_t)i * n + j] * d[j];
        const auto& nd = o.cmat[i];
        c.rho[0](nd[0], nd[1], nd[2]) += dr;
    }
}

// ---------------------------------------------------------------- Poisson
// RootGrid::doSORPartial (src/Grid/RootGrid/RootGridField.cpp:216-264).
static void sor_partial(Ctx& c, double omega, double rho_coeff, int ib, int ie, int jb, int je, int kb, int ke,
                        bool parallel) {
    Arr3& phi = c.phi; const Arr3& rho = c.rho[0];
    int ibt = 0, iet = 0, jbt = 0, jet = 0, kbt = 0, ket = 0;
    if (isBoundary(c, 0, 0) && ib == 1) ibt = 1;
    if (isBoundary(c, 0, 1) && ie == c.cx - 2) iet = -1;
    if (isBoundary(c, 1, 0) && jb == 1) jbt = 1;
    if (isBoundary(c, 1, 1) && je == c.cy - 2) jet = -1;
    if (isBoundary(c, 2, 0) && kb == 1) kbt = 1;
    if (isBoundary(c, 2, 1) && ke == c.cz - 2) ket = -1;
    const int i0 = ib + ibt, i1 = ie + iet, j0 = jb + jbt, j1 = je + jet, k0 = kb + kbt, k1 = ke + ket;
    const int isize = i1 - i0 + 1;
    auto upd = [&](int i, int j, int k) {
        phi(i, j, k) = (1.0 - omega) * phi(i, j, k) +
                       omega * (phi(i + 1, j, k) + phi(i - 1, j, k) + phi(i, j + 1, k) + phi(i, j - 1, k) +
                                phi(i, j, k + 1) + phi(i, j, k - 1) + rho_coeff * rho(i, j, k)) / 6.0;
    };
    if (isize > 2) {
        // red-black over i planes: odd offsets then even offsets
        for (int color = 0; color < 2; ++color) {
            const int nplanes = (i1 - (i0 + color)) >= 0 ? (i1 - (i0 + color)) / 2 + 1 : 0;
#pragma omp parallel for schedule(static) if (parallel)
            for (int t = 0; t < nplanes; ++t) {
                const int i = i0 + color + 2 * t;
                for (int j = j0; j <= j1; ++j)
                    for (int k = k0; k <= k1; ++k) upd(i, j, k);
            }
        }
    } else {
        for (int i = i0; i <= i1; ++i)
            for (int j = j0; j <= j1; ++j)
                for (int k = k0; k <= k1; ++k) upd(i, j, k);
    }
}

// RootGrid::doPSOR (src/Grid/RootGrid/RootGridField.cpp:105-214).
static void do_psor(Ctx& c) {
    const int minimum_radius = std::min({c.nx, c.ny, c.nz});
    const double omega = 2.0 / (1.0 + std::sin(M_PI / minimum_radius));
    const double rho_coeff = 1.0 / c.p.eps0;  // dx^2 / eps0 with dx = 1
    const int X = c.cx, Y = c.cy, Z = c.cz;
    int ib = 1, ie = 1, jb = 1, je = 1, kb = 1, ke = 1;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib, ie, jb, je, kb, ke);
    ib = 2; ie = X - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib - 1, ie + 1, jb, je, kb, ke);
    ib = 1; ie = 1; jb = 2; je = Y - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib, ie, jb, je + 1, kb, ke);
    ib = 2; ie = X - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib - 1, ie + 1, jb - 1, je + 1, kb, ke);
    ib = 1; ie = 1; jb = 1; je = 1; kb = 2; ke = Z - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib, ie, jb, je, kb, ke + 1);
    ib = 2; ie = X - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib - 1, ie + 1, jb, je, kb, ke + 1);
    ib = 1; ie = 1; jb = 2; je = Y - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, false);
    partial_phi(c, ib, ie, jb, je + 1, kb, ke + 1);
    ib = 2; ie = X - 2;
    sor_partial(c, omega, rho_coeff, ib, ie, jb, je, kb, ke, true);  // the one #pragma omp parallel region
    ib = 0; ie = X - 1; jb = 0; je = Y - 1; kb = Z - 2; ke = Z - 2;
    partial_phi(c, ib, ie, jb, je, kb, ke);
    jb = Y - 2; je = Y - 2; kb = 0; ke = Z - 1;
    partial_phi(c, ib, ie, jb, je, kb, ke);
    ib = X - 2; ie = X - 2; jb = 0; je = Y - 1;
    partial_phi(c, ib, ie, jb, je, kb, ke);
}

// RootGrid::checkPhiResidual (src/Grid/RootGrid/RootGridField.cpp:267-317).
static double check_phi_residual(Ctx& c) {
    double residual = 0.0;
    const Arr3& phi = c.phi; const Arr3& rho = c.rho[0];
    const double eps = c.p.eps0;
    const int X = c.cx, Y = c.cy, Z = c.cz;
#pragma omp parallel for reduction(max : residual) schedule(static)
    for (int i = 1; i < X - 1; ++i) {
        if (!((i != 1 || c.notb[0]) && (i != X - 2 || c.notb[1]))) continue;
        for (int j = 1; j < Y - 1; ++j) {
            if (!((j != 1 || c.notb[2]) && (j != Y - 2 || c.notb[3]))) continue;
            for (int k = 1; k < Z - 1; ++k) {
                if (!((k != 1 || c.notb[4]) && (k != Z - 2 || c.notb[5]))) continue;
                const double src = rho(i, j, k) / eps;
                if (std::fabs(src) > 0.0) {
                    const double op = phi(i - 1, j, k) + phi(i + 1, j, k) + phi(i, j - 1, k) + phi(i, j + 1, k) +
                                      phi(i, j, k - 1) + phi(i, j, k + 1) - 6.0 * phi(i, j, k);
                    const double r = std::fabs((op + src) / src);
                    if (r > residual) residual = r;
                }
            }
        }
    }
    return residual;
}

// Field::setBoundaryConditionPhi / setNeumannPhi / setDirichletPhi (src/Grid/Field.cpp:10-96).
static void set_boundary_phi(Ctx& c) {
    Arr3& phi = c.phi;
    const int X = c.cx, Y = c.cy, Z = c.cz;
    for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side) {
            const char b = c.p.boundary[2 * axis + side];
            if (b == 'P') continue;
            const int maxi = axis == 0 ? X : (axis == 1 ? Y : Z);
            const int bi = side == 0 ? 1 : maxi - 2;
            const int ni = side == 0 ? 2 : maxi - 3;
            if (axis == 0) {
                for (int k = 1; k < Z - 1; ++k) for (int j = 1; j < Y - 1; ++j) phi(bi, j, k) = (b == 'D') ? 0.0 : phi(ni, j, k);
            } else if (axis == 1) {
                for (int k = 1; k < Z - 1; ++k) for (int i = 1; i < X - 1; ++i) phi(i, bi, k) = (b == 'D') ? 0.0 : phi(i, ni, k);
            } else {
                for (int j = 1; j < Y - 1; ++j) for (int i = 1; i < X - 1; ++i) phi(i, j, bi) = (b == 'D') ? 0.0 : phi(i, j, ni);
            }
        }
}

// Unknown-node test shared by the exact solver: nodes the PSOR updates.
static inline bool is_unknown(const Ctx& c, int i, int j, int k) {
    auto ok = [&](int idx, int n2, int axis) {
        if (idx < 1 || idx > n2 - 2) return false;
        if (idx == 1 && isBoundary(c, axis, 0)) return false;
        if (idx == n2 - 2 && isBoundary(c, axis, 1)) return false;
        return true;
    };
    return ok(i, c.cx, 0) && ok(j, c.cy, 1) && ok(k, c.cz, 2);
}

// Converged FP64 reference solve: conjugate gradients on A = 6 - sum(neighbours)
// over the unknown nodes, boundary nodes held at their current values, periodic
// neighbours wrapped, mean of the right-hand side removed when every axis is
// periodic; stops at ||r||2 <= tol ||f||2.
static void exact_solve(Ctx& c) {
    const int X = c.cx, Y = c.cy, Z = c.cz;
    const size_t N = (size_t)X * Y * Z;
    std::vector<unsigned char> unk(N, 0);
    for (int i = 0; i < X; ++i) for (int j = 0; j < Y; ++j) for (int k = 0; k < Z; ++k)
        unk[nodeIndex(c, i, j, k)] = is_unknown(c, i, j, k);
    const bool allp = c.notb[0] && c.notb[2] && c.notb[4];
    auto wrap = [&](int idx, int n2, int axis) {
        if (c.notb[2 * axis]) { if (idx == 0) return n2 - 2; if (idx == n2 - 1) return 1; }
        return idx;
    };
    std::vector<double> f(N, 0.0), x(N, 0.0), r(N, 0.0), pp(N, 0.0), Ap(N, 0.0);
    for (size_t t = 0; t < N; ++t) x[t] = c.phi.v[t];
    // Ap = A * v restricted to unknowns, using full field v (boundary values included)
    auto apply = [&](const std::vector<double>& v, std::vector<double>& out, bool with_fixed) {
#pragma omp parallel for schedule(static)
        for (int i = 1; i < X - 1; ++i)
            for (int j = 1; j < Y - 1; ++j)
                for (int k = 1; k < Z - 1; ++k) {
                    const size_t id = nodeIndex(c, i, j, k);
                    if (!unk[id]) { out[id] = 0.0; continue; }
                    double s = 6.0 * v[id];
                    const int nb[6][3] = {{i - 1, j, k}, {i + 1, j, k}, {i, j - 1, k}, {i, j + 1, k}, {i, j, k - 1}, {i, j, k + 1}};
                    for (int t = 0; t < 6; ++t) {
                        const int a = wrap(nb[t][0], X, 0), b = wrap(nb[t][1], Y, 1), d = wrap(nb[t][2], Z, 2);
                        const size_t nid = nodeIndex(c, a, b, d);
                        if (unk[nid] || with_fixed) s -= v[nid];
                    }
                    out[id] = s;
                }
    };
    double fsum = 0.0; size_t nunk = 0;
    for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
        const size_t id = nodeIndex(c, i, j, k);
        if (unk[id]) { f[id] = c.rho[0].v[id] / c.p.eps0; fsum += f[id]; ++nunk; }
    }
    if (allp && nunk) { const double m = fsum / nunk; for (size_t t = 0; t < N; ++t) if (unk[t]) f[t] -= m; }
    apply(x, Ap, true);
    double fn = 0.0, rr = 0.0;
    for (size_t t = 0; t < N; ++t) if (unk[t]) { r[t] = f[t] - Ap[t]; fn += f[t] * f[t]; }
    if (allp) { double m = 0; for (size_t t = 0; t < N; ++t) if (unk[t]) m += r[t]; m /= nunk; for (size_t t = 0; t < N; ++t) if (unk[t]) r[t] -= m; }
    for (size_t t = 0; t < N; ++t) if (unk[t]) { pp[t] = r[t]; rr += r[t] * r[t]; }
    fn = std::sqrt(fn);
    int it = 0;
    const double stop = c.exact_tol * (fn > 0 ? fn : 1.0);
    while (std::sqrt(rr) > stop && it < 20000) {
        apply(pp, Ap, false);
        double pAp = 0.0;
        for (size_t t = 0; t < N; ++t) if (unk[t]) pAp += pp[t] * Ap[t];
        const double alpha = rr / pAp;
        double rr2 = 0.0;
        for (size_t t = 0; t < N; ++t) if (unk[t]) { x[t] += alpha * pp[t]; r[t] -= alpha * Ap[t]; rr2 += r[t] * r[t]; }
        const double beta = rr2 / rr;
        rr = rr2;
        for (size_t t = 0; t < N; ++t) if (unk[t]) pp[t] = r[t] + beta * pp[t];
        ++it;
    }
    if (allp) {  // gauge: mean of the unknowns zero
        double m = 0; for (size_t t = 0; t < N; ++t) if (unk[t]) m += x[t]; m /= nunk;
        for (size_t t = 0; t < N; ++t) if (unk[t]) x[t] -= m;
    }
    for (size_t t = 0; t < N; ++t) if (unk[t]) c.phi.v[t] = x[t];
    // glue copies of the periodic axes, as doPSOR's trailing exchanges leave them
    copy_field_glue(c, c.phi);
    c.last_iterations = it;
    c.last_residual = fn > 0 ? std::sqrt(rr) / fn : 0.0;
}

// RootGrid::solvePoissonPSOR (src/Grid/RootGrid/RootGridField.cpp:65-103).
static void solve_poisson(Ctx& c) {
    c.poisson_error = c.phi;
    if (c.solver_mode == 1) {
        exact_solve(c);
    } else {
        constexpr double required_error = 1.0e-7;
        int loop = 1;
        for (; loop <= c.max_post_loop; ++loop) {
            do_psor(c);
            if ((loop % 10 == 0)) {
                c.last_residual = check_phi_residual(c);
                if (c.last_residual < required_error) break;
            }
        }
        c.last_iterations = loop - 1 < c.max_post_loop ? loop : c.max_post_loop;
    }
    set_boundary_phi(c);
    for (int i = 1; i < c.cx - 1; ++i) for (int j = 1; j < c.cy - 1; ++j) for (int k = 1; k < c.cz - 1; ++k)
        c.poisson_error(i, j, k) = c.phi(i, j, k) - c.poisson_error(i, j, k);
}

// RootGrid::updateRho (src/Grid/RootGrid/RootGridField.cpp:1153-1252).
static int update_rho(Ctx& c) {
    for (auto& r : c.rho) r.zero();
    int bad = 0;
    int64_t absorbed = 0;
    c.incidents_by_species.assign(c.nsp, {});
#pragma omp parallel for schedule(static) reduction(| : bad) reduction(+ : absorbed)
    for (int pid = 0; pid < c.nsp; ++pid) {
        const double q = c.p.species[pid].charge * c.p.species[pid].size;
        Arr3& r = c.rho[pid + 1];
        for (auto& p : c.particles[pid]) {
            if (!p.isValid) continue;
            for (int oi = 0; oi < (int)c.objects.size(); ++oi) {
                int b = 0;
                absorbed += absorb(c, oi, p, b, &c.incidents_by_species[pid]);
                bad |= b;
            }
            if (p.isValid) {
                const Pos pos = posXYZ(p.x, p.y, p.z);
                const int i = pos.i, j = pos.j, k = pos.k;
                r(i, j, k) += pos.dx2 * pos.dy2 * pos.dz2 * q;
                r(i + 1, j, k) += pos.dx1 * pos.dy2 * pos.dz2 * q;
                r(i, j + 1, k) += pos.dx2 * pos.dy1 * pos.dz2 * q;
                r(i + 1, j + 1, k) += pos.dx1 * pos.dy1 * pos.dz2 * q;
                r(i, j, k + 1) += pos.dx2 * pos.dy2 * pos.dz1 * q;
                r(i + 1, j, k + 1) += pos.dx1 * pos.dy2 * pos.dz1 * q;
                r(i, j + 1, k + 1) += pos.dx2 * pos.dy1 * pos.dz1 * q;
                r(i + 1, j + 1, k + 1) += pos.dx1 * pos.dy1 * pos.dz1 * q;
            }
        }
    }
    c.absorbed_step = absorbed;
    for (auto& v : c.incidents_by_species) c.incidents.insert(c.incidents.end(), v.begin(), v.end());
    for (auto& o : c.objects) sum_whole_charge(c, o);
    for (int pid = 1; pid <= c.nsp; ++pid)
        for (size_t t = 0; t < c.rho[0].v.size(); ++t) c.rho[0].v[t] += c.rho[pid].v[t];
    for (auto& r : c.rho) fold_node_scalar(c, r);
    if (!c.objects.empty()) {
        solve_poisson(c);
        for (auto& o : c.objects) redistribute(c, o);
        copy_field_glue(c, c.rho[0]);
    }
    return bad;
}

// RootGrid::updateEfield + updateReferenceEfield (RootGridField.cpp:456-582).
static void update_efield(Ctx& c) {
    const int X = c.cx, Y = c.cy, Z = c.cz;
    Arr3& phi = c.phi;
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Y; ++j)
            for (int k = 0; k < Z; ++k) {
                if (i < X - 1) c.ex(i, j, k) = phi(i, j, k) - phi(i + 1, j, k);
                if (j < Y - 1) c.ey(i, j, k) = phi(i, j, k) - phi(i, j + 1, k);
                if (k < Z - 1) c.ez(i, j, k) = phi(i, j, k) - phi(i, j, k + 1);
            }
#pragma omp parallel for schedule(static)
    for (int i = 1; i < X - 1; ++i)
        for (int j = 1; j < Y - 1; ++j)
            for (int k = 1; k < Z - 1; ++k) {
                c.exref(i, j, k) = 0.5 * (c.ex(i - 1, j, k) + c.ex(i, j, k));
                c.eyref(i, j, k) = 0.5 * (c.ey(i, j - 1, k) + c.ey(i, j, k));
                c.ezref(i, j, k) = 0.5 * (c.ez(i, j, k - 1) + c.ez(i, j, k));
            }
    if (isBoundary(c, 0, 0))
        for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
            c.exref(0, j, k) = 0.0;
            c.exref(1, j, k) = 0.5 * (phi(3, j, k) - 4.0 * phi(2, j, k) + 3.0 * phi(1, j, k));
        }
    if (isBoundary(c, 0, 1))
        for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
            c.exref(X - 1, j, k) = 0.0;
            c.exref(X - 2, j, k) = 0.5 * (-phi(X - 4, j, k) + 4.0 * phi(X - 3, j, k) - 3.0 * phi(X - 2, j, k));
        }
    if (isBoundary(c, 1, 0))
        for (int i = 1; i < X - 1; ++i) for (int k = 1; k < Z - 1; ++k) {
            c.eyref(i, 0, k) = 0.0;
            c.eyref(i, 1, k) = 0.5 * (phi(i, 3, k) - 4.0 * phi(i, 2, k) + 3.0 * phi(i, 1, k));
        }
    if (isBoundary(c, 1, 1))
        for (int i = 1; i < X - 1; ++i) for (int k = 1; k < Z - 1; ++k) {
            c.eyref(i, Y - 1, k) = 0.0;
            c.eyref(i, Y - 2, k) = 0.5 * (-phi(i, Y - 4, k) + 4.0 * phi(i, Y - 3, k) - 3.0 * phi(i, Y - 2, k));
        }
    if (isBoundary(c, 2, 0))
        for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) {
            c.ezref(i, j, 0) = 0.0;
            c.ezref(i, j, 1) = 0.5 * (phi(i, j, 3) - 4.0 * phi(i, j, 2) + 3.0 * phi(i, j, 1));
        }
    if (isBoundary(c, 2, 1))
        for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) {
            c.ezref(i, j, Z - 1) = 0.0;
            c.ezref(i, j, Z - 2) = 0.5 * (-phi(i, j, Z - 4) + 4.0 * phi(i, j, Z - 3) - 3.0 * phi(i, j, Z - 2));
        }
    copy_field_glue(c, c.exref);
    copy_field_glue(c, c.eyref);
    copy_field_glue(c, c.ezref);
}

// ---------------------------------------------------------------- EM mode
// Communicator::sendRecvFieldX/Y/Z self branch on an array with index bases
// (src/MPI/Communicator.cpp:265-343): along a periodic axis (base 0 there)
// index 0 <- index max-2, index max-1 <- index 1, over the whole extent of the
// other two axes; x, then y, then z.
static void copy_field_glue_b(const Ctx& c, ArrB& a) {
    for (int axis = 0; axis < 3; ++axis) {
        if (!c.notb[2 * axis]) continue;
        const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
        const int m = a.up(axis);
        for (int u = a.lo[a1]; u < a.up(a1); ++u)
            for (int w = a.lo[a2]; w < a.up(a2); ++w) {
                int p0[3], p1[3], pm2[3], pm1[3];
                p0[a1] = p1[a1] = pm2[a1] = pm1[a1] = u;
                p0[a2] = p1[a2] = pm2[a2] = pm1[a2] = w;
                p0[axis] = 0; p1[axis] = 1; pm2[axis] = m - 2; pm1[axis] = m - 1;
                const double lo = a(p1[0], p1[1], p1[2]);
                a(p0[0], p0[1], p0[2]) = a(pm2[0], pm2[1], pm2[2]);
                a(pm1[0], pm1[1], pm1[2]) = lo;
            }
    }
}

// MPIw::Environment::sendRecvEdgeScalar (src/MPI/Environment.cpp:74-130) with
// Communicator::sendRecvScalarX/Y/Z's self branch (Communicator.cpp:497-574):
// along each periodic axis the glue planes g-1-t and size-1-t (t < g) both
// become their sum, g = 2 along the current's own direction, 1 across it.
static void fold_edge_scalar(const Ctx& c, Arr3& a, int dir) {
    const int dims[3] = {a.cx, a.cy, a.cz};
    for (int axis = 0; axis < 3; ++axis) {
        if (!c.notb[2 * axis]) continue;
        const int g = axis == dir ? 2 : 1, size = dims[axis];
        const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
        for (int u = 0; u < dims[a1]; ++u)
            for (int w = 0; w < dims[a2]; ++w)
                for (int t = 0; t < g; ++t) {
                    int pl[3], pu[3];
                    pl[a1] = pu[a1] = u; pl[a2] = pu[a2] = w;
                    pl[axis] = g - 1 - t; pu[axis] = size - 1 - t;
                    const double s = a(pl[0], pl[1], pl[2]) + a(pu[0], pu[1], pu[2]);
                    a(pl[0], pl[1], pl[2]) = s; a(pu[0], pu[1], pu[2]) = s;
                }
    }
}

// RootGrid::updateReferenceEfield (RootGridField.cpp:489-582) on the Yee edges
// of the EM mode: nodal means of the two edges, the one-sided phi difference on
// the node next to a non-periodic face and zero on its glue node.
static void reference_efield_em(Ctx& c) {
    const int X = c.cx, Y = c.cy, Z = c.cz;
    Arr3& phi = c.phi;
    for (int i = 1; i < X - 1; ++i)
        for (int j = 1; j < Y - 1; ++j)
            for (int k = 1; k < Z - 1; ++k) {
                c.exref(i, j, k) = 0.5 * (c.fex(i - 1, j, k) + c.fex(i, j, k));
                c.eyref(i, j, k) = 0.5 * (c.fey(i, j - 1, k) + c.fey(i, j, k));
                c.ezref(i, j, k) = 0.5 * (c.fez(i, j, k - 1) + c.fez(i, j, k));
            }
    if (isBoundary(c, 0, 0))
        for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
            c.exref(0, j, k) = 0.0;
            c.exref(1, j, k) = 0.5 * (phi(3, j, k) - 4.0 * phi(2, j, k) + 3.0 * phi(1, j, k));
        }
    if (isBoundary(c, 0, 1))
        for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
            c.exref(X - 1, j, k) = 0.0;
            c.exref(X - 2, j, k) = 0.5 * (-phi(X - 4, j, k) + 4.0 * phi(X - 3, j, k) - 3.0 * phi(X - 2, j, k));
        }
    if (isBoundary(c, 1, 0))
        for (int i = 1; i < X - 1; ++i) for (int k = 1; k < Z - 1; ++k) {
            c.eyref(i, 0, k) = 0.0;
            c.eyref(i, 1, k) = 0.5 * (phi(i, 3, k) - 4.0 * phi(i, 2, k) + 3.0 * phi(i, 1, k));
        }
    if (isBoundary(c, 1, 1))
        for (int i = 1; i < X - 1; ++i) for (int k = 1; k < Z - 1; ++k) {
            c.eyref(i, Y - 1, k) = 0.0;
            c.eyref(i, Y - 2, k) = 0.5 * (-phi(i, Y - 4, k) + 4.0 * phi(i, Y - 3, k) - 3.0 * phi(i, Y - 2, k));
        }
    if (isBoundary(c, 2, 0))
        for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) {
            c.ezref(i, j, 0) = 0.0;
            c.ezref(i, j, 1) = 0.5 * (phi(i, j, 3) - 4.0 * phi(i, j, 2) + 3.0 * phi(i, j, 1));
        }
    if (isBoundary(c, 2, 1))
        for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) {
            c.ezref(i, j, Z - 1) = 0.0;
            c.ezref(i, j, Z - 2) = 0.5 * (-phi(i, j, Z - 4) + 4.0 * phi(i, j, Z - 3) - 3.0 * phi(i, j, Z - 2));
        }
    copy_field_glue(c, c.exref);
    copy_field_glue(c, c.eyref);
    copy_field_glue(c, c.ezref);
}

// RootGrid::updateEfield (RootGridField.cpp:456-487) in the EM mode: the edges of
// the real grid from phi (the damping layers keep their values), then the
// nodal reference.
static void update_efield_em_from_phi(Ctx& c) {
    const int X = c.cx, Y = c.cy, Z = c.cz;
    const Arr3& phi = c.phi;
    for (int i = 0; i < X; ++i)
        for (int j = 0; j < Y; ++j)
            for (int k = 0; k < Z; ++k) {
                if (i < X - 1) c.fex(i, j, k) = phi(i, j, k) - phi(i + 1, j, k);
                if (j < Y - 1) c.fey(i, j, k) = phi(i, j, k) - phi(i, j + 1, k);
                if (k < Z - 1) c.fez(i, j, k) = phi(i, j, k) - phi(i, j, k + 1);
            }
    reference_efield_em(c);
}

// RootGrid::updateReferenceBfield (RootGridField.cpp:1102-1127): nodal means of
// the four faces around each node, then the periodic glue copies.
static void reference_bfield(Ctx& c) {
    const int X = c.cx, Y = c.cy, Z = c.cz;
    for (int i = 1; i < X - 1; ++i)
        for (int j = 1; j < Y - 1; ++j)
            for (int k = 1; k < Z - 1; ++k) {
                c.bxref(i, j, k) = 0.25 * (c.fbx(i, j, k) + c.fbx(i, j - 1, k) + c.fbx(i, j, k - 1) + c.fbx(i, j - 1, k - 1));
                c.byref(i, j, k) = 0.25 * (c.fby(i, j, k) + c.fby(i - 1, j, k) + c.fby(i, j, k - 1) + c.fby(i - 1, j, k - 1));
                c.bzref(i, j, k) = 0.25 * (c.fbz(i, j, k) + c.fbz(i - 1, j, k) + c.fbz(i, j - 1, k) + c.fbz(i - 1, j - 1, k));
            }
    copy_field_glue(c, c.bxref);
    copy_field_glue(c, c.byref);
    copy_field_glue(c, c.bzref);
}

// The damping mask of updateEfieldFDTDDamping / updateBfieldDamping
// (RootGridField.cpp:628-642, 742-756): 1 - (d/L)^2 with d the distance of an
// index from the real grid [1, real-2] (masking_parameter 1).
static inline double damp1(double r, double L, int real) {
    const double d = (r <= 0) ? -r + 1 : (r >= real - 1) ? r - static_cast<double>(real) + 2.0 : 0.0;
    return 1.0 - std::pow(1.0 * d / L, 2);
}
static inline double damp(const Ctx& c, int i, int j, int k) {
    return damp1(i, c.L[0], c.cx) * damp1(j, c.L[1], c.cy) * damp1(k, c.L[2], c.cz);
}
static inline bool real_region(const Ctx& c, int i, int j, int k) {
    return i > 0 && i < c.cx - 1 && j > 0 && j < c.cy - 1 && k > 0 && k < c.cz - 1;
}

// RootGrid::updateEfieldFDTDDamping (RootGridField.cpp:594-710): E += dt/eps0
// (curl B / mu0 - J) on the real edges, the damped update without J on the
// last real edge of each direction and throughout the damping layers, then the
// periodic glue copies and the nodal reference.
static void update_efield_fdtd(Ctx& c) {
    ArrB &ex = c.fex, &ey = c.fey, &ez = c.fez;
    const ArrB &bx = c.fbx, &by = c.fby, &bz = c.fbz;
    const double dte = 1.0 / c.p.eps0;              // dt / eps0, dt = 1
    const double C = dte / (c.p.mu0 * 1.0);        // dt / (mu0 eps0 dx)
    const int i0 = ex.lo[0] + 1, i1 = ex.up(0), j0 = ex.lo[1] + 1, j1 = ex.up(1) - 1;
    const int k0 = ex.lo[2] + 1, k1 = ex.up(2) - 1;
    const int xmax = ex.up(0) + 1, ymax = ex.up(1), zmax = ex.up(2);   // max_x/y/z_index
#pragma omp parallel for schedule(static)
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                const double cx_ = bz(i, j, k) - bz(i, j - 1, k) - by(i, j, k) + by(i, j, k - 1);
                if (real_region(c, i, j, k)) {
                    if (i < c.cx - 2) ex(i, j, k) = ex(i, j, k) - c.jx(i, j, k) * dte + C * cx_;
                    else ex(i, j, k) = 0.5 * (damp(c, i, j, k) + damp(c, i + 1, j, k)) * (ex(i, j, k) + C * cx_);
                } else if (i < xmax - 2) {
                    ex(i, j, k) = 0.5 * (damp(c, i, j, k) + damp(c, i + 1, j, k)) * (ex(i, j, k) + C * cx_);
                }
            }
#pragma omp parallel for schedule(static)
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                const double cy_ = bx(i, j, k) - bx(i, j, k - 1) - bz(i, j, k) + bz(i - 1, j, k);
                const double cz_ = by(i, j, k) - by(i - 1, j, k) - bx(i, j, k) + bx(i, j - 1, k);
                if (real_region(c, i, j, k)) {
                    if (j < c.cy - 2) ey(i, j, k) = ey(i, j, k) - c.jy(i, j, k) * dte + C * cy_;
                    else ey(i, j, k) = 0.5 * (damp(c, i, j, k) + damp(c, i, j + 1, k)) * (ey(i, j, k) + C * cy_);
                    if (k < c.cz - 2) ez(i, j, k) = ez(i, j, k) - c.jz(i, j, k) * dte + C * cz_;
                    else ez(i, j, k) = 0.5 * (damp(c, i, j, k) + damp(c, i, j, k + 1)) * (ez(i, j, k) + C * cz_);
                } else {
                    if (j < ymax - 2)
                        ey(i, j, k) = 0.5 * (damp(c, i, j, k) + damp(c, i, j + 1, k)) * (ey(i, j, k) + C * cy_);
                    if (k < zmax - 2)
                        ez(i, j, k) = 0.5 * (damp(c, i, j, k) + damp(c, i, j, k + 1)) * (ez(i, j, k) + C * cz_);
                }
            }
    copy_field_glue_b(c, ex);
    copy_field_glue_b(c, ey);
    copy_field_glue_b(c, ez);
    reference_efield_em(c);
}

// RootGrid::updateBfieldDamping (RootGridField.cpp:712-820): B -= dt curl E / dx on
// the real faces, damped on the last real face and in the damping layers,
// then the periodic glue copies and the nodal reference.
static void update_bfield(Ctx& c) {
    ArrB &bx = c.fbx, &by = c.fby, &bz = c.fbz;
    const ArrB &ex = c.fex, &ey = c.fey, &ez = c.fez;
    const double d = 1.0;                           // dt / dx
    const int xmax = bx.up(0), ymax = bx.up(1) + 1, zmax = bx.up(2) + 1;   // max_x/y/z_index
    const int X = c.cx, Y = c.cy, Z = c.cz;
#pragma omp parallel for schedule(static)
    for (int i = bx.lo[0] + 1; i < xmax - 1; ++i)
        for (int j = bx.lo[1] + 1; j < ymax - 1; ++j)
            for (int k = bx.lo[2] + 1; k < zmax - 1; ++k) {
                const double gx = (ey(i, j, k + 1) - ey(i, j, k)) - (ez(i, j + 1, k) - ez(i, j, k));
                const double gy = (ez(i + 1, j, k) - ez(i, j, k)) - (ex(i, j, k + 1) - ex(i, j, k));
                const double gz = (ex(i, j + 1, k) - ex(i, j, k)) - (ey(i + 1, j, k) - ey(i, j, k));
                const double mx = 0.25 * (damp(c, i, j, k) + damp(c, i, j + 1, k) + damp(c, i, j, k + 1) + damp(c, i, j + 1, k + 1));
                const double my = 0.25 * (damp(c, i, j, k) + damp(c, i + 1, j, k) + damp(c, i, j, k + 1) + damp(c, i + 1, j, k + 1));
                const double mz = 0.25 * (damp(c, i, j, k) + damp(c, i + 1, j, k) + damp(c, i, j + 1, k) + damp(c, i + 1, j + 1, k));
                if (real_region(c, i, j, k)) {
                    if (j != Y - 2 && k != Z - 2) bx(i, j, k) = bx(i, j, k) + d * gx;
                    else bx(i, j, k) = mx * (bx(i, j, k) + d * gx);
                    if (i != X - 2 && k != Z - 2) by(i, j, k) = by(i, j, k) + d * gy;
                    else by(i, j, k) = my * (by(i, j, k) + d * gy);
                    if (i != X - 2 && j != Y - 2) bz(i, j, k) = bz(i, j, k) + d * gz;
                    else bz(i, j, k) = mz * (bz(i, j, k) + d * gz);
                } else {
                    if (j != ymax - 2 && k != zmax - 2) bx(i, j, k) = mx * (bx(i, j, k) + d * gx);
                    if (i != xmax - 2 && k != zmax - 2) by(i, j, k) = my * (by(i, j, k) + d * gy);
                    if (i != xmax - 2 && j != ymax - 2) bz(i, j, k) = mz * (bz(i, j, k) + d * gz);
                }
            }
    copy_field_glue_b(c, bx);
    copy_field_glue_b(c, by);
    copy_field_glue_b(c, bz);
    reference_bfield(c);
}

// Grid::updateParticleVelocityEM (src/Grid/GridParticleTreatmentEM.cpp:13-105):
// CIC gather of the nodal E and B, both scaled by 0.5 q/m, and the Boris
// kick/rotate/kick with the gathered b (boris = 2 / (1 + |b|^2)).
static void update_velocity_em(Ctx& c) {
    for (int pid = 0; pid < c.nsp; ++pid) {
        const double qm = 0.5 * c.p.species[pid].charge / c.p.species[pid].mass;
        auto& parray = c.particles[pid];
        const long n = (long)parray.size();
#pragma omp parallel for schedule(static)
        for (long pn = 0; pn < n; ++pn) {
            Particle& p = parray[pn];
            if (!p.isValid) continue;
            Pos pos = posXYZ(p.x, p.y, p.z);
            const int i = pos.i, j = pos.j, k = pos.k;
            const double v1 = qm * pos.dx2 * pos.dy2 * pos.dz2, v2 = qm * pos.dx1 * pos.dy2 * pos.dz2;
            const double v3 = qm * pos.dx2 * pos.dy1 * pos.dz2, v4 = qm * pos.dx1 * pos.dy1 * pos.dz2;
            const double v5 = qm * pos.dx2 * pos.dy2 * pos.dz1, v6 = qm * pos.dx1 * pos.dy2 * pos.dz1;
            const double v7 = qm * pos.dx2 * pos.dy1 * pos.dz1, v8 = qm * pos.dx1 * pos.dy1 * pos.dz1;
            auto g = [&](const Arr3& e) {
                return v1 * e(i, j, k) + v2 * e(i + 1, j, k) + v3 * e(i, j + 1, k) + v4 * e(i + 1, j + 1, k) +
                       v5 * e(i, j, k + 1) + v6 * e(i + 1, j, k + 1) + v7 * e(i, j + 1, k + 1) +
                       v8 * e(i + 1, j + 1, k + 1);
            };
            const double exv = g(c.exref), eyv = g(c.eyref), ezv = g(c.ezref);
            const double bx = g(c.bxref), by = g(c.byref), bz = g(c.bzref);
            const double boris = 2.0 / (1.0 + (bx * bx + by * by + bz * bz));
            const double vx1 = p.vx + exv, vy1 = p.vy + eyv, vz1 = p.vz + ezv;
            const double vxt = vx1 + vy1 * bz - vz1 * by;
            const double vyt = vy1 + vz1 * bx - vx1 * bz;
            const double vzt = vz1 + vx1 * by - vy1 * bx;
            p.vx = vx1 + exv + boris * (vyt * bz - vzt * by);
            p.vy = vy1 + eyv + boris * (vzt * bx - vxt * bz);
            p.vz = vz1 + ezv + boris * (vxt * by - vyt * bx);
        }
    }
}

// Position::getReferencePosition (include/position.hpp:88-96): the zigzag's
// relay point, on the shared cell face when the cells differ, else the midpoint.
static inline double relay(int i_new, int i_old, double x_new, double x_old) {
    return std::min(static_cast<double>(std::min(i_new, i_old)),
                    std::max(static_cast<double>(std::max(i_new, i_old)) - 1.0, 0.5 * (x_new + x_old)));
}

// One half of the charge-conserving current of Particle::distributeCurrentAt
// OldPosition / AtNewPosition (src/Particle/particle.cpp:258-338): flux f on
// the edges of the cell of `at`, weights w = mean of the half's two points
// minus the cell's lower node.
static void current_half(Ctx& c, const Pos& at, const double f[3], const double w[3]) {
    const int i = at.i, j = at.j, k = at.k;
    c.jx(i, j, k) += f[0] * (1.0 - w[1]) * (1.0 - w[2]);
    c.jx(i, j + 1, k) += f[0] * w[1] * (1.0 - w[2]);
    c.jx(i, j, k + 1) += f[0] * (1.0 - w[1]) * w[2];
    c.jx(i, j + 1, k + 1) += f[0] * w[1] * w[2];
    c.jy(i, j, k) += f[1] * (1.0 - w[0]) * (1.0 - w[2]);
    c.jy(i + 1, j, k) += f[1] * w[0] * (1.0 - w[2]);
    c.jy(i, j, k + 1) += f[1] * (1.0 - w[0]) * w[2];
    c.jy(i + 1, j, k + 1) += f[1] * w[0] * w[2];
    c.jz(i, j, k) += f[2] * (1.0 - w[0]) * (1.0 - w[1]);
    c.jz(i + 1, j, k) += f[2] * w[0] * (1.0 - w[1]);
    c.jz(i, j + 1, k) += f[2] * (1.0 - w[0]) * w[1];
    c.jz(i + 1, j + 1, k) += f[2] * w[0] * w[1];
}

// RootGrid::updateParticlePositionEM (src/Grid/GridParticleTreatmentEM.cpp:107-201):
// J = 0 (Field::initializeCurrent), for every valid particle the old-cell half
// of the current (from x to x + v), the move and the boundary rules, and for a
// particle still valid the new-cell half (from x - v to x, in the wrapped frame
// after a periodic crossing); then the periodic folds of the edge currents.
// The single-rank migration appends crossing particles in the reference;
// wrapping them in place leaves the same set and the same sums.
static void update_position_em(Ctx& c) {
    c.jx.zero(); c.jy.zero(); c.jz.zero();
    const double slx = c.nx, sly = c.ny, slz = c.nz;
    for (int pid = 0; pid < c.nsp; ++pid) {
        const double q = c.p.species[pid].charge * c.p.species[pid].size / 1.0;   // per dt
        for (auto& p : c.particles[pid]) {
            if (!p.isValid) continue;
            {
                const Pos o = posXYZ(p.x, p.y, p.z);
                const Pos nw = posXYZ(p.x + p.vx, p.y + p.vy, p.z + p.vz);
                const Pos r = posXYZ(relay(nw.i, o.i, nw.x, o.x), relay(nw.j, o.j, nw.y, o.y), relay(nw.k, o.k, nw.z, o.z));
                const double f[3] = {q * (r.x - o.x), q * (r.y - o.y), q * (r.z - o.z)};
                const double w[3] = {0.5 * (r.x + o.x) - (static_cast<double>(o.i) - 1.0),
                                     0.5 * (r.y + o.y) - (static_cast<double>(o.j) - 1.0),
                                     0.5 * (r.z + o.z) - (static_cast<double>(o.k) - 1.0)};
                current_half(c, o, f, w);
            }
            p.x += p.vx; p.y += p.vy; p.z += p.vz;
            boundary_axis(c, p.x, p.isValid, 0, slx);
            boundary_axis(c, p.y, p.isValid, 1, sly);
            boundary_axis(c, p.z, p.isValid, 2, slz);
            if (p.isValid) {
                const Pos o = posXYZ(p.x - p.vx, p.y - p.vy, p.z - p.vz);
                const Pos nw = posXYZ(p.x, p.y, p.z);
                const Pos r = posXYZ(relay(nw.i, o.i, nw.x, o.x), relay(nw.j, o.j, nw.y, o.y), relay(nw.k, o.k, nw.z, o.z));
                const double f[3] = {q * (nw.x - r.x), q * (nw.y - r.y), q * (nw.z - r.z)};
                const double w[3] = {0.5 * (r.x + nw.x) - (static_cast<double>(nw.i) - 1.0),
                                     0.5 * (r.y + nw.y) - (static_cast<double>(nw.j) - 1.0),
                                     0.5 * (r.z + nw.z) - (static_cast<double>(nw.k) - 1.0)};
                current_half(c, nw, f, w);
            }
        }
    }
    fold_edge_scalar(c, c.jx, 0);
    fold_edge_scalar(c, c.jy, 1);
    fold_edge_scalar(c, c.jz, 2);
}

// Field::getBfieldEnergy (src/Grid/Field.cpp:215-234), normalised.
static double bfield_energy(const Ctx& c) {
    const int X = c.cx, Y = c.cy, Z = c.cz;
    double en = 0.0;
    for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
        if (j < Y - 2 && k < Z - 2) en += std::pow(c.fbx(i, j, k), 2);
        if (i < X - 2 && k < Z - 2) en += std::pow(c.fby(i, j, k), 2);
        if (i < X - 2 && j < Y - 2) en += std::pow(c.fbz(i, j, k), 2);
    }
    return 0.5 * en / c.p.mu0;
}

// ---------------------------------------------------------------- sources
static inline double max_extent(const Ctx& c, int axis) {
    const int n = axis == 0 ? c.nx : (axis == 1 ? c.ny : c.nz);
    return isBoundary(c, axis, 1) ? n - 1.0 : (double)n;  // RootGrid.cpp:46-53
}

// RootGrid::RootGrid ambient loading (RootGrid.cpp:45-79) with
// ParticleType::getTotalNumber (ParticleType.cpp:39-47),
// AmbientParticleType::generateNewPosition/Velocity (AmbientParticleType.cpp:76-99).
static void generate_ambient(Ctx& c) {
    const double mx = max_extent(c, 0), my = max_extent(c, 1), mz = max_extent(c, 2);
    for (int s = 0; s < c.nsp; ++s) {
        const fopis_species& sp = c.p.species[s];
        if (sp.kind != FOPIS_SPECIES_AMBIENT) continue;
        const int64_t cxn = isBoundary(c, 0, 1) ? c.nx - 1 : c.nx;
        const int64_t cyn = isBoundary(c, 1, 1) ? c.ny - 1 : c.ny;
        const int64_t czn = isBoundary(c, 2, 1) ? c.nz - 1 : c.nz;
        const int64_t total = cxn * cyn * czn * sp.particle_per_cell;
        std::vector<Particle> out((size_t)total);
        std::vector<unsigned char> keep((size_t)total, 1);
#pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < total; ++t) {
            const uint32_t a = (uint32_t)t, b = (uint32_t)(t >> 32), cc = (uint32_t)s, dtag = TAG_LOAD << 24;
            const U2 r0 = draw2(c.p.seed, a, b, cc, dtag | 0), r1 = draw2(c.p.seed, a, b, cc, dtag | 1);
            const U2 r2 = draw2(c.p.seed, a, b, cc, dtag | 2), r3 = draw2(c.p.seed, a, b, cc, dtag | 3);
            Particle p;
            p.x = 0.0 + (mx - 0.0) * r0.a; p.y = 0.0 + (my - 0.0) * r0.b; p.z = 0.0 + (mz - 0.0) * r1.a;
            double n0, n1, n2, n3;
            box_muller(r1.b, r2.a, n0, n1);
            box_muller(r2.b, r3.a, n2, n3);
            p.vx = sp.drift[0] + sp.deviation * n0;
            p.vy = sp.drift[1] + sp.deviation * n1;
            p.vz = sp.drift[2] + sp.deviation * n2;
            p.typeId = s; p.isValid = 1;
            const Pos pos = posXYZ(p.x, p.y, p.z);
            for (const auto& o : c.objects) if (isContaining(c, o, pos)) keep[(size_t)t] = 0;
            out[(size_t)t] = p;
        }
        for (int64_t t = 0; t < total; ++t) if (keep[(size_t)t]) c.particles[s].push_back(out[(size_t)t]);
    }
}

// Injection velocity by rejection (AmbientParticleType::generateNewInjectionVelocity,
// AmbientParticleType.cpp:101-157): all three components are redrawn until the
// normal component points inward. Returns the attempts used (cap 256).
static int injection_particle(const Ctx& c, int s, int face, int64_t step, uint32_t t, Particle& p) {
    const fopis_species& sp = c.p.species[s];
    const int axis = face / 2;
    const double sign = (face % 2 == 0) ? 1.0 : -1.0;
    const uint32_t cc = (uint32_t)s | ((uint32_t)face << 8), dtag = TAG_INJECT << 24;
    double v[3];
    int attempt = 0;
    for (; attempt < 256; ++attempt) {
        const U2 r0 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | (uint32_t)(2 * attempt));
        const U2 r1 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | (uint32_t)(2 * attempt + 1));
        double n0, n1, n2, n3;
        box_muller(r0.a, r0.b, n0, n1);
        box_muller(r1.a, r1.b, n2, n3);
        const double nn[3] = {n0, n1, n2};
        for (int a = 0; a < 3; ++a) v[a] = sp.drift[a] + (a == axis ? sp.thermal_velocity : sp.deviation) * nn[a];
        if (!((v[axis] * sign) < 0.0)) break;
    }
    const U2 q0 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | 0xFFF0u);
    const U2 q1 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | 0xFFF1u);
    const double u[3] = {q0.a, q0.b, q1.a};
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = 0.0; hi[a] = max_extent(c, a); }
    if (face % 2 == 0) { hi[axis] = v[axis]; }                       // [0, v dt)
    else { lo[axis] = max_extent(c, axis) + v[axis]; }               // [max + v dt, max)
    double x[3];
    for (int a = 0; a < 3; ++a) x[a] = lo[a] + (hi[a] - lo[a]) * u[a];  // uniform_real_distribution(lo, hi)
    p.x = x[0]; p.y = x[1]; p.z = x[2];
    p.vx = v[0]; p.vy = v[1]; p.vz = v[2];
    p.typeId = s; p.isValid = 1;
    return attempt;
}

// Node size along an axis as RootGrid::getXNodeSize (RootGrid.cpp:192-204).
static inline int node_size(const Ctx& c, int axis) {
    const int n = axis == 0 ? c.nx : (axis == 1 ? c.ny : c.nz);
    return c.notb[2 * axis + 1] ? n + 1 : n;
}

// RootGrid::injectParticlesFromBoundary (src/Grid/RootGrid/RootGridParticle.cpp:3-130).
static void inject(Ctx& c, int64_t* counts_out) {
    int64_t injected = 0;
    for (int s = 0; s < c.nsp; ++s) {
        const fopis_species& sp = c.p.species[s];
        if (sp.kind != FOPIS_SPECIES_AMBIENT) continue;
        for (int face = 0; face < 6; ++face) {
            const int axis = face / 2, side = face % 2;
            if (!isBoundary(c, axis, side)) continue;
            const int a1 = (axis + 1) % 3, a2 = (axis + 2) % 3;
            const double area = (double)(node_size(c, a2) - 1) * (node_size(c, a1) - 1);
            const double flux = sp.injection_axis[face] ? sp.flux[face] : 0.0;
            const double num_double = 1.0 * area * flux;
            const int num = (int)std::floor(num_double + c.inject_residual[s][face]);
            c.inject_residual[s][face] += num_double - num;
            if (counts_out) counts_out[s * 6 + face] = num;
            std::vector<Particle> batch(num > 0 ? num : 0);
#pragma omp parallel for schedule(static)
            for (int t = 0; t < num; ++t) injection_particle(c, s, face, c.timestep, (uint32_t)t, batch[t]);
            for (auto& p : batch) c.particles[s].push_back(p);
            injected += num;
        }
    }
    c.injected_step = injected;
}

// Particle::getNext{X,Y,Z}CrossPoint (src/Particle/particle.cpp:206-255).
static Pos next_cross(const Particle& p, int axis) {
    Pos pos = posXYZ(p.x, p.y, p.z);
    const double v[3] = {p.vx, p.vy, p.vz};
    const double d1[3] = {pos.dx1, pos.dy1, pos.dz1}, d2[3] = {pos.dx2, pos.dy2, pos.dz2};
    double xyz[3] = {pos.x, pos.y, pos.z};
    if (v[axis] > 0.0) {
        const double m = d2[axis] / v[axis];
        for (int a = 0; a < 3; ++a) xyz[a] = (a == axis) ? std::ceil(xyz[a]) : xyz[a] + v[a] * m;
        pos.setXYZ(xyz[0], xyz[1], xyz[2]);
    } else if (v[axis] < 0.0) {
        const double m = d1[axis] / (-v[axis]);
        for (int a = 0; a < 3; ++a) xyz[a] = (a == axis) ? std::floor(xyz[a]) : xyz[a] + v[a] * m;
        pos.setXYZ(xyz[0], xyz[1], xyz[2]);
    }
    return pos;
}

// One photoelectron (PhotoElectronParticleType::generateNewParticle/Position/Velocity,
// src/Particle/PhotoElectronParticleType.cpp:9-101, CosineEmission in
// include/random_distribution.hpp:19-28).
static void photo_particle(const Ctx& c, int s, int cm, int64_t step, uint32_t t, const Pos& rel,
                           const double ev[3], int eaxis, Particle& p) {
    const fopis_species& sp = c.p.species[s];
    const uint32_t cc = (uint32_t)s | ((uint32_t)cm << 8), dtag = TAG_EMIT << 24;
    const U2 r0 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | 0);
    const U2 r1 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | 1);
    const U2 r2 = draw2(c.p.seed, t, (uint32_t)step, cc, dtag | 2);
    const double vth = sp.thermal_velocity;
    const double dep = std::asin(2.0 * r0.a - 1.0);
    const double az = 2.0 * M_PI * r0.b;
    double v[3];
    if (eaxis == 0) { v[0] = vth * std::cos(dep) * ev[0]; v[1] = vth * std::sin(dep) * std::cos(az); v[2] = vth * std::sin(dep) * std::sin(az); }
    else if (eaxis == 1) { v[0] = vth * std::sin(dep) * std::sin(az); v[1] = vth * std::cos(dep) * ev[1]; v[2] = vth * std::sin(dep) * std::cos(az); }
    else { v[0] = vth * std::sin(dep) * std::cos(az); v[1] = vth * std::sin(dep) * std::sin(az); v[2] = vth * std::cos(dep) * ev[2]; }
    const double tw = r1.a;
    const double w1 = r1.b, w2 = r2.a;
    double x[3] = {rel.x + (tw - 1.0) * v[0], rel.y + (tw - 1.0) * v[1], rel.z + (tw - 1.0) * v[2]};
    if (eaxis == 0) { x[1] += w1; x[2] += w2; }
    else if (eaxis == 1) { x[0] += w1; x[2] += w2; }
    else { x[0] += w1; x[1] += w2; }
    p.x = x[0]; p.y = x[1]; p.z = x[2]; p.vx = v[0]; p.vy = v[1]; p.vz = v[2];
    p.typeId = s; p.isValid = 1;
}

// Spacecraft::emitParticles, photoelectron branch (src/Spacecraft/Spacecraft.cpp:829-900).
// The loop `for (int i = 0; i < emission_amount_per_area; ++i)` compares an int
// with a double, so ceil(amount) particles leave each lit node.
static int emit(Ctx& c) {
    int bad = 0;
    int64_t emitted = 0;
    const double* sv = c.p.shine_vector;
    int eaxis = -1;
    for (int a = 0; a < 3; ++a) if (std::fabs(sv[a]) == 1.0) { eaxis = a; break; }
    for (auto& o : c.objects) {
        const int s = o.emit_species;
        if (s < 0 || c.p.species[s].kind != FOPIS_SPECIES_PHOTOELECTRON) continue;
        if (eaxis < 0) return -1;  // reference throws std::invalid_argument
        const int surface_sign = (sv[eaxis] > 0.0) ? 1 : -1;
        const double ev[3] = {-sv[0], -sv[1], -sv[2]};
        const double q = c.p.species[s].charge * c.p.species[s].size;
        const double amount = c.p.species[s].emission_amount;
        for (int cm = 0; cm < o.n_cmat; ++cm) {
            Pos pos; pos.setIJK(o.cmat[cm][0], o.cmat[cm][1], o.cmat[cm][2]);
            const bool lit = eaxis == 0 ? isXsurfacePoint(c, o, pos, surface_sign)
                           : eaxis == 1 ? isYsurfacePoint(c, o, pos, surface_sign)
                                        : isZsurfacePoint(c, o, pos, surface_sign);
            if (!lit) continue;
            for (int t = 0; t < amount; ++t) {
                Particle p;
                photo_particle(c, s, cm, c.timestep, (uint32_t)t, pos, ev, eaxis, p);
                const Pos ep = next_cross(p, eaxis);
                if (!surface_charge(c, o, eaxis, ep, s, -q)) bad = 1;
                o.current[s] -= q;
                c.particles[s].push_back(p);
                ++emitted;
            }
        }
    }
    c.emitted_step = emitted;
    return bad;
}
static int emit_secondaries(Ctx& c);
// RootGrid::emitParticlesFromObjects: photoelectrons, then secondaries.
static int emit_all(Ctx& c) {
    const int a = emit(c);
    if (a < 0) return a;
    return a | emit_secondaries(c);
}

// ---------------------------------------------------------------- secondary electrons
// Spacecraft::emitParticles, secondary branch (Spacecraft.cpp:901-937), with
// SecondaryParticleType::generateNewParticles and Whipple's coefficients
// (src/Particle/SecondaryParticleType.cpp:16-194) on the reference's hard-coded
// test material. Deviation: the draws are Philox keyed by the incident's own
// content (crossing point and velocity rounded to 2^-24, species, axis, object)
// and the step, the same function as the GPU path's, not the std::mt19937_64
// streams of the reference, whose values depend on how many incidents came
// before.
static const double kSeeFermi = 9.1, kSeeDeltaMax = 3.0, kSeeEpsMax = 420.0, kSeeZ = 13.0;

static inline uint64_t see_mix(uint64_t h, uint64_t w) {
    h ^= w;
    h *= 0x100000001B3ull;
    h ^= h >> 29;
    return h;
}
static uint64_t incident_key(const Incident& e) {
    const double d[6] = {e.x, e.y, e.z, e.vx, e.vy, e.vz};
    uint64_t h = 0xCBF29CE484222325ull;
    for (int q = 0; q < 6; ++q) h = see_mix(h, (uint64_t)std::llrint(d[q] * 16777216.0));
    return see_mix(h, (uint64_t)e.s | ((uint64_t)e.axis << 8) | ((uint64_t)e.obj << 16));
}
static inline U2 see_draw(const Ctx& c, uint64_t key, uint32_t idx) {
    return draw2(c.p.seed, (uint32_t)key, (uint32_t)(key >> 32), (uint32_t)c.timestep, (TAG_SECONDARY << 24) | idx);
}

// SecondaryParticleType::computeWhipple{TrueSecondary,Inelastic,Elastic}Coeff.
static double whipple_true(double E, double th) {
    return (1.114 * kSeeDeltaMax / std::cos(th)) * std::pow(kSeeEpsMax / E, 0.35) *
           (1.0 - std::exp(-2.28 * std::cos(th) * std::pow(E / kSeeEpsMax, 1.35)));
}
static double whipple_inelastic(double E, double th) {
    const double eta1 = 1.0 - std::pow(2.0 / E, 0.037 * kSeeZ);
    const double eta2 = 0.1 * std::exp(-E / 5000.0);
    double eta0 = 0.0;
    if (E > 50.0 && E < 1000.0) eta0 = std::log(E / 50.0) / std::log(20.0);
    else if (E > 1000.0) eta0 = 1.0;
    return eta0 * (eta1 + eta2) * (7.37 * std::pow(kSeeZ, -0.56875)) * (1.0 - std::cos(th));
}
static double whipple_elastic(double E) {
    return (1.0 / 13.54) * std::pow(kSeeFermi, 4) / (16.0 * (std::pow(E + kSeeFermi, 3) + std::pow(kSeeFermi, 3)));
}

// SecondaryParticleType::generateNewParticles for one incident.
static void see_generate(const Ctx& c, const Incident& e, int sec, std::vector<Particle>& out) {
    const uint64_t key = incident_key(e);
    const double m_in = c.p.species[e.s].mass, q_in = c.p.species[e.s].charge;
    const double v2 = e.vx * e.vx + e.vy * e.vy + e.vz * e.vz;
    const double vin[3] = {e.vx, e.vy, e.vz};
    const double E = 0.5 * m_in * v2 * c.p.energy_ev;                  // getIncidentEnergyInElectronVolt
    const double th = std::acos(std::fabs(vin[e.axis]) / std::sqrt(v2));    // getIncidentAngle
    const double r = q_in < 0.0 ? whipple_elastic(E) : 0.0;
    const double eta = q_in < 0.0 ? whipple_inelastic(E, th) : 0.0;
    double delta = whipple_true(E, th);
    const U2 u = see_draw(c, key, 0);
    int kind, count;
    if (u.a < r) { kind = 1; count = 1; }
    else if (u.a < r + eta) { kind = 2; count = 1; }
    else {
        delta /= (1.0 - r - eta);
        kind = 3;
        count = (int)std::floor(delta) + ((u.b < delta - std::floor(delta)) ? 1 : 0);
    }
    double speed = c.p.species[sec].thermal_velocity;                   // true secondaries
    if (kind == 2) {
        const double share = see_draw(c, key, 1).a;                        // of the incident energy
        speed = std::sqrt(2.0 * (share * 0.5 * m_in * v2) / c.p.species[sec].mass);
    }
    for (int m = 0; m < count; ++m) {
        double v[3] = {vin[0], vin[1], vin[2]};
        if (kind == 1) {
            v[e.axis] = -v[e.axis];
        } else {
            const U2 ua = see_draw(c, key, (uint32_t)(2 + m));
            const double dep = std::asin(2.0 * ua.a - 1.0), az = 2.0 * M_PI * ua.b;
            const double sgn = vin[e.axis] > 0.0 ? -1.0 : 1.0;
            const double cn = speed * std::cos(dep) * sgn;
            const double sa = speed * std::sin(dep) * std::cos(az), sb = speed * std::sin(dep) * std::sin(az);
            if (e.axis == 0) { v[0] = cn; v[1] = sa; v[2] = sb; }
            else if (e.axis == 1) { v[0] = sb; v[1] = cn; v[2] = sa; }
            else { v[0] = sa; v[1] = sb; v[2] = cn; }
        }
        Particle p;
        p.vx = v[0]; p.vy = v[1]; p.vz = v[2];
        p.x = e.x + e.trem * v[0]; p.y = e.y + e.trem * v[1]; p.z = e.z + e.trem * v[2];
        p.typeId = sec; p.isValid = 1;
        out.push_back(p);
    }
}

// The pending incidents' secondaries: a secondary inside the body is absorbed at
// once on a face of another axis (its incident, recorded by the reference into
// the list it is iterating and cleared right after, emits nothing); the others
// take their charge off the face they left, at the next crossing of their
// back-dated position along the incident axis, and are appended. The list is
// then cleared (Spacecraft::clearIncidentEvents).
static int emit_secondaries(Ctx& c) {
    int bad = 0;
    int64_t emitted = 0;
    for (const Incident& e : c.incidents) {
        Object& o = c.objects[e.obj];
        const int sec = o.secondary_species;
        if (sec < 0) continue;
        const double q = c.p.species[sec].charge * c.p.species[sec].size;
        std::vector<Particle> gen;
        see_generate(c, e, sec, gen);
        for (Particle& p : gen) {
            if (isContaining(c, o, posXYZ(p.x, p.y, p.z))) {
                Pos hit;
                const int ax = first_face(c, o, p, e.axis, hit);
                if (ax >= 0 && !surface_charge(c, o, ax, hit, sec, q)) bad = 1;
                o.current[sec] += q;
                continue;
            }
            Particle old = p;
            old.x -= p.vx; old.y -= p.vy; old.z -= p.vz;
            const Pos ep = next_cross(old, e.axis);
            if (!surface_charge(c, o, e.axis, ep, sec, -q)) bad = 1;
            o.current[sec] -= q;
            c.particles[sec].push_back(p);
            ++emitted;
        }
    }
    c.incidents.clear();
    c.emitted_step += emitted;
    return bad;
}

// Grid::removeInvalidParticles (src/Grid/GridParticleTreatment.cpp:93-102).
static void remove_invalid(Ctx& c) {
    for (auto& v : c.particles)
        v.erase(std::remove_if(v.begin(), v.end(), [](const Particle& p) { return p.isValid == 0; }), v.end());
}

// RootGrid::resetObjects (RootGridObject.cpp:162-173).
static void reset_objects(Ctx& c) {
    for (auto& o : c.objects) std::fill(o.current.begin(), o.current.end(), 0.0);
}

// RootGrid::mainLoopEM (src/Grid/RootGrid/RootGrid.cpp:145-191).
static int main_loop_em(Ctx& c) {
    reset_objects(c);
    update_velocity_em(c);
    int bad = emit_all(c);
    update_position_em(c);
    inject(c, nullptr);
    bad |= update_rho(c);
    update_efield_fdtd(c);
    update_bfield(c);
    if (c.timestep % 50 == 0) remove_invalid(c);
    ++c.timestep;
    return bad;
}

// RootGrid::mainLoopES (src/Grid/RootGrid/RootGrid.cpp:82-143).
static int main_loop(Ctx& c) {
    if (c.em) return main_loop_em(c);
    reset_objects(c);
    update_velocity(c);
    int bad = emit_all(c);
    update_position(c);
    inject(c, nullptr);
    bad |= update_rho(c);
    solve_poisson(c);
    update_efield(c);
    if (c.timestep % 50 == 0) remove_invalid(c);
    ++c.timestep;
    return bad;
}

// Gauss-Jordan inverse with partial pivoting (stands in for Eigen's inverse).
static bool invert(std::vector<double>& A, int n) {
    std::vector<double> I((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) I[(size_t)i * n + i] = 1.0;
    for (int k = 0; k < n; ++k) {
        int piv = k; double best = std::fabs(A[(size_t)k * n + k]);
        for (int r = k + 1; r < n; ++r) { double v = std::fabs(A[(size_t)r * n + k]); if (v > best) { best = v; piv = r; } }
        if (best == 0.0) return false;
        if (piv != k) for (int col = 0; col < n; ++col) { std::swap(A[(size_t)k * n + col], A[(size_t)piv * n + col]); std::swap(I[(size_t)k * n + col], I[(size_t)piv * n + col]); }
        const double d = 1.0 / A[(size_t)k * n + k];
        for (int col = 0; col < n; ++col) { A[(size_t)k * n + col] *= d; I[(size_t)k * n + col] *= d; }
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; ++r) {
            if (r == k) continue;
            const double f = A[(size_t)r * n + k];
            if (f == 0.0) continue;
            for (int col = 0; col < n; ++col) { A[(size_t)r * n + col] -= f * A[(size_t)k * n + col]; I[(size_t)r * n + col] -= f * I[(size_t)k * n + col]; }
        }
    }
    A.swap(I);
    return true;
}

// Cmatrix::total (include/Spacecraft/Cmatrix.hpp:36-44).
static double cmat_total(const std::vector<double>& C) { double s = 0; for (double v : C) s += v; return s; }

// Spacecraft::initializeChargeMapOffset (Spacecraft.cpp:160-183).
static void charge_map_offset(Ctx& c, Object& o) {
    if (o.initial_potential_offset == 0.0) return;
    o.potential = o.initial_potential_offset;
    for (int i = 0; i < o.n_cmat; ++i) {
        double d = 0.0;
        for (int j = 0; j < o.n_cmat; ++j) d += o.C[(size_t)i * o.n_cmat + j] * o.potential;
        o.charge_map[i] += d;  // species row 0
    }
}

// RootGrid::initializeObjectsCmatrix (RootGridObject.cpp:77-148): column c holds
// phi at every surface node for rho = 1 at node c; the matrix stored is
// capacity_matrix(col = c, row = r) and is then inverted.
static bool build_cmatrix(Ctx& c, Object& o) {
    const int n = o.n_cmat;
    std::vector<double> M((size_t)n * n);
    for (auto& r : c.rho) r.zero();
    for (int col = 0; col < n; ++col) {
        c.phi.zero();
        const auto& nd = o.cmat[col];
        c.rho[0](nd[0], nd[1], nd[2]) = 1.0;
        solve_poisson(c);
        for (int row = 0; row < n; ++row) {
            const auto& t = o.cmat[row];
            M[(size_t)col * n + row] = c.phi(t[0], t[1], t[2]);
        }
        c.rho[0](nd[0], nd[1], nd[2]) = 0.0;
    }
    c.phi.zero();
    if (!invert(M, n)) return false;
    o.C.swap(M);
    o.total_cmat_value = cmat_total(o.C);
    o.has_C = true;
    charge_map_offset(c, o);
    return true;
}

// ---------------------------------------------------------------- .obj loader
// ObjectUtils::getObjectNodesFromObjFile (src/Spacecraft/ObjectUtils.cpp:9-333),
// without textures and the connectivity list (not used on the ES path).
// Outputs glue-layout indices (getRelativePositionOnRootWithGlue adds 1).
static int parse_obj(const char* path, int nx, int ny, int nz, std::vector<std::array<int, 3>>& nodes,
                     std::vector<std::array<int, 3>>& cells) {
    std::ifstream in(path);
    if (!in) return -1;
    std::vector<int> node_map((size_t)nx * ny * nz, -1);
    auto nm = [&](int i, int j, int k) -> int& { return node_map[((size_t)i * ny + j) * nz + k]; };
    std::vector<unsigned char> xf((size_t)nx * ny * nz, 0), yf(xf.size(), 0), zf(xf.size(), 0);
    auto fi = [&](int i, int j, int k) { return ((size_t)i * ny + j) * nz + k; };
    std::vector<std::array<int, 3>> verts;
    std::vector<std::array<int, 4>> faces;
    std::string line;
    while (std::getline(in, line)) {
        if (line.size() > 2 && line[0] == 'v' && line[1] == ' ') {
            std::istringstream ss(line.substr(2));
            int a, b, d; ss >> a >> b >> d;
            verts.push_back({a + nx / 2, b + ny / 2, d + nz / 2});
        } else if (line.size() > 2 && line[0] == 'f' && line[1] == ' ') {
            std::istringstream ss(line.substr(2));
            std::array<int, 4> f{};
            for (int t = 0; t < 4; ++t) { std::string tok; ss >> tok; f[t] = std::atoi(tok.substr(0, tok.find('/')).c_str()); }
            faces.push_back(f);
        }
    }
    for (const auto& f : faces) {
        const auto& v1 = verts[f[0] - 1]; const auto& v2 = verts[f[1] - 1];
        const auto& v3 = verts[f[2] - 1]; const auto& v4 = verts[f[3] - 1];
        int ax = -1;
        for (int a = 0; a < 3; ++a) if (v1[a] == v2[a] && v1[a] == v3[a] && v1[a] == v4[a]) { ax = a; break; }
        if (ax < 0) return -2;
        const int b1 = (ax == 0) ? 1 : 0, b2 = (ax == 2) ? 1 : 2;
        const int mn1 = std::min({v1[b1], v2[b1], v3[b1], v4[b1]}), mx1 = std::max({v1[b1], v2[b1], v3[b1], v4[b1]});
        const int mn2 = std::min({v1[b2], v2[b2], v3[b2], v4[b2]}), mx2 = std::max({v1[b2], v2[b2], v3[b2], v4[b2]});
        for (int u = mn1; u <= mx1; ++u)
            for (int w = mn2; w <= mx2; ++w) {
                int ijk[3]; ijk[ax] = v1[ax]; ijk[b1] = u; ijk[b2] = w;
                if (nm(ijk[0], ijk[1], ijk[2]) < 0) { nm(ijk[0], ijk[1], ijk[2]) = (int)nodes.size(); nodes.push_back({ijk[0], ijk[1], ijk[2]}); }
                if (u != mx1 && w != mx2) { auto& fm = (ax == 0 ? xf : (ax == 1 ? yf : zf)); fm[fi(ijk[0], ijk[1], ijk[2])] = 1; }
            }
    }
    std::vector<int> cnt((size_t)nx * ny * nz, 0);
    auto scan = [&](int axis) {
        const int na = axis == 0 ? nx : (axis == 1 ? ny : nz);
        const int o1 = axis == 0 ? ny : nx, o2 = axis == 2 ? ny : nz;
        const auto& fm = (axis == 0 ? xf : (axis == 1 ? yf : zf));
        for (int p = 0; p < o1 - 1; ++p)
            for (int q = 0; q < o2 - 1; ++q)
                for (int lo = 0; lo < na - 1; ++lo) {
                    auto at = [&](int s) { int ijk[3]; ijk[axis] = s; ijk[axis == 0 ? 1 : 0] = p; ijk[axis == 2 ? 1 : 2] = q; return fi(ijk[0], ijk[1], ijk[2]); };
                    if (!fm[at(lo)]) continue;
                    for (int up = lo + 1; up < na - 1; ++up) {
                        if (fm[at(up)]) { for (int s = lo; s < up; ++s) cnt[at(s)] += 1; lo = up; break; }
                    }
                }
    };
    scan(0); scan(1); scan(2);
    for (int i = 0; i < nx - 1; ++i) for (int j = 0; j < ny - 1; ++j) for (int k = 0; k < nz - 1; ++k)
        if (cnt[fi(i, j, k)] == 3) cells.push_back({i + 1, j + 1, k + 1});
    for (auto& n : nodes) { n[0] += 1; n[1] += 1; n[2] += 1; }
    return 0;
}

// ---------------------------------------------------------------- fixed-point replay
// Integer CIC weights of the split-precision deposit: each in-cell offset is
// rounded to 17 fractional bits (round half to even) and the eight corner
// weights are products of (2^17 - a) or a per axis, so they sum to 2^51.
static inline int64_t qoff(float o) { return (int64_t)std::nearbyintf(o * 131072.0f); }

}  // namespace orc

using namespace orc;

extern "C" {

void* orc_create(const fopis_params* p) {
    Ctx* c = new Ctx();
    init_ctx(*c, p);
    return c;
}
void orc_destroy(void* h) { delete (Ctx*)h; }
int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

// Philox known-answer access for tests.
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox4x32_10(c, key[0], key[1]);
    for (int t = 0; t < 4; ++t) out[t] = c[t];
}

// The oracle's Position::setXYZ on n points: ijk[3n], d[6n] = dx1,dy1,dz1,dx2,dy2,dz2.
// The oracle's zigzag relay point (relay, used by update_position_em) per pair of
// new and old positions.
void orc_relay(const double* new_xyz, const double* old_xyz, int64_t n, double* out) {
    for (int64_t t = 0; t < n; ++t) {
        const Pos nw = posXYZ(new_xyz[3 * t], new_xyz[3 * t + 1], new_xyz[3 * t + 2]);
        const Pos od = posXYZ(old_xyz[3 * t], old_xyz[3 * t + 1], old_xyz[3 * t + 2]);
        out[3 * t] = relay(nw.i, od.i, nw.x, od.x);
        out[3 * t + 1] = relay(nw.j, od.j, nw.y, od.y);
        out[3 * t + 2] = relay(nw.k, od.k, nw.z, od.z);
    }
}
void orc_position(const double* xyz, int64_t n, int32_t* ijk, double* d) {
    for (int64_t t = 0; t < n; ++t) {
        const Pos p = posXYZ(xyz[3 * t], xyz[3 * t + 1], xyz[3 * t + 2]);
        ijk[3 * t] = p.i; ijk[3 * t + 1] = p.j; ijk[3 * t + 2] = p.k;
        d[6 * t] = p.dx1; d[6 * t + 1] = p.dy1; d[6 * t + 2] = p.dz1;
        d[6 * t + 3] = p.dx2; d[6 * t + 4] = p.dy2; d[6 * t + 5] = p.dz2;
    }
}

void orc_set_solver(void* h, int mode, int max_post_loop, double exact_tol) {
    Ctx* c = (Ctx*)h;
    c->solver_mode = mode;
    if (max_post_loop > 0) c->max_post_loop = max_post_loop;
    if (exact_tol > 0) c->exact_tol = exact_tol;
}
void orc_solver_stats(void* h, int* iterations, double* residual) {
    Ctx* c = (Ctx*)h; *iterations = c->last_iterations; *residual = c->last_residual;
}
// RootGrid::checkPhiResidual on the current phi and rho (glue of periodic axes
// refreshed first, as the PSOR's exchanges leave it).
double orc_pointwise_residual(void* h) {
    Ctx* c = (Ctx*)h;
    copy_field_glue(*c, c->phi);
    return check_phi_residual(*c);
}

int orc_add_object(void* h, const fopis_object_desc* d) {
    Ctx* c = (Ctx*)h;
    Object o;
    o.n_cmat = d->n_cmat;
    o.cmat.resize(d->n_cmat);
    o.node_to_cmat.assign((size_t)c->cx * c->cy * c->cz, -1);
    for (int m = 0; m < d->n_cmat; ++m) {
        o.cmat[m] = {d->cmat_nodes[3 * m], d->cmat_nodes[3 * m + 1], d->cmat_nodes[3 * m + 2]};
        o.node_to_cmat[nodeIndex(*c, o.cmat[m][0], o.cmat[m][1], o.cmat[m][2])] = m;
    }
    o.cell_map.assign((size_t)(c->nx + 1) * (c->ny + 1) * (c->nz + 1), 0);
    for (int m = 0; m < d->n_cells; ++m)
        o.cell_map[cellIndex(*c, d->cells[3 * m], d->cells[3 * m + 1], d->cells[3 * m + 2])] = 1;
    o.charge_map.assign((size_t)c->nsp * o.n_cmat, 0.0);
    o.tmp_charge_map.assign((size_t)c->nsp * o.n_cmat, 0.0);
    o.current.assign(c->nsp, 0.0);
    o.is_potential_fixed = d->is_potential_fixed;
    o.fixed_potential = d->fixed_potential;
    o.initial_potential_offset = d->initial_potential_offset;
    o.emit_species = d->emit_species;
    o.secondary_species = d->secondary_species;
    o.dielectric = d->dielectric;
    if (o.dielectric) o.capacitance.assign(d->capacitance, d->capacitance + d->n_cmat);
    c->objects.push_back(std::move(o));
    return (int)c->objects.size() - 1;
}
int orc_build_cmatrix(void* h, int obj) {
    Ctx* c = (Ctx*)h;
    return build_cmatrix(*c, c->objects[obj]) ? 0 : -1;
}
int orc_set_cmatrix(void* h, int obj, const double* C, int n) {
    Ctx* c = (Ctx*)h; Object& o = c->objects[obj];
    if (n != o.n_cmat) return -1;
    o.C.assign(C, C + (size_t)n * n);
    o.total_cmat_value = cmat_total(o.C);
    o.has_C = true;
    charge_map_offset(*c, o);
    return 0;
}
int orc_get_cmatrix(void* h, int obj, double* C, int n) {
    Ctx* c = (Ctx*)h; Object& o = c->objects[obj];
    if (n != o.n_cmat || !o.has_C) return -1;
    std::memcpy(C, o.C.data(), sizeof(double) * (size_t)n * n);
    return 0;
}
void orc_get_object(void* h, int obj, double* V, double* Q, double* current) {
    Ctx* c = (Ctx*)h; Object& o = c->objects[obj];
    *V = o.potential; *Q = o.total_charge;
    for (int s = 0; s < c->nsp; ++s) current[s] = o.current[s];
}
void orc_get_charge_map(void* h, int obj, double* out) {
    Ctx* c = (Ctx*)h; Object& o = c->objects[obj];
    std::memcpy(out, o.charge_map.data(), sizeof(double) * o.charge_map.size());
}

int64_t orc_load_particles(void* h, int s, const void* aos, int64_t n) {
    Ctx* c = (Ctx*)h;
    const Particle* p = (const Particle*)aos;
    int64_t k = 0;
    for (int64_t t = 0; t < n; ++t) if (p[t].isValid) { Particle q = p[t]; q.typeId = s; c->particles[s].push_back(q); ++k; }
    return k;
}
int64_t orc_num_particles(void* h, int s) {
    Ctx* c = (Ctx*)h; int64_t k = 0;
    for (const auto& p : c->particles[s]) k += p.isValid;
    return k;
}
int64_t orc_get_particles(void* h, int s, void* aos, int64_t cap) {
    Ctx* c = (Ctx*)h; Particle* out = (Particle*)aos; int64_t k = 0;
    for (const auto& p : c->particles[s]) if (p.isValid) { if (k < cap) out[k] = p; ++k; }
    return k;
}
void orc_generate_ambient(void* h) { generate_ambient(*(Ctx*)h); }

void orc_reset_objects(void* h) { reset_objects(*(Ctx*)h); }
void orc_update_velocity(void* h) {
    Ctx* c = (Ctx*)h;
    if (c->em) update_velocity_em(*c); else update_velocity(*c);
}
int orc_emit(void* h) { return emit_all(*(Ctx*)h); }
// The pending incident list as records of 10 doubles (object, species, axis,
// remaining time, x, y, z, vx, vy, vz), the layout of fopis_get_incidents.
int64_t orc_get_incidents(void* h, double* out, int64_t cap) {
    Ctx* c = (Ctx*)h;
    const int64_t n = (int64_t)c->incidents.size();
    for (int64_t t = 0; t < std::min(n, cap); ++t) {
        const Incident& e = c->incidents[t];
        double* r = out + 10 * t;
        r[0] = e.obj; r[1] = e.s; r[2] = e.axis; r[3] = e.trem;
        r[4] = e.x; r[5] = e.y; r[6] = e.z; r[7] = e.vx; r[8] = e.vy; r[9] = e.vz;
    }
    return n;
}
void orc_set_incidents(void* h, const double* in, int64_t n) {
    Ctx* c = (Ctx*)h;
    c->incidents.clear();
    for (int64_t t = 0; t < n; ++t) {
        const double* r = in + 10 * t;
        c->incidents.push_back(Incident{(int)r[0], (int)r[1], (int)r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9]});
    }
}
void orc_update_position(void* h) {
    Ctx* c = (Ctx*)h;
    if (c->em) update_position_em(*c); else update_position(*c);
}
void orc_inject(void* h, int64_t* counts) { inject(*(Ctx*)h, counts); }
int orc_update_rho(void* h) { return update_rho(*(Ctx*)h); }
void orc_solve_poisson(void* h) { solve_poisson(*(Ctx*)h); }
void orc_update_efield(void* h) {
    Ctx* c = (Ctx*)h;
    if (c->em) update_efield_fdtd(*c); else update_efield(*c);
}
void orc_update_bfield(void* h) { if (((Ctx*)h)->em) update_bfield(*(Ctx*)h); }
double orc_bfield_energy(void* h) { return ((Ctx*)h)->em ? bfield_energy(*(Ctx*)h) : 0.0; }
void orc_remove_invalid(void* h) { remove_invalid(*(Ctx*)h); }
int orc_main_loop(void* h, int n) { int bad = 0; for (int t = 0; t < n; ++t) bad |= main_loop(*(Ctx*)h); return bad; }
// Grid::initialize (src/Grid/Grid.cpp:23-36).
int orc_initialize(void* h) {
    Ctx* c = (Ctx*)h;
    int bad = update_rho(*c);
    solve_poisson(*c);
    if (c->em) {
        update_efield_em_from_phi(*c);
        update_bfield(*c);
    } else {
        update_efield(*c);
    }
    return bad;
}
void orc_set_timestep(void* h, int64_t t) { ((Ctx*)h)->timestep = t; }
int64_t orc_get_timestep(void* h) { return ((Ctx*)h)->timestep; }
void orc_step_counts(void* h, int64_t* injected, int64_t* emitted, int64_t* absorbed) {
    Ctx* c = (Ctx*)h; *injected = c->injected_step; *emitted = c->emitted_step; *absorbed = c->absorbed_step;
}

// The EM Yee array of a field selector (32..37), or null.
static ArrB* yee_array(Ctx* c, int which) {
    if (!c->em) return nullptr;
    switch (which) {
        case 32: return &c->fex;
        case 33: return &c->fey;
        case 34: return &c->fez;
        case 35: return &c->fbx;
        case 36: return &c->fby;
        case 37: return &c->fbz;
    }
    return nullptr;
}

// which: 0 phi, 1 rho0, 2..4 E ref, 5..7 B ref, 8..10 J ref, 16+s rho species,
// 32..34 edge E, 35..37 face B, 38..40 edge J (their own shapes, fopis_field numbering)
int orc_get_field(void* h, int which, double* out) {
    Ctx* c = (Ctx*)h;
    if (ArrB* b = yee_array(c, which)) {
        std::memcpy(out, b->v.data(), sizeof(double) * b->v.size());
        return 0;
    }
    if (which >= 8 && which <= 10) {
        if (!c->em) return -1;
        // RootGrid::updateReferenceCurrent (RootGridField.cpp:1256-1285)
        Arr3 r;
        r.resize(c->cx, c->cy, c->cz);
        for (int i = 1; i < c->cx - 1; ++i) for (int j = 1; j < c->cy - 1; ++j) for (int k = 1; k < c->cz - 1; ++k)
            r(i, j, k) = which == 8 ? 0.5 * (c->jx(i - 1, j, k) + c->jx(i, j, k))
                                    : (which == 9 ? 0.5 * (c->jy(i, j - 1, k) + c->jy(i, j, k))
                                                  : 0.5 * (c->jz(i, j, k - 1) + c->jz(i, j, k)));
        copy_field_glue(*c, r);
        std::memcpy(out, r.v.data(), sizeof(double) * r.v.size());
        return 0;
    }
    const Arr3* a = nullptr;
    switch (which) {
        case 0: a = &c->phi; break;
        case 1: a = &c->rho[0]; break;
        case 2: a = &c->exref; break;
        case 3: a = &c->eyref; break;
        case 4: a = &c->ezref; break;
        case 5: a = c->em ? &c->bxref : nullptr; break;
        case 6: a = c->em ? &c->byref : nullptr; break;
        case 7: a = c->em ? &c->bzref : nullptr; break;
        case 32: a = &c->ex; break;
        case 33: a = &c->ey; break;
        case 34: a = &c->ez; break;
        case 38: a = c->em ? &c->jx : nullptr; break;
        case 39: a = c->em ? &c->jy : nullptr; break;
        case 40: a = c->em ? &c->jz : nullptr; break;
        default:
            if (which >= 16 && which < 16 + c->nsp) a = &c->rho[which - 15];
    }
    if (!a) return -1;
    std::memcpy(out, a->v.data(), sizeof(double) * a->v.size());
    return 0;
}

// First index and extent per axis of a field (index bases of the EM arrays).
int orc_field_shape(void* h, int which, int* lo, int* n) {
    Ctx* c = (Ctx*)h;
    if (ArrB* b = yee_array(c, which)) {
        for (int a = 0; a < 3; ++a) { lo[a] = b->lo[a]; n[a] = b->n[a]; }
        return 0;
    }
    const Arr3* a = nullptr;
    if (which >= 32 && which <= 34) a = which == 32 ? &c->ex : (which == 33 ? &c->ey : &c->ez);
    if (which >= 38 && which <= 40 && c->em) a = which == 38 ? &c->jx : (which == 39 ? &c->jy : &c->jz);
    lo[0] = lo[1] = lo[2] = 0;
    if (a) { n[0] = a->cx; n[1] = a->cy; n[2] = a->cz; }
    else { n[0] = c->cx; n[1] = c->cy; n[2] = c->cz; }
    return 0;
}
int orc_set_field(void* h, int which, const double* in) {
    Ctx* c = (Ctx*)h;
    if (ArrB* b = yee_array(c, which)) {
        std::memcpy(b->v.data(), in, sizeof(double) * b->v.size());
        return 0;
    }
    Arr3* a = which == 0 ? &c->phi : (which == 1 ? &c->rho[0] : nullptr);
    if (c->em && which >= 38 && which <= 40) a = which == 38 ? &c->jx : (which == 39 ? &c->jy : &c->jz);
    if (!a) return -1;
    std::memcpy(a->v.data(), in, sizeof(double) * a->v.size());
    return 0;
}

// Grid::getParticleEnergy (GridParticleTreatment.cpp:104-118) and
// Field::getEfieldEnergy (Field.cpp:194-213).
void orc_energy(void* h, double* pe, double* fe) {
    Ctx* c = (Ctx*)h;
    double res = 0.0;
    for (int s = 0; s < c->nsp; ++s) {
        double e = 0.0;
        for (const auto& p : c->particles[s]) if (p.isValid) e += p.vx * p.vx + p.vy * p.vy + p.vz * p.vz;
        res += 0.5 * c->p.species[s].mass * e * c->p.species[s].size;
    }
    *pe = res;
    double en = 0.0;
    const int X = c->cx, Y = c->cy, Z = c->cz;
    for (int i = 1; i < X - 1; ++i) for (int j = 1; j < Y - 1; ++j) for (int k = 1; k < Z - 1; ++k) {
        if (c->em) {   // the Yee edges of the EM mode
            if (i < X - 2) en += c->fex(i, j, k) * c->fex(i, j, k);
            if (j < Y - 2) en += c->fey(i, j, k) * c->fey(i, j, k);
            if (k < Z - 2) en += c->fez(i, j, k) * c->fez(i, j, k);
            continue;
        }
        if (i < X - 2) en += c->ex(i, j, k) * c->ex(i, j, k);
        if (j < Y - 2) en += c->ey(i, j, k) * c->ey(i, j, k);
        if (k < Z - 2) en += c->ez(i, j, k) * c->ez(i, j, k);
    }
    *fe = 0.5 * c->p.eps0 * en;
}

int orc_parse_obj(const char* path, int nx, int ny, int nz, int32_t* nodes, int cap_nodes, int* n_nodes,
                  int32_t* cells, int cap_cells, int* n_cells) {
    std::vector<std::array<int, 3>> nd, cl;
    const int rc = parse_obj(path, nx, ny, nz, nd, cl);
    if (rc) return rc;
    *n_nodes = (int)nd.size(); *n_cells = (int)cl.size();
    for (int t = 0; t < (int)nd.size() && t < cap_nodes; ++t) for (int a = 0; a < 3; ++a) nodes[3 * t + a] = nd[t][a];
    for (int t = 0; t < (int)cl.size() && t < cap_cells; ++t) for (int a = 0; a < 3; ++a) cells[3 * t + a] = cl[t][a];
    return 0;
}

// Fixed-point replay of the split-precision CIC deposit for one species:
// out[node] += integer corner weight (sum 2^51 per particle). cell is the
// particle's glue-layout node cell packed as (i << 20) | (j << 10) | k.
void orc_fixed_deposit(const fopis_params* p, const int32_t* cell, const float* ox, const float* oy,
                       const float* oz, int64_t n, int64_t* out) {
    const int cy = p->ny + 2, cz = p->nz + 2;
    const int64_t A = 131072;
    const int64_t sj = cz, si = (int64_t)cy * cz;
    for (int64_t t = 0; t < n; ++t) {
        if (cell[t] < 0) continue;
        const int64_t a = qoff(ox[t]), b = qoff(oy[t]), d = qoff(oz[t]);
        const int64_t wx[2] = {A - a, a}, wy[2] = {A - b, b}, wz[2] = {A - d, d};
        const int ci = (cell[t] >> 20) & 1023, cj = (cell[t] >> 10) & 1023, ck = cell[t] & 1023;
        const int64_t base = ((int64_t)ci * cy + cj) * cz + ck;
        for (int di = 0; di < 2; ++di) for (int dj = 0; dj < 2; ++dj) for (int dk = 0; dk < 2; ++dk)
            out[base + di * si + dj * sj + dk] += wx[di] * wy[dj] * wz[dk];
    }
}
// Periodic fold of an integer node array (same semantics as fold_node_scalar).
void orc_fixed_fold(const fopis_params* p, int64_t* a) {
    const int X = p->nx + 2, Y = p->ny + 2, Z = p->nz + 2;
    auto at = [&](int i, int j, int k) -> int64_t& { return a[((size_t)i * Y + j) * Z + k]; };
    if (p->boundary[0] == 'P')
        for (int j = 0; j < Y; ++j) for (int k = 0; k < Z; ++k) {
            int64_t s0 = at(0, j, k) + at(X - 2, j, k), s1 = at(1, j, k) + at(X - 1, j, k);
            at(0, j, k) = s0; at(X - 2, j, k) = s0; at(1, j, k) = s1; at(X - 1, j, k) = s1;
        }
    if (p->boundary[2] == 'P')
        for (int i = 0; i < X; ++i) for (int k = 0; k < Z; ++k) {
            int64_t s0 = at(i, 0, k) + at(i, Y - 2, k), s1 = at(i, 1, k) + at(i, Y - 1, k);
            at(i, 0, k) = s0; at(i, Y - 2, k) = s0; at(i, 1, k) = s1; at(i, Y - 1, k) = s1;
        }
    if (p->boundary[4] == 'P')
        for (int i = 0; i < X; ++i) for (int j = 0; j < Y; ++j) {
            int64_t s0 = at(i, j, 0) + at(i, j, Z - 2), s1 = at(i, j, 1) + at(i, j, Z - 1);
            at(i, j, 0) = s0; at(i, j, Z - 2) = s0; at(i, j, 1) = s1; at(i, j, Z - 1) = s1;
        }
}

}  // extern "C"
