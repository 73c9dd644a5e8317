// api.cu — the C ABI of libfopis_gpu.so (include/fopis_gpu.h).
//
// Every entry point catches C++ exceptions and returns an fopis_status; the
// message of the last failure is kept per context (fopis_last_error).
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

using namespace fopis;

namespace {

thread_local std::string g_create_error;

constexpr uint32_t kFatalBits = FOPIS_DEV_PARTICLE_OVERFLOW | FOPIS_DEV_ABSORB_OVERFLOW | FOPIS_DEV_BAD_CMAT_NODE |
                                FOPIS_DEV_NONFINITE | FOPIS_DEV_RHO_OVERFLOW;

template <typename F>
int guarded(void* h, F&& f) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return FOPIS_ERR_ARG;
    try {
        return f(*c);
    } catch (const CudaError& e) {
        c->err = std::string("CUDA error ") + cudaGetErrorString(e.code) + " at " + e.where;
        return FOPIS_ERR_CUDA;
    } catch (const ApiError& e) {
        c->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        c->err = "host allocation failed";
        return FOPIS_ERR_NOMEM;
    } catch (const std::exception& e) {
        c->err = e.what();
        return FOPIS_ERR_ARG;
    }
}

// Reads the device scalars and turns latched device errors into a status.
int check_device(Ctx& c) {
    sync_scalars(c);
    const uint32_t st = c.h_sc->status;
    if (st & (FOPIS_DEV_PARTICLE_OVERFLOW | FOPIS_DEV_ABSORB_OVERFLOW)) {
        c.err = "particle or absorbed-list capacity exceeded (device status " + std::to_string(st) + ")";
        return FOPIS_ERR_CAPACITY;
    }
    if (st & FOPIS_DEV_RHO_OVERFLOW) {
        c.err = "device status " + std::to_string(st) + ": a node's fixed-point charge sum passed 2^64 "
                "(more than 8192 full particle weights of one species on one node)";
        return FOPIS_ERR_DEVICE;
    }
    if (st & kFatalBits) {
        c.err = "device status " + std::to_string(st) + ": invalid surface node or non-finite particle state";
        return FOPIS_ERR_DEVICE;
    }
    return FOPIS_OK;
}

void update_currents(Ctx& c) {
    for (size_t o = 0; o < c.objs.size(); ++o)
        for (int s = 0; s < c.nsp; ++s) {
            const double q = c.p.species[s].charge * c.p.species[s].size;
            c.objs[o].current[s] =
                q * ((double)c.h_sc->absorbed_by[o][s] - (double)c.h_sc->emitted_by[o][s]);
        }
    int64_t ab = 0, em = 0;
    for (size_t o = 0; o < c.objs.size(); ++o)
        for (int s = 0; s < c.nsp; ++s) { ab += c.h_sc->absorbed_by[o][s]; em += c.h_sc->emitted_by[o][s]; }
    c.absorbed_step = ab;
    c.emitted_step = em;
}

void step_begin(Ctx& c) {
    objects_step_begin(c);
    FOPIS_CUDA(cudaMemsetAsync(c.d_sc->energy, 0, sizeof(c.d_sc->energy), c.st));
    c.step_vcycles = 0;
    c.step_solves = 0;
}

double solve_tol(const Ctx& c) { return c.p.poisson_tol > 0 ? c.p.poisson_tol : 1e-8; }
int solve_cap(const Ctx& c) { return c.p.max_vcycles > 0 ? c.p.max_vcycles : 100; }

// One Poisson solve with the start guess of the context's mode.
//  WARM     the current phi (the reference's PSOR continues from it).
//  HISTORY  the first solve of a step (plasma charge only) starts from the
//           previous step's first solve, the second solve (after the
//           capacity-matrix redistribution) from the first plus the two
//           previous steps' conductor responses phi_final - phi_first, scaled
//           by the least-squares fit of this step's redistributed surface
//           charge to theirs.
//  LEARNED  HISTORY with the first solve seeded by the U-Net's increment.
// Every start converges to the same tolerance. A solve that fails to converge
// from the learned guess is redone from the history start, and one from a
// warm start is redone from zero.

// The history becomes usable; on its first valid step phi^{n-2} = phi^{n-1}.
void history_valid(Ctx& c) {
    if (!c.hist_ok)
        FOPIS_CUDA(cudaMemcpyAsync(c.phi_prev2, c.phi_prev, sizeof(double) * c.N, cudaMemcpyDeviceToDevice, c.st));
    c.hist_ok = true;
}

int solve(Ctx& c, int kind) {
    const int mode = c.p.guess_mode;
    const bool hist = mode == FOPIS_GUESS_HISTORY || mode == FOPIS_GUESS_LEARNED;
    const bool track = hist || unet_training(c);
    const bool first = kind != SOLVE_SECOND;
    bool learned = false;
    if (first) {
        if (hist && c.hist_ok)
            FOPIS_CUDA(cudaMemcpyAsync(c.phi, c.phi_prev, sizeof(double) * c.N, cudaMemcpyDeviceToDevice, c.st));
        learned = unet_before_solve(c) != 0;
        c.learned_used = learned ? 1 : 0;
    } else if (hist && c.hist_ok) {
        conductor_start(c);
    }
    if (mode == FOPIS_GUESS_ZERO) FOPIS_CUDA(cudaMemsetAsync(c.phi, 0, sizeof(double) * c.N, c.st));
    int rc = mg_solve(c, solve_tol(c), solve_cap(c));
    int cycles = c.last_vcycles;
    if (rc == FOPIS_ERR_NOT_CONVERGED && learned) {
        FOPIS_CUDA(cudaMemcpyAsync(c.phi, c.phi_prev, sizeof(double) * c.N, cudaMemcpyDeviceToDevice, c.st));
        rc = mg_solve(c, solve_tol(c), solve_cap(c));
        cycles += c.last_vcycles;
        c.learned_used = 0;
    }
    if (rc == FOPIS_ERR_NOT_CONVERGED && mode != FOPIS_GUESS_ZERO) {
        FOPIS_CUDA(cudaMemsetAsync(c.phi, 0, sizeof(double) * c.N, c.st));
        rc = mg_solve(c, solve_tol(c), solve_cap(c));
        cycles += c.last_vcycles;
    }
    if (first) {
        unet_after_solve(c, learned, cycles, rc == FOPIS_OK);
        if (track) {
            std::swap(c.phi_prev, c.phi_prev2);
            FOPIS_CUDA(cudaMemcpyAsync(c.phi_prev, c.phi, sizeof(double) * c.N, cudaMemcpyDeviceToDevice, c.st));
            if (kind == SOLVE_ONLY) history_valid(c);
        }
    } else if (track) {
        conductor_record(c, c.phi_prev);
        history_valid(c);
    }
    if (!track) { c.hist_ok = false; c.obj_hist = 0; }
    return rc;
}

int solve_kind_after_rho(const Ctx& c) { return c.objs.empty() ? SOLVE_ONLY : SOLVE_SECOND; }

// RootGrid::updateRho after the per-particle pass: fold and convert, the
// object charge sums, and with objects the first solve plus the
// redistribution (RootGridField.cpp:1198-1243).
int rho_tail(Ctx& c, int* solve_rc) {
    launch_absorb(c);
    rho_finalize(c);
    int rc = FOPIS_OK;
    if (!c.objs.empty()) {
        objects_step_end(c);
        rc = solve(c, SOLVE_FIRST);
        redistribute(c);
    }
    *solve_rc = rc;
    return FOPIS_OK;
}

void record(Ctx& c, int k) {
    if (c.ev[k]) FOPIS_CUDA(cudaEventRecord(c.ev[k], c.st));
}

// The fused RootGrid::mainLoopES (RootGrid.cpp:82-143).
int one_step(Ctx& c) {
    step_begin(c);
    FOPIS_CUDA(cudaMemsetAsync(c.d_sc->pushed, 0, 3 * sizeof(c.d_sc->pushed), c.st));
    FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->absorbed_n, 0, sizeof(unsigned long long), c.st));
    rho_zero(c);
    record(c, 0);
    launch_push(c, true, true, true);
    record(c, 1);
    launch_emit(c, true);
    record(c, 2);
    launch_inject(c, true);
    record(c, 3);
    int rc1 = FOPIS_OK;
    rho_tail(c, &rc1);
    record(c, 5);
    int rc2 = solve(c, solve_kind_after_rho(c));
    record(c, 6);
    efield_update(c);
    record(c, 7);
    const int si = c.p.sort_interval > 0 ? c.p.sort_interval : 8;
    if (c.timestep % si == 0) particles_sort(c);
    record(c, 8);
    int rc = check_device(c);
    update_currents(c);
    for (int s = 0; s < c.nsp; ++s) {
        c.pushed_step[s] = (int64_t)c.h_sc->pushed[s];
        // after a sort step the sort's exact count stands; otherwise survivors plus new particles
        if (c.timestep % si != 0) c.valid[s] = (int64_t)(c.h_sc->survived[s] + c.h_sc->added[s]);
    }
    c.energy_valid = true;
    c.timestep += 1;
    if (c.ev[0]) {
        FOPIS_CUDA(cudaEventSynchronize(c.ev[8]));
        float ms = 0.f;
        const int map[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 5}, {3, 5}, {5, 6}, {6, 7}, {7, 8}};
        for (int q = 0; q < 8; ++q) {
            cudaEventElapsedTime(&ms, c.ev[map[q][0]], c.ev[map[q][1]]);
            c.ms_phase[q] = ms;
        }
        c.ms_phase[3] = 0.0;   // absorb runs inside the rho phase
    }
    if (rc != FOPIS_OK) return rc;
    if (rc1 != FOPIS_OK) return rc1;
    return rc2;
}

// RootGrid::mainLoopEM (RootGrid.cpp:145-191): velocity (E and B gather),
// emission, position with the edge currents, injection, rho (with the first
// solve and the redistribution when objects exist), then the FDTD E and B
// updates. ms_phase: velocity, emit, position + inject, -, rho, E, B, sort.
int em_step(Ctx& c) {
    step_begin(c);
    FOPIS_CUDA(cudaMemsetAsync(c.d_sc->pushed, 0, 3 * sizeof(c.d_sc->pushed), c.st));
    FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->absorbed_n, 0, sizeof(unsigned long long), c.st));
    // the mixed pass can give the velocity update itself when no body emits: then no
    // particle is created between the velocity and the position updates
    bool emits = false;
    for (const auto& o : c.objs) emits = emits || o.emit_species >= 0 || o.secondary_species >= 0;
    const bool kick_in_pass = !c.fp64 && !emits;
    record(c, 0);
    if (!kick_in_pass) launch_em_velocity(c);
    record(c, 1);
    launch_emit(c, false);
    record(c, 2);
    if (c.fp64) {
        // FP64: the current (FP64 atomics) and the move, the injection, then the rho pass
        launch_em_position(c);
        launch_inject(c, false);
        rho_zero(c);
        launch_deposit_all(c);
    } else {
        // mixed: one particle pass moves, adds the fixed-point current halves, tests the
        // bodies and deposits; injected particles deposit as they are created
        const size_t per = (size_t)(c.cx - 1) * c.cy * c.cz + (size_t)c.cx * (c.cy - 1) * c.cz +
                           (size_t)c.cx * c.cy * (c.cz - 1);
        FOPIS_CUDA(cudaMemsetAsync(c.em.jfix, 0, sizeof(unsigned long long) * per * c.nsp, c.st));
        rho_zero(c);
        launch_em_move(c, kick_in_pass);
        launch_inject(c, true);
    }
    record(c, 3);
    int rc1 = FOPIS_OK;
    rho_tail(c, &rc1);
    record(c, 5);
    em_update_efield(c);
    record(c, 6);
    em_update_bfield(c);
    record(c, 7);
    const int si = c.p.sort_interval > 0 ? c.p.sort_interval : 8;
    if (c.timestep % si == 0) particles_sort(c);
    record(c, 8);
    const int rc = check_device(c);
    update_currents(c);
    for (int s = 0; s < c.nsp; ++s) {
        // the mixed pass counts the particles it moved; the FP64 path's in-use slots stand in
        c.pushed_step[s] = c.fp64 ? (int64_t)c.h_sc->count[s] : (int64_t)c.h_sc->pushed[s];
        if (!c.fp64 && c.timestep % si != 0) c.valid[s] = (int64_t)(c.h_sc->survived[s] + c.h_sc->added[s]);
    }
    c.energy_valid = false;
    c.timestep += 1;
    if (c.ev[0]) {
        FOPIS_CUDA(cudaEventSynchronize(c.ev[8]));
        float ms = 0.f;
        const int map[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 3}, {3, 5}, {5, 6}, {6, 7}, {7, 8}};
        for (int q = 0; q < 8; ++q) {
            cudaEventElapsedTime(&ms, c.ev[map[q][0]], c.ev[map[q][1]]);
            c.ms_phase[q] = ms;
        }
    }
    return rc != FOPIS_OK ? rc : rc1;
}

}  // namespace

extern "C" {

const char* fopis_version(void) { return "fopis-b200 0.1 (sm_100a)"; }

const char* fopis_last_error(void* h) {
    if (!h) return g_create_error.c_str();
    return static_cast<Ctx*>(h)->err.c_str();
}

int fopis_create(const fopis_params* p, int device, void** out) {
    if (!p || !out) return FOPIS_ERR_ARG;
    *out = nullptr;
    Ctx* c = new (std::nothrow) Ctx();
    if (!c) return FOPIS_ERR_NOMEM;
    int rc = guarded(c, [&](Ctx& x) -> int {
        x.p = *p;
        if (p->nx < 3 || p->ny < 3 || p->nz < 3 || p->nx > 1020 || p->ny > 1020 || p->nz > 1020)
            throw ApiError{FOPIS_ERR_ARG, "nx, ny, nz must lie in [3, 1020]"};
        if (p->nspecies < 1 || p->nspecies > FOPIS_MAX_SPECIES) throw ApiError{FOPIS_ERR_ARG, "nspecies out of range"};
        if (!(p->eps0 > 0.0)) throw ApiError{FOPIS_ERR_ARG, "eps0 must be positive"};
        for (int t = 0; t < 6; ++t) {
            const char b = p->boundary[t];
            if (b != 'D' && b != 'N' && b != 'P')
                throw ApiError{FOPIS_ERR_ARG, "Unknown boundary condition type was used"};  // Field.cpp:25-28
        }
        if (p->precision != FOPIS_MIXED && p->precision != FOPIS_FP64)
            throw ApiError{FOPIS_ERR_ARG, "precision must be FOPIS_MIXED or FOPIS_FP64"};
        x.fp64 = p->precision == FOPIS_FP64;
        if (p->solver != FOPIS_SOLVER_ES && p->solver != FOPIS_SOLVER_EM)
            throw ApiError{FOPIS_ERR_ARG, "solver must be FOPIS_SOLVER_ES or FOPIS_SOLVER_EM"};
        if (p->solver == FOPIS_SOLVER_EM) {
            if (!(p->mu0 > 0.0)) throw ApiError{FOPIS_ERR_ARG, "the EM solver needs params.mu0"};
            // Environment::checkCFLCondition (Environment.cpp:193-203): Normalizer::c = 1/sqrt(eps0 mu0)
            if (1.0 / std::sqrt(p->eps0 * p->mu0) > 1.0 + 1e-9)
                throw ApiError{FOPIS_ERR_ARG, "Courant number exceeds 1.0"};
            for (int a = 0; a < 3; ++a)
                if ((p->boundary[2 * a] == 'P') != (p->boundary[2 * a + 1] == 'P'))
                    throw ApiError{FOPIS_ERR_ARG, "the EM solver needs each axis periodic on both sides or on neither"};
        }
        for (int s = 0; s < p->nspecies; ++s)
            if (!(p->species[s].mass > 0.0)) throw ApiError{FOPIS_ERR_ARG, "species mass must be positive"};
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw ApiError{FOPIS_ERR_NO_CUDA, "no CUDA device"};
        x.device = device >= 0 ? device : 0;
        if (device < 0) cudaGetDevice(&x.device);
        FOPIS_CUDA(cudaSetDevice(x.device));
        FOPIS_CUDA(cudaStreamCreateWithFlags(&x.st, cudaStreamNonBlocking));
        {   // the particle arrays grow through this process's default pool: keep freed blocks cached
            cudaMemPool_t pool;
            FOPIS_CUDA(cudaDeviceGetDefaultMemPool(&pool, x.device));
            uint64_t keep = UINT64_MAX;
            FOPIS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        }
        x.nx = p->nx; x.ny = p->ny; x.nz = p->nz;
        x.cx = x.nx + 2; x.cy = x.ny + 2; x.cz = x.nz + 2;
        x.N = (size_t)x.cx * x.cy * x.cz;
        for (int t = 0; t < 6; ++t) x.per[t] = p->boundary[t] == 'P';
        x.nsp = p->nspecies;
        FOPIS_CUDA(cudaMalloc(&x.rho_i64, sizeof(unsigned long long) * x.N * x.nsp));
        FOPIS_CUDA(cudaMalloc(&x.rho0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.phi, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.phi_prev, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.phi_prev2, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.phi_obj, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.phi_obj2, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.scratch64, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMalloc(&x.E, sizeof(float4) * x.N));
        if (x.fp64) {
            FOPIS_CUDA(cudaMalloc(&x.E64, sizeof(Vec4d) * x.N));
            FOPIS_CUDA(cudaMemset(x.E64, 0, sizeof(Vec4d) * x.N));
        }
        FOPIS_CUDA(cudaMalloc(&x.cellmap, x.N));
        FOPIS_CUDA(cudaMalloc(&x.node_cmat, sizeof(int32_t) * x.N));
        const size_t keys = std::max<size_t>(x.N, (size_t)brick_keys(x));
        FOPIS_CUDA(cudaMalloc(&x.sort_count, sizeof(int32_t) * (keys + 1)));
        FOPIS_CUDA(cudaMalloc(&x.sort_offset, sizeof(int32_t) * (keys + 1)));
        const size_t tiles = (keys + 1 + 8191) / 8192;
        FOPIS_CUDA(cudaMalloc(&x.scan_partials, sizeof(int32_t) * (tiles + 1)));
        FOPIS_CUDA(cudaMemset(x.rho_i64, 0, sizeof(unsigned long long) * x.N * x.nsp));
        FOPIS_CUDA(cudaMemset(x.rho0, 0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMemset(x.phi, 0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMemset(x.phi_prev, 0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMemset(x.phi_prev2, 0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMemset(x.phi_obj, 0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMemset(x.phi_obj2, 0, sizeof(double) * x.N));
        FOPIS_CUDA(cudaMemset(x.E, 0, sizeof(float4) * x.N));
        FOPIS_CUDA(cudaMemset(x.cellmap, 0, x.N));
        FOPIS_CUDA(cudaMemset(x.node_cmat, 0xff, sizeof(int32_t) * x.N));
        // absorbed list: generous for conductor-heavy steps
        x.ab.cap = std::max<int64_t>(1 << 20, (int64_t)x.N / 2);
        FOPIS_CUDA(cudaMalloc(&x.ab.cell, sizeof(int32_t) * x.ab.cap));
        double** fl[6] = {&x.ab.ox, &x.ab.oy, &x.ab.oz, &x.ab.vx, &x.ab.vy, &x.ab.vz};
        for (auto* q : fl) FOPIS_CUDA(cudaMalloc(q, sizeof(double) * x.ab.cap));
        FOPIS_CUDA(cudaMalloc(&x.ab.species, x.ab.cap));
        FOPIS_CUDA(cudaMalloc(&x.ab.object, x.ab.cap));
        FOPIS_CUDA(cudaMalloc(&x.d_sc, sizeof(DevScalars)));
        FOPIS_CUDA(cudaMemset(x.d_sc, 0, sizeof(DevScalars)));
        FOPIS_CUDA(cudaMallocHost(&x.h_sc, sizeof(DevScalars)));
        std::memset(x.h_sc, 0, sizeof(DevScalars));
        for (auto& e : x.ev) FOPIS_CUDA(cudaEventCreate(&e));
        if (p->solver == FOPIS_SOLVER_EM) em_alloc(x);
        mg_setup(x);
        mg_prepare(x);
        FOPIS_CUDA(cudaDeviceSynchronize());
        return FOPIS_OK;
    });
    if (rc != FOPIS_OK) {
        g_create_error = c->err;
        fopis_destroy(c);
        return rc;
    }
    *out = c;
    return FOPIS_OK;
}

void fopis_destroy(void* h) {
    Ctx* c = static_cast<Ctx*>(h);
    if (!c) return;
    if (c->st) cudaStreamSynchronize(c->st);
    unet_free(*c);
    em_free(*c);
    for (int s = 0; s < FOPIS_MAX_SPECIES; ++s) {
        Soa* v[2] = {&c->sp[s], &c->sp2[s]};
        for (Soa* q : v) {
            void* arr[7] = {q->cell, q->ox, q->oy, q->oz, q->vx, q->vy, q->vz};
            for (void* a : arr) if (a) cudaFreeAsync(a, c->st);
        }
        Soa64* w[2] = {&c->dp[s], &c->dp2[s]};
        for (Soa64* q : w) {
            void* arr[7] = {q->cell, q->ox, q->oy, q->oz, q->vx, q->vy, q->vz};
            for (void* a : arr) if (a) cudaFreeAsync(a, c->st);
        }
    }
    if (c->st) cudaStreamSynchronize(c->st);
    for (int s = 0; s < FOPIS_MAX_SPECIES; ++s) if (c->brick_start[s]) cudaFree(c->brick_start[s]);
    for (auto& o : c->objs) {
        cudaFree(o.nodes); cudaFree(o.C); cudaFree(o.colsum); cudaFree(o.charge_tmp);
        cudaFree(o.charge_map); cudaFree(o.phis); cudaFree(o.scal); cudaFree(o.lit); cudaFree(o.drho_buf);
        if (o.capacitance) cudaFree(o.capacitance);
    }
    {
        void* inc[] = {c->inc.x, c->inc.y, c->inc.z, c->inc.vx, c->inc.vy, c->inc.vz, c->inc.trem, c->inc.species,
                       c->inc.object, c->inc.axis, c->inc.count};
        for (void* q : inc) if (q) cudaFree(q);
    }
    mg_free(*c);
    void* ptrs[] = {c->rho_i64, c->rho0, c->phi, c->phi_prev, c->phi_prev2, c->phi_obj, c->phi_obj2, c->scratch64, c->E, c->E64, c->cellmap,
                    c->node_cmat, c->sort_count, c->sort_offset, c->scan_partials, c->ab.cell, c->ab.ox,
                    c->ab.oy, c->ab.oz, c->ab.vx, c->ab.vy, c->ab.vz, c->ab.species, c->ab.object, c->d_sc};
    for (void* q : ptrs) if (q) cudaFree(q);
    if (c->h_sc) cudaFreeHost(c->h_sc);
    for (auto& e : c->ev) if (e) cudaEventDestroy(e);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

int fopis_add_object(void* h, const fopis_object_desc* d, int* object_id) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!d || !d->cmat_nodes || (d->n_cells > 0 && !d->cells)) throw ApiError{FOPIS_ERR_ARG, "null object description"};
        if ((int)c.objs.size() >= FOPIS_MAX_OBJECTS) throw ApiError{FOPIS_ERR_ARG, "too many objects"};
        if (d->emit_species >= c.nsp) throw ApiError{FOPIS_ERR_ARG, "emit_species out of range"};
        const int id = (int)c.objs.size();
        c.objs.emplace_back();
        try {
            object_upload(c, c.objs.back(), d, id);
        } catch (...) {
            c.objs.pop_back();
            throw;
        }
        if (object_id) *object_id = id;
        return FOPIS_OK;
    });
}

int fopis_build_capacity_matrix(void* h, int id) {
    return guarded(h, [&](Ctx& c) -> int {
        if (id < 0 || id >= (int)c.objs.size()) throw ApiError{FOPIS_ERR_ARG, "object id"};
        cmatrix_build(c, id);
        return FOPIS_OK;
    });
}

int fopis_set_capacity_matrix(void* h, int id, const double* C, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (id < 0 || id >= (int)c.objs.size() || !C || n != c.objs[id].n) throw ApiError{FOPIS_ERR_ARG, "object id or size"};
        cmatrix_set(c, id, C);
        return FOPIS_OK;
    });
}

int fopis_get_capacity_matrix(void* h, int id, double* C, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (id < 0 || id >= (int)c.objs.size() || !C || n != c.objs[id].n) throw ApiError{FOPIS_ERR_ARG, "object id or size"};
        if (!c.objs[id].has_C) throw ApiError{FOPIS_ERR_STATE, "capacity matrix not built"};
        FOPIS_CUDA(cudaMemcpy(C, c.objs[id].C, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost));
        return FOPIS_OK;
    });
}

int fopis_get_object(void* h, int id, double* V, double* Q, double* I) {
    return guarded(h, [&](Ctx& c) -> int {
        if (id < 0 || id >= (int)c.objs.size()) throw ApiError{FOPIS_ERR_ARG, "object id"};
        const ObjectDev& o = c.objs[id];
        if (V) *V = o.potential;
        if (Q) *Q = o.total_charge;
        if (I) for (int s = 0; s < c.nsp; ++s) I[s] = o.current[s];
        return FOPIS_OK;
    });
}

int fopis_get_charge_map(void* h, int id, double* out, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (id < 0 || id >= (int)c.objs.size() || !out || n != c.nsp * c.objs[id].n) throw ApiError{FOPIS_ERR_ARG, "object id or size"};
        FOPIS_CUDA(cudaMemcpy(out, c.objs[id].charge_map, sizeof(double) * n, cudaMemcpyDeviceToHost));
        return FOPIS_OK;
    });
}

int fopis_set_charge_map(void* h, int id, const double* in, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (id < 0 || id >= (int)c.objs.size() || !in || n != c.nsp * c.objs[id].n) throw ApiError{FOPIS_ERR_ARG, "object id or size"};
        FOPIS_CUDA(cudaMemcpy(c.objs[id].charge_map, in, sizeof(double) * n, cudaMemcpyHostToDevice));
        return FOPIS_OK;
    });
}

// Incident records: object, species, axis, remaining time, x, y, z, vx, vy, vz.
int fopis_get_incidents(void* h, double* out, int64_t cap, int64_t* n_out) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!n_out || cap < 0 || (cap > 0 && !out)) throw ApiError{FOPIS_ERR_ARG, "null output"};
        sync_scalars(c);
        const int64_t n = c.inc.cap ? (int64_t)std::min<unsigned long long>(c.h_sc->incident_n, (unsigned long long)c.inc.cap) : 0;
        *n_out = n;
        const int64_t m = std::min(n, cap);
        if (m == 0) return FOPIS_OK;
        std::vector<double> col[7];
        const double* src[7] = {c.inc.trem, c.inc.x, c.inc.y, c.inc.z, c.inc.vx, c.inc.vy, c.inc.vz};
        for (int q = 0; q < 7; ++q) {
            col[q].resize(m);
            FOPIS_CUDA(cudaMemcpy(col[q].data(), src[q], sizeof(double) * m, cudaMemcpyDeviceToHost));
        }
        std::vector<uint8_t> ob(m), sp(m), ax(m);
        FOPIS_CUDA(cudaMemcpy(ob.data(), c.inc.object, m, cudaMemcpyDeviceToHost));
        FOPIS_CUDA(cudaMemcpy(sp.data(), c.inc.species, m, cudaMemcpyDeviceToHost));
        FOPIS_CUDA(cudaMemcpy(ax.data(), c.inc.axis, m, cudaMemcpyDeviceToHost));
        for (int64_t t = 0; t < m; ++t) {
            double* r = out + FOPIS_INCIDENT_DOUBLES * t;
            r[0] = ob[t]; r[1] = sp[t]; r[2] = ax[t];
            for (int q = 0; q < 7; ++q) r[3 + q] = col[q][t];
        }
        return FOPIS_OK;
    });
}

int fopis_set_incidents(void* h, const double* in, int64_t n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (n < 0 || (n > 0 && !in)) throw ApiError{FOPIS_ERR_ARG, "null input"};
        if (c.inc.cap == 0) throw ApiError{FOPIS_ERR_STATE, "no object emits secondaries"};
        if (n > c.inc.cap) throw ApiError{FOPIS_ERR_CAPACITY, "more incidents than the absorbed-list capacity"};
        std::vector<double> col[7];
        std::vector<uint8_t> ob(n), sp(n), ax(n);
        for (int q = 0; q < 7; ++q) col[q].resize(n);
        for (int64_t t = 0; t < n; ++t) {
            const double* r = in + FOPIS_INCIDENT_DOUBLES * t;
            const int o = (int)r[0], s = (int)r[1], a = (int)r[2];
            if (o < 0 || o >= (int)c.objs.size() || s < 0 || s >= c.nsp || a < 0 || a > 2)
                throw ApiError{FOPIS_ERR_ARG, "incident object, species or axis out of range"};
            ob[t] = (uint8_t)o; sp[t] = (uint8_t)s; ax[t] = (uint8_t)a;
            for (int q = 0; q < 7; ++q) col[q][t] = r[3 + q];
        }
        double* dst[7] = {c.inc.trem, c.inc.x, c.inc.y, c.inc.z, c.inc.vx, c.inc.vy, c.inc.vz};
        if (n > 0) {
            for (int q = 0; q < 7; ++q)
                FOPIS_CUDA(cudaMemcpy(dst[q], col[q].data(), sizeof(double) * n, cudaMemcpyHostToDevice));
            FOPIS_CUDA(cudaMemcpy(c.inc.object, ob.data(), n, cudaMemcpyHostToDevice));
            FOPIS_CUDA(cudaMemcpy(c.inc.species, sp.data(), n, cudaMemcpyHostToDevice));
            FOPIS_CUDA(cudaMemcpy(c.inc.axis, ax.data(), n, cudaMemcpyHostToDevice));
        }
        const unsigned long long nn = (unsigned long long)n;
        FOPIS_CUDA(cudaMemcpy(&c.d_sc->incident_n, &nn, sizeof(nn), cudaMemcpyHostToDevice));
        return FOPIS_OK;
    });
}

int fopis_set_timestep(void* h, int64_t t) {
    return guarded(h, [&](Ctx& c) -> int {
        if (t < 1) throw ApiError{FOPIS_ERR_ARG, "timestep must be >= 1"};
        c.timestep = t;
        return FOPIS_OK;
    });
}

int fopis_get_injection_carry(void* h, double* out, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!out || n != 6 * c.nsp) throw ApiError{FOPIS_ERR_ARG, "carry size must be 6 * nspecies"};
        for (int s = 0; s < c.nsp; ++s) for (int f = 0; f < 6; ++f) out[6 * s + f] = c.inject_residual[s][f];
        return FOPIS_OK;
    });
}

int fopis_set_injection_carry(void* h, const double* in, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!in || n != 6 * c.nsp) throw ApiError{FOPIS_ERR_ARG, "carry size must be 6 * nspecies"};
        for (int s = 0; s < c.nsp; ++s) for (int f = 0; f < 6; ++f) c.inject_residual[s][f] = in[6 * s + f];
        return FOPIS_OK;
    });
}

int fopis_load_particles(void* h, int s, const void* p56, int64_t n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (s < 0 || s >= c.nsp || (n > 0 && !p56) || n < 0) throw ApiError{FOPIS_ERR_ARG, "species or buffer"};
        if (n) particles_append_aos(c, s, p56, n);
        c.energy_valid = false;
        return check_device(c);
    });
}

int fopis_get_particles(void* h, int s, void* p56, int64_t cap, int64_t* n_out) {
    return guarded(h, [&](Ctx& c) -> int {
        if (s < 0 || s >= c.nsp || (cap > 0 && !p56)) throw ApiError{FOPIS_ERR_ARG, "species or buffer"};
        const int64_t n = c.cap[s] ? particles_export_aos(c, s, p56, cap) : 0;
        if (n_out) *n_out = n;
        return FOPIS_OK;
    });
}

int fopis_get_particles_raw(void* h, int s, int32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                            float* vz, int64_t cap, int64_t* n_out) {
    return guarded(h, [&](Ctx& c) -> int {
        if (s < 0 || s >= c.nsp) throw ApiError{FOPIS_ERR_ARG, "species"};
        if (cap > 0 && !(cell && ox && oy && oz && vx && vy && vz)) throw ApiError{FOPIS_ERR_ARG, "buffers"};
        if (c.fp64) throw ApiError{FOPIS_ERR_ARG, "raw split-precision state exists only in the mixed mode"};
        const int64_t n = c.cap[s] ? particles_export_raw(c, s, cell, ox, oy, oz, vx, vy, vz, cap) : 0;
        if (n_out) *n_out = n;
        return FOPIS_OK;
    });
}

int fopis_generate_ambient(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        particles_generate_ambient(c);
        c.energy_valid = false;
        return check_device(c);
    });
}

int fopis_sort_particles(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        particles_sort(c);
        return check_device(c);
    });
}

int fopis_remove_invalid_particles(void* h) { return fopis_sort_particles(h); }

int fopis_initialize(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        particles_sort(c);
        step_begin(c);
        FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->absorbed_n, 0, sizeof(unsigned long long), c.st));
        rho_zero(c);
        launch_deposit_all(c);
        c.hist_ok = false;
        c.obj_hist = 0;
        int rc1 = FOPIS_OK;
        rho_tail(c, &rc1);
        const int rc2 = solve(c, solve_kind_after_rho(c));
        if (c.em.on) {
            em_efield_from_phi(c);
            em_update_bfield(c);
        } else {
            efield_update(c);
        }
        const int rc = check_device(c);
        update_currents(c);
        c.energy_valid = false;
        if (rc != FOPIS_OK) return rc;
        return rc1 != FOPIS_OK ? rc1 : rc2;
    });
}

int fopis_step(void* h, int n) {
    return guarded(h, [&](Ctx& c) -> int {
        int rc = FOPIS_OK;
        for (int t = 0; t < n; ++t) {
            rc = c.em.on ? em_step(c) : one_step(c);
            if (rc != FOPIS_OK && rc != FOPIS_ERR_NOT_CONVERGED) return rc;
        }
        return rc;
    });
}

int fopis_update_velocity(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        step_begin(c);   // RootGrid::resetObjects precedes it in mainLoopES
        if (c.em.on) launch_em_velocity(c);
        else launch_push(c, true, false, false);
        c.energy_valid = false;
        return check_device(c);
    });
}

int fopis_emit_particles(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        launch_emit(c, false);
        c.energy_valid = false;
        return check_device(c);
    });
}

int fopis_update_position(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        if (c.em.on) launch_em_position(c);
        else launch_push(c, false, true, false);
        c.energy_valid = false;
        return check_device(c);
    });
}

int fopis_inject_particles(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        launch_inject(c, false);
        c.energy_valid = false;
        return check_device(c);
    });
}

int fopis_update_rho(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->absorbed_n, 0, sizeof(unsigned long long), c.st));
        rho_zero(c);
        launch_deposit_all(c);
        int rc1 = FOPIS_OK;
        rho_tail(c, &rc1);
        const int rc = check_device(c);
        update_currents(c);
        c.energy_valid = false;
        return rc != FOPIS_OK ? rc : rc1;
    });
}

int fopis_solve_poisson(void* h) {
    return guarded(h, [&](Ctx& c) -> int { return solve(c, solve_kind_after_rho(c)); });
}

int fopis_update_efield(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        if (c.em.on) em_update_efield(c);
        else efield_update(c);
        FOPIS_CUDA(cudaStreamSynchronize(c.st));
        return FOPIS_OK;
    });
}

int fopis_update_reference_fields(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        if (c.em.on) em_reference_fields(c);
        else efield_update(c);
        FOPIS_CUDA(cudaStreamSynchronize(c.st));
        return FOPIS_OK;
    });
}

int fopis_update_bfield(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!c.em.on) throw ApiError{FOPIS_ERR_STATE, "updateBfield belongs to the EM solver"};
        em_update_bfield(c);
        FOPIS_CUDA(cudaStreamSynchronize(c.st));
        return FOPIS_OK;
    });
}

int fopis_field_shape(void* h, int which, int lo[3], int n[3]) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!lo || !n) throw ApiError{FOPIS_ERR_ARG, "null shape output"};
        const int cc[3] = {c.cx, c.cy, c.cz};
        for (int a = 0; a < 3; ++a) { lo[a] = 0; n[a] = cc[a]; }
        if (const YeeArr* y = em_array(c, which)) {
            for (int a = 0; a < 3; ++a) { lo[a] = y->lo[a]; n[a] = y->n[a]; }
        } else if (which >= FOPIS_FIELD_JX && which <= FOPIS_FIELD_JZ) {
            if (!c.em.on) throw ApiError{FOPIS_ERR_ARG, "edge currents exist in the EM mode only"};
            n[which - FOPIS_FIELD_JX] -= 1;
        } else if (which >= FOPIS_FIELD_EX && which <= FOPIS_FIELD_BZ) {
            throw ApiError{FOPIS_ERR_ARG, "Yee arrays exist in the EM mode only"};
        }
        return FOPIS_OK;
    });
}

int fopis_get_bfield_energy(void* h, double* energy) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!energy) throw ApiError{FOPIS_ERR_ARG, "null output"};
        *energy = c.em.on ? em_bfield_energy(c) : 0.0;
        return FOPIS_OK;
    });
}

int fopis_advance_timestep(void* h) {
    return guarded(h, [&](Ctx& c) -> int {
        const int si = c.p.sort_interval > 0 ? c.p.sort_interval : 8;
        if (c.timestep % si == 0) particles_sort(c);
        c.timestep += 1;
        return FOPIS_OK;
    });
}

// Elements of a field selector's array: the Yee arrays and edge currents of the
// EM mode have their own extents, every other field the node grid's.
static size_t field_elements(Ctx& c, int which) {
    if (const YeeArr* y = em_array(c, which)) return y->size();
    if (c.em.on && which >= FOPIS_FIELD_JX && which <= FOPIS_FIELD_JZ) {
        const int d = which - FOPIS_FIELD_JX;
        return (size_t)(c.cx - (d == 0)) * (c.cy - (d == 1)) * (c.cz - (d == 2));
    }
    return c.N;
}

int fopis_get_field(void* h, int which, double* out, size_t n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!out || n != field_elements(c, which))
            throw ApiError{FOPIS_ERR_ARG, "output size must be the field's element count (fopis_field_shape)"};
        const bool em_field = c.em.on && ((which >= FOPIS_FIELD_EXREF && which <= FOPIS_FIELD_JZREF) ||
                                          (which >= FOPIS_FIELD_EX && which <= FOPIS_FIELD_JZ));
        if (em_field) em_field_export(c, which, out);
        else if (which >= FOPIS_FIELD_BXREF && which <= FOPIS_FIELD_JZREF)
            throw ApiError{FOPIS_ERR_ARG, "magnetic field and current exist in the EM mode only"};
        else field_export(c, which, out);
        return FOPIS_OK;
    });
}

int fopis_set_field(void* h, int which, const double* in, size_t n) {
    return guarded(h, [&](Ctx& c) -> int {
        if (const YeeArr* y = em_array(c, which)) {
            if (!in || n != y->size()) throw ApiError{FOPIS_ERR_ARG, "input size must be the Yee array's element count"};
            FOPIS_CUDA(cudaMemcpy(y->v, in, sizeof(double) * n, cudaMemcpyHostToDevice));
            return FOPIS_OK;
        }
        if (c.em.on && which >= FOPIS_FIELD_JX && which <= FOPIS_FIELD_JZ) {
            if (!in || n != field_elements(c, which)) throw ApiError{FOPIS_ERR_ARG, "input size must be the current's element count"};
            FOPIS_CUDA(cudaMemcpy(c.em.j[which - FOPIS_FIELD_JX], in, sizeof(double) * n, cudaMemcpyHostToDevice));
            return FOPIS_OK;
        }
        if (!in || n != c.N) throw ApiError{FOPIS_ERR_ARG, "input size must be (nx+2)(ny+2)(nz+2)"};
        double* dst = which == FOPIS_FIELD_PHI ? c.phi : (which == FOPIS_FIELD_RHO0 ? c.rho0 : nullptr);
        if (!dst) throw ApiError{FOPIS_ERR_ARG, "only PHI and RHO0 can be set"};
        FOPIS_CUDA(cudaMemcpy(dst, in, sizeof(double) * c.N, cudaMemcpyHostToDevice));
        return FOPIS_OK;
    });
}

int fopis_get_energy(void* h, double* pe, double* fe) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!c.energy_valid) { launch_energy(c); sync_scalars(c); c.energy_valid = true; }
        double e = 0.0;
        for (int s = 0; s < c.nsp; ++s) e += 0.5 * c.p.species[s].mass * c.h_sc->energy[s] * c.p.species[s].size;
        if (pe) *pe = e;
        if (fe) *fe = c.em.on ? em_efield_energy(c) : efield_energy(c);
        return FOPIS_OK;
    });
}

int fopis_get_stats(void* h, fopis_stats* st) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!st) throw ApiError{FOPIS_ERR_ARG, "null stats"};
        sync_scalars(c);
        std::memset(st, 0, sizeof(*st));
        st->timestep = c.timestep;
        st->vcycles_last = c.last_vcycles;
        st->vcycles_step = c.step_vcycles;
        st->solves_step = c.step_solves;
        st->converged = c.last_converged;
        st->residual_last = c.last_res;
        st->residual_initial = c.first_res;
        for (int s = 0; s < c.nsp; ++s) {
            st->num_particles[s] = c.nslots[s];
            st->capacity[s] = c.cap[s];
            st->valid_particles[s] = c.valid[s];
            st->pushed_step[s] = c.pushed_step[s];
        }
        st->absorbed_step = c.absorbed_step;
        st->injected_step = c.injected_step;
        st->emitted_step = c.emitted_step;
        st->device_status = c.h_sc->status;
        st->learned_used = c.learned_used;
        for (int q = 0; q < 8; ++q) st->ms_phase[q] = c.ms_phase[q];
        st->kernel_launches = c.launches;
        st->solve_mode = c.solve_state == 1 ? (c.pdl ? 2 : 1) : 0;
        {
            const unsigned long long bits = c.h_sc->pointwise_bits;
            double v;
            std::memcpy(&v, &bits, sizeof(v));
            st->residual_pointwise = v;
        }
        return FOPIS_OK;
    });
}

int fopis_get_stream(void* h, void** stream) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!stream) throw ApiError{FOPIS_ERR_ARG, "null stream pointer"};
        *stream = (void*)c.st;
        return FOPIS_OK;
    });
}

int fopis_set_guess_mode(void* h, int mode) {
    return guarded(h, [&](Ctx& c) -> int {
        if (mode < FOPIS_GUESS_ZERO || mode > FOPIS_GUESS_HISTORY) throw ApiError{FOPIS_ERR_ARG, "guess mode"};
        c.p.guess_mode = mode;
        return FOPIS_OK;
    });
}

int fopis_unet_set_training(void* h, int enable, double lr) {
    return guarded(h, [&](Ctx& c) -> int { return unet_set_training(c, enable, lr); });
}

int fopis_unet_get_state(void* h, double* loss, int64_t* steps) {
    return guarded(h, [&](Ctx& c) -> int { return unet_get_state(c, loss, steps); });
}

int fopis_unet_get_policy(void* h, double* plain_vcycles, double* learned_vcycles, int* learned_enabled) {
    return guarded(h, [&](Ctx& c) -> int { return unet_get_policy(c, plain_vcycles, learned_vcycles, learned_enabled); });
}

int fopis_unet_get_last(void* h, double* warm_residual, double* guess_residual, double* ms_forward,
                        double* ms_train) {
    return guarded(h, [&](Ctx& c) -> int { return unet_get_last(c, warm_residual, guess_residual, ms_forward, ms_train); });
}

int fopis_unet_eval(void* h, const double* rho0, const double* phi1, const double* phi2, const double* phi_target,
                    double* pred, float* grads, double* loss) {
    return guarded(h, [&](Ctx& c) -> int {
        if (!rho0 || !phi1 || !phi2) throw ApiError{FOPIS_ERR_ARG, "null field"};
        return unet_eval(c, rho0, phi1, phi2, phi_target, pred, grads, loss);
    });
}

int fopis_unet_params(void* h, float* get, const float* set, int64_t* count) {
    return guarded(h, [&](Ctx& c) -> int { return unet_params(c, get, set, count); });
}

int fopis_unet_tensor(void* h, int which, float* host, int64_t cap, int64_t* count) {
    return guarded(h, [&](Ctx& c) -> int { return unet_tensor(c, which, host, cap, count); });
}

void fopis_free(void* p) { std::free(p); }

}  // extern "C"
