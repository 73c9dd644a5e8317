// cmatrix.cu — conductors: surface-node maps, the capacity matrix and the
// per-step equipotential correction.
//
// Capacity matrix (RootGrid::initializeObjectsCmatrix, RootGridObject.cpp:77-148):
// column c of B holds phi at every surface node for rho = 1 at surface node c
// (one multigrid solve per column); C = B^-1 by in-place Gauss-Jordan
// elimination in FP64 on the device (B is symmetric positive definite, so no
// pivoting). Per step (Spacecraft::redistributeChargeForPerfectConductor,
// Spacecraft.cpp:708-758): V = (sum_ij C_ij phi_j + Q) / sum_ij C_ij, or the
// fixed potential, then rho0[node_i] += sum_j C_ij (V - phi_j).
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace fopis {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ double wsum(double v) {
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ double bsum(double v) {
    __shared__ double red[32];
    v = wsum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    v = 0.0;
    if (w == 0) {
        v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
        v = wsum(v);
    }
    return v;
}

__global__ void gather_kernel(const double* phi, const int32_t* nodes, int n, double* out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) out[t] = phi[nodes[t]];
}

__global__ void set_node_kernel(double* a, long long idx, double v) { a[idx] = v; }

// Gauss-Jordan step k: copy row k and column k aside.
__global__ void gj_copy_kernel(const double* A, int n, int k, double* rowk, double* colk) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        rowk[t] = A[(long long)k * n + t];
        colk[t] = A[(long long)t * n + k];
    }
}
// In-place Gauss-Jordan inversion step k (no pivoting).
__global__ void gj_update_kernel(double* A, int n, int k, const double* rowk, const double* colk, unsigned* bad) {
    const double akk = colk[k];
    if (blockIdx.x == 0 && threadIdx.x == 0 && !(akk > 0.0)) atomicOr(bad, 1u);
    const double p = 1.0 / akk;
    const long long total = (long long)n * n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / n), j = (int)(t % n);
        double v;
        if (i == k && j == k) v = p;
        else if (i == k) v = rowk[j] * p;
        else if (j == k) v = -colk[i] * p;
        else v = A[t] - colk[i] * rowk[j] * p;
        A[t] = v;
    }
}

// colsum_j = sum_i C_ij; scal[3] = sum_ij C_ij (Cmatrix::total, Cmatrix.hpp:36-44).
__global__ void colsum_kernel(const double* C, int n, double* colsum) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += C[(long long)i * n + j];
        colsum[j] = s;
    }
}
__global__ void total_kernel(const double* colsum, int n, double* out) {
    double s = 0.0;
    for (int t = threadIdx.x; t < n; t += blockDim.x) s += colsum[t];
    s = bsum(s);
    if (threadIdx.x == 0) *out = s;
}

// Spacecraft::initializeChargeMapOffset (Spacecraft.cpp:160-183):
// charge_map[0][i] += sum_j C_ij * offset.
__global__ void offset_kernel(const double* C, int n, double offset, double* charge_map) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nw) {
        double s = 0.0;
        for (int j = lane; j < n; j += 32) s += C[(long long)i * n + j] * offset;
        s = wsum(s);
        if (lane == 0) charge_map[i] += s;
    }
}

// Spacecraft::sumWholeCharge (Spacecraft.cpp:615-626) for the fixed-point
// temporary map, then the total charge (getTotalCharge, :248-259) into scal[1].
__global__ void sum_charge_kernel(long long* tmp, double* map, int nsp, int n, const double* scale, double* scal) {
    double q = 0.0;
    for (int t = threadIdx.x; t < nsp * n; t += blockDim.x) {
        const int s = t / n;
        const long long v = tmp[t];
        if (v) { map[t] += scale[s] * (double)v; tmp[t] = 0; }
        q += map[t];
    }
    q = bsum(q);
    if (threadIdx.x == 0) scal[1] = q;
}

// V of the perfect conductor into scal[0]; scal[2] = sum_j colsum_j phi_j.
// On a dielectric surface (Spacecraft::redistributeChargeForDielectric,
// Spacecraft.cpp:641-706) every node with a capacitance sees phi_j - Q_j / c_j,
// Q_j its accumulated charge over the species: the same formulas then give V
// and delta rho, so phis holds that effective potential.
__global__ void potential_kernel(const double* phi, const int32_t* nodes, const double* colsum, int n, double total,
                                 int fixed, double fixedV, double* phis, double* scal, const double* cap,
                                 const double* charge_map, int nsp) {
    double s = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double p = phi[nodes[j]];
        if (cap && cap[j] > 0.0) {
            double q = 0.0;
            for (int sp = 0; sp < nsp; ++sp) q += charge_map[(long long)sp * n + j];
            p -= q / cap[j];
        }
        phis[j] = p;
        s += colsum[j] * p;
    }
    s = bsum(s);
    if (threadIdx.x == 0) {
        scal[2] = s;
        scal[0] = fixed ? fixedV : (s + scal[1]) / total;
    }
}

// delta rho_i = sum_j C_ij (V - phi_j), added to rho0 at surface node i and
// kept in drho_out for the start of the second solve.
__global__ void drho_kernel(const double* C, int n, const double* phis, const double* scal, const int32_t* nodes,
                            double* rho0, double* drho_out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const double V = scal[0];
    for (int i = warp; i < n; i += nw) {
        double s = 0.0;
        const double* row = C + (long long)i * n;
        for (int j = lane; j < n; j += 32) s += row[j] * (V - phis[j]);
        s = wsum(s);
        if (lane == 0) { rho0[nodes[i]] += s; drho_out[i] = s; }
    }
}

// Start of the second solve: this step's redistributed charge d0 fitted in
// least squares by the two previous steps' (d1, d2) over the surface nodes of
// every object; the coefficients scale the conductor responses those charges
// produced. One term while only one response is recorded, and alpha = 1 (the
// previous response as it is) when the fit is degenerate.
struct ConductorFit {
    int nobj;
    int terms;
    const double* d0[FOPIS_MAX_OBJECTS];
    const double* d1[FOPIS_MAX_OBJECTS];
    const double* d2[FOPIS_MAX_OBJECTS];
    int n[FOPIS_MAX_OBJECTS];
};

__global__ void conductor_fit_kernel(ConductorFit f, double* alpha) {
    double s11 = 0.0, s12 = 0.0, s22 = 0.0, b1 = 0.0, b2 = 0.0;
    for (int o = 0; o < f.nobj; ++o)
        for (int i = threadIdx.x; i < f.n[o]; i += blockDim.x) {
            const double x0 = f.d0[o][i], x1 = f.d1[o][i], x2 = f.terms > 1 ? f.d2[o][i] : 0.0;
            s11 += x1 * x1; s12 += x1 * x2; s22 += x2 * x2; b1 += x0 * x1; b2 += x0 * x2;
        }
    s11 = bsum(s11); s12 = bsum(s12); s22 = bsum(s22); b1 = bsum(b1); b2 = bsum(b2);
    if (threadIdx.x == 0) {
        double a1 = 1.0, a2 = 0.0;
        const double det = s11 * s22 - s12 * s12;
        if (f.terms > 1 && det > 1e-10 * s11 * s22) {
            a1 = (b1 * s22 - b2 * s12) / det;
            a2 = (b2 * s11 - b1 * s12) / det;
        } else if (s11 > 0.0) {
            a1 = b1 / s11;
        }
        alpha[0] = a1;
        alpha[1] = a2;
    }
}

__global__ void conductor_start_kernel(double* phi, const double* r1, const double* r2, const double* alpha,
                                       long long N) {
    const double a1 = alpha[0], a2 = alpha[1];
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x)
        phi[t] += a1 * r1[t] + (a2 != 0.0 ? a2 * r2[t] : 0.0);
}

// Spacecraft::is{X,Y,Z}surfacePoint at an integer node (dx1 = 0), host side.
struct HostObj {
    const Ctx* c;
    std::vector<uint8_t> cells;   // [nx+1][ny+1][nz+1]
    std::vector<int32_t> node_cmat;
    bool valid_cell(int i, int j, int k) const {
        return i >= 0 && i < c->nx + 1 && j >= 0 && j < c->ny + 1 && k >= 0 && k < c->nz + 1;
    }
    bool in(int i, int j, int k) const {
        if (!valid_cell(i, j, k)) return false;
        return cells[((size_t)i * (c->ny + 1) + j) * (c->nz + 1) + k] != 0;
    }
    bool is_cmat(int i, int j, int k) const {
        if (i < 0 || j < 0 || k < 0 || i >= c->cx || j >= c->cy || k >= c->cz) return false;
        return node_cmat[((size_t)i * c->cy + j) * c->cz + k] >= 0;
    }
    bool surface_point(int ax, int i, int j, int k, int sign) const {
        const int di = ax == 0, dj = ax == 1, dk = ax == 2;
        if (valid_cell(i, j, k) && valid_cell(i - di, j - dj, k - dk)) {
            const bool here = in(i, j, k), below = in(i - di, j - dj, k - dk);
            return sign > 0 ? (here && !below) : (!here && below);
        }
        if (ax == 0) return is_cmat(i, j, k) && is_cmat(i, j + 1, k) && is_cmat(i, j, k + 1) && is_cmat(i, j + 1, k + 1);
        if (ax == 1) return is_cmat(i, j, k) && is_cmat(i + 1, j, k) && is_cmat(i, j, k + 1) && is_cmat(i + 1, j, k + 1);
        return is_cmat(i, j, k) && is_cmat(i + 1, j, k) && is_cmat(i, j + 1, k) && is_cmat(i + 1, j + 1, k);
    }
};

int grid1(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + kT - 1) / kT, 148LL * 16)); }

}  // namespace

void object_upload(Ctx& c, ObjectDev& o, const fopis_object_desc* d, int id) {
    if (d->n_cmat <= 0 || d->n_cmat >= (1 << 24)) throw ApiError{FOPIS_ERR_ARG, "n_cmat out of range"};
    o.n = d->n_cmat;
    o.nodes_ijk.assign(d->cmat_nodes, d->cmat_nodes + 3 * (size_t)o.n);
    HostObj h;
    h.c = &c;
    h.cells.assign((size_t)(c.nx + 1) * (c.ny + 1) * (c.nz + 1), 0);
    std::vector<int32_t> lin(o.n);
    std::vector<int32_t> ncm(c.N);
    FOPIS_CUDA(cudaMemcpy(ncm.data(), c.node_cmat, sizeof(int32_t) * c.N, cudaMemcpyDeviceToHost));
    h.node_cmat.assign(c.N, -1);
    for (int m = 0; m < o.n; ++m) {
        const int i = d->cmat_nodes[3 * m], j = d->cmat_nodes[3 * m + 1], k = d->cmat_nodes[3 * m + 2];
        if (i < 0 || j < 0 || k < 0 || i >= c.cx || j >= c.cy || k >= c.cz)
            throw ApiError{FOPIS_ERR_ARG, "surface node outside the grid"};
        const size_t L = ((size_t)i * c.cy + j) * c.cz + k;
        if (ncm[L] >= 0) throw ApiError{FOPIS_ERR_ARG, "surface node shared by two objects"};
        ncm[L] = (id << 24) | m;
        h.node_cmat[L] = m;
        lin[m] = (int32_t)L;
    }
    std::vector<uint8_t> cmap(c.N);
    FOPIS_CUDA(cudaMemcpy(cmap.data(), c.cellmap, c.N, cudaMemcpyDeviceToHost));
    for (int m = 0; m < d->n_cells; ++m) {
        const int i = d->cells[3 * m], j = d->cells[3 * m + 1], k = d->cells[3 * m + 2];
        if (i < 0 || j < 0 || k < 0 || i > c.nx || j > c.ny || k > c.nz) throw ApiError{FOPIS_ERR_ARG, "cell outside the grid"};
        cmap[((size_t)i * c.cy + j) * c.cz + k] = (uint8_t)(id + 1);
        h.cells[((size_t)i * (c.ny + 1) + j) * (c.nz + 1) + k] = 1;
    }
    FOPIS_CUDA(cudaMemcpy(c.node_cmat, ncm.data(), sizeof(int32_t) * c.N, cudaMemcpyHostToDevice));
    FOPIS_CUDA(cudaMemcpy(c.cellmap, cmap.data(), c.N, cudaMemcpyHostToDevice));
    FOPIS_CUDA(cudaMalloc(&o.nodes, sizeof(int32_t) * o.n));
    FOPIS_CUDA(cudaMemcpy(o.nodes, lin.data(), sizeof(int32_t) * o.n, cudaMemcpyHostToDevice));
    FOPIS_CUDA(cudaMalloc(&o.C, sizeof(double) * (size_t)o.n * o.n));
    FOPIS_CUDA(cudaMalloc(&o.colsum, sizeof(double) * o.n));
    FOPIS_CUDA(cudaMalloc(&o.charge_tmp, sizeof(long long) * (size_t)c.nsp * o.n));
    FOPIS_CUDA(cudaMalloc(&o.charge_map, sizeof(double) * (size_t)c.nsp * o.n));
    FOPIS_CUDA(cudaMalloc(&o.phis, sizeof(double) * o.n));
    FOPIS_CUDA(cudaMalloc(&o.drho_buf, sizeof(double) * 3 * o.n));
    FOPIS_CUDA(cudaMemset(o.drho_buf, 0, sizeof(double) * 3 * o.n));
    for (int q = 0; q < 3; ++q) o.drho[q] = o.drho_buf + (size_t)q * o.n;
    FOPIS_CUDA(cudaMalloc(&o.scal, sizeof(double) * 8));
    FOPIS_CUDA(cudaMemset(o.charge_tmp, 0, sizeof(long long) * (size_t)c.nsp * o.n));
    FOPIS_CUDA(cudaMemset(o.charge_map, 0, sizeof(double) * (size_t)c.nsp * o.n));
    FOPIS_CUDA(cudaMemset(o.scal, 0, sizeof(double) * 8));
    o.is_fixed = d->is_potential_fixed;
    o.fixed_potential = d->fixed_potential;
    o.offset = d->initial_potential_offset;
    o.emit_species = d->emit_species;
    o.secondary_species = -1;
    if (d->secondary_species >= 0) {
        if (d->secondary_species >= c.nsp || c.p.species[d->secondary_species].kind != FOPIS_SPECIES_SECONDARY)
            throw ApiError{FOPIS_ERR_ARG, "secondary_species must name a species of kind FOPIS_SPECIES_SECONDARY"};
        if (!(c.p.energy_ev > 0.0)) throw ApiError{FOPIS_ERR_ARG, "secondary emission needs params.energy_ev"};
        o.secondary_species = d->secondary_species;
        if (c.inc.cap == 0) {   // one incident list per context, as long as the absorbed list
            c.inc.cap = c.ab.cap;
            double** fl[7] = {&c.inc.x, &c.inc.y, &c.inc.z, &c.inc.vx, &c.inc.vy, &c.inc.vz, &c.inc.trem};
            for (auto* q : fl) FOPIS_CUDA(cudaMalloc(q, sizeof(double) * c.inc.cap));
            FOPIS_CUDA(cudaMalloc(&c.inc.species, c.inc.cap));
            FOPIS_CUDA(cudaMalloc(&c.inc.object, c.inc.cap));
            FOPIS_CUDA(cudaMalloc(&c.inc.axis, c.inc.cap));
            FOPIS_CUDA(cudaMalloc(&c.inc.count, sizeof(int32_t) * c.inc.cap));
        }
    }
    o.dielectric = d->dielectric ? 1 : 0;
    if (o.dielectric) {
        if (!d->capacitance) throw ApiError{FOPIS_ERR_ARG, "a dielectric surface needs its node capacitances"};
        FOPIS_CUDA(cudaMalloc(&o.capacitance, sizeof(double) * o.n));
        FOPIS_CUDA(cudaMemcpy(o.capacitance, d->capacitance, sizeof(double) * o.n, cudaMemcpyHostToDevice));
    }
    // lit nodes of the emitting face (Spacecraft::emitParticles, Spacecraft.cpp:836-886)
    std::vector<int32_t> lit, lit_ijk;
    if (o.emit_species >= 0 && o.emit_species < c.nsp &&
        c.p.species[o.emit_species].kind == FOPIS_SPECIES_PHOTOELECTRON) {
        int eaxis = -1;
        for (int q = 0; q < 3; ++q) if (std::fabs(c.p.shine_vector[q]) == 1.0) { eaxis = q; break; }
        if (eaxis >= 0) {
            const int sign = c.p.shine_vector[eaxis] > 0.0 ? 1 : -1;
            for (int m = 0; m < o.n; ++m) {
                const int i = d->cmat_nodes[3 * m], j = d->cmat_nodes[3 * m + 1], k = d->cmat_nodes[3 * m + 2];
                if (h.surface_point(eaxis, i, j, k, sign)) {
                    lit.push_back(m);
                    lit_ijk.push_back((i << 20) | (j << 10) | k);
                }
            }
        }
    }
    o.n_lit = (int)lit.size();
    if (o.n_lit) {
        FOPIS_CUDA(cudaMalloc(&o.lit, sizeof(int32_t) * 2 * o.n_lit));
        FOPIS_CUDA(cudaMemcpy(o.lit, lit.data(), sizeof(int32_t) * o.n_lit, cudaMemcpyHostToDevice));
        FOPIS_CUDA(cudaMemcpy(o.lit + o.n_lit, lit_ijk.data(), sizeof(int32_t) * o.n_lit, cudaMemcpyHostToDevice));
    }
}

static void finish_C(Ctx& c, ObjectDev& o) {
    ++c.launches;
    colsum_kernel<<<grid1(o.n), kT, 0, c.st>>>(o.C, o.n, o.colsum);
    ++c.launches;
    total_kernel<<<1, 1024, 0, c.st>>>(o.colsum, o.n, o.scal + 3);
    FOPIS_LAUNCH_CHECK();
    double tot = 0.0;
    FOPIS_CUDA(cudaMemcpyAsync(&tot, o.scal + 3, sizeof(double), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    o.total = tot;
    o.has_C = true;
    if (o.offset != 0.0) {
        o.potential = o.offset;
        ++c.launches;
        offset_kernel<<<grid1((long long)o.n * 32), kT, 0, c.st>>>(o.C, o.n, o.offset, o.charge_map);
        FOPIS_LAUNCH_CHECK();
    }
}

void cmatrix_build(Ctx& c, int id) {
    ObjectDev& o = c.objs[id];
    const int n = o.n;
    double* B = o.C;
    // keep the user's fields: the reference builds C before any particle exists
    FOPIS_CUDA(cudaMemsetAsync(c.rho0, 0, sizeof(double) * c.N, c.st));
    const double tol = std::min(c.p.poisson_tol > 0 ? c.p.poisson_tol : 1e-8, 1e-10);
    for (int col = 0; col < n; ++col) {
        const long long node = ((long long)o.nodes_ijk[3 * col] * c.cy + o.nodes_ijk[3 * col + 1]) * c.cz + o.nodes_ijk[3 * col + 2];
        ++c.launches;
        set_node_kernel<<<1, 1, 0, c.st>>>(c.rho0, node, 1.0);
        FOPIS_CUDA(cudaMemsetAsync(c.phi, 0, sizeof(double) * c.N, c.st));
        const int rc = mg_solve(c, tol, 200);
        if (rc != FOPIS_OK) throw ApiError{rc, "capacity-matrix column solve did not converge"};
        // capacity_matrix(col, row) = phi at row (RootGridObject.cpp:114-126)
        ++c.launches;
        gather_kernel<<<grid1(n), kT, 0, c.st>>>(c.phi, o.nodes, n, B + (size_t)col * n);
        ++c.launches;
        set_node_kernel<<<1, 1, 0, c.st>>>(c.rho0, node, 0.0);
        FOPIS_LAUNCH_CHECK();
    }
    FOPIS_CUDA(cudaMemsetAsync(c.phi, 0, sizeof(double) * c.N, c.st));
    double* rowk = nullptr;
    unsigned* bad = nullptr;
    FOPIS_CUDA(cudaMalloc(&rowk, sizeof(double) * 2 * n));
    FOPIS_CUDA(cudaMalloc(&bad, sizeof(unsigned)));
    FOPIS_CUDA(cudaMemsetAsync(bad, 0, sizeof(unsigned), c.st));
    for (int k = 0; k < n; ++k) {
        ++c.launches;
        gj_copy_kernel<<<grid1(n), kT, 0, c.st>>>(B, n, k, rowk, rowk + n);
        ++c.launches;
        gj_update_kernel<<<grid1((long long)n * n), kT, 0, c.st>>>(B, n, k, rowk, rowk + n, bad);
    }
    FOPIS_LAUNCH_CHECK();
    unsigned hbad = 0;
    FOPIS_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, c.st));
    FOPIS_CUDA(cudaStreamSynchronize(c.st));
    cudaFree(rowk);
    cudaFree(bad);
    if (hbad) throw ApiError{FOPIS_ERR_DEVICE, "capacity matrix B is not positive definite"};
    finish_C(c, o);
}

void cmatrix_set(Ctx& c, int id, const double* hostC) {
    ObjectDev& o = c.objs[id];
    FOPIS_CUDA(cudaMemcpy(o.C, hostC, sizeof(double) * (size_t)o.n * o.n, cudaMemcpyHostToDevice));
    finish_C(c, o);
}

void objects_step_begin(Ctx& c) {
    FOPIS_CUDA(cudaMemsetAsync(&c.d_sc->absorbed_n, 0, sizeof(unsigned long long), c.st));
    FOPIS_CUDA(cudaMemsetAsync(c.d_sc->absorbed_by, 0, sizeof(c.d_sc->absorbed_by), c.st));
    FOPIS_CUDA(cudaMemsetAsync(c.d_sc->emitted_by, 0, sizeof(c.d_sc->emitted_by), c.st));
}

// Moves the step's fixed-point surface charge into the charge maps and the
// total charge into scal[1] (RootGrid::updateRho's sumWholeCharge).
void objects_step_end(Ctx& c) {
    for (auto& o : c.objs) {
        double sc[FOPIS_MAX_SPECIES];
        for (int s = 0; s < c.nsp; ++s) sc[s] = c.p.species[s].charge * c.p.species[s].size * kSurfaceUnit;
        double* dsc = c.scratch64;   // small staging area
        FOPIS_CUDA(cudaMemcpyAsync(dsc, sc, sizeof(double) * c.nsp, cudaMemcpyHostToDevice, c.st));
        ++c.launches;
        sum_charge_kernel<<<1, 1024, 0, c.st>>>(o.charge_tmp, o.charge_map, c.nsp, o.n, dsc, o.scal);
        FOPIS_LAUNCH_CHECK();
        FOPIS_CUDA(cudaStreamSynchronize(c.st));
    }
}

void redistribute(Ctx& c) {
    for (auto& o : c.objs) {
        if (!o.has_C) throw ApiError{FOPIS_ERR_STATE, "capacity matrix not built"};
        ++c.launches;
        potential_kernel<<<1, 1024, 0, c.st>>>(c.phi, o.nodes, o.colsum, o.n, o.total, o.is_fixed, o.fixed_potential,
                                                o.phis, o.scal, o.dielectric ? o.capacitance : nullptr, o.charge_map,
                                                c.nsp);
        ++c.launches;
        drho_kernel<<<grid1((long long)o.n * 32), kT, 0, c.st>>>(o.C, o.n, o.phis, o.scal, o.nodes, c.rho0, o.drho[0]);
        FOPIS_LAUNCH_CHECK();
        double sc[2];
        FOPIS_CUDA(cudaMemcpyAsync(sc, o.scal, sizeof(double) * 2, cudaMemcpyDeviceToHost, c.st));
        FOPIS_CUDA(cudaStreamSynchronize(c.st));
        o.potential = sc[0];
        o.total_charge = sc[1];
    }
    glue_copy(c, c.rho0);
}

// phi (the first solve's result) += the fitted conductor responses.
void conductor_start(Ctx& c) {
    if (c.obj_hist < 1 || c.objs.empty()) return;
    ConductorFit f{};
    f.nobj = (int)c.objs.size();
    f.terms = c.obj_hist >= 2 ? 2 : 1;
    for (int o = 0; o < f.nobj; ++o) {
        f.d0[o] = c.objs[o].drho[0]; f.d1[o] = c.objs[o].drho[1]; f.d2[o] = c.objs[o].drho[2];
        f.n[o] = c.objs[o].n;
    }
    double* alpha = &c.d_sc->red[12];
    ++c.launches;
    conductor_fit_kernel<<<1, 1024, 0, c.st>>>(f, alpha);
    ++c.launches;
    conductor_start_kernel<<<grid1((long long)c.N), kT, 0, c.st>>>(c.phi, c.phi_obj, c.phi_obj2, alpha, (long long)c.N);
    FOPIS_LAUNCH_CHECK();
}

// After the second solve: the response phi_final - phi_first becomes the
// newest history entry, with this step's redistributed charge.
void conductor_record(Ctx& c, const double* phi_first) {
    std::swap(c.phi_obj, c.phi_obj2);
    phi_axpy(c, c.phi_obj, c.phi, phi_first, -1.0);
    for (auto& o : c.objs) {
        double* oldest = o.drho[2];
        o.drho[2] = o.drho[1];
        o.drho[1] = o.drho[0];
        o.drho[0] = oldest;
    }
    c.obj_hist = std::min(2, c.obj_hist + 1);
}

}  // namespace fopis
