// fopis_host.cpp — the host classes of fopis_host.hpp over the C ABI.
#include <iostream>

#include "fopis_host.hpp"
#include "datafile.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sys/stat.h>

#include "json.hpp"

namespace fopis {
namespace host {

// ---------------------------------------------------------------- units
// Normalizer::updatePhysicalConstants (include/normalizer.hpp:24-38) in the
// reference's operation order, so every factor is the reference's to the bit:
// pow(u, 2) is the product u * u (the compiler's form of it), pow(u, 3) the libm pow.
Normalizer::Normalizer(double dx, double dt) : x(dx), t(dt) {
    const double x_pow_3 = std::pow(dx, 3.0);
    V_unit = (dx * dx) * kMe / (kE * (dt * dt));
    A_unit = kE / dt;
    eps0 = kEps0 * (x_pow_3 * kMe) / ((kE * kE) * (dt * dt));   // Normalizer::normalizeEpsilon
    mu0 = kMu0 * (kE * kE) / (kMe * dx);                         // Normalizer::normalizeMu
    c = velocity(kClight);                                       // Normalizer::normalizeVelocity(c)
}

void calc_flux(double vth, double density_norm, double size, const double drift[3], const int injection_axis[6],
               double flux[6]) {
    // numerical integral of v f(v) over [-6, 6] thermal units, step 1e-3, split by the sign of v
    const double ddv = 1e-3;
    const double nvx = 12.0 / ddv;
    for (int axis = 0; axis < 3; ++axis) {
        const double d = drift[axis] / vth;
        double lo = 0.0, hi = 0.0;
        for (int i = 0; i < nvx - 1; ++i) {
            const double arg1 = i * ddv + (d - 6.0);
            const double argx1 = std::pow(arg1 - d, 2.0);
            if (arg1 > 0.0) lo += arg1 * std::exp(-argx1) * ddv;
            else hi += arg1 * std::exp(-argx1) * ddv;
        }
        flux[2 * axis] = lo * (vth / std::sqrt(M_PI)) * density_norm / size;
        flux[2 * axis + 1] = -hi * (vth / std::sqrt(M_PI)) * density_norm / size;
    }
    for (int k = 0; k < 6; ++k) if (!injection_axis[k]) flux[k] = 0.0;
}

fopis_species ParticleType::to_abi(const Normalizer& norm, double dx) const {
    fopis_species s{};
    s.kind = type == "ambient" ? FOPIS_SPECIES_AMBIENT
             : type == "photoelectron" ? FOPIS_SPECIES_PHOTOELECTRON : FOPIS_SPECIES_SECONDARY;
    s.particle_per_cell = particle_per_cell;
    s.charge = charge;
    s.mass = mass;
    s.size = (double)(long long)(std::pow(dx, 3.0) * density / particle_per_cell);   // ParticleType::updateSize
    const double T = kE * temperature;                                               // setTemperature: e * T[eV]
    s.thermal_velocity = norm.velocity(std::sqrt(2.0 * T / (mass * kMe)));
    s.deviation = norm.velocity(std::sqrt(T / (mass * kMe)));
    for (int a = 0; a < 3; ++a) s.drift[a] = drift_kms[a] * (1e3 * norm.velocity(1.0));   // Initialize.cpp:353-355
    for (int a = 0; a < 6; ++a) s.injection_axis[a] = injection_axis[a];
    if (type == "ambient") {
        const double dens_norm = density * std::pow(dx, 3.0);                         // normalizeDensity
        calc_flux(s.thermal_velocity, dens_norm, s.size, s.drift, s.injection_axis, s.flux);
    } else if (type == "photoelectron") {
        const double j = norm.current_density(current_density);
        s.emission_amount = 1.0 * j / (std::fabs(charge) * s.size);                   // dx^2 = 1 (Spacecraft.cpp:876-877)
    }
    return s;
}

// ---------------------------------------------------------------- input.json
namespace {

std::string dir_of(const std::string& path) {
    const size_t s = path.find_last_of('/');
    return s == std::string::npos ? std::string(".") : path.substr(0, s);
}

void parse_obj(const std::string& path, int nx, int ny, int nz, ObjectSpec& o) {
    int32_t *nodes = nullptr, *cells = nullptr;
    int nn = 0, nc = 0;
    const int rc = fopis_parse_obj(path.c_str(), nx, ny, nz, &nodes, &nn, &cells, &nc);
    if (rc != FOPIS_OK) throw Error(rc, "cannot parse " + path);
    o.nodes.assign(nodes, nodes + 3 * (size_t)nn);
    o.cells.assign(cells, cells + 3 * (size_t)nc);
    fopis_free(nodes);
    fopis_free(cells);
}

// Per-node texture lists of the same file (ObjectDataFromFile::textures), turned
// into the dielectric capacitance map of Spacecraft::construct (Spacecraft.cpp:
// 117-149): per node the mean over its quads of normalizeCapacitance(4 pi eps0
// eps_r) of the quad's material; an unknown material name is an error there too.
void node_capacitance(const std::string& path, int nx, int ny, int nz, const std::map<int, std::string>& materials,
                      const Normalizer& norm, ObjectSpec& o) {
    // Spacecraft::material_property_list (SpacecraftMaterialPropertyList.cpp:3-34)
    static const std::map<std::string, double> eps_r = {{"Silicon", 12.0}, {"Aluminum", 9.5}, {"EpoxyGlass", 5.0},
                                                        {"Bakelite", 4.8}, {"GlassReinforcedTeflon", 2.32},
                                                        {"Teflon", 2.1}};
    int32_t *start = nullptr, *tex = nullptr;
    int n = 0;
    const int rc = fopis_parse_obj_textures(path.c_str(), nx, ny, nz, &start, &tex, &n);
    if (rc != FOPIS_OK) throw Error(rc, "cannot parse " + path);
    o.capacitance.assign(n, 0.0);
    try {
        for (int m = 0; m < n; ++m) {
            double acc = 0.0;
            for (int t = start[m]; t < start[m + 1]; ++t) {
                const auto it = materials.find(tex[t]);
                const auto pe = it == materials.end() ? eps_r.end() : eps_r.find(it->second);
                if (pe == eps_r.end())
                    throw Error(FOPIS_ERR_ARG, "Invalid material name " + (it == materials.end() ? std::string("") : it->second) +
                                                   " is specified to be assigned the texture index " + std::to_string(tex[t]) + ".");
                acc += 4.0 * M_PI * kEps0 * pe->second * norm.V_unit / kE;   // normalizeCapacitance
            }
            o.capacitance[m] = acc / (start[m + 1] - start[m]);
        }
    } catch (...) {
        fopis_free(start);
        fopis_free(tex);
        throw;
    }
    fopis_free(start);
    fopis_free(tex);
}

}  // namespace

Input load_input(const std::string& path) {
    const Value js = Value::parse_file(path);
    Input in;
    const Value& env = js["Environment"];
    in.dx = env["dx"].number();
    in.dt = env["dt"].number();
    const int nxyz[3] = {env["nx"].integer(), env["ny"].integer(), env["nz"].integer()};
    if (env.integer_or("proc_x", 1) * env.integer_or("proc_y", 1) * env.integer_or("proc_z", 1) != 1)
        throw Error(FOPIS_ERR_ARG, "the whole domain lives on one GPU: proc_x = proc_y = proc_z = 1");
    in.max_timestep = env.integer_or("max_timestep", 0);
    in.job_type = env.str_or("job_type", "new");
    if (in.job_type != "new" && in.job_type != "load")
        throw Error(FOPIS_ERR_ARG, "Unknown jobtype, neither ``new'' or ``load'', was inputted.");   // Initialize.cpp:97-99
    in.norm = Normalizer(in.dx, in.dt);
    const Normalizer& norm = in.norm;
    const std::string solver = env.str_or("solver_type", "ES");
    if (solver != "ES" && solver != "EM") throw Error(FOPIS_ERR_ARG, "solver_type " + solver + " is neither ES nor EM");
    // Environment::checkCFLCondition (src/Misc/Environment.cpp:193-203) aborts an EM run
    if (solver == "EM" && norm.c > 1.0)
        throw Error(FOPIS_ERR_ARG, "Courant number exceeds 1.0 (c dt / dx = " + std::to_string(norm.c) + ")");

    std::vector<ParticleType> species;
    for (const auto& kv : js["Plasma"].items()) {        // std::map order, as picojson's
        const Value& pl = kv.second;
        ParticleType p;
        p.name = kv.first;
        p.type = pl["type"].str();
        if (p.type != "ambient" && p.type != "photoelectron" && p.type != "secondary")
            throw Error(FOPIS_ERR_ARG, "species type " + p.type + " is outside the ES hot path");
        p.mass = pl["mass"].number();
        p.charge = pl["charge"].number();
        p.density = pl["density"].number();
        p.temperature = pl["temperature"].number();
        p.particle_per_cell = pl["particle_per_cell"].integer();
        if (pl.has("drift_velocity"))
            for (int a = 0; a < 3; ++a) p.drift_kms[a] = pl["drift_velocity"][a].number();
        if (pl.has("injection_axis"))
            for (int a = 0; a < 6; ++a) p.injection_axis[a] = pl["injection_axis"][a].boolean() ? 1 : 0;
        p.current_density = pl.number_or("current_density", 0.0);
        species.push_back(p);
    }
    // Environment::resetParticleTypeOrder (Environment.cpp:360-377): ambient, photoelectron, secondary
    std::stable_partition(species.begin(), species.end(), [](const ParticleType& p) { return p.type == "ambient"; });
    std::stable_partition(species.begin(), species.end(), [](const ParticleType& p) { return p.type != "secondary"; });
    in.species = species;

    double bfield[3] = {0.0, 0.0, 0.0}, shine[3] = {0.0, 0.0, 0.0};
    if (js.has("Field")) {
        const Value& f = js["Field"];
        if (f.has("static_bfield")) for (int a = 0; a < 3; ++a) bfield[a] = f["static_bfield"][a].number();
        if (f.has("shine_vector")) for (int a = 0; a < 3; ++a) shine[a] = f["shine_vector"][a].number();
    }
    if (js.has("Options")) in.use_existing_capacity_matrix = js["Options"].boolean_or("use_existing_capacity_matrix", false);
    // the IO section's energy-log width (Initialize.cpp:219-250, cast from a number as there);
    // the other widths select field files, which are not written here
    if (js.has("IO")) in.plot_energy_width = static_cast<int>(js["IO"].number_or("plot_energy_width", 0.0));

    fopis_params& p = in.params;
    p.nx = nxyz[0]; p.ny = nxyz[1]; p.nz = nxyz[2];
    std::snprintf(p.boundary, sizeof p.boundary, "%s", env["boundary"].str().c_str());
    p.eps0 = norm.eps0;
    for (int a = 0; a < 3; ++a) {
        p.static_bfield[a] = bfield[a] * (norm.bfield(1.0) * 1e-9);   // nT (Initialize.cpp:314-318)
        p.shine_vector[a] = shine[a];
    }
    if ((int)species.size() > FOPIS_MAX_SPECIES) throw Error(FOPIS_ERR_ARG, "too many species");
    p.nspecies = (int)species.size();
    for (size_t i = 0; i < species.size(); ++i) p.species[i] = species[i].to_abi(norm, in.dx);
    p.poisson_tol = 1e-8;
    p.max_vcycles = 100;
    p.guess_mode = FOPIS_GUESS_WARM;
    p.sort_interval = 8;
    p.remove_interval = 50;
    p.capacity_factor = 1.5;
    p.precision = FOPIS_MIXED;
    p.seed = 12345;
    p.energy_ev = norm.unenergy_ev(1.0);   // Normalizer::unnormalizeEnergy(1, "eV")
    p.solver = solver == "EM" ? FOPIS_SOLVER_EM : FOPIS_SOLVER_ES;
    p.mu0 = norm.mu0;

    if (js.has("Object")) {
        const std::string base = dir_of(path);
        for (const auto& kv : js["Object"].items()) {
            const Value& o = kv.second;
            const std::string surface = o.str_or("surface_type", "perfect");
            if (surface != "perfect" && surface != "dielectric")
                throw Error(FOPIS_ERR_ARG, "surface_type " + surface + " is not perfect or dielectric");
            ObjectSpec spec;
            spec.name = kv.first;
            std::string file = o["file_name"].str();
            spec.file_name = file.substr(file.find_last_of('/') == std::string::npos ? 0 : file.find_last_of('/') + 1);
            if (!file.empty() && file[0] != '/') file = base + "/" + file;
            parse_obj(file, nxyz[0], nxyz[1], nxyz[2], spec);
            spec.is_potential_fixed = o.boolean_or("is_potential_fixed", false) ? 1 : 0;
            spec.fixed_potential = norm.potential(o.number_or("fixed_potential", 0.0));
            spec.initial_potential_offset = norm.potential(o.number_or("initial_potential_offset", 0.0));
            if (o.has("emit_particles"))
                for (const auto& e : o["emit_particles"].items())
                    for (size_t s = 0; s < species.size(); ++s) {
                        if (species[s].name == e.first && species[s].type == "photoelectron") spec.emit_species = (int)s;
                        if (species[s].name == e.first && species[s].type == "secondary") spec.secondary_species = (int)s;
                    }
            if (surface == "dielectric") {
                std::map<int, std::string> mats;
                if (o.has("materials"))
                    for (const auto& m : o["materials"].items()) mats[std::stoi(m.first)] = m.second.str();
                spec.dielectric = 1;
                node_capacitance(file, nxyz[0], nxyz[1], nxyz[2], mats, norm, spec);
            }
            in.objects.push_back(spec);
        }
    }
    return in;
}

// ---------------------------------------------------------------- Spacecraft
namespace {
std::string fmt(const char* f, double v) {
    char b[64];
    std::snprintf(b, sizeof b, f, v);
    return b;
}
std::string fmts(const char* f, const std::string& v) {
    char b[256];
    std::snprintf(b, sizeof b, f, v.c_str());
    return b;
}
}  // namespace

std::string Spacecraft::getLogHeader(const std::vector<ParticleType>& species) const {
    std::string h = fmts("%16s", "Potential [V]") + " " + fmts("%16s", "Charge [C]");
    for (const auto& s : species) h += " " + fmts("%16s", s.name + " [A]");
    return h;
}
std::string Spacecraft::getLogEntry(const Normalizer& norm) const {
    std::string e = fmt("%16.7e", norm.unpotential(potential)) + " " + fmt("%16.7e", norm.uncharge(total_charge));
    for (double c : current) e += " " + fmt("%16.7e", norm.uncurrent(c));
    return e;
}

// ---------------------------------------------------------------- RootGrid
RootGrid::RootGrid(const Input& in, int device) : in_(in) {
    const int rc = fopis_create(&in_.params, device, &ctx_);
    if (rc != FOPIS_OK) throw Error(rc, fopis_last_error(nullptr));
    for (const auto& o : in_.objects) {
        fopis_object_desc d{};
        d.n_cmat = o.n_cmat();
        d.cmat_nodes = o.nodes.data();
        d.n_cells = (int)(o.cells.size() / 3);
        d.cells = o.cells.data();
        d.is_potential_fixed = o.is_potential_fixed;
        d.fixed_potential = o.fixed_potential;
        d.initial_potential_offset = o.initial_potential_offset;
        d.emit_species = o.emit_species;
        d.secondary_species = o.secondary_species;
        d.dielectric = o.dielectric;
        d.capacitance = o.dielectric ? o.capacitance.data() : nullptr;
        int id = -1;
        check(fopis_add_object(ctx_, &d, &id));
        object_ids_.push_back(id);
    }
}

RootGrid::~RootGrid() {
    if (ctx_) fopis_destroy(ctx_);
}

void RootGrid::check(int rc, bool allow_not_converged) const {
    if (rc == FOPIS_OK || (allow_not_converged && rc == FOPIS_ERR_NOT_CONVERGED)) return;
    throw Error(rc, fopis_last_error(ctx_));
}

void RootGrid::initializeObjectsCmatrix(const std::string& resume_dir) {
    for (size_t k = 0; k < in_.objects.size(); ++k) {
        if (!resume_dir.empty() && in_.use_existing_capacity_matrix && io::loadCmatrixData(*this, (int)k, resume_dir))
            continue;
        check(fopis_build_capacity_matrix(ctx_, object_ids_[k]));
        if (!resume_dir.empty()) io::writeCmatrixData(*this, (int)k, resume_dir);
    }
}

void RootGrid::setTimestep(int64_t t) { check(fopis_set_timestep(ctx_, t)); }

void RootGrid::saveResumeData(const std::string& dir) const {
    make_dirs(dir);
    DataFile f;
    const int nsp = in_.params.nspecies;
    std::vector<double> carry(6 * (size_t)nsp);
    check(fopis_get_injection_carry(ctx_, carry.data(), 6 * nsp));
    for (int s = 0; s < nsp; ++s) {
        const std::string g = in_.species[s].name + "/";
        const std::vector<Particle> p = getParticles(s);
        const uint64_t n = p.size();
        std::vector<double> col[6];
        for (auto& c : col) c.resize(n);
        for (uint64_t i = 0; i < n; ++i) {
            col[0][i] = p[i].x; col[1][i] = p[i].y; col[2][i] = p[i].z;
            col[3][i] = p[i].vx; col[4][i] = p[i].vy; col[5][i] = p[i].vz;
        }
        f.put_f64(g + "size", (double)n);                     // the reference writes the count as a double
        const char* keys[6] = {"x", "y", "z", "vx", "vy", "vz"};
        for (int q = 0; q < 6; ++q) f.put_f64(g + keys[q], {n}, col[q].data());
        // the reference records its mt19937 draw counts here; the Philox draws are keyed
        // by (seed, timestep), so the seed and the timestep take their place
        const int64_t counts[2] = {(int64_t)in_.params.seed, timestep()};
        f.put_i64(g + "generated_counts", {2}, counts);
        f.put_f64(g + "injection_carry", {6}, carry.data() + 6 * s);
    }
    const uint64_t dims[3] = {(uint64_t)in_.params.nx + 2, (uint64_t)in_.params.ny + 2, (uint64_t)in_.params.nz + 2};
    const std::vector<uint64_t> shape(dims, dims + 3);
    f.put_f64("Potential/phi", shape, getField(FOPIS_FIELD_PHI).data());
    // nodal E (the reference stores its edge E; here it follows from phi)
    f.put_f64("Efield/exref", shape, getField(FOPIS_FIELD_EXREF).data());
    f.put_f64("Efield/eyref", shape, getField(FOPIS_FIELD_EYREF).data());
    f.put_f64("Efield/ezref", shape, getField(FOPIS_FIELD_EZREF).data());
    if (in_.params.solver == FOPIS_SOLVER_EM) {
        // RootGrid::saveResumeFieldData (RootGridIO.cpp:236-271): the Yee E and B, damping layers included
        const char* names[6] = {"Efield/ex", "Efield/ey", "Efield/ez", "Bfield/bx", "Bfield/by", "Bfield/bz"};
        for (int q = 0; q < 6; ++q) {
            int lo[3], n[3];
            check(fopis_field_shape(ctx_, FOPIS_FIELD_EX + q, lo, n));
            std::vector<double> v((size_t)n[0] * n[1] * n[2]);
            check(fopis_get_field(ctx_, FOPIS_FIELD_EX + q, v.data(), v.size()));
            f.put_f64(names[q], {(uint64_t)n[0], (uint64_t)n[1], (uint64_t)n[2]}, v.data());
        }
    }
    for (size_t k = 0; k < in_.objects.size(); ++k) {
        const int n = in_.objects[k].n_cmat();
        std::vector<double> cm((size_t)nsp * n);
        check(fopis_get_charge_map(ctx_, object_ids_[k], cm.data(), nsp * n));
        f.put_f64(in_.objects[k].name + "/charge_map", {(uint64_t)nsp, (uint64_t)n}, cm.data());
    }
    f.save(dir + "/grid_id_0.bin");
}

void RootGrid::loadResumeData(const std::string& dir) {
    const DataFile f = DataFile::load(dir + "/grid_id_0.bin");
    const int nsp = in_.params.nspecies;
    std::vector<double> carry(6 * (size_t)nsp, 0.0);
    for (int s = 0; s < nsp; ++s) {
        const std::string g = in_.species[s].name + "/";
        const uint64_t n = (uint64_t)f.f64_scalar(g + "size");
        if (n == 0) continue;
        const char* keys[6] = {"x", "y", "z", "vx", "vy", "vz"};
        std::vector<double> col[6];
        for (int q = 0; q < 6; ++q) {
            col[q] = f.f64(g + keys[q]);
            if (col[q].size() != n) throw std::runtime_error("resume data: " + g + keys[q] + " has the wrong length");
        }
        std::vector<Particle> p(n);
        for (uint64_t i = 0; i < n; ++i)
            p[i] = Particle{col[0][i], col[1][i], col[2][i], col[3][i], col[4][i], col[5][i], s, 1};
        loadParticles(s, p);
        if (f.has(g + "injection_carry")) {
            const std::vector<double> c = f.f64(g + "injection_carry");
            if (c.size() == 6) for (int q = 0; q < 6; ++q) carry[6 * s + q] = c[q];
        }
    }
    check(fopis_set_injection_carry(ctx_, carry.data(), 6 * nsp));
    const std::vector<double> phi = f.f64("Potential/phi");
    const size_t N = (size_t)(in_.params.nx + 2) * (in_.params.ny + 2) * (in_.params.nz + 2);
    if (phi.size() != N) throw std::runtime_error("resume data: Potential/phi has the wrong size");
    check(fopis_set_field(ctx_, FOPIS_FIELD_PHI, phi.data(), N));
    if (in_.params.solver == FOPIS_SOLVER_EM) {   // RootGrid::loadResumeFieldData (RootGridIO.cpp:181-234)
        const char* names[6] = {"Efield/ex", "Efield/ey", "Efield/ez", "Bfield/bx", "Bfield/by", "Bfield/bz"};
        for (int q = 0; q < 6; ++q) {
            int lo[3], n[3];
            check(fopis_field_shape(ctx_, FOPIS_FIELD_EX + q, lo, n));
            const std::vector<double> v = f.f64(names[q]);
            if (v.size() != (size_t)n[0] * n[1] * n[2])
                throw std::runtime_error(std::string("resume data: ") + names[q] + " has the wrong size");
            check(fopis_set_field(ctx_, FOPIS_FIELD_EX + q, v.data(), v.size()));
        }
    }
    for (size_t k = 0; k < in_.objects.size(); ++k) {
        const int n = in_.objects[k].n_cmat();
        const std::vector<double> cm = f.f64(in_.objects[k].name + "/charge_map");
        if (cm.size() != (size_t)nsp * n) throw std::runtime_error("resume data: charge_map of " + in_.objects[k].name);
        check(fopis_set_charge_map(ctx_, object_ids_[k], cm.data(), nsp * n));
    }
}

// Grid::initializeForLoad (Grid.cpp:38-50): nodal E from the saved potential
// (the reference reads its saved edge E), then updateRho, which with objects
// runs the first solve and the redistribution of the restored charge map.
void RootGrid::initializeForLoad() {
    if (in_.params.solver == FOPIS_SOLVER_EM) {
        // EM: updateRho, then the nodal E and B from the restored Yee arrays
        check(fopis_sort_particles(ctx_));
        updateRho();
        check(fopis_update_reference_fields(ctx_));
        return;
    }
    updateEfield();
    check(fopis_sort_particles(ctx_));
    updateRho();
}

void RootGrid::generateAmbientParticles() { check(fopis_generate_ambient(ctx_)); }
void RootGrid::loadParticles(int species, const std::vector<Particle>& p) {
    check(fopis_load_particles(ctx_, species, p.data(), (int64_t)p.size()));
}
void RootGrid::initialize() { check(fopis_initialize(ctx_), true); }
void RootGrid::mainLoop() { check(fopis_step(ctx_, 1), true); }
void RootGrid::setGuessMode(int mode) { check(fopis_set_guess_mode(ctx_, mode)); }
void RootGrid::updateParticleVelocity() { check(fopis_update_velocity(ctx_)); }
void RootGrid::emitParticlesFromObjects() { check(fopis_emit_particles(ctx_)); }
void RootGrid::updateParticlePosition() { check(fopis_update_position(ctx_)); }
void RootGrid::injectParticlesFromBoundary() { check(fopis_inject_particles(ctx_)); }
void RootGrid::updateRho() { check(fopis_update_rho(ctx_), true); }
void RootGrid::solvePoisson() { check(fopis_solve_poisson(ctx_), true); }
void RootGrid::updateEfield() { check(fopis_update_efield(ctx_)); }
void RootGrid::advanceTimestep() { check(fopis_advance_timestep(ctx_)); }

double RootGrid::getParticleEnergy() const {
    double pe = 0.0, fe = 0.0;
    check(fopis_get_energy(ctx_, &pe, &fe));
    return pe;
}
double RootGrid::getEFieldEnergy() const {
    double pe = 0.0, fe = 0.0;
    check(fopis_get_energy(ctx_, &pe, &fe));
    return fe;
}
double RootGrid::getBFieldEnergy() const {
    double be = 0.0;
    check(fopis_get_bfield_energy(ctx_, &be));
    return be;
}
void RootGrid::updateBfield() { check(fopis_update_bfield(ctx_)); }
fopis_stats RootGrid::stats() const {
    fopis_stats st{};
    check(fopis_get_stats(ctx_, &st));
    return st;
}
std::vector<int64_t> RootGrid::getValidParticleNumbers() const {
    const fopis_stats st = stats();
    return std::vector<int64_t>(st.num_particles, st.num_particles + in_.params.nspecies);
}
std::vector<Particle> RootGrid::getParticles(int species) const {
    const int64_t cap = stats().num_particles[species];
    std::vector<Particle> out((size_t)std::max<int64_t>(cap, 1));
    int64_t n = 0;
    check(fopis_get_particles(ctx_, species, out.data(), cap, &n));
    out.resize((size_t)n);
    return out;
}
std::vector<double> RootGrid::getField(int which) const {
    const size_t n = (size_t)(in_.params.nx + 2) * (in_.params.ny + 2) * (in_.params.nz + 2);
    std::vector<double> out(n);
    check(fopis_get_field(ctx_, which, out.data(), n));
    return out;
}
std::vector<Spacecraft> RootGrid::getObjects() const {
    std::vector<Spacecraft> out;
    for (size_t k = 0; k < in_.objects.size(); ++k) {
        Spacecraft s;
        s.name = in_.objects[k].name;
        s.id = object_ids_[k];
        s.current.assign((size_t)in_.params.nspecies, 0.0);
        check(fopis_get_object(ctx_, s.id, &s.potential, &s.total_charge, s.current.data()));
        out.push_back(std::move(s));
    }
    return out;
}

// ---------------------------------------------------------------- IO
namespace io {
namespace {
void ensure_dir(const std::string& dir) { ::mkdir(dir.c_str(), 0755); }
// IO::putHeader / putLog: "%10s %16s %s" and "%10d %16.7e %s"
void put_header(const std::string& file, const std::string& header) {
    std::ofstream f(file, std::ios::out);
    char b[64];
    std::snprintf(b, sizeof b, "%10s %16s ", "Timestep", "Datatime");
    f << b << header << "\n";
}
void put_log(const std::string& file, int timestep, double datatime, const std::string& entry) {
    std::ofstream f(file, std::ios::app);
    char b[64];
    std::snprintf(b, sizeof b, "%10d %16.7e ", timestep, datatime);
    f << b << entry << "\n";
}
}  // namespace

void plot_energy(const RootGrid& g, int timestep, const std::string& dir) {
    ensure_dir(dir);
    const std::string file = dir + "/energy.txt";
    const Normalizer& n = g.input().norm;
    if (timestep == 1) {
        char h[128];
        std::snprintf(h, sizeof h, "%16s %16s %16s %16s", "Energy [J]", "Particle [J]", "EField [J]", "BField [J]");
        put_header(file, h);
    }
    // IO::plotEnergy (src/Misc/IO.cpp:170-194): the B column is nonzero in the EM mode only
    const double pe = g.getParticleEnergy(), fe = g.getEFieldEnergy(), be = g.getBFieldEnergy();
    char e[128];
    std::snprintf(e, sizeof e, "%16.7e %16.7e %16.7e %16.7e", n.unenergy(pe + fe + be), n.unenergy(pe), n.unenergy(fe),
                  n.unenergy(be));
    put_log(file, timestep, timestep * g.input().dt, e);
}

void plot_objects(const RootGrid& g, int timestep, const std::string& dir) {
    ensure_dir(dir);
    for (const auto& s : g.getObjects()) {
        const std::string file = dir + "/object_" + s.name + ".txt";
        if (timestep == 1) put_header(file, s.getLogHeader(g.input().species));
        put_log(file, timestep, timestep * g.input().dt, s.getLogEntry(g.input().norm));
    }
}

void plot_particle_numbers(const RootGrid& g, int timestep, const std::string& dir) {
    ensure_dir(dir);
    const std::string file = dir + "/total_particle_number.txt";
    const auto counts = g.getValidParticleNumbers();
    if (timestep == 1) {
        std::string h = fmts("%16s", "Total");
        for (const auto& s : g.input().species) h += " " + fmts("%16s", s.name);
        put_header(file, h);
    }
    int64_t total = 0;
    for (int64_t c : counts) total += c;
    char b[32];
    std::snprintf(b, sizeof b, "%16lld", (long long)total);
    std::string e = b;
    for (int64_t c : counts) { std::snprintf(b, sizeof b, " %16lld", (long long)c); e += b; }
    put_log(file, timestep, timestep * g.input().dt, e);
}
}  // namespace io

namespace io {

std::string cmatrix_file(const std::string& resume_dir, const ObjectSpec& o) {
    return resume_dir + "/objects/" + (o.file_name.empty() ? o.name : o.file_name) + ".bin";
}

void writeCmatrixData(const RootGrid& g, int k, const std::string& resume_dir) {
    const ObjectSpec& o = g.input().objects[k];
    const int n = o.n_cmat();
    std::vector<double> C((size_t)n * n);
    const int rc = fopis_get_capacity_matrix(g.context(), g.objectId(k), C.data(), n);
    if (rc != FOPIS_OK) throw Error(rc, fopis_last_error(g.context()));
    DataFile f;
    f.put_f64("capacity_matrix", {(uint64_t)n, (uint64_t)n}, C.data());
    f.put_f64("grid_spacing", g.input().dx);
    f.put_f64("time_spacing", g.input().dt);
    make_dirs(resume_dir + "/objects");
    f.save(cmatrix_file(resume_dir, o));
}

bool loadCmatrixData(RootGrid& g, int k, const std::string& resume_dir) {
    const ObjectSpec& o = g.input().objects[k];
    const std::string file = cmatrix_file(resume_dir, o);
    if (!file_exists(file)) {
        std::cout << "[WARNING] File " << file << " does not exist." << std::endl;
        return false;
    }
    DataFile f;
    try {
        f = DataFile::load(file);
    } catch (const std::runtime_error& e) {
        std::cout << "[WARNING] " << e.what() << std::endl;
        return false;
    }
    if (!f.has("capacity_matrix")) {
        std::cout << "[WARNING] Dataset capacity_matrix does not exist in the file " << file << "." << std::endl;
        return false;
    }
    const int n = o.n_cmat();
    const DataFile::Entry& e = f.get("capacity_matrix");
    const bool valid = e.dims.size() == 2 && e.dims[0] == (uint64_t)n && e.dims[1] == (uint64_t)n &&
                       f.f64_scalar("grid_spacing") == g.input().dx && f.f64_scalar("time_spacing") == g.input().dt;
    if (!valid) return false;
    const std::vector<double> C = f.f64("capacity_matrix");
    const int rc = fopis_set_capacity_matrix(g.context(), g.objectId(k), C.data(), n);
    if (rc != FOPIS_OK) throw Error(rc, fopis_last_error(g.context()));
    return true;
}

}  // namespace io

namespace env {

void saveInfo(const Input& in, int64_t timestep, const std::string& resume_dir) {
    make_dirs(resume_dir);
    DataFile f;
    f.put_f64("dx", in.dx);
    f.put_f64("dt", in.dt);
    f.put_i64("timestep", timestep);
    f.save(resume_dir + "/environment.bin");
}

int64_t loadInfo(const Input& in, const std::string& resume_dir) {
    const std::string file = resume_dir + "/environment.bin";
    if (!file_exists(file))
        throw std::invalid_argument("[ERROR] resume file_name " + file + " does not exist.");
    const DataFile f = DataFile::load(file);
    const double dx = f.f64_scalar("dx"), dt = f.f64_scalar("dt");
    char msg[256];
    if (dx != in.dx) {
        std::snprintf(msg, sizeof msg, "[ERROR] dx %.17g in the resume data does not match the dx %.17g from input.json.",
                      dx, in.dx);
        throw std::invalid_argument(msg);
    }
    if (dt != in.dt) {
        std::snprintf(msg, sizeof msg, "[ERROR] dt %.17g in the resume data does not match the dt %.17g from input.json.",
                      dt, in.dt);
        throw std::invalid_argument(msg);
    }
    return f.i64_scalar("timestep");
}

}  // namespace env

}  // namespace host
}  // namespace fopis
