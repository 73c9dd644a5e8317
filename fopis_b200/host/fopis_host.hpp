// fopis_host.hpp — C++ host side of libfopis_gpu.so with the reference's class
// surface: input.json parsing (Initializer::initTDPIC), Normalizer, particle
// types, Particle records, Field access, Spacecraft logs, RootGrid with the ES
// phase methods, and the IO files main.cpp writes. Every method forwards to the
// C ABI (include/fopis_gpu.h); no device code lives here.
#pragma once

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fopis_gpu.h"

namespace fopis {
namespace host {

// Physical constants of include/normalizer.hpp.
constexpr double kE = 1.60217733e-19;
constexpr double kEps0 = 8.854187817e-12;
constexpr double kMu0 = 4.0 * M_PI * 1.0e-7;
constexpr double kClight = 2.99792458e8;
constexpr double kMe = 9.1093818872e-31;

// Normalizer (include/normalizer.hpp): x_unit = dx, t_unit = dt, m_unit = m_e, e_unit = e.
struct Normalizer {
    double x = 1.0, t = 1.0, m = kMe, e = kE;
    double V_unit = 1.0, A_unit = 1.0, eps0 = 1.0, mu0 = 1.0, c = 1.0;
    Normalizer() = default;
    Normalizer(double dx, double dt);
    double velocity(double v) const { return t * v / x; }
    double unvelocity(double v) const { return v * x / t; }
    double bfield(double b) const { return b * (t * e) / m; }
    double current_density(double j) const { return j * (x * x) / A_unit; }
    double potential(double phi) const { return phi / V_unit; }
    double unpotential(double phi) const { return phi * V_unit; }
    double uncharge(double q) const { return q * e; }
    double uncurrent(double i) const { return i * A_unit; }
    double unenergy(double en) const { return en * m * (x * x) / (t * t); }
    double unenergy_ev(double en) const { return en * m * (x * x) / (e * (t * t)); }   // unnormalizeEnergy(en, "eV")
};

// ParticleType / AmbientParticleType / PhotoElectronParticleType (the fields the ES path reads).
struct ParticleType {
    std::string name;
    std::string type;              // "ambient" | "photoelectron" | "secondary"
    double mass = 1.0;             // m_e
    double charge = -1.0;          // e
    double density = 0.0;          // m^-3
    double temperature = 0.0;      // eV
    int particle_per_cell = 1;
    double drift_kms[3] = {0.0, 0.0, 0.0};
    int injection_axis[6] = {1, 1, 1, 1, 1, 1};
    double current_density = 0.0;  // A/m^2 (photoelectrons)
    fopis_species to_abi(const Normalizer& norm, double dx) const;
};

// AmbientParticleType::calcFlux (src/Particle/AmbientParticleType.cpp:8-57).
void calc_flux(double vth, double density_norm, double size, const double drift[3], const int injection_axis[6],
               double flux[6]);

// One conductor as the C ABI takes it (ObjectDataFromFile + Spacecraft::construct).
struct ObjectSpec {
    std::string name;
    std::string file_name;         // the .obj file's name without directories (Spacecraft::file_name)
    std::vector<int32_t> nodes;    // [n_cmat][3] glue-layout
    std::vector<int32_t> cells;    // [n_cells][3] glue-layout
    int is_potential_fixed = 0;
    double fixed_potential = 0.0;  // normalised
    double initial_potential_offset = 0.0;
    int emit_species = -1;
    int secondary_species = -1;    // secondary-electron species the body emits
    int dielectric = 0;            // surface_type "dielectric"
    std::vector<double> capacitance;   // [n_cmat] normalised node capacitance (dielectric)
    int n_cmat() const { return (int)(nodes.size() / 3); }
};

// The normalised content of input.json.
struct Input {
    fopis_params params{};
    Normalizer norm;
    std::vector<ParticleType> species;   // ABI order: ambient, photoelectron, secondary
    std::vector<ObjectSpec> objects;
    int max_timestep = 0;
    double dx = 1.0, dt = 1.0;
    bool use_existing_capacity_matrix = false;
    std::string job_type = "new";        // Environment.job_type: "new" or "load"
    int plot_energy_width = 0;           // IO.plot_energy_width: energy log every this many steps, 0 = never
};

// Initializer::initTDPIC's parsing (src/Initializer/Initialize.cpp:158-421) for
// the ES path on one GPU (proc_x = proc_y = proc_z = 1).
Input load_input(const std::string& path);

// include/particle.hpp: the 56-byte record the reference stores per particle.
struct Particle {
    double x, y, z, vx, vy, vz;
    int32_t typeId;
    int32_t isValid;
};
static_assert(sizeof(Particle) == 56, "Particle record is 56 bytes");

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
    int code() const { return code_; }
private:
    int code_;
};

// Spacecraft's logged state (Spacecraft::getLogHeader / getLogEntry, Spacecraft.cpp:978-1044).
struct Spacecraft {
    std::string name;
    int id = 0;
    double potential = 0.0;               // normalised
    double total_charge = 0.0;
    std::vector<double> current;          // per species, normalised
    std::string getLogHeader(const std::vector<ParticleType>& species) const;
    std::string getLogEntry(const Normalizer& norm) const;
};

class RootGrid {
public:
    explicit RootGrid(const Input& in, int device = 0);
    ~RootGrid();
    RootGrid(const RootGrid&) = delete;
    RootGrid& operator=(const RootGrid&) = delete;

    void* context() const { return ctx_; }
    const Input& input() const { return in_; }
    int objectId(int k) const { return object_ids_[k]; }

    // RootGrid::initializeObjectsCmatrix (RootGridObject.cpp:77-148): with
    // Options::use_existing_capacity_matrix the matrix is read from
    // <resume_dir>/objects/<file_name> (io::loadCmatrixData) when it fits,
    // otherwise built and written there (io::writeCmatrixData).
    void initializeObjectsCmatrix(const std::string& resume_dir = "");
    // RootGrid::saveResumeData / loadResumeData (RootGridIO.cpp:25-50): the
    // particles of every species, phi and E, and each object's charge map in
    // <resume_dir>/grid_id_0.bin; Grid::initializeForLoad (Grid.cpp:38-50)
    // rebuilds rho and the conductor state from them.
    void saveResumeData(const std::string& resume_dir) const;
    void loadResumeData(const std::string& resume_dir);
    void initializeForLoad();
    int64_t timestep() const { return stats().timestep; }   // Environment::timestep of the next step
    void setTimestep(int64_t t);
    void generateAmbientParticles();                 // Initializer's ambient loading
    void loadParticles(int species, const std::vector<Particle>& p);
    void initialize();                               // Grid::initialize (Grid.cpp:23-36)
    void mainLoop();                                 // RootGrid::mainLoopES (RootGrid.cpp:82-143)
    void setGuessMode(int mode);

    // the phases of mainLoopES, in the reference's order
    void updateParticleVelocity();
    void emitParticlesFromObjects();
    void updateParticlePosition();
    void injectParticlesFromBoundary();
    void updateRho();
    void solvePoisson();
    void updateEfield();
    void advanceTimestep();

    double getParticleEnergy() const;                // Grid::getParticleEnergy
    double getEFieldEnergy() const;                  // Field::getEfieldEnergy
    double getBFieldEnergy() const;                  // Field::getBfieldEnergy (0 in the ES mode)
    void updateBfield();                             // RootGrid::updateBfield (EM mode)
    std::vector<int64_t> getValidParticleNumbers() const;
    std::vector<Particle> getParticles(int species) const;
    std::vector<double> getField(int which) const;   // fopis_field, glue layout (nx+2)(ny+2)(nz+2)
    std::vector<double> getPhi() const { return getField(FOPIS_FIELD_PHI); }
    std::vector<double> getRho() const { return getField(FOPIS_FIELD_RHO0); }
    std::vector<Spacecraft> getObjects() const;
    fopis_stats stats() const;

private:
    void check(int rc, bool allow_not_converged = false) const;
    Input in_;
    void* ctx_ = nullptr;
    std::vector<int> object_ids_;
};

// IO::plotEnergy / plotObjectsData / plotValidParticleNumber (src/Misc/IO.cpp:150-300):
// files data/energy.txt, data/object_<name>.txt, data/total_particle_number.txt.
namespace io {
// IO::writeCmatrixData / loadCmatrixData (src/Misc/IO.cpp:28-120): datasets
// capacity_matrix [n][n], grid_spacing, time_spacing. A file is valid when the
// matrix size and dx, dt match (IO.cpp:88-90); loadCmatrixData then sets the
// object's matrix and returns true.
std::string cmatrix_file(const std::string& resume_dir, const ObjectSpec& o);
void writeCmatrixData(const RootGrid& g, int object, const std::string& resume_dir);
bool loadCmatrixData(RootGrid& g, int object, const std::string& resume_dir);
void plot_energy(const RootGrid& g, int timestep, const std::string& dir);
void plot_objects(const RootGrid& g, int timestep, const std::string& dir);
void plot_particle_numbers(const RootGrid& g, int timestep, const std::string& dir);
}  // namespace io

// Environment::saveInfo / loadInfo (src/Misc/Environment.cpp:379-438):
// <resume_dir>/environment.bin holds dx, dt and the timestep of the next step;
// loadInfo rejects a file whose dx or dt differs from input.json's
// (std::invalid_argument, as the reference) and returns the timestep.
namespace env {
void saveInfo(const Input& in, int64_t timestep, const std::string& resume_dir);
int64_t loadInfo(const Input& in, const std::string& resume_dir);
}  // namespace env

}  // namespace host
}  // namespace fopis
