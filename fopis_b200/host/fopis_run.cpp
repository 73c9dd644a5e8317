// fopis_run — the reference's main loop (src/main.cpp:16-72) on the GPU
// library: read input.json, set up the conductors (capacity matrix built, or
// read from <resume>/objects with Options.use_existing_capacity_matrix), then
// for job_type "new" load the ambient plasma and initialize, for "load" read
// <resume>/environment.bin and grid_id_0.bin and Grid::initializeForLoad
// (Initialize.cpp:75-99); per step RootGrid::mainLoop and the energy / object /
// particle-number logs (the energy log every IO.plot_energy_width steps, never
// when it is 0 or absent); at the end Environment::saveInfo and
// RootGrid::saveResumeData into <resume>.
//
//   fopis_run [input.json] [--steps N] [--out DIR] [--resume DIR] [--device D]
//             [--guess warm|history] [--dump-params FILE]
//
// --steps N runs N steps (default: up to max_timestep, as the reference's
// loop); --resume defaults to "resume". --dump-params writes the normalised
// parameters and object node lists that input.json produces (no GPU work) and
// exits.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>

#include "datafile.hpp"
#include "fopis_host.hpp"

using namespace fopis::host;

namespace {
void dump_params(const Input& in, const std::string& file) {
    std::ofstream f(file, std::ios::binary);
    f.write(reinterpret_cast<const char*>(&in.params), sizeof in.params);
    const int32_t nobj = (int32_t)in.objects.size();
    f.write(reinterpret_cast<const char*>(&nobj), sizeof nobj);
    for (const auto& o : in.objects) {
        const int32_t meta[4] = {(int32_t)(o.nodes.size() / 3), (int32_t)(o.cells.size() / 3), o.is_potential_fixed,
                                 o.emit_species};
        f.write(reinterpret_cast<const char*>(meta), sizeof meta);
        const double pot[2] = {o.fixed_potential, o.initial_potential_offset};
        f.write(reinterpret_cast<const char*>(pot), sizeof pot);
        f.write(reinterpret_cast<const char*>(o.nodes.data()), sizeof(int32_t) * o.nodes.size());
        f.write(reinterpret_cast<const char*>(o.cells.data()), sizeof(int32_t) * o.cells.size());
        const int32_t extra[2] = {o.secondary_species, o.dielectric};
        f.write(reinterpret_cast<const char*>(extra), sizeof extra);
        if (o.dielectric)
            f.write(reinterpret_cast<const char*>(o.capacitance.data()), sizeof(double) * o.capacitance.size());
    }
    const int32_t io[1] = {in.plot_energy_width};
    f.write(reinterpret_cast<const char*>(io), sizeof io);
}
}  // namespace

int main(int argc, char** argv) {
    std::string input = "input.json", out = "data", dump, resume = "resume";
    int steps = -1, device = 0, guess = FOPIS_GUESS_WARM;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) { std::fprintf(stderr, "%s needs a value\n", a.c_str()); std::exit(2); }
            return argv[++i];
        };
        if (a == "--steps") steps = std::stoi(next());
        else if (a == "--out") out = next();
        else if (a == "--resume") resume = next();
        else if (a == "--device") device = std::stoi(next());
        else if (a == "--dump-params") dump = next();
        else if (a == "--datafile-echo") {
            // reads a data file and writes its datasets to another (no GPU work): a
            // check of the file format against other writers and readers
            const std::string src = next(), dst = next();
            try {
                fopis::host::DataFile::load(src).save(dst);
            } catch (const std::exception& e) {
                std::fprintf(stderr, "fopis_run: %s\n", e.what());
                return 1;
            }
            return 0;
        }
        else if (a == "--guess") {
            const std::string g = next();
            guess = g == "history" ? FOPIS_GUESS_HISTORY : FOPIS_GUESS_WARM;
        } else input = a;
    }
    try {
        const Input in = load_input(input);
        if (!dump.empty()) {
            dump_params(in, dump);
            return 0;
        }
        RootGrid grid(in, device);
        grid.setGuessMode(guess);
        grid.initializeObjectsCmatrix(resume);
        int64_t first = 1;
        if (in.job_type == "load") {
            first = env::loadInfo(in, resume);
            std::cout << "--  Resume Data (t = " << first << ") Loading --" << std::endl;
            grid.setTimestep(first);
            grid.loadResumeData(resume);
            grid.initializeForLoad();
        } else {
            grid.generateAmbientParticles();
            grid.initialize();
        }
        const int64_t last = steps >= 0 ? first + steps - 1 : (int64_t)in.max_timestep;
        std::cout << "===== Begin Main Loop =====" << std::endl;
        for (int64_t t = first; t <= last; ++t) {
            grid.mainLoop();
            // Environment::plotEnergy (include/environment.hpp:242, :266-278)
            if (in.plot_energy_width != 0 && t % in.plot_energy_width == 0) io::plot_energy(grid, (int)t, out);
            io::plot_objects(grid, (int)t, out);
            io::plot_particle_numbers(grid, (int)t, out);
        }
        env::saveInfo(in, grid.timestep(), resume);
        grid.saveResumeData(resume);
        const fopis_stats st = grid.stats();
        std::cout << "===== End Main Loop ===== steps " << (last - first + 1) << ", V-cycles in the last step "
                  << st.vcycles_step << std::endl;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "fopis_run: %s\n", e.what());
        return 1;
    }
    return 0;
}
