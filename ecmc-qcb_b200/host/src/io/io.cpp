// io/io.cpp -- heatbath-driver text I/O (see io.h).
#include "io.h"

#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>

namespace fs = std::filesystem;

namespace {
// Opens run_dir/run_name/<run_name + suffix> for appending, creating the directories.
bool open_append(std::ofstream& f, const std::string& filename, const std::string& dirpath, const std::string& suffix,
                 fs::path* where) {
    fs::path dir = fs::path(dirpath) / filename;
    std::error_code ec;
    fs::create_directories(dir, ec);
    if (ec) {
        std::cerr << "Couldn't create folder data : " << ec.message() << std::endl;
        return false;
    }
    *where = dir / (filename + suffix);
    f.open(*where, std::ios::out | std::ios::app);
    if (!f.is_open()) {
        std::cout << "Could not open file " << *where << "\n";
        return false;
    }
    return true;
}

fs::path seed_dir(const std::string& filename, const std::string& dirpath) {
    return fs::path(dirpath) / filename / (filename + "_seed");
}
}  // namespace

std::string io::trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

// Keys and semantics of load_params (src/io/io.cpp:434-481): booleans are true only for the
// literal "true"; N_samples is forced to 1.
void io::load_params(const std::string& filename, RunParamsHbCB& rp) {
    std::ifstream in(filename);
    if (!in.is_open()) throw std::runtime_error("Can't open file " + filename);
    std::map<std::string, std::string> kv;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string value = line.substr(eq + 1);
        if (value.empty()) continue;  // "key =" with nothing after it sets nothing
        kv[trim(line.substr(0, eq))] = trim(value);
    }
    auto geti = [&](const char* k, int& v) {
        if (kv.count(k)) v = std::stoi(kv[k]);
    };
    auto getd = [&](const char* k, double& v) {
        if (kv.count(k)) v = std::stod(kv[k]);
    };
    auto getb = [&](const char* k, bool& v) {
        if (kv.count(k)) v = (kv[k] == "true");
    };
    geti("L_core", rp.L_core);
    geti("n_core_dims", rp.n_core_dims);
    getb("cold_start", rp.cold_start);
    geti("seed", rp.seed);
    geti("N_switch_eo", rp.N_switch_eo);
    geti("N_shift", rp.N_shift);
    getd("beta", rp.hp.beta);
    rp.hp.N_samples = 1;
    geti("N_sweeps", rp.hp.N_sweeps);
    geti("N_hits", rp.hp.N_hits);
    geti("N_shift_plaquette", rp.N_shift_plaquette);
    geti("N_shift_therm", rp.N_therm);
    getb("topo", rp.topo);
    geti("N_shift_topo", rp.N_shift_topo);
    geti("N_steps_gf", rp.N_steps_gf);
    geti("N_rk_steps", rp.N_rk_steps);
    if (kv.count("run_name")) rp.run_name = kv["run_name"];
    if (kv.count("run_dir")) rp.run_dir = kv["run_dir"];
    geti("save_each_shifts", rp.save_each_shifts);
}

bool io::read_params(RunParamsHbCB& params, int rank, const std::string& input) {
    io::load_params(input, params);
    const fs::path base = fs::path(params.run_dir) / params.run_name;
    const fs::path sd = seed_dir(params.run_name, params.run_dir);
    bool existing = fs::exists(base / params.run_name) &&
                    fs::exists(sd / (params.run_name + "_seed_r" + std::to_string(rank) + "_t0.txt")) &&
                    fs::exists(sd / (params.run_name + "_hb_state.txt"));
    if (existing && rank == 0) std::cout << "All ranks found existing configuration. Resuming...\n";
    return existing;
}

void io::save_plaquette(const std::vector<double>& data, const std::string& filename, const std::string& dirpath,
                        int precision) {
    std::ofstream f;
    fs::path p;
    if (!open_append(f, filename, dirpath, "_plaquette.txt", &p)) return;
    f << std::fixed << std::setprecision(precision);
    for (double x : data) f << x << "\n";
    std::cout << "Plaquette written in " << p << "\n";
}

void io::save_topo(const std::vector<double>& tQE, const std::string& filename, const std::string& dirpath,
                   int precision) {
    std::ofstream f;
    fs::path p;
    if (!open_append(f, filename, dirpath, "_topo.txt", &p)) return;
    f << std::fixed << std::setprecision(precision);
    for (size_t i = 0; i + 2 < tQE.size(); i += 3) f << tQE[i] << " " << tQE[i + 1] << " " << tQE[i + 2] << "\n";
    std::cout << "Topology written in " << p << "\n";
}

void io::save_params(const RunParamsHbCB& rp, const std::string& filename, const std::string& dirpath) {
    std::ofstream f;
    fs::path p;
    if (!open_append(f, filename, dirpath, "_params.txt", &p)) return;
    f << std::boolalpha << "\n#########################################################\n\n"
      << "# Lattice params\nL_core=" << rp.L_core << "\nn_core_dims=" << rp.n_core_dims
      << "\ncold_start=" << rp.cold_start << "\n\n"
      << "# Run params\nseed=" << rp.seed << "\nN_shift_therm = " << rp.N_therm << "\nN_shift =" << rp.N_shift
      << "\nN_switch_eo=" << rp.N_switch_eo << "\n\n"
      << "# Heatbath params\nbeta = " << rp.hp.beta << "\nN_sweeps = " << rp.hp.N_sweeps
      << "\nN_hits = " << rp.hp.N_hits << "\n\n"
      << "# Plaquette params\nN_shift_plaquette = " << rp.N_shift_plaquette << "\n\n"
      << "# Topo params\ntopo = " << rp.topo << "\nN_shift_topo = " << rp.N_shift_topo
      << "\nN_steps_gf = " << rp.N_steps_gf << "\nN_rk_steps = " << rp.N_rk_steps << "\n\n"
      << "#Save params\nsave_each_shifts = " << rp.save_each_shifts << "\n\n";
    std::cout << "Parameters saved in " << p << "\n";
}

void io::add_shift(int shift, const std::string& filename, const std::string& dirpath) {
    std::ofstream f;
    fs::path p;
    if (open_append(f, filename, dirpath, "_params.txt", &p)) f << "Saved shift " << shift << "\n";
}

void io::add_finished(const std::string& filename, const std::string& dirpath) {
    std::ofstream f;
    fs::path p;
    if (open_append(f, filename, dirpath, "_params.txt", &p)) f << "Saved final state !\n";
}

void io::save_seed(std::vector<std::mt19937_64>& rng, const std::string& filename, const std::string& dirpath,
                   mpi::MpiTopology& topo) {
    const fs::path dir = seed_dir(filename, dirpath);
    std::error_code ec;
    fs::create_directories(dir, ec);
    for (size_t t = 0; t < rng.size(); t++) {
        std::ofstream f(dir / (filename + "_seed_r" + std::to_string(topo.rank) + "_t" + std::to_string(t) + ".txt"));
        if (f.is_open()) f << rng[t];
    }
    if (topo.rank == 0) std::cout << "All threads seeds (" << rng.size() << ") saved in " << dir << "\n";
}

bool io::load_seed(std::vector<std::mt19937_64>& rng, const std::string& filename, const std::string& dirpath,
                   mpi::MpiTopology& topo) {
    const fs::path dir = seed_dir(filename, dirpath);
    bool all = true;
    for (size_t t = 0; t < rng.size(); t++) {
        std::ifstream f(dir / (filename + "_seed_r" + std::to_string(topo.rank) + "_t" + std::to_string(t) + ".txt"));
        if (f.is_open())
            f >> rng[t];
        else {
            all = false;
            std::cerr << "Rank " << topo.rank << " thread " << t << ": Seed file missing, using initial seed."
                      << std::endl;
        }
    }
    return all;
}

void io::save_hb_state(const GaugeField& field, const std::string& filename, const std::string& dirpath) {
    const fs::path dir = seed_dir(filename, dirpath);
    std::error_code ec;
    fs::create_directories(dir, ec);
    std::ofstream f(dir / (filename + "_hb_state.txt"));
    f << "philox_key " << field.hb_seed << "\nnext_sweep " << field.hb_sweep << "\nseeded " << (field.hb_seeded ? 1 : 0)
      << "\n";
}

bool io::load_hb_state(GaugeField& field, const std::string& filename, const std::string& dirpath) {
    std::ifstream f(seed_dir(filename, dirpath) / (filename + "_hb_state.txt"));
    if (!f.is_open()) return false;
    std::string k1, k2, k3;
    int seeded = 0;
    f >> k1 >> field.hb_seed >> k2 >> field.hb_sweep >> k3 >> seeded;
    field.hb_seeded = seeded != 0;
    return (bool)f;
}

std::string io::format_double(double val, int precision) {
    std::stringstream ss;
    ss << std::fixed << std::setprecision(precision) << val;
    return ss.str();
}

void print_parameters(const RunParamsHbCB& rp, const mpi::MpiTopology& topo) {
    if (topo.rank != 0) return;
    std::cout << "==========================================\nHeatbath - Checkboard\n"
              << "==========================================\nRun name : " << rp.run_name << "\n"
              << "---Lattice params---\nTotal lattice size : " << rp.L_core * rp.n_core_dims << "^4\n"
              << "Local lattice size : " << rp.L_core << "^4\n\n"
              << "---Run params---\nInitial seed : " << rp.seed << "\nThermalization shifts : " << rp.N_therm
              << "\nNumber of shifts : " << rp.N_shift << "\nNumber of e/o switchs per shift : " << rp.N_switch_eo
              << "\nSave each : " << rp.save_each_shifts << " shifts\n\n"
              << "---Heatbath params---\nBeta : " << rp.hp.beta << "\nNumber of sweeps : " << rp.hp.N_sweeps
              << "\nNumber of hits : " << rp.hp.N_hits << "\n\n"
              << "---Measures params---\nNumber of <P> samples : " << rp.N_shift / rp.N_shift_plaquette
              << "\nMeasure <P> each : " << rp.N_shift_plaquette << " shifts\nMeasure topo : "
              << (rp.topo ? "Yes" : "No") << "\n";
    if (rp.topo)
        std::cout << "Number of Q samples : " << rp.N_shift / rp.N_shift_topo << "\nMeasure Q each : " << rp.N_shift_topo
                  << " shifts\n\n---Gradient Flow---\nNumber of RK3 steps per GF step : " << rp.N_rk_steps
                  << "\nNumber of GF steps : " << rp.N_steps_gf << "\n";
    std::cout << "==========================================" << std::endl;
}

// The reference passes a double to print_time(long), which truncates to whole seconds
// (src/io/io.cpp:522-526, src/bin/gauge_hb_cb.cpp:280); kept.
void print_time(long elapsed) {
    std::cout << "==========================================\nElapsed time : " << elapsed
              << "s\n==========================================" << std::endl;
}
