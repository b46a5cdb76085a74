// io/io.h -- heatbath-driver input file, text outputs and resume files, with the reference's key
// names, file names and formats (src/io/io.h; src/io/io.cpp:22-136, 139-218, 312-367, 434-481,
// 484-526, 537-634, 838-885).  No MPI: one process drives one GPU.
#pragma once
#include <cstdint>
#include <random>
#include <string>
#include <vector>

#include "../gauge/GaugeField.h"
#include "../mpi/MpiTopology.h"
#include "params.h"

namespace io {
// ---- input: `key = value` lines, '#' starts a comment line, keys and values trimmed
std::string trim(const std::string& s);
void load_params(const std::string& filename, RunParamsHbCB& rp);  // throws std::runtime_error if unreadable
// Loads the parameters and reports whether the run can resume: the ILDG configuration
// run_dir/run_name/run_name, its RNG state files and the heatbath state file all exist.
bool read_params(RunParamsHbCB& params, int rank, const std::string& input);

// ---- outputs (appended)
void save_plaquette(const std::vector<double>& data, const std::string& filename, const std::string& dirpath,
                    int precision);
void save_topo(const std::vector<double>& tQE, const std::string& filename, const std::string& dirpath,
               int precision);
void save_params(const RunParamsHbCB& rp, const std::string& filename, const std::string& dirpath);
void add_shift(int shift, const std::string& filename, const std::string& dirpath);
void add_finished(const std::string& filename, const std::string& dirpath);

// ---- resume state
// std::mt19937_64 states (used for the global shifts and the hot-start key), one file per engine:
// run_dir/run_name/run_name_seed/run_name_seed_r<rank>_t<i>.txt
void save_seed(std::vector<std::mt19937_64>& rng, const std::string& filename, const std::string& dirpath,
               mpi::MpiTopology& topo);
bool load_seed(std::vector<std::mt19937_64>& rng, const std::string& filename, const std::string& dirpath,
               mpi::MpiTopology& topo);
// The heatbath's counter-based stream state (Philox key, next sweep index):
// run_dir/run_name/run_name_seed/run_name_hb_state.txt
void save_hb_state(const GaugeField& field, const std::string& filename, const std::string& dirpath);
bool load_hb_state(GaugeField& field, const std::string& filename, const std::string& dirpath);

std::string format_double(double val, int precision);
}  // namespace io

void print_parameters(const RunParamsHbCB& rp, const mpi::MpiTopology& topo);
void print_time(long elapsed);
