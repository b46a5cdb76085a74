// gauge_hb_cb -- heatbath run driver on one GPU, with the behaviour of the reference's driver
// (src/bin/gauge_hb_cb.cpp:20-284):
//   * input: the reference's `key = value` file (inputs/h*.txt run unchanged);
//   * lattice: (L_core * n_core_dims)^4, periodic, on one GPU; the global shift draws s_d from
//     [0, L_core - 1] with the run's std::mt19937_64 as the reference does;
//   * schedule: N_therm thermalisation shifts (skipped on resume) then N_shift shifts, each a random
//     global shift followed by N_switch_eo x N_sweeps full checkerboard sweeps (the reference's
//     even-core / odd-core phases update every link once per switch);
//   * outputs: <run>_plaquette.txt, <run>_topo.txt ("t Q E"), <run>_params.txt, the ILDG
//     configuration and the resume state, every save_each_shifts shifts and at the end.
#include <chrono>
#include <iomanip>
#include <iostream>
#include <random>
#include <vector>

#include "../flow/gradient_flow.h"
#include "../gauge/GaugeField.h"
#include "../heatbath/heatbath_mpi.h"
#include "../io/ildg.h"
#include "../io/io.h"
#include "../mpi/HalosShift.h"
#include "../mpi/Shift.h"
#include "../observables/observables_mpi.h"

namespace {

void update_block(GaugeField& field, const GeometryCB& geo, mpi::MpiTopology& topo, const RunParamsHbCB& rp,
                  std::vector<std::mt19937_64>& rng, const char* tag, int i) {
    for (int j = 0; j < rp.N_switch_eo; j++) {
        if (topo.rank == 0) std::cout << tag << "Shift : " << i << ", Switch : " << j << ", Parity : Even\n";
        mpi::heatbathcb::samples(field, geo, topo, rp.hp, rng, even);
        if (topo.rank == 0) std::cout << tag << "Shift : " << i << ", Switch : " << j << ", Parity : Odd\n";
        mpi::heatbathcb::samples(field, geo, topo, rp.hp, rng, odd);
    }
}

void save_all(const RunParamsHbCB& rp, GaugeField& field, const GeometryCB& geo, mpi::MpiTopology& topo,
              std::vector<std::mt19937_64>& rng, std::vector<double>& plaq, std::vector<double>& tqe, int shift,
              bool final_state) {
    const int precision = 10;
    if (topo.rank == 0) {
        std::cout << "\n\n==========================================\n";
        io::save_plaquette(plaq, rp.run_name, rp.run_dir, precision);
        if (rp.topo) io::save_topo(tqe, rp.run_name, rp.run_dir, precision);
        io::add_shift(shift, rp.run_name, rp.run_dir);
        if (final_state) io::add_finished(rp.run_name, rp.run_dir);
    }
    io::save_seed(rng, rp.run_name, rp.run_dir, topo);
    io::save_hb_state(field, rp.run_name, rp.run_dir);
    save_ildg_clime(rp.run_name, rp.run_dir, field, geo, topo);
    if (topo.rank == 0) std::cout << "==========================================\n";
    plaq.clear();
    tqe.clear();
}

void generate_hb_cb(const RunParamsHbCB& rp, bool existing) {
    mpi::MpiTopology topo(rp.n_core_dims);
    GeometryCB geo(rp.L_core * rp.n_core_dims);
    GaugeField field(geo);
    mpi::shift::set_shift_range(rp.L_core);
    std::vector<std::mt19937_64> rng(1);
    rng[0].seed(rp.seed + topo.rank * 1000);
    if (!rp.cold_start) field.hot_start(geo, rng[0]);
    if (existing) {
        read_ildg_clime(rp.run_name, rp.run_dir, field, geo, topo);
        io::load_seed(rng, rp.run_name, rp.run_dir, topo);
        io::load_hb_state(field, rp.run_name, rp.run_dir);
    }
    HalosShift halo_shift(geo);
    GradientFlow flow(0.02, field, geo);
    std::vector<double> plaq, tqe;
    if (topo.rank == 0) io::save_params(rp, rp.run_name, rp.run_dir);
    print_parameters(rp, topo);

    if (!existing) {
        if (topo.rank == 0)
            std::cout << "\n\n===========================================\nThermalisation : " << rp.N_therm
                      << " shifts\n===========================================\n";
        for (int i = 0; i < rp.N_therm; i++) {
            if (topo.rank == 0) std::cout << "\n\n==========(Therm) Shift " << i << "==========\n";
            mpi::shift::random_shift(field, geo, halo_shift, topo, rng[0]);
            update_block(field, geo, topo, rp, rng, "(Therm) ", i);
            if (i % rp.N_shift_plaquette == 0) {
                const double p = mpi::observables::mean_plaquette_global(field, geo, topo);
                if (topo.rank == 0)
                    std::cout << "====== Plaquette ======\n(Therm) Sample " << i / rp.N_shift_plaquette
                              << ", <P> = " << p << "\n";
            }
        }
    }
    if (topo.rank == 0)
        std::cout << "\n\n===========================================\nSampling : " << rp.N_shift / rp.N_shift_plaquette
                  << " <P> samples, " << rp.N_shift / rp.N_shift_topo
                  << " Q samples\n===========================================\n";
    for (int i = 0; i < rp.N_shift; i++) {
        if (topo.rank == 0) std::cout << "\n\n=============Shift " << i << "=============\n";
        mpi::shift::random_shift(field, geo, halo_shift, topo, rng[0]);
        update_block(field, geo, topo, rp, rng, "", i);
        if (i % rp.N_shift_plaquette == 0 && (i > 0 || !existing)) {
            const double p = mpi::observables::mean_plaquette_global(field, geo, topo);
            if (topo.rank == 0)
                std::cout << "====== Plaquette ======\nSample " << i / rp.N_shift_plaquette << ", <P> = " << p << "\n";
            plaq.push_back(p);
        }
        if (rp.topo && i % rp.N_shift_topo == 0 && (i > 0 || !existing)) {
            if (topo.rank == 0) std::cout << "====== Topology ======\n";
            std::vector<double> cur =
                mpi::observables::topo_charge_flowed(field, geo, flow, topo, rp.N_steps_gf, rp.N_rk_steps);
            if (topo.rank == 0)
                std::cout << "Sample " << i / rp.N_shift_topo << ", final Q = " << cur[cur.size() - 2] << "\n";
            tqe.insert(tqe.end(), cur.begin(), cur.end());
        }
        if (i > 0 && i % rp.save_each_shifts == 0) save_all(rp, field, geo, topo, rng, plaq, tqe, i, false);
    }
    save_all(rp, field, geo, topo, rng, plaq, tqe, rp.N_shift, true);
}

}  // namespace

int main(int argc, char* argv[]) {
    if (argc < 2) {
        std::cerr << "Usage: " << argv[0] << " <input_file.txt>" << std::endl;
        return 1;
    }
    RunParamsHbCB params;
    bool existing = false;
    try {
        existing = io::read_params(params, 0, argv[1]);
    } catch (const std::exception& e) {
        std::cerr << "Error reading input : " << e.what() << std::endl;
        return 1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    try {
        generate_hb_cb(params, existing);
    } catch (const std::exception& e) {
        std::cerr << "Fatal: " << e.what() << std::endl;
        return 2;
    }
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << std::fixed << std::setprecision(4);
    print_time((long)total);
    return 0;
}
