// Prints the parameters io::load_params reads from an input file, one "key value" per line.
#include <iostream>

#include "io/io.h"

int main(int argc, char** argv) {
    RunParamsHbCB rp;
    try {
        io::load_params(argv[1], rp);
    } catch (const std::exception& e) {
        std::cout << "error " << e.what() << "\n";
        return 3;
    }
    std::cout << "L_core " << rp.L_core << "\nn_core_dims " << rp.n_core_dims << "\ncold_start " << rp.cold_start
              << "\nseed " << rp.seed << "\nN_therm " << rp.N_therm << "\nN_shift " << rp.N_shift << "\nN_switch_eo "
              << rp.N_switch_eo << "\nbeta " << rp.hp.beta << "\nN_sweeps " << rp.hp.N_sweeps << "\nN_hits "
              << rp.hp.N_hits << "\nN_samples " << rp.hp.N_samples << "\nN_shift_plaquette " << rp.N_shift_plaquette
              << "\ntopo " << rp.topo << "\nN_shift_topo " << rp.N_shift_topo << "\nN_steps_gf " << rp.N_steps_gf
              << "\nN_rk_steps " << rp.N_rk_steps << "\nrun_name " << rp.run_name << "\nrun_dir " << rp.run_dir
              << "\nsave_each_shifts " << rp.save_each_shifts << "\nformat " << io::format_double(3.14159, 2) << "\n";
    return 0;
}
