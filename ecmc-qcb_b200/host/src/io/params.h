// io/params.h -- run parameters of the heatbath driver, with the reference's fields and defaults
// (src/io/params.h:30-63).
#pragma once
#include <string>

struct HbParams {
    double beta = 6.0;
    int N_samples = 10;
    int N_hits = 1;
    int N_sweeps = 1;
    int N_therm = 100;
};

struct RunParamsHbCB {
    int L_core = 6;
    int n_core_dims = 2;
    bool cold_start = true;
    int N_switch_eo = 3;
    int N_shift = 2;
    int seed = 123;
    HbParams hp{};
    int N_therm = 100;
    bool topo = true;
    int N_shift_plaquette = 2;
    int N_shift_topo = 10;
    int N_steps_gf = 10;
    int N_rk_steps = 40;
    std::string run_name = "c";
    std::string run_dir = "data";
    int save_each_shifts = 2;
};
