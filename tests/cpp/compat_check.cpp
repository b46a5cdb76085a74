// Uses the C++ layer the way the reference's drivers use their own classes and prints what the
// Python test compares with the oracle.  argv[1]: scratch directory.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <vector>

#include "flow/gradient_flow.h"
#include "gauge/GaugeField.h"
#include "heatbath/heatbath_mpi.h"
#include "io/ildg.h"
#include "mpi/Shift.h"
#include "observables/observables_mpi.h"

static void dump(const GaugeField& f, const GeometryCB& geo, const std::string& path) {
    std::ofstream out(path, std::ios::binary);
    for (int t = 1; t <= geo.L_int; t++)
        for (int z = 1; z <= geo.L_int; z++)
            for (int y = 1; y <= geo.L_int; y++)
                for (int x = 1; x <= geo.L_int; x++)
                    for (int mu = 0; mu < 4; mu++) {
                        SU3 u = f.view_link_const(geo.index(x, y, z, t), mu);
                        out.write(reinterpret_cast<const char*>(u.m), sizeof(u.m));
                    }
}

int main(int argc, char** argv) {
    const std::string dir = argv[1];
    std::cout << std::setprecision(17);
    mpi::MpiTopology topo(1);
    GeometryCB geo(4);
    GaugeField field(geo);
    std::mt19937_64 rng(2024);
    std::cout << "hot_key " << std::mt19937_64(2024)() << "\n";
    field.hot_start(geo, rng);
    std::cout << "plaq_hot " << mpi::observables::mean_plaquette_global(field, geo, topo) << "\n";
    // the halo is a periodic copy of the opposite face
    SU3 a = field.view_link_const(geo.index(0, 2, 3, 1), 2), b = field.view_link_const(geo.index(4, 2, 3, 1), 2);
    double hd = 0;
    for (int k = 0; k < 9; k++) hd += std::abs(a.m[k] - b.m[k]);
    std::cout << "halo_diff " << hd << "\n";
    SU3 st;
    field.compute_staple(geo, geo.index(1, 1, 1, 1), 1, st);
    std::cout << "staple00 " << st(0, 0).real() << " " << st(0, 0).imag() << "\n";
    dump(field, geo, dir + "/hot.bin");

    std::vector<std::mt19937_64> rngs(1, std::mt19937_64(7));
    std::cout << "hb_key " << std::mt19937_64(7)() << "\n";
    HbParams hp;
    hp.N_samples = 1;
    hp.N_sweeps = 2;
    hp.N_hits = 1;
    hp.beta = 6.0;
    mpi::heatbathcb::samples(field, geo, topo, hp, rngs, even);  // 2 x (sweep EV; sweep OD)
    mpi::heatbathcb::samples(field, geo, topo, hp, rngs, odd);   // single rank has parity even: no update
    std::cout << "hb_sweep " << field.hb_sweep << "\n";
    std::cout << "plaq_hb " << mpi::observables::mean_plaquette_global(field, geo, topo) << "\n";
    dump(field, geo, dir + "/hb.bin");

    GradientFlow gf(0.02, field, geo);
    std::vector<double> tqe = mpi::observables::topo_charge_flowed(field, geo, gf, topo, 3, 2);
    std::cout << "tqe";
    for (double v : tqe) std::cout << " " << v;
    std::cout << "\n";

    save_ildg_clime("cc", dir, field, geo, topo);
    GaugeField g2(geo);
    read_ildg_clime("cc", dir, g2, geo, topo);
    double d = 0;
    for (int s = 0; s < (int)geo.V_ext; s++)
        for (int mu = 0; mu < 4; mu++) {
            SU3 u = field.view_link_const(s, mu), v = g2.view_link_const(s, mu);
            for (int k = 0; k < 9; k++) d += std::abs(u.m[k] - v.m[k]);
        }
    std::cout << "ildg_diff " << d << "\n";

    // host edit through view_link reaches the device on the next hot-path call
    field.view_link(geo.index(1, 1, 1, 1), 0) = SU3::Identity();
    field.projection_su3(geo.index(2, 1, 1, 1), 3);
    std::cout << "plaq_edit " << mpi::observables::mean_plaquette_global(field, geo, topo) << "\n";
    dump(field, geo, dir + "/edit.bin");

    HalosShift hs(geo);
    int s[4] = {1, 2, 0, 3};
    mpi::shift::shift_field(field, geo, hs, topo, s);
    dump(field, geo, dir + "/shift.bin");

    // one hit of link ((2,1,1,1), mu = 1) -- interior site (1,0,0,0), lexicographic index 1 -- with
    // the reference's signature; its staple comes back in A
    std::mt19937_64 hit_rng(11);
    std::cout << "hit_key " << std::mt19937_64(11)() << "\n";
    SU3 A;
    mpi::heatbathcb::hit(field, geo, geo.index(2, 1, 1, 1), 1, 6.0, A, hit_rng);
    std::cout << "hit_staple";
    for (int k = 0; k < 9; k++) std::cout << " " << A.m[k].real() << " " << A.m[k].imag();
    std::cout << "\n";
    dump(field, geo, dir + "/hit.bin");

    // the reference's separate flow members in rk3_step's order equal one rk3_step
    GradientFlow gm(0.02, field, geo), gr(0.02, field, geo);
    gm.compute_force(0);
    gm.compute_w1();
    gm.compute_force(1);
    gm.compute_w2();
    gm.replace_force_0();
    gm.compute_force(1);
    gm.compute_w3();
    gr.rk3_step(topo);
    double fd = 0;
    for (int sx = 0; sx < (int)geo.V_ext; sx++)
        for (int mu = 0; mu < 4; mu++) {
            SU3 u = gm.field_c.view_link_const(sx, mu), v = gr.field_c.view_link_const(sx, mu);
            for (int k = 0; k < 9; k++) fd = std::max(fd, std::abs(u.m[k] - v.m[k]));
        }
    std::cout << "members_vs_rk3 " << fd << "\n";
    SU3 F = mpi::observables::clover_site(field, geo, geo.index(2, 1, 1, 1), 0, 2);
    auto qe = mpi::observables::local_q_e_clover(field, geo, geo.index(2, 1, 1, 1));
    std::cout << "clover_site";
    for (int k = 0; k < 9; k++) std::cout << " " << F.m[k].real() << " " << F.m[k].imag();
    std::cout << "\nlocal_qe " << qe.first << " " << qe.second << "\n";
    std::cout << "levi " << mpi::observables::levi_civita(0, 1, 2, 3) << " " << mpi::observables::levi_civita(1, 0, 2, 3)
              << " " << mpi::observables::levi_civita(0, 0, 2, 3) << "\n";
    return 0;
}
