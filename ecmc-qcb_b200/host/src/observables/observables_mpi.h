// observables/observables_mpi.h -- plaquette and clover observables (reference
// src/observables/observables_mpi.h:8-19) on the GPU.  On one rank, "local" and "global" agree
// up to the reference's normalisations, which are kept.
#pragma once
#include <utility>
#include <vector>

#include "../flow/gradient_flow.h"
#include "../gauge/GaugeField.h"
#include "../mpi/MpiTopology.h"

namespace mpi::observables {
double mean_plaquette_local(const GaugeField& field, const GeometryCB& geo);                    // sum, unnormalised
double mean_plaquette_global(GaugeField& field, const GeometryCB& geo, MpiTopology& topo);      // / (6 V)
SU3 clover_site(const GaugeField& field, const GeometryCB& geo, size_t site, int mu, int nu);  // F_mu_nu(site)
int levi_civita(int mu, int nu, int rho, int sigma);
std::pair<double, double> local_q_e_clover(const GaugeField& field, const GeometryCB& geo,
                                           size_t site);                                        // (q, e) at site
std::pair<double, double> topo_q_e_clover(const GaugeField& field, const GeometryCB& geo);      // (Q, sum e)
std::pair<double, double> topo_q_e_clover_global(const GaugeField& field, const GeometryCB& geo,
                                                 MpiTopology& topo);                            // (Q, E = sum e / V)
std::vector<double> topo_charge_flowed(GaugeField& field, const GeometryCB& geo, GradientFlow& gf,
                                       mpi::MpiTopology& topo, int N_steps_gf, int N_rk_steps);
}  // namespace mpi::observables
