// heatbath/heatbath_mpi.h -- checkerboard Cabibbo-Marinari heatbath (reference
// src/heatbath/heatbath_mpi.h:13-17) on the GPU.
//
// The std::mt19937_64 arguments are kept for signature compatibility.  The first heatbath call on
// a field takes one 64-bit draw from rng[0] as the field's Philox key (GaugeField::hb_seed); every
// sweep() call then uses the next sweep index of the field, so results depend on (seed, sweep
// index) only -- not on thread counts.
#pragma once
#include <random>
#include <vector>

#include "../gauge/GaugeField.h"
#include "../io/params.h"
#include "../mpi/MpiTopology.h"

namespace mpi::heatbathcb {
// One Cabibbo-Marinari hit (subgroups (0,1), (1,2), (0,2)) of link (site, mu) (heatbath_mpi.cpp:10-33);
// site is an index of the halo'd box (halo sites wrap to their periodic interior image).  A receives
// the link's staple, as the reference leaves it.  The hit's uniforms come from the link's Philox
// stream keyed on one 64-bit draw of rng (sweep index 0): consecutive hits on one rng use distinct
// streams, and the result depends on rng's state alone.
void hit(GaugeField& field, const GeometryCB& geo, size_t site, int mu, double beta, SU3& A, std::mt19937_64& rng);
// All links of one site parity, mu = 0..3 as four race-free (parity, mu) sets (heatbath_mpi.cpp:36-57).
void sweep(GaugeField& field, const GeometryCB& geo, double beta, int N_hits, std::vector<std::mt19937_64>& rng,
           site_parity update_parity);
// N_samples x N_sweeps x (sweep EV; sweep OD) if the topology's parity is the active one
// (heatbath_mpi.cpp:60-75).
std::vector<double> samples(GaugeField& field, const GeometryCB& geo, MpiTopology& topo, const HbParams& params,
                            std::vector<std::mt19937_64>& rng, parity active_parity);
}  // namespace mpi::heatbathcb
