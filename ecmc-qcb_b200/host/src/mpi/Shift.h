// mpi/Shift.h -- global random shift (reference src/mpi/Shift.h; Shift.cpp:109-186) of the
// single-GPU lattice: U'(x) = U(x - s).
#pragma once
#include <random>

#include "../gauge/GaugeField.h"
#include "HalosShift.h"
#include "MpiTopology.h"

namespace mpi::shift {
// Applies the global translation by s (U'(x) = U(x - s)).
void shift_field(GaugeField& field, const GeometryCB& geo, HalosShift& h, mpi::MpiTopology& topo, const int s[4]);
// Draws s_d ~ uniform_int(0, range - 1), d = x,y,z,t, from rng exactly as Shift.cpp:165-170 does,
// prints "Shift (sx, sy, sz, st)" and applies it.  range is set_shift_range's value (default: the
// reference's per-rank L_core when the driver sets it, else the lattice extent).
void random_shift(GaugeField& field, const GeometryCB& geo, HalosShift& h, mpi::MpiTopology& topo,
                  std::mt19937_64& rng);
void set_shift_range(int range);
}  // namespace mpi::shift
