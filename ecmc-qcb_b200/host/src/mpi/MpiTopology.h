// mpi/MpiTopology.h -- single-rank stand-in for the reference's Cartesian MPI topology
// (src/mpi/MpiTopology.h:10-30).  One GPU holds the whole periodic lattice, so there is one rank,
// of parity even, whose neighbours are itself.  The constructor argument is kept for signature
// compatibility; the lattice extent is carried by GeometryCB.
#pragma once

enum parity { even, odd };

namespace mpi {
class MpiTopology {
   public:
    int n_core_dim = 1;
    int rank = 0, size = 1;
    int local_rank = 0;
    int local_coords[4] = {0, 0, 0, 0};
    parity p = even;
    int x0 = 0, xL = 0, y0 = 0, yL = 0, z0 = 0, zL = 0, t0 = 0, tL = 0;
    explicit MpiTopology(int /*n_core_dim_*/) {}
};
}  // namespace mpi
