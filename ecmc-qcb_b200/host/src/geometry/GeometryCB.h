// geometry/GeometryCB.h -- host geometry of the compatibility layer.
//
// Keeps the reference's halo'd indexing (src/geometry/GeometryCB.h:22-62): sites of an
// (L+2)^4 box, index(x,y,z,t) with x fastest, interior coordinates 1..L.  On one GPU the lattice
// is periodic, so the halo is a periodic copy of the opposite face, neighbours of interior sites
// are computed directly, and no link is frozen.  L is the whole lattice held by the GPU (the
// reference's L_core * n_core_dims).
#pragma once
#include <cstddef>

#include "types.h"

class GeometryCB {
   public:
    int L_int;
    int L_ext;
    size_t V_int;
    size_t V_ext;

    explicit GeometryCB(int L_) : L_int(L_), L_ext(L_ + 2) {
        V_int = (size_t)L_int * L_int * L_int * L_int;
        V_ext = (size_t)L_ext * L_ext * L_ext * L_ext;
    }
    [[nodiscard]] size_t index(int x, int y, int z, int t) const {
        return ((static_cast<size_t>(t) * L_ext + z) * L_ext + y) * L_ext + x;
    }
    void coords(size_t site, int c[4]) const {
        c[0] = (int)(site % L_ext);
        site /= L_ext;
        c[1] = (int)(site % L_ext);
        site /= L_ext;
        c[2] = (int)(site % L_ext);
        c[3] = (int)(site / L_ext);
    }
    // Neighbour in the halo'd box; steps out of the box wrap periodically through the interior.
    [[nodiscard]] size_t get_neigh(size_t site, int mu, dir d) const {
        int c[4];
        coords(site, c);
        c[mu] += (d == up) ? 1 : -1;
        if (c[mu] > L_int) c[mu] -= L_int;
        if (c[mu] < 1) c[mu] += L_int;
        return index(c[0], c[1], c[2], c[3]);
    }
    // One GPU holds the whole periodic lattice: no boundary links are frozen.
    [[nodiscard]] bool is_frozen(size_t, int) const { return false; }
    [[nodiscard]] site_parity get_parity(size_t site) const {
        int c[4];
        coords(site, c);
        return ((c[0] + c[1] + c[2] + c[3]) % 2 == 0) ? EV : OD;
    }
};
