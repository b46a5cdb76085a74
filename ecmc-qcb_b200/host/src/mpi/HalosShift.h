// mpi/HalosShift.h -- the reference's shift buffers (src/mpi/HalosShift.h); a global shift of a
// single-GPU lattice needs none, so this is an empty object kept for signature compatibility.
#pragma once
#include "../geometry/GeometryCB.h"

struct HalosShift {
    explicit HalosShift(const GeometryCB&) {}
};
