// Kernels and launchers of the float / 6-complex-per-link storage format.
#include "qcb_fmt.cuh"

namespace qcb {
const FmtOps kOpsF12 = FmtImpl<float, 6>::make();
}  // namespace qcb
