// Kernels and launchers of the double / 6-complex-per-link storage format.
#include "qcb_fmt.cuh"

namespace qcb {
const FmtOps kOpsD12 = FmtImpl<double, 6>::make();
}  // namespace qcb
