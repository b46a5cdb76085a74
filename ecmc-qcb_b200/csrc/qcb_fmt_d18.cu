// Kernels and launchers of the double / 9-complex-per-link storage format.
#include "qcb_fmt.cuh"

namespace qcb {
const FmtOps kOpsD18 = FmtImpl<double, 9>::make();
}  // namespace qcb
