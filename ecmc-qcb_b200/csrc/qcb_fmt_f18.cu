// Kernels and launchers of the float / 9-complex-per-link storage format.
#include "qcb_fmt.cuh"

namespace qcb {
const FmtOps kOpsF18 = FmtImpl<float, 9>::make();
}  // namespace qcb
