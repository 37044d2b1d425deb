// Kernel instantiation of the Shake128N32 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsShake128N32 = Launch<Shake128N32, Shake128N32Chain>::table("Shake128N32", XMSS_SHAKE128);
}  // namespace xb
