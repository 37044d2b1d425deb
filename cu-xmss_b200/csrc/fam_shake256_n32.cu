// Kernel instantiation of the Shake256N32 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsShake256N32 = Launch<Shake256N32, Shake256N32Chain>::table("Shake256N32", XMSS_SHAKE256);
}  // namespace xb
