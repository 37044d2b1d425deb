// Kernel instantiation of the Shake256N24 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsShake256N24 = Launch<Shake256N24, Shake256N24Chain>::table("Shake256N24", XMSS_SHAKE256);
}  // namespace xb
