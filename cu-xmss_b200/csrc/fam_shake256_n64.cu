// Kernel instantiation of the Shake256N64 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsShake256N64 = Launch<Shake256N64, Shake256N64Chain>::table("Shake256N64", XMSS_SHAKE256);
}  // namespace xb
