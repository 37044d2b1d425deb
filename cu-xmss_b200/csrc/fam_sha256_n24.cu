// Kernel instantiation of the Sha256N24 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsSha256N24 = Launch<Sha256N24>::table("Sha256N24", XMSS_SHA2);
}  // namespace xb
