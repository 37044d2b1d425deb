// Kernel instantiation of the Sha256N32 hash family (see families.cuh).
#include "../../include/params.h"
#include "family_ops.cuh"

namespace xb {
const FamilyOps kOpsSha256N32 = Launch<Sha256N32>::table("Sha256N32", XMSS_SHA2);
}  // namespace xb
