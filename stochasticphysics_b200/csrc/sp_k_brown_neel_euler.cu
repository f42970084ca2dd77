// Kernel instantiations for one problem (split per problem for parallel builds).
#include "sp_instantiate.cuh"

namespace sp {
void fill_brown_neel_euler(KernelSet* tab) { fill_problem<kBrownNeelEuler>(tab); }
}  // namespace sp
