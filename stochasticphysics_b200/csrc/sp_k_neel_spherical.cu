// Kernel instantiations for one problem (split per problem for parallel builds).
#include "sp_instantiate.cuh"

namespace sp {
void fill_neel_spherical(KernelSet* tab) { fill_problem<kNeelSpherical>(tab); }
}  // namespace sp
