// Kernel instantiations for one problem (split per problem for parallel builds).
#include "sp_instantiate.cuh"

namespace sp {
void fill_neel(KernelSet* tab) { fill_problem<kNeel>(tab); }
}  // namespace sp
