// pk_phys_mhd1.cu -- kernels and launches for ionized fluid + B + psi (solve_cg_ub).
#include "pk_launch.cuh"

namespace pk {
const PhysOps* ops_mhd1() { return make_ops<Phys<K_ION, K_NONE, K_NONE, true>>(); }
}  // namespace pk
