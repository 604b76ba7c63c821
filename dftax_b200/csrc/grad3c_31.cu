// Instantiations of the 3-center derivative kernels of bra class (l1, l2) = (3, 1), see grad3c.cuh.
#include "grad3c.cuh"

namespace dfjk {

bool launch_grad3c_31(int lc, dim3 grid, cudaStream_t s, const Grad3cArgs& a) {
  return launch_grad3c_lc<3, 1>(lc, grid, s, a);
}

void launch_pair_deriv_31(unsigned blocks, cudaStream_t s, const PairDerivArgs& a) {
  launch_pair_deriv_t<3, 1>(blocks, s, a);
}

}  // namespace dfjk
