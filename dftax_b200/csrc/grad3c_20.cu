// Instantiations of the 3-center derivative kernels of bra class (l1, l2) = (2, 0), see grad3c.cuh.
#include "grad3c.cuh"

namespace dfjk {

bool launch_grad3c_20(int lc, dim3 grid, cudaStream_t s, const Grad3cArgs& a) {
  return launch_grad3c_lc<2, 0>(lc, grid, s, a);
}

void launch_pair_deriv_20(unsigned blocks, cudaStream_t s, const PairDerivArgs& a) {
  launch_pair_deriv_t<2, 0>(blocks, s, a);
}

}  // namespace dfjk
