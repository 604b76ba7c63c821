// Instantiations of the 3-center derivative kernels of bra class (l1, l2) = (0, 0), see grad3c.cuh.
#include "grad3c.cuh"

namespace dfjk {

bool launch_grad3c_00(int lc, dim3 grid, cudaStream_t s, const Grad3cArgs& a) {
  return launch_grad3c_lc<0, 0>(lc, grid, s, a);
}

void launch_pair_deriv_00(unsigned blocks, cudaStream_t s, const PairDerivArgs& a) {
  launch_pair_deriv_t<0, 0>(blocks, s, a);
}

}  // namespace dfjk
