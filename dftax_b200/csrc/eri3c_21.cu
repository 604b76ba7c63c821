// Instantiations of the 3-center kernels of bra class (l1, l2) = (2, 1), see eri3c.cuh.
#include "eri3c.cuh"

namespace dfjk {

bool launch_eri3c_21(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a) {
  return launch_lc<2, 1>(lc, grid, s, a);
}

bool launch_eri3c_batch_21(int lc, unsigned blocks, cudaStream_t s, const Eri3cBatch& b) {
  return launch_lc_batch<2, 1>(lc, blocks, s, b);
}

}  // namespace dfjk
