// Instantiations of the 3-center kernels of bra class (l1, l2) = (1, 1), see eri3c.cuh.
#include "eri3c.cuh"

namespace dfjk {

bool launch_eri3c_11(int lc, dim3 grid, cudaStream_t s, const Eri3cArgs& a) {
  return launch_lc<1, 1>(lc, grid, s, a);
}

bool launch_eri3c_batch_11(int lc, unsigned blocks, cudaStream_t s, const Eri3cBatch& b) {
  return launch_lc_batch<1, 1>(lc, blocks, s, b);
}

}  // namespace dfjk
