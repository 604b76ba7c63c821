// Internal declarations of the Kohn-Sham SCF around the DF J/K plan (scf.cu,
// onee.cu, xc.cu). Not part of the C ABI (include/dfscf.h).
#pragma once

#include "internal.h"
#include "../../include/dfscf.h"

namespace dfjk {

// Device view of the orbital shells for the one-electron and AO kernels.
struct OrbView {
  ShellView sh;
  const int* out0;      // first spherical (or cartesian) function of each shell
  const double* c2s;    // transformation blocks, one per l (ncart(l) x nout(l), row-major)
  int c2s_off[8];       // offset of l's block in c2s
  int nout[8];          // functions per shell of each l (2l+1, or ncart(l) without cart2sph)
  int nao;
};

// One-electron integrals (onee.cu): S, T and V = -sum_C Z_C <a|1/|r-C||b> as
// nao x nao matrices (symmetric, both triangles written), for the shell pairs
// of the orbital basis.
void launch_one_electron(const Context& c, const OrbView& ov, int nshell, const std::vector<int>& l,
                         int natom, const double* atom_xyz, const double* atom_z, double* S,
                         double* T, double* V, cudaStream_t s);

// Chunks of spatially sorted grid points, each with the orbital shells that
// are not negligible anywhere in its bounding box (xc_prepare)
constexpr int kXcMaxL = 3;   // orbital l the AO kernel evaluates (f)

struct XcChunks {
  int64_t G = 0;                       // points per chunk (the last may hold fewer)
  std::vector<int64_t> g0, ng;         // first point and count of each chunk
  std::vector<int> sh_off, sh_cnt;     // each chunk's range in the shell list
  std::vector<int> sh_lcnt;            // [chunk][l]: its shells of each l, in this order
  std::vector<int64_t> ao_off;         // each chunk's range in the compact AO map
  std::vector<int> ao_cnt;
  int max_ao = 0;
  int64_t total_ao = 0;                // sum of ao_cnt (the dense form would be nchunk * nao)
  double gemm_flop = 0.0;              // FLOP of one evaluation's two DGEMMs: sum 4 G ao_cnt^2
  DevBuf d_sh, d_sh_out0, d_ao_map;    // shells, their first compact AO, compact -> AO
};

// XC on a point grid (xc.cu)
// The chunks of one XC evaluation run on kXcBranches concurrent branches
// (chunk k on branch k % kXcBranches), each with its own buffers, and the
// context's stream and cuBLAS handle of that branch (no shared GEMM
// workspace), and its own V accumulator; one chunk's kernels fill only part
// of the GPU. The accumulators are summed in branch order at the end and the
// energy partials are per chunk, so the result does not depend on how the
// branches interleave.
struct XcBranch {
  DevBuf phi, dphi, X, W;       // [nsig][G] AO values, 3 gradients, Phi P, weighted AO
  DevBuf Pc, Vc;                // P on a chunk's AOs, its V block
  DevBuf vr, vg;                // per point: v_rho, v_grad (3)
};

struct XcWork {
  XcChunks ch;
  int nbr = kXcBranches;        // branches in use, 1..kXcBranches
  XcBranch br[kXcBranches];
  DevBuf Vacc;                  // kXcBranches x nao x nao: V accumulated per branch
  DevBuf ered;                  // energy partials per chunk and block
  // the evaluation's device work as a CUDA graph, captured on the second call
  // with the same arguments and replayed while they stay the same
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap = nullptr;   // private stream the work is captured on (capture only
                                // records; the graph is launched on the caller's stream)
  const void* g_args[4] = {nullptr, nullptr, nullptr, nullptr};   // P, Vxc, pts, w
  int64_t graph_kernels = 0;    // this library's kernels in the graph
  int calls = 0;
  bool graph_off = false;       // capture failed once: run the launches directly
  ~XcWork() {
    if (exec) cudaGraphExecDestroy(exec);
    if (cap) cudaStreamDestroy(cap);
  }
};

// Sorts the points (and weights) along a Morton curve over 1-Bohr cells;
// pts [n][3] and w [n] are host arrays, reordered in place.
void xc_sort(std::vector<double>& pts, std::vector<double>& w);
// Cuts sorted points into chunks of G points and keeps for each chunk the
// shells whose value-and-gradient bound over the chunk's bounding box exceeds
// thresh (uploads the shell lists); forgets any captured graph of ws.
void xc_chunk(const Shells& sh, const int (&nout)[8], const std::vector<double>& pts, int64_t G,
              double thresh, XcWork& ws);

struct XcParams {
  double x_scale = 0.75;        // PBE exchange share (PBE0)
  double c_scale = 1.0;         // PBE correlation share
  double rho_thresh = 1e-10;    // points at or below this density are left out
};

// E_xc of the closed-shell density P (nao x nao, symmetric, device) and, when
// Vxc != nullptr, its P-gradient symmetrized (device, nao x nao), over the grid
// points pts [n][3] with weights w [n] (device, in xc_prepare's order), chunk
// by chunk as ws.ch lays them out. Uses the context's cuBLAS handle on
// stream s. Returns E_xc (host synchronizing).
double xc_energy_fock(const Context& c, const OrbView& ov, const double* pts, const double* w,
                      const double* P, double* Vxc, const XcParams& xp, XcWork& ws,
                      cudaStream_t s);

// Becke cell weights: w[i] = raw[i] * P_owner(i) / sum_A P_A at point i
void launch_becke_partition(const double* pts, const int* owner, const double* raw, int64_t n,
                            const double* atom_xyz, const double* bragg, int natom, double* w,
                            cudaStream_t s);

}  // namespace dfjk
