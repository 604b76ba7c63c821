// Internal declarations of the dfjk library (not part of the C ABI).
#pragma once

#include "common.h"

#include <functional>

namespace dfjk {

struct Plan;

// Phases timed with CUDA events on the call's stream (see dfjk_phase_times).
enum Phase {
  kPhMetric = 0, kPhPairs, kPhEri3c, kPhBgemm, kPhJ, kPhKhalf, kPhKsyrk, kPhKplanes, kPhCount
};

struct PhaseTimer {
  std::vector<cudaEvent_t> ev[kPhCount];   // begin/end pairs
  size_t used[kPhCount] = {0};
  void reset(int p) { used[p] = 0; }
  void mark(int p, cudaStream_t s);        // records the next event of phase p
  double ms(int p);                        // sum of elapsed over recorded pairs
  void destroy();
  ~PhaseTimer() { destroy(); }
};


// The chunks of one XC evaluation run on this many concurrent branches (xc.cu).
constexpr int kXcBranches = 8;

struct Context {
  int device = 0;
  std::string last_error;
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  // streams, join events and cuBLAS handles of the XC branches, made on first
  // use and kept for the context's life (every SCF of the context reuses them)
  cudaStream_t xc_stream[kXcBranches] = {};
  cudaEvent_t xc_done[kXcBranches] = {};
  cudaEvent_t xc_fork = nullptr;
  cublasHandle_t xc_blas[kXcBranches] = {};
  // each branch handle's GEMM workspace, set explicitly (cublasSetWorkspace)
  // so cuBLAS never allocates one itself around a graph capture
  DevBuf xc_ws[kXcBranches];
  DevBuf boys;   // kBoysNgrid x (kBoysNmax+1) doubles
  DevBuf boys_asym;  // 0.5*Gamma(n+1/2), n = 0..kBoysNmax
  // device address of the no-alloc J path's fixed scratch array on this
  // context's device, looked up when the context is created
  double* noalloc_scratch = nullptr;
};

// Device address of the no-alloc scratch array on the current device
// (cudaGetSymbolAddress; loads the module that holds it).
double* noalloc_scratch_address();

struct ClassRange {   // a contiguous run of shell pairs of one (l1, l2) class
  int l1, l2;
  int64_t begin, count;      // into the pair arrays
  int64_t pp_begin, pp_count;  // primitive pairs
  int64_t esph_off;          // doubles into the Esph buffer
};

struct Plan {
  Context* ctx = nullptr;
  dfjk_options opts{};
  // operator of this plan's integrals: 0 = Coulomb, > 0 = erf(atten r)/r
  double atten = 0.0;
  // range-separated plans (opts.omega > 0) own a second plan for the
  // long-range operator over the same bases and shell pairs; it is built with
  // this one and freed with it
  dfjk_plan* lr = nullptr;
  bool owned_by_parent = false;
  Shells orb, aux;
  Blocks c2s_orb, c2s_aux;
  int nao = 0, naux = 0;
  // kept shell pairs, ordered by class; s1 has the larger l
  std::vector<int> pair_s1, pair_s2, pair_orig_a, pair_orig_b;
  std::vector<int64_t> pair_row0, pair_pp0;
  std::vector<int> pair_npp;
  std::vector<ClassRange> classes;
  int64_t nrows = 0, npp = 0, esph_doubles = 0;
  // aux column layout: shells sorted by l, columns in that order
  std::vector<int> aux_order;        // sorted position -> shell index
  std::vector<int> aux_col0;         // per shell (original index) -> column
  int aux_lbegin[8] = {0}, aux_lcount[8] = {0};
  std::vector<int> aux_perm;         // column (permuted) -> dftax aux index
  // device: pairs
  DevBuf d_pair_s1, d_pair_s2, d_pair_row0, d_pair_pp0, d_pair_npp;
  DevBuf d_pp_P, d_pp_g, d_pp_pref, d_esph;   // primitive-pair data
  DevBuf d_pp_pair, d_pp_pa, d_pp_pb;         // primitive pair -> (pair, prim a, prim b)
  DevBuf d_aux_sorted;   // sorted position -> aux shell index
  DevBuf d_aux_perm;     // column -> dftax index
  // rows -> (m, n) and weights; K lists (CSR over m)
  DevBuf d_row_m, d_row_n, d_row_w, d_kptr, d_krow, d_kn;
  // build products
  int64_t nfit = 0, ldb = 0;
  int built = 0;
  bool metric_ready = false;   // metric factor computed at creation, not yet used by a build
  DevBuf d_metric;   // naux x naux: V, then eigenvectors (column-major)
  DevBuf d_w;        // eigenvalues
  DevBuf d_L;        // naux x ldb factor (column-major, zero padded)
  DevBuf d_B;        // nrows x ldb (row-major)
  std::vector<double> w_host;
  int64_t k0 = 0;    // first kept eigen-direction
  PhaseTimer timer;
  // persistent workspaces (grow-only), reused by every build and J/K call
  DevBuf ws_raw, ws_syevd, ws_info, ws_flag, ws_dvec, ws_gamma, ws_part, ws_X, ws_Cp, ws_sel;
  // streamed plans: one chunk of B rows, the chunk's K-list bounds
  DevBuf ws_bchunk, ws_kb, ws_ke;
  // mixed precision: int8 digit planes of the square B_x for the tensor-core half transform
  DevBuf d_oz_a, d_oz_ea;
  int64_t nao_p16 = 0, naux_p16 = 0;
  DevBuf ws_oz_c, ws_oz_eb, ws_oz_err;
  // mixed precision: digit planes of L^T (per build) and of one raw 3-center chunk
  DevBuf ws_oz_l, ws_oz_el, ws_oz_raw, ws_oz_er;
  // mixed precision: digit slices of X, their exponents and per-slice K partials
  DevBuf ws_oz_x, ws_oz_ex, ws_oz_kp;
  // float64 K = X X^T: lower tile pairs and per-slice partials
  DevBuf ws_syrk_tiles, ws_syrk;
};

// ---- mixed precision on the int8 tensor cores (ozaki.cu) ----
void ozaki_prepare_l(Plan& p, cudaStream_t s);
// error flag of the tensor-core pipeline and non-finite inputs of the digit
// splits since ozaki_prepare_l (one host synchronization)
void ozaki_check(Plan& p, cudaStream_t s);
void ozaki_split_raw(Plan& p, const double* raw, int64_t nr, int8_t* planes, int64_t plane_stride,
                     int* e, cudaStream_t s);
void ozaki_bgemm(Plan& p, const int8_t* planes, int64_t plane_stride, const int* e, int64_t nr,
                 double* Bout, cudaStream_t s);
void build_ozaki_planes(Plan& p, cudaStream_t s);
void ozaki_prepare_c(Plan& p, const double* Cp, int64_t nsel, cudaStream_t s);
void ozaki_k1(Plan& p, int64_t nsel, int64_t x0, int64_t n, double* X, cudaStream_t s);
void ozaki_syrk(Plan& p, const double* X, int64_t kt, double sign, bool beta0, double* K,
                cudaStream_t s);

// ---- 3-center row chunks (api.cu) ----
int64_t chunk_budget(const Plan& p);   // bytes of one chunk of 3-center rows
// runs [first, end) of kept pairs whose rows x ld doubles fit in budget bytes
std::vector<std::pair<int64_t, int64_t>> pair_chunks(const Plan& p, int64_t ld, int64_t budget);
int64_t rows_of(const Plan& p, int64_t b, int64_t e);   // rows of pairs [b, e)
// Streamed plans: rebuilds B chunk by chunk of kept pairs (the build's
// kernels) and calls fn(first row, rows, chunk) for each, in row order; the
// chunk (rows x ldb) is valid during the call on stream s.
void for_each_b_chunk(Plan& p, cudaStream_t s,
                      const std::function<void(int64_t r0, int64_t nr, const double* Bc)>& fn);

// ---- kernels & launchers (md.cu) ----
void boys_table_host(std::vector<double>& tbl, std::vector<double>& asym);
void launch_boys(const Context& c, const double* t, int64_t n, int nmax, double* out, cudaStream_t s);
void launch_pair_setup(Plan& p, cudaStream_t s);
// Every row of several plans (each into its ws_raw, ld = naux) with one
// persistent launch per (l1, l2 | lc) class over a work queue spanning the
// plans.
void launch_eri3c_rows_batch(const std::vector<Plan*>& ps, cudaStream_t s);
// Builds several plans of one context: the 3-center rows of the plans whose
// rows fit in one chunk share their launches (launch_eri3c_rows_batch); the
// others are built one by one.
void build_batch(const std::vector<Plan*>& ps, cudaStream_t s);
void launch_eri3c_rows(Plan& p, int64_t pair_begin, int64_t pair_end, int64_t row_base,
                       void* out, int64_t ld, bool f32, cudaStream_t s);
void launch_eri2c(Plan& p, double* out, int64_t ld, cudaStream_t s);
void launch_schwarz(const Context& c, Shells& sh, const std::vector<int>& pa,
                    const std::vector<int>& pb, std::vector<double>& qmax);

// ---- contractions (jk.cu) ----
void jk_compute(Plan& p, const double* C, const double* w, int64_t ncol, double* J, double* K,
                cudaStream_t s);
// gamma = B^T vec(Ptot) over the plan's rows (ldb doubles; the J intermediate)
void gamma_from_density(Plan& p, const double* Ptot, double* gamma, cudaStream_t s);

// ---- nuclear gradient of the DF energy (grad.cu) ----
// E and dE/dR at a fixed density P (nspin x nao x nao, device): per orbital
// shell and per auxiliary shell (device, [n][3], overwritten)
double energy_gradient(Plan& p, const double* P, int nspin, double hf, double* grad_orb,
                       double* grad_aux, cudaStream_t s);

void check_finite(Plan& p, const double* x, int64_t n, cudaStream_t s, const char* what);

// solid harmonics (api.cu)
void standard_block(int l, std::vector<double>& out);   // ncart(l) x (2l+1)

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

}  // namespace dfjk

struct dfjk_ctx {
  dfjk::Context c;
};

namespace dfjk {
// Runs fn and turns what it throws into a status (and the context's last
// error): every extern "C" entry point goes through this, so no C++ exception
// crosses the C ABI.
template <class Fn>
dfjk_status guard(Context* c, Fn&& fn) {
  try {
    fn();
    if (c) c->last_error.clear();
    return DFJK_OK;
  } catch (const Error& e) {
    if (c) c->last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    if (c) c->last_error = "host allocation failed";
    return DFJK_ERR_MEMORY;
  } catch (const std::exception& e) {
    if (c) c->last_error = e.what();
    return DFJK_ERR_INVALID;
  }
}
}  // namespace dfjk
struct dfjk_plan {
  dfjk::Plan p;
};
