/*
 * dfjk.h — C ABI of the B200 density-fitting Coulomb/exchange library.
 *
 * The library replaces dftax's materialized density-fitting backend
 * (dftax/ks/terms.py:576-613, class DFCoulomb) and the integral build that
 * feeds it (dftax/ks/energy.py:406-433). All arguments are plain pointers and
 * sizes; `stream` is a cudaStream_t passed as void* (NULL = legacy default
 * stream). Compute entry points take DEVICE pointers, as an XLA FFI handler
 * receives them; the *_host variants take host pointers and copy in and out.
 *
 * Every call returns a dfjk_status; on failure dfjk_last_error(ctx) holds a
 * one-line message. Invalid input, unsupported angular momentum, device
 * memory refusal and non-finite values are reported, never trapped.
 *
 * A context or plan is not thread-safe: serialize calls that share one.
 */
#ifndef DFJK_H
#define DFJK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dfjk_ctx dfjk_ctx;
typedef struct dfjk_plan dfjk_plan;

typedef enum {
  DFJK_OK = 0,
  DFJK_ERR_INVALID = 1,     /* bad argument: null pointer, size, basis layout   */
  DFJK_ERR_UNSUPPORTED = 2, /* valid input beyond the kernels (l too high ...)  */
  DFJK_ERR_CUDA = 3,        /* CUDA runtime, cuBLAS or cuSOLVER error           */
  DFJK_ERR_MEMORY = 4,      /* device memory refused (budget or cudaMalloc)     */
  DFJK_ERR_NUMERIC = 5,     /* non-finite value or failed eigensolver           */
  DFJK_ERR_STATE = 6        /* call out of order, e.g. J/K before dfjk_build    */
} dfjk_status;

/* Precision of the build and contractions. */
enum {
  DFJK_FP64 = 0,  /* float64 integrals, B, J and K; B = (ij|P) L on int8 tensor
                     cores with 7 digits per value (2^-56 of each row scale) and
                     exact int32 accumulation, for naux <= 21788            */
  DFJK_MIXED = 1  /* float64 integrals, metric, stored B and J; the products
                     B = (ij|P) L, X = B_x C and K = X X^T (5, 4 and 5 int8
                     digits per value) on int8 tensor cores with exact int32
                     accumulation and float64 epilogues; extra 4*nfit*nao^2
                     bytes of device memory                                     */
};

/* Basis arrays in dftax's BasisData layout (dftax/energy/gto.py:132-156):
 * one row per cartesian AO, host memory, row-major. */
typedef struct {
  int64_t ncart;              /* rows (cartesian AOs)                             */
  int32_t max_prim;           /* padded primitive count per row                   */
  int32_t nsph;               /* columns of cart2sph (ignored when it is NULL)    */
  const double* centers;      /* [ncart][3], Bohr                                 */
  const double* exponents;    /* [ncart][max_prim], zero padded                   */
  const double* coefficients; /* [ncart][max_prim], zero padded                   */
  const int32_t* angular;     /* [ncart][3] (lx, ly, lz)                          */
  const double* cart2sph;     /* [ncart][nsph] block diagonal, or NULL            */
} dfjk_basis;

typedef struct {
  double screen;        /* relative Schwarz shell-pair threshold; <= 0 keeps all
                           (dftax df(screen=...), eri3c_bucketed.py:140-169)     */
  double metric_cutoff; /* relative metric eigenvalue cutoff (terms.py:191)     */
  int32_t precision;    /* DFJK_FP64 or DFJK_MIXED                               */
  int32_t streamed;     /* 0: B is built once and held in device memory; 1: B is
                           not stored: every J/K call rebuilds it chunk by chunk
                           of bra pairs (dftax's StreamedDFCoulomb, terms.py:716-
                           761), for systems whose B exceeds device memory. K
                           then runs the float64 half transform on each chunk */
  int64_t chunk_bytes;  /* staging budget for raw 3-center rows (0 = default)   */
  double omega;         /* > 0: also build the long-range erf(omega r)/r fit for
                           range-separated exchange (energy.py:419-433); 0: off */
} dfjk_options;

typedef struct {
  int64_t nao, naux;            /* spherical (or cartesian) AO / aux counts      */
  int64_t nao_cart, naux_cart;
  int64_t nshell, naux_shell;
  int64_t npair_shell;          /* kept bra shell pairs                          */
  int64_t nrows;                /* rows of B (AO pairs of the kept shell pairs)  */
  int64_t nfit;                 /* columns of B (metric directions kept)         */
  int64_t b_bytes;              /* device bytes held by B                        */
  int32_t built;                /* 1 after a successful dfjk_build               */
  int32_t precision;
} dfjk_plan_info;

/* Fill opts with dftax's defaults: screen off, cutoff 1e-7, FP64, omega 0. */
void dfjk_default_options(dfjk_options* opts);

/* Context: device, library handles and the Boys table (dftax/energy/boys.py:81-123). */
dfjk_status dfjk_create(int device, dfjk_ctx** ctx);
/* Also releases the device memory cached on the context's device (dfjk_trim). */
dfjk_status dfjk_destroy(dfjk_ctx* ctx);
const char* dfjk_last_error(const dfjk_ctx* ctx);

/* Device memory of destroyed plans is kept by the library, per device, and
 * handed to the next plans (plans of one system, made one after another, get
 * their buffers back without cudaMalloc/cudaFree). dfjk_trim synchronizes the
 * context's device and returns that cached memory to the driver; a failed
 * allocation does the same before it retries. No counterpart in the reference. */
dfjk_status dfjk_trim(dfjk_ctx* ctx);

/* Plan: shells, Schwarz-kept shell pairs, class buckets, device layout.
 * Replaces plan_eri3c / plan_pairs / _shell_pair_keep
 * (dftax/integrals/eri3c_bucketed.py:221-283, :448-483, :140-169) and the
 * cart2sph checks (:186-218). It also computes the (P|Q) metric and its
 * factor, on a stream of its own while the host builds the orbital tables,
 * so that a metric failure (DFJK_ERR_NUMERIC) can come from here; the plan's
 * first dfjk_build uses that factor and every later build recomputes it.
 * Returns with its device work complete. */
dfjk_status dfjk_plan_create(dfjk_ctx* ctx, const dfjk_basis* orb, const dfjk_basis* aux,
                             const dfjk_options* opts, dfjk_plan** plan);
dfjk_status dfjk_plan_destroy(dfjk_plan* plan);
dfjk_status dfjk_plan_get_info(const dfjk_plan* plan, dfjk_plan_info* info);

/* Build: (P|Q) metric (eri3c_bucketed.py:746-779), its factor L with
 * L L^T = V+ over eigenvalues above the cutoff (terms.py:155-192, :391-395),
 * the 3-center (ij|P) (eri3c_bucketed.py:782-854) and B = (ij|P) L.
 * Host-synchronizing (the kept-direction count sizes B). */
dfjk_status dfjk_build(dfjk_plan* plan, void* stream);

/* dfjk_build of n plans of one context (molecules of any sizes): the 3-center
 * integrals of every plan whose rows fit in one staging chunk are computed
 * in shared launches, one persistent launch per (l1, l2 | lc) integral class
 * whose blocks walk a work queue of (plan, run of shell pairs) segments, so
 * small molecules do not each pay a launch per class; then each plan's
 * B = (ij|P) L. Larger and streamed plans are built as dfjk_build builds
 * them. Every plan ends exactly as its own dfjk_build leaves it (the same
 * blocks compute the same rows). No counterpart in dftax, whose batched
 * solver (dftax/ks/batched.py:82-304) vmaps one molecule's conformers. */
dfjk_status dfjk_build_batch(dfjk_plan* const* plans, int32_t n, void* stream);

/* J and K of the density D = C diag(w) C^T (w == NULL: all ones), with
 * C [nao][ncol] row-major on the device. J, K: [nao][nao] device outputs.
 * J = sum_PQ (mn|P) V+_PQ (P|D), K = sum_PQ (ml|P) V+_PQ (ns|Q) D_ls
 * (the gradients of DFCoulomb.energy, terms.py:592-613; K as in
 * dftax/energy/hybrid.py:23-41 and terms.py:437-449). Either of J, K may be NULL. */
dfjk_status dfjk_jk(dfjk_plan* plan, const double* C, const double* w, int64_t ncol,
                    double* J, double* K, void* stream);

/* Same with host buffers: copies C (and w) in, J and K out, then synchronizes. */
dfjk_status dfjk_jk_host(dfjk_plan* plan, const double* C, const double* w, int64_t ncol,
                         double* J, double* K, void* stream);

/* The long-range plan of a plan made with omega > 0: the erf(omega r)/r
 * 3-center tensor and metric (eri3c_bucketed.py:746-854 with omega), its own
 * pseudo-inverse and factor, B_lr (int3c_lr / int2c_inv_lr of energy.py:419-433).
 * Owned by the parent (built by the parent's dfjk_build, freed with it;
 * dfjk_plan_destroy refuses it). dfjk_jk on it gives K_lr (and the long-range
 * J); the diagnostics give the attenuated tensors. DFJK_ERR_STATE without omega. */
dfjk_status dfjk_plan_long_range(const dfjk_plan* plan, dfjk_plan** lr);

/* DFCoulomb.energy (terms.py:592-613) and its P-gradient for the spin-stacked
 * density P [nspin][nao][nao] (device): energy -> *e (host scalar) and, when
 * F != NULL, dE/dP -> F [nspin][nao][nao] (device): J - a_x/2 K for nspin 1,
 * J - a_x K_sigma for nspin 2 (terms.py:500-509). Any symmetric P is handled
 * exactly (it is diagonalized on the device). Host-synchronizing. */
dfjk_status dfjk_energy(dfjk_plan* plan, const double* P, int32_t nspin, double hf_coeff,
                        double* e, double* F, void* stream);

/* The same with the long-range exchange term of range-separated hybrids
 * (terms.py:604-612): E += exchange quadratic of K_lr with hf_coeff_lr, and
 * dE/dP gains -hf_coeff_lr/2 K_lr (nspin 1) or -hf_coeff_lr K_lr,sigma
 * (nspin 2). hf_coeff_lr != 0 needs a plan made with omega > 0. */
dfjk_status dfjk_energy_rsh(dfjk_plan* plan, const double* P, int32_t nspin, double hf_coeff,
                            double hf_coeff_lr, double* e, double* F, void* stream);

/* Nuclear gradient of the DF energy at a fixed symmetric density P
 * [nspin][nao][nao] (device): the geometry derivative dftax's forces() take
 * through the integral build (forces.py:245-270), with the metric
 * pseudo-inverse differentiated by d(V+) = -V+ dV V+ (terms.py:196-204).
 * Writes dE/d(center) of every orbital shell, grad_orb [norb_shell][3], and
 * of every auxiliary shell, grad_aux [naux_shell][3] (device, shell order of
 * the bases given to dfjk_plan_create; an atom's gradient is the sum over
 * the shells on it), and the energy -> *e (host). hf_coeff as in
 * dfjk_energy; plans with omega > 0 (attenuated operator) give the gradient
 * of their own operator's energy. Host-synchronizing. */
dfjk_status dfjk_energy_grad(dfjk_plan* plan, const double* P, int32_t nspin, double hf_coeff,
                             double* e, double* grad_orb, double* grad_aux, void* stream);

/* J of D = C diag(w) C^T, as dfjk_jk computes it, without allocating any
 * device memory: for callers that must not call cudaMalloc while they run
 * (an XLA FFI handler inside a JAX program whose allocator already owns the
 * GPU's memory; a serving loop that keeps cudaMalloc/cudaFree, which
 * synchronize the device, off its hot path). No counterpart in the reference.
 * Scratch is a fixed 16.8 MB array in the library's device memory, shared by
 * all calls: plans whose B has more than 8192 columns are rejected
 * (DFJK_ERR_UNSUPPORTED), and calls that overlap on the GPU race on it. The
 * array is placed on a device when dfjk_create makes a context there (its
 * address is looked up then) and is held until the process exits, so this
 * call itself takes no device memory. Float64 plans only. */
dfjk_status dfjk_j_noalloc(dfjk_plan* plan, const double* C, const double* w, int64_t ncol,
                           double* J, void* stream);

/* ---- tracing ------------------------------------------------------------ */

/* Phases timed with CUDA events on the stream of the last dfjk_build / dfjk_jk
 * (dfjk_energy's J and K count as dfjk_jk). */
enum {
  DFJK_PHASE_METRIC = 0, /* (P|Q), eigensolver, factor L                      */
  DFJK_PHASE_PAIRS = 1,  /* primitive-pair setup (E tables in spherical form) */
  DFJK_PHASE_ERI3C = 2,  /* 3-center rows (all chunks)                        */
  DFJK_PHASE_BGEMM = 3,  /* B = (ij|P) L (all chunks)                         */
  DFJK_PHASE_J = 4,      /* gamma and J                                       */
  DFJK_PHASE_KHALF = 5,  /* K half transform                                  */
  DFJK_PHASE_KSYRK = 6,  /* K accumulation                                    */
  DFJK_PHASE_KPLANES = 7, /* mixed precision: int8 digit planes of B for K    */
  DFJK_PHASE_COUNT = 8
};

/* Milliseconds per phase of the last build / J-K call: ms[0..n). Synchronizes
 * on the recorded events. */
dfjk_status dfjk_phase_times(dfjk_plan* plan, double* ms, int32_t n);

/* Kernels this library has launched in this process (cuBLAS/cuSOLVER calls
 * not included). */
int64_t dfjk_kernel_launches(void);

/* ---- parity / diagnostic entry points ---------------------------------- */

/* Dense (nao, nao, naux) 3-center tensor in dftax's index order
 * (eri3c_bucketed.py:782-854 output). Device output; requires a plan small
 * enough for nao*nao*naux doubles. Does not need dfjk_build. */
dfjk_status dfjk_eri3c_dense(dfjk_plan* plan, double* out, void* stream);

/* (naux, naux) metric in dftax's order (eri3c_bucketed.py:746-779). */
dfjk_status dfjk_eri2c_dense(dfjk_plan* plan, double* out, void* stream);

/* V+ (naux, naux) in dftax's order after dfjk_build (terms.py:155-192). */
dfjk_status dfjk_metric_pinv(dfjk_plan* plan, double* out, void* stream);

/* Kept shell pairs as int32 [npair_shell][2] (ia <= ib, dftax shell order). Host output. */
dfjk_status dfjk_kept_pairs(const dfjk_plan* plan, int32_t* out);

/* Boys F_0..F_nmax at n points t (device): out [n][nmax+1]
 * (dftax/energy/boys.py:130-176); nmax <= 18. */
dfjk_status dfjk_boys(dfjk_ctx* ctx, const double* t, int64_t n, int32_t nmax, double* out,
                      void* stream);

/* Runs the bounded wait of the tensor-core pipelines (an mbarrier wait that
 * gives up after a %globaltimer limit and flags the error) on a barrier that
 * nothing completes: one warp with a limit of limit_ns (1e3 .. 4e9), a second
 * with the pipelines' own 4 s limit, which must return as soon as the first
 * one's timeout is flagged. Returns DFJK_ERR_CUDA with the pipelines'
 * timeout message; waited_ms[0..1] (host, optional) receive each warp's wait.
 * Nothing else is in flight in the block, and the context stays usable. */
dfjk_status dfjk_wait_selftest(dfjk_ctx* ctx, int64_t limit_ns, double* waited_ms, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DFJK_H */
