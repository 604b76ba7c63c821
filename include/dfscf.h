/*
 * dfscf.h — C ABI of the Kohn-Sham SCF around the B200 DF J/K plan (dfjk.h).
 *
 * The SCF replaces dftax's KS energy and SCF driver for a closed-shell
 * density-fitted hybrid GGA (dftax/ks/energy.py:549-723, dftax/ks/scf.py:
 * 279-391): the one-electron integrals, the XC energy and its Fock matrix on
 * a caller-supplied quadrature grid (dftax's explicit-grid form,
 * dftax/grid/grid.py: points()), J and K from a built dfjk plan, Pulay DIIS
 * and the float64 Fock diagonalization, all on the device. The functional is
 * PBE0 by default (dftax/energy/xc.py:584-601): x_scale PBE exchange +
 * c_scale PBE correlation + hf_coeff exact exchange.
 *
 * Host arrays are copied at creation; the entry points that take P, F, S,
 * T, V, C take DEVICE pointers (nao x nao, symmetric; C is nao x nmo,
 * column-major, i.e. C[j * nao + i] is orbital j at AO i).
 */
#ifndef DFSCF_H
#define DFSCF_H

#include <stdint.h>

#include "dfjk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dfscf dfscf;

typedef struct {
  double hf_coeff;      /* exact-exchange fraction a_x (PBE0: 0.25)                     */
  double x_scale;       /* PBE exchange share (PBE0: 0.75)                              */
  double c_scale;       /* PBE correlation share (1)                                    */
  double e_tol;         /* |dE| convergence threshold, Ha (scf.py: 1e-8)                */
  double d_tol;         /* commutator-norm threshold (scf.py: 1e-6)                     */
  double lindep;        /* overlap eigenvalue cutoff of the orthonormalizer (1e-7)      */
  double level_shift;   /* Saunders-Hillier virtual shift, Ha (0)                       */
  double rho_thresh;    /* grid points with rho <= this are left out (1e-10)            */
  double ao_thresh;     /* a shell is left out of a chunk of grid points when its value
                           and gradient stay below this over the chunk (1e-14; 0: keep
                           every shell, the dense quadrature)                          */
  int32_t max_iter;     /* 128                                                          */
  int32_t diis_space;   /* DIIS history depth (8)                                        */
  int64_t grid_chunk;   /* grid points per XC chunk, spatially sorted (0: chosen by
                           timing 2048, 4096, 8192 and 16384 on the first molecule of each
                           size and XC stream count; the choice is kept for the
                           process)                                                    */
  int32_t xc_streams;   /* concurrent streams the XC chunks run on, 1..8 (0: 8); the
                           batch engine runs its solves, which already overlap one
                           another, with 1                                             */
  int32_t density;      /* how each iteration's density comes from the DIIS Fock matrix:
                           0: its eigenvectors (cuSOLVER syevd) and aufbau occupations;
                           1: second-order spectral projection (SP2 purification) of
                           X^T F X onto its nocc lowest eigenvalues, which is the same
                           aufbau density when the HOMO-LUMO gap is open, falling back
                           to the eigensolver for that iteration when the projection
                           does not converge (no gap). The orbitals and energies of
                           dfscf_get_orbitals come from the eigensolver either way
                           (after a projected density, the first call computes them
                           from the run's last DIIS Fock matrix)                     */
} dfscf_options;

typedef struct {
  double e_tot;         /* total energy of the last density (Ha)                        */
  double e_one;         /* Tr(P Hcore)                                                  */
  double e_coul;        /* E_J + a_x E_K (DFCoulomb.energy, terms.py:592-613)           */
  double e_xc;          /* XC energy                                                    */
  double e_nn;          /* nuclear repulsion                                            */
  double derr;          /* commutator norm of the last Fock build                       */
  int32_t n_iter;
  int32_t converged;
  int32_t nmo;          /* orbitals kept by the canonical orthonormalizer               */
  int32_t nocc;
  /* milliseconds of the last dfscf_run by part (host clock around
   * synchronized device work): J and K, the XC quadrature, the Fock
   * diagonalizations with the density, the commutator and DIIS */
  double ms_jk, ms_xc, ms_diag, ms_diis;
  int64_t xc_chunk;     /* grid points per XC chunk (set, or chosen by the autotuner)    */
  int32_t xc_graph;     /* 1: the XC evaluations replayed a captured CUDA graph          */
  int32_t n_eig;        /* densities built by the eigensolver in the last dfscf_run: the
                           core guess and every iteration with density 0; the core
                           guess and the fallbacks with density 1                       */
  double xc_gemm_flop;  /* float64 FLOP of the two DGEMMs of one XC evaluation (X = Phi P
                           and Phi^T W per chunk: 4 G n_chunk^2 summed over the chunks) */
} dfscf_result;

/* dftax's defaults for PBE0 (scf.py:279-391, xc.py:584-601, grid.py:10-45). */
void dfscf_default_options(dfscf_options* opts);

/* An SCF over a built dfjk plan (closed shell, nocc doubly occupied orbitals).
 * atoms: natom centers (Bohr) and nuclear charges; grid: npoint points [n][3]
 * (Bohr) and weights, host arrays. The orbital basis is the plan's. Computes
 * S, T, V, the nuclear repulsion and the canonical orthonormalizer (device)
 * on `stream`, and returns with that work complete. Replaces KS.__init__'s
 * non-DF part (energy.py:549-654) and scf.py:73-90. */
dfjk_status dfscf_create(dfjk_plan* plan, int32_t natom, const double* atom_xyz,
                         const double* atom_charge, int64_t npoint, const double* grid_xyz,
                         const double* grid_w, int32_t nocc, const dfscf_options* opts,
                         dfscf** scf, void* stream);
dfjk_status dfscf_destroy(dfscf* scf);

/* Runs the SCF from P0 (device nao x nao; NULL: the core-Hamiltonian guess,
 * guess.py:605-606) to |dE| < e_tol and commutator < d_tol or max_iter
 * (scf.py:279-391). run_opts (may be NULL) overrides this run's max_iter,
 * e_tol, d_tol and level_shift; the other fields are fixed at creation.
 * Host-synchronizing a few times per iteration. */
dfjk_status dfscf_run(dfscf* scf, const double* P0, const dfscf_options* run_opts, void* stream);
dfjk_status dfscf_get_result(const dfscf* scf, dfscf_result* res);
/* The last density P (device nao x nao) and orbitals: eps (device nmo) and C
 * (device nao x nmo, column-major). Either pointer may be NULL. */
dfjk_status dfscf_get_density(dfscf* scf, double* P, void* stream);
dfjk_status dfscf_get_orbitals(dfscf* scf, double* eps, double* C, void* stream);

/* ---- parity / diagnostic entry points ---------------------------------- */

/* S, T, V (device nao x nao each; any may be NULL): overlap_kinetic_bucketed
 * and nuclear_attraction_bucketed (eri3c_bucketed.py:486-694). */
dfjk_status dfscf_one_electron(dfscf* scf, double* S, double* T, double* V, void* stream);
/* E_xc of P -> *exc (host) and its symmetrized P-gradient -> Vxc (device, may
 * be NULL): GridXC.energy (terms.py:776-828) with xc_energy (grid.py:10-45). */
dfjk_status dfscf_xc(dfscf* scf, const double* P, double* exc, double* Vxc, void* stream);
/* Total energy of P -> *e (host) and the Fock matrix sym(dE/dP) -> F (device,
 * may be NULL): KS.total and scf.py:42-46 for a closed shell. */
dfjk_status dfscf_energy_fock(dfscf* scf, const double* P, double* e, double* F, void* stream);

/* Becke fuzzy-cell weights of an atom-centered grid (dftax/grid/becke.py,
 * becke_partition with the Bragg-radius size adjustment): w[i] = raw[i] *
 * P_owner[i](p_i) / sum_A P_A(p_i). pts [n][3], owner [n], raw [n], w [n] are
 * device arrays; atom_xyz [natom][3] and bragg [natom] (Bohr) host arrays. */
dfjk_status dfjk_becke_partition(dfjk_ctx* ctx, const double* pts, const int32_t* owner,
                                 const double* raw, int64_t n, int32_t natom,
                                 const double* atom_xyz, const double* bragg, double* w,
                                 void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DFSCF_H */
