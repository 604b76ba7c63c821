/*
 * dfbatch.h — many Kohn-Sham SCF solves of uneven size on one GPU, admitted
 * by a device-memory budget and run concurrently (batching and serving).
 *
 * dftax solves conformers of one molecule in a vmapped batch
 * (dftax/ks/batched.py:82-304); here the molecules may differ in size and
 * composition, and requests may arrive while others run. An engine owns W
 * workers, each with its own library context (cuBLAS/cuSOLVER handles) and
 * CUDA stream. A submitted request is admitted first-in, first-out once its
 * estimated device bytes fit in the budget beside the solves already running
 * (continuous admission: as solves finish, their memory frees and the next
 * requests start); the device work of the running solves overlaps on the GPU.
 * Each admitted solve builds its DF plan (dfjk.h), keeps B, P, C, the DIIS
 * history and its grid on the device for the whole solve, runs the SCF
 * (dfscf.h) and frees its memory. Every result is computed by the same
 * deterministic kernels as a solve made alone.
 *
 * All request arrays are host arrays, copied at submission.
 */
#ifndef DFBATCH_H
#define DFBATCH_H

#include <stdint.h>

#include "dfjk.h"
#include "dfscf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dfbatch dfbatch;

typedef struct {
  int32_t workers;      /* concurrent solves (streams), default 4                       */
  int32_t reserved;
  int64_t hbm_budget;   /* device bytes the running solves may hold together; 0: 85% of
                           the device memory free when the engine is created            */
} dfbatch_options;

typedef struct {
  const dfjk_basis* orb;        /* orbital and auxiliary bases (dfjk.h layout)          */
  const dfjk_basis* aux;
  dfjk_options plan_opts;       /* precision, screen, ... of the DF plan                */
  int32_t natom;
  int32_t nocc;                 /* doubly occupied orbitals (closed shell)              */
  const double* atom_xyz;       /* [natom][3] Bohr                                      */
  const double* atom_charge;    /* [natom]                                              */
  int64_t npoint;               /* XC grid points and weights (dfscf.h)                 */
  const double* grid_xyz;
  const double* grid_w;
  dfscf_options scf_opts;
  double* P_out;                /* optional host [nao][nao]: the converged density      */
  const double* P_guess;        /* optional host [nao][nao] initial density (a
                                   superposition of atomic densities, guess.py:529-546,
                                   or a previous solve's); NULL: the core-Hamiltonian
                                   guess                                                */
} dfbatch_request;

typedef struct {
  int32_t status;               /* dfjk_status of the solve                             */
  int32_t worker;               /* the worker that ran it                               */
  dfscf_result scf;
  double t_submit, t_start, t_end;  /* seconds since the engine was created             */
  int64_t bytes;                /* device bytes reserved for it                         */
  char message[256];            /* error message when status != DFJK_OK                 */
} dfbatch_result;

void dfbatch_default_options(dfbatch_options* opts);
dfjk_status dfbatch_create(int device, const dfbatch_options* opts, dfbatch** engine);
/* Waits for every submitted solve, then stops the workers. */
dfjk_status dfbatch_destroy(dfbatch* engine);

/* Copies the request and queues it; returns at once with its id. A request
 * whose estimate exceeds the whole budget is refused (DFJK_ERR_MEMORY). */
dfjk_status dfbatch_submit(dfbatch* engine, const dfbatch_request* req, int64_t* id);
/* Blocks until solve `id` has finished and copies its result. */
dfjk_status dfbatch_wait(dfbatch* engine, int64_t id, dfbatch_result* res);
/* *done = 1 once solve `id` has finished (non-blocking). */
dfjk_status dfbatch_poll(dfbatch* engine, int64_t id, int32_t* done);
/* Device bytes a solve of this request would reserve (the admission estimate). */
dfjk_status dfbatch_estimate(const dfbatch_request* req, int64_t* bytes);

#ifdef __cplusplus
}
#endif

#endif /* DFBATCH_H */
