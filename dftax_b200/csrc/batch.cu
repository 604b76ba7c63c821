// Batched and served SCF solves (include/dfbatch.h).
//
// The engine's workers each own a library context (their own cuBLAS and
// cuSOLVER handles) and a non-blocking CUDA stream. Requests wait in a FIFO;
// a free worker takes the head once its estimated device bytes fit in the
// budget beside the solves already running, so requests that arrive while
// others run start as soon as memory frees up, and the device work of the
// running solves overlaps. A solve is: plan creation and DF build
// (dfjk_plan_create, dfjk_build), the SCF (dfscf_create, dfscf_run), the
// optional density copy, then everything freed. The kernels are the ones a
// solve made alone runs, with the same fixed-order reductions, so a result
// does not depend on what else is running.
#include "internal.h"
#include "scf.h"
#include "../../include/dfbatch.h"

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

namespace {

using clock_type = std::chrono::steady_clock;

struct OwnedBasis {
  dfjk_basis b{};
  std::vector<double> centers, exps, coefs, c2s;
  std::vector<int32_t> ang;
  void copy(const dfjk_basis* s) {
    if (!s || s->ncart <= 0 || s->max_prim <= 0 || !s->centers || !s->exponents ||
        !s->coefficients || !s->angular)
      dfjk::fail(DFJK_ERR_INVALID, "request basis: null array or empty basis");
    const int64_t n = s->ncart, mp = s->max_prim;
    centers.assign(s->centers, s->centers + 3 * n);
    exps.assign(s->exponents, s->exponents + n * mp);
    coefs.assign(s->coefficients, s->coefficients + n * mp);
    ang.assign(s->angular, s->angular + 3 * n);
    if (s->cart2sph) c2s.assign(s->cart2sph, s->cart2sph + n * (int64_t)s->nsph);
    b = *s;
    b.centers = centers.data();
    b.exponents = exps.data();
    b.coefficients = coefs.data();
    b.angular = ang.data();
    b.cart2sph = s->cart2sph ? c2s.data() : nullptr;
  }
};

struct Job {
  int64_t id = 0;
  OwnedBasis orb, aux;
  dfjk_options popts{};
  dfscf_options sopts{};
  int natom = 0, nocc = 0;
  int64_t npoint = 0;
  std::vector<double> xyz, charge, gxyz, gw;
  double* P_out = nullptr;
  std::vector<double> P0;   // initial density (empty: core guess)
  int64_t bytes = 0;
  dfbatch_result res{};
  bool done = false;
};

double since(clock_type::time_point t0) {
  return std::chrono::duration<double>(clock_type::now() - t0).count();
}

// functions of a basis: spherical columns with cart2sph, else cartesian rows;
// sum over shell pairs a <= b of n_a n_b (the rows of B, diagonal blocks full)
void basis_sizes(const dfjk_basis* b, int64_t* nfun, int64_t* pair_rows) {
  std::vector<int> nf;
  for (int64_t i = 0; i < b->ncart;) {
    const int* a = b->angular + 3 * i;
    const int l = a[0] + a[1] + a[2];
    const int nc = (l + 1) * (l + 2) / 2;
    nf.push_back(b->cart2sph ? 2 * l + 1 : nc);
    i += nc;
  }
  int64_t n = 0, sq = 0;
  for (int v : nf) {
    n += v;
    sq += (int64_t)v * v;
  }
  *nfun = n;
  *pair_rows = (n * n + sq) / 2;
}

// device bytes of one solve: the plan (B, metric and factor, raw 3-center
// chunk and its digit planes, mixed K digit planes), the J/K workspaces, the
// SCF matrices and DIIS history, and the XC chunk buffers; upper bounds with
// every metric direction kept, plus 10% and 256 MB
int64_t estimate(const dfbatch_request* r) {
  int64_t nao, rows, naux, arows;
  basis_sizes(r->orb, &nao, &rows);
  basis_sizes(r->aux, &naux, &arows);
  const int64_t ldb = (naux + 7) / 8 * 8, naux16 = (naux + 15) / 16 * 16, nao16 = (nao + 15) / 16 * 16;
  const bool mixed = r->plan_opts.precision == DFJK_MIXED;
  const int digits = mixed ? 5 : 7;
  const int64_t chunk = r->plan_opts.chunk_bytes > 0 ? r->plan_opts.chunk_bytes : (int64_t)2 << 30;
  const int64_t raw_rows = std::min<int64_t>(rows, std::max<int64_t>(1, chunk / (8 * naux)) + 256);
  int64_t b = rows * ldb * 8;                                   // B
  b += 3 * naux * naux * 8 + naux * ldb * 8;                    // metric, eigenvectors, work, L
  b += raw_rows * naux * 8 + digits * raw_rows * naux16;        // raw chunk and its planes
  b += digits * ldb * naux16;                                   // planes of L
  if (mixed) b += 4 * ldb * nao * nao16;                        // K digit planes
  const int64_t nocc = std::max(1, r->nocc);
  const int64_t x = std::min<int64_t>((int64_t)6 << 30, nao * ldb * nocc * 8);
  b += x + x * 5 / 8 + (ldb * nocc / 8192 + 2) * nao * nao * 8;  // K half transform, slices, partials
  const int64_t diis = r->scf_opts.diis_space > 0 ? r->scf_opts.diis_space : 8;
  b += (18 + 2 * diis) * nao * nao * 8;                          // SCF matrices (purification too), DIIS
  const int64_t G = r->scf_opts.grid_chunk > 0 ? r->scf_opts.grid_chunk : 16384;
  // XC chunk buffers and a V accumulator on each of the solve's XC streams
  // (one unless the request asks for more: xc.cu), the grid
  const int64_t nbr = r->scf_opts.xc_streams > 0 ? r->scf_opts.xc_streams : 1;
  b += nbr * (6 * nao * G * 8 + 2 * nao * nao * 8) + r->npoint * 4 * 8;
  return b + b / 10 + ((int64_t)256 << 20);
}

}  // namespace

struct dfbatch {
  int device = 0;
  dfbatch_options o{};
  int64_t budget = 0, in_use = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> pending;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  int64_t next_id = 0;
  bool stop = false;
  std::vector<std::thread> workers;
  clock_type::time_point t0;
};

namespace {

void run_job(dfjk_ctx* ctx, cudaStream_t s, Job& j) {
  dfjk_plan* plan = nullptr;
  dfscf* scf = nullptr;
  auto check = [&](dfjk_status st) {
    if (st != DFJK_OK) dfjk::fail(st, "%s", dfjk_last_error(ctx));
  };
  dfjk_status st = DFJK_OK;
  std::string msg;
  try {
    // the engine's solves overlap one another: each runs its XC chunks on one
    // stream unless the request asks otherwise
    if (j.sopts.xc_streams == 0) j.sopts.xc_streams = 1;
    check(dfjk_plan_create(ctx, &j.orb.b, &j.aux.b, &j.popts, &plan));
    check(dfjk_build(plan, s));
    check(dfscf_create(plan, j.natom, j.xyz.data(), j.charge.data(), j.npoint,
                       j.npoint ? j.gxyz.data() : nullptr, j.npoint ? j.gw.data() : nullptr, j.nocc,
                       &j.sopts, &scf, s));
    dfjk::DevBuf P0;
    if (!j.P0.empty()) {
      P0.alloc(j.P0.size() * sizeof(double));
      DFJK_CUDA(cudaMemcpyAsync(P0.p, j.P0.data(), j.P0.size() * sizeof(double),
                                cudaMemcpyHostToDevice, s));
    }
    check(dfscf_run(scf, j.P0.empty() ? nullptr : P0.as<double>(), nullptr, s));
    check(dfscf_get_result(scf, &j.res.scf));
    if (j.P_out) {
      dfjk_plan_info info;
      check(dfjk_plan_get_info(plan, &info));
      dfjk::DevBuf P;
      P.alloc((size_t)info.nao * info.nao * sizeof(double));
      check(dfscf_get_density(scf, P.as<double>(), s));
      DFJK_CUDA(cudaMemcpyAsync(j.P_out, P.p, (size_t)info.nao * info.nao * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
      DFJK_CUDA(cudaStreamSynchronize(s));
    }
  } catch (const dfjk::Error& e) {
    st = e.code;
    msg = e.msg;
  } catch (const std::exception& e) {
    st = DFJK_ERR_INVALID;
    msg = e.what();
  }
  if (scf) dfscf_destroy(scf);
  if (plan) dfjk_plan_destroy(plan);
  // the inputs are no longer needed; the record keeps only the result
  j.orb = OwnedBasis{};
  j.aux = OwnedBasis{};
  std::vector<double>().swap(j.gxyz);
  std::vector<double>().swap(j.gw);
  j.res.status = st;
  std::snprintf(j.res.message, sizeof j.res.message, "%s", msg.c_str());
}

void worker_main(dfbatch* e, int w) {
  dfjk_ctx* ctx = nullptr;
  cudaStream_t s = nullptr;
  const dfjk_status cst = dfjk_create(e->device, &ctx);
  if (cst == DFJK_OK) {
    cudaSetDevice(e->device);
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
  }
  for (;;) {
    Job* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(e->mu);
      e->cv_work.wait(lk, [&] {
        if (e->pending.empty()) return e->stop;
        return e->in_use + e->pending.front()->bytes <= e->budget;
      });
      if (e->pending.empty()) break;
      j = e->pending.front();
      e->pending.pop_front();
      e->in_use += j->bytes;
    }
    j->res.worker = w;
    j->res.t_start = since(e->t0);
    if (cst != DFJK_OK || !s) {
      j->res.status = cst != DFJK_OK ? cst : DFJK_ERR_CUDA;
      std::snprintf(j->res.message, sizeof j->res.message, "worker %d has no device context", w);
    } else {
      cudaSetDevice(e->device);
      run_job(ctx, s, *j);
    }
    j->res.t_end = since(e->t0);
    {
      std::lock_guard<std::mutex> lk(e->mu);
      e->in_use -= j->bytes;
      j->done = true;
    }
    e->cv_done.notify_all();
    e->cv_work.notify_all();
  }
  if (s) cudaStreamDestroy(s);
  if (ctx) dfjk_destroy(ctx);
}

}  // namespace

using namespace dfjk;

extern "C" {

void dfbatch_default_options(dfbatch_options* o) {
  if (!o) return;
  *o = dfbatch_options{};
  o->workers = 4;
  o->hbm_budget = 0;
}

dfjk_status dfbatch_create(int device, const dfbatch_options* opts, dfbatch** out) {
  if (!out) return DFJK_ERR_INVALID;
  *out = nullptr;
  auto e = std::make_unique<dfbatch>();
  dfjk_status st = guard(nullptr, [&] {
    int n = 0;
    DFJK_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) fail(DFJK_ERR_INVALID, "device %d out of range (%d)", device, n);
    DFJK_CUDA(cudaSetDevice(device));
    e->device = device;
    if (opts) e->o = *opts;
    else dfbatch_default_options(&e->o);
    if (e->o.workers < 1 || e->o.workers > 64) fail(DFJK_ERR_INVALID, "workers=%d", e->o.workers);
    size_t free_b = 0, total_b = 0;
    DFJK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    e->budget = e->o.hbm_budget > 0 ? e->o.hbm_budget : (int64_t)(0.85 * (double)free_b);
    e->t0 = clock_type::now();
    try {
      for (int w = 0; w < e->o.workers; ++w) e->workers.emplace_back(worker_main, e.get(), w);
    } catch (...) {
      // a worker that cannot be started: stop and join those that were
      {
        std::lock_guard<std::mutex> lk(e->mu);
        e->stop = true;
      }
      e->cv_work.notify_all();
      for (auto& t : e->workers) t.join();
      e->workers.clear();
      throw;
    }
  });
  if (st != DFJK_OK) return st;
  *out = e.release();
  return DFJK_OK;
}

dfjk_status dfbatch_destroy(dfbatch* e) {
  if (!e) return DFJK_OK;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    e->stop = true;
  }
  e->cv_work.notify_all();
  for (auto& t : e->workers) t.join();
  delete e;
  return DFJK_OK;
}

dfjk_status dfbatch_estimate(const dfbatch_request* r, int64_t* bytes) {
  if (!r || !bytes || !r->orb || !r->aux || !r->orb->angular || !r->aux->angular)
    return DFJK_ERR_INVALID;
  return guard(nullptr, [&] { *bytes = estimate(r); });
}

dfjk_status dfbatch_submit(dfbatch* e, const dfbatch_request* r, int64_t* id) {
  if (!e || !r || !id) return DFJK_ERR_INVALID;
  auto j = std::make_unique<Job>();
  dfjk_status st = guard(nullptr, [&] {
    if (r->natom <= 0 || !r->atom_xyz || !r->atom_charge) fail(DFJK_ERR_INVALID, "no atoms");
    if (r->nocc <= 0) fail(DFJK_ERR_INVALID, "nocc=%d", r->nocc);
    if (r->npoint < 0 || (r->npoint > 0 && (!r->grid_xyz || !r->grid_w)))
      fail(DFJK_ERR_INVALID, "bad grid");
    j->orb.copy(r->orb);
    j->aux.copy(r->aux);
    j->popts = r->plan_opts;
    j->sopts = r->scf_opts;
    j->natom = r->natom;
    j->nocc = r->nocc;
    j->npoint = r->npoint;
    j->xyz.assign(r->atom_xyz, r->atom_xyz + 3 * r->natom);
    j->charge.assign(r->atom_charge, r->atom_charge + r->natom);
    if (r->npoint > 0) {
      j->gxyz.assign(r->grid_xyz, r->grid_xyz + 3 * r->npoint);
      j->gw.assign(r->grid_w, r->grid_w + r->npoint);
    }
    j->P_out = r->P_out;
    if (r->P_guess) {
      const int64_t nao = r->orb->cart2sph ? r->orb->nsph : r->orb->ncart;
      j->P0.assign(r->P_guess, r->P_guess + nao * nao);
    }
    j->bytes = estimate(r);
    if (j->bytes > e->budget)
      fail(DFJK_ERR_MEMORY, "request needs about %lld bytes, above the budget of %lld",
           (long long)j->bytes, (long long)e->budget);
  });
  if (st != DFJK_OK) return st;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    j->id = e->next_id++;
    j->res.t_submit = since(e->t0);
    j->res.bytes = j->bytes;
    *id = j->id;
    e->pending.push_back(j.get());
    e->jobs[j->id] = std::move(j);
  }
  e->cv_work.notify_all();
  return DFJK_OK;
}

dfjk_status dfbatch_wait(dfbatch* e, int64_t id, dfbatch_result* res) {
  if (!e || !res) return DFJK_ERR_INVALID;
  std::unique_lock<std::mutex> lk(e->mu);
  auto it = e->jobs.find(id);
  if (it == e->jobs.end()) return DFJK_ERR_INVALID;
  Job* j = it->second.get();
  e->cv_done.wait(lk, [&] { return j->done; });
  *res = j->res;
  return DFJK_OK;
}

dfjk_status dfbatch_poll(dfbatch* e, int64_t id, int32_t* done) {
  if (!e || !done) return DFJK_ERR_INVALID;
  std::lock_guard<std::mutex> lk(e->mu);
  auto it = e->jobs.find(id);
  if (it == e->jobs.end()) return DFJK_ERR_INVALID;
  *done = it->second->done ? 1 : 0;
  return DFJK_OK;
}

}  // extern "C"
