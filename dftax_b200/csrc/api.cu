// Host side of the dfjk library: context, plan (shells, screening, layouts),
// build (metric factor, 3-center rows, B) and the C ABI entry points.
#include "internal.h"
#include "ozaki.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <numeric>
#include <exception>
#include <functional>
#include <thread>

namespace dfjk {

void fail(dfjk_status code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw Error{code, buf};
}

// ---------------------------------------------------------------------------
// Device memory cache. Plans are made one after another (one per geometry,
// one per request of a serving loop) with buffers of the same sizes, and
// cudaMalloc of tens of GB plus cudaFree (which synchronizes the device) cost
// ~100 ms per (H2O)_32 plan. Freed buffers are kept per device and handed out
// again to requests of at most their size and at least 3/4 of it. A cached
// buffer may still be used by work queued before it was freed (on any stream,
// by any thread), so every free takes a sequence number, and a reuse first
// synchronizes the device unless a device synchronization that began after
// the free has completed. A failed cudaMalloc empties the cache and retries;
// dfjk_trim empties it on request.
// ---------------------------------------------------------------------------

namespace {
struct Cached {
  void* p;
  size_t bytes;
  uint64_t stamp;   // sequence number of the free
};
std::mutex g_cache_mu;
// never destroyed: cudaFree at process exit could run after the driver shut down
std::vector<std::vector<Cached>>& cache() {
  static auto* c = new std::vector<std::vector<Cached>>(64);
  return *c;
}
// per device: the last sequence number handed out, and the largest one known idle
std::vector<uint64_t>& free_seq() {
  static auto* e = new std::vector<uint64_t>(64, 0);
  return *e;
}
std::vector<uint64_t>& idle_upto() {
  static auto* e = new std::vector<uint64_t>(64, 0);
  return *e;
}

void* cache_take(int dev, size_t n, size_t* got) {
  bool need_sync = false;
  void* p = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto& v = cache()[dev];
    size_t best = v.size();
    for (size_t i = 0; i < v.size(); ++i)
      if (v[i].bytes >= n && n >= v[i].bytes / 4 * 3 &&
          (best == v.size() || v[i].bytes < v[best].bytes))
        best = i;
    if (best == v.size()) return nullptr;
    p = v[best].p;
    *got = v[best].bytes;
    need_sync = v[best].stamp > idle_upto()[dev];
    v.erase(v.begin() + best);
  }
  if (need_sync) sync_device(dev);
  return p;
}
}  // namespace

std::recursive_mutex& capture_mutex() {
  static std::recursive_mutex m;
  return m;
}

void sync_device(int dev) {
  uint64_t s0;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    s0 = free_seq()[dev];
  }
  {
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    DFJK_CUDA(cudaDeviceSynchronize());
  }
  std::lock_guard<std::mutex> lk(g_cache_mu);
  idle_upto()[dev] = std::max(idle_upto()[dev], s0);
}

void cache_trim(int dev) {
  std::vector<Cached> v;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (dev < 0 || dev >= (int)cache().size()) return;
    v.swap(cache()[dev]);
  }
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(dev);
  std::lock_guard<std::recursive_mutex> cap(capture_mutex());
  for (auto& c : v) cudaFree(c.p);
  cudaSetDevice(cur);
}

void DevBuf::alloc(size_t n) {
  free();
  if (n == 0) n = 16;
  int d = 0;
  DFJK_CUDA(cudaGetDevice(&d));
  if (d >= (int)cache().size()) fail(DFJK_ERR_INVALID, "device ordinal %d out of range", d);
  size_t got = 0;
  if (void* c = cache_take(d, n, &got)) {
    p = c;
    bytes = got;
    dev = d;
    return;
  }
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cache_trim(d);
    e = cudaMalloc(&p, n);
  }
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    fail(DFJK_ERR_MEMORY, "cudaMalloc of %zu bytes failed: %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  dev = d;
}

static std::atomic<int64_t> g_launches{0};
void count_launch(int64_t n) { g_launches += n; }

void PhaseTimer::mark(int p, cudaStream_t s) {
  if (used[p] == ev[p].size()) {
    cudaEvent_t e;
    DFJK_CUDA(cudaEventCreate(&e));
    ev[p].push_back(e);
  }
  DFJK_CUDA(cudaEventRecord(ev[p][used[p]++], s));
}

double PhaseTimer::ms(int p) {
  double tot = 0.0;
  for (size_t i = 0; i + 1 < used[p]; i += 2) {
    DFJK_CUDA(cudaEventSynchronize(ev[p][i + 1]));
    float f = 0.f;
    DFJK_CUDA(cudaEventElapsedTime(&f, ev[p][i], ev[p][i + 1]));
    tot += f;
  }
  return tot;
}

void PhaseTimer::destroy() {
  for (auto& v : ev) {
    for (cudaEvent_t e : v) cudaEventDestroy(e);
    v.clear();
  }
  for (auto& u : used) u = 0;
}

void DevBuf::free() {
  if (p) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    cache()[dev].push_back({p, bytes, ++free_seq()[dev]});
  }
  p = nullptr;
  bytes = 0;
}

// ---------------------------------------------------------------------------
// Basis parsing and validation
// ---------------------------------------------------------------------------

static int comp_index(int l, int lx, int ly) {
  int idx = 0;
  for (int x = l; x > lx; --x) idx += l - x + 1;
  return idx + (l - lx - ly);
}

// Real solid harmonics r^l Y_lm (unit-sphere normalized, m = -l..l) as an
// ncart(l) x (2l+1) block in dftax's cartesian order; identity for l <= 1.
// Closed form of Helgaker, Jorgensen & Olsen, eqs. 6.4.47-6.4.50.
void standard_block(int l, std::vector<double>& out) {
  const int nc = ncart(l), ns = 2 * l + 1;
  out.assign((size_t)nc * ns, 0.0);
  if (l <= 1) {
    for (int i = 0; i < ns; ++i) out[i * ns + i] = 1.0;
    return;
  }
  auto fact = [](int n) { double r = 1; for (int i = 2; i <= n; ++i) r *= i; return r; };
  auto binom = [](int n, int k) {
    if (k < 0 || k > n) return 0.0;
    double r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
  };
  for (int col = 0; col < ns; ++col) {
    const int m = col - l, am = std::abs(m), vm2 = m < 0 ? 1 : 0;
    const double nrm = std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0)) /
                       (std::pow(2.0, am) * fact(l));
    for (int t = 0; t <= (l - am) / 2; ++t)
      for (int u = 0; u <= t; ++u) {
        const int vmax2 = 2 * ((am - vm2) / 2) + vm2;
        for (int tv = vm2; tv <= vmax2; tv += 2) {
          const double sign = ((t + (tv - vm2) / 2) % 2) ? -1.0 : 1.0;
          const double c = sign * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                           binom(t, u) * binom(am, tv);
          // the z power is l - px - py = l - 2t - am
          const int py = 2 * u + tv, px = 2 * t + am - 2 * u - tv;
          out[comp_index(l, px, py) * ns + col] += c * nrm;
        }
      }
  }
  const double scale = std::sqrt((2 * l + 1) / (4.0 * M_PI));
  for (double& v : out) v *= scale;
}

// Laplacian of every column polynomial must vanish (harmonic components).
static bool harmonic(int l, const double* blk, int ns) {
  if (l <= 1) return true;
  double big = 0.0;
  for (int i = 0; i < ncart(l) * ns; ++i) big = std::max(big, std::fabs(blk[i]));
  const int nlow = ncart(l - 2);
  for (int col = 0; col < ns; ++col) {
    std::vector<double> lap(nlow, 0.0);
    for (int lx = l; lx >= 0; --lx)
      for (int ly = l - lx; ly >= 0; --ly) {
        const int lz = l - lx - ly;
        const double c = blk[comp_index(l, lx, ly) * ns + col];
        if (c == 0.0) continue;
        if (lx >= 2) lap[comp_index(l - 2, lx - 2, ly)] += c * lx * (lx - 1);
        if (ly >= 2) lap[comp_index(l - 2, lx, ly - 2)] += c * ly * (ly - 1);
        if (lz >= 2) lap[comp_index(l - 2, lx, ly)] += c * lz * (lz - 1);
      }
    for (double v : lap)
      if (std::fabs(v) > 1e-9 * std::max(big, 1.0)) return false;
  }
  return true;
}

// Shells from static metadata (dftax/integrals/eri3c_bucketed.py:119-137):
// a shell starts where the component sequence restarts at (l, 0, 0).
static void parse_basis(const dfjk_basis* b, const char* what, int lmax_supported,
                        bool need_harmonic, Shells& sh, Blocks& blk) {
  if (!b || !b->centers || !b->exponents || !b->coefficients || !b->angular)
    fail(DFJK_ERR_INVALID, "%s basis: null array", what);
  if (b->ncart <= 0 || b->max_prim <= 0)
    fail(DFJK_ERR_INVALID, "%s basis: ncart=%lld max_prim=%d", what, (long long)b->ncart, b->max_prim);
  const int64_t n = b->ncart;
  const int mp = b->max_prim;
  for (int64_t i = 0; i < n * 3; ++i)
    if (!std::isfinite(b->centers[i])) fail(DFJK_ERR_NUMERIC, "%s basis: non-finite center", what);
  for (int64_t i = 0; i < n * mp; ++i)
    if (!std::isfinite(b->exponents[i]) || !std::isfinite(b->coefficients[i]))
      fail(DFJK_ERR_NUMERIC, "%s basis: non-finite exponent or coefficient", what);
  std::vector<int64_t> starts;
  for (int64_t i = 0; i < n; ++i) {
    const int* a = b->angular + 3 * i;
    if (a[0] < 0 || a[1] < 0 || a[2] < 0) fail(DFJK_ERR_INVALID, "%s basis: negative power", what);
    const int l = a[0] + a[1] + a[2];
    if (a[0] == l && a[1] == 0 && a[2] == 0) starts.push_back(i);
  }
  if (starts.empty() || starts[0] != 0)
    fail(DFJK_ERR_INVALID, "%s basis rows do not start shells at (l,0,0)", what);
  starts.push_back(n);
  sh.reset();
  sh.n = (int)starts.size() - 1;
  sh.spherical = b->cart2sph != nullptr;
  int out = 0;
  for (int s = 0; s < sh.n; ++s) {
    const int64_t r0 = starts[s], r1 = starts[s + 1];
    const int* a0 = b->angular + 3 * r0;
    const int l = a0[0] + a0[1] + a0[2];
    if (l > lmax_supported)
      fail(DFJK_ERR_UNSUPPORTED, "%s basis: angular momentum l=%d exceeds the compiled l<=%d",
           what, l, lmax_supported);
    if (r1 - r0 != ncart(l))
      fail(DFJK_ERR_INVALID, "%s basis: shell at row %lld has %lld rows, expected %d", what,
           (long long)r0, (long long)(r1 - r0), ncart(l));
    // canonical component order and uniform per-shell data
    for (int k = 0; k < ncart(l); ++k) {
      const int* ak = b->angular + 3 * (r0 + k);
      int lx = l, kk = k;
      while (kk > l - lx) { kk -= (l - lx + 1); --lx; }
      const int ly = (l - lx) - kk;
      if (ak[0] != lx || ak[1] != ly || ak[2] != l - lx - ly)
        fail(DFJK_ERR_INVALID, "%s basis: shell at row %lld is not in (lx desc, ly desc) order",
             what, (long long)r0);
      for (int d = 0; d < 3; ++d)
        if (b->centers[3 * (r0 + k) + d] != b->centers[3 * r0 + d])
          fail(DFJK_ERR_INVALID, "%s basis: components of one shell on different centers", what);
      for (int q = 0; q < mp; ++q) {
        if (b->exponents[(r0 + k) * mp + q] != b->exponents[r0 * mp + q])
          fail(DFJK_ERR_INVALID, "%s basis: components of one shell with different exponents", what);
        const double c0 = b->coefficients[r0 * mp + q], ck = b->coefficients[(r0 + k) * mp + q];
        if (std::fabs(ck - c0) > 1e-13 * std::fabs(c0))
          fail(DFJK_ERR_UNSUPPORTED,
               "%s basis: per-component coefficients differ within the shell at row %lld", what,
               (long long)r0);
      }
    }
    int np = 0;
    for (int q = 0; q < mp; ++q)
      if (b->exponents[r0 * mp + q] != 0.0) ++np;
    if (np == 0) fail(DFJK_ERR_INVALID, "%s basis: shell at row %lld has no primitive", what, (long long)r0);
    sh.l.push_back(l);
    sh.nprim.push_back(np);
    sh.prim0.push_back((int)sh.pexp.size());
    sh.row0.push_back((int)r0);
    sh.ncomp.push_back(ncart(l));
    sh.out0.push_back(out);
    out += sh.spherical ? 2 * l + 1 : ncart(l);
    for (int d = 0; d < 3; ++d) sh.cen.push_back(b->centers[3 * r0 + d]);
    for (int q = 0; q < mp; ++q)
      if (b->exponents[r0 * mp + q] != 0.0) {
        if (!(b->exponents[r0 * mp + q] > 0.0))
          fail(DFJK_ERR_INVALID, "%s basis: non-positive exponent", what);
        sh.pexp.push_back(b->exponents[r0 * mp + q]);
        sh.pcoef.push_back(b->coefficients[r0 * mp + q]);
      }
    sh.lmax = std::max(sh.lmax, l);
  }
  sh.ncart = (int)n;
  sh.nout = out;
  // transformation blocks (eri3c_bucketed.py:186-218): block diagonal, one per l
  blk.reset();
  int off = 0;
  std::vector<int> have(8, 0);
  for (int l = 0; l <= 7; ++l) blk.off[l] = 0;
  std::vector<std::vector<double>> per_l(8);
  if (!sh.spherical) {
    if (sh.lmax >= 2)
      fail(DFJK_ERR_UNSUPPORTED, "%s basis: cartesian shells with l>=2 are not supported "
           "(pass cart2sph)", what);
    for (int l = 0; l <= sh.lmax; ++l) standard_block(l, per_l[l]);
  } else {
    if (b->nsph <= 0) fail(DFJK_ERR_INVALID, "%s basis: nsph=%d with cart2sph", what, b->nsph);
    if (b->nsph != sh.nout)
      fail(DFJK_ERR_INVALID, "%s basis: cart2sph has %d columns, shells need %d", what, b->nsph, sh.nout);
    const double* C = b->cart2sph;
    const int ns = b->nsph;
    // sum |C| over each shell's rows, read by several host threads (the
    // auxiliary matrix is hundreds of MB); four partial sums per row
    std::vector<double> row_abs(sh.n, 0.0);
    auto scan = [&](int sa, int sb) {
      for (int s = sa; s < sb; ++s) {
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = 0; i < ncart(sh.l[s]); ++i) {
          const double* r = C + (int64_t)(sh.row0[s] + i) * ns;
          int j = 0;
          for (; j + 4 <= ns; j += 4)
            for (int u = 0; u < 4; ++u) acc[u] += std::fabs(r[j + u]);
          for (; j < ns; ++j) acc[0] += std::fabs(r[j]);
        }
        row_abs[s] = (acc[0] + acc[1]) + (acc[2] + acc[3]);
      }
    };
    const int64_t cells = (int64_t)sh.ncart * ns;
    const int nth = cells > (1 << 22)
                        ? (int)std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()))
                        : 1;
    run_on_threads(nth, [&](int t) {
      scan((int)((int64_t)sh.n * t / nth), (int)((int64_t)sh.n * (t + 1) / nth));
    });
    for (int s = 0; s < sh.n; ++s) {
      const int l = sh.l[s], nc = ncart(l), no = 2 * l + 1, r0 = sh.row0[s], c0 = sh.out0[s];
      const double rows = row_abs[s];
      double inb = 0.0;
      std::vector<double> blkv((size_t)nc * no);
      for (int i = 0; i < nc; ++i) {
        for (int j = 0; j < no; ++j) {
          const double v = C[(int64_t)(r0 + i) * ns + c0 + j];
          blkv[i * no + j] = v;
          inb += std::fabs(v);
        }
      }
      if (std::fabs(rows - inb) > 1e-12 * std::max(1.0, rows))
        fail(DFJK_ERR_INVALID, "%s cart2sph is not block diagonal over shells (shell l=%d at row %d)",
             what, l, r0);
      if (have[l]) {
        for (size_t q = 0; q < blkv.size(); ++q)
          if (blkv[q] != per_l[l][q])
            fail(DFJK_ERR_INVALID, "%s cart2sph blocks differ between shells of l=%d", what, l);
      } else {
        per_l[l] = blkv;
        have[l] = 1;
        if (need_harmonic && !harmonic(l, blkv.data(), no))
          fail(DFJK_ERR_UNSUPPORTED, "%s cart2sph block for l=%d is not harmonic", what, l);
      }
    }
  }
  for (int l = 0; l <= sh.lmax; ++l) {
    blk.off[l] = off;
    if (per_l[l].empty()) standard_block(l, per_l[l]);
    blk.host.insert(blk.host.end(), per_l[l].begin(), per_l[l].end());
    off += (int)per_l[l].size();
  }
  upload(blk.dev, blk.host);
  upload(sh.d_l, sh.l);
  upload(sh.d_nprim, sh.nprim);
  upload(sh.d_prim0, sh.prim0);
  upload(sh.d_cen, sh.cen);
  upload(sh.d_pexp, sh.pexp);
  upload(sh.d_pcoef, sh.pcoef);
}

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------

// host threads for the plan tables (0 .. nth-1 each take [n t / nth, n (t+1) / nth))
static int table_threads(int64_t n, int64_t min_chunk) {
  const int64_t hw = std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
  return (int)std::max<int64_t>(1, std::min<int64_t>(hw, n / min_chunk));
}

template <class F>
static void for_ranges(int nth, int64_t n, F f) {
  if (nth <= 1) {
    f(0, (int64_t)0, n);
    return;
  }
  run_on_threads(nth, [&](int t) { f(t, n * t / nth, n * (t + 1) / nth); });
}

static void make_orbital_tables(Plan& p);
void compute_metric_factor(Plan& p, cudaStream_t s);

static void make_plan(Plan& p, const dfjk_basis* orb, const dfjk_basis* aux) {
  parse_basis(orb, "orbital", kLmaxOrb, false, p.orb, p.c2s_orb);
  parse_basis(aux, "auxiliary", kLmaxAux, true, p.aux, p.c2s_aux);
  p.nao = p.orb.nout;
  p.naux = p.aux.nout;
  // aux columns: shells sorted by l (stable), column runs per l
  p.aux_order.resize(p.aux.n);
  std::iota(p.aux_order.begin(), p.aux_order.end(), 0);
  std::stable_sort(p.aux_order.begin(), p.aux_order.end(),
                   [&](int x, int y) { return p.aux.l[x] < p.aux.l[y]; });
  p.aux_col0.assign(p.aux.n, 0);
  p.aux_perm.assign(p.naux, 0);
  for (int l = 0; l < 8; ++l) { p.aux_lbegin[l] = 0; p.aux_lcount[l] = 0; }
  int col = 0;
  for (int pos = 0; pos < p.aux.n; ++pos) {
    const int s = p.aux_order[pos], l = p.aux.l[s];
    if (p.aux_lcount[l] == 0) p.aux_lbegin[l] = pos;
    p.aux_lcount[l]++;
    p.aux_col0[s] = col;
    for (int k = 0; k < 2 * l + 1; ++k) p.aux_perm[col + k] = p.aux.out0[s] + k;
    col += 2 * l + 1;
  }
  upload(p.d_aux_sorted, p.aux_order);
  upload(p.d_aux_perm, p.aux_perm);
  // The metric and its factor need only the auxiliary tables: a host thread
  // computes them on a stream of its own while this thread builds the
  // orbital pair tables, and the plan's first build uses them. (The metric
  // reads its eigenvalues back, so it cannot simply be queued.)
  const int dev = p.ctx->device;
  std::exception_ptr metric_err;
  std::thread metric([&] {
    cudaStream_t ms = nullptr;
    try {
      DFJK_CUDA(cudaSetDevice(dev));
      DFJK_CUDA(cudaStreamCreateWithFlags(&ms, cudaStreamNonBlocking));
      p.timer.reset(kPhMetric);
      p.timer.mark(kPhMetric, ms);
      compute_metric_factor(p, ms);
      p.timer.mark(kPhMetric, ms);
      DFJK_CUDA(cudaStreamSynchronize(ms));
      p.metric_ready = true;
    } catch (...) {
      metric_err = std::current_exception();
    }
    if (ms) {
      cudaStreamSynchronize(ms);
      cudaStreamDestroy(ms);
    }
  });
  try {
    make_orbital_tables(p);
  } catch (...) {
    metric.join();
    throw;
  }
  metric.join();
  if (metric_err) std::rethrow_exception(metric_err);
}

// bra shell pairs, class buckets, row and K-list tables of the orbital basis
static void make_orbital_tables(Plan& p) {
  const int ns = p.orb.n;
  // bra shell pairs ia <= ib, optionally Schwarz screened
  std::vector<int> pa, pb;
  for (int i = 0; i < ns; ++i)
    for (int j = i; j < ns; ++j) {
      pa.push_back(i);
      pb.push_back(j);
    }
  if (p.opts.screen > 0.0) {
    std::vector<double> q;
    launch_schwarz(*p.ctx, p.orb, pa, pb, q);
    double qmax = 0.0;
    for (double v : q) qmax = std::max(qmax, v);
    std::vector<int> ka, kb;
    for (size_t i = 0; i < q.size(); ++i)
      if (q[i] >= p.opts.screen * qmax) {
        ka.push_back(pa[i]);
        kb.push_back(pb[i]);
      }
    pa.swap(ka);
    pb.swap(kb);
  }
  // canonical orientation (larger l first) and class buckets
  struct PR { int l1, l2, s1, s2, a, b; };
  // stable order by (l1, l2): a counting sort over the 64 keys l1 * 8 + l2
  std::vector<PR> prs(pa.size());
  {
    std::vector<int64_t> start(65, 0);
    for (size_t i = 0; i < pa.size(); ++i) {
      const int la = p.orb.l[pa[i]], lb = p.orb.l[pb[i]];
      start[1 + std::max(la, lb) * 8 + std::min(la, lb)]++;
    }
    for (int k = 0; k < 64; ++k) start[k + 1] += start[k];
    for (size_t i = 0; i < pa.size(); ++i) {
      int a = pa[i], b = pb[i], s1 = a, s2 = b;
      if (p.orb.l[a] < p.orb.l[b]) std::swap(s1, s2);
      const int l1 = p.orb.l[s1], l2 = p.orb.l[s2];
      prs[start[l1 * 8 + l2]++] = {l1, l2, s1, s2, a, b};
    }
  }
  p.classes.clear();
  const size_t npair = prs.size();
  p.pair_s1.resize(npair); p.pair_s2.resize(npair); p.pair_orig_a.resize(npair);
  p.pair_orig_b.resize(npair); p.pair_row0.resize(npair); p.pair_pp0.resize(npair);
  p.pair_npp.resize(npair);
  int64_t row = 0, pp = 0, esph = 0;
  for (size_t i = 0; i < npair; ++i) {
    const PR& r = prs[i];
    if (p.classes.empty() || p.classes.back().l1 != r.l1 || p.classes.back().l2 != r.l2) {
      ClassRange c{r.l1, r.l2, (int64_t)i, 0, pp, 0, esph};
      p.classes.push_back(c);
    }
    ClassRange& c = p.classes.back();
    c.count++;
    p.pair_s1[i] = r.s1;
    p.pair_s2[i] = r.s2;
    p.pair_orig_a[i] = r.a;
    p.pair_orig_b[i] = r.b;
    p.pair_row0[i] = row;
    p.pair_pp0[i] = pp;
    const int n1 = p.orb.nprim[r.s1], n2 = p.orb.nprim[r.s2];
    p.pair_npp[i] = n1 * n2;
    pp += n1 * n2;
    c.pp_count += n1 * n2;
    const int na = 2 * r.l1 + 1, nb = 2 * r.l2 + 1;
    const int nh = (r.l1 + r.l2 + 1) * (r.l1 + r.l2 + 2) * (r.l1 + r.l2 + 3) / 6;
    esph += (int64_t)n1 * n2 * na * nb * nh;
    row += na * nb;
  }
  p.nrows = row;
  p.npp = pp;
  p.esph_doubles = esph;
  // primitive pairs -> (pair, x, y) and rows -> (m, n), kinds: each range of
  // pairs fills its own slices, in parallel
  std::vector<int> pp_pair(pp), pp_pa(pp), pp_pb(pp);
  std::vector<int> rm(row), rn(row);
  std::vector<int8_t> kind(row);
  for_ranges(table_threads((int64_t)npair, 4096), (int64_t)npair, [&](int, int64_t i0, int64_t i1) {
    for (int64_t i = i0; i < i1; ++i) {
      const int s1 = p.pair_s1[i], s2 = p.pair_s2[i];
      const int n1 = p.orb.nprim[s1], n2 = p.orb.nprim[s2];
      int64_t k = p.pair_pp0[i];
      for (int x = 0; x < n1; ++x)
        for (int y = 0; y < n2; ++y, ++k) {
          pp_pair[k] = (int)i;
          pp_pa[k] = x;
          pp_pb[k] = y;
        }
      const int na = 2 * p.orb.l[s1] + 1, nb = 2 * p.orb.l[s2] + 1;
      for (int x = 0; x < na; ++x)
        for (int y = 0; y < nb; ++y) {
          const int64_t r = p.pair_row0[i] + x * nb + y;
          const int m = p.orb.out0[s1] + x, n = p.orb.out0[s2] + y;
          rm[r] = m;
          rn[r] = n;
          kind[r] = (s1 == s2) ? (m >= n ? 1 : 0) : 2;
        }
    }
  });
  // K lists: per m, the rows that touch m in ascending row order (a counting
  // sort over row ranges; each range's histogram places its entries after
  // those of the ranges before it, so the order is the sequential one)
  const int nth = table_threads(row, 65536);
  std::vector<std::vector<int>> hist(nth, std::vector<int>(p.nao, 0));
  for_ranges(nth, row, [&](int t, int64_t r0, int64_t r1) {
    std::vector<int>& h = hist[t];
    for (int64_t r = r0; r < r1; ++r) {
      h[rm[r]]++;
      if (kind[r] == 2) h[rn[r]]++;
    }
  });
  std::vector<int> cnt(p.nao + 1, 0);
  for (int m = 0; m < p.nao; ++m) {
    int acc = 0;
    for (int t = 0; t < nth; ++t) {
      const int h = hist[t][m];
      hist[t][m] = acc;   // offset of range t within m's list
      acc += h;
    }
    cnt[m + 1] = cnt[m] + acc;
  }
  std::vector<int> krow(cnt[p.nao]), kn(cnt[p.nao]);
  for_ranges(nth, row, [&](int t, int64_t r0, int64_t r1) {
    std::vector<int> fill(p.nao);
    for (int m = 0; m < p.nao; ++m) fill[m] = cnt[m] + hist[t][m];
    for (int64_t r = r0; r < r1; ++r) {
      krow[fill[rm[r]]] = (int)r;
      kn[fill[rm[r]]++] = rn[r];
      if (kind[r] == 2) {
        krow[fill[rn[r]]] = (int)r;
        kn[fill[rn[r]]++] = rm[r];
      }
    }
  });
  // upload
  upload(p.d_pair_s1, p.pair_s1);
  upload(p.d_pair_s2, p.pair_s2);
  upload(p.d_pair_row0, p.pair_row0);
  upload(p.d_pair_pp0, p.pair_pp0);
  upload(p.d_pair_npp, p.pair_npp);
  upload(p.d_pp_pair, pp_pair);
  upload(p.d_pp_pa, pp_pa);
  upload(p.d_pp_pb, pp_pb);
  p.d_pp_P.alloc(std::max<int64_t>(pp, 1) * 3 * sizeof(double));
  p.d_pp_g.alloc(std::max<int64_t>(pp, 1) * sizeof(double));
  p.d_pp_pref.alloc(std::max<int64_t>(pp, 1) * sizeof(double));
  p.d_esph.alloc(std::max<int64_t>(esph, 1) * sizeof(double));
  upload(p.d_row_m, rm);
  upload(p.d_row_n, rn);
  upload(p.d_row_w, kind);
  upload(p.d_kptr, cnt);
  upload(p.d_krow, krow);
  upload(p.d_kn, kn);
  // the uploads (legacy stream) are complete before any stream of the caller
  // uses the tables; the metric's own stream is not waited for here
  DFJK_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
}

// ---------------------------------------------------------------------------
// Build: metric factor, primitive pairs, 3-center rows, B
// ---------------------------------------------------------------------------

__global__ void scale_factor_kernel(const double* __restrict__ U, const double* __restrict__ w,
                                    int64_t naux, int64_t k0, int64_t nfit, int64_t ldb,
                                    double* __restrict__ L) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= naux * ldb) return;
  const int64_t col = i / naux, r = i % naux;
  L[i] = col < nfit ? U[(k0 + col) * naux + r] / sqrt(w[k0 + col]) : 0.0;
}

__global__ void finite_check_kernel(const double* __restrict__ x, int64_t n, int* __restrict__ bad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && !isfinite(x[i])) atomicExch(bad, 1);
}

void check_finite(Plan& p, const double* x, int64_t n, cudaStream_t s, const char* what) {
  DevBuf& flag = p.ws_flag;
  flag.ensure(sizeof(int));
  DFJK_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
  if (n > 0) {
    finite_check_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, n, flag.as<int>());
    DFJK_LAUNCHED();
  }
  int h = 0;
  DFJK_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (h) fail(DFJK_ERR_NUMERIC, "non-finite values in %s", what);
}

int64_t chunk_budget(const Plan& p) {
  return p.opts.chunk_bytes > 0 ? p.opts.chunk_bytes : (int64_t)2 << 30;
}

void compute_metric_factor(Plan& p, cudaStream_t s) {
  Context& c = *p.ctx;
  const int64_t n = p.naux;
  p.d_metric.ensure((size_t)n * n * sizeof(double));
  DFJK_CUDA(cudaMemsetAsync(p.d_metric.p, 0, (size_t)n * n * sizeof(double), s));
  launch_eri2c(p, p.d_metric.as<double>(), n, s);
  check_finite(p, p.d_metric.as<double>(), n * n, s, "the (P|Q) metric");
  p.d_w.ensure(n * sizeof(double));
  DFJK_CUSOLVER(cusolverDnSetStream(c.cusolver, s));
  int lwork = 0;
  DFJK_CUSOLVER(cusolverDnDsyevd_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR,
                                            CUBLAS_FILL_MODE_LOWER, (int)n, p.d_metric.as<double>(),
                                            (int)n, p.d_w.as<double>(), &lwork));
  DevBuf& work = p.ws_syevd;
  DevBuf& info = p.ws_info;
  work.ensure((size_t)std::max(lwork, 1) * sizeof(double));
  info.ensure(sizeof(int));
  DFJK_CUSOLVER(cusolverDnDsyevd(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                 (int)n, p.d_metric.as<double>(), (int)n, p.d_w.as<double>(),
                                 work.as<double>(), lwork, info.as<int>()));
  int hinfo = 0;
  p.w_host.resize(n);
  DFJK_CUDA(cudaMemcpyAsync(&hinfo, info.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaMemcpyAsync(p.w_host.data(), p.d_w.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  DFJK_CUDA(cudaStreamSynchronize(s));
  if (hinfo != 0) fail(DFJK_ERR_NUMERIC, "metric eigensolver failed (info=%d)", hinfo);
  // keep w > cutoff * w_max (dftax/ks/terms.py:191); w ascending -> kept set is a suffix
  const double thr = p.opts.metric_cutoff * p.w_host[n - 1];
  int64_t k0 = 0;
  while (k0 < n && !(p.w_host[k0] > thr)) ++k0;
  p.k0 = k0;
  p.nfit = n - k0;
  if (p.nfit <= 0) fail(DFJK_ERR_NUMERIC, "metric has no eigenvalue above the cutoff");
  p.ldb = (p.nfit + 7) / 8 * 8;
  p.d_L.ensure((size_t)n * p.ldb * sizeof(double));
  const int64_t tot = n * p.ldb;
  scale_factor_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
      p.d_metric.as<double>(), p.d_w.as<double>(), n, k0, p.nfit, p.ldb, p.d_L.as<double>());
  DFJK_LAUNCHED();
}

// Pair chunks of at most `budget` bytes of raw rows (ld doubles each).
std::vector<std::pair<int64_t, int64_t>> pair_chunks(const Plan& p, int64_t ld, int64_t budget) {
  std::vector<std::pair<int64_t, int64_t>> out;
  const int64_t npair = (int64_t)p.pair_s1.size();
  const int64_t max_rows = std::max<int64_t>(budget / (ld * (int64_t)sizeof(double)), 49);
  int64_t b = 0;
  while (b < npair) {
    int64_t e = b;
    while (e < npair) {
      const int64_t end_row = (e + 1 < npair) ? p.pair_row0[e + 1] : p.nrows;
      if (end_row - p.pair_row0[b] > max_rows && e > b) break;
      ++e;
    }
    out.push_back({b, e});
    b = e;
  }
  return out;
}

int64_t rows_of(const Plan& p, int64_t b, int64_t e) {
  const int64_t npair = (int64_t)p.pair_s1.size();
  const int64_t end_row = e < npair ? p.pair_row0[e] : p.nrows;
  return end_row - p.pair_row0[b];
}

// Everything a build does before its 3-center rows: the metric factor, the
// primitive pairs, the workspaces and L's digit planes. Returns the pair
// chunks of the rows, or no chunks when the plan is streamed (built then).
static std::vector<std::pair<int64_t, int64_t>> build_begin(Plan& p, cudaStream_t s) {
  p.built = 0;
  // the first build of a plan uses the metric factor computed while the plan
  // was created (same code and inputs); every later build recomputes it
  const bool have_metric = p.metric_ready;
  p.metric_ready = false;
  for (int ph = kPhMetric; ph <= kPhBgemm; ++ph)
    if (ph != kPhMetric || !have_metric) p.timer.reset(ph);
  p.timer.reset(kPhKplanes);
  // The eigensolver keeps the whole device busy: running the 3-center rows
  // beside it on a second stream (at either priority) was measured to save
  // under 3% of a (H2O)_32 build while holding the whole tensor, so the
  // phases run in order on s.
  if (!have_metric) {
    p.timer.mark(kPhMetric, s);
    compute_metric_factor(p, s);
    p.timer.mark(kPhMetric, s);
  }
  p.timer.mark(kPhPairs, s);
  launch_pair_setup(p, s);
  p.timer.mark(kPhPairs, s);
  const int64_t ld = p.naux;
  const int64_t kp = (p.naux + 15) / 16 * 16;
  auto chunks = pair_chunks(p, ld, chunk_budget(p));
  int64_t maxrows = 1;
  for (auto& ch : chunks) maxrows = std::max(maxrows, rows_of(p, ch.first, ch.second));
  DevBuf& raw = p.ws_raw;
  raw.ensure((size_t)maxrows * ld * sizeof(double));
  // B = (ij|P) L on the int8 tensor cores with exact accumulation: 5 digits
  // per value in mixed precision, 7 (2^-56 of each row's scale, below
  // float64's own rounding of the row maximum) for float64 plans
  ozaki_prepare_l(p, s);
  p.ws_oz_raw.ensure((size_t)build_digits(p) * maxrows * kp);
  p.ws_oz_er.ensure((size_t)maxrows * sizeof(int));
  if (p.opts.streamed) {
    // B is rebuilt chunk by chunk by every J/K call (for_each_b_chunk)
    p.d_B.free();
    p.ws_bchunk.ensure((size_t)maxrows * p.ldb * sizeof(double));
    ozaki_check(p, s);
    p.built = 1;
    return {};
  }
  p.d_B.ensure((size_t)std::max<int64_t>(p.nrows, 1) * p.ldb * sizeof(double));
  return chunks;
}

// B[r0 : r0 + nr] = raw (nr x naux, in ws_raw) . L on the int8 tensor cores
static void build_product(Plan& p, int64_t r0, int64_t nr, cudaStream_t s) {
  const int64_t kp = (p.naux + 15) / 16 * 16;
  p.timer.mark(kPhBgemm, s);
  ozaki_split_raw(p, p.ws_raw.as<double>(), nr, p.ws_oz_raw.as<int8_t>(), nr * kp,
                  p.ws_oz_er.as<int>(), s);
  ozaki_bgemm(p, p.ws_oz_raw.as<int8_t>(), nr * kp, p.ws_oz_er.as<int>(), nr,
              p.d_B.as<double>() + r0 * p.ldb, s);
  p.timer.mark(kPhBgemm, s);
}

// after the last chunk: the checks and, in mixed precision, the K planes
static void build_end(Plan& p, cudaStream_t s) {
  // the digit splits flagged any non-finite input (a NaN's digits are
  // finite); float64 plans also scan B for an overflow in the product
  ozaki_check(p, s);
  const bool mixed = p.opts.precision == DFJK_MIXED;
  if (!mixed) check_finite(p, p.d_B.as<double>(), p.nrows * p.ldb, s, "B");
  if (mixed) {
    p.timer.mark(kPhKplanes, s);
    build_ozaki_planes(p, s);
    p.timer.mark(kPhKplanes, s);
  }
  p.built = 1;
}

void build(Plan& p, cudaStream_t s) {
  auto chunks = build_begin(p, s);
  if (p.built) return;   // streamed
  for (auto& ch : chunks) {
    const int64_t r0 = p.pair_row0[ch.first], nr = rows_of(p, ch.first, ch.second);
    p.timer.mark(kPhEri3c, s);
    launch_eri3c_rows(p, ch.first, ch.second, r0, p.ws_raw.p, p.naux, false, s);
    p.timer.mark(kPhEri3c, s);
    build_product(p, r0, nr, s);
  }
  build_end(p, s);
}

void build_batch(const std::vector<Plan*>& ps, cudaStream_t s) {
  // plans whose rows fit in one chunk share the 3-center launches; the
  // others (and streamed plans) are built alone
  std::vector<Plan*> together;
  for (Plan* p : ps) {
    if (p->opts.streamed || pair_chunks(*p, p->naux, chunk_budget(*p)).size() > 1) {
      build(*p, s);
      continue;
    }
    build_begin(*p, s);
    together.push_back(p);
  }
  launch_eri3c_rows_batch(together, s);
  for (Plan* p : together) {
    build_product(*p, 0, p->nrows, s);
    build_end(*p, s);
  }
}

void for_each_b_chunk(Plan& p, cudaStream_t s,
                      const std::function<void(int64_t r0, int64_t nr, const double* Bc)>& fn) {
  const int64_t kp = (p.naux + 15) / 16 * 16;
  auto chunks = pair_chunks(p, p.naux, chunk_budget(p));
  for (auto& ch : chunks) {
    const int64_t r0 = p.pair_row0[ch.first], nr = rows_of(p, ch.first, ch.second);
    launch_eri3c_rows(p, ch.first, ch.second, r0, p.ws_raw.p, p.naux, false, s);
    ozaki_split_raw(p, p.ws_raw.as<double>(), nr, p.ws_oz_raw.as<int8_t>(), nr * kp,
                    p.ws_oz_er.as<int>(), s);
    ozaki_bgemm(p, p.ws_oz_raw.as<int8_t>(), nr * kp, p.ws_oz_er.as<int>(), nr,
                p.ws_bchunk.as<double>(), s);
    fn(r0, nr, p.ws_bchunk.as<double>());
  }
  ozaki_check(p, s);
}

// ---------------------------------------------------------------------------
// Diagnostics: dense tensors in dftax's order
// ---------------------------------------------------------------------------

__global__ void scatter_dense3_kernel(const double* __restrict__ raw, int64_t nrows, int64_t naux,
                                      int64_t row_base, const int* __restrict__ rm,
                                      const int* __restrict__ rn, const int8_t* __restrict__ kind,
                                      const int* __restrict__ perm, int64_t nao,
                                      double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nrows * naux) return;
  const int64_t r = i / naux, col = i % naux;
  const int64_t gr = r + row_base;
  const int m = rm[gr], n = rn[gr];
  const double v = raw[i];
  const int P = perm[col];
  out[((int64_t)m * nao + n) * naux + P] = v;
  if (kind[gr] == 2) out[((int64_t)n * nao + m) * naux + P] = v;
}

__global__ void unpermute2_kernel(const double* __restrict__ in, int64_t n,
                                  const int* __restrict__ perm, double* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * n) return;
  const int64_t r = i / n, c = i % n;
  out[(int64_t)perm[r] * n + perm[c]] = in[i];
}

void eri3c_dense(Plan& p, double* out, cudaStream_t s) {
  const int64_t nao = p.nao, naux = p.naux;
  DFJK_CUDA(cudaMemsetAsync(out, 0, (size_t)nao * nao * naux * sizeof(double), s));
  launch_pair_setup(p, s);
  auto chunks = pair_chunks(p, naux, chunk_budget(p));
  int64_t maxrows = 1;
  for (auto& ch : chunks) maxrows = std::max(maxrows, rows_of(p, ch.first, ch.second));
  DevBuf raw;
  raw.alloc((size_t)maxrows * naux * sizeof(double));
  for (auto& ch : chunks) {
    const int64_t r0 = p.pair_row0[ch.first], nr = rows_of(p, ch.first, ch.second);
    launch_eri3c_rows(p, ch.first, ch.second, r0, raw.p, naux, false, s);
    const int64_t tot = nr * naux;
    scatter_dense3_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
        raw.as<double>(), nr, naux, r0, p.d_row_m.as<int>(), p.d_row_n.as<int>(),
        p.d_row_w.as<int8_t>(), p.d_aux_perm.as<int>(), nao, out);
    DFJK_LAUNCHED();
  }
  DFJK_CUDA(cudaStreamSynchronize(s));
}

void eri2c_dense(Plan& p, double* out, cudaStream_t s) {
  const int64_t n = p.naux;
  DevBuf v;
  v.alloc((size_t)n * n * sizeof(double));
  DFJK_CUDA(cudaMemsetAsync(v.p, 0, (size_t)n * n * sizeof(double), s));
  launch_eri2c(p, v.as<double>(), n, s);
  unpermute2_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(v.as<double>(), n,
                                                                     p.d_aux_perm.as<int>(), out);
  DFJK_LAUNCHED();
  DFJK_CUDA(cudaStreamSynchronize(s));
}

void metric_pinv(Plan& p, double* out, cudaStream_t s) {
  if (!p.built) fail(DFJK_ERR_STATE, "metric_pinv before dfjk_build");
  Context& c = *p.ctx;
  const int64_t n = p.naux;
  DevBuf v;
  v.alloc((size_t)n * n * sizeof(double));
  DFJK_CUBLAS(cublasSetStream(c.cublas, s));
  const double one = 1.0, zero = 0.0;
  // V+ = L L^T (column-major L: naux x ldb)
  DFJK_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)n, (int)n, (int)p.ldb, &one,
                          p.d_L.as<double>(), (int)n, p.d_L.as<double>(), (int)n, &zero,
                          v.as<double>(), (int)n));
  unpermute2_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, s>>>(v.as<double>(), n,
                                                                     p.d_aux_perm.as<int>(), out);
  DFJK_LAUNCHED();
  DFJK_CUDA(cudaStreamSynchronize(s));
}

double energy(Plan& p, const double* P, int nspin, double hf, double hf_lr, double* F,
              cudaStream_t s);

}  // namespace dfjk

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

using namespace dfjk;

static cudaStream_t st(void* s) { return static_cast<cudaStream_t>(s); }

extern "C" {

void dfjk_default_options(dfjk_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->screen = 0.0;
  o->metric_cutoff = 1e-7;
  o->precision = DFJK_FP64;
  o->chunk_bytes = 0;
}

dfjk_status dfjk_create(int device, dfjk_ctx** out) {
  if (!out) return DFJK_ERR_INVALID;
  *out = nullptr;
  dfjk_ctx* h = new (std::nothrow) dfjk_ctx;
  if (!h) return DFJK_ERR_MEMORY;
  dfjk_status st_ = guard(nullptr, [&] {
    int n = 0;
    DFJK_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) fail(DFJK_ERR_INVALID, "device %d out of range (%d)", device, n);
    DFJK_CUDA(cudaSetDevice(device));
    h->c.device = device;
    DFJK_CUBLAS(cublasCreate(&h->c.cublas));
    DFJK_CUSOLVER(cusolverDnCreate(&h->c.cusolver));
    // the no-alloc J path's fixed scratch: its module is loaded (and the array
    // placed in device memory) here, not in that path's first call
    h->c.noalloc_scratch = noalloc_scratch_address();
    std::vector<double> tbl, asym;
    boys_table_host(tbl, asym);
    upload(h->c.boys, tbl);
    upload(h->c.boys_asym, asym);
  });
  if (st_ != DFJK_OK) {
    delete h;
    return st_;
  }
  *out = h;
  return DFJK_OK;
}

dfjk_status dfjk_destroy(dfjk_ctx* h) {
  if (!h) return DFJK_OK;
  cudaSetDevice(h->c.device);
  if (h->c.cublas) cublasDestroy(h->c.cublas);
  if (h->c.cusolver) cusolverDnDestroy(h->c.cusolver);
  for (int q = 0; q < dfjk::kXcBranches; ++q) {
    if (h->c.xc_blas[q]) cublasDestroy(h->c.xc_blas[q]);
    if (h->c.xc_done[q]) cudaEventDestroy(h->c.xc_done[q]);
    if (h->c.xc_stream[q]) cudaStreamDestroy(h->c.xc_stream[q]);
  }
  if (h->c.xc_fork) cudaEventDestroy(h->c.xc_fork);
  const int dev = h->c.device;
  {
    std::lock_guard<std::recursive_mutex> cap(dfjk::capture_mutex());
    cudaDeviceSynchronize();
  }
  delete h;
  dfjk::cache_trim(dev);
  return DFJK_OK;
}

const char* dfjk_last_error(const dfjk_ctx* h) { return h ? h->c.last_error.c_str() : "null context"; }

dfjk_status dfjk_plan_create(dfjk_ctx* h, const dfjk_basis* orb, const dfjk_basis* aux,
                             const dfjk_options* opts, dfjk_plan** out) {
  if (!h || !out) return DFJK_ERR_INVALID;
  *out = nullptr;
  dfjk_plan* pl = new (std::nothrow) dfjk_plan;
  if (!pl) return DFJK_ERR_MEMORY;
  dfjk_status r = guard(&h->c, [&] {
    DFJK_CUDA(cudaSetDevice(h->c.device));
    pl->p.ctx = &h->c;
    if (opts) pl->p.opts = *opts;
    else dfjk_default_options(&pl->p.opts);
    if (!(pl->p.opts.metric_cutoff >= 0.0) || !std::isfinite(pl->p.opts.screen))
      fail(DFJK_ERR_INVALID, "invalid options");
    if (pl->p.opts.precision != DFJK_FP64 && pl->p.opts.precision != DFJK_MIXED)
      fail(DFJK_ERR_INVALID, "unknown precision %d", pl->p.opts.precision);
    if (!(pl->p.opts.omega >= 0.0) || !std::isfinite(pl->p.opts.omega))
      fail(DFJK_ERR_INVALID, "omega must be finite and >= 0");
    if (pl->p.opts.streamed != 0 && pl->p.opts.streamed != 1)
      fail(DFJK_ERR_INVALID, "streamed must be 0 or 1");
    make_plan(pl->p, orb, aux);
    if (pl->p.opts.omega > 0.0) {
      // the long-range operator over the same bases; its Schwarz screen is the
      // same full-range one, so it keeps the same shell pairs
      dfjk_plan* lr = new dfjk_plan;
      pl->p.lr = lr;
      lr->p.ctx = &h->c;
      lr->p.opts = pl->p.opts;
      lr->p.atten = pl->p.opts.omega;
      lr->p.owned_by_parent = true;
      make_plan(lr->p, orb, aux);
    }
    // the int8 products are exact for dot products of at most kOzMaxK terms
    // (kOzMaxK7 for the 7-digit build product of float64 plans)
    if (pl->p.opts.precision == DFJK_MIXED &&
        (pl->p.naux > kOzMaxK || pl->p.nao > kOzMaxK))
      fail(DFJK_ERR_UNSUPPORTED, "mixed precision supports nao, naux <= %lld (got %d, %d)",
           (long long)kOzMaxK, pl->p.nao, pl->p.naux);
    if (pl->p.opts.precision == DFJK_FP64 && pl->p.naux > kOzMaxK7)
      fail(DFJK_ERR_UNSUPPORTED, "float64 plans support naux <= %lld (got %d)",
           (long long)kOzMaxK7, pl->p.naux);
  });
  if (r != DFJK_OK) {
    delete pl->p.lr;
    delete pl;
    return r;
  }
  *out = pl;
  return DFJK_OK;
}

dfjk_status dfjk_plan_destroy(dfjk_plan* pl) {
  if (!pl) return DFJK_OK;
  if (pl->p.owned_by_parent) return DFJK_ERR_INVALID;   // freed with its parent
  cudaSetDevice(pl->p.ctx->device);
  // the buffers go back to the cache without a device synchronization: work
  // still queued on them (on this or another stream) is waited for when a
  // buffer is handed out again, so solves on other streams keep running
  delete pl->p.lr;
  delete pl;
  return DFJK_OK;
}

dfjk_status dfjk_trim(dfjk_ctx* h) {
  if (!h) return DFJK_ERR_INVALID;
  cudaSetDevice(h->c.device);
  {
    std::lock_guard<std::recursive_mutex> cap(dfjk::capture_mutex());
    cudaDeviceSynchronize();
  }
  dfjk::cache_trim(h->c.device);
  return DFJK_OK;
}

dfjk_status dfjk_plan_get_info(const dfjk_plan* pl, dfjk_plan_info* info) {
  if (!pl || !info) return DFJK_ERR_INVALID;
  const Plan& p = pl->p;
  info->nao = p.nao;
  info->naux = p.naux;
  info->nao_cart = p.orb.ncart;
  info->naux_cart = p.aux.ncart;
  info->nshell = p.orb.n;
  info->naux_shell = p.aux.n;
  info->npair_shell = (int64_t)p.pair_s1.size();
  info->nrows = p.nrows;
  info->nfit = p.nfit;
  info->b_bytes = (int64_t)(p.d_B.bytes + p.d_oz_a.bytes);
  info->built = p.built;
  info->precision = p.opts.precision;
  return DFJK_OK;
}

dfjk_status dfjk_build_batch(dfjk_plan* const* plans, int32_t n, void* stream) {
  if (!plans || n < 0) return DFJK_ERR_INVALID;
  if (n == 0) return DFJK_OK;
  for (int32_t i = 0; i < n; ++i)
    if (!plans[i]) return DFJK_ERR_INVALID;
  Context* c = plans[0]->p.ctx;
  return guard(c, [&] {
    std::vector<Plan*> ps;
    for (int32_t i = 0; i < n; ++i) {
      if (plans[i]->p.ctx != c) fail(DFJK_ERR_INVALID, "plans of one batch need one context");
      if (plans[i]->p.lr) fail(DFJK_ERR_UNSUPPORTED, "batched builds take no long-range plans");
      for (int32_t k = 0; k < i; ++k)
        if (plans[k] == plans[i]) fail(DFJK_ERR_INVALID, "plan %d appears twice", i);
      ps.push_back(&plans[i]->p);
    }
    DFJK_CUDA(cudaSetDevice(c->device));
    build_batch(ps, st(stream));
  });
}

dfjk_status dfjk_build(dfjk_plan* pl, void* stream) {
  if (!pl) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    build(pl->p, st(stream));
    if (pl->p.lr) build(pl->p.lr->p, st(stream));
  });
}

dfjk_status dfjk_plan_long_range(const dfjk_plan* pl, dfjk_plan** lr) {
  if (!pl || !lr) return DFJK_ERR_INVALID;
  *lr = pl->p.lr;
  return pl->p.lr ? DFJK_OK : DFJK_ERR_STATE;
}

dfjk_status dfjk_jk(dfjk_plan* pl, const double* C, const double* w, int64_t ncol, double* J,
                    double* K, void* stream) {
  if (!pl) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    if (!pl->p.built) fail(DFJK_ERR_STATE, "dfjk_jk before dfjk_build");
    if (!C || ncol <= 0) fail(DFJK_ERR_INVALID, "C is null or ncol=%lld", (long long)ncol);
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    jk_compute(pl->p, C, w, ncol, J, K, st(stream));
  });
}

dfjk_status dfjk_jk_host(dfjk_plan* pl, const double* C, const double* w, int64_t ncol, double* J,
                         double* K, void* stream) {
  if (!pl) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    Plan& p = pl->p;
    if (!p.built) fail(DFJK_ERR_STATE, "dfjk_jk_host before dfjk_build");
    if (!C || ncol <= 0) fail(DFJK_ERR_INVALID, "C is null or ncol=%lld", (long long)ncol);
    DFJK_CUDA(cudaSetDevice(p.ctx->device));
    cudaStream_t s = st(stream);
    const size_t nc = (size_t)p.nao * ncol * sizeof(double), nn = (size_t)p.nao * p.nao * sizeof(double);
    DevBuf dC, dw, dJ, dK;
    dC.alloc(nc);
    DFJK_CUDA(cudaMemcpyAsync(dC.p, C, nc, cudaMemcpyHostToDevice, s));
    if (w) {
      dw.alloc(ncol * sizeof(double));
      DFJK_CUDA(cudaMemcpyAsync(dw.p, w, ncol * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    if (J) dJ.alloc(nn);
    if (K) dK.alloc(nn);
    jk_compute(p, dC.as<double>(), w ? dw.as<double>() : nullptr, ncol, J ? dJ.as<double>() : nullptr,
               K ? dK.as<double>() : nullptr, s);
    if (J) DFJK_CUDA(cudaMemcpyAsync(J, dJ.p, nn, cudaMemcpyDeviceToHost, s));
    if (K) DFJK_CUDA(cudaMemcpyAsync(K, dK.p, nn, cudaMemcpyDeviceToHost, s));
    DFJK_CUDA(cudaStreamSynchronize(s));
  });
}

dfjk_status dfjk_energy(dfjk_plan* pl, const double* P, int32_t nspin, double hf_coeff, double* e,
                        double* F, void* stream) {
  return dfjk_energy_rsh(pl, P, nspin, hf_coeff, 0.0, e, F, stream);
}

dfjk_status dfjk_energy_rsh(dfjk_plan* pl, const double* P, int32_t nspin, double hf_coeff,
                            double hf_coeff_lr, double* e, double* F, void* stream) {
  if (!pl) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    if (!pl->p.built) fail(DFJK_ERR_STATE, "dfjk_energy before dfjk_build");
    if (!P || !e || (nspin != 1 && nspin != 2)) fail(DFJK_ERR_INVALID, "bad energy arguments");
    if (!std::isfinite(hf_coeff) || !std::isfinite(hf_coeff_lr))
      fail(DFJK_ERR_INVALID, "non-finite exchange coefficient");
    if (hf_coeff_lr != 0.0 && !pl->p.lr)
      fail(DFJK_ERR_STATE, "hf_coeff_lr needs a plan made with omega > 0");
    if (hf_coeff_lr != 0.0 && !pl->p.lr->p.built)
      fail(DFJK_ERR_STATE, "the long-range plan is not built");
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    *e = energy(pl->p, P, nspin, hf_coeff, hf_coeff_lr, F, st(stream));
  });
}

dfjk_status dfjk_energy_grad(dfjk_plan* pl, const double* P, int32_t nspin, double hf_coeff,
                             double* e, double* grad_orb, double* grad_aux, void* stream) {
  if (!pl) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    if (!pl->p.built) fail(DFJK_ERR_STATE, "dfjk_energy_grad before dfjk_build");
    if (pl->p.opts.streamed)
      fail(DFJK_ERR_UNSUPPORTED, "dfjk_energy_grad needs B held in device memory (not streamed)");
    if (!P || !e || !grad_orb || !grad_aux || (nspin != 1 && nspin != 2))
      fail(DFJK_ERR_INVALID, "bad gradient arguments");
    if (!std::isfinite(hf_coeff)) fail(DFJK_ERR_INVALID, "non-finite exchange coefficient");
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    *e = energy_gradient(pl->p, P, nspin, hf_coeff, grad_orb, grad_aux, st(stream));
  });
}

dfjk_status dfjk_eri3c_dense(dfjk_plan* pl, double* out, void* stream) {
  if (!pl || !out) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    eri3c_dense(pl->p, out, st(stream));
  });
}

dfjk_status dfjk_eri2c_dense(dfjk_plan* pl, double* out, void* stream) {
  if (!pl || !out) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    eri2c_dense(pl->p, out, st(stream));
  });
}

dfjk_status dfjk_metric_pinv(dfjk_plan* pl, double* out, void* stream) {
  if (!pl || !out) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    DFJK_CUDA(cudaSetDevice(pl->p.ctx->device));
    metric_pinv(pl->p, out, st(stream));
  });
}

dfjk_status dfjk_phase_times(dfjk_plan* pl, double* ms, int32_t n) {
  if (!pl || !ms || n < 0) return DFJK_ERR_INVALID;
  return guard(pl->p.ctx, [&] {
    for (int i = 0; i < n && i < kPhCount; ++i) ms[i] = pl->p.timer.ms(i);
    for (int i = kPhCount; i < n; ++i) ms[i] = 0.0;
  });
}

int64_t dfjk_kernel_launches(void) { return g_launches.load(); }

dfjk_status dfjk_kept_pairs(const dfjk_plan* pl, int32_t* out) {
  if (!pl || !out) return DFJK_ERR_INVALID;
  const Plan& p = pl->p;
  // dftax order: sorted by (ia, ib)
  std::vector<std::pair<int, int>> v;
  for (size_t i = 0; i < p.pair_orig_a.size(); ++i) v.push_back({p.pair_orig_a[i], p.pair_orig_b[i]});
  std::sort(v.begin(), v.end());
  for (size_t i = 0; i < v.size(); ++i) {
    out[2 * i] = v[i].first;
    out[2 * i + 1] = v[i].second;
  }
  return DFJK_OK;
}

dfjk_status dfjk_boys(dfjk_ctx* h, const double* t, int64_t n, int32_t nmax, double* out, void* stream) {
  if (!h) return DFJK_ERR_INVALID;
  return guard(&h->c, [&] {
    if (!t || !out || n < 0 || nmax < 0 || nmax > 18) fail(DFJK_ERR_INVALID, "bad boys arguments");
    DFJK_CUDA(cudaSetDevice(h->c.device));
    launch_boys(h->c, t, n, nmax, out, st(stream));
  });
}

dfjk_status dfjk_wait_selftest(dfjk_ctx* h, int64_t limit_ns, double* waited_ms, void* stream) {
  if (!h) return DFJK_ERR_INVALID;
  return guard(&h->c, [&] {
    if (limit_ns < 1000 || limit_ns > 4000000000ll)
      fail(DFJK_ERR_INVALID, "wait limit %lld ns outside [1e3, 4e9]", (long long)limit_ns);
    DFJK_CUDA(cudaSetDevice(h->c.device));
    wait_selftest(h->c, limit_ns, waited_ms, st(stream));
  });
}

}  // extern "C"
