// Host side of the SRM path: uniform source, setup scalars and the harmonic
// sampler. Compiled without FMA contraction so that every single-precision
// operation rounds exactly as the reference's Fortran statement does.
#include "srm_host.h"

#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "srm_kernels.h"

namespace scarf {

// pi as the reference declares it (scarflib_common.f90:94): nearest float.
constexpr float kPi = 3.14159265358979323846f;

// ------------------------------------------------------------ Yarn2 source --
uint64_t Yarn2::mulmod(uint64_t a, uint64_t b) {
  // Mersenne reduction: for p < 2^62, p mod (2^31-1) by folding 31-bit digits.
  uint64_t p = a * b;
  p = (p & kMod) + (p >> 31);
  p = (p & kMod) + (p >> 31);
  return p >= kMod ? p - kMod : p;
}

namespace {
// g^r = g^(r & 0xFFFF) * (g^65536)^(r >> 16): two tables of exact residues.
struct PowTables {
  std::vector<uint32_t> lo, hi;
  PowTables() : lo(1u << 16), hi(1u << 15) {
    uint64_t v = 1;
    for (uint32_t k = 0; k < (1u << 16); ++k) {
      lo[k] = static_cast<uint32_t>(v);
      v = Yarn2::mulmod(v, Yarn2::kGen);
    }
    const uint64_t g16 = v;  // g^65536
    v = 1;
    for (uint32_t k = 0; k < (1u << 15); ++k) {
      hi[k] = static_cast<uint32_t>(v);
      v = Yarn2::mulmod(v, g16);
    }
  }
};
const PowTables& pow_tables() {
  static const PowTables t;
  return t;
}
}  // namespace

// The device's split of the same transform: g^k, g^(k 2^11), g^(k 2^22).
std::vector<uint32_t> device_pow_tables() {
  std::vector<uint32_t> w;
  w.reserve(2048 + 2048 + 512);
  uint64_t step = Yarn2::kGen;
  const int sizes[3] = {2048, 2048, 512};
  for (int part = 0; part < 3; ++part) {
    uint64_t v = 1;
    for (int k = 0; k < sizes[part]; ++k) {
      w.push_back(static_cast<uint32_t>(v));
      v = Yarn2::mulmod(v, step);
    }
    for (int b = 0; b < 11; ++b) step = Yarn2::mulmod(step, step);  // step^(2^11)
  }
  return w;
}

uint32_t Yarn2::output(uint64_t r) {
  if (r == 0) return 0u;
  const PowTables& t = pow_tables();
  return static_cast<uint32_t>(mulmod(t.lo[r & 0xFFFFu], t.hi[r >> 16]));
}

void Yarn2::seed(int s) {
  // prng.cpp:147 passes the int seed as unsigned long to yarn2::seed, whose
  // published rule reduces it, read as a signed 64-bit integer, into [0, m)
  // and sets the older state word to 1 (the state is never all-zero).
  int64_t t = static_cast<int64_t>(static_cast<unsigned long>(static_cast<long>(s)));
  t %= static_cast<int64_t>(kMod);
  if (t < 0) t += static_cast<int64_t>(kMod);
  r0 = static_cast<uint64_t>(t);
  r1 = 1;
}

uint32_t Yarn2::next_raw() {
  uint64_t t = mulmod(kA1, r0) + mulmod(kA2, r1);
  if (t >= kMod) t -= kMod;
  r1 = r0;
  r0 = t;
  return output(t);
}

void Yarn2::jump(uint64_t n) {
  // State transition (r0, r1) -> (a1 r0 + a2 r1, r0) as a 2x2 matrix power.
  uint64_t m00 = kA1, m01 = kA2, m10 = 1, m11 = 0;  // base matrix
  uint64_t p00 = 1, p01 = 0, p10 = 0, p11 = 1;      // accumulated power
  auto addm = [](uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    return s >= kMod ? s - kMod : s;
  };
  while (n) {
    if (n & 1) {
      const uint64_t q00 = addm(mulmod(p00, m00), mulmod(p01, m10));
      const uint64_t q01 = addm(mulmod(p00, m01), mulmod(p01, m11));
      const uint64_t q10 = addm(mulmod(p10, m00), mulmod(p11, m10));
      const uint64_t q11 = addm(mulmod(p10, m01), mulmod(p11, m11));
      p00 = q00, p01 = q01, p10 = q10, p11 = q11;
    }
    const uint64_t s00 = addm(mulmod(m00, m00), mulmod(m01, m10));
    const uint64_t s01 = addm(mulmod(m00, m01), mulmod(m01, m11));
    const uint64_t s10 = addm(mulmod(m10, m00), mulmod(m11, m10));
    const uint64_t s11 = addm(mulmod(m10, m01), mulmod(m11, m11));
    m00 = s00, m01 = s01, m10 = s10, m11 = s11;
    n >>= 1;
  }
  const uint64_t n0 = addm(mulmod(p00, r0), mulmod(p01, r1));
  const uint64_t n1 = addm(mulmod(p10, r0), mulmod(p11, r1));
  r0 = n0;
  r1 = n1;
}

// ------------------------------------------------------------- spectra -----
// psdf.f90:65 (von Karman) and :88 (Gaussian), evaluated in FP32.
static inline float psd_vk(float x, float nu) { return 1.0f / powf(1.0f + x * x, nu); }
static inline float psd_gs(float x) { return expf(-0.25f * (x * x)); }

double srm_fn(double x, int ndim, int acf, float nu) {
  const float xf = static_cast<float>(x);
  const float fv = (acf == 0) ? psd_vk(xf, nu) : psd_gs(xf);
  double r = x * static_cast<double>(fv);
  if (ndim == 3) r = r * x;
  return r;
}

// --------------------------------------------------------------- setup -----
int srm_setup(const scarf_srm_params& p, scarf_srm_setup* s) {
  std::memset(s, 0, sizeof(*s));
  if (p.acf != 0 && p.acf != 1) return SCARF_ERR_UNSUPPORTED;
  if (p.nharm <= 0) return SCARF_ERR_ARG;
  const int ndim = (p.cl[2] > 0.0f) ? 3 : 2;
  s->ndim = ndim;
  float span[3];
  for (int c = 0; c < 3; ++c) span[c] = p.fc[c] - p.nc[c];
  for (int c = 0; c < ndim; ++c)
    if (!(span[c] > 0.0f) || !(p.cl[c] > 0.0f)) return SCARF_ERR_ARG;
  if (!(p.ds > 0.0f) || !(p.dh > 0.0f)) return SCARF_ERR_ARG;
  // kmin/kmax/kc (scarflib_srm.f90:647-652): MAXVAL(cl/span), MINVAL(cl).
  float mx = p.cl[0] / span[0], mn = p.cl[0];
  for (int c = 1; c < ndim; ++c) {
    mx = std::max(mx, p.cl[c] / span[c]);
    mn = std::min(mn, p.cl[c]);
  }
  s->kmin = (2.0f * kPi) * mx;
  s->kmax = (kPi / p.dh) * mn;
  s->kc = (kPi / p.ds) * mn;
  // Representation warnings (:660-662).
  for (int c = 0; c < ndim; ++c) {
    if ((2.0f * kPi) / span[c] >= 1.0f / p.cl[c]) s->info0 = 1.0f;
    if (p.ds > p.cl[c] / 2.0f) s->info1 = 1.0f;
  }
  s->scaling = p.sigma / sqrtf(static_cast<float>(p.nharm));
  // Rotation about z (alpha), y (beta), x (gamma) (:678-691), row-major.
  const float ca = cosf(p.alpha * kPi / 180.0f), sa = sinf(p.alpha * kPi / 180.0f);
  const float cb = cosf(p.beta * kPi / 180.0f), sb = sinf(p.beta * kPi / 180.0f);
  const float cg = cosf(p.gamma * kPi / 180.0f), sg = sinf(p.gamma * kPi / 180.0f);
  float* m = s->m;
  m[0] = ca * cb;
  m[3] = sa * cb;
  m[6] = -sb;
  m[1] = ca * sb * sg - sa * cg;
  m[4] = sa * sb * sg + ca * cg;
  m[7] = cb * sg;
  m[2] = ca * sb * cg + sa * sg;
  m[5] = sa * sb * cg - ca * sg;
  m[8] = cb * cg;
  // Rotation about the half span (:694-700).
  float half[3], rot[3];
  for (int c = 0; c < 3; ++c) half[c] = (p.fc[c] - p.nc[c]) / 2.0f;
  for (int r = 0; r < 3; ++r) rot[r] = m[3 * r] * half[0] + m[3 * r + 1] * half[1] + m[3 * r + 2] * half[2];
  for (int c = 0; c < 3; ++c) s->bar[c] = half[c] - rot[c];
  s->nu = p.hurst + static_cast<float>(ndim) / 2.0f;
  // Majorant constant (:706-716). The reference leaves it unset for a 2D
  // Gaussian; 1 bounds k*exp(-k^2/4) there, so 1 is used.
  s->cnst = (p.acf == 1 && ndim == 3) ? 1.0f / sqrtf(kPi) : 1.0f;
  // Scaling from the spectral integrals (:720, :935-969).
  double band = 0, full = 0, err = 0;
  s->ier_band = quad_dqng(ndim, p.acf, s->nu, static_cast<double>(s->kmin), static_cast<double>(s->kmax), 1.0e-8,
                          1.0e-5, &band, &err);
  s->ier_full = quad_dqagi(ndim, p.acf, s->nu, 0.0, 1.0e-8, 1.0e-5, 500, &full, &err);
  s->intg_band = static_cast<float>(band);
  s->intg_full = static_cast<float>(full);
  s->scaling0 = s->scaling;
  s->scaling = s->scaling * sqrtf(s->intg_band / s->intg_full);
  return SCARF_OK;
}

int host_threads() {
  if (const char* e = std::getenv("SCARF_HOST_THREADS")) {
    const int v = std::atoi(e);
    if (v > 0) return v;
  }
  const unsigned hc = std::thread::hardware_concurrency();
  return static_cast<int>(std::max(1u, std::min(hc, 64u)));
}

// ------------------------------------------------------ host worker pool --
namespace {

// Persistent host workers for the sampler's short parallel loops (field
// walks, table rows, rejection rounds): creating threads per loop costs tens
// of microseconds per thread, more than a 20 000-row loop itself. A job is a
// shared object with its own task counter, so a worker that wakes late for a
// finished job finds no task left and never calls a stale function; the
// caller takes tasks too and waits only for tasks, never for workers.
class HostPool {
 public:
  // Runs fn(0) .. fn(ntasks - 1) on at most `width` threads (the caller's
  // included) and returns when all have returned; the first exception a task
  // threw is rethrown then. Jobs from several caller threads run one after
  // another; fn must not start another job.
  void run(int ntasks, int width, const std::function<void(int)>& fn) {
    if (ntasks <= 0) return;
    width = std::min(width, ntasks);
    if (width <= 1) {
      for (int i = 0; i < ntasks; ++i) fn(i);
      return;
    }
    std::lock_guard<std::mutex> serial(run_mu_);
    auto job = std::make_shared<Job>();
    job->fn = &fn;
    job->ntasks = ntasks;
    job->slots = width - 1;
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (; nworkers_ < width - 1; ++nworkers_) std::thread([this] { worker_loop(); }).detach();
      job_ = job;
      ++gen_;
    }
    cv_.notify_all();
    work(*job);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return job->done.load() == job->ntasks; });
    job_.reset();
    if (job->error) std::rethrow_exception(job->error);
  }

 private:
  struct Job {
    const std::function<void(int)>* fn = nullptr;
    int ntasks = 0;
    std::atomic<int> slots{0}, next{0}, done{0};
    std::mutex error_mu;
    std::exception_ptr error;  // the first exception a task threw
  };

  void work(Job& j) {
    for (int i = j.next.fetch_add(1); i < j.ntasks; i = j.next.fetch_add(1)) {
      try {
        (*j.fn)(i);
      } catch (...) {
        std::lock_guard<std::mutex> lk(j.error_mu);
        if (!j.error) j.error = std::current_exception();
      }
      if (j.done.fetch_add(1) + 1 == j.ntasks) {
        std::lock_guard<std::mutex> lk(mu_);
        done_cv_.notify_all();
      }
    }
  }

  void worker_loop() {
    unsigned long long seen = 0;
    for (;;) {
      std::shared_ptr<Job> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        job = job_;
      }
      if (job && job->slots.fetch_sub(1) > 0) work(*job);
    }
  }

  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  std::shared_ptr<Job> job_;
  unsigned long long gen_ = 0;
  int nworkers_ = 0;  // detached threads; they live as long as the process
};

// One pool per process: a child made by fork() has none of its parent's
// workers (and may hold copies of locked mutexes), so it starts a new pool;
// the parent's object is left as it is.
HostPool& host_pool() {
  static std::mutex mu;
  static HostPool* pool = nullptr;
  static pid_t owner = 0;
  std::lock_guard<std::mutex> lk(mu);
  const pid_t pid = getpid();
  if (!pool || owner != pid) {
    pool = new HostPool();
    owner = pid;
  }
  return *pool;
}

}  // namespace

void parallel_tasks(int ntasks, int width, const std::function<void(int)>& fn) {
  host_pool().run(ntasks, width, fn);
}

// ------------------------------------------------------------- sampler -----
namespace {

// Everything the per-harmonic math needs from the draws of one harmonic.
struct Draws {
  float u;
  float ang[2], ra[2], rb[2];
  bool skip;
};

// Per-harmonic arithmetic (scarflib_srm.f90:754-778) in statement order.
inline void harmonic_row(const Draws& d, int ndim, const float cl[3], float* row) {
  const float phi = d.ang[0] * 2.0f * kPi;
  float v1, v2, v3;
  if (ndim == 3) {
    const float theta = acosf(1.0f - 2.0f * d.ang[1]);
    v1 = d.u * sinf(phi) * sinf(theta) / cl[0];
    v2 = d.u * cosf(phi) * sinf(theta) / cl[1];
    v3 = d.u * cosf(theta) / cl[2];
  } else {
    v1 = d.u * cosf(phi) / cl[0];
    v2 = d.u * sinf(phi) / cl[1];
    v3 = 0.0f;
  }
  row[0] = v1;
  row[1] = v2;
  row[2] = v3;
  row[3] = sqrtf(-2.0f * logf(d.ra[0])) * cosf(2.0f * kPi * d.ra[1]);
  row[4] = sqrtf(-2.0f * logf(d.rb[0])) * cosf(2.0f * kPi * d.rb[1]);
}

inline bool accept(float r1, float r2, const scarf_srm_setup& s, int acf, float* u_out) {
  const float u = r1 * (s.kmax - s.kmin) + s.kmin;
  const float d = static_cast<float>(srm_fn(static_cast<double>(u), s.ndim, acf, s.nu) * static_cast<double>(s.cnst));
  *u_out = u;
  return r2 < d;
}

// Serial walk over an arbitrary pair source (the reference's own loop).
template <class NextPair>
int walk_serial(const scarf_srm_params& p, const scarf_srm_setup& s, NextPair next, float* table, long long* used) {
  int kept = 0;
  long long np = 0;
  float r[2];
  for (int l = 0; l < p.nharm; ++l) {
    Draws d{};
    for (;;) {
      next(r);
      ++np;
      if (accept(r[0], r[1], s, p.acf, &d.u)) break;
    }
    next(r);
    ++np;
    if (d.u > s.kc) continue;
    d.ang[0] = r[0];
    d.ang[1] = r[1];
    next(r);
    ++np;
    d.ra[0] = r[0];
    d.ra[1] = r[1];
    next(r);
    ++np;
    d.rb[0] = r[0];
    d.rb[1] = r[1];
    harmonic_row(d, s.ndim, p.cl, table + 5 * static_cast<size_t>(kept));
    ++kept;
  }
  if (used) *used = np;
  return kept;
}

// Parallel form for the built-in generator. The pair stream is cut into
// rounds; in each round `threads` workers evaluate the rejection test for
// consecutive chunks of pairs from jumped copies of the generator, and one
// walker then consumes the round in stream order exactly as the serial loop
// would. Decisions and values are those of the serial loop by construction.
int walk_parallel(const scarf_srm_params& p, const scarf_srm_setup& s, int threads, float* table, long long* used) {
  // Round size from the expected number of pairs: a pair is accepted with
  // probability int_{kmin}^{kmax} d(k) dk / (kmax - kmin), and every kept
  // harmonic consumes three more pairs.
  double acc_rate = static_cast<double>(s.intg_band) * s.cnst / std::max(1e-30, double(s.kmax) - double(s.kmin));
  acc_rate = std::min(1.0, std::max(acc_rate, 1e-6));
  const double expect = p.nharm * (1.0 / acc_rate + 3.0) * 1.05 + 64.0;
  const int64_t chunk = std::min<int64_t>(1 << 18, std::max<int64_t>(4096, static_cast<int64_t>(expect / threads) + 1));
  const int64_t round_pairs = chunk * threads;
  std::vector<float> cur(2 * round_pairs), nxt(2 * round_pairs);
  std::vector<uint8_t> acc_cur(round_pairs), acc_nxt(round_pairs);
  std::vector<float> u_cur(round_pairs), u_nxt(round_pairs);
  Yarn2 base;
  base.seed(p.seed);

  auto fill = [&](int64_t first_pair, std::vector<float>& r, std::vector<uint8_t>& acc, std::vector<float>& uu) {
    parallel_tasks(threads, threads, [&](int t) {
      Yarn2 g = base;
      g.jump(2ull * static_cast<uint64_t>(first_pair + t * chunk));
      for (int64_t q = t * chunk; q < (t + 1) * chunk; ++q) {
        const float r1 = g.next_u01(), r2 = g.next_u01();
        r[2 * q] = r1;
        r[2 * q + 1] = r2;
        float u;
        acc[q] = accept(r1, r2, s, p.acf, &u) ? 1 : 0;
        uu[q] = u;
      }
    });
  };

  int64_t cur_first = 0;
  fill(0, cur, acc_cur, u_cur);
  bool have_next = false;
  auto ensure_next = [&]() {
    if (!have_next) {
      fill(cur_first + round_pairs, nxt, acc_nxt, u_nxt);
      have_next = true;
    }
  };
  auto advance_round = [&]() {
    ensure_next();
    std::swap(cur, nxt);
    std::swap(acc_cur, acc_nxt);
    std::swap(u_cur, u_nxt);
    cur_first += round_pairs;
    have_next = false;
  };
  // Pair q (global index) values; q may reach into the next round.
  auto pair_at = [&](int64_t q, float out[2]) {
    int64_t k = q - cur_first;
    if (k < round_pairs) {
      out[0] = cur[2 * k];
      out[1] = cur[2 * k + 1];
    } else {
      ensure_next();
      k -= round_pairs;
      out[0] = nxt[2 * k];
      out[1] = nxt[2 * k + 1];
    }
  };

  int kept = 0;
  int64_t pos = 0;  // next unconsumed pair
  for (int l = 0; l < p.nharm; ++l) {
    // First accepted pair at or after pos.
    float u = 0.0f;
    for (;;) {
      while (pos - cur_first >= round_pairs) advance_round();
      const int64_t k = pos - cur_first;
      const int64_t end = round_pairs;
      int64_t j = k;
      while (j < end && !acc_cur[j]) ++j;
      if (j < end) {
        u = u_cur[j];
        pos = cur_first + j + 1;
        break;
      }
      pos = cur_first + end;
    }
    Draws d{};
    d.u = u;
    pair_at(pos, d.ang);
    ++pos;
    if (u > s.kc) continue;
    pair_at(pos, d.ra);
    ++pos;
    pair_at(pos, d.rb);
    ++pos;
    harmonic_row(d, s.ndim, p.cl, table + 5 * static_cast<size_t>(kept));
    ++kept;
  }
  if (used) *used = pos;
  return kept;
}

}  // namespace

double acceptance_rate(const scarf_srm_setup& s) {
  const double width = static_cast<double>(s.kmax) - static_cast<double>(s.kmin);
  if (!(width > 0.0)) return 0.0;
  return static_cast<double>(s.intg_band) * s.cnst / width;
}

// ------------------------------------------------ device memory accounting --
namespace {
std::atomic<size_t> g_dev_in_use{0};
std::atomic<size_t> g_dev_cap{0};  // 0: no cap
thread_local bool t_alloc_failed = false;
}  // namespace

int device_alloc(void** p, size_t bytes) {
  *p = nullptr;
  const size_t cap = g_dev_cap.load();
  size_t used = g_dev_in_use.load();
  do {
    if (cap && bytes > cap - std::min(cap, used)) {
      t_alloc_failed = true;
      return cudaErrorMemoryAllocation;
    }
  } while (!g_dev_in_use.compare_exchange_weak(used, used + bytes));
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    g_dev_in_use -= bytes;
    *p = nullptr;
    if (e == cudaErrorMemoryAllocation) {
      t_alloc_failed = true;
      cudaGetLastError();
    }
  }
  return e;
}

bool take_device_alloc_failure() {
  const bool f = t_alloc_failed;
  t_alloc_failed = false;
  return f;
}

void device_free(void* p, size_t bytes) {
  if (!p) return;
  cudaFree(p);
  g_dev_in_use -= bytes;
}

void set_device_memory_cap(size_t bytes) { g_dev_cap = bytes; }
size_t device_memory_in_use() { return g_dev_in_use.load(); }

// ------------------------------------------------- device-assisted sampler --
namespace {

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t need) {
    if (need <= bytes) return cudaSuccess;
    device_free(p, bytes);
    p = nullptr;
    bytes = 0;
    const cudaError_t e = static_cast<cudaError_t>(device_alloc(&p, need));
    if (e == cudaSuccess) bytes = need;
    return e;
  }
  void release() {
    device_free(p, bytes);
    p = nullptr;
    bytes = 0;
  }
};

struct DeviceSamplerState {
  int device = -1;
  bool tables = false;
  DevBuf counts, offsets, entries, slots, batch_args, batch_tbeg, reject;
  SampleEntry* host_entries = nullptr;  // page-locked staging of candidate entries
  long long host_entries_cap = 0;
  // Two sets of the same for a batch's groups: one group's gather fills one
  // while the host walks the previous group's entries in the other.
  DevBuf gentries[2];
  SampleEntry* ghost[2] = {nullptr, nullptr};
  long long ghost_cap[2] = {0, 0};
  cudaStream_t side = nullptr;        // gathers and copies beside the scans
  std::vector<cudaEvent_t> events;    // end of each group's scan
};
DeviceSamplerState g_dev_sampler;
std::mutex g_dev_sampler_mu;
long long g_pass_pairs_cap = 0;  // 0: size passes from the acceptance rate
// Scan launches of a batch: the host's walks and table rows of one group run
// while the following groups scan.
constexpr int kSamplerGroups = 8;

// Host decision for a pair the device left open (glibc spectrum).
bool host_accept(const scarf_srm_setup& s, int acf, float r1, float r2) {
  float u;
  return accept(r1, r2, s, acf, &u);
}

}  // namespace

void sampler_reject_thresholds(const scarf_srm_setup& s, int acf, float margin, uint32_t* thr) {
  const int pw = s.ndim - 1;
  const double nu = s.nu;
  auto F = [&](double x) {
    const double psd = acf == 0 ? std::pow(1.0 + x * x, -nu) : std::exp(-0.25 * x * x);
    return (pw == 2 ? x * x : x) * psd * static_cast<double>(s.cnst);
  };
  double peak = 0.0;
  if (acf == 0) {
    const double den = 2.0 * nu - pw;
    peak = den > 0.0 ? std::sqrt(pw / den) : HUGE_VAL;  // (den <= 0: increasing)
  } else {
    peak = std::sqrt(2.0 * pw);
  }
  // u as the scan computes it from r1, in FP32 without contraction.
  const float w = s.kmax - s.kmin;
  auto u_of = [&](uint32_t y) { return Yarn2::to_u01(y) * w + s.kmin; };
  for (int b = 0; b < kRejectBins; ++b) {
    const uint32_t y0 = static_cast<uint32_t>(b) << kRejectShift;
    const uint32_t y1 = static_cast<uint32_t>(std::min<uint64_t>((static_cast<uint64_t>(b) + 1) << kRejectShift,
                                                                 Yarn2::kMod) - 1);
    const double a = u_of(y0), c = u_of(y1);
    const double x = std::min(std::max(peak, a), c);
    // relative room for the FP32 spectrum (expf's argument error grows with
    // |arg| to ~1e-5 before it underflows), absolute room for its subnormals
    const double bound = F(x) * (1.0 + static_cast<double>(margin)) * (1.0 + 1e-4) + 1e-30;
    // smallest raw y with to_u01(y) >= bound (to_u01 is non-decreasing)
    uint32_t t = 0xFFFFFFFFu;
    if (!(bound > 1.0) && std::isfinite(bound)) {
      uint32_t lo = 0, hi = static_cast<uint32_t>(Yarn2::kMod);  // to_u01(m) = 1 >= bound
      while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (static_cast<double>(Yarn2::to_u01(mid)) >= bound) hi = mid;
        else lo = mid + 1;
      }
      t = lo;
    }
    thr[b] = t;
  }
}

void set_device_sampler_pass_cap(long long pairs) {
  std::lock_guard<std::mutex> lk(g_dev_sampler_mu);
  g_pass_pairs_cap = pairs > 0 ? pairs : 0;
}

namespace {

SamplerArgs make_sampler_args(const scarf_srm_params& p, const scarf_srm_setup& s) {
  Yarn2 g;
  g.seed(p.seed);
  SamplerArgs A{};
  A.r0 = g.r0;
  A.r1 = g.r1;
  A.kmin = s.kmin;
  A.kmax = s.kmax;
  A.cnst = s.cnst;
  A.nu = s.nu;
  A.ndim = s.ndim;
  A.acf = p.acf;
  A.margin = kSamplerMargin;
  return A;
}

long long capped_pairs(long long n) { return g_pass_pairs_cap > 0 ? std::min(n, g_pass_pairs_cap) : n; }

// Pairs of the first pass of a field: enough for every harmonic at the
// expected acceptance with a 10 % margin.
long long first_pass_pairs(const scarf_srm_params& p, double acc) {
  return capped_pairs(static_cast<long long>(p.nharm * (1.0 / acc + 3.0) * 1.1) + 4096);
}

}  // namespace

void release_sampler_device_memory() {
  std::lock_guard<std::mutex> lk(g_dev_sampler_mu);
  DeviceSamplerState& D = g_dev_sampler;
  for (DevBuf* b : {&D.counts, &D.offsets, &D.entries, &D.slots, &D.batch_args, &D.batch_tbeg, &D.reject,
                    &D.gentries[0], &D.gentries[1]})
    b->release();
}

namespace {

// Uploads the pow tables once per device (caller holds g_dev_sampler_mu).
bool ensure_sampler_device(DeviceSamplerState& D) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (D.device != dev) {
    // the previous device's buffers (freed through unified addressing)
    for (DevBuf* b : {&D.counts, &D.offsets, &D.entries, &D.slots, &D.batch_args, &D.batch_tbeg, &D.reject,
                      &D.gentries[0], &D.gentries[1]})
      b->release();
    if (D.host_entries) cudaFreeHost(D.host_entries);
    for (SampleEntry* h : D.ghost)
      if (h) cudaFreeHost(h);
    D = DeviceSamplerState();
    D.device = dev;
  }
  if (!D.tables) {
    static const std::vector<uint32_t> t = device_pow_tables();
    if (sampler_upload_tables(t.data()) != cudaSuccess) return false;
    D.tables = true;
  }
  return true;
}

// One device pass of one field over pairs [q_begin, q_begin + count): the
// candidate entries (accepted or undecided pairs) in stream order.
bool single_pass(DeviceSamplerState& D, SamplerArgs A, long long q_begin, long long count,
                 std::vector<SampleEntry>& entries, cudaStream_t stream) {
  A.q_begin = q_begin;
  A.q_count = count;
  A.pairs_per_thread = static_cast<int>(std::min<long long>(8192, std::max<long long>(256, count / (148 * 2048))));
  A.nthreads = (count + A.pairs_per_thread - 1) / A.pairs_per_thread;
  if (D.counts.ensure(sizeof(int) * A.nthreads) != cudaSuccess) return false;
  if (D.offsets.ensure(sizeof(long long) * A.nthreads) != cudaSuccess) return false;
  A.counts = static_cast<int*>(D.counts.p);
  A.offsets = static_cast<const long long*>(D.offsets.p);
  A.write = 0;
  if (launch_sampler(A, stream) != cudaSuccess) return false;
  std::vector<int> counts(A.nthreads);
  if (cudaMemcpyAsync(counts.data(), D.counts.p, sizeof(int) * A.nthreads, cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return false;
  std::vector<long long> offsets(A.nthreads);
  long long total = 0;
  for (long long t = 0; t < A.nthreads; ++t) {
    offsets[t] = total;
    total += counts[t];
  }
  entries.resize(total);
  if (total > 0) {
    if (D.entries.ensure(sizeof(SampleEntry) * total) != cudaSuccess) return false;
    if (cudaMemcpyAsync(D.offsets.p, offsets.data(), sizeof(long long) * A.nthreads, cudaMemcpyHostToDevice,
                        stream) != cudaSuccess)
      return false;
    A.out = static_cast<SampleEntry*>(D.entries.p);
    A.write = 1;
    if (launch_sampler(A, stream) != cudaSuccess) return false;
    if (cudaMemcpyAsync(entries.data(), D.entries.p, sizeof(SampleEntry) * total, cudaMemcpyDeviceToHost, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return false;
  }
  return true;
}

// The host walk of one field over its candidate entries, in stream order
// exactly as the serial loop consumes pairs: reject until an accepted pair,
// then one pair of angles, then (for a kept harmonic) two pairs for a and b.
// Resumable: walk() returns false when the entries ran out before every
// harmonic was decided; the caller then supplies the next pass.
struct DeviceWalk {
  const scarf_srm_params* p = nullptr;
  const scarf_srm_setup* s = nullptr;
  float* table = nullptr;
  double acc = 0.0;
  // Candidates of the current pass: a view into a shared buffer (first pass
  // of a batch) or into `owned` (passes of this field alone).
  const SampleEntry* ent = nullptr;
  size_t nent = 0;
  std::vector<SampleEntry> owned;
  std::vector<Draws> draws;  // kept harmonics' draws; their rows are computed after the walk
  size_t ei = 0;
  long long pos = 0, open = 0, pass_end = 0;
  int kept = 0, l = 0;

  bool walk() {
    if (draws.empty()) draws.reserve(p->nharm);
    for (; l < p->nharm; ++l) {
      for (;;) {
        while (ei < nent && ent[ei].q < pos) ++ei;
        if (ei == nent) return false;
        const SampleEntry& e = ent[ei];
        bool ok = e.flag == 1;
        if (e.flag == 2) {
          ++open;
          ok = host_accept(*s, p->acf, e.r[0], e.r[1]);
        }
        if (!ok) {
          ++ei;
          continue;
        }
        Draws d{};
        d.u = e.r[0] * (s->kmax - s->kmin) + s->kmin;
        if (d.u > s->kc) {
          pos = e.q + 2;
          break;
        }
        d.ang[0] = e.r[2];
        d.ang[1] = e.r[3];
        d.ra[0] = e.r[4];
        d.ra[1] = e.r[5];
        d.rb[0] = e.r[6];
        d.rb[1] = e.r[7];
        draws.push_back(d);
        ++kept;
        pos = e.q + 4;
        break;
      }
    }
    return true;
  }

  // Further passes until the walk completes.
  bool finish(DeviceSamplerState& D, const SamplerArgs& A, cudaStream_t stream) {
    while (!walk()) {
      const long long more = capped_pairs(static_cast<long long>((p->nharm - l) * (1.0 / acc + 3.0) * 1.2) + 4096);
      if (!single_pass(D, A, pass_end, more, owned, stream)) return false;
      pass_end += more;
      ent = owned.data();
      nent = owned.size();
      ei = 0;
    }
    return true;
  }
};

}  // namespace

int srm_sample_device(const scarf_srm_params& p, const scarf_srm_setup& s, float* table, long long* pairs_used,
                      void* stream_handle, long long* uncertain) {
  // The batched path with one field: its first pass is a single scan.
  int kept = 0;
  long long used = 0;
  float* tables[1] = {table};
  const int rc = srm_sample_device_batch(1, &p, &s, tables, &kept, &used, stream_handle, uncertain);
  if (rc == -1) return -1;
  if (rc < 0) return -2;
  if (pairs_used) *pairs_used = used;
  return kept;
}

int srm_sample_device_batch(int nfields, const scarf_srm_params* p, const scarf_srm_setup* s, float* const* tables,
                            int* kept, long long* pairs_used, void* stream_handle, long long* uncertain) {
  const cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
  if (nfields <= 0) return 0;
  std::vector<double> acc(nfields);
  for (int f = 0; f < nfields; ++f) {
    acc[f] = acceptance_rate(s[f]);
    if (acc[f] < kMinAcceptance) return -1 - f;
  }
  std::lock_guard<std::mutex> lk(g_dev_sampler_mu);
  DeviceSamplerState& D = g_dev_sampler;
  if (!ensure_sampler_device(D)) return -2 - nfields;
  // First pass of every field in one scan: each thread keeps up to `cap`
  // candidates in its own slot (cap sized from the expected count, with a
  // wide Poisson margin); a gather launch compacts them. The fields share
  // ~300k threads or more (2 048 at least each), 256 to 4 096 pairs per
  // thread: each thread's pairs form one serial chain of generator steps, so
  // longer chains leave the scan waiting on its slowest threads.
  const long long thread_goal = std::max<long long>(2048, 148LL * 2048 / nfields);
  std::vector<SamplerArgs> args(nfields);
  std::vector<long long> tbeg(nfields + 1, 0), sbeg(nfields + 1, 0);
  for (int f = 0; f < nfields; ++f) {
    SamplerArgs& A = args[f];
    A = make_sampler_args(p[f], s[f]);
    A.q_begin = 0;
    A.q_count = first_pass_pairs(p[f], acc[f]);
    A.pairs_per_thread =
        static_cast<int>(std::min<long long>(4096, std::max<long long>(256, A.q_count / thread_goal)));
    A.nthreads = (A.q_count + A.pairs_per_thread - 1) / A.pairs_per_thread;
    const double lambda = A.pairs_per_thread * std::min(1.0, acc[f]);
    A.cap = static_cast<int>(std::ceil(1.25 * lambda + 6.0 * std::sqrt(lambda) + 8.0));
    // Test hook: a smaller slot forces the overflow path (fields redone with
    // their own passes), which the margin above makes vanishingly rare.
    if (const char* e = std::getenv("SCARF3D_B200_SAMPLER_SLOT_CAP")) A.cap = std::max(1, std::min(A.cap, std::atoi(e)));
    tbeg[f + 1] = tbeg[f] + A.nthreads;
    sbeg[f + 1] = sbeg[f] + A.nthreads * A.cap;
  }
  const long long T = tbeg[nfields];
  const int err = -2 - nfields;
  if (D.counts.ensure(sizeof(int) * T) != cudaSuccess || D.offsets.ensure(sizeof(long long) * T) != cudaSuccess ||
      D.slots.ensure(sizeof(unsigned long long) * sbeg[nfields]) != cudaSuccess ||
      D.batch_args.ensure(sizeof(SamplerArgs) * nfields) != cudaSuccess ||
      D.batch_tbeg.ensure(sizeof(long long) * (nfields + 1)) != cudaSuccess ||
      D.reject.ensure(sizeof(uint32_t) * kRejectBins * nfields) != cudaSuccess)
    return err;
  // Certain-reject thresholds of every field, uploaded before the scans.
  std::vector<uint32_t> reject(static_cast<size_t>(kRejectBins) * nfields);
  parallel_tasks(nfields, host_threads(), [&](int f) {
    sampler_reject_thresholds(s[f], p[f].acf, args[f].margin, reject.data() + static_cast<size_t>(f) * kRejectBins);
  });
  if (cudaMemcpyAsync(D.reject.p, reject.data(), sizeof(uint32_t) * reject.size(), cudaMemcpyHostToDevice, stream) !=
      cudaSuccess)
    return err;
  int* d_counts = static_cast<int*>(D.counts.p);
  long long* d_offsets = static_cast<long long*>(D.offsets.p);
  unsigned long long* d_slots = static_cast<unsigned long long*>(D.slots.p);
  for (int f = 0; f < nfields; ++f) {
    args[f].counts = d_counts + tbeg[f];
    args[f].offsets = nullptr;
    args[f].out = nullptr;
    args[f].keys = d_slots + sbeg[f];
    args[f].reject = static_cast<const unsigned int*>(D.reject.p) + static_cast<size_t>(f) * kRejectBins;
  }
  // Groups of consecutive fields, balanced by their first-pass pairs. Each
  // group's scan is its own launch on `stream`; while later groups scan, the
  // host copies the finished group's counts, gathers its candidates on the
  // side stream, walks its fields and fills their table rows, so the host
  // work of all but the last group runs under the scans. tbeg_rel holds the
  // thread offsets relative to each group's first thread, group after group
  // (group g's fields [gbeg[g], gbeg[g+1]) at entries gbeg[g] + g ...).
  const int G = std::max(1, std::min(nfields, kSamplerGroups));
  std::vector<int> gbeg(G + 1, nfields);
  gbeg[0] = 0;
  {
    double all = 0.0, run = 0.0;
    for (int f = 0; f < nfields; ++f) all += static_cast<double>(args[f].q_count);
    int g = 1;
    for (int f = 0; f < nfields && g < G; ++f) {
      run += static_cast<double>(args[f].q_count);
      if (run >= all * g / G) gbeg[g++] = f + 1;
    }
  }
  std::vector<long long> tbeg_rel(nfields + G, 0);
  for (int g = 0; g < G; ++g)
    for (int f = gbeg[g]; f <= gbeg[g + 1]; ++f) tbeg_rel[f + g] = tbeg[f] - tbeg[gbeg[g]];
  if (D.batch_tbeg.ensure(sizeof(long long) * (nfields + G)) != cudaSuccess) return err;
  if (!D.side && cudaStreamCreateWithFlags(&D.side, cudaStreamNonBlocking) != cudaSuccess) {
    D.side = nullptr;
    return err;
  }

  while (static_cast<int>(D.events.size()) < G) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return err;
    D.events.push_back(e);
  }
  if (cudaMemcpyAsync(D.batch_args.p, args.data(), sizeof(SamplerArgs) * nfields, cudaMemcpyHostToDevice, stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(D.batch_tbeg.p, tbeg_rel.data(), sizeof(long long) * (nfields + G), cudaMemcpyHostToDevice,
                      stream) != cudaSuccess)
    return err;
  const SamplerArgs* d_args = static_cast<const SamplerArgs*>(D.batch_args.p);
  const long long* d_tbeg = static_cast<const long long*>(D.batch_tbeg.p);
  // One launch per group on the caller's stream (scans of consecutive groups
  // run on two streams measured slower: the groups then finish later and
  // the host stages behind them start later).
  for (int g = 0; g < G; ++g) {
    const int f0 = gbeg[g], f1 = gbeg[g + 1];
    if (f1 > f0 &&
        launch_sampler_batch(d_args + f0, d_tbeg + f0 + g, f1 - f0, tbeg[f1] - tbeg[f0], 2, stream) != cudaSuccess)
      return err;
    if (cudaEventRecord(D.events[g], stream) != cudaSuccess) return err;
  }

  std::vector<int> counts(T);
  std::vector<long long> offsets(T);        // relative to the group's first entry
  std::vector<char> overflow(nfields, 0);   // a slot overflowed: the field is redone alone
  std::vector<DeviceWalk> walks(nfields);
  std::vector<char> done(nfields, 0);
  for (int f = 0; f < nfields; ++f) {
    DeviceWalk& w = walks[f];
    w.p = &p[f];
    w.s = &s[f];
    w.table = tables[f];
    w.acc = acc[f];
    w.pass_end = args[f].q_count;
  }
  // Table rows from the kept draws (libm trig per row), spread over host
  // threads in blocks of rows; each row depends on its own draw only.
  auto fill_rows = [&](const std::vector<int>& fields) {
    std::vector<long long> rbeg(fields.size() + 1, 0);
    for (size_t i = 0; i < fields.size(); ++i) rbeg[i + 1] = rbeg[i] + walks[fields[i]].kept;
    constexpr long long kRowBlock = 512;
    const long long nblocks = (rbeg.back() + kRowBlock - 1) / kRowBlock;
    parallel_tasks(static_cast<int>(nblocks), host_threads(), [&](int b) {
      const long long r0 = b * kRowBlock, r1 = std::min(rbeg.back(), r0 + kRowBlock);
      size_t i = static_cast<size_t>(std::upper_bound(rbeg.begin(), rbeg.end(), r0) - rbeg.begin()) - 1;
      for (long long r = r0; r < r1; ++r) {
        while (r >= rbeg[i + 1]) ++i;
        const int f = fields[i];
        const long long k = r - rbeg[i];
        harmonic_row(walks[f].draws[k], s[f].ndim, p[f].cl, tables[f] + 5 * k);
      }
    });
  };
  // Walks of a group whose entries sit in staging set `b` (complete once the
  // side stream has passed the group's copy), then the table rows of the
  // fields it finished.
  auto walk_group = [&](int g, int b, const std::vector<long long>& ebeg) {
    const int f0 = gbeg[g], f1 = gbeg[g + 1];
    for (int f = f0; f < f1; ++f) {
      DeviceWalk& w = walks[f];
      w.ent = overflow[f] ? nullptr : D.ghost[b] + ebeg[f - f0];
      w.nent = overflow[f] ? 0 : static_cast<size_t>(ebeg[f - f0 + 1] - ebeg[f - f0]);
      if (overflow[f]) w.pass_end = 0;
    }
    parallel_tasks(f1 - f0, host_threads(), [&](int i) { done[f0 + i] = walks[f0 + i].walk() ? 1 : 0; });
    std::vector<int> finished;
    for (int f = f0; f < f1; ++f) {
      // the staging set belongs to a later group now
      walks[f].ent = nullptr;
      walks[f].nent = 0;
      walks[f].ei = 0;
      if (done[f]) finished.push_back(f);
    }
    fill_rows(finished);
  };
  // Group g: its counts (which also waits for the previous group's gather
  // and copy on the side stream), then its gather into the staging set the
  // previous non-empty group did not use; the previous group is walked
  // while that gather runs.
  int prev = -1, prev_b = 1;
  std::vector<long long> prev_ebeg;
  for (int g = 0; g < G; ++g) {
    const int f0 = gbeg[g], f1 = gbeg[g + 1];
    if (f1 == f0) continue;
    const long long t0 = tbeg[f0], Tg = tbeg[f1] - t0;
    if (cudaStreamWaitEvent(D.side, D.events[g], 0) != cudaSuccess ||
        cudaMemcpyAsync(counts.data() + t0, d_counts + t0, sizeof(int) * Tg, cudaMemcpyDeviceToHost, D.side) !=
            cudaSuccess ||
        cudaStreamSynchronize(D.side) != cudaSuccess)
      return err;
    std::vector<long long> ebeg(f1 - f0 + 1, 0);  // entry range of each field of the group
    long long total = 0;
    for (int f = f0; f < f1; ++f) {
      for (long long t = tbeg[f]; t < tbeg[f + 1]; ++t) {
        offsets[t] = total;
        if (counts[t] > args[f].cap) overflow[f] = 1;
        total += std::min(counts[t], args[f].cap);
      }
      ebeg[f - f0 + 1] = total;
    }
    const int b = prev_b ^ 1;
    if (total > 0) {
      // Set b was last read by the walks of the group before the previous
      // one, which are done.
      if (D.gentries[b].ensure(sizeof(SampleEntry) * total) != cudaSuccess) return err;
      if (D.ghost_cap[b] < total) {
        if (D.ghost[b]) cudaFreeHost(D.ghost[b]);
        D.ghost[b] = nullptr;
        D.ghost_cap[b] = 0;
        void* h = nullptr;
        if (cudaHostAlloc(&h, sizeof(SampleEntry) * total, cudaHostAllocDefault) != cudaSuccess) return err;
        D.ghost[b] = static_cast<SampleEntry*>(h);
        D.ghost_cap[b] = total;
      }
      if (cudaMemcpyAsync(d_offsets + t0, offsets.data() + t0, sizeof(long long) * Tg, cudaMemcpyHostToDevice,
                          D.side) != cudaSuccess ||
          launch_sampler_gather(d_args + f0, d_tbeg + f0 + g, f1 - f0, Tg, d_offsets + t0,
                                static_cast<SampleEntry*>(D.gentries[b].p), D.side) != cudaSuccess ||
          cudaMemcpyAsync(D.ghost[b], D.gentries[b].p, sizeof(SampleEntry) * total, cudaMemcpyDeviceToHost,
                          D.side) != cudaSuccess)
        return err;
    }
    if (prev >= 0) walk_group(prev, prev_b, prev_ebeg);
    prev = g;
    prev_b = b;
    prev_ebeg.swap(ebeg);
  }
  if (prev >= 0) {
    if (cudaStreamSynchronize(D.side) != cudaSuccess) return err;
    walk_group(prev, prev_b, prev_ebeg);
  }
  // Fields whose first pass ran short (or overflowed) continue with their own
  // device passes, one field at a time, once every group's scan is done.
  long long open_total = 0;
  std::vector<int> rest;
  for (int f = 0; f < nfields; ++f) {
    DeviceWalk& w = walks[f];
    if (!done[f]) {
      SamplerArgs A = args[f];
      A.counts = nullptr;
      A.offsets = nullptr;
      A.out = nullptr;
      if (!w.finish(D, A, stream)) return err;
      rest.push_back(f);
    }
    if (kept) kept[f] = w.kept;
    if (pairs_used) pairs_used[f] = w.pos;
    open_total += w.open;
  }
  fill_rows(rest);
  if (uncertain) *uncertain = open_total;
  return 0;
}

int srm_sample(const scarf_srm_params& p, const scarf_srm_setup& s, const UniformSource* src, int threads,
               float* table, long long* pairs_used) {
  // The rejection loop (scarflib_srm.f90:731-745) draws until r2 < d(u); its
  // success probability is the spectral mass in [kmin, kmax] over the
  // interval width. Below kMinAcceptance a field would take hours of host
  // time (the reference spins the same way), so such inputs are refused.
  if (acceptance_rate(s) < kMinAcceptance) return -1;
  if (src && src->srng) {
    if (src->set_seed) src->set_seed(p.seed);
    return walk_serial(p, s, [&](float r[2]) { src->srng(r); }, table, pairs_used);
  }
  if (threads <= 1 || p.nharm < 64) {
    Yarn2 g;
    g.seed(p.seed);
    return walk_serial(
        p, s,
        [&](float r[2]) {
          r[0] = g.next_u01();
          r[1] = g.next_u01();
        },
        table, pairs_used);
  }
  return walk_parallel(p, s, threads, table, pairs_used);
}

}  // namespace scarf
