// Host code of the library and the C oracle under AddressSanitizer and
// UndefinedBehaviorSanitizer (built and run by test_sanitizers.py, no GPU).
// Exercises setup, quadrature, the serial and multi-threaded samplers, the
// host worker pool and the host side of the device-assisted sampler, and
// cross-checks them bit for bit (the oracle for setup and serial tables, the
// serial sampler for the device-assisted one). Any sanitizer report aborts.
//
// No GPU is reached: the CUDA runtime calls the sampler's host code makes
// are defined here over host memory (copies synchronous, streams and events
// inert), and the four sampler kernels are emulated on the host from their
// device semantics (srm_sampler.cu), so the orchestration -- grouped scans,
// per-group gathers, walks, slot overflow, further passes -- runs for real.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../oracle/srm_oracle.h"
#include "srm_host.h"
#include "srm_kernels.h"

// ---- CUDA runtime over host memory ----------------------------------------
namespace {
int g_handle;  // streams and events are inert: any non-null handle will do
}
extern "C" {
cudaError_t cudaGetDevice(int* d) {
  *d = 0;
  return cudaSuccess;
}
cudaError_t cudaMalloc(void** p, size_t n) {
  *p = std::malloc(n ? n : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned int) { return cudaMalloc(p, n); }
cudaError_t cudaFreeHost(void* p) { return cudaFree(p); }
cudaError_t cudaMemcpyAsync(void* dst, const void* src, size_t n, cudaMemcpyKind, cudaStream_t) {
  if (n) std::memcpy(dst, src, n);
  return cudaSuccess;
}
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* s, unsigned int) {
  *s = reinterpret_cast<cudaStream_t>(&g_handle);
  return cudaSuccess;
}
cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned int) {
  *e = reinterpret_cast<cudaEvent_t>(&g_handle);
  return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaStreamWaitEvent(cudaStream_t, cudaEvent_t, unsigned int) { return cudaSuccess; }
cudaError_t cudaGetLastError(void) { return cudaSuccess; }
}

// ---- the sampler kernels, emulated -----------------------------------------
namespace scarf {
namespace {

Yarn2 at_pair(const SamplerArgs& A, long long q) {
  Yarn2 g;
  g.r0 = A.r0;
  g.r1 = A.r1;
  g.jump(2ull * static_cast<uint64_t>(q));
  return g;
}

// 0 = certain reject, 1 = certain accept, 2 = uncertain (as the device tests).
int classify(const SamplerArgs& A, float r1, float r2) {
  const float u = r1 * (A.kmax - A.kmin) + A.kmin;
  const float fv = A.acf == 0 ? 1.0f / powf(1.0f + u * u, A.nu) : expf(-0.25f * (u * u));
  double srm = static_cast<double>(u) * static_cast<double>(fv);
  if (A.ndim == 3) srm = srm * static_cast<double>(u);
  const float d = static_cast<float>(srm * static_cast<double>(A.cnst));
  if (r2 < d * (1.0f - A.margin)) return 1;
  if (r2 >= d * (1.0f + A.margin)) return 0;
  return 2;
}

void sample_range(const SamplerArgs& A, long long t, int write) {
  const long long q0 = A.q_begin + t * A.pairs_per_thread;
  const long long q1 = std::min(q0 + A.pairs_per_thread, A.q_begin + A.q_count);
  Yarn2 g = at_pair(A, q0);
  int count = 0;
  long long slot = write == 1 ? A.offsets[t] : (write == 2 ? t * A.cap : 0);
  const long long slot_end = write == 2 ? slot + A.cap : (1ll << 62);
  for (long long q = q0; q < q1; ++q) {
    const float r1 = Yarn2::to_u01(g.next_raw());
    const float r2 = Yarn2::to_u01(g.next_raw());
    const int c = classify(A, r1, r2);
    if (c == 0) continue;
    ++count;
    if (write == 2) {
      if (slot < slot_end) A.keys[slot++] = (static_cast<unsigned long long>(q) << 2) | static_cast<unsigned>(c);
    } else if (write && slot < slot_end) {
      SampleEntry e{};
      e.q = q;
      e.flag = c;
      e.r[0] = r1;
      e.r[1] = r2;
      Yarn2 look = g;
      for (int k = 2; k < 8; ++k) e.r[k] = Yarn2::to_u01(look.next_raw());
      A.out[slot++] = e;
    }
  }
  if (write != 1) A.counts[t] = count;
}

int field_of(const long long* tbeg, int nfields, long long t) {
  int lo = 0, hi = nfields - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tbeg[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

}  // namespace

cudaError_t sampler_upload_tables(const unsigned int*) { return cudaSuccess; }

cudaError_t launch_sampler(const SamplerArgs& A, cudaStream_t) {
  for (long long t = 0; t < A.nthreads; ++t) sample_range(A, t, A.write);
  return cudaSuccess;
}

cudaError_t launch_sampler_batch(const SamplerArgs* fields, const long long* tbeg, int nfields, long long total,
                                 int write, cudaStream_t) {
  for (long long t = 0; t < total; ++t) {
    const int f = field_of(tbeg, nfields, t);
    sample_range(fields[f], t - tbeg[f], write);
  }
  return cudaSuccess;
}

cudaError_t launch_sampler_gather(const SamplerArgs* fields, const long long* tbeg, int nfields, long long total,
                                  const long long* offsets, SampleEntry* dst, cudaStream_t) {
  for (long long t = 0; t < total; ++t) {
    const int f = field_of(tbeg, nfields, t);
    const SamplerArgs& A = fields[f];
    const long long tl = t - tbeg[f];
    const int n = std::min(A.counts[tl], A.cap);
    const unsigned long long* src = A.keys + tl * A.cap;
    SampleEntry* o = dst + offsets[t];
    for (int i = 0; i < n; ++i) {
      const unsigned long long q = src[i] >> 2;
      Yarn2 look = at_pair(A, static_cast<long long>(q));
      SampleEntry e{};
      e.q = static_cast<long long>(q);
      e.flag = static_cast<int>(src[i] & 3u);
      for (int k = 0; k < 8; ++k) e.r[k] = Yarn2::to_u01(look.next_raw());
      o[i] = e;
    }
  }
  return cudaSuccess;
}

}  // namespace scarf

namespace {

int failures = 0;
void expect(bool ok, const char* what, int c) {
  if (!ok) {
    std::fprintf(stderr, "case %d: %s\n", c, what);
    ++failures;
  }
}

struct Case {
  int acf, nharm, seed, rescale;
  float hurst, sigma, ds, dh;
  float cl[3], fc[3];
  float alpha, beta, gamma;
};

const Case kCases[] = {
    {0, 300, 1234, 0, 0.25f, 0.05f, 50.0f, 50.0f, {2000, 2000, 2000}, {800, 600, 500}, 0, 0, 0},
    {1, 250, 7, 0, 0.0f, 0.1f, 100.0f, 100.0f, {1500, 1500, 500}, {3900, 2300, 1900}, 0, 0, 0},
    {0, 333, 99, 1, 0.5f, 0.05f, 25.0f, 25.0f, {3000, 3000, 1000}, {1375, 1175, 775}, 30, -10, 5},
    {0, 200, 11, 0, 0.3f, 0.08f, 50.0f, 20.0f, {2000, 2000, 800}, {1150, 950, 750}, 0, 0, 0},  // dh < ds: drops
    {1, 260, 1235, 0, 0.0f, 0.05f, 50.0f, 50.0f, {2000, 1200, 0}, {4950, 3450, 0}, 20, 0, 0},  // 2-D
};

scarf_srm_params params_of(const Case& k, int seed_offset) {
  scarf_srm_params p{};
  p.acf = k.acf, p.nharm = k.nharm, p.seed = k.seed + seed_offset, p.rescale = k.rescale;
  p.hurst = k.hurst, p.sigma = k.sigma, p.ds = k.ds, p.dh = k.dh;
  for (int a = 0; a < 3; ++a) p.cl[a] = k.cl[a], p.nc[a] = 0.0f, p.fc[a] = k.fc[a];
  p.alpha = k.alpha, p.beta = k.beta, p.gamma = k.gamma;
  return p;
}

// The device-assisted sampler over batches of nf fields against the serial
// host sampler: tables bit for bit, kept counts and pairs consumed equal.
int check_device_batches(const char* what) {
  int batches = 0;
  for (int nf : {1, 2, 3, 5, 9, 17, 40}) {
    std::vector<scarf_srm_params> P;
    std::vector<scarf_srm_setup> S(nf);
    for (int f = 0; f < nf; ++f) {
      P.push_back(params_of(kCases[f % 5], 1000 * nf + f));
      expect(scarf::srm_setup(P[f], &S[f]) == SCARF_OK, "srm_setup failed", f);
    }
    std::vector<std::vector<float>> tabs(nf);
    std::vector<float*> ptrs(nf);
    for (int f = 0; f < nf; ++f) {
      tabs[f].assign(5 * P[f].nharm, 0.0f);
      ptrs[f] = tabs[f].data();
    }
    std::vector<int> kept(nf, -1);
    std::vector<long long> used(nf, -1);
    long long open = 0;
    const int rc = scarf::srm_sample_device_batch(nf, P.data(), S.data(), ptrs.data(), kept.data(), used.data(),
                                                  nullptr, &open);
    expect(rc == 0, what, nf);
    for (int f = 0; f < nf; ++f) {
      std::vector<float> ref(5 * P[f].nharm);
      long long ref_pairs = 0;
      const int n = scarf::srm_sample(P[f], S[f], nullptr, 1, ref.data(), &ref_pairs);
      const bool same = kept[f] == n && used[f] == ref_pairs &&
                        !std::memcmp(tabs[f].data(), ref.data(), sizeof(float) * 5 * std::max(n, 0));
      if (!same) std::fprintf(stderr, "%s: batch of %d, field %d differs from the serial sampler\n", what, nf, f);
      expect(same, what, nf);
    }
    ++batches;
  }
  // one field through the single-field entry point
  scarf_srm_params p = params_of(kCases[2], 77);
  scarf_srm_setup s{};
  scarf::srm_setup(p, &s);
  std::vector<float> got(5 * p.nharm), ref(5 * p.nharm);
  long long gp = 0, rp = 0, unc = 0;
  const int ng = scarf::srm_sample_device(p, s, got.data(), &gp, nullptr, &unc);
  const int nr = scarf::srm_sample(p, s, nullptr, 1, ref.data(), &rp);
  expect(ng == nr && gp == rp && !std::memcmp(got.data(), ref.data(), sizeof(float) * 5 * nr), what, -2);
  return batches;
}

}  // namespace

int main() {
  int c = 0;
  for (const Case& k : kCases) {
    scarf_srm_params p{};
    p.acf = k.acf, p.nharm = k.nharm, p.seed = k.seed, p.rescale = k.rescale;
    p.hurst = k.hurst, p.sigma = k.sigma, p.ds = k.ds, p.dh = k.dh;
    for (int a = 0; a < 3; ++a) p.cl[a] = k.cl[a], p.nc[a] = 0.0f, p.fc[a] = k.fc[a];
    p.alpha = k.alpha, p.beta = k.beta, p.gamma = k.gamma;
    orc_params o{};
    o.acf = k.acf, o.nharm = k.nharm, o.seed = k.seed, o.rescale = k.rescale;
    o.hurst = k.hurst, o.sigma = k.sigma, o.ds = k.ds, o.dh = k.dh;
    for (int a = 0; a < 3; ++a) o.cl[a] = k.cl[a], o.nc[a] = 0.0f, o.fc[a] = k.fc[a];
    o.alpha = k.alpha, o.beta = k.beta, o.gamma = k.gamma;

    scarf_srm_setup s{};
    orc_setup os{};
    expect(scarf::srm_setup(p, &s) == SCARF_OK, "srm_setup failed", c);
    expect(orc_setup_compute(&o, &os) == 0, "orc_setup_compute failed", c);
    expect(s.ndim == os.ndim && s.kmin == os.kmin && s.kmax == os.kmax && s.kc == os.kc && s.nu == os.nu &&
               s.scaling == os.scaling && !std::memcmp(s.m, os.m, sizeof(s.m)) &&
               !std::memcmp(s.bar, os.bar, sizeof(s.bar)),
           "setup differs from the oracle", c);

    std::vector<float> serial(5 * k.nharm), threaded(5 * k.nharm), orc(5 * k.nharm);
    long long pairs_serial = 0, pairs_threaded = 0;
    int64_t pairs_orc = 0;
    const int n1 = scarf::srm_sample(p, s, nullptr, 1, serial.data(), &pairs_serial);
    const int n4 = scarf::srm_sample(p, s, nullptr, 4, threaded.data(), &pairs_threaded);
    const int no = orc_sample(&o, &os, orc.data(), &pairs_orc);
    expect(n1 > 0 && n1 == n4 && n1 == no, "kept counts differ", c);
    expect(pairs_serial == pairs_threaded && pairs_serial == pairs_orc, "pairs consumed differ", c);
    expect(!std::memcmp(serial.data(), threaded.data(), sizeof(float) * 5 * n1), "threaded table differs", c);
    expect(!std::memcmp(serial.data(), orc.data(), sizeof(float) * 5 * n1), "table differs from the oracle", c);

    // the oracle's whole structured execute, with rescale and a taper
    const int fs[3] = {1, 1, 1};
    const int fe[3] = {9, 7, os.ndim == 3 ? 5 : 1};
    std::vector<float> field(9 * 7 * 5);
    float info[6] = {0};
    const float poi[3] = {100.0f, 100.0f, 0.0f};
    expect(orc_execute_structured(&o, fs, fe, poi, 1, 50.0f, 200.0f, field.data(), info, 2) == 0,
           "orc_execute_structured failed", c);
    ++c;
  }

  // Device-assisted sampler (emulated device): as it runs, with one candidate
  // slot per scan thread (most fields overflow and are redone alone), and
  // with short passes (most fields need further passes).
  int batches = check_device_batches("device sampler");
  setenv("SCARF3D_B200_SAMPLER_SLOT_CAP", "1", 1);
  batches += check_device_batches("device sampler, overflowing slots");
  unsetenv("SCARF3D_B200_SAMPLER_SLOT_CAP");
  scarf::set_device_sampler_pass_cap(1500);
  batches += check_device_batches("device sampler, short passes");
  scarf::set_device_sampler_pass_cap(0);

  // Worker pool: jobs of every width, from two caller threads at once.
  auto jobs = [](int base, std::atomic<long long>* sum) {
    for (int w = 1; w <= 9; ++w)
      for (int n : {0, 1, 3, 64, 1000}) {
        std::vector<int> hit(n, 0);
        scarf::parallel_tasks(n, w, [&](int i) { hit[i] += 1; });
        for (int i = 0; i < n; ++i) *sum += hit[i] * (base + i);
      }
  };
  std::atomic<long long> s1{0}, s2{0};
  std::thread t1(jobs, 1, &s1), t2(jobs, 2, &s2);
  t1.join();
  t2.join();
  long long want1 = 0, want2 = 0;
  for (int w = 1; w <= 9; ++w)
    for (int n : {0, 1, 3, 64, 1000})
      for (int i = 0; i < n; ++i) want1 += 1 + i, want2 += 2 + i;
  expect(s1 == want1 && s2 == want2, "worker pool ran a task other than once", -1);

  // A task that throws: every other task still runs, and the caller gets the
  // exception once all have returned.
  {
    std::vector<int> hit(200, 0);
    bool caught = false;
    try {
      scarf::parallel_tasks(200, 6, [&](int i) {
        hit[i] = 1;
        if (i == 17) throw std::runtime_error("task 17");
      });
    } catch (const std::runtime_error& e) {
      caught = std::strcmp(e.what(), "task 17") == 0;
    }
    int ran = 0;
    for (int h : hit) ran += h;
    expect(caught && ran == 200, "a throwing task lost other tasks or its exception", -1);
  }

  std::printf("%d cases, %d device-sampler batches, %d failures\n", c, batches, failures);
  return failures ? 1 : 0;
}
