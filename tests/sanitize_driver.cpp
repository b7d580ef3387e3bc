// Host code of the library and the C oracle under AddressSanitizer and
// UndefinedBehaviorSanitizer (built and run by test_sanitizers.py, no GPU).
// Exercises setup, quadrature, the serial and multi-threaded samplers and the
// host worker pool, and cross-checks them against the oracle bit for bit;
// any sanitizer report aborts the run. The device launchers the sampler
// references are stubbed: nothing here reaches a GPU.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../oracle/srm_oracle.h"
#include "srm_host.h"
#include "srm_kernels.h"

namespace scarf {
cudaError_t sampler_upload_tables(const unsigned int*) { return cudaErrorNoDevice; }
cudaError_t launch_sampler(const SamplerArgs&, cudaStream_t) { return cudaErrorNoDevice; }
cudaError_t launch_sampler_batch(const SamplerArgs*, const long long*, int, long long, int, cudaStream_t) {
  return cudaErrorNoDevice;
}
cudaError_t launch_sampler_gather(const SamplerArgs*, const long long*, int, long long, const long long*,
                                  SampleEntry*, cudaStream_t) {
  return cudaErrorNoDevice;
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

  std::printf("%d cases, %d failures\n", c, failures);
  return failures ? 1 : 0;
}
