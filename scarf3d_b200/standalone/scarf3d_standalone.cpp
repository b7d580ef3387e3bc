// scarf3d_standalone -- keyword-file driver of the SRM library, the counterpart
// of the reference's standalone application (standalone/main.f90).
//
//   scarf3d_standalone <input file>            compute the field on one GPU and
//                                              write random_field.bin (raw
//                                              column-major FP32, x fastest)
//   scarf3d_standalone --check <input file>    parse and validate only, print
//                                              the summary (no device work)
//
// Input format (standalone/main.f90:141-221): a line holding exactly one of the
// descriptors below (leading blanks make it a different line, trailing blanks
// do not count) is followed by its value(s), read list-directed from the next
// line(s): blanks, tabs or commas separate values, "r*v" repeats v r times.
//   # dimension  2 or 3              # npts      ndim integers
//   # ds         grid step (m)       # cl        ndim correlation lengths
//   # sigma      standard deviation  # acf       0 von Karman, 1 Gaussian
//   # hurst      Hurst exponent      # seed      non-zero integer
//   # poi        ndim coordinates (one line per point of interest)
//   # mute, # taper                  radii around the points of interest
//   # rescale    0 or 1              # pad       0 or 1 (FIM option)
//   # alpha, # beta, # gamma         rotation angles (degrees)
//   # method     0 FIM, 1 SRM        # nwriters  I/O processes (> 0)
// Defaults and checks follow main.f90:111-127 and 270-345, including their
// messages; as in the reference, the Hurst-range check can never fire
// (main.f90:333: hurst < 0 .and. hurst > 1). The reference's default method
// is FIM (0); both methods run here. One process computes the whole grid
// (fs = 1, fe = npts), where the reference splits it over MPI ranks.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "scarf3d.h"
#include "scarf3d_b200.h"

namespace {

struct Input {
  int ndim = 0;
  std::vector<int> n;
  std::vector<float> cl;
  std::vector<std::vector<float>> poi;
  float ds = 0.0f, sigma = -1.0f, hurst = -1.0f, mute = 0.0f, taper = 0.0f;
  float alpha = 0.0f, beta = 0.0f, gamma = 0.0f;
  int acf = -1, seed = 0, rescale = 0, pad = 0, method = 0, nwriters = 2;
};

std::string rtrim(const std::string& s) {
  size_t e = s.find_last_not_of(" \t\r\n");
  return e == std::string::npos ? std::string() : s.substr(0, e + 1);
}

// List-directed reader over the lines that follow a descriptor.
class Values {
 public:
  Values(const std::vector<std::string>& lines, size_t next) : lines_(lines), line_(next) {}
  // Next value as text, or empty when the file ends first.
  std::string next() {
    while (pending_.empty()) {
      if (line_ >= lines_.size()) return std::string();
      std::string l = lines_[line_++];
      for (char& c : l)
        if (c == ',' || c == '\t') c = ' ';
      std::istringstream is(l);
      std::string tok;
      while (is >> tok) {
        if (tok == "/") break;  // list terminator
        const size_t star = tok.find('*');
        if (star != std::string::npos && star > 0) {
          const int r = std::atoi(tok.substr(0, star).c_str());
          for (int k = 0; k < r; ++k) pending_.push_back(tok.substr(star + 1));
        } else {
          pending_.push_back(tok);
        }
      }
    }
    std::string v = pending_.front();
    pending_.erase(pending_.begin());
    return v;
  }

 private:
  const std::vector<std::string>& lines_;
  size_t line_;
  std::vector<std::string> pending_;
};

bool read_ints(Values v, int count, std::vector<int>& out) {
  out.assign(count, 0);
  for (int i = 0; i < count; ++i) {
    const std::string t = v.next();
    if (t.empty()) return false;
    out[i] = static_cast<int>(std::strtol(t.c_str(), nullptr, 10));
  }
  return true;
}
bool read_floats(Values v, int count, std::vector<float>& out) {
  out.assign(count, 0.0f);
  for (int i = 0; i < count; ++i) {
    std::string t = v.next();
    if (t.empty()) return false;
    for (char& c : t)
      if (c == 'd' || c == 'D') c = 'e';  // Fortran double-precision exponents
    out[i] = std::strtof(t.c_str(), nullptr);
  }
  return true;
}

// Returns 0, or 1 with a message printed (the reference aborts with code 1).
int parse(const char* path, Input& in) {
  std::ifstream f(path);
  if (!f) {
    std::printf(" Error: cannot open input file %s\n", path);
    return 1;
  }
  std::vector<std::string> lines;
  for (std::string l; std::getline(f, l);) lines.push_back(rtrim(l.substr(0, 100)));
  for (size_t i = 0; i < lines.size(); ++i) {
    if (lines[i] == "# dimension") {
      std::vector<int> d;
      if (read_ints(Values(lines, i + 1), 1, d)) in.ndim = d[0];
    }
  }
  if (in.ndim != 2 && in.ndim != 3) {
    std::printf(" Error: dimension must be equal to 2 or 3\n");
    return 1;
  }
  const int nd = in.ndim;
  in.n.assign(nd, 0);
  in.cl.assign(nd, 0.0f);
  for (size_t i = 0; i < lines.size(); ++i) {
    const std::string& key = lines[i];
    Values v(lines, i + 1);
    std::vector<int> iv;
    std::vector<float> fv;
    if (key == "# npts") {
      if (read_ints(v, nd, iv)) in.n = iv;
    } else if (key == "# poi") {
      std::vector<float> p(nd, -1.0f);
      if (read_floats(v, nd, fv)) p = fv;
      in.poi.push_back(p);
    } else if (key == "# cl") {
      if (read_floats(v, nd, fv)) in.cl = fv;
    } else {
      struct F { const char* k; float* p; } floats[] = {{"# ds", &in.ds}, {"# sigma", &in.sigma}, {"# hurst", &in.hurst},
                                                        {"# mute", &in.mute}, {"# taper", &in.taper}, {"# alpha", &in.alpha},
                                                        {"# beta", &in.beta}, {"# gamma", &in.gamma}};
      struct I { const char* k; int* p; } ints[] = {{"# acf", &in.acf}, {"# seed", &in.seed}, {"# rescale", &in.rescale},
                                                    {"# pad", &in.pad}, {"# method", &in.method}, {"# nwriters", &in.nwriters}};
      for (const F& e : floats)
        if (key == e.k && read_floats(v, 1, fv)) *e.p = fv[0];
      for (const I& e : ints)
        if (key == e.k && read_ints(v, 1, iv)) *e.p = iv[0];
    }
  }
  auto fail = [](const char* msg) {
    std::printf(" %s\n", msg);
    return 1;
  };
  for (int v : in.n)
    if (v <= 0) return fail("Error: number of points must be larger than zero");
  for (const auto& p : in.poi)
    for (float c : p)
      if (c < 0.0f) return fail("Error: POI must be inside the model");
  if (in.acf != 0 && in.acf != 1) return fail("Error: accepted ACF are Von Karman (0) and Gaussian (1)");
  if (in.mute < 0.0f) return fail("Error: mute parameter can be only positive");
  if (in.taper < 0.0f) return fail("Error: taper parameter can be only positive");
  if (in.rescale != 0 && in.rescale != 1) return fail("Error: rescale parameter can be only off (0) or on (1)");
  if (in.nwriters <= 0) return fail("Error: nwriters parameter can be only larger than zero");
  if (in.sigma <= 0.0f) return fail("Error: standard deviation (sigma) must be larger than zero");
  if (in.ds <= 0.0f) return fail("Error: grid-step must be larger than zero");
  if (in.acf == 0 && in.hurst < 0.0f && in.hurst > 1.0f) return fail("Error: Hurst exponent must be in the range [0 1]");
  if (in.seed == 0) return fail("Error: seed number (any integer not equal zero) not specified");
  return 0;
}

void summary(const Input& in) {
  auto row_i = [](const char* k, long long v) { std::printf(" %-26s|%12lld%24s|\n", k, v, ""); };
  auto row_f = [](const char* k, double v) { std::printf(" %-26s|%12.3f%24s|\n", k, v, ""); };
  auto rule = []() { std::printf(" --------------------------|------------------------------------|\n"); };
  std::printf("\n Summary of input parameters\n ****************************************************************\n");
  row_i("Number of dimensions", in.ndim);
  rule();
  row_i("method", in.method);
  rule();
  std::printf(" %-26s|", "Number of points");
  for (int v : in.n) std::printf("%12d", v);
  std::printf("\n");
  rule();
  row_f("Grid-step", in.ds);
  rule();
  row_i("Auto-correlation function", in.acf);
  std::printf(" %-26s|", "Correlation length");
  for (float v : in.cl) std::printf("%12.3f", v);
  std::printf("\n");
  row_f("Std. dev.", in.sigma);
  if (in.acf == 0) {
    row_f("Hurst exponent", in.hurst);
    rule();
  }
  row_i("Seed number", in.seed);
  rule();
  if (!in.poi.empty()) {
    row_i("Number of POIs", static_cast<long long>(in.poi.size()));
    row_f("Muting radius", in.mute);
    row_f("Tapering radius", in.taper);
    rule();
  }
  row_f("Alpha angle", in.alpha);
  row_f("Beta angle", in.beta);
  row_f("Gamma angle", in.gamma);
  rule();
  row_i("MPI processes for I/O", in.nwriters);
  std::printf(" ****************************************************************\n\n");
  std::fflush(stdout);
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char** argv) {
  const bool check = argc == 3 && std::string(argv[1]) == "--check";
  if (!(argc == 2 || check)) {
    std::printf(" Please specify an input file!\n");
    return 0;
  }
  Input in;
  if (parse(argv[argc - 1], in) != 0) return 1;
  summary(in);
  if (check) return 0;

  const int nd = in.ndim;
  int fs[3] = {1, 1, 1}, fe[3] = {1, 1, 1};
  long long npts = 1;
  for (int a = 0; a < nd; ++a) {
    fe[a] = in.n[a];
    npts *= in.n[a];
  }
  std::vector<float> poi;
  for (const auto& p : in.poi) poi.insert(poi.end(), p.begin(), p.end());
  scarf_opt opt;
  scarf_opt_init(&opt);
  opt.method = in.method;
  opt.hurst = in.hurst;
  opt.alpha = in.alpha;
  opt.beta = in.beta;
  opt.gamma = in.gamma;
  opt.rescale = in.rescale;
  opt.pad = in.pad;
  if (!poi.empty()) {
    opt.poi = poi.data();
    opt.npoi = static_cast<int>(in.poi.size());
    opt.mute = in.mute;
    opt.taper = in.taper;
  }
  scarf_cart_initialize(nd, fs, fe, in.ds, in.acf, in.cl.data(), in.sigma, &opt);
  std::vector<float> field(static_cast<size_t>(npts));
  float stats[8] = {0};
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = scarf_execute_ex(in.seed, field.data(), stats, 0);
  const double t_exec = seconds_since(t0);
  if (rc != SCARF_OK) {
    std::printf(" Error: %s\n", scarf_last_error());
    scarf_finalize();
    return 1;
  }
  std::printf("\n %-35s\n *************************************************\n", "Statistics for current simulation");
  std::printf(" %-30s|%12.5f sec|\n", "Elapsed time", t_exec);
  std::printf(" ------------------------------|-----------------|\n");
  std::printf(" %-30s|%12s%5s|\n", "Domain too small?", std::lround(stats[0]) != 0 ? "T" : "F", "");
  std::printf(" %-30s|%12s%5s|\n", "Grid-step too large?", std::lround(stats[1]) != 0 ? "T" : "F", "");
  std::printf(" ------------------------------|-----------------|\n");
  std::printf(" %-30s|%12.5f%5s|\n", "Discrete standard deviation", stats[2], "");
  std::printf(" %-30s|%12.5f%5s|\n", "Discrete mean value", stats[3], "");
  std::printf(" ------------------------------|-----------------|\n");
  const auto t1 = std::chrono::steady_clock::now();
  scarf_io_one(nd, in.n.data(), field.data(), "random_field.bin", &in.nwriters);
  std::printf(" %-30s|%12.5f sec|\n", "I/O time", seconds_since(t1));
  std::printf(" *************************************************\n\n");
  scarf_finalize();
  std::printf("\n Program completed successfully\n");
  return 0;
}
