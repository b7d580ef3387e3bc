// QUADPACK routines used by the SRM scaling (quadpack.f90): DQNG (:8137),
// DQAGI (:1177) -> DQAGIE (:712) with DQK15I (:6589), DQELG (:6230) and
// DQPSRT (:8529). The SRM scaling sqrt(intg(kmin,kmax)/intg(0,inf)) sets the
// field's absolute scale at the 1e-5 level (epsrel = 1e-5), so the same
// routines with the same control flow are restated here; the node and weight
// tables are the published Gauss-Kronrod(-Patterson) constants
// (Piessens et al., QUADPACK, 1983).
#include <cfloat>
#include <cmath>
#include <vector>

#include "srm_host.h"

namespace scarf {
namespace {

struct Integrand {
  int ndim, acf;
  float nu;
  double operator()(double x) const { return srm_fn(x, ndim, acf, nu); }
};

constexpr double kX1[5] = {0.973906528517171720077964012084452, 0.865063366688984510732096688423493,
                           0.679409568299024406234327365114874, 0.433395394129247190799265943165784,
                           0.148874338981631210884826001129720};
constexpr double kW10[5] = {0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
                            0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
                            0.295524224714752870173892994651338};
constexpr double kX2[5] = {0.995657163025808080735527280689003, 0.930157491355708226001207180059508,
                           0.780817726586416897063717578345042, 0.562757134668604683339000099272694,
                           0.294392862701460198131126603103866};
constexpr double kW21a[5] = {0.032558162307964727478818972459390, 0.075039674810919952767043140916190,
                             0.109387158802297641899210590325805, 0.134709217311473325928054001771707,
                             0.147739104901338491374841515972068};
constexpr double kW21b[6] = {0.011694638867371874278064396062192, 0.054755896574351996031381300244580,
                             0.093125454583697605535065465083366, 0.123491976262065851077958109831074,
                             0.142775938577060080797094273138717, 0.149445554002916905664936468389821};
constexpr double kX3[11] = {0.999333360901932081394099323919911, 0.987433402908088869795961478381209,
                            0.954807934814266299257919200290473, 0.900148695748328293625099494069092,
                            0.825198314983114150847066732588520, 0.732148388989304982612354848755461,
                            0.622847970537725238641159120344323, 0.499479574071056499952214885499755,
                            0.364901661346580768043989548502644, 0.222254919776601296498260928066212,
                            0.074650617461383322043914435796506};
constexpr double kW43a[10] = {0.016296734289666564924281974617663, 0.037522876120869501461613795898115,
                              0.054694902058255442147212685465005, 0.067355414609478086075553166302174,
                              0.073870199632393953432140695251367, 0.005768556059769796184184327908655,
                              0.027371890593248842081276069289151, 0.046560826910428830743339154433824,
                              0.061744995201442564496240336030883, 0.071387267268693397768559114425516};
constexpr double kW43b[12] = {0.001844477640212414100389106552965, 0.010798689585891651740465406741293,
                              0.021895363867795428102523123075149, 0.032597463975345689443882222526137,
                              0.042163137935191811847627924327955, 0.050741939600184577780189020092084,
                              0.058379395542619248375475369330206, 0.064746404951445885544689259517511,
                              0.069566197912356484528633315038405, 0.072824441471833208150939535192842,
                              0.074507751014175118273571813842889, 0.074722147517403005594425168280423};
constexpr double kX4[22] = {0.999902977262729234490529830591582, 0.997989895986678745427496322365960,
                            0.992175497860687222808523352251425, 0.981358163572712773571916941623894,
                            0.965057623858384619128284110607926, 0.943167613133670596816416634507426,
                            0.915806414685507209591826430720050, 0.883221657771316501372117548744163,
                            0.845710748462415666605902011504855, 0.803557658035230982788739474980964,
                            0.757005730685495558328942793432020, 0.706273209787321819824094274740840,
                            0.651589466501177922534422205016736, 0.593223374057961088875273770349144,
                            0.531493605970831932285268948562671, 0.466763623042022844871966781659270,
                            0.399424847859218804732101665817923, 0.329874877106188288265053371824597,
                            0.258503559202161551802280975429025, 0.185695396568346652015917141167606,
                            0.111842213179907468172398359241362, 0.037352123394619870814998165437704};
constexpr double kW87a[21] = {0.008148377384149172900002878448190, 0.018761438201562822243935059003794,
                              0.027347451050052286161582829741283, 0.033677707311637930046581056957588,
                              0.036935099820427907614589586742499, 0.002884872430211530501334156248695,
                              0.013685946022712701888950035273128, 0.023280413502888311123409291030404,
                              0.030872497611713358675466394126442, 0.035693633639418770719351355457044,
                              0.000915283345202241360843392549948, 0.005399280219300471367738743391053,
                              0.010947679601118931134327826856808, 0.016298731696787335262665703223280,
                              0.021081568889203835112433060188190, 0.025370969769253827243467999831710,
                              0.029189697756475752501446154084920, 0.032373202467202789685788194889595,
                              0.034783098950365142750781997949596, 0.036412220731351787562801163687577,
                              0.037253875503047708539592001191226};
constexpr double kW87b[23] = {0.000274145563762072350016527092881, 0.001807124155057942948341311753254,
                              0.004096869282759164864458070683480, 0.006758290051847378699816577897424,
                              0.009549957672201646536053581325377, 0.012329447652244853694626639963780,
                              0.015010447346388952376697286041943, 0.017548967986243191099665352925900,
                              0.019938037786440888202278192730714, 0.022194935961012286796332102959499,
                              0.024339147126000805470360647041454, 0.026374505414839207241503786552615,
                              0.028286910788771200659968002987960, 0.030052581128092695322521110347341,
                              0.031646751371439929404586051078883, 0.033050413419978503290785944862689,
                              0.034255099704226061787082821046821, 0.035262412660156681033782717998428,
                              0.036076989622888701185500318003895, 0.036698604498456094498018047441094,
                              0.037120549269832576114119958413599, 0.037334228751935040321235449094698,
                              0.037361073762679023410321241766599};
constexpr double kWg15[8] = {0.0, 0.129484966168869693270611432679082, 0.0, 0.279705391489276667901467771423780,
                             0.0, 0.381830050505118944950369775488975, 0.0, 0.417959183673469387755102040816327};
constexpr double kXgk15[8] = {0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                              0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                              0.586087235467691130294144838258730, 0.405845151377397166906606412076961,
                              0.207784955007898467600689403773245, 0.0};
constexpr double kWgk15[8] = {0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                              0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                              0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                              0.204432940075298892414161999234649, 0.209482141084727828012999174891714};

constexpr double kEps = DBL_EPSILON;

// Error-estimate refinement shared by the Kronrod rules.
inline double refine_err(double abserr, double resabs, double resasc) {
  if (resasc != 0.0 && abserr != 0.0) abserr = resasc * std::fmin(1.0, std::pow(200.0 * abserr / resasc, 1.5));
  if (resabs > DBL_MIN / (50.0 * kEps)) abserr = std::fmax((kEps * 50.0) * resabs, abserr);
  return abserr;
}

int dqng(const Integrand& f, double a, double b, double epsabs, double epsrel, double* result, double* abserr) {
  double fv1[5], fv2[5], fv3[5], fv4[5], savfun[21];
  double res10 = 0, res21 = 0, res43 = 0, resabs = 0, resasc = 0;
  *result = 0.0;
  *abserr = 0.0;
  if (epsabs <= 0.0 && epsrel < std::fmax(50.0 * kEps, 0.5e-28)) return 6;
  const double hlgth = 0.5 * (b - a), dhlgth = std::fabs(hlgth), centr = 0.5 * (b + a);
  const double fcentr = f(centr);
  int ipx = 0;
  for (int rule = 1; rule <= 3; ++rule) {
    if (rule == 1) {
      res10 = 0.0;
      res21 = kW21b[5] * fcentr;
      resabs = kW21b[5] * std::fabs(fcentr);
      for (int k = 0; k < 5; ++k) {
        const double absc = hlgth * kX1[k];
        const double f1 = f(centr + absc), f2 = f(centr - absc), fs = f1 + f2;
        res10 = res10 + kW10[k] * fs;
        res21 = res21 + kW21a[k] * fs;
        resabs = resabs + kW21a[k] * (std::fabs(f1) + std::fabs(f2));
        savfun[k] = fs;
        fv1[k] = f1;
        fv2[k] = f2;
      }
      ipx = 5;
      for (int k = 0; k < 5; ++k) {
        ++ipx;
        const double absc = hlgth * kX2[k];
        const double f1 = f(centr + absc), f2 = f(centr - absc), fs = f1 + f2;
        res21 = res21 + kW21b[k] * fs;
        resabs = resabs + kW21b[k] * (std::fabs(f1) + std::fabs(f2));
        savfun[ipx - 1] = fs;
        fv3[k] = f1;
        fv4[k] = f2;
      }
      *result = res21 * hlgth;
      resabs = resabs * dhlgth;
      const double reskh = 0.5 * res21;
      resasc = kW21b[5] * std::fabs(fcentr - reskh);
      for (int k = 0; k < 5; ++k)
        resasc = resasc + kW21a[k] * (std::fabs(fv1[k] - reskh) + std::fabs(fv2[k] - reskh)) +
                 kW21b[k] * (std::fabs(fv3[k] - reskh) + std::fabs(fv4[k] - reskh));
      *abserr = std::fabs((res21 - res10) * hlgth);
      resasc = resasc * dhlgth;
    } else if (rule == 2) {
      res43 = kW43b[11] * fcentr;
      for (int k = 0; k < 10; ++k) res43 = res43 + savfun[k] * kW43a[k];
      for (int k = 0; k < 11; ++k) {
        ++ipx;
        const double absc = hlgth * kX3[k];
        const double fs = f(absc + centr) + f(centr - absc);
        res43 = res43 + fs * kW43b[k];
        savfun[ipx - 1] = fs;
      }
      *result = res43 * hlgth;
      *abserr = std::fabs((res43 - res21) * hlgth);
    } else {
      double res87 = kW87b[22] * fcentr;
      for (int k = 0; k < 21; ++k) res87 = res87 + savfun[k] * kW87a[k];
      for (int k = 0; k < 22; ++k) {
        const double absc = hlgth * kX4[k];
        res87 = res87 + kW87b[k] * (f(absc + centr) + f(centr - absc));
      }
      *result = res87 * hlgth;
      *abserr = std::fabs((res87 - res43) * hlgth);
    }
    *abserr = refine_err(*abserr, resabs, resasc);
    if (*abserr <= std::fmax(epsabs, epsrel * std::fabs(*result))) return 0;
  }
  return 1;
}

void dqk15i(const Integrand& f, double boun, int inf, double a, double b, double* result, double* abserr,
            double* resabs, double* resasc) {
  double fv1[7], fv2[7];
  const double dinf = static_cast<double>(inf < 1 ? inf : 1);
  const double centr = 0.5 * (a + b), hlgth = 0.5 * (b - a);
  const double t0 = boun + dinf * (1.0 - centr) / centr;
  double fval = f(t0);
  if (inf == 2) fval = fval + f(-t0);
  const double fc = (fval / centr) / centr;
  double resg = kWg15[7] * fc, resk = kWgk15[7] * fc;
  *resabs = std::fabs(resk);
  for (int j = 0; j < 7; ++j) {
    const double absc = hlgth * kXgk15[j];
    const double x1 = centr - absc, x2 = centr + absc;
    const double t1 = boun + dinf * (1.0 - x1) / x1, t2 = boun + dinf * (1.0 - x2) / x2;
    double f1 = f(t1), f2 = f(t2);
    if (inf == 2) f1 = f1 + f(-t1);
    if (inf == 2) f2 = f2 + f(-t2);
    f1 = (f1 / x1) / x1;
    f2 = (f2 / x2) / x2;
    fv1[j] = f1;
    fv2[j] = f2;
    const double fs = f1 + f2;
    resg = resg + kWg15[j] * fs;
    resk = resk + kWgk15[j] * fs;
    *resabs = *resabs + kWgk15[j] * (std::fabs(f1) + std::fabs(f2));
  }
  const double reskh = resk * 0.5;
  *resasc = kWgk15[7] * std::fabs(fc - reskh);
  for (int j = 0; j < 7; ++j) *resasc = *resasc + kWgk15[j] * (std::fabs(fv1[j] - reskh) + std::fabs(fv2[j] - reskh));
  *result = resk * hlgth;
  *resasc = *resasc * hlgth;
  *resabs = *resabs * hlgth;
  *abserr = refine_err(std::fabs((resk - resg) * hlgth), *resabs, *resasc);
}

// Keeps iord[1..] ordered by decreasing error (1-based arrays).
void dqpsrt(int limit, int last, int* maxerr, double* ermax, const double* elist, int* iord, int* nrmax) {
  if (last <= 2) {
    iord[1] = 1;
    iord[2] = 2;
  } else {
    const double errmax = elist[*maxerr];
    const int ido = *nrmax - 1;
    for (int i = 1; i <= ido; ++i) {
      const int isucc = iord[*nrmax - 1];
      if (errmax <= elist[isucc]) break;
      iord[*nrmax] = isucc;
      --(*nrmax);
    }
    int jupbn = last;
    if (last > (limit / 2 + 2)) jupbn = limit + 3 - last;
    const double errmin = elist[last];
    const int jbnd = jupbn - 1;
    int i = *nrmax + 1;
    bool inserted = false;
    for (; i <= jbnd; ++i) {
      const int isucc = iord[i];
      if (errmax >= elist[isucc]) {
        inserted = true;
        break;
      }
      iord[i - 1] = isucc;
    }
    if (!inserted) {
      iord[jbnd] = *maxerr;
      iord[jupbn] = last;
    } else {
      iord[i - 1] = *maxerr;
      int k = jbnd;
      bool placed = false;
      for (int j = i; j <= jbnd; ++j) {
        const int isucc = iord[k];
        if (errmin < elist[isucc]) {
          iord[k + 1] = last;
          placed = true;
          break;
        }
        iord[k + 1] = isucc;
        --k;
      }
      if (!placed) iord[i] = last;
    }
  }
  *maxerr = iord[*nrmax];
  *ermax = elist[*maxerr];
}

// Wynn epsilon extrapolation (1-based epstab[1..52], res3la[1..3]).
void dqelg(int* n, double* epstab, double* result, double* abserr, double* res3la, int* nres) {
  const double oflow = DBL_MAX;
  ++(*nres);
  *abserr = oflow;
  *result = epstab[*n];
  if (*n >= 3) {
    const int limexp = 50;
    epstab[*n + 2] = epstab[*n];
    const int newelm = (*n - 1) / 2;
    epstab[*n] = oflow;
    const int num = *n;
    int k1 = *n;
    bool converged = false;
    for (int i = 1; i <= newelm; ++i) {
      const int k2 = k1 - 1, k3 = k1 - 2;
      double res = epstab[k1 + 2];
      const double e0 = epstab[k3], e1 = epstab[k2], e2 = res;
      const double e1abs = std::fabs(e1);
      const double delta2 = e2 - e1, err2 = std::fabs(delta2), tol2 = std::fmax(std::fabs(e2), e1abs) * kEps;
      const double delta3 = e1 - e0, err3 = std::fabs(delta3), tol3 = std::fmax(e1abs, std::fabs(e0)) * kEps;
      if (!(err2 > tol2 || err3 > tol3)) {
        *result = res;
        *abserr = err2 + err3;
        converged = true;
        break;
      }
      const double e3 = epstab[k1];
      epstab[k1] = e1;
      const double delta1 = e1 - e3, err1 = std::fabs(delta1), tol1 = std::fmax(e1abs, std::fabs(e3)) * kEps;
      bool shrink = (err1 <= tol1 || err2 <= tol2 || err3 <= tol3);
      double ss = 0.0;
      if (!shrink) {
        ss = 1.0 / delta1 + 1.0 / delta2 - 1.0 / delta3;
        shrink = !(std::fabs(ss * e1) > 1.0e-4);
      }
      if (shrink) {
        *n = i + i - 1;
        break;
      }
      res = e1 + 1.0 / ss;
      epstab[k1] = res;
      k1 = k1 - 2;
      const double error = err2 + std::fabs(res - e2) + err3;
      if (error <= *abserr) {
        *abserr = error;
        *result = res;
      }
    }
    if (!converged) {
      if (*n == limexp) *n = 2 * (limexp / 2) - 1;
      int ib = ((num / 2) * 2 == num) ? 2 : 1;
      const int ie = newelm + 1;
      for (int i = 1; i <= ie; ++i) {
        epstab[ib] = epstab[ib + 2];
        ib += 2;
      }
      if (num != *n) {
        int indx = num - *n + 1;
        for (int i = 1; i <= *n; ++i) epstab[i] = epstab[indx++];
      }
      if (*nres < 4) {
        res3la[*nres] = *result;
        *abserr = oflow;
      } else {
        *abserr = std::fabs(*result - res3la[3]) + std::fabs(*result - res3la[2]) + std::fabs(*result - res3la[1]);
        res3la[1] = res3la[2];
        res3la[2] = res3la[3];
        res3la[3] = *result;
      }
    }
  }
  *abserr = std::fmax(*abserr, 5.0 * kEps * std::fabs(*result));
}

int dqagie(const Integrand& f, double bound, int inf, double epsabs, double epsrel, int limit, double* result,
           double* abserr) {
  std::vector<double> alist(limit + 1), blist(limit + 1), rlist(limit + 1), elist(limit + 1);
  std::vector<int> iord(limit + 1);
  double rlist2[56] = {0}, res3la[4] = {0};
  double area = 0, area1, area2, a1, a2, b1 = 0, b2, correc = 0, defabs, defab1, defab2, erlarg = 0, erlast,
         errbnd, errmax = 0, error1, error2, erro12 = 0, errsum = 0, ertest = 0, resabs, reseps, abseps,
         small = 0;
  const double oflow = DBL_MAX, uflow = DBL_MIN;
  int ier = 0, ierro = 0, iroff1 = 0, iroff2 = 0, iroff3 = 0, ksgn = -1, ktmin = 0, maxerr = 1, nres = 0,
      nrmax = 1, numrl2 = 2, last = 0;
  bool extrap = false, noext = false;
  *result = 0.0;
  *abserr = 0.0;
  alist[1] = 0.0;
  blist[1] = 1.0;
  if (epsabs <= 0.0 && epsrel < std::fmax(50.0 * kEps, 0.5e-28)) return 6;
  const double boun = (inf == 2) ? 0.0 : bound;
  dqk15i(f, boun, inf, 0.0, 1.0, result, abserr, &defabs, &resabs);
  last = 1;
  rlist[1] = *result;
  elist[1] = *abserr;
  iord[1] = 1;
  const double dres = std::fabs(*result);
  errbnd = std::fmax(epsabs, epsrel * dres);
  if (*abserr <= 100.0 * kEps * defabs && *abserr > errbnd) ier = 2;
  if (limit == 1) ier = 1;
  if (ier != 0 || (*abserr <= errbnd && *abserr != resabs) || *abserr == 0.0) goto finish;
  rlist2[1] = *result;
  errmax = *abserr;
  maxerr = 1;
  area = *result;
  errsum = *abserr;
  *abserr = oflow;
  if (dres >= (1.0 - 50.0 * kEps) * defabs) ksgn = 1;
  for (last = 2; last <= limit; ++last) {
    a1 = alist[maxerr];
    b1 = 0.5 * (alist[maxerr] + blist[maxerr]);
    a2 = b1;
    b2 = blist[maxerr];
    erlast = errmax;
    dqk15i(f, boun, inf, a1, b1, &area1, &error1, &resabs, &defab1);
    dqk15i(f, boun, inf, a2, b2, &area2, &error2, &resabs, &defab2);
    const double area12 = area1 + area2;
    erro12 = error1 + error2;
    errsum = errsum + erro12 - errmax;
    area = area + area12 - rlist[maxerr];
    if (!(defab1 == error1 || defab2 == error2)) {
      if (!(std::fabs(rlist[maxerr] - area12) > 0.1e-4 * std::fabs(area12) || erro12 < 0.99 * errmax)) {
        if (extrap) ++iroff2;
        if (!extrap) ++iroff1;
      }
      if (last > 10 && erro12 > errmax) ++iroff3;
    }
    rlist[maxerr] = area1;
    rlist[last] = area2;
    errbnd = std::fmax(epsabs, epsrel * std::fabs(area));
    if (iroff1 + iroff2 >= 10 || iroff3 >= 20) ier = 2;
    if (iroff2 >= 5) ierro = 3;
    if (last == limit) ier = 1;
    if (std::fmax(std::fabs(a1), std::fabs(b2)) <= (1.0 + 100.0 * kEps) * (std::fabs(a2) + 1000.0 * uflow)) ier = 4;
    if (error2 > error1) {
      alist[maxerr] = a2;
      alist[last] = a1;
      blist[last] = b1;
      rlist[maxerr] = area2;
      rlist[last] = area1;
      elist[maxerr] = error2;
      elist[last] = error1;
    } else {
      alist[last] = a2;
      blist[maxerr] = b1;
      blist[last] = b2;
      elist[maxerr] = error1;
      elist[last] = error2;
    }
    dqpsrt(limit, last, &maxerr, &errmax, elist.data(), iord.data(), &nrmax);
    if (errsum <= errbnd) goto sum_all;
    if (ier != 0) goto post;
    if (last == 2) {
      small = 0.375;
      erlarg = errsum;
      ertest = errbnd;
      rlist2[2] = area;
      continue;
    }
    if (noext) continue;
    erlarg = erlarg - erlast;
    if (std::fabs(b1 - a1) > small) erlarg = erlarg + erro12;
    if (!extrap) {
      if (std::fabs(blist[maxerr] - alist[maxerr]) > small) continue;
      extrap = true;
      nrmax = 2;
    }
    if (!(ierro == 3 || erlarg <= ertest)) {
      const int id = nrmax;
      int jupbnd = last;
      if (last > (2 + limit / 2)) jupbnd = limit + 3 - last;
      bool leave = false;
      for (int k = id; k <= jupbnd; ++k) {
        maxerr = iord[nrmax];
        errmax = elist[maxerr];
        if (std::fabs(blist[maxerr] - alist[maxerr]) > small) {
          leave = true;
          break;
        }
        ++nrmax;
      }
      if (leave) continue;
    }
    ++numrl2;
    rlist2[numrl2] = area;
    dqelg(&numrl2, rlist2, &reseps, &abseps, res3la, &nres);
    ++ktmin;
    if (ktmin > 5 && *abserr < 0.1e-2 * errsum) ier = 5;
    if (abseps < *abserr) {
      ktmin = 0;
      *abserr = abseps;
      *result = reseps;
      correc = erlarg;
      ertest = std::fmax(epsabs, epsrel * std::fabs(reseps));
      if (*abserr <= ertest) goto post;
    }
    if (numrl2 == 1) noext = true;
    if (ier == 5) goto post;
    maxerr = iord[1];
    errmax = elist[maxerr];
    nrmax = 1;
    extrap = false;
    small = small * 0.5;
    erlarg = errsum;
  }
post:
  if (*abserr == oflow) goto sum_all;
  if (ier + ierro != 0) {
    if (ierro == 3) *abserr = *abserr + correc;
    if (ier == 0) ier = 3;
    if (*result != 0.0 && area != 0.0) {
      if (*abserr / std::fabs(*result) > errsum / std::fabs(area)) goto sum_all;
    } else {
      if (*abserr > errsum) goto sum_all;
      if (area == 0.0) goto finish;
    }
  }
  if (ksgn == -1 && std::fmax(std::fabs(*result), std::fabs(area)) <= defabs * 0.1e-1) goto finish;
  if (0.1e-1 > (*result / area) || (*result / area) > 0.1e3 || errsum > std::fabs(area)) ier = 6;
  goto finish;
sum_all:
  *result = 0.0;
  for (int k = 1; k <= last; ++k) *result = *result + rlist[k];
  *abserr = errsum;
finish:
  if (ier > 2) ier = ier - 1;
  return ier;
}

}  // namespace

int quad_dqng(int ndim, int acf, float nu, double a, double b, double epsabs, double epsrel, double* result,
              double* abserr) {
  return dqng(Integrand{ndim, acf, nu}, a, b, epsabs, epsrel, result, abserr);
}

int quad_dqagi(int ndim, int acf, float nu, double bound, double epsabs, double epsrel, int limit, double* result,
               double* abserr) {
  if (limit < 1) return 6;
  return dqagie(Integrand{ndim, acf, nu}, bound, 1, epsabs, epsrel, limit, result, abserr);
}

}  // namespace scarf
