/*
 * srm_oracle.c -- CPU restatement of SCARF3D's SRM path. TEST INFRASTRUCTURE
 * ONLY (tests/, the smoke check, bench.py's CPU-baseline leg); the product
 * library never links it. Parity status: UNPINNED (see srm_oracle.h).
 *
 * Arithmetic contract: single-precision operations in the reference's written
 * order (Fortran evaluates a+b+c as (a+b)+c), no FMA contraction (compiled with
 * -ffp-contract=off), glibc single-precision libm (sinf, cosf, acosf, logf,
 * powf, expf, sqrtf) as gfortran calls it, and the mixed FP32/FP64 chain of
 * srm_fn. Citations are file:line in the reference tree.
 */
#include "srm_oracle.h"

#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* pi as the reference declares it: REAL(real32) 3.141592653589793
 * (scarflib_common.f90:94), i.e. the float nearest to pi. */
#define ORC_PI 3.14159265358979323846f

/* ======================================================================== */
/* Uniform source: YARN2-type generator (TRNG's published parameters).        */
/* prng.cpp:60 holds a static trng::yarn2 seeded by set_seed (prng.cpp:147);  */
/* srng returns two uniform01_dist<float> draws (prng.cpp:152-165).           */
/* ======================================================================== */
#define ORC_MOD 2147483647LL /* 2^31 - 1 */
#define ORC_A1 1498809829LL
#define ORC_A2 1160990996LL
#define ORC_GEN 123567893LL

static int64_t orc_powmod(int64_t base, int64_t e) {
  int64_t r = 1;
  base %= ORC_MOD;
  while (e > 0) {
    if (e & 1) r = (r * base) % ORC_MOD;
    base = (base * base) % ORC_MOD;
    e >>= 1;
  }
  return r;
}

void orc_rng_seed(orc_rng *g, int seed) {
  /* prng.cpp:147 converts the int seed to unsigned long and calls
   * trng::yarn2::seed(unsigned long). The published seeding of TRNG's
   * multiple recursive generators reduces the seed, read back as a signed
   * 64-bit integer, into [0, m) (adding m to a negative remainder) and sets
   * the older state word to 1, so the state is never all-zero. */
  int64_t t = (int64_t)(unsigned long)(long)seed;
  t %= ORC_MOD;
  if (t < 0) t += ORC_MOD;
  g->r0 = t;
  g->r1 = 1;
}

uint32_t orc_rng_next(orc_rng *g) {
  int64_t t = (ORC_A1 * g->r0 + ORC_A2 * g->r1) % ORC_MOD;
  g->r1 = g->r0;
  g->r0 = t;
  return t == 0 ? 0u : (uint32_t)orc_powmod(ORC_GEN, t);
}

float orc_u01(uint32_t y) {
  /* trng::uniform01_dist<> (prng.cpp:159-163) takes its default result type,
   * double: one generator output y in [0, m-1] scaled into [0,1) by the
   * generator's range, y * (1/m) in double precision. srng stores each draw
   * into a float, rounding to nearest (the result can be 0, and can round up
   * to 1.0f for the largest y). 1/m is 0x1.00000002p-31 in double. */
  return (float)((double)y * 0x1.00000002p-31);
}

void orc_srng(orc_rng *g, float r[2]) {
  r[0] = orc_u01(orc_rng_next(g));
  r[1] = orc_u01(orc_rng_next(g));
}

/* ======================================================================== */
/* Spectra (psdf.f90:50-90) and the SRM integrand (scarflib_srm.f90:975-995) */
/* ======================================================================== */
float orc_fn_vk(float x, float nu) { return 1.0f / powf(1.0f + x * x, nu); }

float orc_fn_gs(float x) { return expf(-0.25f * (x * x)); }

double orc_srm_fn(double x, int ndim, int acf, float nu) {
  float xf = (float)x;
  float fv = (acf == 0) ? orc_fn_vk(xf, nu) : orc_fn_gs(xf);
  double r = x * (double)fv;
  if (ndim == 3) r = r * x;
  return r;
}

typedef struct { int ndim, acf; float nu; } orc_psd;
static double orc_f(double x, const orc_psd *p) { return orc_srm_fn(x, p->ndim, p->acf, p->nu); }

/* ======================================================================== */
/* QUADPACK restatement (quadpack.f90). Node and weight tables are the       */
/* published Gauss-Kronrod(-Patterson) constants of Piessens et al. (1983).  */
/* Control flow mirrors the Fortran labels so results match to the bit.      */
/* ======================================================================== */
static const double ORC_X1[5] = {
    0.973906528517171720077964012084452, 0.865063366688984510732096688423493,
    0.679409568299024406234327365114874, 0.433395394129247190799265943165784,
    0.148874338981631210884826001129720};
static const double ORC_W10[5] = {
    0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
    0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
    0.295524224714752870173892994651338};
static const double ORC_X2[5] = {
    0.995657163025808080735527280689003, 0.930157491355708226001207180059508,
    0.780817726586416897063717578345042, 0.562757134668604683339000099272694,
    0.294392862701460198131126603103866};
static const double ORC_W21A[5] = {
    0.032558162307964727478818972459390, 0.075039674810919952767043140916190,
    0.109387158802297641899210590325805, 0.134709217311473325928054001771707,
    0.147739104901338491374841515972068};
static const double ORC_W21B[6] = {
    0.011694638867371874278064396062192, 0.054755896574351996031381300244580,
    0.093125454583697605535065465083366, 0.123491976262065851077958109831074,
    0.142775938577060080797094273138717, 0.149445554002916905664936468389821};
static const double ORC_X3[11] = {
    0.999333360901932081394099323919911, 0.987433402908088869795961478381209,
    0.954807934814266299257919200290473, 0.900148695748328293625099494069092,
    0.825198314983114150847066732588520, 0.732148388989304982612354848755461,
    0.622847970537725238641159120344323, 0.499479574071056499952214885499755,
    0.364901661346580768043989548502644, 0.222254919776601296498260928066212,
    0.074650617461383322043914435796506};
static const double ORC_W43A[10] = {
    0.016296734289666564924281974617663, 0.037522876120869501461613795898115,
    0.054694902058255442147212685465005, 0.067355414609478086075553166302174,
    0.073870199632393953432140695251367, 0.005768556059769796184184327908655,
    0.027371890593248842081276069289151, 0.046560826910428830743339154433824,
    0.061744995201442564496240336030883, 0.071387267268693397768559114425516};
static const double ORC_W43B[12] = {
    0.001844477640212414100389106552965, 0.010798689585891651740465406741293,
    0.021895363867795428102523123075149, 0.032597463975345689443882222526137,
    0.042163137935191811847627924327955, 0.050741939600184577780189020092084,
    0.058379395542619248375475369330206, 0.064746404951445885544689259517511,
    0.069566197912356484528633315038405, 0.072824441471833208150939535192842,
    0.074507751014175118273571813842889, 0.074722147517403005594425168280423};
static const double ORC_X4[22] = {
    0.999902977262729234490529830591582, 0.997989895986678745427496322365960,
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
static const double ORC_W87A[21] = {
    0.008148377384149172900002878448190, 0.018761438201562822243935059003794,
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
static const double ORC_W87B[23] = {
    0.000274145563762072350016527092881, 0.001807124155057942948341311753254,
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

/* 15-point Kronrod / 7-point Gauss on the transformed infinite interval. */
static const double ORC_WG15[8] = {
    0.0, 0.129484966168869693270611432679082, 0.0, 0.279705391489276667901467771423780,
    0.0, 0.381830050505118944950369775488975, 0.0, 0.417959183673469387755102040816327};
static const double ORC_XGK15[8] = {
    0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
    0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
    0.586087235467691130294144838258730, 0.405845151377397166906606412076961,
    0.207784955007898467600689403773245, 0.0};
static const double ORC_WGK15[8] = {
    0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
    0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
    0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
    0.204432940075298892414161999234649, 0.209482141084727828012999174891714};

/* DQNG: non-adaptive 21/43/87-point rule (quadpack.f90:8137). */
static void dqng_impl(const orc_psd *ps, double a, double b, double epsabs, double epsrel,
                      double *result, double *abserr, int *neval, int *ier) {
  const double epmach = DBL_EPSILON, uflow = DBL_MIN;
  double fv1[5], fv2[5], fv3[5], fv4[5], savfun[21];
  double res10 = 0, res21 = 0, res43 = 0, res87, resabs = 0, resasc = 0, reskh;
  int ipx = 0;
  *result = 0.0;
  *abserr = 0.0;
  *neval = 0;
  *ier = 6;
  if (epsabs <= 0.0 && epsrel < fmax(50.0 * epmach, 0.5e-28)) return;
  double hlgth = 0.5 * (b - a);
  double dhlgth = fabs(hlgth);
  double centr = 0.5 * (b + a);
  double fcentr = orc_f(centr, ps);
  *neval = 21;
  *ier = 1;
  for (int l = 1; l <= 3; l++) {
    if (l == 1) {
      res10 = 0.0;
      res21 = ORC_W21B[5] * fcentr;
      resabs = ORC_W21B[5] * fabs(fcentr);
      for (int k = 0; k < 5; k++) {
        double absc = hlgth * ORC_X1[k];
        double fval1 = orc_f(centr + absc, ps);
        double fval2 = orc_f(centr - absc, ps);
        double fval = fval1 + fval2;
        res10 = res10 + ORC_W10[k] * fval;
        res21 = res21 + ORC_W21A[k] * fval;
        resabs = resabs + ORC_W21A[k] * (fabs(fval1) + fabs(fval2));
        savfun[k] = fval;
        fv1[k] = fval1;
        fv2[k] = fval2;
      }
      ipx = 5;
      for (int k = 0; k < 5; k++) {
        ipx++;
        double absc = hlgth * ORC_X2[k];
        double fval1 = orc_f(centr + absc, ps);
        double fval2 = orc_f(centr - absc, ps);
        double fval = fval1 + fval2;
        res21 = res21 + ORC_W21B[k] * fval;
        resabs = resabs + ORC_W21B[k] * (fabs(fval1) + fabs(fval2));
        savfun[ipx - 1] = fval;
        fv3[k] = fval1;
        fv4[k] = fval2;
      }
      *result = res21 * hlgth;
      resabs = resabs * dhlgth;
      reskh = 0.5 * res21;
      resasc = ORC_W21B[5] * fabs(fcentr - reskh);
      for (int k = 0; k < 5; k++)
        resasc = resasc + ORC_W21A[k] * (fabs(fv1[k] - reskh) + fabs(fv2[k] - reskh)) +
                 ORC_W21B[k] * (fabs(fv3[k] - reskh) + fabs(fv4[k] - reskh));
      *abserr = fabs((res21 - res10) * hlgth);
      resasc = resasc * dhlgth;
    } else if (l == 2) {
      res43 = ORC_W43B[11] * fcentr;
      *neval = 43;
      for (int k = 0; k < 10; k++) res43 = res43 + savfun[k] * ORC_W43A[k];
      for (int k = 0; k < 11; k++) {
        ipx++;
        double absc = hlgth * ORC_X3[k];
        double fval = orc_f(absc + centr, ps) + orc_f(centr - absc, ps);
        res43 = res43 + fval * ORC_W43B[k];
        savfun[ipx - 1] = fval;
      }
      *result = res43 * hlgth;
      *abserr = fabs((res43 - res21) * hlgth);
    } else {
      res87 = ORC_W87B[22] * fcentr;
      *neval = 87;
      for (int k = 0; k < 21; k++) res87 = res87 + savfun[k] * ORC_W87A[k];
      for (int k = 0; k < 22; k++) {
        double absc = hlgth * ORC_X4[k];
        res87 = res87 + ORC_W87B[k] * (orc_f(absc + centr, ps) + orc_f(centr - absc, ps));
      }
      *result = res87 * hlgth;
      *abserr = fabs((res87 - res43) * hlgth);
    }
    if (resasc != 0.0 && *abserr != 0.0)
      *abserr = resasc * fmin(1.0, pow(200.0 * *abserr / resasc, 1.5));
    if (resabs > uflow / (50.0 * epmach)) *abserr = fmax((epmach * 50.0) * resabs, *abserr);
    if (*abserr <= fmax(epsabs, epsrel * fabs(*result))) {
      *ier = 0;
      return;
    }
  }
}

/* DQK15I: 15-point transformed rule on a subinterval of (0,1] (quadpack.f90:6589). */
static void dqk15i_impl(const orc_psd *ps, double boun, int inf, double a, double b,
                        double *result, double *abserr, double *resabs, double *resasc) {
  const double epmach = DBL_EPSILON, uflow = DBL_MIN;
  double fv1[7], fv2[7];
  double dinf = (double)(inf < 1 ? inf : 1);
  double centr = 0.5 * (a + b);
  double hlgth = 0.5 * (b - a);
  double tabsc1 = boun + dinf * (1.0 - centr) / centr;
  double fval1 = orc_f(tabsc1, ps);
  if (inf == 2) fval1 = fval1 + orc_f(-tabsc1, ps);
  double fc = (fval1 / centr) / centr;
  double resg = ORC_WG15[7] * fc;
  double resk = ORC_WGK15[7] * fc;
  *resabs = fabs(resk);
  for (int j = 0; j < 7; j++) {
    double absc = hlgth * ORC_XGK15[j];
    double absc1 = centr - absc;
    double absc2 = centr + absc;
    double t1 = boun + dinf * (1.0 - absc1) / absc1;
    double t2 = boun + dinf * (1.0 - absc2) / absc2;
    double f1 = orc_f(t1, ps);
    double f2 = orc_f(t2, ps);
    if (inf == 2) f1 = f1 + orc_f(-t1, ps);
    if (inf == 2) f2 = f2 + orc_f(-t2, ps);
    f1 = (f1 / absc1) / absc1;
    f2 = (f2 / absc2) / absc2;
    fv1[j] = f1;
    fv2[j] = f2;
    double fsum = f1 + f2;
    resg = resg + ORC_WG15[j] * fsum;
    resk = resk + ORC_WGK15[j] * fsum;
    *resabs = *resabs + ORC_WGK15[j] * (fabs(f1) + fabs(f2));
  }
  double reskh = resk * 0.5;
  *resasc = ORC_WGK15[7] * fabs(fc - reskh);
  for (int j = 0; j < 7; j++)
    *resasc = *resasc + ORC_WGK15[j] * (fabs(fv1[j] - reskh) + fabs(fv2[j] - reskh));
  *result = resk * hlgth;
  *resasc = *resasc * hlgth;
  *resabs = *resabs * hlgth;
  *abserr = fabs((resk - resg) * hlgth);
  if (*resasc != 0.0 && *abserr != 0.0)
    *abserr = *resasc * fmin(1.0, pow(200.0 * *abserr / *resasc, 1.5));
  if (*resabs > uflow / (50.0 * epmach)) *abserr = fmax((epmach * 50.0) * *resabs, *abserr);
}

/* DQPSRT: maintain the descending ordering of error estimates
 * (quadpack.f90:8529). Arrays are 1-based. */
static void dqpsrt_impl(int limit, int last, int *maxerr, double *ermax, const double *elist,
                        int *iord, int *nrmax) {
  double errmax, errmin;
  int i, ibeg, ido, isucc, j, jbnd, jupbn, k;
  if (last > 2) goto L10;
  iord[1] = 1;
  iord[2] = 2;
  goto L90;
L10:
  errmax = elist[*maxerr];
  ido = *nrmax - 1;
  for (i = 1; i <= ido; i++) {
    isucc = iord[*nrmax - 1];
    if (errmax <= elist[isucc]) break;
    iord[*nrmax] = isucc;
    (*nrmax)--;
  }
  jupbn = last;
  if (last > (limit / 2 + 2)) jupbn = limit + 3 - last;
  errmin = elist[last];
  jbnd = jupbn - 1;
  ibeg = *nrmax + 1;
  for (i = ibeg; i <= jbnd; i++) {
    isucc = iord[i];
    if (errmax >= elist[isucc]) goto L60;
    iord[i - 1] = isucc;
  }
  iord[jbnd] = *maxerr;
  iord[jupbn] = last;
  goto L90;
L60:
  iord[i - 1] = *maxerr;
  k = jbnd;
  for (j = i; j <= jbnd; j++) {
    isucc = iord[k];
    if (errmin < elist[isucc]) goto L80;
    iord[k + 1] = isucc;
    k--;
  }
  iord[i] = last;
  goto L90;
L80:
  iord[k + 1] = last;
L90:
  *maxerr = iord[*nrmax];
  *ermax = elist[*maxerr];
}

/* DQELG: Wynn's epsilon algorithm (quadpack.f90:6230). epstab 1-based [1..52]. */
static void dqelg_impl(int *n, double *epstab, double *result, double *abserr, double *res3la,
                       int *nres) {
  const double epmach = DBL_EPSILON, oflow = DBL_MAX;
  int i, ib, ib2, ie, indx, k1, k2, k3, limexp, newelm, num;
  double delta1, delta2, delta3, e0, e1, e1abs, e2, e3, epsinf, error, err1, err2, err3, res, ss,
      tol1, tol2, tol3;
  (*nres)++;
  *abserr = oflow;
  *result = epstab[*n];
  if (*n < 3) goto L100;
  limexp = 50;
  epstab[*n + 2] = epstab[*n];
  newelm = (*n - 1) / 2;
  epstab[*n] = oflow;
  num = *n;
  k1 = *n;
  for (i = 1; i <= newelm; i++) {
    k2 = k1 - 1;
    k3 = k1 - 2;
    res = epstab[k1 + 2];
    e0 = epstab[k3];
    e1 = epstab[k2];
    e2 = res;
    e1abs = fabs(e1);
    delta2 = e2 - e1;
    err2 = fabs(delta2);
    tol2 = fmax(fabs(e2), e1abs) * epmach;
    delta3 = e1 - e0;
    err3 = fabs(delta3);
    tol3 = fmax(e1abs, fabs(e0)) * epmach;
    if (err2 > tol2 || err3 > tol3) goto L10;
    *result = res;
    *abserr = err2 + err3;
    goto L100;
  L10:
    e3 = epstab[k1];
    epstab[k1] = e1;
    delta1 = e1 - e3;
    err1 = fabs(delta1);
    tol1 = fmax(e1abs, fabs(e3)) * epmach;
    if (err1 <= tol1 || err2 <= tol2 || err3 <= tol3) goto L20;
    ss = 1.0 / delta1 + 1.0 / delta2 - 1.0 / delta3;
    epsinf = fabs(ss * e1);
    if (epsinf > 1.0e-4) goto L30;
  L20:
    *n = i + i - 1;
    goto L50;
  L30:
    res = e1 + 1.0 / ss;
    epstab[k1] = res;
    k1 = k1 - 2;
    error = err2 + fabs(res - e2) + err3;
    if (error <= *abserr) {
      *abserr = error;
      *result = res;
    }
  }
L50:
  if (*n == limexp) *n = 2 * (limexp / 2) - 1;
  ib = 1;
  if ((num / 2) * 2 == num) ib = 2;
  ie = newelm + 1;
  for (i = 1; i <= ie; i++) {
    ib2 = ib + 2;
    epstab[ib] = epstab[ib2];
    ib = ib2;
  }
  if (num == *n) goto L80;
  indx = num - *n + 1;
  for (i = 1; i <= *n; i++) {
    epstab[i] = epstab[indx];
    indx++;
  }
L80:
  if (*nres >= 4) goto L90;
  res3la[*nres] = *result;
  *abserr = oflow;
  goto L100;
L90:
  *abserr = fabs(*result - res3la[3]) + fabs(*result - res3la[2]) + fabs(*result - res3la[1]);
  res3la[1] = res3la[2];
  res3la[2] = res3la[3];
  res3la[3] = *result;
L100:
  *abserr = fmax(*abserr, 5.0 * epmach * fabs(*result));
}

/* DQAGIE: adaptive integration over (bound, +inf) with extrapolation
 * (quadpack.f90:712). Work arrays 1-based, length limit+1. */
static void dqagie_impl(const orc_psd *ps, double bound, int inf, double epsabs, double epsrel,
                        int limit, double *result, double *abserr, int *neval, int *ier,
                        double *alist, double *blist, double *rlist, double *elist, int *iord,
                        int *last) {
  const double epmach = DBL_EPSILON;
  double rlist2[56], res3la[4];
  double area = 0, area1, area12, area2, a1, a2, b1 = 0, b2, boun, correc = 0, defabs, defab1,
         defab2, dres, erlarg = 0, erlast, errbnd, errmax = 0, error1, error2, erro12 = 0,
         errsum = 0, ertest = 0, resabs, reseps, abseps, small = 0, oflow = DBL_MAX,
         uflow = DBL_MIN;
  int id, ierro = 0, iroff1 = 0, iroff2 = 0, iroff3 = 0, jupbnd, k, ksgn = -1, ktmin = 0,
          maxerr = 1, nres = 0, nrmax = 1, numrl2 = 2;
  int extrap = 0, noext = 0;
  memset(rlist2, 0, sizeof(rlist2));
  memset(res3la, 0, sizeof(res3la));
  *ier = 0;
  *neval = 0;
  *last = 0;
  *result = 0.0;
  *abserr = 0.0;
  alist[1] = 0.0;
  blist[1] = 1.0;
  rlist[1] = 0.0;
  elist[1] = 0.0;
  iord[1] = 0;
  if (epsabs <= 0.0 && epsrel < fmax(50.0 * epmach, 0.5e-28)) *ier = 6;
  if (*ier == 6) return;
  boun = bound;
  if (inf == 2) boun = 0.0;
  dqk15i_impl(ps, boun, inf, 0.0, 1.0, result, abserr, &defabs, &resabs);
  *last = 1;
  rlist[1] = *result;
  elist[1] = *abserr;
  iord[1] = 1;
  dres = fabs(*result);
  errbnd = fmax(epsabs, epsrel * dres);
  if (*abserr <= 100.0 * epmach * defabs && *abserr > errbnd) *ier = 2;
  if (limit == 1) *ier = 1;
  if (*ier != 0 || (*abserr <= errbnd && *abserr != resabs) || *abserr == 0.0) goto L130;
  uflow = DBL_MIN;
  oflow = DBL_MAX;
  rlist2[1] = *result;
  errmax = *abserr;
  maxerr = 1;
  area = *result;
  errsum = *abserr;
  *abserr = oflow;
  nrmax = 1;
  nres = 0;
  ktmin = 0;
  numrl2 = 2;
  extrap = 0;
  noext = 0;
  ierro = 0;
  iroff1 = 0;
  iroff2 = 0;
  iroff3 = 0;
  ksgn = -1;
  if (dres >= (1.0 - 50.0 * epmach) * defabs) ksgn = 1;
  for (*last = 2; *last <= limit; (*last)++) {
    a1 = alist[maxerr];
    b1 = 0.5 * (alist[maxerr] + blist[maxerr]);
    a2 = b1;
    b2 = blist[maxerr];
    erlast = errmax;
    dqk15i_impl(ps, boun, inf, a1, b1, &area1, &error1, &resabs, &defab1);
    dqk15i_impl(ps, boun, inf, a2, b2, &area2, &error2, &resabs, &defab2);
    area12 = area1 + area2;
    erro12 = error1 + error2;
    errsum = errsum + erro12 - errmax;
    area = area + area12 - rlist[maxerr];
    if (defab1 == error1 || defab2 == error2) goto L15;
    if (fabs(rlist[maxerr] - area12) > 0.1e-4 * fabs(area12) || erro12 < 0.99 * errmax) goto L10;
    if (extrap) iroff2++;
    if (!extrap) iroff1++;
  L10:
    if (*last > 10 && erro12 > errmax) iroff3++;
  L15:
    rlist[maxerr] = area1;
    rlist[*last] = area2;
    errbnd = fmax(epsabs, epsrel * fabs(area));
    if (iroff1 + iroff2 >= 10 || iroff3 >= 20) *ier = 2;
    if (iroff2 >= 5) ierro = 3;
    if (*last == limit) *ier = 1;
    if (fmax(fabs(a1), fabs(b2)) <= (1.0 + 100.0 * epmach) * (fabs(a2) + 1000.0 * uflow)) *ier = 4;
    if (error2 > error1) goto L20;
    alist[*last] = a2;
    blist[maxerr] = b1;
    blist[*last] = b2;
    elist[maxerr] = error1;
    elist[*last] = error2;
    goto L30;
  L20:
    alist[maxerr] = a2;
    alist[*last] = a1;
    blist[*last] = b1;
    rlist[maxerr] = area2;
    rlist[*last] = area1;
    elist[maxerr] = error2;
    elist[*last] = error1;
  L30:
    dqpsrt_impl(limit, *last, &maxerr, &errmax, elist, iord, &nrmax);
    if (errsum <= errbnd) goto L115;
    if (*ier != 0) goto L100;
    if (*last == 2) goto L80;
    if (noext) continue;
    erlarg = erlarg - erlast;
    if (fabs(b1 - a1) > small) erlarg = erlarg + erro12;
    if (extrap) goto L40;
    if (fabs(blist[maxerr] - alist[maxerr]) > small) continue;
    extrap = 1;
    nrmax = 2;
  L40:
    if (ierro == 3 || erlarg <= ertest) goto L60;
    id = nrmax;
    jupbnd = *last;
    if (*last > (2 + limit / 2)) jupbnd = limit + 3 - *last;
    {
      int leave = 0;
      for (k = id; k <= jupbnd; k++) {
        maxerr = iord[nrmax];
        errmax = elist[maxerr];
        if (fabs(blist[maxerr] - alist[maxerr]) > small) {
          leave = 1;
          break;
        }
        nrmax++;
      }
      if (leave) continue;
    }
  L60:
    numrl2++;
    rlist2[numrl2] = area;
    dqelg_impl(&numrl2, rlist2, &reseps, &abseps, res3la, &nres);
    ktmin++;
    if (ktmin > 5 && *abserr < 0.1e-2 * errsum) *ier = 5;
    if (abseps >= *abserr) goto L70;
    ktmin = 0;
    *abserr = abseps;
    *result = reseps;
    correc = erlarg;
    ertest = fmax(epsabs, epsrel * fabs(reseps));
    if (*abserr <= ertest) goto L100;
  L70:
    if (numrl2 == 1) noext = 1;
    if (*ier == 5) goto L100;
    maxerr = iord[1];
    errmax = elist[maxerr];
    nrmax = 1;
    extrap = 0;
    small = small * 0.5;
    erlarg = errsum;
    continue;
  L80:
    small = 0.375;
    erlarg = errsum;
    ertest = errbnd;
    rlist2[2] = area;
  }
L100:
  if (*abserr == oflow) goto L115;
  if ((*ier + ierro) == 0) goto L110;
  if (ierro == 3) *abserr = *abserr + correc;
  if (*ier == 0) *ier = 3;
  if (*result != 0.0 && area != 0.0) goto L105;
  if (*abserr > errsum) goto L115;
  if (area == 0.0) goto L130;
  goto L110;
L105:
  if (*abserr / fabs(*result) > errsum / fabs(area)) goto L115;
L110:
  if (ksgn == -1 && fmax(fabs(*result), fabs(area)) <= defabs * 0.1e-1) goto L130;
  if (0.1e-1 > (*result / area) || (*result / area) > 0.1e3 || errsum > fabs(area)) *ier = 6;
  goto L130;
L115:
  *result = 0.0;
  for (k = 1; k <= *last; k++) *result = *result + rlist[k];
  *abserr = errsum;
L130:
  *neval = 30 * (*last) - 15;
  if (inf == 2) *neval = 2 * (*neval);
  if (*ier > 2) *ier = *ier - 1;
}

void orc_dqng(int ndim, int acf, float nu, double a, double b, double epsabs, double epsrel,
              double *result, double *abserr, int *neval, int *ier) {
  orc_psd ps = {ndim, acf, nu};
  dqng_impl(&ps, a, b, epsabs, epsrel, result, abserr, neval, ier);
}

void orc_dqagi(int ndim, int acf, float nu, double bound, int inf, double epsabs, double epsrel,
               int limit, double *result, double *abserr, int *neval, int *ier, int *last) {
  orc_psd ps = {ndim, acf, nu};
  double *w = (double *)calloc((size_t)4 * (limit + 1), sizeof(double));
  int *iw = (int *)calloc((size_t)limit + 1, sizeof(int));
  dqagie_impl(&ps, bound, inf, epsabs, epsrel, limit, result, abserr, neval, ier, w,
              w + (limit + 1), w + 2 * (limit + 1), w + 3 * (limit + 1), iw, last);
  free(w);
  free(iw);
}

/* ======================================================================== */
/* Setup (scarflib_srm.f90:617-720; unstructured copy :214-317)              */
/* ======================================================================== */
int orc_setup_compute(const orc_params *p, orc_setup *s) {
  memset(s, 0, sizeof(*s));
  if (p->acf != 0 && p->acf != 1) return -1;
  if (p->nharm <= 0) return -2;
  int ndim = (p->cl[2] > 0.0f) ? 3 : 2;
  s->ndim = ndim;
  float span[3];
  for (int c = 0; c < 3; c++) span[c] = p->fc[c] - p->nc[c];
  float mx = p->cl[0] / span[0];
  float mn = p->cl[0];
  for (int c = 1; c < ndim; c++) {
    float q = p->cl[c] / span[c];
    if (q > mx) mx = q;
    if (p->cl[c] < mn) mn = p->cl[c];
  }
  s->kmin = (2.0f * ORC_PI) * mx;
  s->kmax = (ORC_PI / p->dh) * mn;
  s->kc = (ORC_PI / p->ds) * mn;
  for (int c = 0; c < ndim; c++) {
    if ((2.0f * ORC_PI) / span[c] >= 1.0f / p->cl[c]) s->info0 = 1.0f;
    if (p->ds > p->cl[c] / 2.0f) s->info1 = 1.0f;
  }
  s->scaling = p->sigma / sqrtf((float)p->nharm);

  float ca = cosf(p->alpha * ORC_PI / 180.0f), sa = sinf(p->alpha * ORC_PI / 180.0f);
  float cb = cosf(p->beta * ORC_PI / 180.0f), sb = sinf(p->beta * ORC_PI / 180.0f);
  float cg = cosf(p->gamma * ORC_PI / 180.0f), sg = sinf(p->gamma * ORC_PI / 180.0f);
  float *m = s->m;
  m[0] = ca * cb;
  m[3] = sa * cb;
  m[6] = -sb;
  m[1] = ca * sb * sg - sa * cg;
  m[4] = sa * sb * sg + ca * cg;
  m[7] = cb * sg;
  m[2] = ca * sb * cg + sa * sg;
  m[5] = sa * sb * cg - ca * sg;
  m[8] = cb * cg;
  float bar[3], obar[3];
  for (int c = 0; c < 3; c++) bar[c] = (p->fc[c] - p->nc[c]) / 2.0f;
  for (int r = 0; r < 3; r++) obar[r] = m[3 * r] * bar[0] + m[3 * r + 1] * bar[1] + m[3 * r + 2] * bar[2];
  for (int c = 0; c < 3; c++) s->bar[c] = bar[c] - obar[c];

  s->nu = p->hurst + (float)ndim / 2.0f;
  if (p->acf == 0) {
    s->cnst = 1.0f;
  } else {
    /* 3D: 1/sqrt(pi) (scarflib_srm.f90:711). 2D is left undefined by the
     * reference; 1 is a valid majorant there (max of k*exp(-k^2/4) < 1). */
    s->cnst = (ndim == 3) ? 1.0f / sqrtf(ORC_PI) : 1.0f;
  }
  double r, e;
  int nev, last;
  orc_dqng(ndim, p->acf, s->nu, (double)s->kmin, (double)s->kmax, 1.0e-8, 1.0e-5, &r, &e, &nev,
           &s->ier_band);
  s->intg_band = (float)r;
  orc_dqagi(ndim, p->acf, s->nu, 0.0, 1, 1.0e-8, 1.0e-5, 500, &r, &e, &nev, &s->ier_full, &last);
  s->intg_full = (float)r;
  s->scaling0 = s->scaling;
  s->scaling = s->scaling * sqrtf(s->intg_band / s->intg_full);
  return 0;
}

/* ======================================================================== */
/* Harmonic sampler (scarflib_srm.f90:731-778; unstructured :328-375)        */
/* ======================================================================== */
int orc_sample(const orc_params *p, const orc_setup *s, float *tab, int64_t *pairs) {
  orc_rng g;
  orc_rng_seed(&g, p->seed);
  int kept = 0;
  int64_t np = 0;
  float r[2];
  for (int l = 0; l < p->nharm; l++) {
    float u, d;
    for (;;) {
      orc_srng(&g, r);
      np++;
      u = r[0] * (s->kmax - s->kmin) + s->kmin;
      d = (float)(orc_srm_fn((double)u, s->ndim, p->acf, s->nu) * (double)s->cnst);
      if (r[1] < d) break;
    }
    orc_srng(&g, r);
    np++;
    if (u > s->kc) continue;
    float phi = r[0] * 2.0f * ORC_PI;
    float v1, v2, v3;
    if (s->ndim == 3) {
      float theta = acosf(1.0f - 2.0f * r[1]);
      v1 = u * sinf(phi) * sinf(theta) / p->cl[0];
      v2 = u * cosf(phi) * sinf(theta) / p->cl[1];
      v3 = u * cosf(theta) / p->cl[2];
    } else {
      v1 = u * cosf(phi) / p->cl[0];
      v2 = u * sinf(phi) / p->cl[1];
      v3 = 0.0f;
    }
    orc_srng(&g, r);
    np++;
    float a = sqrtf(-2.0f * logf(r[0])) * cosf(2.0f * ORC_PI * r[1]);
    orc_srng(&g, r);
    np++;
    float b = sqrtf(-2.0f * logf(r[0])) * cosf(2.0f * ORC_PI * r[1]);
    float *t = tab + 5 * (int64_t)kept;
    t[0] = v1;
    t[1] = v2;
    t[2] = v3;
    t[3] = a;
    t[4] = b;
    kept++;
  }
  if (pairs) *pairs = np;
  return kept;
}

/* ======================================================================== */
/* Sums (structured :794-809 + normalise :843-851; unstructured :397-406)    */
/* ======================================================================== */
static inline void orc_rotate_f32(const orc_setup *s, float x, float y, float z, float P[3]) {
  const float *m = s->m;
  for (int r = 0; r < 3; r++) P[r] = m[3 * r] * x + m[3 * r + 1] * y + m[3 * r + 2] * z + s->bar[r];
}

static inline float orc_point_f32(const float P[3], const float *tab, int nh, float scaling) {
  float f = 0.0f;
  for (int h = 0; h < nh; h++) {
    const float *t = tab + 5 * (int64_t)h;
    float arg = t[0] * P[0] + t[1] * P[1] + t[2] * P[2];
    f = f + t[3] * sinf(arg) + t[4] * cosf(arg);
  }
  return f * scaling;
}

static inline double orc_point_f64(const double P[3], const float *tab, int nh, double scaling) {
  double f = 0.0;
  for (int h = 0; h < nh; h++) {
    const float *t = tab + 5 * (int64_t)h;
    double arg = (double)t[0] * P[0] + (double)t[1] * P[1] + (double)t[2] * P[2];
    f = f + (double)t[3] * sin(arg) + (double)t[4] * cos(arg);
  }
  return f * scaling;
}

static inline void orc_rotate_f64(const orc_setup *s, double x, double y, double z, double P[3]) {
  const float *m = s->m;
  for (int r = 0; r < 3; r++)
    P[r] = (double)m[3 * r] * x + (double)m[3 * r + 1] * y + (double)m[3 * r + 2] * z +
           (double)s->bar[r];
}

void orc_sum_structured_f32(const orc_setup *s, const int fs[3], const int n[3], float ds,
                            const float *tab, int nh, const int64_t *idx, int64_t nidx,
                            float *out) {
  for (int64_t q = 0; q < nidx; q++) {
    int64_t p = idx[q];
    int i = (int)(p % n[0]) + 1;
    int j = (int)((p / n[0]) % n[1]) + 1;
    int k = (int)(p / ((int64_t)n[0] * n[1])) + 1;
    float x = (float)(i + fs[0] - 2) * ds;
    float y = (float)(j + fs[1] - 2) * ds;
    float z = (float)(k + fs[2] - 2) * ds;
    float P[3];
    orc_rotate_f32(s, x, y, z, P);
    out[q] = orc_point_f32(P, tab, nh, s->scaling);
  }
}

void orc_sum_structured_f64(const orc_setup *s, const int fs[3], const int n[3], float ds,
                            const float *tab, int nh, const int64_t *idx, int64_t nidx,
                            double *out) {
  for (int64_t q = 0; q < nidx; q++) {
    int64_t p = idx[q];
    int i = (int)(p % n[0]) + 1;
    int j = (int)((p / n[0]) % n[1]) + 1;
    int k = (int)(p / ((int64_t)n[0] * n[1])) + 1;
    double P[3];
    orc_rotate_f64(s, (double)(i + fs[0] - 2) * (double)ds, (double)(j + fs[1] - 2) * (double)ds,
                   (double)(k + fs[2] - 2) * (double)ds, P);
    out[q] = orc_point_f64(P, tab, nh, (double)s->scaling);
  }
}

void orc_sum_points_f32(const orc_setup *s, const float *x, const float *y, const float *z,
                        const float *tab, int nh, const int64_t *idx, int64_t nidx, float *out) {
  for (int64_t q = 0; q < nidx; q++) {
    int64_t p = idx[q];
    float P[3];
    orc_rotate_f32(s, x[p], y[p], z[p], P);
    out[q] = orc_point_f32(P, tab, nh, s->scaling);
  }
}

void orc_sum_points_f64(const orc_setup *s, const float *x, const float *y, const float *z,
                        const float *tab, int nh, const int64_t *idx, int64_t nidx, double *out) {
  for (int64_t q = 0; q < nidx; q++) {
    int64_t p = idx[q];
    double P[3];
    orc_rotate_f64(s, (double)x[p], (double)y[p], (double)z[p], P);
    out[q] = orc_point_f64(P, tab, nh, (double)s->scaling);
  }
}

typedef struct {
  const orc_setup *s;
  const int *fs, *n;
  float ds;
  const float *x, *y, *z;
  const float *tab;
  int nh;
  float *field;
  int64_t lo, hi;
} orc_job;

static void *orc_job_structured(void *arg) {
  orc_job *jb = (orc_job *)arg;
  for (int64_t p = jb->lo; p < jb->hi; p++) {
    int i = (int)(p % jb->n[0]) + 1;
    int j = (int)((p / jb->n[0]) % jb->n[1]) + 1;
    int k = (int)(p / ((int64_t)jb->n[0] * jb->n[1])) + 1;
    float P[3];
    orc_rotate_f32(jb->s, (float)(i + jb->fs[0] - 2) * jb->ds, (float)(j + jb->fs[1] - 2) * jb->ds,
                   (float)(k + jb->fs[2] - 2) * jb->ds, P);
    jb->field[p] = orc_point_f32(P, jb->tab, jb->nh, jb->s->scaling);
  }
  return NULL;
}

static void *orc_job_points(void *arg) {
  orc_job *jb = (orc_job *)arg;
  for (int64_t p = jb->lo; p < jb->hi; p++) {
    float P[3];
    orc_rotate_f32(jb->s, jb->x[p], jb->y[p], jb->z[p], P);
    jb->field[p] = orc_point_f32(P, jb->tab, jb->nh, jb->s->scaling);
  }
  return NULL;
}

static void orc_run_jobs(orc_job *proto, int64_t npts, int nthreads, void *(*fn)(void *)) {
  if (nthreads < 1) nthreads = 1;
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  orc_job *jobs = (orc_job *)calloc((size_t)nthreads, sizeof(orc_job));
  for (int t = 0; t < nthreads; t++) {
    jobs[t] = *proto;
    jobs[t].lo = npts * t / nthreads;
    jobs[t].hi = npts * (t + 1) / nthreads;
    pthread_create(&th[t], NULL, fn, &jobs[t]);
  }
  for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
  free(th);
  free(jobs);
}

void orc_sum_structured_f32_mt(const orc_setup *s, const int fs[3], const int n[3], float ds,
                               const float *tab, int nh, float *field, int nthreads) {
  orc_job proto;
  memset(&proto, 0, sizeof(proto));
  proto.s = s;
  proto.fs = fs;
  proto.n = n;
  proto.ds = ds;
  proto.tab = tab;
  proto.nh = nh;
  proto.field = field;
  orc_run_jobs(&proto, (int64_t)n[0] * n[1] * n[2], nthreads, orc_job_structured);
}

void orc_sum_points_f32_mt(const orc_setup *s, const float *x, const float *y, const float *z,
                           int64_t npts, const float *tab, int nh, float *field, int nthreads) {
  orc_job proto;
  memset(&proto, 0, sizeof(proto));
  proto.s = s;
  proto.x = x;
  proto.y = y;
  proto.z = z;
  proto.tab = tab;
  proto.nh = nh;
  proto.field = field;
  orc_run_jobs(&proto, npts, nthreads, orc_job_points);
}

/* ======================================================================== */
/* Statistics (scarflib_common.f90:694-875), rescale (scarflib_srm.f90:897-912) */
/* and taper (scarflib_common.f90:881-994)                                   */
/* ======================================================================== */
float orc_mean(const float *f, int64_t n) {
  double v = 0.0, c = 1.0;
  for (int64_t i = 0; i < n; i++) {
    v = v + ((double)f[i] - v) / c;
    c = c + 1.0;
  }
  return (float)v;
}

float orc_variance(const float *f, int64_t n) {
  double mu = (double)orc_mean(f, n);
  double s1 = 0.0, s2 = 0.0;
  for (int64_t i = 0; i < n; i++) {
    double x = (double)f[i] - mu;
    s1 = s1 + x;
    s2 = s2 + x * x;
  }
  s1 = (s1 * s1) / (double)n;
  double v = (s2 - s1) / (double)(n - 1);
  return (float)v;
}

void orc_parallel_variance(const float *var, const float *avg, const int *nset, int nsets,
                           float *var_out, float *avg_out) {
  double sig = (double)var[0], mu = (double)avg[0], n = (double)nset[0];
  for (int i = 1; i < nsets; i++) {
    double delta = (double)avg[i] - mu;
    double m1 = sig * (n - 1.0);
    double m2 = (double)var[i] * ((double)nset[i] - 1.0);
    double m = m1 + m2 + delta * delta * n * (double)nset[i] / (n + (double)nset[i]);
    mu = (mu * n + (double)avg[i] * (double)nset[i]) / (n + (double)nset[i]);
    n = n + (double)nset[i];
    sig = m / (n - 1.0);
  }
  *var_out = (float)sig;
  *avg_out = (float)mu;
}

void orc_rescale(float *f, int64_t n, float sigma, float std, float mean) {
  float scaling = sigma / std;
  for (int64_t i = 0; i < n; i++) f[i] = f[i] * scaling - mean;
}

static inline float orc_taper_value(float f, float d, float mute, float taper, float dsum) {
  if (d <= mute) return 0.0f;
  if (d > mute && d <= dsum) {
    float t = (d - mute) / taper;
    return f * (0.5f - 0.5f * cosf(t * ORC_PI));
  }
  return f;
}

void orc_taper_structured(float dh, const int fs[3], const int fe[3], float *field,
                          const float poi[3], float mute, float taper) {
  float dsum = mute + taper;
  int64_t nx = fe[0] - fs[0] + 1, ny = fe[1] - fs[1] + 1;
  for (int k = fs[2]; k <= fe[2]; k++) {
    float dz = (float)(k - 1) * dh - poi[2];
    dz = dz * dz;
    for (int j = fs[1]; j <= fe[1]; j++) {
      float dy = (float)(j - 1) * dh - poi[1];
      dy = dy * dy;
      for (int i = fs[0]; i <= fe[0]; i++) {
        float dx = (float)(i - 1) * dh - poi[0];
        dx = dx * dx;
        float d = sqrtf(dx + dy + dz);
        int64_t p = (i - fs[0]) + nx * ((j - fs[1]) + ny * (int64_t)(k - fs[2]));
        field[p] = orc_taper_value(field[p], d, mute, taper, dsum);
      }
    }
  }
}

void orc_taper_points(const float *x, const float *y, const float *z, int64_t n, float *field,
                      const float poi[3], float mute, float taper) {
  float dsum = mute + taper;
  for (int64_t i = 0; i < n; i++) {
    float ex = x[i] - poi[0], ey = y[i] - poi[1], ez = z[i] - poi[2];
    float d = sqrtf(ex * ex + ey * ey + ez * ez);
    field[i] = orc_taper_value(field[i], d, mute, taper, dsum);
  }
}

/* ======================================================================== */
/* Whole structured execute (scarflib_srm.f90:505-929), single rank          */
/* ======================================================================== */
int orc_execute_structured(const orc_params *p, const int fs[3], const int fe[3], const float *poi,
                           int npoi, float mute, float taper, float *field, float info[6],
                           int nthreads) {
  orc_setup s;
  int rc = orc_setup_compute(p, &s);
  if (rc) return rc;
  float *tab = (float *)malloc(sizeof(float) * 5 * (size_t)p->nharm);
  if (!tab) return -3;
  int64_t pairs;
  int nh = orc_sample(p, &s, tab, &pairs);
  int n[3] = {fe[0] - fs[0] + 1, fe[1] - fs[1] + 1, fe[2] - fs[2] + 1};
  int64_t npts = (int64_t)n[0] * n[1] * n[2];
  orc_sum_structured_f32_mt(&s, fs, n, p->ds, tab, nh, field, nthreads);
  free(tab);
  for (int i = 0; i < 6; i++) info[i] = 0.0f;
  info[0] = s.info0;
  info[1] = s.info1;
  float var = orc_variance(field, npts);
  float mu = orc_mean(field, npts);
  int nn = (int)npts;
  orc_parallel_variance(&var, &mu, &nn, 1, &info[2], &info[3]);
  info[2] = sqrtf(info[2]);
  if (p->rescale == 1) {
    orc_rescale(field, npts, p->sigma, info[2], info[3]);
    info[2] = p->sigma;
    info[3] = 0.0f;
  }
  for (int q = 0; q < npoi; q++) {
    float pt[3] = {0.0f, 0.0f, 0.0f};
    for (int c = 0; c < s.ndim; c++) pt[c] = poi[s.ndim * q + c];
    orc_taper_structured(p->ds, fs, fe, field, pt, mute, taper);
  }
  return 0;
}
