/* fr_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see fr_oracle.h).
 *
 * A CPU, FP64 restatement of the FlurryPP residual + RK path.  Every routine
 * cites the reference routine it follows (paths relative to the reference
 * project root).  Arithmetic expressions keep the reference's operation order
 * so that, on the 3D cases the reference can run, the two agree to rounding
 * (the GEMMs use the same i-p-j loop order as oracle/refshim/cblas_shim.c).
 *
 * What is new relative to the reference (it cannot run these):
 *   - 2D quads: the reference's own QUAD/2D branches (operators, shape
 *     functions, calcTransforms, 2D faces) are used, with quad face-vertex
 *     lists {0,1},{1,2},{2,3},{3,0} matching the QUAD flux-point order of
 *     getLocFpts (src/points.cpp:72-87);
 *   - periodic pairing: faces are matched on caller-supplied vertex ids in
 *     which periodic images share an id, so the reference's own matching and
 *     relRot logic (src/geo.cpp:197-246, :789-908) pairs them;
 *   - the Taylor-Green initial condition (icType 10).
 */
#include "fr_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>
#include <thread>

namespace {
using std::max;
using std::min;
using std::vector;

const double PI = 4.0 * atan(1); /* include/global.hpp:37 */
int g_threads = 1;

/* Runs f(i) for i in [0,n) on g_threads host threads, in contiguous blocks.
 * Every loop parallelised this way writes disjoint memory per i. */
template <class Fn> void pfor(int n, Fn f) {
  int T = std::min(g_threads, n);
  if (T <= 1) {
    for (int i = 0; i < n; i++) f(i);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < T; t++)
    th.emplace_back([&, t] {
      int i0 = (int)((long)n * t / T), i1 = (int)((long)n * (t + 1) / T);
      for (int i = i0; i < i1; i++) f(i);
    });
  for (auto &x : th) x.join();
}

/* BC_TYPE values of include/global.hpp:63-78 */
enum { BC_NONE = -1, BC_PERIODIC = 0, BC_CHAR = 1, BC_SUP_IN = 2, BC_SUP_OUT = 3,
       BC_SUB_IN = 4, BC_SUB_OUT = 5, BC_SLIP = 8, BC_ISO_NOSLIP = 9,
       BC_ADI_NOSLIP = 10, BC_SYMMETRY = 12, BC_ISO_NOSLIP_MOVING = 13 };

/* ------------------------------------------------------------ points.cpp */
/* Gauss-Legendre nodes as the reference tabulates them (15 decimals,
 * src/points.cpp:169-196), orders 0..5. */
vector<double> gaussPts(int order) {
  static const double t[6][6] = {
      {0.0},
      {-0.577350269189626, 0.577350269189626},
      {-0.774596669241483, 0.000000000000000, 0.774596669241483},
      {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
      {-0.906179845938664, -0.538469310105683, 0.000000000000000, 0.538469310105683,
       0.906179845938664},
      {-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197,
       0.661209386466265, 0.932469514203152}};
  if (order < 0 || order > 5) { fprintf(stderr, "oracle: order %d unsupported\n", order); abort(); }
  return vector<double>(t[order], t[order] + order + 1);
}
vector<double> equidistantPts(int order) { /* src/points.cpp:164-167 */
  vector<double> o(order + 1);
  double dxi = 2. / order;
  for (int i = 0; i < order + 1; i++) o[i] = -1 + dxi * i;
  return o;
}
/* Gauss weights, src/points.cpp:347-400 (orders 0..5). */
vector<double> qptWeights1D(int order) {
  static const double t[6][6] = {
      {2.0},
      {1.0, 1.0},
      {0.5555555555555556, 0.8888888888888888, 0.5555555555555556},
      {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538},
      {0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665,
       0.2369268850561891},
      {0.1713244923791704, 0.3607615730481386, 0.4679139345726910, 0.4679139345726910,
       0.3607615730481386, 0.1713244923791704}};
  return vector<double>(t[order], t[order] + order + 1);
}
/* getQptWeights (src/points.cpp:320-345) */
vector<double> qptWeights(int order, int nDims) {
  vector<double> w1 = qptWeights1D(order);
  if (nDims == 1) return w1;
  int n = order + 1;
  vector<double> out;
  if (nDims == 2) {
    out.resize(n * n);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) out[j + i * n] = w1[i] * w1[j];
  } else {
    out.resize(n * n * n);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) out[k + n * (j + i * n)] = w1[i] * w1[j] * w1[k];
  }
  return out;
}

/* -------------------------------------------------------- polynomials.cpp */
double Lagrange(const vector<double> &x, double y, int mode) { /* :9-19 */
  double lag = 1.0;
  for (int i = 0; i < (int)x.size(); i++)
    if (i != mode) lag = lag * ((y - x[i]) / (x[mode] - x[i]));
  return lag;
}
double dLagrange(const vector<double> &x, double y, int mode) { /* :21-45 */
  double dLag = 0.0;
  int n = x.size();
  for (int i = 0; i < n; i++) {
    if (i == mode) continue;
    double num = 1.0, den = 1.0;
    for (int j = 0; j < n; j++) {
      if (j != mode && j != i) num = num * (y - x[j]);
      if (j != mode) den = den * (x[mode] - x[j]);
    }
    dLag = dLag + (num / den);
  }
  return dLag;
}
double Legendre(double r, int mode) { /* :83-94 */
  if (mode < 0) return 0.;
  if (mode == 0) return 1.0;
  if (mode == 1) return r;
  return ((2 * mode - 1) * r * Legendre(r, mode - 1) - (mode - 1) * Legendre(r, mode - 2)) / mode;
}
double dLegendre(double r, int mode) { /* :96-116 */
  double d = 0.;
  if (mode == 0) return 0;
  if (r > -1.0 && r < 1.0) {
    d = mode * ((r * Legendre(r, mode)) - Legendre(r, mode - 1)) / (r * r - 1.0);
  } else {
    if (r == -1.0) d = pow(-1.0, mode - 1.0) * 0.5 * mode * (mode + 1.0);
    if (r == 1.0) d = 0.5 * mode * (mode + 1.0);
  }
  return d;
}
int factorial(int n) { return (n == 1 || n == 0) ? 1 : factorial(n - 1) * n; }
double computeEta(int vcjh, int order) { /* :392-428 */
  if (vcjh == 0) return 0.0;
  if (vcjh == 1) return (1.0 * order) / (1.0 * (order + 1));
  if (vcjh == 2) return (1.0 * (order + 1)) / (1.0 * order);
  double c = 0;
  if (order == 2) c = 0.206;
  else if (order == 3) c = 3.80e-3;
  else if (order == 4) c = 4.67e-5;
  else if (order == 5) c = 4.28e-7;
  else { fprintf(stderr, "oracle: C+ not available for order %d\n", order); abort(); }
  double ap = 1. / pow(2.0, order) * factorial(2 * order) / (factorial(order) * factorial(order));
  return c * (2 * order + 1) / 2 * (factorial(order) * ap) * (factorial(order) * ap);
}
double dVCJH_1d(double r, int mode, int order, double eta) { /* :447-474 */
  if (mode == 0) {
    if (order == 0)
      return 0.5 * pow(-1.0, order) * (dLegendre(r, order) - ((dLegendre(r, order + 1)) / (1.0 + eta)));
    return 0.5 * pow(-1.0, order) *
           (dLegendre(r, order) - (((eta * dLegendre(r, order - 1)) + dLegendre(r, order + 1)) / (1.0 + eta)));
  }
  if (order == 0) return 0.5 * (dLegendre(r, order) + ((dLegendre(r, order + 1)) / (1.0 + eta)));
  return 0.5 * (dLegendre(r, order) + (((eta * dLegendre(r, order - 1)) + dLegendre(r, order + 1)) / (1.0 + eta)));
}

/* ------------------------------------------------------------ funcs.cpp */
/* Lagrange quad shape functions of any order, node order of shape_quad /
 * dshape_quad (src/funcs.cpp:126-176, :587-661): corners, edges, interior. */
void shapeQuad(double xi, double eta, int nNodes, double *sh, double *dsh /*[nNodes][2] or null*/) {
  int nSide = (int)lround(sqrt((double)nNodes));
  vector<double> xl(nSide);
  double dxi = 2. / (nSide - 1);
  for (int i = 0; i < nSide; i++) xl[i] = -1. + i * dxi;
  auto put = [&](int n, int a, int b) {
    if (sh) sh[n] = Lagrange(xl, xi, a) * Lagrange(xl, eta, b);
    if (dsh) {
      dsh[2 * n + 0] = dLagrange(xl, xi, a) * Lagrange(xl, eta, b);
      dsh[2 * n + 1] = Lagrange(xl, xi, a) * dLagrange(xl, eta, b);
    }
  };
  int nLevels = nSide / 2, nPts = 0;
  for (int i = 0; i < nLevels; i++) {
    int i2 = (nSide - 1) - i;
    put(nPts + 0, i, i);
    put(nPts + 1, i2, i);
    put(nPts + 2, i2, i2);
    put(nPts + 3, i, i2);
    nPts += 4;
    int n2 = nSide - 2 * (i + 1);
    for (int j = 0; j < n2; j++) {
      put(nPts + 0 * n2 + j, i + 1 + j, i);
      put(nPts + 1 * n2 + j, i2, i + 1 + j);
      put(nPts + 2 * n2 + j, i2 - 1 - j, i2);
      put(nPts + 3 * n2 + j, i, i2 - 1 - j);
    }
    nPts += 4 * n2;
  }
  if (nSide % 2) put(nNodes - 1, nSide / 2, nSide / 2);
}
/* Linear hexahedron (8 nodes) shape functions, corner level of shape_hex /
 * dshape_hex (src/funcs.cpp:183-260, :680-800). */
void shapeHex8(double xi, double eta, double mu, double *sh, double *dsh /*[8][3]*/) {
  vector<double> xl = {-1., 1.};
  static const int c[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                              {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int n = 0; n < 8; n++) {
    int a = c[n][0], b = c[n][1], g = c[n][2];
    if (sh) sh[n] = Lagrange(xl, xi, a) * Lagrange(xl, eta, b) * Lagrange(xl, mu, g);
    if (dsh) {
      dsh[3 * n + 0] = dLagrange(xl, xi, a) * Lagrange(xl, eta, b) * Lagrange(xl, mu, g);
      dsh[3 * n + 1] = Lagrange(xl, xi, a) * dLagrange(xl, eta, b) * Lagrange(xl, mu, g);
      dsh[3 * n + 2] = Lagrange(xl, xi, a) * Lagrange(xl, eta, b) * dLagrange(xl, mu, g);
    }
  }
}

}  // namespace

/* ====================================================================== */
struct OFace {
  int eL, fL, eR, fR, relRot, bc;
  vector<int> fptL, fptR; /* element-local flux point ids */
  vector<double> Fn;      /* face-resident common flux [nFptsFace][nV] */
};

struct orc_solver {
  orc_params p;
  int nDims, P, nS, nF, nE, nV, nNodes, nFaceEle, nFptFace, nRK;
  vector<double> RKa, RKb;
  /* operators (row-major) */
  vector<double> locS, locF, tNorm; /* [nS][d], [nF][d], [nF][d] */
  vector<double> E, C;              /* [nF][nS], [nS][nF] */
  vector<double> D[3], Efn[3], CU[3];
  /* geometry */
  vector<double> nodes; /* [nNodes][nE][d] */
  vector<double> pos_spts, JGinv_spts, JGinv_fpts, Jac_spts, Jac_fpts;
  vector<double> detJ_spts, detJ_fpts, norm_fpts, dA_fpts;
  vector<OFace> faces;
  /* solution */
  vector<double> U, U0, U_fpts, F_spts, dU_spts, dU_fpts, dUc_fpts, disFn, Fn_fpts;
  vector<vector<double>> divF;
  vector<double> waveSp, eleDt; /* [nE][nF], [nE] */
  double time = 0, dt = 0, rkTime = 0;
  int iter = 0, initIter = 0;

  /* index helpers, reference layouts */
  inline double &u(vector<double> &a, int pt, int e, int k) { return a[((size_t)pt * nE + e) * nV + k]; }
  inline size_t i4(int d, int pt, int nPt, int e, int k) const { return (((size_t)d * nPt + pt) * nE + e) * nV + k; }
  inline size_t g4(int d1, int pt, int nPt, int e, int d2) const { return (((size_t)d1 * nPt + pt) * nE + e) * nDims + d2; }
};

namespace {

/* cblas_dgemm row-major no-transpose with the loop order of the shim used to
 * build the reference (oracle/refshim/cblas_shim.c); columns are split over
 * threads, which leaves every element's arithmetic unchanged. */
void dgemm(int m, int n, int k, double alpha, const double *a, const double *b, double beta, double *c) {
  const int CH = 4096;
  int nChunks = (n + CH - 1) / CH;
  pfor(nChunks, [&](int ch) {
    int j0 = ch * CH, j1 = min(n, j0 + CH);
    for (int i = 0; i < m; i++) {
      double *ci = c + (size_t)i * n;
      if (beta == 0.0) { for (int j = j0; j < j1; j++) ci[j] = 0.0; }
      else if (beta != 1.0) { for (int j = j0; j < j1; j++) ci[j] *= beta; }
      for (int p = 0; p < k; p++) {
        const double aip = alpha * a[(size_t)i * k + p];
        const double *bp = b + (size_t)p * n;
        for (int j = j0; j < j1; j++) ci[j] += aip * bp[j];
      }
    }
  });
}

/* Reference-space unit normal of each flux point's face:
 * QUAD src/operators.cpp:820-840, HEX src/solver.cpp:155-195. */
void faceTNorm(int nDims, int iFace, double *t) {
  if (nDims == 2) {
    static const double q[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};
    t[0] = q[iFace][0]; t[1] = q[iFace][1];
  } else {
    static const double h[6][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}};
    for (int d = 0; d < 3; d++) t[d] = h[iFace][d];
  }
}

/* oper::setupOperators restricted to the matrices the residual path uses
 * (src/operators.cpp:13-76, :78-111, :660-805, :807-889, :891-914, :1008-1092,
 * :1544-1619); points getLocSpts / getLocFpts (src/points.cpp:37-128). */
void setupOperators(orc_solver &s) {
  int P = s.P, n1 = P + 1, d = s.nDims;
  vector<double> sp = gaussPts(P);
  s.nS = d == 2 ? n1 * n1 : n1 * n1 * n1;
  s.nF = d == 2 ? 4 * n1 : 6 * n1 * n1;
  s.nFptFace = d == 2 ? n1 : n1 * n1;
  s.nFaceEle = d == 2 ? 4 : 6;
  int nS = s.nS, nF = s.nF;
  s.locS.assign(nS * d, 0);
  s.locF.assign(nF * d, 0);
  if (d == 2) {
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++) { s.locS[(j + i * n1) * 2 + 0] = sp[j]; s.locS[(j + i * n1) * 2 + 1] = sp[i]; }
    for (int i = 0; i < n1; i++) {
      double *f = s.locF.data();
      f[2 * i] = sp[i]; f[2 * i + 1] = -1.;
      f[2 * (i + n1)] = 1.; f[2 * (i + n1) + 1] = sp[i];
      f[2 * (i + 2 * n1)] = sp[P - i]; f[2 * (i + 2 * n1) + 1] = 1.;
      f[2 * (i + 3 * n1)] = -1.; f[2 * (i + 3 * n1) + 1] = sp[P - i];
    }
  } else {
    for (int k = 0; k < n1; k++)
      for (int j = 0; j < n1; j++)
        for (int i = 0; i < n1; i++) {
          int id = i + n1 * (j + n1 * k);
          s.locS[3 * id] = sp[i]; s.locS[3 * id + 1] = sp[j]; s.locS[3 * id + 2] = sp[k];
        }
    int P12 = n1 * n1;
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++) {
        int ind = i + j * n1;
        double *f = s.locF.data();
        auto set = [&](int id, double x, double y, double z) { f[3 * id] = x; f[3 * id + 1] = y; f[3 * id + 2] = z; };
        set(ind, sp[i], sp[j], -1.);
        set(ind + P12, sp[P - i], sp[j], 1.);
        set(ind + 2 * P12, -1, sp[i], sp[j]);
        set(ind + 3 * P12, 1, sp[P - i], sp[j]);
        set(ind + 4 * P12, sp[P - i], -1, sp[j]);
        set(ind + 5 * P12, sp[i], 1, sp[j]);
      }
  }
  s.tNorm.assign(nF * d, 0);
  for (int f = 0; f < nF; f++) faceTNorm(d, f / s.nFptFace, &s.tNorm[f * d]);

  /* opp_spts_to_fpts */
  s.E.assign((size_t)nF * nS, 0);
  for (int f = 0; f < nF; f++)
    for (int sp_ = 0; sp_ < nS; sp_++) {
      if (d == 2) {
        int is = sp_ % n1, js = sp_ / n1;
        s.E[f * nS + sp_] = Lagrange(sp, s.locF[2 * f], is) * Lagrange(sp, s.locF[2 * f + 1], js);
      } else {
        int ks = sp_ / (n1 * n1), js = (sp_ - n1 * n1 * ks) / n1, is = sp_ - n1 * js - n1 * n1 * ks;
        s.E[f * nS + sp_] = Lagrange(sp, s.locF[3 * f], is) * Lagrange(sp, s.locF[3 * f + 1], js) *
                            Lagrange(sp, s.locF[3 * f + 2], ks);
      }
    }
  /* opp_grad_spts: setupGradPts(basis = pts = Gauss points) */
  for (int dim = 0; dim < d; dim++) {
    s.D[dim].assign((size_t)nS * nS, 0);
    for (int g = 0; g < nS; g++)
      for (int b = 0; b < nS; b++) {
        double v;
        if (d == 2) {
          int i1 = g % n1, j1 = g / n1, i2 = b % n1, j2 = b / n1;
          v = dim == 0 ? dLagrange(sp, sp[i1], i2) * Lagrange(sp, sp[j1], j2)
                       : dLagrange(sp, sp[j1], j2) * Lagrange(sp, sp[i1], i2);
        } else {
          int kg = g / (n1 * n1), jg = (g - n1 * n1 * kg) / n1, ig = g - n1 * jg - n1 * n1 * kg;
          int kb = b / (n1 * n1), jb = (b - n1 * n1 * kb) / n1, ib = b - n1 * jb - n1 * n1 * kb;
          if (dim == 0) v = dLagrange(sp, sp[ig], ib) * Lagrange(sp, sp[jg], jb) * Lagrange(sp, sp[kg], kb);
          else if (dim == 1) v = dLagrange(sp, sp[jg], jb) * Lagrange(sp, sp[ig], ib) * Lagrange(sp, sp[kg], kb);
          else v = dLagrange(sp, sp[kg], kb) * Lagrange(sp, sp[ig], ib) * Lagrange(sp, sp[jg], jb);
        }
        s.D[dim][g * nS + b] = v;
      }
  }
  /* opp_extrapolateFn */
  for (int dim = 0; dim < d; dim++) {
    s.Efn[dim].assign((size_t)nF * nS, 0);
    for (int sp_ = 0; sp_ < nS; sp_++)
      for (int f = 0; f < nF; f++) s.Efn[dim][f * nS + sp_] = s.E[f * nS + sp_] * s.tNorm[f * d + dim];
  }
  /* opp_correction: divVCJH_quad / divVCJH_hex */
  double eta = s.p.vcjhScheme == 0 ? 0. : computeEta(s.p.vcjhScheme, P);
  s.C.assign((size_t)nS * nF, 0);
  for (int sp_ = 0; sp_ < nS; sp_++)
    for (int fp = 0; fp < nF; fp++) {
      const double *loc = &s.locS[sp_ * d];
      double v = 0;
      if (d == 2) {
        int i = fp / n1, j = fp - n1 * i;
        if (i == 0) v = -Lagrange(sp, loc[0], j) * dVCJH_1d(loc[1], 0, P, eta);
        else if (i == 1) v = Lagrange(sp, loc[1], j) * dVCJH_1d(loc[0], 1, P, eta);
        else if (i == 2) v = Lagrange(sp, loc[0], P - j) * dVCJH_1d(loc[1], 1, P, eta);
        else v = -Lagrange(sp, loc[1], P - j) * dVCJH_1d(loc[0], 0, P, eta);
      } else {
        int P12 = n1 * n1, f = fp / P12, j = (fp - P12 * f) / n1, i = fp - P12 * f - n1 * j;
        double x = loc[0], y = loc[1], z = loc[2];
        if (f == 0) v = Lagrange(sp, x, i) * Lagrange(sp, y, j) * -dVCJH_1d(z, 0, P, eta);
        else if (f == 1) v = Lagrange(sp, x, P - i) * Lagrange(sp, y, j) * dVCJH_1d(z, 1, P, eta);
        else if (f == 2) v = Lagrange(sp, y, i) * Lagrange(sp, z, j) * -dVCJH_1d(x, 0, P, eta);
        else if (f == 3) v = Lagrange(sp, y, P - i) * Lagrange(sp, z, j) * dVCJH_1d(x, 1, P, eta);
        else if (f == 4) v = Lagrange(sp, x, P - i) * Lagrange(sp, z, j) * -dVCJH_1d(y, 0, P, eta);
        else v = Lagrange(sp, x, i) * Lagrange(sp, z, j) * dVCJH_1d(y, 1, P, eta);
      }
      s.C[sp_ * nF + fp] = v;
    }
  /* opp_correctU */
  for (int dim = 0; dim < d; dim++) {
    s.CU[dim].assign((size_t)nS * nF, 0);
    for (int fp = 0; fp < nF; fp++)
      for (int sp_ = 0; sp_ < nS; sp_++) s.CU[dim][sp_ * nF + fp] = s.C[sp_ * nF + fp] * s.tNorm[fp * d + dim];
  }
}

/* setPosSptsFpts + calcTransforms (src/solver.cpp:904-951, :1227-1356). */
bool setupGeometry(orc_solver &s) {
  int d = s.nDims, nS = s.nS, nF = s.nF, nE = s.nE, nN = s.nNodes;
  vector<double> shS(nS * nN), dshS(d * nS * nN), dshF(d * nF * nN), tmp(nN * 3);
  auto shapeAt = [&](const double *loc, double *sh, double *dsh) {
    if (d == 2) shapeQuad(loc[0], loc[1], nN, sh, dsh);
    else shapeHex8(loc[0], loc[1], loc[2], sh, dsh);
  };
  for (int sp_ = 0; sp_ < nS; sp_++) {
    shapeAt(&s.locS[sp_ * d], &shS[sp_ * nN], tmp.data());
    for (int n = 0; n < nN; n++)
      for (int dim = 0; dim < d; dim++) dshS[(dim * nS + sp_) * nN + n] = tmp[n * d + dim];
  }
  for (int f = 0; f < nF; f++) {
    shapeAt(&s.locF[f * d], nullptr, tmp.data());
    for (int n = 0; n < nN; n++)
      for (int dim = 0; dim < d; dim++) dshF[(dim * nF + f) * nN + n] = tmp[n * d + dim];
  }
  int n = nE * d;
  s.pos_spts.assign((size_t)nS * nE * d, 0);
  dgemm(nS, n, nN, 1.0, shS.data(), s.nodes.data(), 0.0, s.pos_spts.data());
  s.Jac_spts.assign((size_t)d * nS * nE * d, 0);
  s.Jac_fpts.assign((size_t)d * nF * nE * d, 0);
  for (int dim = 0; dim < d; dim++) {
    dgemm(nS, n, nN, 1.0, &dshS[dim * nS * nN], s.nodes.data(), 0.0, &s.Jac_spts[(size_t)dim * nS * nE * d]);
    dgemm(nF, n, nN, 1.0, &dshF[dim * nF * nN], s.nodes.data(), 0.0, &s.Jac_fpts[(size_t)dim * nF * nE * d]);
  }
  s.JGinv_spts.assign(s.Jac_spts.size(), 0);
  s.JGinv_fpts.assign(s.Jac_fpts.size(), 0);
  s.detJ_spts.assign((size_t)nS * nE, 0);
  s.detJ_fpts.assign((size_t)nF * nE, 0);
  auto transform = [&](vector<double> &Jac, vector<double> &JG, vector<double> &det, int nPt, int pt, int e) {
    auto J = [&](int a, int b) -> double & { return Jac[s.g4(a, pt, nPt, e, b)]; };
    auto G = [&](int a, int b) -> double & { return JG[s.g4(a, pt, nPt, e, b)]; };
    double &dj = det[(size_t)pt * nE + e];
    if (d == 2) {
      dj = J(0, 0) * J(1, 1) - J(0, 1) * J(1, 0);
      G(0, 0) = J(1, 1); G(0, 1) = -J(1, 0); G(1, 0) = -J(0, 1); G(1, 1) = J(0, 0);
    } else {
      double xr = J(0, 0), xs = J(1, 0), xt = J(2, 0), yr = J(0, 1), ys = J(1, 1), yt = J(2, 1);
      double zr = J(0, 2), zs = J(1, 2), zt = J(2, 2);
      dj = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
      G(0, 0) = ys * zt - yt * zs; G(0, 1) = xt * zs - xs * zt; G(0, 2) = xs * yt - xt * ys;
      G(1, 0) = yt * zr - yr * zt; G(1, 1) = xr * zt - xt * zr; G(1, 2) = xt * yr - xr * yt;
      G(2, 0) = yr * zs - ys * zr; G(2, 1) = xs * zr - xr * zs; G(2, 2) = xr * ys - xs * yr;
    }
  };
  for (int sp_ = 0; sp_ < nS; sp_++)
    for (int e = 0; e < nE; e++) {
      transform(s.Jac_spts, s.JGinv_spts, s.detJ_spts, nS, sp_, e);
      if (s.detJ_spts[(size_t)sp_ * nE + e] < 0) {
        fprintf(stderr, "oracle: Negative Jacobian at solution points (element %d)\n", e);
        return false;
      }
    }
  s.norm_fpts.assign((size_t)nF * nE * d, 0);
  s.dA_fpts.assign((size_t)nF * nE, 0);
  for (int f = 0; f < nF; f++)
    for (int e = 0; e < nE; e++) {
      transform(s.Jac_fpts, s.JGinv_fpts, s.detJ_fpts, nF, f, e);
      double *nv = &s.norm_fpts[((size_t)f * nE + e) * d];
      for (int d1 = 0; d1 < d; d1++) {
        nv[d1] = 0.;
        for (int d2 = 0; d2 < d; d2++) nv[d1] += s.JGinv_fpts[s.g4(d2, f, nF, e, d1)] * s.tNorm[f * d + d2];
      }
      double &dA = s.dA_fpts[(size_t)f * nE + e];
      dA = 0;
      for (int dim = 0; dim < d; dim++) dA += nv[dim] * nv[dim];
      dA = sqrt(dA);
      if (std::fabs(dA) < 1e-10) {
        dA = 0.;
        for (int dim = 0; dim < d; dim++) nv[dim] = 0;
      } else {
        for (int dim = 0; dim < d; dim++) nv[dim] /= dA;
      }
    }
  return true;
}

/* Face-vertex lists: HEX from geo::processConn3D (src/geo.cpp:85-90); QUAD
 * edges follow the QUAD flux-point order of getLocFpts. */
const int HEXFV[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {3, 0, 4, 7}, {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};
const int QUADFV[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
/* Oriented face-vertex lists of geo::compareOrientation (src/geo.cpp:800-880) */
const int HEXORI[6][4] = {{0, 1, 2, 3}, {5, 4, 7, 6}, {0, 3, 7, 4}, {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};

/* processConn3D face matching + setupElesFaces + intFace::setupRightState
 * (src/geo.cpp:75-246, :322-446; src/intFace.cpp:6-63). */
bool setupFaces(orc_solver &s, const int *c2v, const int *bc) {
  int d = s.nDims, nE = s.nE, nFE = s.nFaceEle, nC = d == 2 ? 4 : 8, P = s.P, nFF = s.nFptFace;
  std::map<vector<int>, std::pair<int, int>> first;
  for (int e = 0; e < nE; e++)
    for (int f = 0; f < nFE; f++) {
      vector<int> key;
      if (d == 2) key = {c2v[e * nC + QUADFV[f][0]], c2v[e * nC + QUADFV[f][1]]};
      else for (int i = 0; i < 4; i++) key.push_back(c2v[e * nC + HEXFV[f][i]]);
      std::sort(key.begin(), key.end());
      auto it = first.find(key);
      if (it == first.end()) {
        first[key] = {e, f};
        continue;
      }
      OFace F;
      F.eL = it->second.first; F.fL = it->second.second; F.eR = e; F.fR = f; F.bc = -1;
      if (F.eL == e) { fprintf(stderr, "oracle: element %d neighbours itself\n", e); return false; }
      if (d == 3) {
        int t1[4], t2[4];
        for (int i = 0; i < 4; i++) {
          t1[i] = c2v[F.eL * nC + HEXORI[F.fL][i]];
          t2[i] = c2v[F.eR * nC + HEXORI[F.fR][i]];
        }
        F.relRot = -1;
        for (int r = 0; r < 4; r++) if (t1[r] == t2[0]) { F.relRot = r; break; }
        if (F.relRot < 0) { fprintf(stderr, "oracle: Internal faces improperly matched\n"); return false; }
      } else {
        F.relRot = 1;
      }
      it->second.first = -2; /* matched */
      s.faces.push_back(F);
    }
  for (auto &kv : first) {
    if (kv.second.first == -2) continue;
    int e = kv.second.first, f = kv.second.second;
    int b = bc[e * nFE + f];
    if (b < 0) { fprintf(stderr, "oracle: unmatched face %d of element %d has no BC\n", f, e); return false; }
    OFace F;
    F.eL = e; F.fL = f; F.eR = -1; F.fR = -1; F.relRot = -1; F.bc = b;
    s.faces.push_back(F);
  }
  /* interior faces first, as geo::setupElesFaces orders them */
  std::stable_sort(s.faces.begin(), s.faces.end(), [](const OFace &a, const OFace &b) { return (a.eR < 0) < (b.eR < 0); });
  for (auto &F : s.faces) {
    F.fptL.resize(nFF);
    for (int i = 0; i < nFF; i++) F.fptL[i] = F.fL * nFF + i;
    if (F.eR >= 0) {
      F.fptR.resize(nFF);
      if (d == 2) {
        for (int i = 0; i < nFF; i++) F.fptR[i] = F.fR * nFF + nFF - 1 - i;
      } else {
        int start = nFF * F.fR, end = nFF * (F.fR + 1);
        for (int i = 0; i < nFF; i++) {
          int ifp = i % (P + 1), jfp = i / (P + 1);
          switch (F.relRot) {
            case 0: F.fptR[i] = start + ifp * (P + 1) + jfp; break;
            case 1: F.fptR[i] = start + P - ifp + jfp * (P + 1); break;
            case 2: F.fptR[i] = end - 1 - (ifp * (P + 1) + jfp); break;
            case 3: F.fptR[i] = end - (P + 1) * (jfp + 1) + ifp; break;
          }
        }
      }
    }
    F.Fn.assign((size_t)nFF * s.nV, 0.0);
  }
  return true;
}

/* ---------------------------------------------------------------- flux.cpp */
void inviscidFlux(const orc_params &p, const double *U, double F[3][5]) { /* :37-88 */
  if (p.equation == 0) {
    F[0][0] = p.advectVx * U[0];
    F[1][0] = p.advectVy * U[0];
    if (p.nDims == 3) F[2][0] = p.advectVz * U[0];
  } else if (p.nDims == 2) {
    double rho = U[0], u = U[1] / rho, v = U[2] / rho, E = U[3];
    double pr = (p.gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
    F[0][0] = rho * u; F[1][0] = rho * v;
    F[0][1] = rho * u * u + pr; F[1][1] = rho * u * v;
    F[0][2] = rho * v * u; F[1][2] = rho * v * v + pr;
    F[0][3] = (E + pr) * u; F[1][3] = (E + pr) * v;
  } else {
    double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = U[3] / rho, E = U[4];
    double pr = (p.gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v + w * w));
    F[0][0] = rho * u; F[1][0] = rho * v; F[2][0] = rho * w;
    F[0][1] = rho * u * u + pr; F[1][1] = rho * u * v; F[2][1] = rho * u * w;
    F[0][2] = rho * v * u; F[1][2] = rho * v * v + pr; F[2][2] = rho * v * w;
    F[0][3] = rho * w * u; F[1][3] = rho * w * v; F[2][3] = rho * w * w + pr;
    F[0][4] = (E + pr) * u; F[1][4] = (E + pr) * v; F[2][4] = (E + pr) * w;
  }
}

/* viscousFlux (src/flux.cpp:90-226), including its index quirks:
 * tauxz = mu(du/dz + dv/dx), tauyz = mu(du/dz + dv/dy) (:197-198) and
 * Fvis[0][3] = -tauzz, Fvis[1][3] = -tauyz (:216-217). gradU is [d][nV]. */
void viscousFlux(const orc_params &p, const double *U, const double *g, double Fv[3][5]) {
  int nD = p.nDims, nV = nD + 2;
  auto G = [&](int a, int b) { return g[a * nV + b]; };
  double rho = U[0], u = U[1] / rho, v = U[2] / rho;
  double e = U[nD + 1] / rho - 0.5 * (u * u + v * v);
  double w;
  if (nD == 3) { w = U[3] / rho; e -= 0.5 * (w * w); } else w = 0.;
  double dRho_dx = G(0, 0), dRhoU_dx = G(0, 1), dRhoV_dx = G(0, 2), dE_dx = G(0, nD + 1);
  double dRho_dy = G(1, 0), dRhoU_dy = G(1, 1), dRhoV_dy = G(1, 2), dE_dy = G(1, nD + 1);
  double dRho_dz = 0, dRhoU_dz = 0, dRhoV_dz = 0, dRhoW_dx = 0, dRhoW_dy = 0, dRhoW_dz = 0, dE_dz = 0;
  if (nD == 3) {
    dRho_dz = G(2, 0); dRhoU_dz = G(2, 1); dRhoV_dz = G(2, 2);
    dRhoW_dx = G(0, 3); dRhoW_dy = G(1, 3); dRhoW_dz = G(2, 3); dE_dz = G(2, 4);
  }
  double mu = p.mu_inf;
  if (!p.fixVis) {
    double rt = (p.gamma - 1.0) * e / (p.rt_inf);
    mu *= pow(rt, 1.5) * (1. + (p.c_sth)) / (rt + (p.c_sth));
  }
  double du_dx = (dRhoU_dx - dRho_dx * u) / rho, du_dy = (dRhoU_dy - dRho_dy * u) / rho;
  double dv_dx = (dRhoV_dx - dRho_dx * v) / rho, dv_dy = (dRhoV_dy - dRho_dy * v) / rho;
  double du_dz = 0, dv_dz = 0, dw_dx = 0, dw_dy = 0, dw_dz = 0;
  if (nD == 3) {
    du_dz = (dRhoU_dz - dRho_dz * u) / rho;
    dv_dz = (dRhoV_dz - dRho_dz * v) / rho;
    dw_dx = (dRhoW_dx - dRho_dx * w) / rho;
    dw_dy = (dRhoW_dy - dRho_dy * w) / rho;
    dw_dz = (dRhoW_dz - dRho_dz * w) / rho;
  }
  (void)dv_dz;
  double dK_dx, dK_dy, dK_dz;
  if (nD == 2) {
    dK_dx = 0.5 * (u * u + v * v) * dRho_dx + rho * (u * du_dx + v * dv_dx);
    dK_dy = 0.5 * (u * u + v * v) * dRho_dy + rho * (u * du_dy + v * dv_dy);
    dK_dz = 0;
  } else {
    dK_dx = 0.5 * (u * u + v * v + w * w) * dRho_dx + rho * (u * du_dx + v * dv_dx + w * dw_dx);
    dK_dy = 0.5 * (u * u + v * v + w * w) * dRho_dy + rho * (u * du_dy + v * dv_dy + w * dw_dy);
    dK_dz = 0.5 * (u * u + v * v + w * w) * dRho_dz + rho * (u * du_dz + v * dv_dz + w * dw_dz);
  }
  double de_dx = (dE_dx - dK_dx - dRho_dx * e) / rho;
  double de_dy = (dE_dy - dK_dy - dRho_dy * e) / rho;
  double de_dz = 0;
  if (nD == 3) de_dz = (dE_dz - dK_dz - dRho_dz * e) / rho;
  double diag = (du_dx + dv_dy + dw_dz) / 3.0;
  double tauxx = 2.0 * mu * (du_dx - diag), tauyy = 2.0 * mu * (dv_dy - diag);
  double tauxy = mu * (du_dy + dv_dx);
  double tauxz = 0, tauyz = 0, tauzz = 0;
  if (nD == 3) {
    tauxz = mu * (du_dz + dv_dx);
    tauyz = mu * (du_dz + dv_dy);
    tauzz = 2.0 * mu * (dw_dz - diag);
  }
  Fv[0][0] = 0.0; Fv[0][1] = -tauxx; Fv[0][2] = -tauxy;
  Fv[0][nD + 1] = -(u * tauxx + v * tauxy + w * tauxz + (mu / p.prandtl) * (p.gamma) * de_dx);
  Fv[1][0] = 0.0; Fv[1][1] = -tauxy; Fv[1][2] = -tauyy;
  Fv[1][nD + 1] = -(u * tauxy + v * tauyy + w * tauyz + (mu / p.prandtl) * (p.gamma) * de_dy);
  if (nD == 3) {
    Fv[0][3] = -tauzz; Fv[1][3] = -tauyz;
    Fv[2][0] = 0.0; Fv[2][1] = -tauxz; Fv[2][2] = -tauyz; Fv[2][3] = -tauzz;
    Fv[2][4] = -(u * tauxz + v * tauyz + w * tauzz + (mu / p.prandtl) * (p.gamma) * de_dz);
  }
}
void viscousFluxAD(const orc_params &p, const double *g /*[d][1]*/, double Fv[3][5]) { /* :361-366 */
  Fv[0][0] = -p.diffD * g[0];
  Fv[1][0] = -p.diffD * g[1];
  if (p.nDims == 3) Fv[2][0] = -p.diffD * g[2];
}

/* ------------------------------------------------ face.cpp / boundFace.cpp */
/* Rusanov, one flux point (src/face.cpp:289-356). Returns the wave speed. */
double rusanov(const orc_params &p, const double *UL, const double *UR, const double *n, double *Fn) {
  double FL[3][5], FR[3][5];
  inviscidFlux(p, UL, FL);
  inviscidFlux(p, UR, FR);
  double FnL[5] = {0, 0, 0, 0, 0}, FnR[5] = {0, 0, 0, 0, 0};
  double rhoL = UL[0], rhoR = UR[0];
  double uL = UL[1] / rhoL, uR = UR[1] / rhoR, vL = UL[2] / rhoL, vR = UR[2] / rhoR;
  double wL, pL, vnL = 0., wR, pR, vnR = 0.;
  if (p.nDims == 2) {
    pL = (p.gamma - 1.0) * (UL[3] - 0.5 * rhoL * (uL * uL + vL * vL));
    pR = (p.gamma - 1.0) * (UR[3] - 0.5 * rhoR * (uR * uR + vR * vR));
  } else {
    wL = UL[3] / rhoL; wR = UR[3] / rhoR;
    pL = (p.gamma - 1.0) * (UL[4] - 0.5 * rhoL * (uL * uL + vL * vL + wL * wL));
    pR = (p.gamma - 1.0) * (UR[4] - 0.5 * rhoR * (uR * uR + vR * vR + wR * wR));
  }
  int nV = p.nDims + 2;
  for (int dim = 0; dim < p.nDims; dim++) {
    vnL += n[dim] * UL[dim + 1] / rhoL;
    vnR += n[dim] * UR[dim + 1] / rhoR;
    for (int i = 0; i < nV; i++) { FnL[i] += n[dim] * FL[dim][i]; FnR[i] += n[dim] * FR[dim][i]; }
  }
  double csqL = max(p.gamma * pL / rhoL, 0.0), csqR = max(p.gamma * pR / rhoR, 0.0);
  double eigL = std::fabs(vnL) + sqrt(csqL), eigR = std::fabs(vnR) + sqrt(csqR);
  double eig = max(eigL, eigR);
  for (int i = 0; i < nV; i++) Fn[i] = 0.5 * (FnL[i] + FnR[i] - eig * (UR[i] - UL[i]));
  return max(eigL, eigR);
}

/* Roe with entropy fix, 2D (src/face.cpp:358-484). */
void roe(const orc_params &p, const double *UL, const double *UR, const double *n, double *Fn) {
  double gamma = p.gamma;
  int nD = p.nDims;
  double vL[3], vR[3], um[3], du[5];
  for (int i = 0; i < nD; i++) { vL[i] = UL[i + 1] / UL[0]; vR[i] = UR[i + 1] / UR[0]; }
  double pL, pR;
  if (nD == 2) {
    pL = (gamma - 1.0) * (UL[3] - (0.5 * UL[0] * (vL[0] * vL[0] + vL[1] * vL[1])));
    pR = (gamma - 1.0) * (UR[3] - (0.5 * UR[0] * (vR[0] * vR[0] + vR[1] * vR[1])));
  } else {
    pL = (gamma - 1.0) * (UL[4] - (0.5 * UL[0] * (vL[0] * vL[0] + vL[1] * vL[1] + vL[2] * vL[2])));
    pR = (gamma - 1.0) * (UR[4] - (0.5 * UR[0] * (vR[0] * vR[0] + vR[1] * vR[1] + vR[2] * vR[2])));
  }
  double hL = (UL[nD + 1] + pL) / UL[0], hR = (UR[nD + 1] + pR) / UR[0];
  double sq_rho = sqrt(UR[0] / UL[0]);
  double rrho = 1. / (sq_rho + 1.);
  double usq = 0., unm = 0., vgn = 0.;
  for (int i = 0; i < nD; i++) {
    um[i] = rrho * (vL[i] + sq_rho * vR[i]);
    usq += 0.5 * um[i] * um[i];
    unm += um[i] * n[i];
  }
  double hm = rrho * (hL + sq_rho * hR);
  double am_sq = (gamma - 1.) * (hm - usq);
  double am = sqrt(am_sq);
  double rhoUnL = 0., rhoUnR = 0.;
  for (int i = 0; i < nD; i++) { rhoUnL += UL[i + 1] * n[i]; rhoUnR += UR[i + 1] * n[i]; }
  Fn[0] = rhoUnL + rhoUnR;
  Fn[1] = rhoUnL * vL[0] + rhoUnR * vR[0] + (pL + pR) * n[0];
  Fn[2] = rhoUnL * vL[1] + rhoUnR * vR[1] + (pL + pR) * n[1];
  Fn[3] = rhoUnL * hL + rhoUnR * hR;
  for (int i = 0; i < nD + 2; i++) du[i] = UR[i] - UL[i];
  double lambda0 = std::abs(unm - vgn), lambdaP = std::abs(unm - vgn + am), lambdaM = std::abs(unm - vgn - am);
  double eps = 0.5 * (std::abs(rhoUnL / UL[0] - rhoUnR / UR[0]) +
                      std::abs(sqrt(gamma * pL / UL[0]) - sqrt(gamma * pR / UR[0])));
  if (lambda0 < 2. * eps) lambda0 = 0.25 * lambda0 * lambda0 / eps + eps;
  if (lambdaP < 2. * eps) lambdaP = 0.25 * lambdaP * lambdaP / eps + eps;
  if (lambdaM < 2. * eps) lambdaM = 0.25 * lambdaM * lambdaM / eps + eps;
  double a2 = 0.5 * (lambdaP + lambdaM) - lambda0;
  double a3 = 0.5 * (lambdaP - lambdaM) / am;
  double a1 = a2 * (gamma - 1.) / am_sq;
  double a4 = a3 * (gamma - 1.);
  double a5 = usq * du[0] - um[0] * du[1] - um[1] * du[2] + du[3];
  double a6 = unm * du[0] - n[0] * du[1] - n[1] * du[2];
  double aL1 = a1 * a5 - a3 * a6, bL1 = a4 * a5 - a2 * a6;
  Fn[0] -= lambda0 * du[0] + aL1;
  Fn[1] -= lambda0 * du[1] + aL1 * um[0] + bL1 * n[0];
  Fn[2] -= lambda0 * du[2] + aL1 * um[1] + bL1 * n[1];
  Fn[3] -= lambda0 * du[3] + aL1 * hm + bL1 * unm;
  for (int i = 0; i < nD + 2; i++) Fn[i] *= 0.5;
}

/* Lax-Friedrichs for advection (src/face.cpp:486-514). Returns wave speed. */
double laxFriedrichs(const orc_params &p, double uL, double uR, const double *n, double *Fn) {
  double uAvg = 0.5 * (uL + uR), uDiff = uL - uR;
  double vNorm = p.advectVx * n[0] + p.advectVy * n[1];
  if (p.nDims == 3) vNorm += p.advectVz * n[2];
  Fn[0] = vNorm * uAvg + 0.5 * p.lambda * std::abs(vNorm) * uDiff;
  return std::abs(vNorm);
}

/* boundFace::applyBCs for Navier-Stokes (src/boundFace.cpp:33-277). */
void applyBC(const orc_params &p, int bcType, const double *UL, const double *n, double *UR) {
  int nD = p.nDims;
  double rhoR = 0, pR = 0, ER = 0, TR;
  double vL[3] = {0, 0, 0}, vR[3] = {0, 0, 0}, vG[3] = {0, 0, 0};
  double vBound[3] = {p.uBound, p.vBound, p.wBound};
  double gamma = p.gamma, gmo = gamma - 1.;
  double rhoL = UL[0], eL = UL[nD + 1];
  for (int i = 0; i < nD; i++) vL[i] = UL[i + 1] / UL[0];
  double vSq = 0;
  for (int i = 0; i < nD; i++) vSq += (vL[i] * vL[i]);
  double pL = (gamma - 1.0) * (eL - 0.5 * rhoL * vSq);
  if (bcType == BC_SUB_IN) {
    rhoR = p.rhoBound;
    for (int i = 0; i < nD; i++) vR[i] = vBound[i];
    pR = pL;
    vSq = 0;
    for (int i = 0; i < nD; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
  } else if (bcType == BC_SUB_OUT) {
    rhoR = rhoL;
    for (int i = 0; i < nD; i++) vR[i] = vL[i];
    pR = p.pBound;
    vSq = 0.;
    for (int i = 0; i < nD; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
  } else if (bcType == BC_SUP_IN) {
    rhoR = p.rhoBound;
    vR[0] = p.uBound; vR[1] = p.vBound; vR[2] = p.wBound;
    pR = p.pBound;
    vSq = 0.;
    for (int i = 0; i < nD; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
  } else if (bcType == BC_SUP_OUT) {
    rhoR = rhoL;
    for (int i = 0; i < nD; i++) vR[i] = vL[i];
    ER = eL;
  } else if (bcType == BC_SLIP || bcType == BC_SYMMETRY) {
    rhoR = rhoL;
    double vnL = 0.;
    for (int i = 0; i < nD; i++) vnL += (vL[i] - vG[i]) * n[i];
    for (int i = 0; i < nD; i++) vR[i] = vL[i] - (2.0) * vnL * n[i];
    ER = eL;
  } else if (bcType == BC_ISO_NOSLIP_MOVING) {
    pR = pL;
    TR = p.TWall;
    rhoR = pR / (p.RGas * TR);
    vR[0] = vG[0] + p.uWall; vR[1] = vG[1] + p.vWall;
    if (nD == 3) vR[2] = vG[2] + p.wWall;
    vSq = 0.;
    for (int i = 0; i < nD; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
  } else if (bcType == BC_ISO_NOSLIP) {
    pR = pL;
    TR = p.TWall;
    rhoR = pR / (p.RGas * TR);
    for (int i = 0; i < nD; i++) vR[i] = vG[i];
    vSq = 0.;
    for (int i = 0; i < nD; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
  } else if (bcType == BC_ADI_NOSLIP) {
    rhoR = rhoL;
    pR = pL;
    for (int i = 0; i < nD; i++) vR[i] = vG[i];
    vSq = 0.;
    for (int i = 0; i < nD; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - 1.0)) + 0.5 * rhoR * vSq;
  } else if (bcType == BC_CHAR) {
    double vnL = 0., vnB = 0.;
    for (int i = 0; i < nD; i++) vnL += vL[i] * n[i];
    for (int i = 0; i < nD; i++) vnB += vBound[i] * n[i];
    double cL = sqrt(gamma * pL / rhoL);
    double cB = sqrt(gamma * p.pBound / p.rhoBound);
    double R_L, R_B;
    if (std::abs(vnB) >= cB && vnL >= 0) R_L = vnB + 2. / gmo * cB;
    else R_L = vnL + 2. / gmo * cL;
    if (std::abs(vnB) >= cB && vnL < 0) R_B = vnL - 2. / gmo * cL;
    else R_B = vnB - 2. / gmo * cB;
    double rhoFac = .25 * (gamma - 1.) * (R_L - R_B);
    double rhoBG = rhoFac * rhoFac / gamma;
    if (vnL < 0) rhoBG *= pow(p.rhoBound, gamma) / p.pBound;
    else rhoBG *= pow(rhoL, gamma) / pL;
    rhoR = pow(rhoBG, 1. / gmo);
    pR = rhoFac * rhoFac * rhoR / gamma;
    double VB = 0.5 * (R_L + R_B);
    for (int i = 0; i < nD; i++) {
      if (vnL < 0) vR[i] = vBound[i] + (VB - vnB) * n[i];
      else vR[i] = vL[i] + (VB - vnL) * n[i];
    }
    double vMag2 = 0;
    for (int i = 0; i < nD; i++) vMag2 += vR[i] * vR[i];
    ER = pR / gmo + .5 * rhoR * vMag2;
  } else {
    fprintf(stderr, "oracle: Boundary condition %d not recognized\n", bcType);
    abort();
  }
  UR[0] = rhoR;
  for (int i = 0; i < nD; i++) UR[i + 1] = rhoR * vR[i];
  UR[nD + 1] = ER;
}

/* boundFace::applyViscousBCs (src/boundFace.cpp:279-320), adiabatic wall. */
void applyViscousBC(const orc_params &p, int bcType, const double *UL, const double *UR,
                    const double *gL /*[d][nV]*/, double *gR) {
  int nD = p.nDims, nV = nD + 2;
  if (bcType != BC_ADI_NOSLIP) return;
  for (int i = 0; i < nD * nV; i++) gR[i] = gL[i];
  double rhovSq = 0.;
  for (int dim = 0; dim < nD; dim++) rhovSq += UL[dim + 1] * UL[dim + 1];
  double pL = (p.gamma - 1.) * (UL[nD + 1] - 0.5 * rhovSq / UL[0]);
  double pR = pL;
  double e = pR / ((p.gamma - 1.) * UR[0]);
  double gradVel[3][3];
  for (int d1 = 0; d1 < nD; d1++)
    for (int d2 = 0; d2 < nD; d2++)
      gradVel[d1][d2] = (gR[d1 * nV + d2 + 1] - gR[d1 * nV + 0] * UR[d2 + 1] / UR[0]) / UR[0];
  double vSq = 0.;
  for (int dim = 0; dim < nD; dim++) vSq += UR[dim + 1] * UR[dim + 1] / (UR[0] * UR[0]);
  for (int d1 = 0; d1 < nD; d1++) {
    gR[d1 * nV + nD + 1] = (e + 0.5 * vSq) * gR[d1 * nV + 0];
    for (int d2 = 0; d2 < nD; d2++) gR[d1 * nV + nD + 1] += UR[d2 + 1] * gradVel[d2][d1];
  }
}

/* face::calcInviscidFlux (src/face.cpp:132-175) for one face. */
void faceInviscid(orc_solver &s, OFace &F) {
  const orc_params &p = s.p;
  int nFF = s.nFptFace, nV = s.nV, d = s.nDims, nE = s.nE;
  vector<double> UL(nV), UR(nV, 0.0), UC(nV);
  for (int i = 0; i < nFF; i++) {
    int fl = F.fptL[i];
    for (int k = 0; k < nV; k++) UL[k] = s.U_fpts[((size_t)fl * nE + F.eL) * nV + k];
    const double *n = &s.norm_fpts[((size_t)fl * nE + F.eL) * d];
    double dAL = s.dA_fpts[(size_t)fl * nE + F.eL];
    int fr = F.eR >= 0 ? F.fptR[i] : -1;
    if (F.eR >= 0) {
      for (int k = 0; k < nV; k++) UR[k] = s.U_fpts[((size_t)fr * nE + F.eR) * nV + k];
    } else if (p.equation == 1) {
      applyBC(p, F.bc, UL.data(), n, UR.data());
    } else {
      for (int k = 0; k < nV; k++) UR[k] = 0.0; /* advection BCs leave the ghost state at zero */
    }
    double *Fn = &F.Fn[(size_t)i * nV];
    double ws;
    if (p.equation == 0) ws = laxFriedrichs(p, UL[0], UR[0], n, Fn), s.waveSp[(size_t)F.eL * s.nF + fl] = ws;
    else if (F.eR < 0 || p.riemannType == 0) s.waveSp[(size_t)F.eL * s.nF + fl] = rusanov(p, UL.data(), UR.data(), n, Fn);
    else roe(p, UL.data(), UR.data(), n, Fn);
    for (int k = 0; k < nV; k++) s.Fn_fpts[((size_t)fl * nE + F.eL) * nV + k] = Fn[k] * dAL;
    if (p.viscous) {
      /* ldgSolution (src/face.cpp:582-607) */
      if (F.eR < 0) {
        for (int k = 0; k < nV; k++) UC[k] = 0.5 * (UL[k] + UR[k]);
      } else {
        double pf = p.penFact;
        if (d == 2) { if (n[0] + n[1] < 0) pf = -p.penFact; }
        else if (n[0] + n[1] + sqrt(2.) * n[2] < 0) pf = -p.penFact;
        for (int k = 0; k < nV; k++) UC[k] = 0.5 * (UL[k] + UR[k]) - pf * (UL[k] - UR[k]);
      }
      for (int k = 0; k < nV; k++) s.dUc_fpts[((size_t)fl * nE + F.eL) * nV + k] = UC[k] - UL[k];
    }
    if (F.eR >= 0) {
      double dAR = s.dA_fpts[(size_t)fr * nE + F.eR];
      for (int k = 0; k < nV; k++) s.Fn_fpts[((size_t)fr * nE + F.eR) * nV + k] = -Fn[k] * dAR;
      if (p.viscous)
        for (int k = 0; k < nV; k++) s.dUc_fpts[((size_t)fr * nE + F.eR) * nV + k] = UC[k] - UR[k];
    }
  }
}

/* face::calcViscousFlux (src/face.cpp:177-287) for one face. */
void faceViscous(orc_solver &s, OFace &F) {
  const orc_params &p = s.p;
  int nFF = s.nFptFace, nV = s.nV, d = s.nDims, nE = s.nE, nF = s.nF;
  vector<double> UL(nV), UR(nV, 0.0), gL(d * nV), gR(d * nV, 0.0);
  double FL[3][5], FR[3][5], Fc[3][5];
  for (int i = 0; i < nFF; i++) {
    int fl = F.fptL[i];
    int fr = F.eR >= 0 ? F.fptR[i] : -1;
    for (int k = 0; k < nV; k++) UL[k] = s.U_fpts[((size_t)fl * nE + F.eL) * nV + k];
    const double *n = &s.norm_fpts[((size_t)fl * nE + F.eL) * d];
    for (int dim = 0; dim < d; dim++)
      for (int k = 0; k < nV; k++) gL[dim * nV + k] = s.dU_fpts[s.i4(dim, fl, nF, F.eL, k)];
    if (F.eR >= 0) {
      for (int k = 0; k < nV; k++) UR[k] = s.U_fpts[((size_t)fr * nE + F.eR) * nV + k];
      for (int dim = 0; dim < d; dim++)
        for (int k = 0; k < nV; k++) gR[dim * nV + k] = s.dU_fpts[s.i4(dim, fr, nF, F.eR, k)];
    } else if (p.equation == 1) {
      applyBC(p, F.bc, UL.data(), n, UR.data());
      applyViscousBC(p, F.bc, UL.data(), UR.data(), gL.data(), gR.data());
    }
    double *Fn = &F.Fn[(size_t)i * nV];
    if (p.equation == 1) {
      if (F.eR < 0) {
        if (F.bc == BC_ADI_NOSLIP) {
          viscousFlux(p, UR.data(), gR.data(), FR);
          for (int dim = 0; dim < d; dim++)
            for (int k = 0; k < nV; k++) Fc[dim][k] = FR[dim][k] + p.tau * n[dim] * (UL[k] - UR[k]);
        } else {
          viscousFlux(p, UL.data(), gL.data(), FL);
          for (int dim = 0; dim < d; dim++)
            for (int k = 0; k < nV; k++) Fc[dim][k] = FL[dim][k] + p.tau * n[dim] * (UL[k] - UR[k]);
        }
      } else {
        viscousFlux(p, UL.data(), gL.data(), FL);
        viscousFlux(p, UR.data(), gR.data(), FR);
        double pf = p.penFact;
        if (d == 2) { if (n[0] + n[1] < 0) pf = -p.penFact; }
        else if (n[0] + n[1] + sqrt(2.) * n[2] < 0) pf = -p.penFact;
        double nx = n[0], ny = n[1], nz = d == 3 ? n[2] : 0;
        for (int k = 0; k < nV; k++) {
          double dF0 = FL[0][k] - FR[0][k], dF1 = FL[1][k] - FR[1][k];
          double dU = UL[k] - UR[k];
          if (d == 2) {
            Fc[0][k] = 0.5 * (FL[0][k] + FR[0][k]) + pf * nx * (nx * (dF0) + ny * (dF1)) + p.tau * nx * (dU);
            Fc[1][k] = 0.5 * (FL[1][k] + FR[1][k]) + pf * ny * (nx * (dF0) + ny * (dF1)) + p.tau * ny * (dU);
          } else {
            double dF2 = FL[1][k] - FR[2][k]; /* as written at src/face.cpp:245 */
            Fc[0][k] = 0.5 * (FL[0][k] + FR[0][k]) + pf * nx * (nx * (dF0) + ny * (dF1) + nz * (dF2)) + p.tau * nx * (dU);
            Fc[1][k] = 0.5 * (FL[1][k] + FR[1][k]) + pf * ny * (nx * (dF0) + ny * (dF1) + nz * (dF2)) + p.tau * ny * (dU);
            Fc[2][k] = 0.5 * (FL[2][k] + FR[2][k]) + pf * nz * (nx * (dF0) + ny * (dF1) + nz * (dF2)) + p.tau * nz * (dU);
          }
        }
      }
      for (int dim = 0; dim < d; dim++)
        for (int k = 0; k < nV; k++) Fn[k] += Fc[dim][k] * n[dim];
    } else {
      viscousFluxAD(p, gL.data(), FL);
      viscousFluxAD(p, gR.data(), FR);
      double t = 0; /* centralFlux (src/flux.cpp:379-387) */
      for (int j = 0; j < d; j++) t += 0.5 * (FL[j][0] + FR[j][0]) * n[j];
      Fn[0] += t;
    }
    double dAL = s.dA_fpts[(size_t)fl * nE + F.eL];
    for (int k = 0; k < nV; k++) s.Fn_fpts[((size_t)fl * nE + F.eL) * nV + k] = Fn[k] * dAL;
    if (F.eR >= 0) {
      double dAR = s.dA_fpts[(size_t)fr * nE + F.eR];
      for (int k = 0; k < nV; k++) s.Fn_fpts[((size_t)fr * nE + F.eR) * nV + k] = -Fn[k] * dAR;
    }
  }
}

double cflLimit(int order) { /* getCFLLimit, src/global.cpp:45-66 */
  static const double t[6] = {1.393, 0.464, 0.235, 0.1453, 0.100, 0.0736};
  if (order < 0 || order > 5) { fprintf(stderr, "oracle: CFL limit not available\n"); abort(); }
  return t[order];
}

/* ele::calcWaveSpFpts (src/ele.cpp:1031-1084) for every element. */
void calcWaveSpFpts(orc_solver &s) {
  const orc_params &p = s.p;
  int nF = s.nF, nE = s.nE, nV = s.nV, d = s.nDims;
  for (int e = 0; e < nE; e++)
    for (int f = 0; f < nF; f++) {
      const double *n = &s.norm_fpts[((size_t)f * nE + e) * d];
      double &ws = s.waveSp[(size_t)e * nF + f];
      if (p.equation == 0) {
        double u = p.advectVx, v = p.advectVy, w = 0.;
        if (d == 3) w = p.advectVz;
        double vN = u * n[0] + v * n[1];
        if (d == 3) vN += w * n[2];
        double vgN = 0;
        double vTot = std::abs(vN - vgN);
        vN = std::abs(vN);
        vgN = std::abs(vgN);
        ws = max(vTot, max(vN, vgN));
      } else {
        const double *U = &s.U_fpts[((size_t)f * nE + e) * nV];
        double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = 0;
        if (d == 3) w = U[3] / rho;
        double rhoVSq = rho * (u * u + v * v + w * w);
        double pr = (p.gamma - 1) * (U[d + 1] - 0.5 * rhoVSq);
        double vN = u * n[0] + v * n[1];
        if (d == 3) vN += w * n[2];
        double vgN = 0;
        double csq = max(p.gamma * pr / rho, 0.0);
        ws = (std::abs(vN - vgN) + sqrt(csq));
      }
    }
}

}  // namespace

/* ================================================================== API */
extern "C" {

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

void orc_point_flux(const orc_params *p, const double *U, const double *gradU, double *Finv, double *Fvis) {
  int d = p->nDims, nV = p->equation == 0 ? 1 : d + 2;
  double F[3][5] = {{0}}, G[3][5] = {{0}};
  inviscidFlux(*p, U, F);
  if (gradU && Fvis) {
    if (p->equation == 1) viscousFlux(*p, U, gradU, G);
    else viscousFluxAD(*p, gradU, G);
  }
  for (int a = 0; a < d; a++)
    for (int k = 0; k < nV; k++) {
      Finv[a * nV + k] = F[a][k];
      if (Fvis) Fvis[a * nV + k] = G[a][k];
    }
}
double orc_point_rusanov(const orc_params *p, const double *UL, const double *UR, const double *n, double *Fn) {
  return rusanov(*p, UL, UR, n, Fn);
}
void orc_point_roe(const orc_params *p, const double *UL, const double *UR, const double *n, double *Fn) {
  roe(*p, UL, UR, n, Fn);
}
double orc_point_lf(const orc_params *p, double uL, double uR, const double *n, double *Fn) {
  return laxFriedrichs(*p, uL, uR, n, Fn);
}
void orc_point_ldg_uc(const orc_params *p, const double *UL, const double *UR, const double *n, double *UC) {
  int d = p->nDims, nV = d + 2;
  double pf = p->penFact;
  if (d == 2) { if (n[0] + n[1] < 0) pf = -p->penFact; }
  else if (n[0] + n[1] + sqrt(2.) * n[2] < 0) pf = -p->penFact;
  for (int k = 0; k < nV; k++) UC[k] = 0.5 * (UL[k] + UR[k]) - pf * (UL[k] - UR[k]);
}
void orc_point_bc(const orc_params *p, int bcType, const double *UL, const double *n, double *UR) {
  applyBC(*p, bcType, UL, n, UR);
}

orc_solver *orc_create(const orc_params *p, int nEles, int nNodes, const double *xv, const int *c2v, const int *bc) {
  orc_solver *s = new orc_solver();
  s->p = *p;
  s->nDims = p->nDims;
  s->P = p->order;
  s->nE = nEles;
  s->nNodes = nNodes;
  s->nV = p->equation == 0 ? 1 : p->nDims + 2;
  if (p->nDims == 3 && nNodes != 8) { fprintf(stderr, "oracle: only 8-node hexahedra\n"); delete s; return nullptr; }
  if (p->nDims == 3 && p->equation == 1 && p->riemannType == 1) {
    fprintf(stderr, "oracle: Roe not implemented in 3D (src/face.cpp:362)\n"); delete s; return nullptr;
  }
  /* RK tables, src/input.cpp:424-461 */
  switch (p->timeType) {
    case 0: s->nRK = 1; s->RKa = {0}; s->RKb = {1}; break;
    case 2: s->nRK = 2; s->RKa = {0, 1.}; s->RKb = {1. / 2., 1. / 2.}; break;
    case 4: s->nRK = 4; s->RKa = {0., .5, .5, 1.}; s->RKb = {1. / 6., 1. / 3., 1. / 3., 1. / 6.}; break;
    case 5: s->nRK = 4; s->RKa = {0., 1. / 4., 1. / 3., 1. / 2., 1.0}; s->RKb = {0.}; break;
    default: fprintf(stderr, "oracle: timeType %d unsupported\n", p->timeType); delete s; return nullptr;
  }
  setupOperators(*s);
  s->nodes.assign((size_t)nNodes * nEles * s->nDims, 0);
  for (int e = 0; e < nEles; e++)
    for (int n = 0; n < nNodes; n++)
      for (int d = 0; d < s->nDims; d++)
        s->nodes[((size_t)n * nEles + e) * s->nDims + d] = xv[((size_t)e * nNodes + n) * s->nDims + d];
  if (!setupGeometry(*s) || !setupFaces(*s, c2v, bc)) { delete s; return nullptr; }
  size_t nSE = (size_t)s->nS * nEles * s->nV, nFE = (size_t)s->nF * nEles * s->nV;
  s->U.assign(nSE, 0); s->U0.assign(nSE, 0);
  s->U_fpts.assign(nFE, 0); s->Fn_fpts.assign(nFE, 0); s->disFn.assign(nFE, 0); s->dUc_fpts.assign(nFE, 0);
  s->F_spts.assign(nSE * s->nDims, 0);
  s->dU_spts.assign(nSE * s->nDims, 0);
  s->dU_fpts.assign(nFE * s->nDims, 0);
  s->divF.assign(s->nRK, vector<double>(nSE, 0));
  s->waveSp.assign((size_t)nEles * s->nF, 0);
  s->eleDt.assign(nEles, 0);
  s->dt = p->dtType == 0 ? p->dt : 0;
  return s;
}

void orc_destroy(orc_solver *s) { delete s; }
int orc_nspts(const orc_solver *s) { return s->nS; }
int orc_nfpts(const orc_solver *s) { return s->nF; }
int orc_nfields(const orc_solver *s) { return s->nV; }
int orc_nfaces(const orc_solver *s) { return (int)s->faces.size(); }
double orc_get_dt(const orc_solver *s) { return s->dt; }
double orc_get_time(const orc_solver *s) { return s->time; }
int orc_get_iter(const orc_solver *s) { return s->iter; }

static const vector<double> *named(const orc_solver *s_, const std::string &nm) {
  orc_solver *s = const_cast<orc_solver *>(s_);
  if (nm == "U_spts") return &s->U;
  if (nm == "U0") return &s->U0;
  if (nm == "U_fpts") return &s->U_fpts;
  if (nm == "F_spts") return &s->F_spts;
  if (nm == "Fn_fpts") return &s->Fn_fpts;
  if (nm == "disFn_fpts") return &s->disFn;
  if (nm == "dU_spts") return &s->dU_spts;
  if (nm == "dU_fpts") return &s->dU_fpts;
  if (nm == "dUc_fpts") return &s->dUc_fpts;
  if (nm.rfind("divF_spts", 0) == 0 && nm.size() == 10) {
    int k = nm[9] - '0';
    if (k >= 0 && k < s->nRK) return &s->divF[k];
  }
  if (nm == "pos_spts") return &s->pos_spts;
  if (nm == "JGinv_spts") return &s->JGinv_spts;
  if (nm == "detJac_spts") return &s->detJ_spts;
  if (nm == "norm_fpts") return &s->norm_fpts;
  if (nm == "dA_fpts") return &s->dA_fpts;
  if (nm == "waveSp") return &s->waveSp;
  if (nm == "opp_spts_to_fpts") return &s->E;
  if (nm == "opp_correction") return &s->C;
  for (int d = 0; d < s->nDims; d++) {
    if (nm == "opp_grad_spts" + std::to_string(d)) return &s->D[d];
    if (nm == "opp_extrapolateFn" + std::to_string(d)) return &s->Efn[d];
    if (nm == "opp_correctU" + std::to_string(d)) return &s->CU[d];
  }
  return nullptr;
}
long orc_get(const orc_solver *s, const char *name, double *out) {
  const vector<double> *v = named(s, name);
  if (!v) return -1;
  if (out) std::memcpy(out, v->data(), v->size() * sizeof(double));
  return (long)v->size();
}
long orc_set(orc_solver *s, const char *name, const double *in) {
  vector<double> *v = const_cast<vector<double> *>(named(s, name));
  if (!v) return -1;
  std::memcpy(v->data(), in, v->size() * sizeof(double));
  return (long)v->size();
}
void orc_get_faces(const orc_solver *s, int *out) {
  for (size_t i = 0; i < s->faces.size(); i++) {
    const OFace &F = s->faces[i];
    int r[6] = {F.eL, F.fL, F.eR, F.fR, F.eR >= 0 ? F.relRot : -1, F.bc};
    std::memcpy(out + 6 * i, r, sizeof r);
  }
}

/* ele::setInitialCondition (src/ele.cpp:683-790) + Taylor-Green (new). */
void orc_set_ic(orc_solver *s, int icType, double a0) {
  const orc_params &p = s->p;
  int nS = s->nS, nE = s->nE, d = s->nDims, nV = s->nV;
  double gamma = p.gamma;
  for (int sp = 0; sp < nS; sp++)
    for (int e = 0; e < nE; e++) {
      double *U = &s->U[((size_t)sp * nE + e) * nV];
      const double *x = &s->pos_spts[((size_t)sp * nE + e) * d];
      if (p.equation == 1) {
        double rho, vx, vy, vz = 0, pr;
        if (icType == 0) {
          rho = p.rhoBound; vx = p.uBound; vy = p.vBound; vz = d == 3 ? p.wBound : 0; pr = p.pBound;
          U[0] = rho; U[1] = rho * vx; U[2] = rho * vy;
          if (d == 3) U[3] = rho * vz;
          U[d + 1] = pr / (gamma - 1) + (0.5 * rho * (vx * vx + vy * vy + vz * vz));
        } else if (icType == 1) {
          double eps = 5.0, X = x[0], Y = x[1];
          double f = 1.0 - (X * X + Y * Y);
          rho = max(pow(1. - eps * eps * (gamma - 1.) / (8. * gamma * PI * PI) * exp(f), 1.0 / (gamma - 1.0) + 1e-5), 1e-3);
          vx = 1. - eps * Y / (2. * PI) * exp(f / 2.);
          vy = 1. + eps * X / (2. * PI) * exp(f / 2.);
          pr = pow(rho, gamma);
          U[0] = rho; U[1] = rho * vx; U[2] = rho * vy;
          if (d == 3) U[3] = 0.;
          U[d + 1] = pr / (gamma - 1) + (0.5 * rho * (vx * vx + vy * vy));
        } else if (icType == 10) {
          double Ma = a0, X = x[0], Y = x[1], Z = d == 3 ? x[2] : 0.0;
          double p0 = 1.0 / (gamma * Ma * Ma);
          rho = 1.0;
          vx = sin(X) * cos(Y) * cos(Z);
          vy = -cos(X) * sin(Y) * cos(Z);
          vz = 0.0;
          pr = p0 + (rho / 16.0) * (cos(2 * X) + cos(2 * Y)) * (cos(2 * Z) + 2);
          U[0] = rho; U[1] = rho * vx; U[2] = rho * vy;
          if (d == 3) U[3] = rho * vz;
          U[d + 1] = pr / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
        }
      } else {
        if (icType == 0) {
          double r2 = x[0] * x[0] + x[1] * x[1] + (d == 3 ? x[2] * x[2] : 0.0);
          U[0] = exp(-r2);
        } else if (icType == 1) {
          U[0] = 1. + sin(2. * PI * (x[0] + 5) / 10.);
        }
      }
    }
}

void orc_extrapolate_u(orc_solver *s) { /* solver::extrapolateU, src/solver.cpp:401-412 */
  dgemm(s->nF, s->nE * s->nV, s->nS, 1.0, s->E.data(), s->U.data(), 0.0, s->U_fpts.data());
}

/* solver::calcResidual (src/solver.cpp:252-291) */
void orc_calc_residual(orc_solver *s, int step) {
  const orc_params &p = s->p;
  int nS = s->nS, nF = s->nF, nE = s->nE, nV = s->nV, d = s->nDims, N = nE * nV;
  size_t sz = (size_t)nS * nE * nV;
  orc_extrapolate_u(s);
  if (p.viscous) /* calcGradU_spts :808-821 */
    for (int dim = 0; dim < d; dim++) dgemm(nS, N, nS, 1.0, s->D[dim].data(), s->U.data(), 0.0, &s->dU_spts[dim * sz]);
  /* calcInviscidFlux_spts :514-539 */
  pfor(nE, [&](int e) {
    for (int sp = 0; sp < nS; sp++) {
      double tF[3][5];
      inviscidFlux(p, &s->U[((size_t)sp * nE + e) * nV], tF);
      for (int d1 = 0; d1 < d; d1++)
        for (int k = 0; k < nV; k++) {
          double &Fo = s->F_spts[s->i4(d1, sp, nS, e, k)];
          if (p.viscous) { Fo = tF[d1][k]; continue; }
          Fo = 0.;
          for (int d2 = 0; d2 < d; d2++) Fo += s->JGinv_spts[s->g4(d1, sp, nS, e, d2)] * tF[d2][k];
        }
    }
  });
  /* calcInviscidFlux_faces :541-545 */
  int nFc = (int)s->faces.size();
  pfor(nFc, [&](int i) { faceInviscid(*s, s->faces[i]); });
  if (p.viscous) {
    /* correctGradU :823-879 */
    for (int dim = 0; dim < d; dim++) dgemm(nS, N, nF, 1.0, s->CU[dim].data(), s->dUc_fpts.data(), 1.0, &s->dU_spts[dim * sz]);
    for (int sp = 0; sp < nS; sp++)
      for (int e = 0; e < nE; e++) {
        double invDet = 1. / s->detJ_spts[(size_t)sp * nE + e];
        auto G = [&](int a, int b) { return s->JGinv_spts[s->g4(a, sp, nS, e, b)]; };
        for (int k = 0; k < nV; k++) {
          double &a0 = s->dU_spts[s->i4(0, sp, nS, e, k)], &a1 = s->dU_spts[s->i4(1, sp, nS, e, k)];
          if (d == 2) {
            double ur = a0, us = a1;
            a0 = invDet * (ur * G(0, 0) + us * G(1, 0));
            a1 = invDet * (ur * G(0, 1) + us * G(1, 1));
          } else {
            double &a2 = s->dU_spts[s->i4(2, sp, nS, e, k)];
            double ur = a0, us = a1, ut = a2;
            a0 = invDet * (ur * G(0, 0) + us * G(1, 0) + ut * G(2, 0));
            a1 = invDet * (ur * G(0, 1) + us * G(1, 1) + ut * G(2, 1));
            a2 = invDet * (ur * G(0, 2) + us * G(1, 2) + ut * G(2, 2));
          }
        }
      }
    /* extrapolateGradU :881-895 */
    size_t fz = (size_t)nF * nE * nV;
    for (int dim = 0; dim < d; dim++) dgemm(nF, N, nS, 1.0, s->E.data(), &s->dU_spts[dim * sz], 0.0, &s->dU_fpts[dim * fz]);
    /* calcViscousFlux_spts :562-596 */
    pfor(nE, [&](int e) {
      for (int sp = 0; sp < nS; sp++) {
        double tF[3][5], g[3 * 5];
        for (int dim = 0; dim < d; dim++)
          for (int k = 0; k < nV; k++) g[dim * nV + k] = s->dU_spts[s->i4(dim, sp, nS, e, k)];
        if (p.equation == 1) viscousFlux(p, &s->U[((size_t)sp * nE + e) * nV], g, tF);
        else viscousFluxAD(p, g, tF);
        for (int dim = 0; dim < d; dim++)
          for (int k = 0; k < nV; k++) tF[dim][k] += s->F_spts[s->i4(dim, sp, nS, e, k)];
        for (int d1 = 0; d1 < d; d1++)
          for (int k = 0; k < nV; k++) s->F_spts[s->i4(d1, sp, nS, e, k)] = 0.;
        for (int d1 = 0; d1 < d; d1++)
          for (int k = 0; k < nV; k++)
            for (int d2 = 0; d2 < d; d2++)
              s->F_spts[s->i4(d1, sp, nS, e, k)] += s->JGinv_spts[s->g4(d1, sp, nS, e, d2)] * tF[d2][k];
      }
    });
    /* calcViscousFlux_faces :598-603 */
    pfor(nFc, [&](int i) { faceViscous(*s, s->faces[i]); });
  }
  /* extrapolateNormalFlux (static branch) :764-786 */
  dgemm(nF, N, nS, 1.0, s->Efn[0].data(), &s->F_spts[0], 0.0, s->disFn.data());
  for (int dim = 1; dim < d; dim++) dgemm(nF, N, nS, 1.0, s->Efn[dim].data(), &s->F_spts[dim * sz], 1.0, s->disFn.data());
  /* calcDivF_spts :707-727 */
  double *div = s->divF[step].data();
  dgemm(nS, N, nS, 1.0, s->D[0].data(), &s->F_spts[0], 0.0, div);
  for (int dim = 1; dim < d; dim++) dgemm(nS, N, nS, 1.0, s->D[dim].data(), &s->F_spts[dim * sz], 1.0, div);
  /* correctDivFlux :789-806 */
  for (size_t i = 0; i < s->disFn.size(); i++) s->disFn[i] = s->Fn_fpts[i] - s->disFn[i];
  dgemm(nS, N, nF, 1.0, s->C.data(), s->disFn.data(), 1.0, div);
}

/* solver::timeStepA / timeStepB (src/solver.cpp:307-385), no PMG source. */
void orc_time_step_a(orc_solver *s, int step, double rkval) {
  int nS = s->nS, nE = s->nE, nV = s->nV;
  const double *div = s->divF[step].data();
  for (int sp = 0; sp < nS; sp++)
    for (int e = 0; e < nE; e++) {
      double dtl = s->p.dtType != 2 ? s->dt : s->eleDt[e];
      for (int k = 0; k < nV; k++) {
        size_t i = ((size_t)sp * nE + e) * nV + k;
        s->U[i] = s->U0[i] - rkval * div[i] / s->detJ_spts[(size_t)sp * nE + e] * dtl;
      }
    }
}
void orc_time_step_b(orc_solver *s, int step) {
  int nS = s->nS, nE = s->nE, nV = s->nV;
  const double *div = s->divF[step].data();
  for (int sp = 0; sp < nS; sp++)
    for (int e = 0; e < nE; e++) {
      double dtl = s->p.dtType != 2 ? s->dt : s->eleDt[e];
      for (int k = 0; k < nV; k++) {
        size_t i = ((size_t)sp * nE + e) * nV + k;
        s->U[i] -= s->RKb[step] * div[i] / s->detJ_spts[(size_t)sp * nE + e] * dtl;
      }
    }
}

/* solver::calcDt (src/solver.cpp:293-305) + ele::calcDt (src/ele.cpp:1086-1105) */
void orc_calc_dt(orc_solver *s) {
  if (s->iter == s->initIter + 1) {
    orc_extrapolate_u(s); /* U_fpts as initializeSolution / the last extrapolation left it */
    calcWaveSpFpts(*s);
  }
  int nS = s->nS, nF = s->nF, nE = s->nE, P = s->P;
  vector<double> wts = qptWeights(P, s->nDims), wS = qptWeights(P, s->nDims - 1);
  double dt = INFINITY;
  for (int e = 0; e < nE; e++) {
    double vol = 0;
    for (int sp = 0; sp < nS; sp++) vol += s->detJ_spts[(size_t)sp * nE + e] * wts[sp];
    double iw = 0;
    for (int f = 0; f < nF; f++) iw += s->waveSp[(size_t)e * nF + f] * wS[f % s->nFptFace] * s->dA_fpts[(size_t)f * nE + e];
    s->eleDt[e] = s->p.CFL * cflLimit(P) * 2 * vol / iw;
    dt = min(dt, s->eleDt[e]);
  }
  s->dt = dt;
}

/* solver::update (src/solver.cpp:212-250) preceded by the main loop's iter++ */
void orc_update(orc_solver *s) {
  s->iter++;
  int nRK = s->nRK;
  for (int step = 0; step < nRK - 1; step++) {
    s->rkTime = s->time + s->RKa[step] * s->dt;
    if (step == 0 && s->p.dtType != 0) orc_calc_dt(s);
    if (step == 0) s->U0 = s->U;
    orc_calc_residual(s, step);
    orc_time_step_a(s, step, s->RKa[step + 1]);
  }
  s->rkTime = s->time + s->RKa[nRK - 1] * s->dt;
  orc_calc_residual(s, nRK - 1);
  if (s->p.timeType < 5) {
    if (nRK > 1) s->U = s->U0;
    else if (s->p.dtType != 0) orc_calc_dt(s);
    for (int step = 0; step < nRK; step++) orc_time_step_b(s, step);
  } else {
    orc_time_step_a(s, nRK - 1, s->RKa[nRK]);
  }
  s->time += s->dt;
}

/* ele::getNormResidual (src/ele.cpp:1882-1903) summed over elements */
void orc_residual_norm(const orc_solver *s, int normType, double *out) {
  int nS = s->nS, nE = s->nE, nV = s->nV;
  vector<double> w = qptWeights(s->P, s->nDims);
  for (int k = 0; k < nV; k++) out[k] = 0;
  for (int e = 0; e < nE; e++) {
    vector<double> r(nV, 0.0);
    for (int sp = 0; sp < nS; sp++)
      for (int k = 0; k < nV; k++) {
        double dv = s->divF[0][((size_t)sp * nE + e) * nV + k], dj = s->detJ_spts[(size_t)sp * nE + e];
        if (normType == 1) r[k] += std::abs(dv) * w[sp];
        else if (normType == 2) r[k] += dv * dv / dj * w[sp];
        else r[k] = max(std::abs(dv) / dj, r[k]);
      }
    for (int k = 0; k < nV; k++) out[k] = normType == 3 ? max(out[k], r[k]) : out[k] + r[k];
  }
}

/* Gauss-Legendre nodes and weights of n points, ascending, by Newton's
 * method on the Legendre polynomial (the reference tabulates them to 16
 * digits, src/points.cpp:169-248, :376-470; the values agree to rounding). */
static void gaussLegendre(int n, vector<double> &x, vector<double> &w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    double z = -cos(PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0; }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (std::abs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; k++) {
      double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    if (n == 1) { p1 = z; p0 = 1.0; }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

/* viscousStressTensor (src/flux.cpp:228-358) */
static void stressTensor(const orc_params &p, int d, const double *U, const double *g /*[d][nV]*/, double tau[3][3]) {
  int nV = d + 2;
  auto G = [&](int a, int b) { return g[a * nV + b]; };
  double rho = U[0], u = U[1] / rho, v = U[2] / rho;
  double e = U[d + 1] / rho - 0.5 * (u * u + v * v), w = 0.;
  if (d == 3) { w = U[3] / rho; e -= 0.5 * (w * w); }
  double dRho_dx = G(0, 0), dRhoU_dx = G(0, 1), dRhoV_dx = G(0, 2);
  double dRho_dy = G(1, 0), dRhoU_dy = G(1, 1), dRhoV_dy = G(1, 2);
  double dRho_dz = 0, dRhoU_dz = 0, dRhoW_dz = 0;
  if (d == 3) { dRho_dz = G(2, 0); dRhoU_dz = G(2, 1); dRhoW_dz = G(2, 3); }
  double mu = p.mu_inf;
  if (!p.fixVis) {
    double rt = (p.gamma - 1.0) * e / p.rt_inf;
    mu *= pow(rt, 1.5) * (1. + p.c_sth) / (rt + p.c_sth);
  }
  double du_dx = (dRhoU_dx - dRho_dx * u) / rho, du_dy = (dRhoU_dy - dRho_dy * u) / rho;
  double dv_dx = (dRhoV_dx - dRho_dx * v) / rho, dv_dy = (dRhoV_dy - dRho_dy * v) / rho;
  double du_dz = 0, dw_dz = 0;
  if (d == 3) { du_dz = (dRhoU_dz - dRho_dz * u) / rho; dw_dz = (dRhoW_dz - dRho_dz * w) / rho; }
  double diag = (du_dx + dv_dy + dw_dz) / 3.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) tau[i][j] = 0;
  tau[0][0] = 2.0 * mu * (du_dx - diag);
  tau[1][1] = 2.0 * mu * (dv_dy - diag);
  tau[0][1] = tau[1][0] = mu * (du_dy + dv_dx);
  if (d == 3) {
    tau[0][2] = tau[2][0] = mu * (du_dz + dv_dx);
    tau[1][2] = tau[2][1] = mu * (du_dz + dv_dy);
    tau[2][2] = 2.0 * mu * (dw_dz - diag);
  }
}

/* solver::computeWallForce (src/solver.cpp:1367-1378) summing
 * boundFace::computeWallForce (src/boundFace.cpp:330-378) over the slip,
 * adiabatic and isothermal wall faces, from the face data of the last
 * orc_calc_residual: force[0..2] pressure, force[3..5] viscous stress. */
void orc_wall_force(const orc_solver *s, double *force) {
  const orc_params &p = s->p;
  int d = s->nDims, nV = s->nV, nE = s->nE, nF = s->nF, P = s->P;
  vector<double> w = qptWeights1D(P);
  for (int j = 0; j < 6; j++) force[j] = 0;
  for (const OFace &F : s->faces) {
    if (F.eR >= 0 || !(F.bc == BC_SLIP || F.bc == BC_ADI_NOSLIP || F.bc == BC_ISO_NOSLIP)) continue;
    double ff[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < s->nFptFace; i++) {
      double weight = d == 2 ? w[i] : w[i % (P + 1)] * w[i / (P + 1)];
      int fl = F.fptL[i];
      const double *U = &s->U_fpts[((size_t)fl * nE + F.eL) * nV];
      const double *n = &s->norm_fpts[((size_t)fl * nE + F.eL) * d];
      double dA = s->dA_fpts[(size_t)fl * nE + F.eL];
      double rho = U[0], vMagSq = 0;
      for (int dim = 0; dim < d; dim++) vMagSq += U[dim + 1] * U[dim + 1] / (rho * rho);
      double pr = (p.gamma - 1) * (U[d + 1] - 0.5 * rho * vMagSq);
      for (int dim = 0; dim < d; dim++) ff[dim] += pr * n[dim] * dA * weight;
      if (p.viscous) {
        double g[3 * 5], tau[3][3];
        for (int dim = 0; dim < d; dim++)
          for (int k = 0; k < nV; k++) g[dim * nV + k] = s->dU_fpts[s->i4(dim, fl, nF, F.eL, k)];
        stressTensor(p, d, U, g, tau);
        for (int a = 0; a < d; a++)
          for (int b = 0; b < d; b++) ff[3 + a] -= tau[a][b] * n[b] * dA * weight;
      }
    }
    for (int j = 0; j < 6; j++) force[j] += ff[j];
  }
}

/* solver::computeMassFlux (src/solver.cpp:1380-1391) summing
 * boundFace::computeMassFlux (src/boundFace.cpp:380-418) over the
 * characteristic / supersonic / subsonic in- and outflow faces, from the
 * faces' common fluxes of the last orc_calc_residual. */
void orc_mass_flux(const orc_solver *s, int errorNorm, double *flux) {
  int d = s->nDims, nV = s->nV, nE = s->nE, P = s->P;
  vector<double> w = qptWeights1D(P);
  for (int k = 0; k < nV; k++) flux[k] = 0;
  for (const OFace &F : s->faces) {
    if (F.eR >= 0 || !(F.bc == BC_CHAR || F.bc == BC_SUP_IN || F.bc == BC_SUP_OUT || F.bc == BC_SUB_IN ||
                       F.bc == BC_SUB_OUT))
      continue;
    vector<double> ff(nV, 0.0);
    for (int i = 0; i < s->nFptFace; i++) {
      double weight = d == 2 ? w[i] : w[i % (P + 1)] * w[i / (P + 1)];
      int fl = F.fptL[i];
      double dA = s->dA_fpts[(size_t)fl * nE + F.eL];
      double nx = s->norm_fpts[((size_t)fl * nE + F.eL) * d];
      const double *Fn = &F.Fn[(size_t)i * nV];
      for (int k = 0; k < nV; k++) {
        if (errorNorm == 0) ff[k] += Fn[k] * dA * weight;
        else if (errorNorm == 1) ff[k] += std::abs(Fn[k]) * dA * weight * nx;
        else ff[k] += (Fn[k] * dA) * (Fn[k] * dA) * weight * nx;
      }
    }
    for (int k = 0; k < nV; k++) flux[k] += ff[k];
  }
}

/* calcError (src/funcs.cpp:1875-1979), testCase 1: the state minus the
 * analytic solution at x (icType 0 entropy error / Gaussian, 1 isentropic
 * vortex of strength eps / sine wave, 2 cosine product for advection);
 * box = xmin, xmax, ymin, ymax of the periodic domain. */
static void calcError(const orc_params &p, int d, int icType, double eps, const double *box, double time,
                      const double *U, const double *x, int errorNorm, double *err) {
  int nV = p.equation == 0 ? 1 : d + 2;
  double xmin = box[0], xmax = box[1], ymin = box[2], ymax = box[3];
  for (int k = 0; k < nV; k++) err[k] = 0;
  if (p.equation == 1) {
    double gamma = p.gamma;
    if (icType == 0) {
      double pfs = p.pBound, rhofsg = pow(p.rhoBound, gamma);
      double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = d == 2 ? 0 : U[3] / rho;
      double pr = (gamma - 1.) * (U[d + 1] - .5 * rho * (u * u + v * v + w * w));
      err[0] = pr * rhofsg / (pow(rho, gamma) * pfs) - 1.;
    } else {
      double X = fmod((x[0] - time), (xmax - xmin)), Y = fmod((x[1] - time), (ymax - ymin));
      if (X > xmax) X -= (xmax - xmin);
      if (Y > ymax) Y -= (ymax - ymin);
      if (X < xmin) X += (xmax - xmin);
      if (Y < ymin) Y += (ymax - ymin);
      double f = 1.0 - (X * X + Y * Y);
      double rho = max(pow(1. - eps * eps * (gamma - 1.) / (8. * gamma * PI * PI) * exp(f), 1.0 / (gamma - 1.0)), 1e-10);
      double vx = 1. - eps * Y / (2. * PI) * exp(f / 2.), vy = 1. + eps * X / (2. * PI) * exp(f / 2.);
      double pr = pow(rho, gamma);
      err[0] = rho;
      err[1] = rho * vx;
      err[2] = rho * vy;
      if (d == 3) err[3] = 0.;
      err[d + 1] = pr / (gamma - 1) + (0.5 * rho * (vx * vx + vy * vy));
      for (int k = 0; k < nV; k++) err[k] = U[k] - err[k];
    }
  } else {
    double X = std::abs(fmod((x[0] - time), (xmax - xmin))), Y = std::abs(fmod((x[1] - time), (ymax - ymin)));
    if (X > (xmax - xmin) / 2) X -= (xmax - xmin);
    if (Y > (ymax - ymin) / 2) Y -= (ymax - ymin);
    if (icType == 0) err[0] = exp(-(X * X + Y * Y));
    else if (icType == 1) err[0] = 1 + sin(2. * PI * (x[0] + 5. - time) / 10.);
    else err[0] = cos(2 * PI * x[0] / 6.) * cos(2 * PI * x[1] / 6.) * cos(2 * PI * (d == 3 ? x[2] : 0.0) / 6.);
    err[0] = U[0] - err[0];
  }
  if (errorNorm == 1)
    for (int k = 0; k < nV; k++) err[k] = std::abs(err[k]);
  else if (errorNorm == 2)
    for (int k = 0; k < nV; k++) err[k] *= err[k];
}

/* solver::integrateError (src/solver.cpp:1507-1574), testCase 1: errorNorm
 * 0 integrates state minus solution and the state at the solution points and
 * returns |difference|; 1 / 2 interpolate the state and detJ to the
 * Gauss points of quadOrder (oper::setupInterpolateSptsQpts,
 * src/operators.cpp:305-316) and integrate |error| / error^2 (2: square
 * root of the sum).  eps is the vortex strength (5 for icType 1). */
void orc_integrate_error(const orc_solver *s, int icType, double eps, int errorNorm, int quadOrder,
                         const double *box, double *out) {
  const orc_params &p = s->p;
  int d = s->nDims, nV = s->nV, nE = s->nE, nS = s->nS, nN = s->nNodes, P = s->P;
  for (int k = 0; k < nV; k++) out[k] = 0;
  vector<double> err(nV);
  if (errorNorm == 0) {
    vector<double> wts = qptWeights(P, d), intU(nV, 0.0);
    for (int e = 0; e < nE; e++)
      for (int sp = 0; sp < nS; sp++) {
        const double *U = &s->U[((size_t)sp * nE + e) * nV];
        calcError(p, d, icType, eps, box, s->time, U, &s->pos_spts[((size_t)sp * nE + e) * d], 0, err.data());
        double wd = s->detJ_spts[(size_t)sp * nE + e];
        for (int k = 0; k < nV; k++) {
          out[k] += err[k] * wts[sp] * wd;
          intU[k] += U[k] * wts[sp] * wd;
        }
      }
    for (int k = 0; k < nV; k++) out[k] = std::abs(out[k] - intU[k]);
    return;
  }
  int nq1 = quadOrder + 1, nQ = d == 2 ? nq1 * nq1 : nq1 * nq1 * nq1;
  vector<double> xq, wq1;
  gaussLegendre(nq1, xq, wq1);
  vector<double> wq(nQ);
  vector<double> loc((size_t)nQ * 3, 0.0);
  for (int q = 0; q < nQ; q++) {
    int a = q % nq1, b = (q / nq1) % nq1, c = q / (nq1 * nq1);
    loc[3 * q] = xq[a];
    loc[3 * q + 1] = xq[b];
    if (d == 3) loc[3 * q + 2] = xq[c];
    wq[q] = d == 2 ? wq1[b] * wq1[a] : wq1[c] * wq1[b] * wq1[a]; /* getQptWeights ordering */
  }
  /* opp_spts_to_qpts (setupInterpolateSptsIpts, src/operators.cpp:259-302) */
  vector<double> sp = gaussPts(P), A((size_t)nQ * nS);
  for (int q = 0; q < nQ; q++)
    for (int t = 0; t < nS; t++) {
      int i = t % (P + 1), j = (t / (P + 1)) % (P + 1), k = t / ((P + 1) * (P + 1));
      double v = Lagrange(sp, loc[3 * q], i) * Lagrange(sp, loc[3 * q + 1], j);
      if (d == 3) v *= Lagrange(sp, loc[3 * q + 2], k);
      A[(size_t)q * nS + t] = v;
    }
  vector<double> Uq((size_t)nQ * nE * nV), dq((size_t)nQ * nE), sh(nN), tmp(nN * 3);
  dgemm(nQ, nE * nV, nS, 1.0, A.data(), s->U.data(), 0.0, Uq.data());
  dgemm(nQ, nE, nS, 1.0, A.data(), s->detJ_spts.data(), 0.0, dq.data());
  for (int e = 0; e < nE; e++)
    for (int q = 0; q < nQ; q++) {
      if (d == 2) shapeQuad(loc[3 * q], loc[3 * q + 1], nN, sh.data(), nullptr);
      else shapeHex8(loc[3 * q], loc[3 * q + 1], loc[3 * q + 2], sh.data(), nullptr);
      double x[3] = {0, 0, 0};
      for (int n = 0; n < nN; n++)
        for (int dim = 0; dim < d; dim++) x[dim] += sh[n] * s->nodes[((size_t)n * nE + e) * d + dim];
      calcError(p, d, icType, eps, box, s->time, &Uq[((size_t)q * nE + e) * nV], x, errorNorm, err.data());
      for (int k = 0; k < nV; k++) out[k] += err[k] * wq[q] * dq[(size_t)q * nE + e];
    }
  if (errorNorm == 2)
    for (int k = 0; k < nV; k++) out[k] = std::sqrt(std::abs(out[k]));
}

}  // extern "C"
