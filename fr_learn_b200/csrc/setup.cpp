// setup.cpp -- host set-up of operators, metrics and connectivity.
//
// The FR operators of the reference are Kronecker products of 1D Lagrange
// data (oper::setupOperators, src/operators.cpp:78-111, :660-805, :891-914,
// :1544-1619): at Gauss solution points every factor along a face-tangential
// direction is exactly 0 or 1, so each dense entry equals one 1D value.  The
// kernels apply the 1D tables directly (sum factorisation); the dense matrices
// are rebuilt here only so they can be compared with the reference's.
#include "setup.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <unordered_map>

namespace frg {
namespace {

// Gauss-Legendre nodes and weights exactly as the reference tabulates them
// (src/points.cpp:169-196 nodes, :347-400 weights): 15 / 16 decimals, with the
// reference's asymmetric last digits kept so node locations agree bitwise.
const double kGaussPts[MAXP + 1][MAXP + 1] = {
    {0.0},
    {-0.577350269189626, 0.577350269189626},
    {-0.774596669241483, 0.000000000000000, 0.774596669241483},
    {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
    {-0.906179845938664, -0.538469310105683, 0.000000000000000, 0.538469310105683, 0.906179845938664},
    {-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197, 0.661209386466265,
     0.932469514203152}};
const double kGaussW[MAXP + 1][MAXP + 1] = {
    {2.0},
    {1.0, 1.0},
    {0.5555555555555556, 0.8888888888888888, 0.5555555555555556},
    {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538},
    {0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665, 0.2369268850561891},
    {0.1713244923791704, 0.3607615730481386, 0.4679139345726910, 0.4679139345726910, 0.3607615730481386,
     0.1713244923791704}};

// Lagrange basis `m` on nodes x[0..n) at y, as a running product (the
// reference's form, src/polynomials.cpp:9-19).
double lagr(const double *x, int n, double y, int m) {
  double v = 1.0;
  for (int i = 0; i < n; i++)
    if (i != m) v = v * ((y - x[i]) / (x[m] - x[i]));
  return v;
}
// Its derivative: sum over dropped factors (src/polynomials.cpp:21-45).
double dlagr(const double *x, int n, double y, int m) {
  double d = 0.0;
  for (int i = 0; i < n; i++) {
    if (i == m) continue;
    double num = 1.0, den = 1.0;
    for (int j = 0; j < n; j++) {
      if (j != m && j != i) num = num * (y - x[j]);
      if (j != m) den = den * (x[m] - x[j]);
    }
    d = d + (num / den);
  }
  return d;
}
// Legendre polynomial by the three-term recurrence and its derivative from
// (x^2-1) P_n' = n (x P_n - P_{n-1}), with the endpoint values n(n+1)/2 *
// (+-1)^(n-1) (src/polynomials.cpp:83-116).
double legendre(double r, int n) {
  if (n < 0) return 0.;
  if (n == 0) return 1.0;
  if (n == 1) return r;
  return ((2 * n - 1) * r * legendre(r, n - 1) - (n - 1) * legendre(r, n - 2)) / n;
}
double dlegendre(double r, int n) {
  if (n == 0) return 0;
  if (r > -1.0 && r < 1.0) return n * ((r * legendre(r, n)) - legendre(r, n - 1)) / (r * r - 1.0);
  if (r == -1.0) return pow(-1.0, n - 1.0) * 0.5 * n * (n + 1.0);
  if (r == 1.0) return 0.5 * n * (n + 1.0);
  return 0.;
}
int fact(int n) { return n <= 1 ? 1 : n * fact(n - 1); }
// VCJH parameter eta (src/polynomials.cpp:392-428): DG 0, SD P/(P+1),
// HU (P+1)/P, C+ from the tabulated c.
double vcjh_eta(int scheme, int P) {
  switch (scheme) {
    case 0: return 0.0;
    case 1: return (1.0 * P) / (1.0 * (P + 1));
    case 2: return (1.0 * (P + 1)) / (1.0 * P);
    default: {
      const double c[6] = {0, 0, 0.206, 3.80e-3, 4.67e-5, 4.28e-7};
      double ap = 1. / pow(2.0, P) * fact(2 * P) / (fact(P) * fact(P));
      return c[P] * (2 * P + 1) / 2 * (fact(P) * ap) * (fact(P) * ap);
    }
  }
}
// d/dxi of the left (side 0) / right (side 1) VCJH correction function,
// g = (-1)^P/2 [L_P - (eta L_{P-1} + L_{P+1})/(1+eta)] and its mirror
// (src/polynomials.cpp:447-474).
double dvcjh(double r, int side, int P, double eta) {
  double lo = P == 0 ? dlegendre(r, P + 1) : (eta * dlegendre(r, P - 1)) + dlegendre(r, P + 1);
  if (side == 0) return 0.5 * pow(-1.0, P) * (dlegendre(r, P) - (lo / (1.0 + eta)));
  return 0.5 * (dlegendre(r, P) + (lo / (1.0 + eta)));
}

// Flux-point face bookkeeping shared by the dense builder and connectivity.
// 2D faces: 0 eta=-1, 1 xi=+1, 2 eta=+1, 3 xi=-1; face-local index k runs
// counter-clockwise (getLocFpts, src/points.cpp:72-87).
// 3D faces: 0 z-, 1 z+, 2 x-, 3 x+, 4 y-, 5 y+, local index a + b*(P+1)
// (getLocFpts, src/points.cpp:88-126).
struct FptLine {
  int dir, side;          // normal direction, 0 = -1 face, 1 = +1 face
  int idx[3];             // 1D indices of the tangential coordinates (dir slot unused)
};
FptLine fpt_line(int nDims, int P, int f) {
  FptLine L{};
  if (nDims == 2) {
    int face = f / (P + 1), k = f % (P + 1);
    switch (face) {
      case 0: L.dir = 1; L.side = 0; L.idx[0] = k; break;
      case 1: L.dir = 0; L.side = 1; L.idx[1] = k; break;
      case 2: L.dir = 1; L.side = 1; L.idx[0] = P - k; break;
      default: L.dir = 0; L.side = 0; L.idx[1] = P - k; break;
    }
  } else {
    int n1 = P + 1, face = f / (n1 * n1), k = f % (n1 * n1), a = k % n1, b = k / n1;
    switch (face) {
      case 0: L.dir = 2; L.side = 0; L.idx[0] = a; L.idx[1] = b; break;
      case 1: L.dir = 2; L.side = 1; L.idx[0] = P - a; L.idx[1] = b; break;
      case 2: L.dir = 0; L.side = 0; L.idx[1] = a; L.idx[2] = b; break;
      case 3: L.dir = 0; L.side = 1; L.idx[1] = P - a; L.idx[2] = b; break;
      case 4: L.dir = 1; L.side = 0; L.idx[0] = P - a; L.idx[2] = b; break;
      default: L.dir = 1; L.side = 1; L.idx[0] = a; L.idx[2] = b; break;
    }
  }
  return L;
}
int spt_index(int nDims, int P, const int *ijk) {
  int n1 = P + 1;
  return nDims == 2 ? ijk[0] + n1 * ijk[1] : ijk[0] + n1 * (ijk[1] + n1 * ijk[2]);
}

// Shape functions of the mesh elements.  Quads: Lagrange on equidistant
// nodes, node order corners / edges / centre level by level (the recursion of
// src/funcs.cpp:126-176); hexes: 8 corners (src/funcs.cpp:183-230).
struct Shape {
  int nN = 0, nSide = 0;
  std::vector<std::array<int, 3>> ij;  // 1D node index per direction of each node
  std::vector<double> xl;
};
bool make_shape(int nDims, int nN, Shape &s) {
  s.nN = nN;
  if (nDims == 3) {
    if (nN != 8) return false;
    s.nSide = 2;
    s.ij = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  } else {
    int n = (int)lround(sqrt((double)nN));
    if (n * n != nN || n < 2) return false;
    s.nSide = n;
    s.ij.assign(nN, {0, 0, 0});
    int c = 0;
    for (int lev = 0; lev < n / 2; lev++) {
      int i2 = n - 1 - lev;
      s.ij[c++] = {lev, lev, 0};
      s.ij[c++] = {i2, lev, 0};
      s.ij[c++] = {i2, i2, 0};
      s.ij[c++] = {lev, i2, 0};
      int m = n - 2 * (lev + 1);
      for (int j = 0; j < m; j++) s.ij[c + j] = {lev + 1 + j, lev, 0};
      for (int j = 0; j < m; j++) s.ij[c + m + j] = {i2, lev + 1 + j, 0};
      for (int j = 0; j < m; j++) s.ij[c + 2 * m + j] = {i2 - 1 - j, i2, 0};
      for (int j = 0; j < m; j++) s.ij[c + 3 * m + j] = {lev, i2 - 1 - j, 0};
      c += 4 * m;
    }
    if (n % 2) s.ij[nN - 1] = {n / 2, n / 2, 0};
  }
  s.xl.resize(s.nSide);
  double dxi = 2. / (s.nSide - 1);
  for (int i = 0; i < s.nSide; i++) s.xl[i] = -1. + i * dxi;
  return true;
}
// d(shape)/d(xi_dim) of every node at reference point loc.
void dshape(const Shape &s, int nDims, const double *loc, int dim, double *out) {
  for (int n = 0; n < s.nN; n++) {
    double v = 1.0;
    for (int d = 0; d < nDims; d++) {
      double f = d == dim ? dlagr(s.xl.data(), s.nSide, loc[d], s.ij[n][d])
                          : lagr(s.xl.data(), s.nSide, loc[d], s.ij[n][d]);
      v = d == 0 ? f : v * f;
    }
    out[n] = v;
  }
}
void shape(const Shape &s, int nDims, const double *loc, double *out) {
  for (int n = 0; n < s.nN; n++) {
    double v = 1.0;
    for (int d = 0; d < nDims; d++) {
      double f = lagr(s.xl.data(), s.nSide, loc[d], s.ij[n][d]);
      v = d == 0 ? f : v * f;
    }
    out[n] = v;
  }
}

// Reference coordinates of solution / flux points (getLocSpts/getLocFpts).
void loc_spt(int nDims, const Ops1D &o, int s, double *x) {
  int n1 = o.P + 1;
  x[0] = o.pts[s % n1];
  x[1] = o.pts[(s / n1) % n1];
  if (nDims == 3) x[2] = o.pts[s / (n1 * n1)];
}
void loc_fpt(int nDims, const Ops1D &o, int f, double *x) {
  FptLine L = fpt_line(nDims, o.P, f);
  for (int d = 0; d < nDims; d++) x[d] = d == L.dir ? (L.side ? 1.0 : -1.0) : o.pts[L.idx[d]];
}

struct KeyHash {
  size_t operator()(const std::array<int, 4> &k) const {
    size_t h = 1469598103934665603ull;
    for (int v : k) h = (h ^ (size_t)(unsigned)v) * 1099511628211ull;
    return h;
  }
};

}  // namespace

Ops1D build_ops1d(int P, int vcjh) {
  Ops1D o;
  o.P = P;
  int n = P + 1;
  for (int i = 0; i < n; i++) { o.pts[i] = kGaussPts[P][i]; o.w[i] = kGaussW[P][i]; }
  for (int j = 0; j < n; j++) {
    o.lag[0][j] = lagr(o.pts, n, -1.0, j);
    o.lag[1][j] = lagr(o.pts, n, 1.0, j);
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) o.dlag[i][j] = dlagr(o.pts, n, o.pts[i], j);
  double eta = vcjh_eta(vcjh, P);
  for (int i = 0; i < n; i++) {
    o.gL[i] = dvcjh(o.pts[i], 0, P, eta);
    o.gR[i] = dvcjh(o.pts[i], 1, P, eta);
  }
  return o;
}

void dense_operator(int nDims, const Ops1D &o, int which, int dim, std::vector<double> &out) {
  int P = o.P, n1 = P + 1;
  int nS = nDims == 2 ? n1 * n1 : n1 * n1 * n1, nF = nDims == 2 ? 4 * n1 : 6 * n1 * n1;
  auto sidx = [&](int s, int d) { return d == 0 ? s % n1 : d == 1 ? (s / n1) % n1 : s / (n1 * n1); };
  if (which == 0 || which == 2) {  // spts_to_fpts, extrapolateFn[dim]
    out.assign((size_t)nF * nS, 0.0);
    for (int f = 0; f < nF; f++) {
      FptLine L = fpt_line(nDims, P, f);
      double t = which == 0 ? 1.0 : (dim == L.dir ? (L.side ? 1.0 : -1.0) : 0.0);
      for (int j = 0; j < n1; j++) {
        int ijk[3] = {L.idx[0], L.idx[1], L.idx[2]};
        ijk[L.dir] = j;
        out[(size_t)f * nS + spt_index(nDims, P, ijk)] = o.lag[L.side][j] * t;
      }
    }
  } else if (which == 1) {  // grad_spts[dim]
    out.assign((size_t)nS * nS, 0.0);
    for (int s = 0; s < nS; s++)
      for (int j = 0; j < n1; j++) {
        int ijk[3] = {sidx(s, 0), sidx(s, 1), nDims == 3 ? sidx(s, 2) : 0};
        int i = ijk[dim];
        ijk[dim] = j;
        out[(size_t)s * nS + spt_index(nDims, P, ijk)] = o.dlag[i][j];
      }
  } else {  // correction, correctU[dim]
    out.assign((size_t)nS * nF, 0.0);
    for (int f = 0; f < nF; f++) {
      FptLine L = fpt_line(nDims, P, f);
      double t = which == 3 ? 1.0 : (dim == L.dir ? (L.side ? 1.0 : -1.0) : 0.0);
      for (int j = 0; j < n1; j++) {
        int ijk[3] = {L.idx[0], L.idx[1], L.idx[2]};
        ijk[L.dir] = j;
        double g = L.side ? o.gR[j] : -o.gL[j];
        out[(size_t)spt_index(nDims, P, ijk) * nF + f] = g * t;
      }
    }
  }
}

bool metric_tables(int d, int P, int vcjh, int nN, MetricTables &t, std::string &err) {
  const int n1 = P + 1, nS = d == 2 ? n1 * n1 : n1 * n1 * n1, nFF = d == 2 ? n1 : n1 * n1, nF = 2 * d * nFF;
  Shape sh;
  if (!make_shape(d, nN, sh)) {
    err = d == 3 ? "3D elements must be 8-node hexahedra" : "quad node count must be a square >= 4";
    return false;
  }
  Ops1D o = build_ops1d(P, vcjh);
  t.nDims = d; t.nS = nS; t.nF = nF; t.nN = nN;
  t.shS.assign((size_t)nS * nN, 0.0);
  t.dS.assign((size_t)d * nS * nN, 0.0);
  t.dF.assign((size_t)d * nF * nN, 0.0);
  for (int s = 0; s < nS; s++) {
    double x[3];
    loc_spt(d, o, s, x);
    shape(sh, d, x, &t.shS[(size_t)s * nN]);
    for (int dim = 0; dim < d; dim++) dshape(sh, d, x, dim, &t.dS[((size_t)dim * nS + s) * nN]);
  }
  t.fdir.resize(nF);
  t.fsgn.resize(nF);
  for (int f = 0; f < nF; f++) {
    double x[3];
    loc_fpt(d, o, f, x);
    for (int dim = 0; dim < d; dim++) dshape(sh, d, x, dim, &t.dF[((size_t)dim * nF + f) * nN]);
    FptLine L = fpt_line(d, P, f);
    t.fdir[f] = L.dir;
    t.fsgn[f] = L.side ? 1 : -1;
  }
  t.wv.resize(nS);
  t.ws.resize(nF);
  for (int s = 0; s < nS; s++) {
    int i = s % n1, j = (s / n1) % n1, k = s / (n1 * n1);
    // getQptWeights order: products w_slow * w_mid (* w_fast)
    t.wv[s] = d == 2 ? o.w[j] * o.w[i] : o.w[k] * o.w[j] * o.w[i];
  }
  for (int f = 0; f < nF; f++) {
    int k = f % nFF, a = k % n1, b = k / n1;
    t.ws[f] = d == 2 ? o.w[k] : o.w[b] * o.w[a];
  }
  return true;
}

bool plot_tables(int d, int P, int nN, std::vector<double> &shapeP, std::vector<double> &interpP, std::string &err) {
  Shape sh;
  if (!make_shape(d, nN, sh)) {
    err = d == 3 ? "3D elements must be 8-node hexahedra" : "quad node count must be a square >= 4";
    return false;
  }
  const Ops1D o = build_ops1d(P, 0);
  const int n1 = P + 1, n3 = P + 3, nS = d == 2 ? n1 * n1 : n1 * n1 * n1, nP = d == 2 ? n3 * n3 : n3 * n3 * n3;
  std::vector<double> x1(n3);
  x1[0] = -1.0;
  for (int i = 0; i < n1; i++) x1[i + 1] = o.pts[i];
  x1[n3 - 1] = 1.0;
  shapeP.assign((size_t)nP * nN, 0.0);
  interpP.assign((size_t)nP * nS, 0.0);
  for (int q = 0; q < nP; q++) {
    const int i = q % n3, j = (q / n3) % n3, k = q / (n3 * n3);
    const double loc[3] = {x1[i], x1[j], d == 3 ? x1[k] : 0.0};
    shape(sh, d, loc, &shapeP[(size_t)q * nN]);
    for (int s = 0; s < nS; s++) {
      const int is = s % n1, js = (s / n1) % n1, ks = s / (n1 * n1);
      double v = lagr(o.pts, n1, loc[0], is) * lagr(o.pts, n1, loc[1], js);
      if (d == 3) v = v * lagr(o.pts, n1, loc[2], ks);
      interpP[(size_t)q * nS + s] = v;
    }
  }
  return true;
}

// Gauss-Legendre nodes (ascending) and weights of n points by Newton's
// method on the Legendre polynomial; the reference tabulates them to 16
// digits (src/points.cpp:169-248, :376-470), which agree to rounding.
static void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  const double pi = 3.141592653589793;
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; i++) {
    double z = -std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; k++) {
      const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

bool quad_tables(int d, int P, int nN, int quadOrder, std::vector<double> &shapeQ, std::vector<double> &interpQ,
                 std::vector<double> &wq, std::string &err) {
  Shape sh;
  if (!make_shape(d, nN, sh)) {
    err = d == 3 ? "3D elements must be 8-node hexahedra" : "quad node count must be a square >= 4";
    return false;
  }
  if (quadOrder < 0 || quadOrder > 20) {
    err = "quadOrder out of range (0..20)";
    return false;
  }
  const Ops1D o = build_ops1d(P, 0);
  const int n1 = P + 1, nq = quadOrder + 1, nS = d == 2 ? n1 * n1 : n1 * n1 * n1;
  const int nQ = d == 2 ? nq * nq : nq * nq * nq;
  std::vector<double> xq, w1;
  gauss_legendre(nq, xq, w1);
  shapeQ.assign((size_t)nQ * nN, 0.0);
  interpQ.assign((size_t)nQ * nS, 0.0);
  wq.assign(nQ, 0.0);
  for (int q = 0; q < nQ; q++) {
    const int i = q % nq, j = (q / nq) % nq, k = q / (nq * nq);
    const double loc[3] = {xq[i], xq[j], d == 3 ? xq[k] : 0.0};
    // getQptWeights: the slowest index's weight first
    wq[q] = d == 2 ? w1[j] * w1[i] : w1[k] * w1[j] * w1[i];
    shape(sh, d, loc, &shapeQ[(size_t)q * nN]);
    for (int s = 0; s < nS; s++) {
      const int is = s % n1, js = (s / n1) % n1, ks = s / (n1 * n1);
      double v = lagr(o.pts, n1, loc[0], is) * lagr(o.pts, n1, loc[1], js);
      if (d == 3) v = v * lagr(o.pts, n1, loc[2], ks);
      interpQ[(size_t)q * nS + s] = v;
    }
  }
  return true;
}

bool spt_shape_table(int d, int P, int nN, std::vector<double> &shapeS, std::string &err) {
  Shape sh;
  if (!make_shape(d, nN, sh)) {
    err = d == 3 ? "3D elements must be 8-node hexahedra" : "quad node count must be a square >= 4";
    return false;
  }
  const Ops1D o = build_ops1d(P, 0);
  const int nS = d == 2 ? (P + 1) * (P + 1) : (P + 1) * (P + 1) * (P + 1);
  shapeS.assign((size_t)nS * nN, 0.0);
  for (int s = 0; s < nS; s++) {
    double loc[3] = {0, 0, 0};
    loc_spt(d, o, s, loc);
    shape(sh, d, loc, &shapeS[(size_t)s * nN]);
  }
  return true;
}

void order_interp(int d, int Pf, int Pt, std::vector<double> &out) {
  const Ops1D of = build_ops1d(Pf, 0), ot = build_ops1d(Pt, 0);
  const int nf = Pf + 1, nt = Pt + 1, nSf = d == 2 ? nf * nf : nf * nf * nf, nSt = d == 2 ? nt * nt : nt * nt * nt;
  out.assign((size_t)nSt * nSf, 0.0);
  for (int t = 0; t < nSt; t++) {
    const double x = ot.pts[t % nt], y = ot.pts[(t / nt) % nt], z = d == 3 ? ot.pts[t / (nt * nt)] : 0.0;
    for (int r = 0; r < nSf; r++) {
      double v = lagr(of.pts, nf, x, r % nf) * lagr(of.pts, nf, y, (r / nf) % nf);
      if (d == 3) v = v * lagr(of.pts, nf, z, r / (nf * nf));
      out[(size_t)t * nSf + r] = v;
    }
  }
}

frg_status build_geometry(const frg_params &p, const frg_mesh &m, HostGeom &g, std::string &err) {
  const int d = p.nDims, P = p.order, nE = m.nEles, n1 = P + 1;
  g.nDims = d; g.P = P; g.nE = nE;
  g.nS = d == 2 ? n1 * n1 : n1 * n1 * n1;
  g.nFF = d == 2 ? n1 : n1 * n1;
  g.nFaceEle = 2 * d;
  g.nF = g.nFaceEle * g.nFF;
  const int nS = g.nS, nF = g.nF, nN = m.nNodes;
  MetricTables t;
  if (!metric_tables(d, P, p.vcjhScheme, nN, t, err)) return FRG_ERR_ARG;
  const std::vector<double> &shS = t.shS, &dS = t.dS, &dF = t.dF, &wv = t.wv, &ws = t.ws;
  g.pos_spts.assign((size_t)nS * nE * d, 0.0);
  g.JG.assign((size_t)d * d * nS * nE, 0.0);
  g.detJ.assign((size_t)nS * nE, 0.0);
  g.nrmOwn.assign((size_t)d * nF * nE, 0.0);
  g.dA.assign((size_t)nF * nE, 0.0);
  g.vol.assign(nE, 0.0);
  g.dAw.assign((size_t)nF * nE, 0.0);
  auto X = [&](int e, int n, int k) { return m.xv[((size_t)e * nN + n) * d + k]; };
  // jacobian at a point from dshape rows: J[a][k] = d x_k / d xi_a
  auto jac = [&](const double *dsh, int nPt, int pt, int e, double J[3][3]) {
    for (int a = 0; a < d; a++)
      for (int k = 0; k < d; k++) {
        double v = 0.0;
        const double *row = dsh + ((size_t)a * nPt + pt) * nN;
        for (int n = 0; n < nN; n++) v += row[n] * X(e, n, k);
        J[a][k] = v;
      }
  };
  // adjugate (JGinv) and determinant, reference calcTransforms formulas
  // (src/solver.cpp:1247-1282)
  auto adj = [&](double J[3][3], double G[3][3], double &det) {
    if (d == 2) {
      det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
      G[0][0] = J[1][1]; G[0][1] = -J[1][0]; G[1][0] = -J[0][1]; G[1][1] = J[0][0];
    } else {
      double xr = J[0][0], xs = J[1][0], xt = J[2][0], yr = J[0][1], ys = J[1][1], yt = J[2][1];
      double zr = J[0][2], zs = J[1][2], zt = J[2][2];
      det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
      G[0][0] = ys * zt - yt * zs; G[0][1] = xt * zs - xs * zt; G[0][2] = xs * yt - xt * ys;
      G[1][0] = yt * zr - yr * zt; G[1][1] = xr * zt - xt * zr; G[1][2] = xt * yr - xr * yt;
      G[2][0] = yr * zs - ys * zr; G[2][1] = xs * zr - xr * zs; G[2][2] = xr * ys - xs * yr;
    }
  };
  for (int e = 0; e < nE; e++) {
    for (int s = 0; s < nS; s++) {
      for (int k = 0; k < d; k++) {
        double v = 0.0;
        for (int n = 0; n < nN; n++) v += shS[(size_t)s * nN + n] * X(e, n, k);
        g.pos_spts[((size_t)s * nE + e) * d + k] = v;
      }
      double J[3][3], G[3][3], det;
      jac(dS.data(), nS, s, e, J);
      adj(J, G, det);
      if (det < 0) {
        char buf[128];
        snprintf(buf, sizeof buf, "Negative Jacobian at solution points (element %d)", e);
        err = buf;
        return FRG_ERR_NEG_JAC;
      }
      g.detJ[(size_t)s * nE + e] = det;
      for (int a = 0; a < d; a++)
        for (int b = 0; b < d; b++) g.JG[(((size_t)a * d + b) * nS + s) * nE + e] = G[a][b];
      g.vol[e] += det * wv[s];
    }
    for (int f = 0; f < nF; f++) {
      double J[3][3], G[3][3], det;
      jac(dF.data(), nF, f, e, J);
      adj(J, G, det);
      const double tn = t.fsgn[f];
      double nv[3], mag = 0.0;
      // norm = JGinv^T tNorm: only the face-normal reference direction is non-zero
      for (int k = 0; k < d; k++) {
        nv[k] = 0.0;
        for (int a = 0; a < d; a++) nv[k] += G[a][k] * (a == t.fdir[f] ? tn : 0.0);
      }
      for (int k = 0; k < d; k++) mag += nv[k] * nv[k];
      mag = sqrt(mag);
      if (std::fabs(mag) < 1e-10) {
        mag = 0.;
        for (int k = 0; k < d; k++) nv[k] = 0;
      } else {
        for (int k = 0; k < d; k++) nv[k] /= mag;
      }
      for (int k = 0; k < d; k++) g.nrmOwn[((size_t)k * nF + f) * nE + e] = nv[k];
      g.dA[(size_t)f * nE + e] = mag;
      g.dAw[(size_t)f * nE + e] = ws[f] * mag;
    }
  }
  // ---- connectivity: faces keyed by sorted corner ids (src/geo.cpp:197-246)
  static const int QFV[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
  static const int HFV[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {3, 0, 4, 7}, {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};
  // face vertex lists in the orientation geo::compareOrientation uses (src/geo.cpp:800-880)
  static const int HOR[6][4] = {{0, 1, 2, 3}, {5, 4, 7, 6}, {0, 3, 7, 4}, {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};
  const int nC = d == 2 ? 4 : 8, nFE = g.nFaceEle, nFF = g.nFF;
  std::unordered_map<std::array<int, 4>, long, KeyHash> open;
  open.reserve((size_t)nE * nFE);
  g.nbr.assign((size_t)nF * nE, 0);
  g.nrmC = g.nrmOwn;
  g.faceTable.clear();
  std::vector<char> done((size_t)nE * nFE, 0);
  for (int e = 0; e < nE; e++)
    for (int f = 0; f < nFE; f++) {
      std::array<int, 4> key{-1, -1, -1, -1};
      if (d == 2) { key[0] = m.c2v[e * nC + QFV[f][0]]; key[1] = m.c2v[e * nC + QFV[f][1]]; }
      else for (int i = 0; i < 4; i++) key[i] = m.c2v[e * nC + HFV[f][i]];
      std::sort(key.begin(), key.begin() + (d == 2 ? 2 : 4));
      auto it = open.find(key);
      if (it == open.end()) { open.emplace(key, (long)e * nFE + f); continue; }
      long lf = it->second;
      open.erase(it);
      int eL = (int)(lf / nFE), fL = (int)(lf % nFE), eR = e, fR = f;
      if (eL == eR) { err = "element is its own neighbour (periodic direction with one element)"; return FRG_ERR_MESH; }
      int rel = 1;
      if (d == 3) {
        rel = -1;
        int first = m.c2v[eR * nC + HOR[fR][0]];
        for (int r = 0; r < 4; r++)
          if (m.c2v[eL * nC + HOR[fL][r]] == first) { rel = r; break; }
        if (rel < 0) { err = "internal faces improperly matched"; return FRG_ERR_MESH; }
      }
      // flux-point pairing of intFace::setupRightState (src/intFace.cpp:30-59)
      for (int i = 0; i < nFF; i++) {
        int fr;
        if (d == 2) fr = fR * nFF + nFF - 1 - i;
        else {
          int a = i % n1, b = i / n1, st = nFF * fR, en = nFF * (fR + 1);
          switch (rel) {
            case 0: fr = st + a * n1 + b; break;
            case 1: fr = st + P - a + b * n1; break;
            case 2: fr = en - 1 - (a * n1 + b); break;
            default: fr = en - n1 * (b + 1) + a; break;
          }
        }
        int fl = fL * nFF + i;
        long tR = (long)fr * nE + eR, tL = (long)fl * nE + eL;
        if (tR >= (1L << 30) || tL >= (1L << 30)) { err = "mesh too large for 30-bit trace index"; return FRG_ERR_ARG; }
        g.nbr[(size_t)fl * nE + eL] = (int)(tR << 1);
        g.nbr[(size_t)fr * nE + eR] = (int)((tL << 1) | 1);
        for (int k = 0; k < d; k++)
          g.nrmC[((size_t)k * nF + fr) * nE + eR] = g.nrmOwn[((size_t)k * nF + fl) * nE + eL];
      }
      done[(size_t)eL * nFE + fL] = done[(size_t)eR * nFE + fR] = 1;
      g.faceTable.insert(g.faceTable.end(), {eL, fL, eR, fR, d == 3 ? rel : 1, -1});
      g.nIntFaces++;
    }
  for (int e = 0; e < nE; e++)
    for (int f = 0; f < nFE; f++) {
      if (done[(size_t)e * nFE + f]) continue;
      int b = m.bc ? m.bc[e * nFE + f] : -1;
      if (b < 1) {
        char buf[160];
        snprintf(buf, sizeof buf, "face %d of element %d has no neighbour and no boundary condition", f, e);
        err = buf;
        return FRG_ERR_MESH;
      }
      for (int i = 0; i < nFF; i++) g.nbr[((size_t)f * nFF + i) * nE + e] = -1 - b;
      g.faceTable.insert(g.faceTable.end(), {e, f, -1, -1, -1, b});
      g.nBndFaces++;
    }
  return FRG_OK;
}

frg_status initial_condition(const frg_params &p, const HostGeom &g, int icType, double a0,
                             std::vector<double> &U, std::string &err) {
  const int d = g.nDims, nS = g.nS, nE = g.nE, nV = p.equation == 0 ? 1 : d + 2;
  const double gm = p.gamma, pi = 4.0 * atan(1);
  U.assign((size_t)nS * nE * nV, 0.0);
  for (int s = 0; s < nS; s++)
    for (int e = 0; e < nE; e++) {
      const double *x = &g.pos_spts[((size_t)s * nE + e) * d];
      double *u = &U[((size_t)s * nE + e) * nV];
      if (p.equation == 0) {
        if (icType == 0) {  // Gaussian bump exp(-|x|^2)
          double r2 = x[0] * x[0] + x[1] * x[1] + (d == 3 ? x[2] * x[2] : 0.0);
          u[0] = exp(-r2);
        } else if (icType == 1) {
          u[0] = 1. + sin(2. * pi * (x[0] + 5) / 10.);
        } else { err = "unknown advection icType"; return FRG_ERR_ARG; }
        continue;
      }
      double rho, vx, vy, vz = 0, pr;
      if (icType == 0) {  // uniform freestream
        rho = p.rhoBound; vx = p.uBound; vy = p.vBound; vz = d == 3 ? p.wBound : 0; pr = p.pBound;
        u[0] = rho; u[1] = rho * vx; u[2] = rho * vy;
        if (d == 3) u[3] = rho * vz;
        u[d + 1] = pr / (gm - 1) + (0.5 * rho * (vx * vx + vy * vy + vz * vz));
      } else if (icType == 1 || icType == 11) {  // isentropic vortex, eps 5 (or a0)
        double eps = icType == 1 ? 5.0 : a0;
        double f = 1.0 - (x[0] * x[0] + x[1] * x[1]);
        rho = std::max(pow(1. - eps * eps * (gm - 1.) / (8. * gm * pi * pi) * exp(f), 1.0 / (gm - 1.0) + 1e-5), 1e-3);
        vx = 1. - eps * x[1] / (2. * pi) * exp(f / 2.);
        vy = 1. + eps * x[0] / (2. * pi) * exp(f / 2.);
        pr = pow(rho, gm);
        u[0] = rho; u[1] = rho * vx; u[2] = rho * vy;
        if (d == 3) u[3] = 0.;
        u[d + 1] = pr / (gm - 1) + (0.5 * rho * (vx * vx + vy * vy));
      } else if (icType == 10) {  // Taylor-Green vortex, rho0 = V0 = 1, p0 = 1/(gamma Ma^2)
        double X = x[0], Y = x[1], Z = d == 3 ? x[2] : 0.0;
        double p0 = 1.0 / (gm * a0 * a0);
        rho = 1.0;
        vx = sin(X) * cos(Y) * cos(Z);
        vy = -cos(X) * sin(Y) * cos(Z);
        vz = 0.0;
        pr = p0 + (rho / 16.0) * (cos(2 * X) + cos(2 * Y)) * (cos(2 * Z) + 2);
        u[0] = rho; u[1] = rho * vx; u[2] = rho * vy;
        if (d == 3) u[3] = rho * vz;
        u[d + 1] = pr / (gm - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
      } else { err = "unknown icType"; return FRG_ERR_ARG; }
    }
  return FRG_OK;
}

}  // namespace frg
