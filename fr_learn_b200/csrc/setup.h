// setup.h -- host-side set-up of the FR path: 1D operator tables, dense
// operator matrices (for inspection), element metrics and face connectivity,
// laid out for the device kernels.  Runs once per solver, on the host, as the
// reference's setup does (solver::setup, src/solver.cpp:21-63).
#pragma once
#include <string>
#include <vector>

#include "../../include/frgpu.h"

namespace frg {

constexpr int MAXP = 5;

// 1D ingredients of every tensor-product operator of one order P.
//   pts   Gauss-Legendre solution points (the reference's 15-decimal table)
//   lag[s][j]  Lagrange basis j at xi = -1 (s=0) / +1 (s=1)
//   dlag[i][j] d/dxi of basis j at solution point i
//   gL/gR[i]   derivative of the left/right VCJH correction function at point i
//   w     Gauss weights (the reference's table)
struct Ops1D {
  int P = 0;
  double pts[MAXP + 1] = {0}, w[MAXP + 1] = {0};
  double lag[2][MAXP + 1] = {{0}};
  double dlag[MAXP + 1][MAXP + 1] = {{0}};
  double gL[MAXP + 1] = {0}, gR[MAXP + 1] = {0};
};
Ops1D build_ops1d(int P, int vcjh);

// Dense matrices as oper::setupOperators stores them (row-major).
void dense_operator(int nDims, const Ops1D &o, int which, int dim, std::vector<double> &out);

// Per-solver geometry in device layout ([..][point][element], element fastest).
struct HostGeom {
  int nDims = 0, P = 0, nS = 0, nF = 0, nFF = 0, nE = 0, nFaceEle = 0;
  std::vector<double> pos_spts;  // [nS][nE][d]  (reference layout, host only)
  std::vector<double> JG;        // [d1][d2][nS][nE]   JGinv(d1, spt, e, d2)
  std::vector<double> detJ;      // [nS][nE]
  std::vector<double> nrmC;      // [d][nF][nE]  normal of the face's left element
  std::vector<double> nrmOwn;    // [d][nF][nE]  this element's own outward normal
  std::vector<double> dA;        // [nF][nE]
  std::vector<double> vol;       // [nE]         sum detJ * w
  std::vector<double> dAw;       // [nF][nE]     dA * surface weight
  std::vector<int> nbr;          // [nF][nE]     (traceIndex<<1 | isRight) or -1-bc
  std::vector<int> faceTable;    // [nFaces][6]  eL, fL, eR, fR, relRot, bc
  long nIntFaces = 0, nBndFaces = 0;
};

// Shape-function tables of the element metrics of one order and node count,
// shared by the host set-up and the device metric kernel:
//   shS [nS][nN]     node shape functions at the solution points
//   dS  [d][nS][nN]  their reference derivatives at the solution points
//   dF  [d][nF][nN]  ... and at the flux points
//   fdir [nF]        normal reference direction of the flux point's face
//   fsgn [nF]        +1 / -1 for the face at xi_dir = +1 / -1
//   wv [nS], ws [nF] volume / surface quadrature weights
struct MetricTables {
  int nDims = 0, nS = 0, nF = 0, nN = 0;
  std::vector<double> shS, dS, dF, wv, ws;
  std::vector<int> fdir, fsgn;
};
bool metric_tables(int nDims, int P, int vcjh, int nNodes, MetricTables &t, std::string &err);

// Plot points of the reference's ParaView / restart files: the tensor grid of
// the 1D points {-1, solution points, +1}, x fastest (getLocPpts,
// src/points.cpp:130-160), (P+3)^d per element.
//   shapeP  [nP][nN]  node shape functions at the plot points
//   interpP [nP][nS]  opp_spts_to_ppts (src/operators.cpp:114-140)
bool plot_tables(int nDims, int P, int nNodes, std::vector<double> &shapeP, std::vector<double> &interpP,
                 std::string &err);
// Gauss points of quadOrder (the reference's loc_qpts, src/operators.cpp:305-316)
// for integrateError: node shape functions there [nQ][nN], the solution-point
// interpolation opp_spts_to_qpts [nQ][nS] and the weights [nQ] in
// getQptWeights's order (src/points.cpp:347-374).
bool quad_tables(int nDims, int P, int nNodes, int quadOrder, std::vector<double> &shapeQ,
                 std::vector<double> &interpQ, std::vector<double> &wq, std::string &err);
// Node shape functions at the solution points [nS][nN].
bool spt_shape_table(int nDims, int P, int nNodes, std::vector<double> &shapeS, std::string &err);
// Lagrange interpolation between the solution points of two orders
// ([nS_to][nS_from], the restart's inter-order operator, src/ele.cpp:1506-1555).
void order_interp(int nDims, int Pfrom, int Pto, std::vector<double> &out);

// Builds metrics and connectivity.  Returns FRG_OK or an error with `err` set.
frg_status build_geometry(const frg_params &p, const frg_mesh &m, HostGeom &g, std::string &err);

// Initial condition of ele::setInitialCondition on the host, reference layout
// [nS][nE][nV].
frg_status initial_condition(const frg_params &p, const HostGeom &g, int icType, double a0,
                             std::vector<double> &U, std::string &err);

}  // namespace frg
