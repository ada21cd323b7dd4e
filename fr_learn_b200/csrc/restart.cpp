// restart.cpp -- the reference's ParaView output, which is also its restart
// file: writeParaview (src/output.cpp:103-391) and solver::readRestartFile /
// ele::restart (src/solver.cpp:1420-1482, src/ele.cpp:1451-1880).
//
// Per element one <Piece> of (P+3)^d plot points -- the tensor grid of the 1D
// points {-1, solution points, +1}, x fastest -- holding the primitive
// variables interpolated from the solution points (extrapolateUPpts,
// src/solver.cpp:449-483), the plot-point coordinates and the linear
// sub-cells.  Numbers are written with 16 significant digits as the
// reference's stream does.  A restart reads back the interior plot points,
// which are the solution points, converts them to conservative variables and
// interpolates to the solver's order when the file's order differs.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "setup.h"

namespace frg {
frg_status set_error(frg_status st, const std::string &msg);
}

namespace {

using frg::set_error;

std::string file_name(const char *base, int iter) {
  char buf[32];
  snprintf(buf, sizeof buf, "_%.09d.vtu", iter);
  return std::string(base) + buf;
}

void put(std::string &o, double v) {
  char buf[40];
  snprintf(buf, sizeof buf, "%.16g ", v);
  o += buf;
}
void put(std::string &o, long v) {
  char buf[24];
  snprintf(buf, sizeof buf, "%ld ", v);
  o += buf;
}

int n_fields(const frg_params &p) { return p.equation == 0 ? 1 : p.nDims + 2; }

// The value of Name="..." on a tag line, or "".
std::string attr(const std::string &line, const char *key) {
  const std::string k = std::string(key) + "=\"";
  size_t a = line.find(k);
  if (a == std::string::npos) return "";
  a += k.size();
  size_t b = line.find('"', a);
  return b == std::string::npos ? "" : line.substr(a, b - a);
}

}  // namespace

extern "C" {

frg_status frg_write_paraview_host(const frg_params *params, const frg_mesh *mesh, const double *U, double time,
                                   int iter, const char *dataFileName) {
  if (!params || !mesh || !mesh->xv || !U || !dataFileName) return set_error(FRG_ERR_ARG, "null argument");
  const frg_params &p = *params;
  const int d = p.nDims, P = p.order, nE = mesh->nEles, nN = mesh->nNodes, nV = n_fields(p);
  if ((d != 2 && d != 3) || P < 1 || P > 5 || nE < 1) return set_error(FRG_ERR_ARG, "bad parameters");
  std::vector<double> shapeP, interpP;
  std::string err;
  if (!frg::plot_tables(d, P, nN, shapeP, interpP, err)) return set_error(FRG_ERR_ARG, err);
  const int n1 = P + 1, n3 = P + 3, nS = d == 2 ? n1 * n1 : n1 * n1 * n1;
  const int nP = d == 2 ? n3 * n3 : n3 * n3 * n3, nSub = d == 2 ? (n3 - 1) * (n3 - 1) : (n3 - 1) * (n3 - 1) * (n3 - 1);
  const std::string path = file_name(dataFileName, iter);
  FILE *f = fopen(path.c_str(), "w");
  if (!f) return set_error(FRG_ERR_ARG, "cannot open " + path);
  std::string o;
  o.reserve(1 << 20);
  char buf[96];
  o += "<?xml version=\"1.0\" ?>\n";
  o += "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" "
       "compressor=\"vtkZLibDataCompressor\">\n";
  snprintf(buf, sizeof buf, "<!-- TIME %.16g -->\n<!-- ITER %d -->\n", time, iter);
  o += buf;
  o += "\t<UnstructuredGrid>\n";
  std::vector<double> V((size_t)nS * nV), Vp((size_t)nP * nV);
  for (int e = 0; e < nE; e++) {
    // primitives at the solution points, then V_ppts = opp_spts_to_ppts V_spts
    for (int s = 0; s < nS; s++) {
      const double *u = U + ((size_t)s * nE + e) * nV;
      double *v = &V[(size_t)s * nV];
      if (p.equation == 0) {
        v[0] = u[0];
        continue;
      }
      const double rho = u[0], ux = u[1] / rho, uy = u[2] / rho;
      double w = 0, vMagSq = ux * ux + uy * uy;
      if (d == 3) {
        w = u[3] / rho;
        vMagSq += w * w;
        v[3] = w;
      }
      v[0] = rho;
      v[1] = ux;
      v[2] = uy;
      v[d + 1] = (p.gamma - 1) * (u[d + 1] - 0.5 * rho * vMagSq);
    }
    for (int q = 0; q < nP; q++)
      for (int k = 0; k < nV; k++) {
        double acc = 0.0;
        for (int s = 0; s < nS; s++) acc += interpP[(size_t)q * nS + s] * V[(size_t)s * nV + k];
        Vp[(size_t)q * nV + k] = acc;
      }
    snprintf(buf, sizeof buf, "\t\t<Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", nP, nSub);
    o += buf;
    o += "\t\t\t<PointData>\n";
    o += "\t\t\t\t<DataArray type=\"Float32\" Name=\"Density\" format=\"ascii\">\n";
    for (int q = 0; q < nP; q++) put(o, Vp[(size_t)q * nV]);
    o += "\n\t\t\t\t</DataArray>\n";
    if (p.equation == 1) {
      o += "\t\t\t\t<DataArray type=\"Float32\" NumberOfComponents=\"3\" Name=\"Velocity\" format=\"ascii\">\n";
      // 2D: ParaView needs three components; the third is written as 0
      for (int q = 0; q < nP; q++) {
        put(o, Vp[(size_t)q * nV + 1]);
        put(o, Vp[(size_t)q * nV + 2]);
        put(o, d == 3 ? Vp[(size_t)q * nV + 3] : 0.0);
      }
      o += "\n\t\t\t\t</DataArray>\n";
      o += "\t\t\t\t<DataArray type=\"Float32\" Name=\"Pressure\" format=\"ascii\">\n";
      for (int q = 0; q < nP; q++) put(o, Vp[(size_t)q * nV + d + 1]);
      o += "\n\t\t\t\t</DataArray>\n";
    }
    o += "\t\t\t</PointData>\n";
    o += "\t\t\t<Points>\n";
    o += "\t\t\t\t<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n";
    const double *X = mesh->xv + (size_t)e * nN * d;
    for (int q = 0; q < nP; q++) {
      for (int k = 0; k < d; k++) {
        double acc = 0.0;
        for (int n = 0; n < nN; n++) acc += shapeP[(size_t)q * nN + n] * X[n * d + k];
        put(o, acc);
      }
      if (d == 2) o += "0 ";
    }
    o += "\n\t\t\t\t</DataArray>\n";
    o += "\t\t\t</Points>\n";
    o += "\t\t\t<Cells>\n";
    o += "\t\t\t\t<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n";
    const long m = n3;
    if (d == 2) {
      for (long j = 0; j < m - 1; j++)
        for (long i = 0; i < m - 1; i++) {
          put(o, j * m + i);
          put(o, j * m + i + 1);
          put(o, (j + 1) * m + i + 1);
          put(o, (j + 1) * m + i);
          o += "\n";
        }
    } else {
      for (long k = 0; k < m - 1; k++)
        for (long j = 0; j < m - 1; j++)
          for (long i = 0; i < m - 1; i++) {
            for (long kk = k; kk <= k + 1; kk++) {
              put(o, i + m * (j + m * kk));
              put(o, i + 1 + m * (j + m * kk));
              put(o, i + 1 + m * (j + 1 + m * kk));
              put(o, i + m * (j + 1 + m * kk));
            }
            o += "\n";
          }
    }
    o += "\t\t\t\t</DataArray>\n";
    o += "\t\t\t\t<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n";
    const long nv = d == 2 ? 4 : 8;
    for (long k = 0; k < nSub; k++) put(o, (k + 1) * nv);
    o += "\n\t\t\t\t</DataArray>\n";
    o += "\t\t\t\t<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
    for (long k = 0; k < nSub; k++) put(o, d == 2 ? 9L : 12L);
    o += "\n\t\t\t\t</DataArray>\n";
    o += "\t\t\t</Cells>\n";
    o += "\t\t</Piece>\n";
    if (o.size() > (1u << 20)) {
      fwrite(o.data(), 1, o.size(), f);
      o.clear();
    }
  }
  o += "\t</UnstructuredGrid>\n";
  o += "</VTKFile>\n";
  fwrite(o.data(), 1, o.size(), f);
  const bool bad = ferror(f) != 0;
  if (fclose(f) != 0 || bad) return set_error(FRG_ERR_ARG, "write error on " + path);
  return FRG_OK;
}

frg_status frg_read_restart_host(const frg_params *params, int nEles, const char *dataFileName, int restartIter,
                                 double *U, double *time) {
  if (!params || !dataFileName || !U || nEles < 1) return set_error(FRG_ERR_ARG, "null argument");
  const frg_params &p = *params;
  const int d = p.nDims, P = p.order, nE = nEles, nV = n_fields(p);
  const int n1 = P + 1, nS = d == 2 ? n1 * n1 : n1 * n1 * n1;
  const std::string path = file_name(dataFileName, restartIter);
  std::ifstream in(path);
  if (!in.is_open()) return set_error(FRG_ERR_ARG, "Cannot open restart file " + path);
  std::string line;
  bool foundUG = false;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::string a, b;
    ss >> a;
    if (a == "<!--") {
      ss >> b;
      if (b == "TIME" && time) ss >> *time;
    } else if (a == "<UnstructuredGrid>") {
      foundUG = true;
      break;
    }
  }
  if (!foundUG) return set_error(FRG_ERR_ARG, "Cannot find UnstructuredData tag in restart file.");
  std::vector<double> interp;
  int interpFrom = -1;
  for (int e = 0; e < nE; e++) {
    bool piece = false;
    while (std::getline(in, line))
      if (line.find("<Piece") != std::string::npos) {
        piece = true;
        break;
      }
    if (!piece) {
      // ele::restart (src/ele.cpp:1469-1478): an element the file does not
      // hold is reported and its solution set to 100 in every field; the
      // read goes on with the next element
      printf("Restart-file element doesn't exist!\n");
      for (int s = 0; s < nS; s++)
        for (int k = 0; k < nV; k++) U[((size_t)s * nE + e) * nV + k] = 100.;
      continue;
    }
    const long nPts = atol(attr(line, "NumberOfPoints").c_str()), nCells = atol(attr(line, "NumberOfCells").c_str());
    // nCells = (order + 2)^d sub-cells
    const int Pf = (int)lround(d == 2 ? std::sqrt((double)nCells) : std::cbrt((double)nCells)) - 2;
    const long n3 = Pf + 3;
    if (Pf < 0 || Pf > 5 || nPts != (d == 2 ? n3 * n3 : n3 * n3 * n3))
      return set_error(FRG_ERR_ARG, "restart file: unexpected piece size");
    const int nf1 = Pf + 1, nSf = d == 2 ? nf1 * nf1 : nf1 * nf1 * nf1;
    std::vector<double> rho(nSf), vel((size_t)nSf * 3), pr(nSf);
    bool gotR = false, gotV = false, gotP = false;
    while (std::getline(in, line) && line.find("</PointData>") == std::string::npos) {
      if (line.find("<DataArray") == std::string::npos) continue;
      const std::string name = attr(line, "Name");
      const int nc = name == "Velocity" ? 3 : 1;
      double *dst = name == "Density" ? rho.data() : name == "Velocity" ? vel.data() : name == "Pressure" ? pr.data()
                                                                                                           : nullptr;
      if (!std::getline(in, line)) break;
      if (!dst) continue;
      // plot point (i+1, j+1, k+1) holds solution point (i, j, k)
      const char *c = line.c_str();
      char *end = nullptr;
      long q = 0;
      for (; q < nPts * nc; q++) {
        const double v = strtod(c, &end);
        if (end == c) break;
        c = end;
        const long pt = q / nc, comp = q % nc;
        const long i = pt % n3 - 1, j = (pt / n3) % n3 - 1, k = d == 3 ? pt / (n3 * n3) - 1 : 0;
        if (i < 0 || i > Pf || j < 0 || j > Pf || k < 0 || k > Pf) continue;
        dst[(size_t)(i + nf1 * (j + nf1 * k)) * nc + comp] = v;
      }
      if (q != nPts * nc) return set_error(FRG_ERR_ARG, "restart file: short data array " + name);
      if (name == "Density") gotR = true;
      if (name == "Velocity") gotV = true;
      if (name == "Pressure") gotP = true;
    }
    if (!gotR || (p.equation == 1 && !(gotV && gotP)))
      return set_error(FRG_ERR_ARG, "restart file: missing Density / Velocity / Pressure");
    while (line.find("</Piece>") == std::string::npos && std::getline(in, line)) {
    }
    // primitives -> conservative (src/ele.cpp:1764-1783)
    std::vector<double> tU((size_t)nSf * nV);
    for (int s = 0; s < nSf; s++) {
      double *u = &tU[(size_t)s * nV];
      u[0] = rho[s];
      if (p.equation == 0) continue;
      const double *v = &vel[(size_t)s * 3];
      u[1] = u[0] * v[0];
      u[2] = u[0] * v[1];
      double vSq = v[0] * v[0] + v[1] * v[1];
      if (d == 3) {
        u[3] = u[0] * v[2];
        vSq += v[2] * v[2];
      }
      u[d + 1] = pr[s] / (p.gamma - 1) + 0.5 * u[0] * vSq;
    }
    if (Pf != P) {
      if (interpFrom != Pf) {
        frg::order_interp(d, Pf, P, interp);
        interpFrom = Pf;
      }
      for (int s = 0; s < nS; s++)
        for (int k = 0; k < nV; k++) {
          double acc = 0.0;
          for (int r = 0; r < nSf; r++) acc += interp[(size_t)s * nSf + r] * tU[(size_t)r * nV + k];
          U[((size_t)s * nE + e) * nV + k] = acc;
        }
    } else {
      for (int s = 0; s < nS; s++)
        for (int k = 0; k < nV; k++) U[((size_t)s * nE + e) * nV + k] = tU[(size_t)s * nV + k];
    }
  }
  return FRG_OK;
}

}  // extern "C"
