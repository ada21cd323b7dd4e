// gmsh.cpp -- Gmsh v2 ASCII mesh files: geo::readGmsh (src/geo.cpp:448-769)
// and the boundary-condition matching of geo::processConn3D
// (src/geo.cpp:169-193), producing the frg_mesh arrays that frg_create
// pairs faces from (hashed on vertex ids, where the reference compares every
// face with every other).
//
// Host code; no device work.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/frgpu.h"

namespace frg {
frg_status set_error(frg_status st, const std::string &msg);
}
using frg::set_error;

namespace {

std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
  return s;
}

// bcStr2Num (src/global.cpp:11-25); "fluid" / "none" mark the volume
int bc_number(const std::string &name, bool &ok) {
  static const std::map<std::string, int> m = {
      {"none", -1}, {"fluid", -1}, {"periodic", 0}, {"char", 1}, {"sup_in", 2}, {"sup_out", 3},
      {"sub_in", 4}, {"sub_out", 5}, {"slip_wall", 8}, {"isothermal_noslip", 9},
      {"isothermal_noslip_moving", 13}, {"adiabatic_noslip", 10}, {"overset", 11}, {"symmetry", 12}};
  auto it = m.find(name);
  ok = it != m.end();
  return ok ? it->second : -1;
}

// Element face corner lists in the reference's face order: quads
// (src/geo.cpp:789-797) and hexahedra (:798-808).
const int kQuadFV[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
const int kHexFV[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {3, 0, 4, 7}, {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};

// Gmsh's node order of the 4-, 9- and 16-node quads (corners; edge nodes
// edge by edge along the boundary; the interior nodes, themselves a quad)
// is the order of the 2D shape functions (src/funcs.cpp:126-176), and the
// 8-node hexahedron's that of shape_hex, so the nodes are taken as listed.
struct Parsed {
  int nDims = 0, nodesPerEle = 0;
  std::vector<double> verts;          // [nVerts][3]
  std::vector<std::vector<int>> eles;  // 0-based vertex ids, Gmsh node order
  std::vector<std::set<int>> bndPts;   // per boundary, its vertices
  std::vector<int> bndBc;              // per boundary, its BC number
};

frg_status parse(const char *fileName, const char *meshBounds, Parsed &P) {
  std::ifstream in(fileName);
  if (!in.is_open()) return set_error(FRG_ERR_ARG, std::string("Unable to open mesh file ") + fileName);
  // mesh_bound map: "<gmsh name> <bc name>" pairs separated by ';' or newlines
  std::map<std::string, std::string> bounds;
  {
    std::string mb = meshBounds ? meshBounds : "";
    for (char &c : mb)
      if (c == ';' || c == ',') c = '\n';
    std::istringstream ss(mb);
    std::string line;
    while (std::getline(ss, line)) {
      std::istringstream ls(line);
      std::string a, b;
      if (ls >> a >> b) bounds[lower(a)] = lower(b);
    }
  }
  std::string line;
  auto seek = [&](const char *tag) {
    in.clear();
    in.seekg(0, std::ios::beg);
    while (std::getline(in, line))
      if (line.find(tag) != std::string::npos) return true;
    return false;
  };
  // --- $PhysicalNames: each boundary's condition, the volume's dimension
  if (!seek("$PhysicalNames")) return set_error(FRG_ERR_MESH, "$PhysicalNames tag not found in Gmsh file!");
  int nPhys = 0;
  in >> nPhys;
  std::getline(in, line);
  std::map<int, int> bcIdMap;  // Gmsh physical id -> boundary index, -1 = volume
  for (int i = 0; i < nPhys; i++) {
    std::getline(in, line);
    std::istringstream ss(line);
    int dim = 0, id = 0;
    std::string name;
    ss >> dim >> id >> name;
    name.erase(std::remove(name.begin(), name.end(), '"'), name.end());
    name = lower(name);
    auto it = bounds.find(name);
    if (it == bounds.end())
      return set_error(FRG_ERR_MESH, "Unrecognized mesh boundary: \"" + name +
                                         "\" (boundary names must match those in the mesh file)");
    bool ok = false;
    const int bc = bc_number(it->second, ok);
    if (!ok) return set_error(FRG_ERR_MESH, "Unrecognized boundary condition: \"" + it->second + "\"");
    if (it->second == "fluid") {
      P.nDims = dim;
      bcIdMap[id] = -1;
    } else {
      bcIdMap[id] = (int)P.bndBc.size();
      P.bndBc.push_back(bc);
    }
  }
  if (P.nDims != 2 && P.nDims != 3) return set_error(FRG_ERR_MESH, "no \"fluid\" volume of dimension 2 or 3");
  P.bndPts.assign(P.bndBc.size(), {});
  // --- $Nodes
  if (!seek("$Nodes")) return set_error(FRG_ERR_MESH, "$Nodes tag not found in Gmsh file!");
  long nV = 0;
  in >> nV;
  std::getline(in, line);
  P.verts.assign((size_t)nV * 3, 0.0);
  for (long i = 0; i < nV; i++) {
    long id;
    if (!(in >> id >> P.verts[3 * i] >> P.verts[3 * i + 1] >> P.verts[3 * i + 2]))
      return set_error(FRG_ERR_MESH, "short $Nodes section");
    std::getline(in, line);
  }
  // --- $Elements: volume cells and boundary faces
  if (!seek("$Elements")) return set_error(FRG_ERR_MESH, "$Elements tag not found in Gmsh file!");
  long nEl = 0;
  in >> nEl;
  std::getline(in, line);
  for (long k = 0; k < nEl; k++) {
    int id, type, nTags, phys, tmp;
    if (!(in >> id >> type >> nTags >> phys)) return set_error(FRG_ERR_MESH, "short $Elements section");
    for (int t = 0; t < nTags - 1; t++) in >> tmp;
    auto bit = bcIdMap.find(phys);
    const int b = bit == bcIdMap.end() ? -2 : bit->second;
    if (b == -2) return set_error(FRG_ERR_MESH, "element with an undeclared physical id " + std::to_string(phys));
    if (b == -1) {
      // volume cell: linear hexahedra in 3D; linear / quadratic / cubic quads in 2D
      int nn = 0;
      if (P.nDims == 3) {
        if (type != 5)
          return set_error(FRG_ERR_ARG, "Gmsh element type " + std::to_string(type) +
                                            ": 3D volumes must be 8-node hexahedra here");
        nn = 8;
      } else {
        nn = type == 3 ? 4 : type == 10 ? 9 : type == 36 ? 16 : 0;
        if (!nn) return set_error(FRG_ERR_ARG, "Gmsh element type " + std::to_string(type) +
                                                   ": 2D volumes must be 4-, 9- or 16-node quads");
      }
      if (P.nodesPerEle && nn != P.nodesPerEle) return set_error(FRG_ERR_ARG, "mixed element node counts");
      P.nodesPerEle = nn;
      std::vector<int> v(nn);
      for (int i = 0; i < nn; i++) {
        long iv;
        in >> iv;
        if (iv < 1 || iv > nV) return set_error(FRG_ERR_MESH, "node id out of range");
        v[i] = (int)(iv - 1);
      }
      P.eles.push_back(std::move(v));
    } else {
      // boundary face: its corner vertices join the boundary's point set
      // (the reference collects the first 2 / 3 / 4 nodes by face type)
      int nPts = 0;
      switch (type) {
        case 1: case 8: case 26: case 27: case 28: nPts = 2; break;  // edges: the end points
        case 2: nPts = 3; break;
        case 3: case 10: case 16: case 36: case 37: case 38: nPts = 4; break;
        default:
          return set_error(FRG_ERR_MESH, "Boundary Element (Face) Type Not Recognized! (Gmsh type " +
                                             std::to_string(type) + ")");
      }
      for (int i = 0; i < nPts; i++) {
        long iv;
        in >> iv;
        P.bndPts[b].insert((int)(iv - 1));
      }
    }
    std::getline(in, line);
  }
  if (P.eles.empty()) return set_error(FRG_ERR_MESH, "no volume elements");
  return FRG_OK;
}

}  // namespace

extern "C" {

frg_status frg_read_gmsh(const char *fileName, const char *meshBounds, int *nDims, int *nEles, int *nNodes,
                         double *xv, int *c2v, int *bc) {
  if (!fileName || !nDims || !nEles || !nNodes) return set_error(FRG_ERR_ARG, "null argument");
  Parsed P;
  frg_status st = parse(fileName, meshBounds, P);
  if (st) return st;
  const int d = P.nDims, nE = (int)P.eles.size(), nN = P.nodesPerEle, nC = d == 2 ? 4 : 8, nFc = d == 2 ? 4 : 6;
  *nDims = d;
  *nEles = nE;
  *nNodes = nN;
  if (!xv && !c2v && !bc) return FRG_OK;
  if (!xv || !c2v || !bc) return set_error(FRG_ERR_ARG, "null output array");
  for (int e = 0; e < nE; e++) {
    const std::vector<int> &v = P.eles[e];
    for (int n = 0; n < nN; n++)
      for (int k = 0; k < d; k++) xv[((size_t)e * nN + n) * d + k] = P.verts[3 * (size_t)v[n] + k];
    for (int c = 0; c < nC; c++) c2v[(size_t)e * nC + c] = v[c];
  }
  // faces: a face no other element shares is a boundary face; it takes the
  // condition of the first boundary whose point set holds all its corners
  // (processConn3D, src/geo.cpp:169-193); faces two elements share get -1
  std::map<std::vector<int>, int> count;
  auto face_key = [&](int e, int f) {
    std::vector<int> k;
    for (int j = 0; j < (d == 2 ? 2 : 4); j++) k.push_back(P.eles[e][d == 2 ? kQuadFV[f][j] : kHexFV[f][j]]);
    std::sort(k.begin(), k.end());
    return k;
  };
  for (int e = 0; e < nE; e++)
    for (int f = 0; f < nFc; f++) count[face_key(e, f)]++;
  for (int e = 0; e < nE; e++)
    for (int f = 0; f < nFc; f++) {
      const std::vector<int> k = face_key(e, f);
      int b = -1;
      if (count[k] == 1) {
        for (size_t q = 0; q < P.bndBc.size() && b < 0; q++) {
          bool on = true;
          for (int x : k) on = on && P.bndPts[q].count(x);
          if (on) b = P.bndBc[q];
        }
        if (b < 0) {
          char m[128];
          snprintf(m, sizeof m, "boundary face %d of element %d lies on no boundary of the mesh file", f, e);
          return set_error(FRG_ERR_MESH, m);
        }
      }
      bc[(size_t)e * nFc + f] = b;
    }
  return FRG_OK;
}

}  // extern "C"
