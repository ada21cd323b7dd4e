// optab_upload.cuh -- fills this translation unit's copy of the 1D operator
// tables (c_opd / c_opf, internal linkage in kernels.cuh) for every VCJH
// scheme and order.  Included once by each kernel unit.
#pragma once
#include "kernels.cuh"
#include "setup.h"

namespace frg {
namespace {

inline cudaError_t upload_tables_impl() {
  static OpTab<double> hd[4][KMAXP + 1];
  static OpTab<float> hf[4][KMAXP + 1];
  for (int sch = 0; sch < 4; sch++)
    for (int P = 0; P <= KMAXP; P++) {
      if ((sch == 3 && P < 2) || (sch == 2 && P == 0)) continue;  // eta undefined there
      Ops1D o = build_ops1d(P, sch);
      OpTab<double> &d = hd[sch][P];
      OpTab<float> &f = hf[sch][P];
      for (int i = 0; i <= KMAXP; i++) {
        d.lag[0][i] = o.lag[0][i]; d.lag[1][i] = o.lag[1][i];
        d.gL[i] = o.gL[i]; d.gR[i] = o.gR[i]; d.w[i] = o.w[i];
        f.lag[0][i] = (float)o.lag[0][i]; f.lag[1][i] = (float)o.lag[1][i];
        f.gL[i] = (float)o.gL[i]; f.gR[i] = (float)o.gR[i]; f.w[i] = (float)o.w[i];
        for (int j = 0; j <= KMAXP; j++) { d.dlag[i][j] = o.dlag[i][j]; f.dlag[i][j] = (float)o.dlag[i][j]; }
      }
    }
  cudaError_t e = cudaMemcpyToSymbol(c_opd, hd, sizeof hd);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_opf, hf, sizeof hf);
  return e;
}

}  // namespace
}  // namespace frg
