// Header lines of the two output files, shared by the host writers
// (writers.cpp) and the GPU writer (ipg_write_outputs in api.cu).
#pragma once

#include <string>

namespace ipg {

// "# dummy 1 etamax= ... tau= ...\n" of the hydro file (MyEigen.cpp:380-398)
std::string hydro_header(int N, double L, int sizeOutput, double LOutput, int etaSizeOutput,
                         double detaOutput, int it, double dtau);
// the same without tau, of the KoMPoST file (MyEigen.cpp:810-830)
std::string tmunu_header(int N, double L, int sizeOutput, double LOutput, int etaSizeOutput,
                         double detaOutput);

}  // namespace ipg
