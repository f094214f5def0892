// Wannier tight-binding model as the reference reads it (src/wannier_tb.cpp:15-113).
#pragma once
#include <complex>
#include <string>
#include <vector>

namespace hhg {

using cd = std::complex<double>;

struct TBModel {
  std::string comment;
  double lattice[3][3] = {};       // rows a1, a2, a3 (Angstrom)
  int nw = 0;                      // orbitals
  int nsites = 0;                  // R cells
  std::vector<int> degeneracy;     // parsed and, as in the reference, never applied
  std::vector<int> R;              // [nsites][3]
  std::vector<cd> hop;             // [nsites][nw][nw]; line "m n" stored at [n-1][m-1]
  std::vector<cd> bc[3];           // position elements x, y, z in the same layout (Angstrom)
};

// Throws std::runtime_error with a message on a missing or malformed file.
TBModel parse_tb(const std::string& path);

}  // namespace hhg
