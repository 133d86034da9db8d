// Host-side z-operator construction (FP64) shared by libturbid_gpu.so and
// the CPU unit tests of the eigen-solver.
#pragma once
#include <vector>

namespace tg {

// Chebyshev-Gauss-Lobatto grid z_i = cos((n-1-i) pi/(n-1)), D1, D2 (row-major
// n x n); gridzc is the mapped grid (== gridz without mapping).
void chebyshev_operators(int n, int mapping, double coef, std::vector<double>& gridz, std::vector<double>& D1,
                         std::vector<double>& D2, std::vector<double>& gridzc);

struct Decomposition {
  int n = 0;
  std::vector<double> E, Einv, lam;            // n x n with identity corners; lam[n]
  std::vector<double> fbb, ftb, fbf, ftf;      // fix rows
};

// F (n x n row-major) = V diag(lam) V^-1 with a real spectrum.
void real_eigen(const std::vector<double>& F, int n, std::vector<double>& lam, std::vector<double>& V,
                std::vector<double>& Vinv);

// bc = {a_bottom, b_bottom, a_top, b_top}: a f + b f' = c.
void build_decomposition(int n, const std::vector<double>& D1, const std::vector<double>& D2, const double* bc,
                         Decomposition& out);

// Folds the fix rows into the two matrices applied by the GPU solve:
//   Einvf = Einv * T   (T: forward fix, or zeroed boundary rows for the pressure)
//   Ef    = B * E      (B: backward fix rows 0 and N-1, row N-1 after row 0)
void fold_decomposition(const Decomposition& d, bool pressure, std::vector<double>& Einvf, std::vector<double>& Ef);

}  // namespace tg
