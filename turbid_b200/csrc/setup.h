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
  // interior eigenvectors with exact parity: columns 1..h even, h+1..n-2 odd
  // (h = (n-1)/2), from the folded halves of a centro-symmetric operator
  bool parity = false;
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

// Split form of the folded solve for a decomposition with parity (Dirichlet or
// Neumann on both walls of an odd grid): with W taking the boundary pair
// (y0, yN) to (y0 + yN, y0 - yN),
//   Einvs = W Einvf  (rows 0..h even in the column index, rows h+1..n-1 odd)
//   Es    = Ef W^-1  (columns 0..h even in the row index, h+1..n-1 odd)
// so that Es diag(R) Einvs == Ef diag(R) Einvf (R0 = RN = 1), each a pair of
// half-size products.  Ef's row N-1 is taken without the reference's top-row
// quirk, which the kernel adds back as x[N-1] += quirk * x[0] (the pressure:
// quirk = ftb[0]; other solves qualify only when ftb[0] == 0).  Returns false
// when the decomposition has no parity or the parity check fails.
bool split_operators(const Decomposition& d, bool pressure, std::vector<double>& Einvs, std::vector<double>& Es,
                     double& quirk);

}  // namespace tg
