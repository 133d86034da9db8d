// Host-side construction of the z-operators (FP64), done once per case:
//   * Chebyshev-Gauss-Lobatto D1 with the negative-sum diagonal and optional
//     grid mapping, D2 = D1*D1 with the negative-sum diagonal
//     (reference src/stepper_space_chebyshev.cc:101-228);
//   * the boundary-condensed Helmholtz decomposition of CmDz2DecompositionCplx
//     (reference src/cmdz2_decomposition.cc:19-227): BC rows, four fix rows,
//     condensed interior operator F, eigen-decomposition F = V diag(lam) V^-1.
// The eigen-decomposition is our own: Parlett-Reinsch balancing, Householder
// reduction to Hessenberg form, Francis double-shift QR for the eigenvalues
// (Golub & Van Loan, Matrix Computations, alg. 7.5.1-7.5.2) and inverse
// iteration on the Hessenberg matrix for the eigenvectors; eigenvalues are
// then refined by the two-sided Rayleigh quotient in extended precision.
// The spectrum of these collocation operators is real; a complex pair is
// reported as a setup error.
#include "setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace tg {

static const double kPi = 3.141592653589793238462643383279502884;

void chebyshev_operators(int n, int mapping, double coef, std::vector<double>& gridz, std::vector<double>& D1,
                         std::vector<double>& D2, std::vector<double>& gridzc) {
  gridz.assign(n, 0.0);
  for (int i = 0; i < n; ++i) gridz[i] = std::cos((n - i - 1) * kPi / (n - 1));
  D1.assign((size_t)n * n, 0.0);
  auto d1 = [&](int i, int j) -> double& { return D1[(size_t)i * n + j]; };
  for (int i = 1; i < n; ++i)
    for (int j = 0; j < i; ++j) d1(i, j) = (((i + j) & 1) ? -1.0 : 1.0) / (gridz[i] - gridz[j]);
  for (int i = 0; i < n; ++i) d1(i, 0) *= 0.5;
  for (int j = 0; j < n; ++j) d1(n - 1, j) *= 2.0;
  for (int i = 0; i < n - 1; ++i)
    for (int j = i + 1; j < n; ++j) d1(i, j) = -d1(n - 1 - i, n - 1 - j);
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) s -= d1(i, j);
    d1(i, i) = s;
  }
  gridzc = gridz;
  if (mapping != 0) {
    std::vector<double> dc(n);
    for (int i = 0; i < n; ++i) {
      double z = gridz[i];
      if (mapping == 1) {
        double t = std::tan(kPi / 2 * z);
        gridzc[i] = 2 / kPi * std::atan(coef * t);
        dc[i] = 1 / coef * (1 + (coef * t) * (coef * t)) / (1 + t * t);
      } else if (mapping == 2) {
        gridzc[i] = std::asin(coef * z) / std::asin(coef);
        dc[i] = 1 / coef * std::cos(std::asin(coef * z)) * std::asin(coef);
      } else if (mapping == 3) {
        double t = std::tan(kPi / 4 * (z - 1));
        gridzc[i] = 4 / kPi * std::atan(coef * t) + 1;
        dc[i] = 1 / coef * (1 + (coef * t) * (coef * t)) / (1 + t * t);
      } else {
        throw std::runtime_error("SpaceStepper > Unsupported Mapping Function!");
      }
    }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) d1(i, j) *= dc[i];
  }
  D2.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) {
      double a = D1[(size_t)i * n + k];
      if (a == 0.0) continue;
      const double* row = &D1[(size_t)k * n];
      double* out = &D2[(size_t)i * n];
      for (int j = 0; j < n; ++j) out[j] += a * row[j];
    }
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < n; ++j)
      if (j != i) s -= D2[(size_t)i * n + j];
    D2[(size_t)i * n + i] = s;
  }
}

// ---------------------------------------------------------------------------
// eigen-solver pieces (row-major dense n x n)
// ---------------------------------------------------------------------------
namespace {

struct Mat {
  int n;
  std::vector<double> a;
  explicit Mat(int n_) : n(n_), a((size_t)n_ * n_, 0.0) {}
  double& operator()(int i, int j) { return a[(size_t)i * n + j]; }
  double operator()(int i, int j) const { return a[(size_t)i * n + j]; }
};

// Parlett-Reinsch balancing with powers of two; returns scale d (A <- D^-1 A D)
std::vector<double> balance(Mat& A) {
  const int n = A.n;
  std::vector<double> d(n, 1.0);
  const double radix = 2.0, sqrdx = 4.0;
  bool done = false;
  while (!done) {
    done = true;
    for (int i = 0; i < n; ++i) {
      double r = 0.0, c = 0.0;
      for (int j = 0; j < n; ++j)
        if (j != i) {
          c += std::fabs(A(j, i));
          r += std::fabs(A(i, j));
        }
      if (c != 0.0 && r != 0.0) {
        double g = r / radix, f = 1.0, s = c + r;
        while (c < g) {
          f *= radix;
          c *= sqrdx;
        }
        g = r * radix;
        while (c > g) {
          f /= radix;
          c /= sqrdx;
        }
        if ((c + r) / f < 0.95 * s) {
          done = false;
          g = 1.0 / f;
          d[i] *= f;
          for (int j = 0; j < n; ++j) A(i, j) *= g;
          for (int j = 0; j < n; ++j) A(j, i) *= f;
        }
      }
    }
  }
  return d;
}

// Householder reduction to upper Hessenberg: A <- Q^T A Q, returns Q
Mat hessenberg(Mat& A) {
  const int n = A.n;
  Mat Q(n);
  for (int i = 0; i < n; ++i) Q(i, i) = 1.0;
  std::vector<double> v(n);
  for (int k = 0; k < n - 2; ++k) {
    double alpha = 0.0;
    for (int i = k + 1; i < n; ++i) alpha += A(i, k) * A(i, k);
    alpha = std::sqrt(alpha);
    if (alpha == 0.0) continue;
    if (A(k + 1, k) > 0) alpha = -alpha;
    double vnorm2 = 0.0;
    for (int i = 0; i < n; ++i) v[i] = 0.0;
    v[k + 1] = A(k + 1, k) - alpha;
    for (int i = k + 2; i < n; ++i) v[i] = A(i, k);
    for (int i = k + 1; i < n; ++i) vnorm2 += v[i] * v[i];
    if (vnorm2 == 0.0) continue;
    const double beta = 2.0 / vnorm2;
    // A <- (I - beta v v^T) A
    for (int j = 0; j < n; ++j) {
      double s = 0.0;
      for (int i = k + 1; i < n; ++i) s += v[i] * A(i, j);
      s *= beta;
      for (int i = k + 1; i < n; ++i) A(i, j) -= s * v[i];
    }
    // A <- A (I - beta v v^T) ; Q <- Q (I - beta v v^T)
    for (int i = 0; i < n; ++i) {
      double s = 0.0, t = 0.0;
      for (int j = k + 1; j < n; ++j) {
        s += A(i, j) * v[j];
        t += Q(i, j) * v[j];
      }
      s *= beta;
      t *= beta;
      for (int j = k + 1; j < n; ++j) {
        A(i, j) -= s * v[j];
        Q(i, j) -= t * v[j];
      }
    }
    for (int i = k + 2; i < n; ++i) A(i, k) = 0.0;
  }
  return Q;
}

// apply a 3- (or 2-) element Householder reflector P = I - 2 u u^T/(u^T u)
// from the left on rows r..r+len-1 over columns [c0, c1] and from the right
// on columns r..r+len-1 over rows [q0, q1]
void reflect(Mat& H, const double* u, int len, int r, int c0, int c1, int q0, int q1) {
  double uu = 0.0;
  for (int i = 0; i < len; ++i) uu += u[i] * u[i];
  if (uu == 0.0) return;
  const double beta = 2.0 / uu;
  for (int j = c0; j <= c1; ++j) {
    double s = 0.0;
    for (int i = 0; i < len; ++i) s += u[i] * H(r + i, j);
    s *= beta;
    for (int i = 0; i < len; ++i) H(r + i, j) -= s * u[i];
  }
  for (int i = q0; i <= q1; ++i) {
    double s = 0.0;
    for (int j = 0; j < len; ++j) s += H(i, r + j) * u[j];
    s *= beta;
    for (int j = 0; j < len; ++j) H(i, r + j) -= s * u[j];
  }
}

void householder_vec(double x, double y, double z, int len, double* u) {
  double nrm = std::sqrt(x * x + y * y + (len == 3 ? z * z : 0.0));
  double s = (x >= 0) ? nrm : -nrm;
  u[0] = x + s;
  u[1] = y;
  if (len == 3) u[2] = z;
}

// Francis double-shift QR on an upper Hessenberg matrix (eigenvalues only)
void hessenberg_qr(Mat H, std::vector<double>& wr, std::vector<double>& wi) {
  const int n = H.n;
  wr.assign(n, 0.0);
  wi.assign(n, 0.0);
  const double eps = 2.220446049250313e-16;
  int hi = n - 1;
  int iter = 0;
  while (hi >= 0) {
    // find the start of the active unreduced block
    int lo = hi;
    while (lo > 0) {
      double s = std::fabs(H(lo - 1, lo - 1)) + std::fabs(H(lo, lo));
      if (s == 0.0) s = 1.0;
      if (std::fabs(H(lo, lo - 1)) <= eps * s) {
        H(lo, lo - 1) = 0.0;
        break;
      }
      --lo;
    }
    if (lo == hi) {  // 1x1 block converged
      wr[hi] = H(hi, hi);
      wi[hi] = 0.0;
      --hi;
      iter = 0;
      continue;
    }
    if (lo == hi - 1) {  // 2x2 block
      double a = H(hi - 1, hi - 1), b = H(hi - 1, hi), c = H(hi, hi - 1), d = H(hi, hi);
      double p = 0.5 * (a - d), q = p * p + b * c;
      if (q >= 0) {
        double z = std::sqrt(q);
        z = (p >= 0) ? p + z : p - z;
        double l1 = d + z;
        double l2 = (z != 0.0) ? d - b * c / z : d + z;
        wr[hi - 1] = l1;
        wr[hi] = l2;
      } else {
        wr[hi - 1] = wr[hi] = d + p;
        wi[hi - 1] = std::sqrt(-q);
        wi[hi] = -std::sqrt(-q);
      }
      hi -= 2;
      iter = 0;
      continue;
    }
    if (++iter > 200) throw std::runtime_error("CmDz2Decomposition > QR iteration did not converge");
    // double shift from the trailing 2x2 (exceptional shift every 11 iterations)
    double s, t;
    if (iter % 11 == 10) {
      double w = std::fabs(H(hi, hi - 1)) + std::fabs(H(hi - 1, hi - 2));
      s = 1.5 * w;
      t = w * w;
    } else {
      s = H(hi - 1, hi - 1) + H(hi, hi);
      t = H(hi - 1, hi - 1) * H(hi, hi) - H(hi - 1, hi) * H(hi, hi - 1);
    }
    double x = H(lo, lo) * H(lo, lo) + H(lo, lo + 1) * H(lo + 1, lo) - s * H(lo, lo) + t;
    double y = H(lo + 1, lo) * (H(lo, lo) + H(lo + 1, lo + 1) - s);
    double z = H(lo + 1, lo) * H(lo + 2, lo + 1);
    for (int k = lo; k <= hi - 2; ++k) {
      double u[3];
      householder_vec(x, y, z, 3, u);
      int c0 = std::max(lo, k - 1);
      int q1 = std::min(k + 3, hi);
      reflect(H, u, 3, k, c0, hi, lo, q1);
      if (k > lo) H(k + 1, k - 1) = H(k + 2, k - 1) = 0.0;
      x = H(k + 1, k);
      y = H(k + 2, k);
      if (k < hi - 2) z = H(k + 3, k);
    }
    double u[3];
    householder_vec(x, y, 0.0, 2, u);
    reflect(H, u, 2, hi - 1, hi - 2, hi, lo, hi);
    H(hi, hi - 2) = 0.0;
  }
}

// solve (H - mu I) x = b for upper Hessenberg H by LU with partial pivoting
void hess_solve(const Mat& H, double mu, std::vector<double>& x, double tiny) {
  const int n = H.n;
  Mat U(n);
  for (int i = 0; i < n; ++i)
    for (int j = std::max(0, i - 1); j < n; ++j) U(i, j) = H(i, j) - (i == j ? mu : 0.0);
  // eliminate subdiagonal with row swaps; apply to x
  for (int k = 0; k < n - 1; ++k) {
    if (std::fabs(U(k + 1, k)) > std::fabs(U(k, k))) {
      for (int j = k; j < n; ++j) std::swap(U(k, j), U(k + 1, j));
      std::swap(x[k], x[k + 1]);
    }
    double piv = U(k, k);
    if (piv == 0.0) piv = U(k, k) = tiny;
    double l = U(k + 1, k) / piv;
    U(k + 1, k) = 0.0;
    for (int j = k + 1; j < n; ++j) U(k + 1, j) -= l * U(k, j);
    x[k + 1] -= l * x[k];
  }
  if (U(n - 1, n - 1) == 0.0) U(n - 1, n - 1) = tiny;
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int j = i + 1; j < n; ++j) s -= U(i, j) * x[j];
    x[i] = s / U(i, i);
  }
}

// dense inverse by LU with partial pivoting
std::vector<double> invert(const std::vector<double>& M, int n) {
  std::vector<double> a = M, inv((size_t)n * n, 0.0);
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(a[(size_t)i * n + k]) > std::fabs(a[(size_t)p * n + k])) p = i;
    if (a[(size_t)p * n + k] == 0.0) throw std::runtime_error("CmDz2Decomposition > singular eigenvector matrix");
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)p * n + j], a[(size_t)k * n + j]);
      std::swap(perm[p], perm[k]);
    }
    for (int i = k + 1; i < n; ++i) {
      double l = a[(size_t)i * n + k] / a[(size_t)k * n + k];
      a[(size_t)i * n + k] = l;
      for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
    }
  }
  for (int c = 0; c < n; ++c) {
    std::vector<double> x(n);
    for (int i = 0; i < n; ++i) x[i] = (perm[i] == c) ? 1.0 : 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < i; ++j) x[i] -= a[(size_t)i * n + j] * x[j];
    for (int i = n - 1; i >= 0; --i) {
      for (int j = i + 1; j < n; ++j) x[i] -= a[(size_t)i * n + j] * x[j];
      x[i] /= a[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + c] = x[i];
  }
  return inv;
}

}  // namespace

void real_eigen(const std::vector<double>& F, int n, std::vector<double>& lam, std::vector<double>& V,
                std::vector<double>& Vinv) {
  Mat A(n);
  A.a = F;
  std::vector<double> d = balance(A);
  Mat H = A;
  Mat Q = hessenberg(H);
  std::vector<double> wr, wi;
  hessenberg_qr(H, wr, wi);
  double hnorm = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = std::max(0, i - 1); j < n; ++j) hnorm = std::max(hnorm, std::fabs(H(i, j)));
  for (int i = 0; i < n; ++i)
    if (wi[i] != 0.0 && std::fabs(wi[i]) > 1e-8 * std::max(1.0, std::fabs(wr[i])))
      throw std::runtime_error("CmDz2Decomposition > complex eigenvalue in collocation operator");
  lam = wr;
  V.assign((size_t)n * n, 0.0);
  const double eps = 2.220446049250313e-16;
  for (int e = 0; e < n; ++e) {
    const double mu = lam[e] + eps * hnorm * 8.0;
    std::vector<double> x(n);
    for (int i = 0; i < n; ++i) x[i] = 1.0 + 0.01 * std::sin(1.0 + i * 0.7);
    for (int it = 0; it < 3; ++it) {
      hess_solve(H, mu, x, eps * hnorm);
      double nrm = 0.0;
      for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
      nrm = std::sqrt(nrm);
      for (int i = 0; i < n; ++i) x[i] /= nrm;
    }
    // back-transform: v = D Q x, unit 2-norm
    std::vector<double> v(n, 0.0);
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = 0; j < n; ++j) s += Q(i, j) * x[j];
      v[i] = d[i] * s;
    }
    double nrm = 0.0;
    for (int i = 0; i < n; ++i) nrm += v[i] * v[i];
    nrm = std::sqrt(nrm);
    int imax = 0;
    for (int i = 1; i < n; ++i)
      if (std::fabs(v[i]) > std::fabs(v[imax])) imax = i;
    const double sgn = v[imax] < 0 ? -1.0 : 1.0;
    for (int i = 0; i < n; ++i) V[(size_t)i * n + e] = sgn * v[i] / nrm;
  }
  Vinv = invert(V, n);
  // two-sided Rayleigh quotient in extended precision: lam_e = w_e^T F v_e
  for (int e = 0; e < n; ++e) {
    long double acc = 0.0L;
    for (int i = 0; i < n; ++i) {
      long double fv = 0.0L;
      for (int j = 0; j < n; ++j) fv += (long double)F[(size_t)i * n + j] * (long double)V[(size_t)j * n + e];
      acc += (long double)Vinv[(size_t)e * n + i] * fv;
    }
    lam[e] = (double)acc;
  }
}

// F[n-1-i][n-1-j] == F[i][j] to 1e-12 of the largest entry (odd n >= 3)
static bool centro_symmetric(const std::vector<double>& F, int n) {
  if (n < 3 || !(n & 1)) return false;
  double fmax = 0.0, dev = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      fmax = std::max(fmax, std::fabs(F[(size_t)i * n + j]));
      dev = std::max(dev, std::fabs(F[(size_t)(n - 1 - i) * n + (n - 1 - j)] - F[(size_t)i * n + j]));
    }
  return dev <= 1e-12 * fmax;
}

// Eigen-decomposition of a centro-symmetric F (odd n = 2m+1) from its two
// folded halves: even vectors v[k] = v[n-1-k] = u[k] (k < m), v[m] = u[m]
// see Fe = F[i][k] + F[i][n-1-k] (k < m), Fe[i][m] = F[i][m]; odd vectors
// v[k] = -v[n-1-k] = u[k], v[m] = 0 see Fo = F[i][k] - F[i][n-1-k].  Columns
// of V: the m+1 even eigenvectors, then the m odd ones; every eigenvector has
// exact parity, which the split Helmholtz kernels rely on.
static void folded_eigen(const std::vector<double>& F, int n, std::vector<double>& lam, std::vector<double>& V,
                         std::vector<double>& Vinv) {
  const int m = (n - 1) / 2, ne = m + 1, no = m;
  std::vector<double> Fe((size_t)ne * ne), Fo((size_t)no * no);
  for (int i = 0; i < ne; ++i) {
    for (int k = 0; k < m; ++k) Fe[(size_t)i * ne + k] = F[(size_t)i * n + k] + F[(size_t)i * n + (n - 1 - k)];
    Fe[(size_t)i * ne + m] = F[(size_t)i * n + m];
  }
  for (int i = 0; i < no; ++i)
    for (int k = 0; k < m; ++k) Fo[(size_t)i * no + k] = F[(size_t)i * n + k] - F[(size_t)i * n + (n - 1 - k)];
  std::vector<double> le, Ve, Vie, lo, Vo, Vio;
  real_eigen(Fe, ne, le, Ve, Vie);
  real_eigen(Fo, no, lo, Vo, Vio);
  lam = le;
  lam.insert(lam.end(), lo.begin(), lo.end());
  V.assign((size_t)n * n, 0.0);
  Vinv.assign((size_t)n * n, 0.0);
  for (int j = 0; j < ne; ++j) {
    for (int k = 0; k < m; ++k) {
      V[(size_t)k * n + j] = V[(size_t)(n - 1 - k) * n + j] = Ve[(size_t)k * ne + j];
      Vinv[(size_t)j * n + k] = Vinv[(size_t)j * n + (n - 1 - k)] = 0.5 * Vie[(size_t)j * ne + k];
    }
    V[(size_t)m * n + j] = Ve[(size_t)m * ne + j];
    Vinv[(size_t)j * n + m] = Vie[(size_t)j * ne + m];
  }
  for (int j = 0; j < no; ++j) {
    const int c = ne + j;
    for (int k = 0; k < m; ++k) {
      V[(size_t)k * n + c] = Vo[(size_t)k * no + j];
      V[(size_t)(n - 1 - k) * n + c] = -Vo[(size_t)k * no + j];
      Vinv[(size_t)c * n + k] = 0.5 * Vio[(size_t)j * no + k];
      Vinv[(size_t)c * n + (n - 1 - k)] = -0.5 * Vio[(size_t)j * no + k];
    }
  }
}

void build_decomposition(int n, const std::vector<double>& D1, const std::vector<double>& D2, const double* bc,
                         Decomposition& out) {
  out.n = n;
  std::vector<double> A = D2;
  auto a = [&](int i, int j) -> double& { return A[(size_t)i * n + j]; };
  for (int j = 0; j < n; ++j) {
    a(0, j) = bc[1] * D1[j];
    a(n - 1, j) = bc[3] * D1[(size_t)(n - 1) * n + j];
  }
  a(0, 0) += bc[0];
  a(n - 1, n - 1) += bc[2];
  const double a11 = a(0, 0), ann = a(n - 1, n - 1), a1n = a(0, n - 1), an1 = a(n - 1, 0);
  const double den = 1.0 / (an1 * a1n - a11 * ann);
  out.fbb.assign(n, 0.0);
  out.ftb.assign(n, 0.0);
  out.fbf.assign(n, 0.0);
  out.ftf.assign(n, 0.0);
  for (int i = 1; i < n - 1; ++i) {
    out.fbb[i] = (ann * a(0, i) - a1n * a(n - 1, i)) * den;
    out.ftb[i] = (a11 * a(n - 1, i) - an1 * a(0, i)) * den;
    out.fbf[i] = (ann * a(i, 0) - an1 * a(i, n - 1)) * den;
    out.ftf[i] = (a11 * a(i, n - 1) - a1n * a(i, 0)) * den;
  }
  out.fbb[0] = -1 * ann * den;
  out.fbb[n - 1] = +1 * a1n * den;
  out.ftb[0] = +1 * an1 * den;
  out.ftb[n - 1] = -1 * a11 * den;
  const int ni = n - 2;
  std::vector<double> F((size_t)ni * ni);
  for (int iz = 1; iz < n - 1; ++iz)
    for (int ix = 1; ix < n - 1; ++ix)
      F[(size_t)(ix - 1) * ni + (iz - 1)] = a(ix, iz) + a(ix, 0) * out.fbb[iz] + a(ix, n - 1) * out.ftb[iz];
  std::vector<double> lam, V, Vi;
  out.parity = centro_symmetric(F, ni);
  if (out.parity)
    folded_eigen(F, ni, lam, V, Vi);
  else
    real_eigen(F, ni, lam, V, Vi);
  out.E.assign((size_t)n * n, 0.0);
  out.Einv.assign((size_t)n * n, 0.0);
  out.lam.assign(n, 0.0);
  for (int i = 0; i < ni; ++i) {
    out.lam[i + 1] = lam[i];
    for (int j = 0; j < ni; ++j) {
      out.E[(size_t)(i + 1) * n + (j + 1)] = V[(size_t)i * ni + j];
      out.Einv[(size_t)(i + 1) * n + (j + 1)] = Vi[(size_t)i * ni + j];
    }
  }
  out.E[0] = out.E[(size_t)n * n - 1] = 1.0;
  out.Einv[0] = out.Einv[(size_t)n * n - 1] = 1.0;
}

void fold_decomposition(const Decomposition& d, bool pressure, std::vector<double>& Einvf, std::vector<double>& Ef) {
  const int n = d.n;
  Einvf = d.Einv;
  if (pressure) {
    // rows 0, N-1 of the target are zeroed before E^-1 (phase_carrier_flat.cc:966-967)
    for (int i = 0; i < n; ++i) {
      Einvf[(size_t)i * n + 0] = 0.0;
      Einvf[(size_t)i * n + n - 1] = 0.0;
    }
  } else {
    // interior rows += fbf*row0 + ftf*row(N-1) before E^-1: Einv*(I + fbf e0' + ftf eN')
    for (int i = 0; i < n; ++i) {
      double s0 = 0.0, s1 = 0.0;
      for (int k = 0; k < n; ++k) {
        s0 += d.Einv[(size_t)i * n + k] * d.fbf[k];
        s1 += d.Einv[(size_t)i * n + k] * d.ftf[k];
      }
      Einvf[(size_t)i * n + 0] += s0;
      Einvf[(size_t)i * n + n - 1] += s1;
    }
  }
  // row 0 := fbb . y, then row N-1 := ftb . y with the replaced row 0
  Ef = d.E;
  std::vector<double> r0(n, 0.0), rn(n, 0.0);
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += d.fbb[k] * d.E[(size_t)k * n + j];
    r0[j] = s;
  }
  for (int j = 0; j < n; ++j) {
    double s = d.ftb[0] * r0[j];
    for (int k = 1; k < n; ++k) s += d.ftb[k] * d.E[(size_t)k * n + j];
    rn[j] = s;
  }
  for (int j = 0; j < n; ++j) {
    Ef[j] = r0[j];
    Ef[(size_t)(n - 1) * n + j] = rn[j];
  }
}

bool split_operators(const Decomposition& d, bool pressure, std::vector<double>& Einvs, std::vector<double>& Es,
                     double& quirk) {
  const int n = d.n;
  if (!d.parity || n < 5 || !(n & 1)) return false;
  // the quirk x[n-1] += ftb[0] (x[0] - y[0]) reduces to ftb[0] x[0] only when
  // y[0] == 0, i.e. for the pressure (boundary rows zeroed before E^-1)
  if (!pressure && d.ftb[0] != 0.0) return false;
  quirk = pressure ? d.ftb[0] : 0.0;
  const int h = (n - 1) / 2;
  std::vector<double> Ei, Ef;
  fold_decomposition(d, pressure, Ei, Ef);
  for (int j = 0; j < n; ++j) {  // row N-1 := ftb . E with E's own row 0 (the quirk is applied by the kernel)
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += d.ftb[k] * d.E[(size_t)k * n + j];
    Ef[(size_t)(n - 1) * n + j] = s;
  }
  Einvs = Ei;
  Es = Ef;
  for (int j = 0; j < n; ++j) {
    const double r0 = Ei[j], rn = Ei[(size_t)(n - 1) * n + j];
    Einvs[j] = r0 + rn;
    Einvs[(size_t)(n - 1) * n + j] = r0 - rn;
    const double c0 = Ef[(size_t)j * n], cn = Ef[(size_t)j * n + n - 1];
    Es[(size_t)j * n] = 0.5 * (c0 + cn);
    Es[(size_t)j * n + n - 1] = 0.5 * (c0 - cn);
  }
  if (pressure)  // y'0 = y'N = 0 (rows 0, N-1 of Einvs vanish): the boundary columns multiply zeros
    for (int i = 0; i < n; ++i) Es[(size_t)i * n] = Es[(size_t)i * n + n - 1] = 0.0;
  // parity of the rows of Einvs and of the columns of Es (even block 0..h)
  double ai = 0.0, ae = 0.0, di = 0.0, de = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const double sg = (i <= h) ? 1.0 : -1.0, sc = (j <= h) ? 1.0 : -1.0;
      ai = std::max(ai, std::fabs(Einvs[(size_t)i * n + j]));
      ae = std::max(ae, std::fabs(Es[(size_t)i * n + j]));
      di = std::max(di, std::fabs(Einvs[(size_t)i * n + (n - 1 - j)] - sg * Einvs[(size_t)i * n + j]));
      de = std::max(de, std::fabs(Es[(size_t)(n - 1 - i) * n + j] - sc * Es[(size_t)i * n + j]));
    }
  return di <= 1e-11 * ai && de <= 1e-11 * ae;
}

}  // namespace tg
