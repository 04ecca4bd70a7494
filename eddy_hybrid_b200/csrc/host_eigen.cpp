// host_eigen.cpp -- eigen-decomposition of the symmetrised stretched-grid
// operator used by the Poisson plan: implicit symmetric tridiagonal QR with
// Wilkinson shifts and Givens bulge chasing (Golub & Van Loan, "Matrix
// Computations", the symmetric QR algorithm for tridiagonal matrices),
// accumulating the eigenvectors.
#include <cmath>
#include <vector>

#include "eddy_internal.h"

// d: diagonal (n), e: off-diagonal (n-1); on return d holds the eigenvalues
// and q (n*n, row-major, q[i*n+m] = component i of eigenvector m).
int tridiag_eigen(int n, std::vector<double> &d, std::vector<double> &e, std::vector<double> &q) {
  q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) q[(size_t)i * n + i] = 1.0;
  if (n == 1) return 0;
  e.resize(n - 1);
  const double eps = 2.220446049250313e-16;
  int m = n - 1;
  long iters = 0, maxit = 60L * n;
  while (m > 0) {
    // deflate converged trailing entries
    if (std::fabs(e[m - 1]) <= eps * (std::fabs(d[m - 1]) + std::fabs(d[m]))) {
      e[m - 1] = 0.0;
      m--;
      continue;
    }
    // start of the unreduced block ending at m
    int l = m - 1;
    while (l > 0 && std::fabs(e[l - 1]) > eps * (std::fabs(d[l - 1]) + std::fabs(d[l]))) l--;
    if (l > 0) e[l - 1] = 0.0;
    if (++iters > maxit) return -1;
    // Wilkinson shift from the trailing 2x2 of the block
    double delta = 0.5 * (d[m - 1] - d[m]);
    double b2 = e[m - 1] * e[m - 1];
    double sg = delta >= 0.0 ? 1.0 : -1.0;
    double mu = d[m] - b2 / (delta + sg * std::sqrt(delta * delta + b2));
    double x = d[l] - mu, z = e[l];
    for (int k = l; k < m; k++) {
      double r = std::hypot(x, z);
      double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : z / r;
      if (k > l) e[k - 1] = r;
      double dk = d[k], dk1 = d[k + 1], ek = e[k];
      d[k] = c * c * dk + 2.0 * c * s * ek + s * s * dk1;
      d[k + 1] = s * s * dk - 2.0 * c * s * ek + c * c * dk1;
      e[k] = c * s * (dk1 - dk) + (c * c - s * s) * ek;
      if (k < m - 1) {
        x = e[k];
        z = s * e[k + 1];
        e[k + 1] = c * e[k + 1];
      }
      for (int i = 0; i < n; i++) {
        double a = q[(size_t)i * n + k], b = q[(size_t)i * n + k + 1];
        q[(size_t)i * n + k] = c * a + s * b;
        q[(size_t)i * n + k + 1] = -s * a + c * b;
      }
    }
  }
  return 0;
}
