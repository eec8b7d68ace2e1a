#include "quadrature.hpp"

#include <cmath>
#include <stdexcept>

namespace sfb {

double legendre(double z, int n) {
  double p0 = 1.0, p1 = z;
  if (n == 0) return 1.0;
  for (int k = 1; k < n; ++k) {
    const double p2 = ((2.0 * k + 1.0) * z * p1 - k * p0) / (k + 1.0);
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

double legendre_deriv(double z, int n) {
  if (n == 0) return 0.0;
  double p0 = 1.0, p1 = z, d0 = 0.0, d1 = 1.0;
  for (int k = 1; k < n; ++k) {
    const double p2 = ((2.0 * k + 1.0) * z * p1 - k * p0) / (k + 1.0);
    const double d2 = ((2.0 * k + 1.0) * (p1 + z * d1) - k * d0) / (k + 1.0);
    p0 = p1;
    p1 = p2;
    d0 = d1;
    d1 = d2;
  }
  return d1;
}

Quadrature::Quadrature(int n) : ngll(n), xi(n), w(n), hprime(n * n) {
  if (n < 3) throw std::invalid_argument("GLL quadrature needs >= 3 points");
  const int N = n - 1;  // polynomial degree
  // Interior points are the roots of P_N'(x).  Newton iteration on P_N' from
  // Chebyshev-Gauss-Lobatto starting guesses; P_N'' follows from the Legendre
  // ODE: (1 - x^2) P'' = 2x P' - N(N+1) P.
  xi[0] = -1.0;
  xi[N] = 1.0;
  for (int i = 1; i < N; ++i) {
    double x = -std::cos(M_PI * i / N);
    for (int it = 0; it < 100; ++it) {
      const double p = legendre(x, N);
      const double dp = legendre_deriv(x, N);
      const double d2p = (2.0 * x * dp - N * (N + 1.0) * p) / (1.0 - x * x);
      const double dx = dp / d2p;
      x -= dx;
      if (std::abs(dx) < 1e-16) break;
    }
    xi[i] = x;
  }
  if (n % 2 == 1) xi[N / 2] = 0.0;  // symmetric rule: exact centre point
  for (int i = 0; i < n; ++i) {
    const double p = legendre(xi[i], N);
    w[i] = 2.0 / (N * (N + 1.0) * p * p);
  }
  // hprime(i, j) = l_j'(xi_i) (derivative of the j-th basis function at the
  // i-th point), the standard closed form for the GLL nodal basis.
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      double v;
      if (i == 0 && j == 0) {
        v = -0.25 * N * (N + 1.0);
      } else if (i == N && j == N) {
        v = 0.25 * N * (N + 1.0);
      } else if (i == j) {
        v = 0.0;
      } else {
        v = legendre(xi[i], N) / (legendre(xi[j], N) * (xi[i] - xi[j]));
      }
      hprime[i * n + j] = v;
    }
  }
}

void lagrange_interpolants(const Quadrature &q, double x, double *h,
                           double *hp) {
  const int n = q.ngll;
  for (int k = 0; k < n; ++k) {
    double num = 1.0, den = 1.0, dsum = 0.0;
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      num *= (x - q.xi[i]);
      den *= (q.xi[k] - q.xi[i]);
      double prod = 1.0;
      for (int j = 0; j < n; ++j)
        if (j != k && j != i) prod *= (x - q.xi[j]);
      dsum += prod;
    }
    h[k] = num / den;
    if (hp) hp[k] = dsum / den;
  }
}

}  // namespace sfb
