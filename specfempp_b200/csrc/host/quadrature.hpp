// Gauss-Lobatto-Legendre quadrature on [-1, 1]: points, weights, the
// derivative matrix of the Lagrange basis and Lagrange interpolants at an
// arbitrary point.  All set-up arithmetic is FP64; the solver stores FP32
// copies.
//
// Reference behaviour restated (SPECFEM++):
//   src/quadrature/gll/gll.cpp:59-65        points/weights then derivatives
//   src/quadrature/gll/gll_library.cpp:133  zwgljd (GLL points and weights)
//   src/quadrature/gll/lagrange_poly.cpp:159-193  hprime(i, j) = l_j'(xi_i)
//   src/quadrature/gll/lagrange_poly.cpp:128-157  Lagrange interpolants at xi
#pragma once
#include <vector>

namespace sfb {

struct Quadrature {
  int ngll = 0;
  std::vector<double> xi;      // [ngll] GLL points, xi[0] = -1, xi[n-1] = +1
  std::vector<double> w;       // [ngll] GLL weights
  std::vector<double> hprime;  // [ngll*ngll] hprime[i*ngll + j] = l_j'(xi_i)

  explicit Quadrature(int ngll);
  Quadrature() = default;
};

// Legendre polynomial P_n(z) and its derivative, three-term recurrence.
double legendre(double z, int n);
double legendre_deriv(double z, int n);

// Lagrange interpolants h_k(x) and derivatives h_k'(x) through the GLL points.
void lagrange_interpolants(const Quadrature &q, double x, double *h,
                           double *hprime);

}  // namespace sfb
