#pragma once
#include <vector>

namespace edk {

// lowest m eigenvalues (ascending) of the symmetric tridiagonal (d[n], e[n-1])
void tridiag_lowest(int n, const double *d, const double *e, int m, double *w);
// unit eigenvector for eigenvalue lambda, orthogonal to nprev earlier vectors (n each)
void tridiag_vector(int n, const double *d, const double *e, double lambda, const double *prev,
                    int nprev, double *v);
// all eigenpairs of a dense symmetric matrix (row-major); V column j = vector j
void dense_eigh(int n, std::vector<double> A, std::vector<double> &w, std::vector<double> &V);
// lowest m eigenpairs of a dense symmetric matrix (row-major): Householder
// reduction to tridiagonal, Sturm bisection, inverse iteration, back
// transformation.  V (n x m, column j = vector j), w ascending.
void dense_lowest(int n, std::vector<double> A, int m, std::vector<double> &w, std::vector<double> &V);

}  // namespace edk
