// LU factorisation with partial pivoting and inversion from the LU factors, exposed under
// the LAPACKE names the reference calls (math/LapackInterface.hpp, reached from
// math/unary_ops/matrix_unary_ops/MatrixInverse.hpp:87-97 for the 5x5 inverse and from
// mesh/shape_function/ShapeFunction.cpp:51-55 for the Vandermonde inverse).
//
// Test-oracle code: it stands in for netlib LAPACK 3.8.0 (the version pinned by the
// reference's dependency installer), which is not available here. The algorithm is the
// textbook right-looking Gaussian elimination with row partial pivoting (Golub & Van Loan,
// "Matrix Computations", Alg. 3.4.1) followed by inv(A) = inv(U) inv(L) P, computed column
// by column. Results agree with LAPACK to rounding, not bit for bit.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "lapacke.h"

namespace
{

// Element accessor for row- or column-major storage with leading dimension lda.
template <typename T>
inline T &at(T *a, int layout, int lda, int i, int j)
{
  return layout == LAPACK_ROW_MAJOR ? a[i * lda + j] : a[j * lda + i];
}

template <typename T>
int getrf(int layout, int m, int n, T *a, int lda, int *ipiv)
{
  const int kmax = m < n ? m : n;
  int info       = 0;
  for (int k = 0; k < kmax; ++k)
  {
    int p    = k;
    T maxabs = std::fabs(at(a, layout, lda, k, k));
    for (int i = k + 1; i < m; ++i)
    {
      const T v = std::fabs(at(a, layout, lda, i, k));
      if (v > maxabs)
      {
        maxabs = v;
        p      = i;
      }
    }
    ipiv[k] = p + 1; // LAPACK pivots are 1-based
    if (maxabs == T(0))
    {
      if (info == 0)
        info = k + 1;
      continue;
    }
    if (p != k)
    {
      for (int j = 0; j < n; ++j)
      {
        T tmp                    = at(a, layout, lda, k, j);
        at(a, layout, lda, k, j) = at(a, layout, lda, p, j);
        at(a, layout, lda, p, j) = tmp;
      }
    }
    const T inv_piv = T(1) / at(a, layout, lda, k, k);
    for (int i = k + 1; i < m; ++i)
    {
      at(a, layout, lda, i, k) *= inv_piv;
    }
    for (int i = k + 1; i < m; ++i)
    {
      const T lik = at(a, layout, lda, i, k);
      for (int j = k + 1; j < n; ++j)
      {
        at(a, layout, lda, i, j) -= lik * at(a, layout, lda, k, j);
      }
    }
  }
  return info;
}

template <typename T>
int getri(int layout, int n, T *a, int lda, const int *ipiv)
{
  // Solve A X = I column by column using the packed L\U factors and the pivots.
  std::vector<T> lu(static_cast<size_t>(n) * n);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      lu[i * n + j] = at(a, layout, lda, i, j);

  for (int i = 0; i < n; ++i)
    if (lu[i * n + i] == T(0))
      return i + 1;

  std::vector<T> col(n);
  for (int c = 0; c < n; ++c)
  {
    for (int i = 0; i < n; ++i)
      col[i] = (i == c) ? T(1) : T(0);
    // apply the row interchanges in the order they were made
    for (int k = 0; k < n; ++k)
    {
      const int p = ipiv[k] - 1;
      if (p != k)
      {
        T tmp  = col[k];
        col[k] = col[p];
        col[p] = tmp;
      }
    }
    // forward substitution with unit lower L
    for (int i = 1; i < n; ++i)
      for (int k = 0; k < i; ++k)
        col[i] -= lu[i * n + k] * col[k];
    // back substitution with U
    for (int i = n - 1; i >= 0; --i)
    {
      for (int k = i + 1; k < n; ++k)
        col[i] -= lu[i * n + k] * col[k];
      col[i] /= lu[i * n + i];
    }
    for (int i = 0; i < n; ++i)
      at(a, layout, lda, i, c) = col[i];
  }
  return 0;
}

[[noreturn]] void not_on_path(const char *name)
{
  std::fprintf(stderr, "oracle LAPACKE shim: %s is not provided (not on the RDS path)\n", name);
  std::abort();
}

} // namespace

extern "C" {

int LAPACKE_dgetrf(int layout, int m, int n, double *a, int lda, int *ipiv)
{
  return getrf<double>(layout, m, n, a, lda, ipiv);
}

int LAPACKE_sgetrf(int layout, int m, int n, float *a, int lda, int *ipiv)
{
  return getrf<float>(layout, m, n, a, lda, ipiv);
}

int LAPACKE_dgetri(int layout, int n, double *a, int lda, const int *ipiv)
{
  return getri<double>(layout, n, a, lda, ipiv);
}

int LAPACKE_sgetri(int layout, int n, float *a, int lda, const int *ipiv)
{
  return getri<float>(layout, n, a, lda, ipiv);
}

double LAPACKE_dlange(int, char, int, int, const double *, int)
{
  not_on_path("LAPACKE_dlange");
}

float LAPACKE_slange(int, char, int, int, const float *, int)
{
  not_on_path("LAPACKE_slange");
}

int LAPACKE_dgecon(int, char, int, const double *, int, double, double *)
{
  not_on_path("LAPACKE_dgecon");
}

int LAPACKE_sgecon(int, char, int, const float *, int, float, float *)
{
  not_on_path("LAPACKE_sgecon");
}

int LAPACKE_dgeev(int, char, char, int, double *, int, double *, double *, double *, int,
                  double *, int)
{
  not_on_path("LAPACKE_dgeev");
}

int LAPACKE_sgeev(int, char, char, int, float *, int, float *, float *, float *, int, float *,
                  int)
{
  not_on_path("LAPACKE_sgeev");
}
}
