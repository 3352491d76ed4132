// Minimal LAPACKE declarations for building the reference oracle without a LAPACK install.
// Only dgetrf/dgetri (used by the reference's 5x5 and Vandermonde inverses) do real work;
// the other entry points exist so the reference's LapackInterface.hpp compiles and abort
// if they are ever reached (they are not on the residual-distribution path).
#pragma once
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
extern "C" {
float LAPACKE_slange(int layout, char norm, int m, int n, const float *a, int lda);
double LAPACKE_dlange(int layout, char norm, int m, int n, const double *a, int lda);
int LAPACKE_sgetrf(int layout, int m, int n, float *a, int lda, int *ipiv);
int LAPACKE_dgetrf(int layout, int m, int n, double *a, int lda, int *ipiv);
int LAPACKE_sgetri(int layout, int n, float *a, int lda, const int *ipiv);
int LAPACKE_dgetri(int layout, int n, double *a, int lda, const int *ipiv);
int LAPACKE_sgecon(int layout, char norm, int n, const float *a, int lda, float anorm,
                   float *rcond);
int LAPACKE_dgecon(int layout, char norm, int n, const double *a, int lda, double anorm,
                   double *rcond);
int LAPACKE_sgeev(int layout, char jobvl, char jobvr, int n, float *a, int lda, float *wr,
                  float *wi, float *vl, int ldvl, float *vr, int ldvr);
int LAPACKE_dgeev(int layout, char jobvl, char jobvr, int n, double *a, int lda, double *wr,
                  double *wi, double *vl, int ldvl, double *vr, int ldvr);
}
