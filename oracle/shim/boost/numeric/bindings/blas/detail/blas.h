// ORACLE shim (test infrastructure): Fortran BLAS entry points used by the
// reference's gemm/axpy templates, bound to the scipy-bundled OpenBLAS.
#pragma once
#include <complex>
typedef int fortran_int_t;
extern "C" {
void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                  const int*, const double*, const int*, const double*, double*, const int*);
void scipy_sgemm_(const char*, const char*, const int*, const int*, const int*, const float*, const float*,
                  const int*, const float*, const int*, const float*, float*, const int*);
void scipy_zgemm_(const char*, const char*, const int*, const int*, const int*, const void*, const void*,
                  const int*, const void*, const int*, const void*, void*, const int*);
void scipy_cgemm_(const char*, const char*, const int*, const int*, const int*, const void*, const void*,
                  const int*, const void*, const int*, const void*, void*, const int*);
void scipy_daxpy_(const int*, const double*, const double*, const int*, double*, const int*);
void scipy_saxpy_(const int*, const float*, const float*, const int*, float*, const int*);
void scipy_zaxpy_(const int*, const void*, const void*, const int*, void*, const int*);
void scipy_caxpy_(const int*, const void*, const void*, const int*, void*, const int*);
}
#define BLAS_DGEMM scipy_dgemm_
#define BLAS_SGEMM scipy_sgemm_
#define BLAS_ZGEMM scipy_zgemm_
#define BLAS_CGEMM scipy_cgemm_
#define BLAS_DAXPY scipy_daxpy_
#define BLAS_SAXPY scipy_saxpy_
#define BLAS_ZAXPY scipy_zaxpy_
#define BLAS_CAXPY scipy_caxpy_
