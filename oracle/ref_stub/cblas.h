/* Stand-in for the CBLAS declarations that the reference's MatrixMulBLAS.hpp
 * includes, so that its Distance.hpp compiles unmodified into oracle/_ref
 * (no BLAS library is installed here).  The oracle binds only Distance.hpp's
 * vectorSetDistance, which calls no BLAS routine; each stand-in aborts if it
 * is ever reached, and none computes anything. */
#pragma once
#include <cstdlib>
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
inline float cblas_sdot(int, const float *, int, const float *, int) { std::abort(); }
inline void cblas_sgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int, int, float, const float *, int,
                        const float *, int, float, float *, int) { std::abort(); }
inline void cblas_sgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, float,
                        const float *, int, const float *, int, float, float *, int) {
  std::abort();
}
inline void cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int, double,
                        const double *, int, const double *, int, double, double *, int) {
  std::abort();
}
