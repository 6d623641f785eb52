/* cblas.h -- the few CBLAS entry points the reference's CPU contraction code
 * (src/ML-TENSORMD/cppblas.hpp) calls, as plain loops, so that file compiles
 * here without a system BLAS.  Used only to build oracle/_ref (the checker);
 * nothing in the product links it. */
#ifndef TMD_REF_SHIM_CBLAS_H
#define TMD_REF_SHIM_CBLAS_H

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef CBLAS_ORDER CBLAS_LAYOUT;

#define TMD_SHIM_AXPY(name, T)                                               \
  static inline void name(int n, T alpha, const T *x, int incx, T *y,        \
                          int incy) {                                        \
    for (int i = 0; i < n; i++) y[i * incy] += alpha * x[i * incx];          \
  }
TMD_SHIM_AXPY(cblas_saxpy, float)
TMD_SHIM_AXPY(cblas_daxpy, double)

#define TMD_SHIM_COPY(name, T)                                               \
  static inline void name(int n, const T *x, int incx, T *y, int incy) {    \
    for (int i = 0; i < n; i++) y[i * incy] = x[i * incx];                   \
  }
TMD_SHIM_COPY(cblas_scopy, float)
TMD_SHIM_COPY(cblas_dcopy, double)

#define TMD_SHIM_DOT(name, T)                                                \
  static inline T name(int n, const T *x, int incx, const T *y, int incy) { \
    T s = 0;                                                                 \
    for (int i = 0; i < n; i++) s += x[i * incx] * y[i * incy];              \
    return s;                                                                \
  }
TMD_SHIM_DOT(cblas_sdot, float)
TMD_SHIM_DOT(cblas_ddot, double)

/* C = alpha op(A) op(B) + beta C with the usual CBLAS layout rules. */
#define TMD_SHIM_GEMM(name, T)                                               \
  static inline void name(CBLAS_ORDER order, CBLAS_TRANSPOSE ta,             \
                          CBLAS_TRANSPOSE tb, int M, int N, int K, T alpha,  \
                          const T *A, int lda, const T *B, int ldb, T beta,  \
                          T *C, int ldc) {                                   \
    const int row = order == CblasRowMajor;                                  \
    for (int i = 0; i < M; i++)                                              \
      for (int j = 0; j < N; j++) {                                          \
        T s = 0;                                                             \
        for (int k = 0; k < K; k++) {                                        \
          /* element (i,k) of op(A), (k,j) of op(B) */                       \
          const int ai = ta == CblasNoTrans ? i : k, ak = ta == CblasNoTrans ? k : i; \
          const int bk = tb == CblasNoTrans ? k : j, bj = tb == CblasNoTrans ? j : k; \
          const T a = row ? A[ai * lda + ak] : A[ak * lda + ai];             \
          const T b = row ? B[bk * ldb + bj] : B[bj * ldb + bk];             \
          s += a * b;                                                        \
        }                                                                    \
        T *c = row ? &C[i * ldc + j] : &C[j * ldc + i];                      \
        *c = alpha * s + (beta == 0 ? (T)0 : beta * *c);                     \
      }                                                                      \
  }
TMD_SHIM_GEMM(cblas_sgemm, float)
TMD_SHIM_GEMM(cblas_dgemm, double)

#endif
