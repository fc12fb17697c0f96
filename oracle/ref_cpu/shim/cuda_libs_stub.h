// Declarations standing in for cuSPARSE, cuSOLVER, cuBLAS and cuRAND, used
// ONLY to compile include/solver/gnSolver/gnSolver.cu for the CPU (test
// infrastructure).  Its sparse-solver and vector-sum helpers name these
// libraries; the drivers here never call them, and every function aborts.
#pragma once
#include <cstdio>
#include <cstdlib>

namespace dynref_libs {
inline int unavailable(const char* f) {
  std::fprintf(stderr, "cuda library shim: %s is not provided\n", f);
  std::abort();
}
}  // namespace dynref_libs

typedef void* cusparseHandle_t;
typedef void* cusparseMatDescr_t;
typedef void* cusolverSpHandle_t;
typedef void* cusolverDnHandle_t;
typedef void* cublasHandle_t;
typedef void* curandGenerator_t;
enum { CUSPARSE_MATRIX_TYPE_GENERAL = 0 };
enum { CUSPARSE_INDEX_BASE_ZERO = 0 };
enum { CUSPARSE_DIRECTION_ROW = 0 };
enum { CUBLAS_OP_N = 0, CUBLAS_OP_T = 1 };

template <class... A>
inline int cusparseCreate(A...) { return dynref_libs::unavailable("cusparseCreate"); }
template <class... A>
inline int cusparseCreateMatDescr(A...) { return dynref_libs::unavailable("cusparseCreateMatDescr"); }
template <class... A>
inline int cusparseSetMatType(A...) { return dynref_libs::unavailable("cusparseSetMatType"); }
template <class... A>
inline int cusparseSetMatIndexBase(A...) { return dynref_libs::unavailable("cusparseSetMatIndexBase"); }
template <class... A>
inline int cusparseSnnz(A...) { return dynref_libs::unavailable("cusparseSnnz"); }
template <class... A>
inline int cusparseSdense2csr(A...) { return dynref_libs::unavailable("cusparseSdense2csr"); }
template <class... A>
inline int cusolverSpCreate(A...) { return dynref_libs::unavailable("cusolverSpCreate"); }
template <class... A>
inline int cusolverSpScsrlsvcholHost(A...) {
  return dynref_libs::unavailable("cusolverSpScsrlsvcholHost");
}
template <class... A>
inline int cublasCreate(A...) { return dynref_libs::unavailable("cublasCreate"); }
template <class... A>
inline int cublasDestroy(A...) { return dynref_libs::unavailable("cublasDestroy"); }
template <class... A>
inline int cublasSgeam(A...) { return dynref_libs::unavailable("cublasSgeam"); }
