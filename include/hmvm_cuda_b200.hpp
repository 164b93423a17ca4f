// hmvm_cuda_b200.hpp -- C++ drop-in for the reference harness's CUDA entry
// points, over the C ABI of hmvm_b200.h.
//
// Include it after the reference's hacapk.h (it needs the matrix<T> /
// matrix2<T> templates of src_hmvm/src_cpp/hacapk.h:5-36).  It provides
//
//   template <class T> void hmvm_cuda0..3(matrix2<T>* mat2, T* b, int kernel,
//                                          int dump_result, int nbench);
//     the signatures of src_hmvm/src_cpp/hmvm_cuda.h:4-7.  Every variant runs the
//     same B200 kernels (the reference's `kernel` selects a thread mapping that
//     has no meaning here; it only names the outputs).  With dump_result the
//     result goes to result_cuda<N>_b200_k<kernel>_<d|f>.txt at %.3E
//     (hmvm_cuda2.cu:285-290); with nbench>0 a line
//     "TIME <nbench> hmvm_cuda<N>_b200_k<kernel>_<d|f> min .. max .. avg .." is
//     printed over nbench runs after 5 untimed ones (hmvm_cuda2.cu:234-302),
//     timed with CUDA events around the kernels only, like the reference.
//     Errors are printed and the call returns; it never exits the process.
//
//   With HMVM_B200_DEFINE_LOADERS defined in exactly one translation unit:
//   loadHmatrix / loadHmatrix2 / convertD2F with the signatures of
//   src_hmvm/src_cpp/hacapk.h:39-41, replacing loadmatrix.cpp (return 0 on
//   success, -1 on failure as the reference does).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <typeinfo>
#include <vector>

#include "hmvm_b200.h"

namespace hmvm_b200_detail {

template <class T>
struct Abi;
template <>
struct Abi<double> {
  using M2 = hmvm_matrix2_d;
  static int create(matrix2<double>* m, hmvm_plan** p) {
    return hmvm_b200_plan_create_d(reinterpret_cast<const M2*>(m), nullptr, p);
  }
  static const char* tag() { return "d"; }
};
template <>
struct Abi<float> {
  using M2 = hmvm_matrix2_f;
  static int create(matrix2<float>* m, hmvm_plan** p) {
    return hmvm_b200_plan_create_f(reinterpret_cast<const M2*>(m), nullptr, p);
  }
  static const char* tag() { return "f"; }
};

// The reference structures and the C-ABI ones must be the same bytes.
static_assert(sizeof(matrix2<double>) == sizeof(hmvm_matrix2_d), "matrix2<double> layout");
static_assert(sizeof(matrix2<float>) == sizeof(hmvm_matrix2_f), "matrix2<float> layout");
static_assert(offsetof(matrix2<double>, rowmat) == offsetof(hmvm_matrix2_d, rowmat), "matrix2 rowmat offset");
static_assert(offsetof(matrix2<double>, dense) == offsetof(hmvm_matrix2_d, dense), "matrix2 tail offset");
static_assert(sizeof(matrix<double>) == sizeof(hmvm_matrix_d), "matrix<double> layout");
static_assert(sizeof(submatrix<double>) == sizeof(hmvm_submatrix_d), "submatrix<double> layout");

inline void report(int rc, const char* where) {
  std::printf("%s failed: %s: %s\n", where, hmvm_b200_strerror(rc), hmvm_b200_last_error());
}

template <class T>
void run(int which, matrix2<T>* mat2, T* b, int kernel, int dump_result, int nbench) {
  char name[128];
  std::snprintf(name, sizeof name, "cuda%d_b200_k%d_%s", which, kernel, Abi<T>::tag());
  hmvm_plan* plan = nullptr;
  int rc = Abi<T>::create(mat2, &plan);
  if (rc) {
    report(rc, name);
    return;
  }
  const int nd = mat2->nd;
  std::vector<T> v(nd > 0 ? nd : 1);
  T *d_b = nullptr, *d_v = nullptr;
  if (cudaMalloc(&d_b, sizeof(T) * (nd > 0 ? nd : 1)) != cudaSuccess ||
      cudaMalloc(&d_v, sizeof(T) * (nd > 0 ? nd : 1)) != cudaSuccess) {
    std::printf("%s failed: device allocation\n", name);
    cudaFree(d_b);
    hmvm_b200_plan_destroy(plan);
    return;
  }
  cudaMemcpy(d_b, b, sizeof(T) * nd, cudaMemcpyHostToDevice);
  if (dump_result) {
    rc = hmvm_b200_apply(plan, d_b, d_v, nullptr);
    if (!rc && cudaMemcpy(v.data(), d_v, sizeof(T) * nd, cudaMemcpyDeviceToHost) != cudaSuccess) rc = HMVM_ECUDA;
    if (rc) {
      report(rc, name);
    } else {
      char fname[160];
      std::snprintf(fname, sizeof fname, "result_%s.txt", name);
      std::FILE* F = std::fopen(fname, "w");
      if (F) {
        for (int i = 0; i < nd; i++) std::fprintf(F, "%.3E\n", (double)v[i]);
        std::fclose(F);
      }
    }
  }
  if (nbench > 0 && !rc) {
    const int M = 5, L = M + nbench;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double dmin = 9999.99, dmax = 0.0, davg = 0.0;
    for (int l = 0; l < L && !rc; l++) {
      cudaEventRecord(e0, nullptr);
      rc = hmvm_b200_apply(plan, d_b, d_v, nullptr);
      cudaEventRecord(e1, nullptr);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (l >= M) {
        double s = ms * 1e-3;
        davg += s;
        if (dmin > s) dmin = s;
        if (dmax < s) dmax = s;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) report(rc, name);
    else std::printf("TIME %d hmvm_%s min %e max %e avg %e\n", nbench, name, dmin, dmax, davg / nbench);
  }
  cudaFree(d_b);
  cudaFree(d_v);
  hmvm_b200_plan_destroy(plan);
}

}  // namespace hmvm_b200_detail

template <class T>
void hmvm_cuda0(matrix2<T>* mat2, T* b, int kernel, int dump_result, int nbench) {
  hmvm_b200_detail::run<T>(0, mat2, b, kernel, dump_result, nbench);
}
template <class T>
void hmvm_cuda1(matrix2<T>* mat2, T* b, int kernel, int dump_result, int nbench) {
  hmvm_b200_detail::run<T>(1, mat2, b, kernel, dump_result, nbench);
}
template <class T>
void hmvm_cuda2(matrix2<T>* mat2, T* b, int kernel, int dump_result, int nbench) {
  hmvm_b200_detail::run<T>(2, mat2, b, kernel, dump_result, nbench);
}
template <class T>
void hmvm_cuda3(matrix2<T>* mat2, T* b, int kernel, int dump_result, int nbench) {
  hmvm_b200_detail::run<T>(3, mat2, b, kernel, dump_result, nbench);
}

#ifdef HMVM_B200_DEFINE_LOADERS
int loadHmatrix(const char* fname, matrix<double>* mat, matrix2<double>* mat2) {
  int rc = hmvm_b200_load_hmatrix(fname, reinterpret_cast<hmvm_matrix_d*>(mat), reinterpret_cast<hmvm_matrix2_d*>(mat2));
  if (rc) std::printf("loadHmatrix %s: %s\n", fname, hmvm_b200_last_error());
  return rc ? -1 : 0;
}
int loadHmatrix2(const char* fname, matrix2<double>* mat2) {
  int rc = hmvm_b200_load_hmatrix2(fname, reinterpret_cast<hmvm_matrix2_d*>(mat2));
  if (rc) std::printf("loadHmatrix2 %s: %s\n", fname, hmvm_b200_last_error());
  return rc ? -1 : 0;
}
int convertD2F(matrix<float>* matF, matrix2<float>* matF2, const matrix<double>* matD, const matrix2<double>* matD2) {
  int rc = hmvm_b200_convert_d2f(reinterpret_cast<hmvm_matrix_f*>(matF), reinterpret_cast<hmvm_matrix2_f*>(matF2),
                                 reinterpret_cast<const hmvm_matrix_d*>(matD),
                                 reinterpret_cast<const hmvm_matrix2_d*>(matD2));
  return rc ? -1 : 0;
}
#endif
