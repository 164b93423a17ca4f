// Test and baseline infrastructure only: the reference's own GPU HMVM
// (src_hmvm/src_cpp/hmvm_cuda2.cu, the "hybrid2" kernels) built unchanged for
// sm_100a, as a same-box GPU reference point.
//
// This translation unit is compiled by oracle/Makefile with the reference's
// src_hmvm/src_cpp directory on the include path and includes hmvm_cuda2.cu
// unchanged.  Two entry points:
//
//   refgpu_cuda2_bench   the reference's own host wrapper hmvm_cuda2<T>(mat2,
//                        b, kernel, 0, nbench) (hmvm_cuda2.cu:312-446): it
//                        uploads the matrix, splits the leaves, runs the
//                        kernel 5 + nbench times and prints "TIME <n> <name>
//                        min max avg" (kernel launch + synchronize, timed with
//                        omp_get_wtime, the first 5 runs discarded,
//                        hmvm_cuda2.cu:236-302); that output goes to out_path.
//   refgpu_hybrid2_y     one launch of the same kernel
//                        hmvm_cuda_hybrid2<T,div> with the launch shape of the
//                        wrapper (napprox + ndense blocks of 32*mul threads,
//                        ktmax*sizeof(T) shared bytes), returning y in full
//                        precision (the wrapper only writes it at %.3E).
//
// The matrix comes from the CPU harness (oracle/ref_harness.cpp:
// ref_matrix2_d / ref_matrix2_f).  Nothing in the product links this library.

#include <unistd.h>

#include <cstdio>
#include <vector>

#include "hmvm_cuda2.cu"

namespace {

template <class T>
int hybrid2_y(matrix2<T>* m, const T* x, int div, int mul, int a2t, int a2i, int aa, int da, T* y) {
  const int nlf = m->nlf, nd = m->nd;
  const size_t len = (size_t)m->len;
  std::vector<int> approx, dense;
  for (int ip = 0; ip < nlf; ip++) (m->ltmtx[ip] == 1 ? approx : dense).push_back(ip);
  int *d_ltmtx, *d_ndt, *d_ndl, *d_nstrtl, *d_nstrtt, *d_kt, *d_a1, *d_a2, *d_approx, *d_dense;
  T *d_rowmat, *d_rowmat_t, *d_x, *d_y;
  int* const* ints[] = {&d_ltmtx, &d_ndt, &d_ndl, &d_nstrtl, &d_nstrtt, &d_kt, &d_a1, &d_a2};
  const int* srcs[] = {m->ltmtx, m->ndt, m->ndl, m->nstrtl, m->nstrtt, m->kt, m->a1, m->a2};
  for (int k = 0; k < 8; k++) {
    if (cudaMalloc((void**)ints[k], sizeof(int) * (nlf > 0 ? nlf : 1)) != cudaSuccess) return -1;
    cudaMemcpy(*ints[k], srcs[k], sizeof(int) * nlf, cudaMemcpyHostToDevice);
  }
  if (cudaMalloc((void**)&d_approx, sizeof(int) * (approx.size() + 1)) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&d_dense, sizeof(int) * (dense.size() + 1)) != cudaSuccess) return -1;
  cudaMemcpy(d_approx, approx.data(), sizeof(int) * approx.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(d_dense, dense.data(), sizeof(int) * dense.size(), cudaMemcpyHostToDevice);
  if (cudaMalloc((void**)&d_rowmat, sizeof(T) * len) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&d_rowmat_t, sizeof(T) * len) != cudaSuccess) return -1;
  cudaMemcpy(d_rowmat, m->rowmat, sizeof(T) * len, cudaMemcpyHostToDevice);
  cudaMemcpy(d_rowmat_t, m->rowmat_t, sizeof(T) * len, cudaMemcpyHostToDevice);
  if (cudaMalloc((void**)&d_x, sizeof(T) * nd) != cudaSuccess) return -1;
  if (cudaMalloc((void**)&d_y, sizeof(T) * nd) != cudaSuccess) return -1;
  cudaMemcpy(d_x, x, sizeof(T) * nd, cudaMemcpyHostToDevice);
  cudaMemset(d_y, 0, sizeof(T) * nd);
  const int blocks = (int)(approx.size() + dense.size()), threads = 32 * mul, shms = m->ktmax * (int)sizeof(T);
#define HYB2_LAUNCH(D)                                                                                             \
  hmvm_cuda_hybrid2<T, D><<<blocks, threads, shms>>>(d_y, d_x, nlf, m->ktmax, d_ltmtx, d_ndt, d_ndl, d_nstrtl,     \
                                                     d_nstrtt, d_kt, d_a1, d_a2, d_rowmat, d_rowmat_t,             \
                                                     (int)approx.size(), d_approx, (int)dense.size(), d_dense, mul, \
                                                     a2t, a2i, aa, da)
  switch (div) {
    case 1: HYB2_LAUNCH(1); break;
    case 2: HYB2_LAUNCH(2); break;
    case 4: HYB2_LAUNCH(4); break;
    case 8: HYB2_LAUNCH(8); break;
    case 16: HYB2_LAUNCH(16); break;
    default: HYB2_LAUNCH(32); break;
  }
#undef HYB2_LAUNCH
  const cudaError_t e = cudaDeviceSynchronize();
  cudaMemcpy(y, d_y, sizeof(T) * nd, cudaMemcpyDeviceToHost);
  for (int k = 0; k < 8; k++) cudaFree(*ints[k]);
  cudaFree(d_approx);
  cudaFree(d_dense);
  cudaFree(d_rowmat);
  cudaFree(d_rowmat_t);
  cudaFree(d_x);
  cudaFree(d_y);
  return e == cudaSuccess ? 0 : -2;
}

}  // namespace

extern "C" {

int refgpu_cuda2_bench(void* mat2, int is_float, const void* x, int kernel, int nbench, const char* out_path) {
  FILE* f = fopen(out_path, "w");
  if (!f) return -1;
  fflush(stdout);
  const int saved = dup(1);
  dup2(fileno(f), 1);
  if (is_float)
    hmvm_cuda2<float>(static_cast<matrix2<float>*>(mat2), (float*)x, kernel, 0, nbench);
  else
    hmvm_cuda2<double>(static_cast<matrix2<double>*>(mat2), (double*)x, kernel, 0, nbench);
  fflush(stdout);
  dup2(saved, 1);
  close(saved);
  fclose(f);
  return 0;
}

int refgpu_hybrid2_y(void* mat2, int is_float, const void* x, int div, int mul, int a2t, int a2i, int aa, int da,
                     void* y) {
  if (is_float)
    return hybrid2_y<float>(static_cast<matrix2<float>*>(mat2), static_cast<const float*>(x), div, mul, a2t, a2i,
                            aa, da, static_cast<float*>(y));
  return hybrid2_y<double>(static_cast<matrix2<double>*>(mat2), static_cast<const double*>(x), div, mul, a2t, a2i,
                           aa, da, static_cast<double*>(y));
}

}  // extern "C"
