// A driver in the shape of the reference's src_hmvm/src_cpp/hmvm1.cpp
// (argv: file [dump(0,1) nbench]) that reaches the B200 library only through
// the reference-shaped C++ entry points of hmvm_cuda_b200.hpp.  It loads the
// file with loadHmatrix, builds b[i] = sin(i+1), runs hmvm_cuda2<double>, then
// convertD2F and hmvm_cuda2<float>, and (extra) writes the FP64 result as raw
// doubles to result_raw_d.bin so tests can compare it exactly.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "hacapk.h"
#define HMVM_B200_DEFINE_LOADERS
#include "hmvm_cuda_b200.hpp"

int main(int argc, char **argv) {
  int dump_result = 0, nbench = 5;
  if (argc < 2) {
    printf("usage: %s filename [dump(0,1) nbench]\n", argv[0]);
    return -1;
  }
  if (argc >= 3) dump_result = atoi(argv[2]);
  if (argc >= 4) nbench = atoi(argv[3]);
  matrix<double> *matD = new matrix<double>();
  matrix2<double> *matD2 = new matrix2<double>();
  if (loadHmatrix(argv[1], matD, matD2)) return -1;
  int nd = matD->nd;
  double *b = new double[nd];
  for (int i = 0; i < nd; i++) b[i] = sin((double)(i + 1));
  hmvm_cuda2<double>(matD2, b, 0, dump_result, nbench);
  {
    // raw FP64 result through the C ABI, for exact comparison
    std::vector<double> y(nd);
    hmvm_stats st;
    if (hmvm_cuda_d(reinterpret_cast<hmvm_matrix2_d *>(matD2), b, y.data(), 0, &st) == 0) {
      FILE *F = fopen("result_raw_d.bin", "wb");
      fwrite(y.data(), sizeof(double), nd, F);
      fclose(F);
    }
  }
  matrix<float> *matF = new matrix<float>();
  matrix2<float> *matF2 = new matrix2<float>();
  float *fb = new float[nd];
  for (int i = 0; i < nd; i++) fb[i] = sinf((float)(i + 1));
  convertD2F(matF, matF2, matD, matD2);
  hmvm_cuda2<float>(matF2, fb, 0, dump_result, nbench);
  delete[] b;
  delete[] fb;
  hmvm_b200_free_matrix_d(reinterpret_cast<hmvm_matrix_d *>(matD));
  hmvm_b200_free_matrix2_d(reinterpret_cast<hmvm_matrix2_d *>(matD2));
  hmvm_b200_free_matrix_f(reinterpret_cast<hmvm_matrix_f *>(matF));
  hmvm_b200_free_matrix2_f(reinterpret_cast<hmvm_matrix2_f *>(matF2));
  delete matD; delete matD2; delete matF; delete matF2;
  return 0;
}
