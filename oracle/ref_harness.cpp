// Test infrastructure only: a C-ABI shim over the reference's own HMVM code.
//
// This translation unit is compiled by oracle/Makefile with the reference's
// src_hmvm/src_cpp directory on the include path.  It includes the reference's
// template definition files unchanged (src_hmvm/src_cpp/hmvm_seq.cpp and
// src_hmvm/src_cpp/hmvm_omp.cpp) and links the reference's loadmatrix.cpp, so
// the functions exported below run the reference's own arithmetic:
//
//   hmvm_seq_2<T,a2i>  src_hmvm/src_cpp/hmvm_seq.cpp:154-227  (the FP64 oracle)
//   hmvm_seq_1<T,a2i>  src_hmvm/src_cpp/hmvm_seq.cpp:10-79    (AoS variant)
//   hmvm_omp_2<T,a2i>  src_hmvm/src_cpp/hmvm_omp.cpp:374-463  (the timed CPU baseline)
//   loadHmatrix        src_hmvm/src_cpp/loadmatrix.cpp:7-150
//   loadHmatrix2       src_hmvm/src_cpp/loadmatrix.cpp:152-250
//   convertD2F         src_hmvm/src_cpp/loadmatrix.cpp:252-342
//
// Only tests, the smoke check and bench.py's CPU-baseline leg load the built
// library (oracle/_ref/libhmvm_ref.so).  Nothing in the product links it.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>
#include <unistd.h>

#include "hacapk.h"
#include "hmvm_seq.cpp"
#include "hmvm_omp.cpp"

namespace {

struct RefHandle {
  matrix<double>* matD = nullptr;    // AoS (only filled by loadHmatrix)
  matrix2<double>* matD2 = nullptr;  // SoA
  matrix<float>* matF = nullptr;
  matrix2<float>* matF2 = nullptr;
  bool wrapped = false;              // matD2 points at caller-owned arrays
};

// The reference loaders print progress to stdout; route it to stderr while they
// run so callers that print machine-readable lines on stdout stay clean.
struct StdoutToStderr {
  int saved = -1;
  StdoutToStderr() {
    fflush(stdout);
    saved = dup(1);
    dup2(2, 1);
  }
  ~StdoutToStderr() {
    fflush(stdout);
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};

}  // namespace

extern "C" {

// hmatrix_1.bin -> AoS + SoA (reference loadHmatrix). Returns NULL on failure.
void* ref_load1(const char* fname) {
  StdoutToStderr quiet;
  RefHandle* h = new RefHandle();
  h->matD = new matrix<double>();
  h->matD2 = new matrix2<double>();
  if (loadHmatrix(fname, h->matD, h->matD2) != 0) {
    delete h->matD2;
    delete h->matD;
    delete h;
    return nullptr;
  }
  return h;
}

// hmatrix_2.bin -> SoA (reference loadHmatrix2). Returns NULL on failure.
void* ref_load2(const char* fname) {
  StdoutToStderr quiet;
  RefHandle* h = new RefHandle();
  h->matD2 = new matrix2<double>();
  if (loadHmatrix2(fname, h->matD2) != 0) {
    delete h->matD2;
    delete h;
    return nullptr;
  }
  return h;
}

// Wrap caller-owned SoA arrays (layout of src_hmvm/src_cpp/hacapk.h:23-36) without copying.
void* ref_wrap2(int nd, int nlf, int ktmax, int len, int* ltmtx, int* kt, int* ndl, int* ndt,
                int* nstrtl, int* nstrtt, int* a1, int* a2, double* rowmat) {
  RefHandle* h = new RefHandle();
  h->wrapped = true;
  h->matD2 = new matrix2<double>();
  matrix2<double>* m = h->matD2;
  m->nd = nd;
  m->nlf = nlf;
  m->ktmax = ktmax;
  m->len = len;
  m->nleavs = nullptr;
  m->ltmtx = ltmtx;
  m->kt = kt;
  m->ndl = ndl;
  m->ndt = ndt;
  m->nstrtl = nstrtl;
  m->nstrtt = nstrtt;
  m->a1 = a1;
  m->a2 = a2;
  m->rowmat = rowmat;
  // rowmat_t as the reference loader builds it (loadmatrix.cpp:216-242): the
  // reference's convertD2F copies it, so it must exist.
  m->rowmat_t = (double*)malloc(sizeof(double) * (size_t)(len > 0 ? len : 1));
  for (int i = 0; i < nlf; i++) {
    if (ltmtx[i] == 1) {
      memcpy(&m->rowmat_t[a1[i]], &rowmat[a1[i]], sizeof(double) * (size_t)kt[i] * ndt[i]);
      for (int y = 0; y < kt[i]; y++)
        for (int x = 0; x < ndl[i]; x++)
          m->rowmat_t[a2[i] + y + x * kt[i]] = rowmat[a2[i] + y * ndl[i] + x];
    } else {
      memcpy(&m->rowmat_t[a1[i]], &rowmat[a1[i]], sizeof(double) * (size_t)ndl[i] * ndt[i]);
    }
  }
  m->napprox = 0;
  m->ndense = 0;
  m->approx = nullptr;
  m->dense = nullptr;
  return h;
}

void ref_info(void* hv, int* out4) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  out4[0] = h->matD2->nd;
  out4[1] = h->matD2->nlf;
  out4[2] = h->matD2->ktmax;
  out4[3] = h->matD2->len;
}

// Copy the SoA view out (arrays must have room for nlf ints / len doubles).
void ref_export2(void* hv, int* ltmtx, int* kt, int* ndl, int* ndt, int* nstrtl, int* nstrtt,
                 int* a1, int* a2, double* rowmat) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  matrix2<double>* m = h->matD2;
  size_t n = (size_t)m->nlf;
  memcpy(ltmtx, m->ltmtx, n * sizeof(int));
  memcpy(kt, m->kt, n * sizeof(int));
  memcpy(ndl, m->ndl, n * sizeof(int));
  memcpy(ndt, m->ndt, n * sizeof(int));
  memcpy(nstrtl, m->nstrtl, n * sizeof(int));
  memcpy(nstrtt, m->nstrtt, n * sizeof(int));
  memcpy(a1, m->a1, n * sizeof(int));
  memcpy(a2, m->a2, n * sizeof(int));
  memcpy(rowmat, m->rowmat, (size_t)m->len * sizeof(double));
}

// convertD2F on the SoA part (and the AoS part when present).
int ref_make_float(void* hv) {
  StdoutToStderr quiet;
  RefHandle* h = static_cast<RefHandle*>(hv);
  if (h->matF2) return 0;
  h->matF2 = new matrix2<float>();
  if (h->matD) h->matF = new matrix<float>();
  return convertD2F(h->matF, h->matF2, h->matD, h->matD2);
}

// y = H x with the reference sequential SoA kernel (y zeroed first, as the
// reference proxy does at hmvm_seq.cpp:398-401).
void ref_seq2_d(void* hv, const double* x, double* y, int a2i) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  int nd = h->matD2->nd;
  for (int i = 0; i < nd; i++) y[i] = 0.0;
  if (a2i) hmvm_seq_2<double, 1>(y, h->matD2, x);
  else     hmvm_seq_2<double, 0>(y, h->matD2, x);
}

void ref_seq2_f(void* hv, const float* x, float* y, int a2i) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  int nd = h->matF2->nd;
  for (int i = 0; i < nd; i++) y[i] = 0.0f;
  if (a2i) hmvm_seq_2<float, 1>(y, h->matF2, x);
  else     hmvm_seq_2<float, 0>(y, h->matF2, x);
}

// AoS sequential kernel; requires a handle from ref_load1.
int ref_seq1_d(void* hv, const double* x, double* y, int a2i) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  if (!h->matD) return -1;
  int nd = h->matD->nd;
  for (int i = 0; i < nd; i++) y[i] = 0.0;
  if (a2i) hmvm_seq_1<double, 1>(y, h->matD, x);
  else     hmvm_seq_1<double, 0>(y, h->matD, x);
  return 0;
}

// OpenMP SoA kernel (zeroes y itself, hmvm_omp.cpp:391-392).  nthreads<=0 keeps
// the OpenMP default.
void ref_omp2_d(void* hv, const double* x, double* y, int nthreads) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  hmvm_omp_2<double, 0>(y, h->matD2, x);
}

void ref_omp2_f(void* hv, const float* x, float* y, int nthreads) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  hmvm_omp_2<float, 0>(y, h->matF2, x);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// The handle's matrix2<double> / matrix2<float> (after ref_make_float), for the
// reference's CUDA code in the companion library (ref_cuda_harness.cu).
void* ref_matrix2_d(void* hv) { return static_cast<RefHandle*>(hv)->matD2; }
void* ref_matrix2_f(void* hv) { return static_cast<RefHandle*>(hv)->matF2; }

// The reference's own timed sweep of its SoA OpenMP variants,
// hmvm_omp_bench<double>(NULL, mat2, x, 0) (src_hmvm/src_cpp/hmvm_omp.cpp:992-1347;
// with mat == NULL it skips the AoS variants).  It prints "TIME <L> <name> min
// max avg" lines on stdout; they are written to out_path instead, for the
// caller to parse.  Returns 0, or -1 if out_path cannot be opened.
int ref_omp_bench_d(void* hv, const double* x, const char* out_path, int nthreads) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  FILE* f = fopen(out_path, "w");
  if (!f) return -1;
  fflush(stdout);
  int saved = dup(1);
  dup2(fileno(f), 1);
  hmvm_omp_bench<double>(NULL, h->matD2, x, 0);
  fflush(stdout);
  dup2(saved, 1);
  close(saved);
  fclose(f);
  return 0;
}

void ref_free(void* hv) {
  RefHandle* h = static_cast<RefHandle*>(hv);
  if (!h) return;
  // The reference never frees its matrices; release what the loaders allocated.
  if (h->matD2 && h->wrapped) free(h->matD2->rowmat_t);
  if (h->matD2 && !h->wrapped) {
    free(h->matD2->ltmtx); free(h->matD2->kt); free(h->matD2->ndl); free(h->matD2->ndt);
    free(h->matD2->nstrtl); free(h->matD2->nstrtt); free(h->matD2->a1); free(h->matD2->a2);
    free(h->matD2->rowmat); free(h->matD2->rowmat_t);
  }
  if (h->matD) {
    for (int i = 0; i < h->matD->nlf; i++) {
      free(h->matD->submat[i].a1); free(h->matD->submat[i].a2); free(h->matD->submat[i].a2t);
    }
    free(h->matD->submat);
    delete h->matD;
  }
  if (h->matF2) {
    delete[] h->matF2->ltmtx; delete[] h->matF2->kt; delete[] h->matF2->ndl; delete[] h->matF2->ndt;
    delete[] h->matF2->nstrtl; delete[] h->matF2->nstrtt; delete[] h->matF2->a1; delete[] h->matF2->a2;
    delete[] h->matF2->rowmat; delete[] h->matF2->rowmat_t;
    delete h->matF2;
  }
  if (h->matF) {
    for (int i = 0; i < h->matF->nlf; i++) {
      delete[] h->matF->submat[i].a1; delete[] h->matF->submat[i].a2; delete[] h->matF->submat[i].a2t;
    }
    delete[] h->matF->submat;
    delete h->matF;
  }
  delete h->matD2;
  delete h;
}

}  // extern "C"
