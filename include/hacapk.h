// hacapk.h -- the H-matrix structures of the reference harness, for code that
// moves to this library without the reference sources.
//
// The three templates must keep the member order and types of the
// reference's src_hmvm/src_cpp/hacapk.h:5-36 (existing drivers fill and read
// them directly, and hmvm_b200.h's hmvm_matrix2_d/_f are the same bytes); the
// loader prototypes are those of src_hmvm/src_cpp/hacapk.h:39-41, defined by
// hmvm_cuda_b200.hpp when HMVM_B200_DEFINE_LOADERS is set.  The include guard
// is the reference's, so either copy of the header can be included first.
#ifndef _HACAPK_C_HPP
#define _HACAPK_C_HPP

// One leaf.  ltmtx 1: low-rank, a1 = V^T [kt][ndt], a2 = U [kt][ndl],
// a2t = U [ndl][kt];  ltmtx 2: dense, a1 = [ndl][ndt].  nstrtl/nstrtt 1-based.
template <class T>
struct submatrix {
  int ltmtx, kt, ndl, ndt, nstrtl, nstrtt;
  T *a1, *a2, *a2t;
};

// Array-of-structures form.
template <class T>
struct matrix {
  int nd;
  int nlf;
  int ktmax;
  int *nleavs;
  submatrix<T> *submat;
  int b1, b2, b3;
  int e1, e2, e3;
};

// Structure-of-arrays form: leaf fields in separate arrays, all leaf data in
// rowmat at element offsets a1/a2 (rowmat_t: U transposed to [ndl][kt]).
template <class T>
struct matrix2 {
  int nd;
  int nlf;
  int ktmax;
  int len;
  int *nleavs;
  int *ltmtx, *kt, *ndl, *ndt, *nstrtl, *nstrtt;
  int *a1, *a2;
  T *rowmat, *rowmat_t;
  int napprox, ndense;
  int *approx, *dense;
};

int loadHmatrix(const char *fname, matrix<double> *, matrix2<double> *);
int loadHmatrix2(const char *fname, matrix2<double> *);
int convertD2F(matrix<float> *matF, matrix2<float> *matF2, const matrix<double> *matD, const matrix2<double> *matD2);

#endif
