// File loaders and the FP64->FP32 conversion, with the reference's signatures
// and results (src_hmvm/src_cpp/loadmatrix.cpp) but checked input: record
// markers, leaf fields and sizes are validated, errors are returned as status
// codes, nothing is printed and nothing stays allocated after a failure.

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "hmvm_b200.h"

namespace hmvm {
int set_error(int status, const std::string& msg);
}
using hmvm::set_error;

namespace {

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

// One Fortran unformatted sequential record of exactly `nbytes` payload bytes.
int read_record(FILE* f, void* dst, size_t nbytes, const char* what) {
  int32_t m1 = 0, m2 = 0;
  if (fread(&m1, 4, 1, f) != 1) return set_error(HMVM_EFORMAT, std::string("truncated before ") + what);
  if ((int64_t)m1 != (int64_t)nbytes)
    return set_error(HMVM_EFORMAT, std::string("record length mismatch in ") + what + ": marker " +
                                       std::to_string(m1) + ", expected " + std::to_string(nbytes));
  if (nbytes && fread(dst, 1, nbytes, f) != nbytes)
    return set_error(HMVM_EFORMAT, std::string("truncated in ") + what);
  if (fread(&m2, 4, 1, f) != 1 || m2 != m1)
    return set_error(HMVM_EFORMAT, std::string("bad closing record marker after ") + what);
  return HMVM_OK;
}

int check_leaf(int nd, int ktmax, int i, int ltmtx, int ndl, int ndt, int nstrtl, int nstrtt, int kt) {
  char buf[200];
  const char* why = nullptr;
  if (ltmtx != 1 && ltmtx != 2) why = "ltmtx is not 1 or 2";
  else if (ndl < 0 || ndt < 0) why = "negative ndl/ndt";
  else if (ndl > 0 && (nstrtl < 1 || (long long)nstrtl - 1 + ndl > nd)) why = "nstrtl+ndl-1 > nd";
  else if (ndt > 0 && (nstrtt < 1 || (long long)nstrtt - 1 + ndt > nd)) why = "nstrtt+ndt-1 > nd";
  else if (ltmtx == 1 && (kt < 0 || kt > ktmax)) why = "kt outside 0..ktmax";
  if (!why) return HMVM_OK;
  snprintf(buf, sizeof buf, "leaf %d: %s", i, why);
  return set_error(HMVM_EFORMAT, buf);
}

long long leaf_elems(int ltmtx, int kt, int ndl, int ndt) {
  return ltmtx == 1 ? (long long)kt * ndt + (long long)kt * ndl : (long long)ndl * ndt;
}

template <class M2>
bool alloc_soa_heads(M2* m2, int nlf) {
  size_t n = (size_t)(nlf > 0 ? nlf : 1);
  m2->ltmtx = (int*)malloc(n * 4);
  m2->kt = (int*)malloc(n * 4);
  m2->ndl = (int*)malloc(n * 4);
  m2->ndt = (int*)malloc(n * 4);
  m2->nstrtl = (int*)malloc(n * 4);
  m2->nstrtt = (int*)malloc(n * 4);
  m2->a1 = (int*)malloc(n * 4);
  m2->a2 = (int*)malloc(n * 4);
  return m2->ltmtx && m2->kt && m2->ndl && m2->ndt && m2->nstrtl && m2->nstrtt && m2->a1 && m2->a2;
}

// rowmat_t: a1 block copied, U transposed to [ndl][kt] (loadmatrix.cpp:227-234).
template <class T>
void fill_rowmat_t(const int* ltmtx, const int* kt, const int* ndl, const int* ndt, const int* a1, const int* a2,
                   int nlf, const T* rowmat, T* rowmat_t) {
  for (int i = 0; i < nlf; i++) {
    if (ltmtx[i] == 1) {
      std::memcpy(rowmat_t + a1[i], rowmat + a1[i], sizeof(T) * (size_t)kt[i] * ndt[i]);
      const T* u = rowmat + a2[i];
      T* ut = rowmat_t + a2[i];
      for (int y = 0; y < kt[i]; y++)
        for (int x = 0; x < ndl[i]; x++) ut[y + (size_t)x * kt[i]] = u[(size_t)y * ndl[i] + x];
    } else {
      std::memcpy(rowmat_t + a1[i], rowmat + a1[i], sizeof(T) * (size_t)ndl[i] * ndt[i]);
    }
  }
}

// The owned arrays of a 64-bit leaf table being loaded.
struct Table64 {
  int32_t *ltmtx = nullptr, *kt = nullptr, *ndl = nullptr, *ndt = nullptr, *nstrtl = nullptr, *nstrtt = nullptr;
  int64_t *a1 = nullptr, *a2 = nullptr;
  double* rowmat = nullptr;
  ~Table64() {
    free(ltmtx); free(kt); free(ndl); free(ndt); free(nstrtl); free(nstrtt); free(a1); free(a2); free(rowmat);
  }
  bool alloc(int32_t nlf) {
    const size_t n = (size_t)(nlf > 0 ? nlf : 1);
    ltmtx = (int32_t*)malloc(n * 4); kt = (int32_t*)malloc(n * 4); ndl = (int32_t*)malloc(n * 4);
    ndt = (int32_t*)malloc(n * 4); nstrtl = (int32_t*)malloc(n * 4); nstrtt = (int32_t*)malloc(n * 4);
    a1 = (int64_t*)malloc(n * 8); a2 = (int64_t*)malloc(n * 8);
    return ltmtx && kt && ndl && ndt && nstrtl && nstrtt && a1 && a2;
  }
  // hands the arrays to `lv` (which then owns them)
  void release_to(hmvm_leaves64* lv) {
    lv->ltmtx = ltmtx; lv->kt = kt; lv->ndl = ndl; lv->ndt = ndt; lv->nstrtl = nstrtl; lv->nstrtt = nstrtt;
    lv->a1 = a1; lv->a2 = a2; lv->rowmat = rowmat;
    ltmtx = kt = ndl = ndt = nstrtl = nstrtt = nullptr;
    a1 = a2 = nullptr;
    rowmat = nullptr;
  }
};

// Reads leaf i's data records at rowmat[off..] and sets a1/a2 (file order).
int read_leaf_data64(FILE* f, Table64& T, int32_t i, int64_t& off) {
  int rc;
  if (T.ltmtx[i] == 1) {
    const size_t n1 = (size_t)T.kt[i] * T.ndt[i], n2 = (size_t)T.kt[i] * T.ndl[i];
    T.a1[i] = off;
    if ((rc = read_record(f, T.rowmat + off, n1 * 8, "low-rank a1"))) return rc;
    off += (int64_t)n1;
    T.a2[i] = off;
    if ((rc = read_record(f, T.rowmat + off, n2 * 8, "low-rank a2"))) return rc;
    off += (int64_t)n2;
  } else {
    const size_t n1 = (size_t)T.ndl[i] * T.ndt[i];
    T.a1[i] = off;
    T.a2[i] = 0;
    if ((rc = read_record(f, T.rowmat + off, n1 * 8, "dense a1"))) return rc;
    off += (int64_t)n1;
  }
  return HMVM_OK;
}

}  // namespace

extern "C" {

int hmvm_b200_load_leaves64(const char* fname, hmvm_leaves64* out, int32_t* format) {
  if (!fname || !out) return set_error(HMVM_EINVAL, "NULL argument");
  File F;
  F.f = fopen(fname, "rb");
  if (!F.f) return set_error(HMVM_EIO, std::string("cannot open ") + fname);
  int32_t m0 = 0;
  if (fread(&m0, 4, 1, F.f) != 1 || fseek(F.f, 0, SEEK_SET) != 0)
    return set_error(HMVM_EFORMAT, "truncated before header");
  const int fmt = m0 == 12 ? HMVM_BIN1 : m0 == 16 ? HMVM_BIN2 : m0 == 20 ? HMVM_BIN64 : 0;
  if (!fmt)
    return set_error(HMVM_EFORMAT, "header record of " + std::to_string(m0) + " bytes (12, 16 or 20 expected)");
  unsigned char hdr[20];
  int rc = read_record(F.f, hdr, (size_t)m0, "header");
  if (rc) return rc;
  int32_t h3[3];
  std::memcpy(h3, hdr, 12);
  const int32_t nd = h3[0], nlf = h3[1], ktmax = h3[2];
  int64_t len = -1;  // bin1 carries none
  if (fmt == HMVM_BIN2) {
    int32_t l32;
    std::memcpy(&l32, hdr + 12, 4);
    len = l32;
  } else if (fmt == HMVM_BIN64) {
    std::memcpy(&len, hdr + 12, 8);
  }
  if (nd < 0 || nlf < 0 || ktmax < 0 || (fmt != HMVM_BIN1 && len < 0))
    return set_error(HMVM_EFORMAT, "negative field in header");
  Table64 T;
  if (!T.alloc(nlf)) return set_error(HMVM_ENOMEM, "host allocation failed");
  int64_t off = 0;
  if (fmt == HMVM_BIN1) {
    // per leaf: header record, then its data (loadmatrix.cpp:98-127); rowmat grows
    size_t cap = 1 << 16;
    T.rowmat = (double*)malloc(cap * sizeof(double));
    if (!T.rowmat) return set_error(HMVM_ENOMEM, "host allocation failed");
    for (int32_t i = 0; i < nlf; i++) {
      int32_t h6[6];
      if ((rc = read_record(F.f, h6, sizeof h6, "leaf header"))) return rc;
      T.ltmtx[i] = h6[0]; T.ndl[i] = h6[1]; T.ndt[i] = h6[2]; T.nstrtl[i] = h6[3]; T.nstrtt[i] = h6[4];
      T.kt[i] = h6[5];
      if ((rc = check_leaf(nd, ktmax, i, T.ltmtx[i], T.ndl[i], T.ndt[i], T.nstrtl[i], T.nstrtt[i], T.kt[i])))
        return rc;
      const size_t need = (size_t)leaf_elems(T.ltmtx[i], T.kt[i], T.ndl[i], T.ndt[i]);
      if ((size_t)off + need > cap) {
        while ((size_t)off + need > cap) cap *= 2;
        double* p = (double*)realloc(T.rowmat, cap * sizeof(double));
        if (!p) return set_error(HMVM_ENOMEM, "host allocation failed");
        T.rowmat = p;
      }
      if ((rc = read_leaf_data64(F.f, T, i, off))) return rc;
    }
    len = off;
  } else {
    // six int32[nlf] columns, then every leaf's data (loadmatrix.cpp:152-250)
    int32_t* cols[6] = {T.ltmtx, T.ndl, T.ndt, T.nstrtl, T.nstrtt, T.kt};
    const char* names[6] = {"ltmtx", "ndl", "ndt", "nstrtl", "nstrtt", "kt"};
    for (int c = 0; c < 6; c++)
      if ((rc = read_record(F.f, cols[c], (size_t)nlf * 4, names[c]))) return rc;
    int64_t total = 0;
    for (int32_t i = 0; i < nlf; i++) {
      if ((rc = check_leaf(nd, ktmax, i, T.ltmtx[i], T.ndl[i], T.ndt[i], T.nstrtl[i], T.nstrtt[i], T.kt[i])))
        return rc;
      total += leaf_elems(T.ltmtx[i], T.kt[i], T.ndl[i], T.ndt[i]);
    }
    const bool saturated = fmt == HMVM_BIN2 && len == INT32_MAX && total >= INT32_MAX;
    if (total != len && !saturated)
      return set_error(HMVM_EFORMAT, "header len " + std::to_string(len) + " differs from the leaf sizes (" +
                                         std::to_string(total) + ")");
    len = total;
    T.rowmat = (double*)malloc((size_t)(len > 0 ? len : 1) * sizeof(double));
    if (!T.rowmat) return set_error(HMVM_ENOMEM, "host allocation failed");
    for (int32_t i = 0; i < nlf; i++)
      if ((rc = read_leaf_data64(F.f, T, i, off))) return rc;
  }
  std::memset(out, 0, sizeof(*out));
  out->nd = nd;
  out->nlf = nlf;
  out->ktmax = ktmax;
  out->len = len;
  T.release_to(out);
  if (format) *format = fmt;
  return HMVM_OK;
}

void hmvm_b200_free_leaves64(hmvm_leaves64* lv) {
  if (!lv) return;
  free(const_cast<int32_t*>(lv->ltmtx)); free(const_cast<int32_t*>(lv->kt));
  free(const_cast<int32_t*>(lv->ndl)); free(const_cast<int32_t*>(lv->ndt));
  free(const_cast<int32_t*>(lv->nstrtl)); free(const_cast<int32_t*>(lv->nstrtt));
  free(const_cast<int64_t*>(lv->a1)); free(const_cast<int64_t*>(lv->a2));
  free(const_cast<void*>(lv->rowmat));
  std::memset(lv, 0, sizeof(*lv));
}

void hmvm_b200_free_matrix2_d(hmvm_matrix2_d* m) {
  if (!m) return;
  free(m->nleavs); free(m->ltmtx); free(m->kt); free(m->ndl); free(m->ndt); free(m->nstrtl); free(m->nstrtt);
  free(m->a1); free(m->a2); free(m->rowmat); free(m->rowmat_t); free(m->approx); free(m->dense);
  std::memset(m, 0, sizeof(*m));
}
void hmvm_b200_free_matrix2_f(hmvm_matrix2_f* m) {
  if (!m) return;
  free(m->nleavs); free(m->ltmtx); free(m->kt); free(m->ndl); free(m->ndt); free(m->nstrtl); free(m->nstrtt);
  free(m->a1); free(m->a2); free(m->rowmat); free(m->rowmat_t); free(m->approx); free(m->dense);
  std::memset(m, 0, sizeof(*m));
}
void hmvm_b200_free_matrix_d(hmvm_matrix_d* m) {
  if (!m) return;
  if (m->submat)
    for (int i = 0; i < m->nlf; i++) {
      free(m->submat[i].a1); free(m->submat[i].a2); free(m->submat[i].a2t);
    }
  free(m->submat);
  free(m->nleavs);
  std::memset(m, 0, sizeof(*m));
}
void hmvm_b200_free_matrix_f(hmvm_matrix_f* m) {
  if (!m) return;
  if (m->submat)
    for (int i = 0; i < m->nlf; i++) {
      free(m->submat[i].a1); free(m->submat[i].a2); free(m->submat[i].a2t);
    }
  free(m->submat);
  free(m->nleavs);
  std::memset(m, 0, sizeof(*m));
}

int hmvm_b200_load_hmatrix(const char* fname, hmvm_matrix_d* mat, hmvm_matrix2_d* mat2) {
  if (!fname || !mat2) return set_error(HMVM_EINVAL, "NULL argument");
  File F;
  F.f = fopen(fname, "rb");
  if (!F.f) return set_error(HMVM_EIO, std::string("cannot open ") + fname);
  int hdr[3];
  int rc = read_record(F.f, hdr, sizeof hdr, "header");
  if (rc) return rc;
  const int nd = hdr[0], nlf = hdr[1], ktmax = hdr[2];
  if (nd < 0 || nlf < 0 || ktmax < 0) return set_error(HMVM_EFORMAT, "negative nd/nlf/ktmax in header");
  hmvm_matrix2_d m2;
  std::memset(&m2, 0, sizeof m2);
  hmvm_matrix_d m1;
  std::memset(&m1, 0, sizeof m1);
  auto fail = [&](int code) {
    hmvm_b200_free_matrix2_d(&m2);
    hmvm_b200_free_matrix_d(&m1);
    return code;
  };
  m2.nd = m1.nd = nd;
  m2.nlf = m1.nlf = nlf;
  m2.ktmax = m1.ktmax = ktmax;
  if (!alloc_soa_heads(&m2, nlf)) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
  // Pass 1: headers and data into a growing rowmat (file order, as :98-127).
  size_t cap = 1 << 16, used = 0;
  m2.rowmat = (double*)malloc(cap * sizeof(double));
  if (!m2.rowmat) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
  for (int i = 0; i < nlf; i++) {
    int h6[6];
    if ((rc = read_record(F.f, h6, sizeof h6, "leaf header"))) return fail(rc);
    const int ltmtx = h6[0], ndl = h6[1], ndt = h6[2], nstrtl = h6[3], nstrtt = h6[4], kt = h6[5];
    if ((rc = check_leaf(nd, ktmax, i, ltmtx, ndl, ndt, nstrtl, nstrtt, kt))) return fail(rc);
    long long need = leaf_elems(ltmtx, kt, ndl, ndt);
    if ((long long)used + need > INT_MAX)
      return fail(set_error(HMVM_ERANGE, "stored elements exceed the int len of matrix2"));
    while (used + (size_t)need > cap) {
      cap *= 2;
      double* p = (double*)realloc(m2.rowmat, cap * sizeof(double));
      if (!p) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
      m2.rowmat = p;
    }
    m2.ltmtx[i] = ltmtx; m2.ndl[i] = ndl; m2.ndt[i] = ndt; m2.nstrtl[i] = nstrtl; m2.nstrtt[i] = nstrtt;
    m2.kt[i] = kt;
    if (ltmtx == 1) {
      size_t n1 = (size_t)kt * ndt, n2 = (size_t)kt * ndl;
      m2.a1[i] = (int)used;
      if ((rc = read_record(F.f, m2.rowmat + used, n1 * 8, "low-rank a1"))) return fail(rc);
      used += n1;
      m2.a2[i] = (int)used;
      if ((rc = read_record(F.f, m2.rowmat + used, n2 * 8, "low-rank a2"))) return fail(rc);
      used += n2;
    } else {
      size_t n1 = (size_t)ndl * ndt;
      m2.a1[i] = (int)used;
      m2.a2[i] = 0;
      if ((rc = read_record(F.f, m2.rowmat + used, n1 * 8, "dense a1"))) return fail(rc);
      used += n1;
    }
  }
  m2.len = (int)used;
  m2.rowmat_t = (double*)malloc((used > 0 ? used : 1) * sizeof(double));
  if (!m2.rowmat_t) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
  fill_rowmat_t(m2.ltmtx, m2.kt, m2.ndl, m2.ndt, m2.a1, m2.a2, nlf, m2.rowmat, m2.rowmat_t);
  if (mat) {
    // AoS copies with a2t = U transposed (loadmatrix.cpp:58-85).
    m1.submat = (hmvm_submatrix_d*)calloc((size_t)(nlf > 0 ? nlf : 1), sizeof(hmvm_submatrix_d));
    if (!m1.submat) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
    for (int i = 0; i < nlf; i++) {
      hmvm_submatrix_d& s = m1.submat[i];
      s.ltmtx = m2.ltmtx[i]; s.kt = m2.kt[i]; s.ndl = m2.ndl[i]; s.ndt = m2.ndt[i];
      s.nstrtl = m2.nstrtl[i]; s.nstrtt = m2.nstrtt[i];
      if (s.ltmtx == 1) {
        size_t n1 = (size_t)s.kt * s.ndt, n2 = (size_t)s.kt * s.ndl;
        s.a1 = (double*)malloc((n1 ? n1 : 1) * 8);
        s.a2 = (double*)malloc((n2 ? n2 : 1) * 8);
        s.a2t = (double*)malloc((n2 ? n2 : 1) * 8);
        if (!s.a1 || !s.a2 || !s.a2t) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
        std::memcpy(s.a1, m2.rowmat + m2.a1[i], n1 * 8);
        std::memcpy(s.a2, m2.rowmat + m2.a2[i], n2 * 8);
        std::memcpy(s.a2t, m2.rowmat_t + m2.a2[i], n2 * 8);
      } else {
        size_t n1 = (size_t)s.ndl * s.ndt;
        s.a1 = (double*)malloc((n1 ? n1 : 1) * 8);
        if (!s.a1) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
        std::memcpy(s.a1, m2.rowmat + m2.a1[i], n1 * 8);
      }
    }
    *mat = m1;
  }
  *mat2 = m2;
  return HMVM_OK;
}

int hmvm_b200_load_hmatrix2(const char* fname, hmvm_matrix2_d* mat2) {
  if (!fname || !mat2) return set_error(HMVM_EINVAL, "NULL argument");
  File F;
  F.f = fopen(fname, "rb");
  if (!F.f) return set_error(HMVM_EIO, std::string("cannot open ") + fname);
  int hdr[4];
  int rc = read_record(F.f, hdr, sizeof hdr, "header");
  if (rc) return rc;
  const int nd = hdr[0], nlf = hdr[1], ktmax = hdr[2], len = hdr[3];
  if (nd < 0 || nlf < 0 || ktmax < 0 || len < 0) return set_error(HMVM_EFORMAT, "negative field in header");
  hmvm_matrix2_d m2;
  std::memset(&m2, 0, sizeof m2);
  auto fail = [&](int code) {
    hmvm_b200_free_matrix2_d(&m2);
    return code;
  };
  m2.nd = nd;
  m2.nlf = nlf;
  m2.ktmax = ktmax;
  if (!alloc_soa_heads(&m2, nlf)) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
  size_t nb = (size_t)nlf * 4;
  int* cols[6] = {m2.ltmtx, m2.ndl, m2.ndt, m2.nstrtl, m2.nstrtt, m2.kt};
  const char* names[6] = {"ltmtx", "ndl", "ndt", "nstrtl", "nstrtt", "kt"};
  for (int c = 0; c < 6; c++)
    if ((rc = read_record(F.f, cols[c], nb, names[c]))) return fail(rc);
  long long total = 0;
  for (int i = 0; i < nlf; i++) {
    if ((rc = check_leaf(nd, ktmax, i, m2.ltmtx[i], m2.ndl[i], m2.ndt[i], m2.nstrtl[i], m2.nstrtt[i], m2.kt[i])))
      return fail(rc);
    total += leaf_elems(m2.ltmtx[i], m2.kt[i], m2.ndl[i], m2.ndt[i]);
  }
  if (total > INT_MAX) return fail(set_error(HMVM_ERANGE, "stored elements exceed the int len of matrix2"));
  if (total != len)
    return fail(set_error(HMVM_EFORMAT, "header len " + std::to_string(len) + " differs from the leaf sizes (" +
                                            std::to_string(total) + ")"));
  m2.len = len;
  m2.rowmat = (double*)malloc((size_t)(len > 0 ? len : 1) * 8);
  m2.rowmat_t = (double*)malloc((size_t)(len > 0 ? len : 1) * 8);
  if (!m2.rowmat || !m2.rowmat_t) return fail(set_error(HMVM_ENOMEM, "host allocation failed"));
  size_t off = 0;
  for (int i = 0; i < nlf; i++) {
    if (m2.ltmtx[i] == 1) {
      size_t n1 = (size_t)m2.kt[i] * m2.ndt[i], n2 = (size_t)m2.kt[i] * m2.ndl[i];
      m2.a1[i] = (int)off;
      if ((rc = read_record(F.f, m2.rowmat + off, n1 * 8, "low-rank a1"))) return fail(rc);
      off += n1;
      m2.a2[i] = (int)off;
      if ((rc = read_record(F.f, m2.rowmat + off, n2 * 8, "low-rank a2"))) return fail(rc);
      off += n2;
    } else {
      size_t n1 = (size_t)m2.ndl[i] * m2.ndt[i];
      m2.a1[i] = (int)off;
      m2.a2[i] = 0;
      if ((rc = read_record(F.f, m2.rowmat + off, n1 * 8, "dense a1"))) return fail(rc);
      off += n1;
    }
  }
  fill_rowmat_t(m2.ltmtx, m2.kt, m2.ndl, m2.ndt, m2.a1, m2.a2, nlf, m2.rowmat, m2.rowmat_t);
  *mat2 = m2;
  return HMVM_OK;
}

int hmvm_b200_convert_d2f(hmvm_matrix_f* matF, hmvm_matrix2_f* matF2, const hmvm_matrix_d* matD,
                          const hmvm_matrix2_d* matD2) {
  if (matD && matF) {
    hmvm_matrix_f f;
    std::memset(&f, 0, sizeof f);
    f.nd = matD->nd;
    f.nlf = matD->nlf;
    f.ktmax = matD->ktmax;
    f.submat = (hmvm_submatrix_f*)calloc((size_t)(f.nlf > 0 ? f.nlf : 1), sizeof(hmvm_submatrix_f));
    if (!f.submat) return set_error(HMVM_ENOMEM, "host allocation failed");
    for (int i = 0; i < f.nlf; i++) {
      const hmvm_submatrix_d& s = matD->submat[i];
      hmvm_submatrix_f& o = f.submat[i];
      o.ltmtx = s.ltmtx; o.kt = s.kt; o.ndl = s.ndl; o.ndt = s.ndt; o.nstrtl = s.nstrtl; o.nstrtt = s.nstrtt;
      size_t n1 = s.ltmtx == 1 ? (size_t)s.kt * s.ndt : (size_t)s.ndl * s.ndt;
      size_t n2 = s.ltmtx == 1 ? (size_t)s.kt * s.ndl : 0;
      o.a1 = (float*)malloc((n1 ? n1 : 1) * 4);
      if (n2) {
        o.a2 = (float*)malloc(n2 * 4);
        o.a2t = (float*)malloc(n2 * 4);
      }
      if (!o.a1 || (n2 && (!o.a2 || !o.a2t))) {
        hmvm_b200_free_matrix_f(&f);
        return set_error(HMVM_ENOMEM, "host allocation failed");
      }
      for (size_t j = 0; j < n1; j++) o.a1[j] = (float)s.a1[j];
      for (size_t j = 0; j < n2; j++) o.a2[j] = (float)s.a2[j];
      for (size_t j = 0; j < n2; j++) o.a2t[j] = (float)s.a2t[j];
    }
    *matF = f;
  }
  if (matD2 && matF2) {
    hmvm_matrix2_f f;
    std::memset(&f, 0, sizeof f);
    f.nd = matD2->nd;
    f.nlf = matD2->nlf;
    f.ktmax = matD2->ktmax;
    f.len = matD2->len;
    if (!alloc_soa_heads(&f, f.nlf)) {
      hmvm_b200_free_matrix2_f(&f);
      return set_error(HMVM_ENOMEM, "host allocation failed");
    }
    size_t n = (size_t)f.nlf * 4;
    std::memcpy(f.ltmtx, matD2->ltmtx, n); std::memcpy(f.kt, matD2->kt, n);
    std::memcpy(f.ndl, matD2->ndl, n); std::memcpy(f.ndt, matD2->ndt, n);
    std::memcpy(f.nstrtl, matD2->nstrtl, n); std::memcpy(f.nstrtt, matD2->nstrtt, n);
    std::memcpy(f.a1, matD2->a1, n); std::memcpy(f.a2, matD2->a2, n);
    size_t len = (size_t)(f.len > 0 ? f.len : 1);
    f.rowmat = (float*)malloc(len * 4);
    if (!f.rowmat) {
      hmvm_b200_free_matrix2_f(&f);
      return set_error(HMVM_ENOMEM, "host allocation failed");
    }
    for (int64_t j = 0; j < matD2->len; j++) f.rowmat[j] = (float)matD2->rowmat[j];
    if (matD2->rowmat_t) {
      f.rowmat_t = (float*)malloc(len * 4);
      if (!f.rowmat_t) {
        hmvm_b200_free_matrix2_f(&f);
        return set_error(HMVM_ENOMEM, "host allocation failed");
      }
      for (int64_t j = 0; j < matD2->len; j++) f.rowmat_t[j] = (float)matD2->rowmat_t[j];
    }
    *matF2 = f;
  }
  return HMVM_OK;
}

}  // extern "C"
