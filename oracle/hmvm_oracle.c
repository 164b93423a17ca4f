/*
 * ORACLE -- test infrastructure only.  Never linked into the product.
 *
 * A plain-C restatement of the reference HMVM path, used as the checker for the
 * CUDA library in tests/, in __graft_entry__.smoke() and (as the "port" CPU
 * baseline) in bench.py.  It differs from the reference only in using 64-bit
 * element offsets, so it also covers matrices whose stored element count
 * overflows the reference's `int len` / `int a1[], a2[]`
 * (src_hmvm/src_cpp/hacapk.h:28,31).
 *
 * Pinning: tests/test_oracle.py checks this file bit-for-bit against the
 * reference's own hmvm_seq_2 / loadHmatrix / loadHmatrix2 compiled from the
 * reference sources (oracle/_ref, built by oracle/Makefile) on the reference's
 * shipped hmatrix_sample.bin and on generated matrices, and against the golden
 * vectors under tests/golden/ (written by tests/golden/make_golden.py from the
 * reference build).
 *
 * Restated functions (reference file:line):
 *   orc_load_bin1   src_hmvm/src_cpp/loadmatrix.cpp:7-150   (hmatrix_1.bin)
 *   orc_load_bin2   src_hmvm/src_cpp/loadmatrix.cpp:152-250 (hmatrix_2.bin)
 *   orc_hmvm_seq2_d src_hmvm/src_cpp/hmvm_seq.cpp:154-227   (hmvm_seq_2<double,a2i>)
 *   orc_hmvm_seq2_f src_hmvm/src_cpp/hmvm_seq.cpp:154-227   (hmvm_seq_2<float,a2i>)
 *   orc_omp2_d      src_hmvm/src_cpp/hmvm_omp.cpp:374-463   (hmvm_omp_2<double,0>)
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EOPEN -1
#define ORC_ETRUNC -2
#define ORC_ERECORD -3
#define ORC_EVALUE -4
#define ORC_ENOMEM -5

/* Loaded SoA matrix: the matrix2<double> of src_hmvm/src_cpp/hacapk.h:23-36 with
 * 64-bit a1/a2 offsets and 64-bit len. */
typedef struct {
  int32_t nd, nlf, ktmax;
  int64_t len;
  int32_t *ltmtx, *kt, *ndl, *ndt, *nstrtl, *nstrtt;
  int64_t *a1, *a2;
  double *rowmat;
} orc_hmat;

static int rd(FILE *f, void *p, size_t sz, size_t n) {
  return fread(p, sz, n, f) == n ? ORC_OK : ORC_ETRUNC;
}

/* One Fortran unformatted sequential record: 4-byte length, payload, 4-byte length. */
static int rd_record(FILE *f, void *p, size_t nbytes) {
  int32_t m1, m2;
  if (rd(f, &m1, 4, 1)) return ORC_ETRUNC;
  if ((int64_t)m1 != (int64_t)nbytes) return ORC_ERECORD;
  if (nbytes && rd(f, p, 1, nbytes)) return ORC_ETRUNC;
  if (rd(f, &m2, 4, 1)) return ORC_ETRUNC;
  if (m2 != m1) return ORC_ERECORD;
  return ORC_OK;
}

void orc_free(orc_hmat *m) {
  free(m->ltmtx); free(m->kt); free(m->ndl); free(m->ndt);
  free(m->nstrtl); free(m->nstrtt); free(m->a1); free(m->a2); free(m->rowmat);
  memset(m, 0, sizeof(*m));
}

static int alloc_heads(orc_hmat *m) {
  size_t n = (size_t)(m->nlf > 0 ? m->nlf : 1);
  m->ltmtx = malloc(n * 4); m->kt = malloc(n * 4); m->ndl = malloc(n * 4); m->ndt = malloc(n * 4);
  m->nstrtl = malloc(n * 4); m->nstrtt = malloc(n * 4);
  m->a1 = malloc(n * 8); m->a2 = malloc(n * 8);
  if (!m->ltmtx || !m->kt || !m->ndl || !m->ndt || !m->nstrtl || !m->nstrtt || !m->a1 || !m->a2)
    return ORC_ENOMEM;
  return ORC_OK;
}

static int64_t leaf_elems(int32_t ltmtx, int32_t kt, int32_t ndl, int32_t ndt) {
  return ltmtx == 1 ? (int64_t)kt * ndt + (int64_t)kt * ndl : (int64_t)ndl * ndt;
}

/* hmatrix_1.bin: header record (nd,nlf,ktmax); per leaf a record
 * (ltmtx,ndl,ndt,nstrtl,nstrtt,kt) then a1 (and a2 for ltmtx==1) records
 * (loadmatrix.cpp:20-86).  Offsets are assigned in leaf order as at :98-127. */
int orc_load_bin1(const char *fname, orc_hmat *m) {
  memset(m, 0, sizeof(*m));
  FILE *f = fopen(fname, "rb");
  if (!f) return ORC_EOPEN;
  int32_t hdr[3];
  int rc = rd_record(f, hdr, sizeof hdr);
  if (rc) goto fail;
  m->nd = hdr[0]; m->nlf = hdr[1]; m->ktmax = hdr[2];
  if (m->nd < 0 || m->nlf < 0) { rc = ORC_EVALUE; goto fail; }
  if ((rc = alloc_heads(m))) goto fail;
  /* First pass: read the whole file into a growing buffer. */
  size_t cap = 1 << 20, used = 0;
  m->rowmat = malloc(cap * sizeof(double));
  if (!m->rowmat) { rc = ORC_ENOMEM; goto fail; }
  for (int32_t i = 0; i < m->nlf; i++) {
    int32_t h6[6];
    if ((rc = rd_record(f, h6, sizeof h6))) goto fail;
    m->ltmtx[i] = h6[0]; m->ndl[i] = h6[1]; m->ndt[i] = h6[2];
    m->nstrtl[i] = h6[3]; m->nstrtt[i] = h6[4]; m->kt[i] = h6[5];
    if (h6[1] < 0 || h6[2] < 0 || h6[5] < 0) { rc = ORC_EVALUE; goto fail; }
    int64_t need = leaf_elems(h6[0], h6[5], h6[1], h6[2]);
    while (used + (size_t)need > cap) {
      cap *= 2;
      double *p = realloc(m->rowmat, cap * sizeof(double));
      if (!p) { rc = ORC_ENOMEM; goto fail; }
      m->rowmat = p;
    }
    if (h6[0] == 1) {
      int64_t n1 = (int64_t)h6[5] * h6[2], n2 = (int64_t)h6[5] * h6[1];
      m->a1[i] = (int64_t)used;
      if ((rc = rd_record(f, m->rowmat + used, (size_t)n1 * 8))) goto fail;
      used += (size_t)n1;
      m->a2[i] = (int64_t)used;
      if ((rc = rd_record(f, m->rowmat + used, (size_t)n2 * 8))) goto fail;
      used += (size_t)n2;
    } else {
      int64_t n1 = (int64_t)h6[1] * h6[2];
      m->a1[i] = (int64_t)used;
      m->a2[i] = 0;
      if ((rc = rd_record(f, m->rowmat + used, (size_t)n1 * 8))) goto fail;
      used += (size_t)n1;
    }
  }
  m->len = (int64_t)used;
  fclose(f);
  return ORC_OK;
fail:
  fclose(f);
  orc_free(m);
  return rc;
}

/* hmatrix_2.bin: header record (nd,nlf,ktmax,len); six int[nlf] records in the
 * order ltmtx, ndl, ndt, nstrtl, nstrtt, kt; then the per-leaf a1/a2 records
 * (loadmatrix.cpp:165-245).  The stored int32 len is checked against the sum of
 * leaf sizes when it fits, and ignored when the sum overflows int32. */
int orc_load_bin2(const char *fname, orc_hmat *m) {
  memset(m, 0, sizeof(*m));
  FILE *f = fopen(fname, "rb");
  if (!f) return ORC_EOPEN;
  int32_t hdr[4];
  int rc = rd_record(f, hdr, sizeof hdr);
  if (rc) goto fail;
  m->nd = hdr[0]; m->nlf = hdr[1]; m->ktmax = hdr[2];
  if (m->nd < 0 || m->nlf < 0) { rc = ORC_EVALUE; goto fail; }
  if ((rc = alloc_heads(m))) goto fail;
  size_t nb = (size_t)m->nlf * 4;
  if ((rc = rd_record(f, m->ltmtx, nb))) goto fail;
  if ((rc = rd_record(f, m->ndl, nb))) goto fail;
  if ((rc = rd_record(f, m->ndt, nb))) goto fail;
  if ((rc = rd_record(f, m->nstrtl, nb))) goto fail;
  if ((rc = rd_record(f, m->nstrtt, nb))) goto fail;
  if ((rc = rd_record(f, m->kt, nb))) goto fail;
  int64_t len = 0;
  for (int32_t i = 0; i < m->nlf; i++) {
    if (m->ndl[i] < 0 || m->ndt[i] < 0 || m->kt[i] < 0) { rc = ORC_EVALUE; goto fail; }
    len += leaf_elems(m->ltmtx[i], m->kt[i], m->ndl[i], m->ndt[i]);
  }
  if (len <= INT32_MAX && (int64_t)hdr[3] != len) { rc = ORC_EVALUE; goto fail; }
  m->len = len;
  m->rowmat = malloc((size_t)(len > 0 ? len : 1) * sizeof(double));
  if (!m->rowmat) { rc = ORC_ENOMEM; goto fail; }
  int64_t off = 0;
  for (int32_t i = 0; i < m->nlf; i++) {
    if (m->ltmtx[i] == 1) {
      int64_t n1 = (int64_t)m->kt[i] * m->ndt[i], n2 = (int64_t)m->kt[i] * m->ndl[i];
      m->a1[i] = off;
      if ((rc = rd_record(f, m->rowmat + off, (size_t)n1 * 8))) goto fail;
      off += n1;
      m->a2[i] = off;
      if ((rc = rd_record(f, m->rowmat + off, (size_t)n2 * 8))) goto fail;
      off += n2;
    } else {
      int64_t n1 = (int64_t)m->ndl[i] * m->ndt[i];
      m->a1[i] = off;
      m->a2[i] = 0;
      if ((rc = rd_record(f, m->rowmat + off, (size_t)n1 * 8))) goto fail;
      off += n1;
    }
  }
  fclose(f);
  return ORC_OK;
fail:
  fclose(f);
  orc_free(m);
  return rc;
}

/* Copy helpers so callers (ctypes) can take the arrays over. */
void orc_export(const orc_hmat *m, int32_t *ltmtx, int32_t *kt, int32_t *ndl, int32_t *ndt,
                int32_t *nstrtl, int32_t *nstrtt, int64_t *a1, int64_t *a2, double *rowmat) {
  size_t n = (size_t)m->nlf;
  memcpy(ltmtx, m->ltmtx, n * 4); memcpy(kt, m->kt, n * 4);
  memcpy(ndl, m->ndl, n * 4); memcpy(ndt, m->ndt, n * 4);
  memcpy(nstrtl, m->nstrtl, n * 4); memcpy(nstrtt, m->nstrtt, n * 4);
  memcpy(a1, m->a1, n * 8); memcpy(a2, m->a2, n * 8);
  memcpy(rowmat, m->rowmat, (size_t)m->len * 8);
}

/* Heap-allocated handle API for ctypes. */
orc_hmat *orc_open(const char *fname, int format, int *rc) {
  orc_hmat *m = malloc(sizeof(orc_hmat));
  if (!m) { *rc = ORC_ENOMEM; return NULL; }
  *rc = format == 2 ? orc_load_bin2(fname, m) : orc_load_bin1(fname, m);
  if (*rc) { free(m); return NULL; }
  return m;
}
void orc_close(orc_hmat *m) { if (m) { orc_free(m); free(m); } }
void orc_info(const orc_hmat *m, int64_t *out4) {
  out4[0] = m->nd; out4[1] = m->nlf; out4[2] = m->ktmax; out4[3] = m->len;
}

/* hmvm_seq_2<T,a2i> (hmvm_seq.cpp:154-227), y zeroed first as the reference
 * proxy does (hmvm_seq.cpp:398-401).  Leaves in file order; low-rank leaves
 * (ltmtx==1) compute t = V x[cols] into a ktmax-long scratch (:176-185) then
 * add U t into y with the il-outer loop (a2i==0, :187-195) or the row-dot loop
 * (a2i==1, :196-205); every other ltmtx is treated as dense (:207-219). */
#define ORC_SEQ2(NAME, T)                                                                   \
  void NAME(int32_t nd, int32_t nlf, int32_t ktmax, const int32_t *ltmtx_, const int32_t *kt_,   \
            const int32_t *ndl_, const int32_t *ndt_, const int32_t *nstrtl_,                   \
            const int32_t *nstrtt_, const int64_t *a1, const int64_t *a2, const T *rowmat,       \
            const T *b, T *v, int a2i) {                                                       \
    T *tmp2 = malloc(sizeof(T) * (size_t)(ktmax > 0 ? ktmax : 1));                              \
    for (int32_t i = 0; i < nd; i++) v[i] = (T)0.0;                                             \
    for (int32_t i = 0; i < nlf; i++) {                                                         \
      int32_t ndl = ndl_[i], ndt = ndt_[i], nstrtl = nstrtl_[i], nstrtt = nstrtt_[i], kt = kt_[i]; \
      if (ltmtx_[i] == 1) {                                                                     \
        for (int32_t j = 0; j < kt; j++) tmp2[j] = (T)0.0;                                      \
        int64_t head = a1[i];                                                                   \
        for (int32_t il = 0; il < kt; il++)                                                     \
          for (int32_t it = 0; it < ndt; it++)                                                  \
            tmp2[il] += rowmat[head + it + (int64_t)il * ndt] * b[it + nstrtt - 1];             \
        head = a2[i];                                                                           \
        if (a2i == 0) {                                                                         \
          for (int32_t il = 0; il < kt; il++)                                                   \
            for (int32_t it = 0; it < ndl; it++)                                                \
              v[it + nstrtl - 1] += rowmat[head + it + (int64_t)il * ndl] * tmp2[il];           \
        } else {                                                                                \
          for (int32_t it = 0; it < ndl; it++) {                                                \
            T tmp1 = (T)0.0;                                                                    \
            for (int32_t il = 0; il < kt; il++)                                                 \
              tmp1 += rowmat[head + it + (int64_t)il * ndl] * tmp2[il];                         \
            v[it + nstrtl - 1] += tmp1;                                                         \
          }                                                                                     \
        }                                                                                       \
      } else {                                                                                  \
        int64_t head = a1[i];                                                                   \
        for (int32_t il = 0; il < ndl; il++) {                                                  \
          T tmp1 = (T)0.0;                                                                      \
          for (int32_t it = 0; it < ndt; it++)                                                  \
            tmp1 += rowmat[head + it + (int64_t)il * ndt] * b[it + nstrtt - 1];                 \
          v[il + nstrtl - 1] += tmp1;                                                           \
        }                                                                                       \
      }                                                                                         \
    }                                                                                           \
    free(tmp2);                                                                                 \
  }

ORC_SEQ2(orc_hmvm_seq2_d, double)
ORC_SEQ2(orc_hmvm_seq2_f, float)

/* FP64 -> FP32 cast of the stored elements (convertD2F, loadmatrix.cpp:300-330). */
void orc_cast_f(const double *src, float *dst, int64_t n) {
  for (int64_t i = 0; i < n; i++) dst[i] = (float)src[i];
}

/* Multi-RHS: column j of Y (leading dim ldy) = H * column j of X (leading dim
 * ldx); each column is an independent hmvm_seq_2<double,0>. */
void orc_hmvm_seq2_multi_d(int32_t nd, int32_t nlf, int32_t ktmax, const int32_t *ltmtx,
                           const int32_t *kt, const int32_t *ndl, const int32_t *ndt,
                           const int32_t *nstrtl, const int32_t *nstrtt, const int64_t *a1,
                           const int64_t *a2, const double *rowmat, const double *X, int64_t ldx,
                           double *Y, int64_t ldy, int32_t nrhs) {
  for (int32_t j = 0; j < nrhs; j++)
    orc_hmvm_seq2_d(nd, nlf, ktmax, ltmtx, kt, ndl, ndt, nstrtl, nstrtt, a1, a2, rowmat,
                    X + (int64_t)j * ldx, Y + (int64_t)j * ldy, 0);
}

/* hmvm_omp_2<double,0> (hmvm_omp.cpp:374-463): leaves split over threads with
 * `omp for` (static schedule), each thread accumulating into a private y
 * (zaut[nd]) over the rows [ls,le] it touched, then merged with `omp atomic`.
 * The merge order depends on thread timing, so results can differ from the
 * sequential order in the last bits. */
void orc_omp2_d(int32_t nd, int32_t nlf, int32_t ktmax, const int32_t *ltmtx_, const int32_t *kt_,
                const int32_t *ndl_, const int32_t *ndt_, const int32_t *nstrtl_,
                const int32_t *nstrtt_, const int64_t *a1, const int64_t *a2, const double *rowmat,
                const double *zu, double *zau, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel
  {
#pragma omp for
    for (int32_t i = 0; i < nd; i++) zau[i] = 0.0;
    double *zaut = calloc((size_t)(nd > 0 ? nd : 1), sizeof(double));
    double *zbut = malloc(sizeof(double) * (size_t)(ktmax > 0 ? ktmax : 1));
    int32_t ls = nd, le = 1;
#pragma omp for
    for (int32_t ip = 0; ip < nlf; ip++) {
      int32_t ndl = ndl_[ip], ndt = ndt_[ip], nstrtl = nstrtl_[ip], nstrtt = nstrtt_[ip];
      if (nstrtl < ls) ls = nstrtl;
      if (nstrtl + ndl - 1 > le) le = nstrtl + ndl - 1;
      if (ltmtx_[ip] == 1) {
        int32_t kt = kt_[ip];
        int64_t head = a1[ip];
        for (int32_t il = 0; il < kt; il++) {
          zbut[il] = 0.0;
          for (int32_t it = 0; it < ndt; it++)
            zbut[il] += rowmat[head + it + (int64_t)il * ndt] * zu[it + nstrtt - 1];
        }
        head = a2[ip];
        for (int32_t il = 0; il < kt; il++)
          for (int32_t it = 0; it < ndl; it++)
            zaut[it + nstrtl - 1] += rowmat[head + it + (int64_t)il * ndl] * zbut[il];
      } else if (ltmtx_[ip] == 2) {
        int64_t head = a1[ip];
        for (int32_t il = 0; il < ndl; il++) {
          double tmp1 = 0.0;
          for (int32_t it = 0; it < ndt; it++)
            tmp1 += rowmat[head + it + (int64_t)il * ndt] * zu[it + nstrtt - 1];
          zaut[il + nstrtl - 1] += tmp1;
        }
      }
    }
    for (int32_t il = ls - 1; il <= le - 1; il++) {
#pragma omp atomic
      zau[il] += zaut[il];
    }
    free(zaut);
    free(zbut);
  }
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
