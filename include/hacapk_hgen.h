/*
 * hacapk_hgen.h -- H-matrix generator and writer (C ABI).
 *
 * Builds an H-matrix with HACApK's construction rules for the point kernel
 * K(i,j) = 1/(4*pi*|p_i - p_j|) (K(i,i) = 1.0) on seeded point clouds, and
 * writes it in the reference's hmatrix_1.bin / hmatrix_2.bin formats.  It
 * stands in for the reference's Fortran construction + dump path, which needs
 * MPI and a Fortran compiler:
 *
 *   hgen_build         HACApK_generate (src_hdump/m_HACApK_use.f90:62-166):
 *                        cluster tree   HACApK_generate_cbitree  (src_hdump/m_HACApK_base.f90:994-1054)
 *                        bounding boxes HACApK_bndbox            (src_hdump/m_HACApK_base.f90:953-991)
 *                        block tree     HACApK_generate_leafmtx  (src_hdump/m_HACApK_base.f90:845-891)
 *                        leaf order     qsort_row/qsort_col      (src_hdump/m_HACApK_base.f90:245-255,893-935)
 *                        ACA            HACApK_aca               (src_hdump/m_HACApK_base.f90:494-577)
 *                        leaf fill      HACApK_fill_leafmtx_hyp  (src_hdump/m_HACApK_base.f90:580-662)
 *   hgen_write_bin1    HACApK_hdump_dump_leafmtx  (src_hdump/m_HACApK_hdump.f90:84-108)
 *   hgen_write_bin2    HACApK_hdump_dump_leafmtx2 (src_hdump/m_HACApK_hdump.f90:114-180)
 *
 * All functions return 0 on success and a negative HGEN_E* code on failure;
 * none of them exits the process.
 */
#ifndef HACAPK_HGEN_H
#define HACAPK_HGEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HGEN_OK 0
#define HGEN_EINVAL -1
#define HGEN_ENOMEM -2
#define HGEN_EIO -3
#define HGEN_ERANGE -4 /* a count does not fit the file format's int32 fields */

enum hgen_geometry {
  HGEN_SPHERE = 0,       /* uniform on the unit sphere */
  HGEN_CUBE_SURFACE = 1, /* uniform on the surface of the unit cube [0,1]^3 */
  HGEN_PLATE_2X1 = 2     /* uniform on the flat plate [0,2]x[0,1]x{0} */
};

typedef struct hgen_params {
  int64_t n;              /* number of points (= matrix order nd) */
  int32_t geometry;       /* enum hgen_geometry */
  int32_t leaf_size;      /* param(21): a cluster with <= leaf_size points is a leaf */
  double eta;             /* param(51): admissibility parameter */
  double eps;             /* param(71): ACA tolerance */
  double aca_eps_factor;  /* param(72): ACA_EPS = aca_eps_factor * eps (HACApK default 1e-3) */
  int32_t kmax;           /* param(63): rank cap per leaf (HACApK default 1000) */
  int32_t nthreads;       /* <= 0: OpenMP default */
  uint64_t seed;          /* point-cloud seed */
} hgen_params;

/* A triangle mesh in ppohBEM's .pbf text format (read by the reference driver,
 * src_hdump/bem-bb-fw-HACApK-0.5.0.f90:396-500): node count, node xyz lines,
 * face count, nodes per face (3), integer and real parameter counts per face,
 * the faces' 0-based node indices, then the per-face parameters. */
typedef struct hgen_mesh {
  int32_t nond, nofc, nond_on_face, nint_para_fc, ndble_para_fc, _pad0;
  double *nodes;        /* [nond * 3] xyz */
  int32_t *face2node;   /* [nofc * nond_on_face], 0-based */
  int32_t *int_para_fc; /* [nofc * nint_para_fc] (NULL if none) */
  double *dble_para_fc; /* [nofc * ndble_para_fc] (NULL if none) */
} hgen_mesh;

/* The generated matrix: the SoA view of src_hmvm/src_cpp/hacapk.h:23-36 with
 * 64-bit element offsets (a1/a2/len), plus the construction by-products. */
typedef struct hgen_hmatrix {
  int32_t nd, nlf, ktmax, _pad0;
  int64_t len;
  int32_t *ltmtx, *kt, *ndl, *ndt, *nstrtl, *nstrtt; /* [nlf]; nstrtl/nstrtt are 1-based */
  int64_t *a1, *a2;                                  /* [nlf] element offsets into rowmat */
  double *rowmat;                                    /* [len] leaf data, file order */
  int32_t *lod;       /* [nd] permutation: position (0-based) -> original point (1-based) */
  double *coords;     /* [nd*3] original points, xyz interleaved */
  int64_t n_lowrank, n_dense;
  int64_t aca_incomplete; /* leaves where HACApK would have stopped (m_HACApK_base.f90:565-575) */
  const hgen_mesh* mesh;  /* hgen_build_tree_mesh: the mesh (borrowed; keep it until the fill); else NULL */
} hgen_hmatrix;

void hgen_default_params(hgen_params* p);
/* hgen_build = hgen_build_tree + hgen_fill_leaves. */
int hgen_build(const hgen_params* p, hgen_hmatrix** out);
/* Points, cluster tree, block tree and leaf order only: the leaf arrays are
 * set, kt / a1 / a2 are 0, rowmat is NULL and len 0.  Fill it with
 * hgen_fill_leaves (host, OpenMP) or hmvm_b200_aca_fill (GPU, libhmvm_b200). */
int hgen_build_tree(const hgen_params* p, hgen_hmatrix** out);
/* The same for the ppohBEM collocation matrix of a triangle mesh: points are
 * the face centroids (src_hdump/m_ppohBEM_bembb2hacapk.f90), entry (i, j) is
 * face j's integral at face i's centroid (m_ppohBEM_matrix_element_ij.f90,
 * face_integral in m_ppohBEM_user_func.f90:49-100); nd = the face count and
 * p->n / p->geometry / p->seed are ignored.  The matrix keeps a pointer to the
 * mesh for its fill.  HACApK's own settings are leaf_size 15, eta 2, kmax 1000,
 * aca_eps_factor 1e-3 and eps = the driver's tolerance. */
int hgen_build_tree_mesh(const hgen_params* p, const hgen_mesh* mesh, hgen_hmatrix** out);
int hgen_read_pbf(const char* fname, hgen_mesh** out);
void hgen_free_mesh(hgen_mesh* mesh);
/* ACA for the low-rank leaves and kernel entries for the dense ones
 * (HACApK_fill_leafmtx_hyp, src_hdump/m_HACApK_base.f90:580-662); sets kt,
 * a1, a2, len, ktmax, aca_incomplete and allocates rowmat. */
int hgen_fill_leaves(hgen_hmatrix* m, const hgen_params* p);
void hgen_free(hgen_hmatrix* m);

/* Writers.  bin2's int32 `len` header field is written saturated at INT32_MAX
 * when the element count does not fit. */
int hgen_write_bin1(const hgen_hmatrix* m, const char* fname);
int hgen_write_bin2(const hgen_hmatrix* m, const char* fname);
/* The 64-bit variant of hmatrix_2.bin: the same records, but the header record
 * holds len as int64 (nd, nlf, ktmax: int32; 20 bytes), as
 * HACApK_hdump_dump_leafmtx2 writes it with `integer*8 :: len`. */
int hgen_write_bin64(const hgen_hmatrix* m, const char* fname);

/* Exact entry of the permuted matrix, row/col 1-based positions (for tests). */
double hgen_entry(const hgen_hmatrix* m, int32_t ill, int32_t itt);

#ifdef __cplusplus
}
#endif

#endif /* HACAPK_HGEN_H */
