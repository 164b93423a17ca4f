/*
 * hmvm_b200.h -- H-matrix-vector multiplication on one NVIDIA B200 (C ABI).
 *
 * A drop-in for the HMVM path of the reference harness (hacapk_hmvm,
 * src_hmvm/src_cpp): the same H-matrix structures and files, and y = H x over
 * the HACApK leaf list, computed by hand-written sm_100a kernels.
 *
 * Conventions
 *   - Every function returns HMVM_OK (0) or a negative HMVM_E* status; none of
 *     them exits the process (the reference prints and calls exit(-1),
 *     src_hmvm/src_cpp/hmvm_cuda0.cu:11).  hmvm_b200_last_error() gives the
 *     message of the calling thread's last failure.
 *   - Row/column indices nstrtl/nstrtt are 1-based, as written by HACApK.
 *   - The library owns the device memory of a plan; the caller owns x and y.
 *   - There is no CPU fallback: without a usable CUDA device, plan creation and
 *     every compute call return HMVM_ENODEV.
 */
#ifndef HMVM_B200_H
#define HMVM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define HMVM_OK 0
#define HMVM_EINVAL -1   /* bad argument or inconsistent leaf table */
#define HMVM_ENOMEM -2   /* host or device allocation failed */
#define HMVM_ECUDA -3    /* a CUDA runtime call failed */
#define HMVM_EIO -4      /* file could not be opened or read */
#define HMVM_EFORMAT -5  /* file is not a well-formed hmatrix_1.bin / hmatrix_2.bin */
#define HMVM_ERANGE -6   /* a count exceeds what the structure or format can hold */
#define HMVM_ENODEV -7   /* no usable CUDA device */
#define HMVM_EDEVICE -8  /* a kernel reported an error status */

/* ---- H-matrix structures ------------------------------------------------ */
/* Byte-compatible with the reference templates (src_hmvm/src_cpp/hacapk.h:5-36)
 * instantiated for double / float.  Low-rank leaf (ltmtx==1): rowmat[a1..] is
 * V^T as [kt][ndt], rowmat[a2..] is U as [kt][ndl]; dense leaf (ltmtx==2):
 * rowmat[a1..] is [ndl][ndt] row-major.  rowmat_t holds the same data with U
 * transposed to [ndl][kt] (loadmatrix.cpp:227-234). */
typedef struct hmvm_submatrix_d {
  int ltmtx, kt, ndl, ndt, nstrtl, nstrtt;
  double *a1, *a2, *a2t;
} hmvm_submatrix_d;
typedef struct hmvm_submatrix_f {
  int ltmtx, kt, ndl, ndt, nstrtl, nstrtt;
  float *a1, *a2, *a2t;
} hmvm_submatrix_f;

typedef struct hmvm_matrix_d {
  int nd, nlf, ktmax;
  int *nleavs;
  hmvm_submatrix_d *submat;
  int b1, b2, b3, e1, e2, e3;
} hmvm_matrix_d;
typedef struct hmvm_matrix_f {
  int nd, nlf, ktmax;
  int *nleavs;
  hmvm_submatrix_f *submat;
  int b1, b2, b3, e1, e2, e3;
} hmvm_matrix_f;

typedef struct hmvm_matrix2_d {
  int nd, nlf, ktmax, len;
  int *nleavs;
  int *ltmtx, *kt, *ndl, *ndt, *nstrtl, *nstrtt;
  int *a1, *a2;
  double *rowmat, *rowmat_t;
  int napprox, ndense;
  int *approx, *dense;
} hmvm_matrix2_d;
typedef struct hmvm_matrix2_f {
  int nd, nlf, ktmax, len;
  int *nleavs;
  int *ltmtx, *kt, *ndl, *ndt, *nstrtl, *nstrtt;
  int *a1, *a2;
  float *rowmat, *rowmat_t;
  int napprox, ndense;
  int *approx, *dense;
} hmvm_matrix2_f;

/* The same leaf table with 64-bit element offsets, for matrices whose stored
 * element count overflows matrix2's int `len` / `a1` / `a2`
 * (src_hmvm/src_cpp/hacapk.h:28,31).  `rowmat` is double or float as named by
 * the create call it is passed to. */
typedef struct hmvm_leaves64 {
  int32_t nd, nlf, ktmax, _pad0;
  int64_t len;
  const int32_t *ltmtx, *kt, *ndl, *ndt, *nstrtl, *nstrtt;
  const int64_t *a1, *a2;
  const void *rowmat;
} hmvm_leaves64;

/* ---- loaders (replace src_hmvm/src_cpp/loadmatrix.cpp) ------------------ */
/* Replaces loadHmatrix (loadmatrix.cpp:7-150): reads hmatrix_1.bin into the AoS
 * and SoA forms (mat may be NULL to skip the AoS copies).  Record markers and
 * leaf fields are validated; on error nothing is left allocated. */
int hmvm_b200_load_hmatrix(const char *fname, hmvm_matrix_d *mat, hmvm_matrix2_d *mat2);
/* Replaces loadHmatrix2 (loadmatrix.cpp:152-250): reads hmatrix_2.bin into SoA. */
int hmvm_b200_load_hmatrix2(const char *fname, hmvm_matrix2_d *mat2);
/* Replaces convertD2F (loadmatrix.cpp:252-342): FP64 -> FP32 copies; either
 * source may be NULL. */
int hmvm_b200_convert_d2f(hmvm_matrix_f *matF, hmvm_matrix2_f *matF2, const hmvm_matrix_d *matD,
                          const hmvm_matrix2_d *matD2);
/* File formats recognised by hmvm_b200_load_leaves64 (by the byte count of
 * the first record: 12, 16 and 20). */
#define HMVM_BIN1 1  /* hmatrix_1.bin: header nd, nlf, ktmax; per leaf a header record and its data */
#define HMVM_BIN2 2  /* hmatrix_2.bin: header nd, nlf, ktmax, int32 len; six int32[nlf] columns; data */
#define HMVM_BIN64 3 /* the bin2 layout with an int64 len (a 20-byte header record) */
/* Reads any of the three formats into a 64-bit leaf table whose arrays the
 * library allocates (rowmat: double); *format (may be NULL) receives the
 * format found.  Lifts the int len / a1 / a2 ceiling of loadHmatrix /
 * loadHmatrix2 (src_hmvm/src_cpp/hacapk.h:28,31; loadmatrix.cpp:13,38,70,100)
 * for the HACApK dump formats (src_hdump/m_HACApK_hdump.f90:84-108,114-180),
 * with the same validation as the loaders above.  A bin2 header whose len is
 * INT32_MAX is taken as saturated (its leaves may hold more elements). */
int hmvm_b200_load_leaves64(const char *fname, hmvm_leaves64 *out, int32_t *format);
/* Release a table filled by hmvm_b200_load_leaves64 (and only such a table). */
void hmvm_b200_free_leaves64(hmvm_leaves64 *lv);
/* Release what the loaders / convert allocated (the reference never frees). */
void hmvm_b200_free_matrix_d(hmvm_matrix_d *mat);
void hmvm_b200_free_matrix_f(hmvm_matrix_f *mat);
void hmvm_b200_free_matrix2_d(hmvm_matrix2_d *mat2);
void hmvm_b200_free_matrix2_f(hmvm_matrix2_f *mat2);

/* ---- plans: a leaf table repacked and resident on the GPU ---------------- */
typedef struct hmvm_plan hmvm_plan;

enum hmvm_precision {
  HMVM_FP64 = 0,  /* FP64 storage, FP64 arithmetic */
  HMVM_FP32 = 1,  /* FP32 storage, FP32 arithmetic (the reference's float mode) */
  HMVM_MIXED = 2  /* x, y in FP64; low-rank factors FP16 (or BF16) with per-column FP32-range
                     scales, FP8 E4M3 for columns whose rank-1 term is below
                     mixed_fp8_eps * |block|, FP32 for columns at or above
                     mixed_fp32_tau * |block|; dense leaves FP32, diagonal dense blocks FP64;
                     products summed in FP32 per segment, rows summed in FP64 */
};

enum hmvm_lr_format { HMVM_LR_FP16 = 0, HMVM_LR_BF16 = 1 };

typedef struct hmvm_plan_opts {
  int32_t precision;      /* enum hmvm_precision */
  int32_t device;         /* CUDA device ordinal, -1 = current device */
  int32_t max_tile_rows;  /* rows per row tile, 1..32 (0 = 32) */
  int32_t split_cols;     /* V panels are also cut every split_cols columns (0 = only by size) */
  int32_t stage1_cfg;     /* kernel configuration index for the V stage (-1 = default) */
  int32_t stage2_cfg;     /* kernel configuration index for the row stage (-1 = default) */
  int32_t ctas_per_sm;    /* persistent CTAs per SM (0 = default) */
  int32_t kernel;         /* 0: register-streaming tile kernel; 1 (default, -1): TMA-ring stream kernel */
  /* HMVM_MIXED only.  |block| is the largest rank-1 term norm |u_k||v_k| of the leaf. */
  double mixed_fp8_eps;   /* FP8 below this * |block| (default 1e-4, the ACA tolerance; 0 = no FP8) */
  double mixed_fp32_tau;  /* FP32 at or above this * |block| (> 1 = none; < 0, the default = 0.5 for FP16
                             factors, 0.05 for BF16, whose 8-bit significand needs more FP32 columns) */
  int32_t mixed_lr_format;/* enum hmvm_lr_format (default FP16) */
  int32_t nrhs_max;       /* right-hand sides per pass of hmvm_b200_apply_multi, 1..8 (default 1; items are
                             sized so that nrhs_max inputs per column fit the multi-RHS kernel's buffer);
                             16 on HMVM_MIXED plans: 16-column passes with the 16-bit factor runs on the
                             tensor cores (tcgen05); 32 or more on HMVM_FP32 and HMVM_MIXED plans: the wide
                             tensor-core form, 128 right-hand sides per pass with every product on tcgen05
                             (the matrix stored as FP16 -- BF16 for BF16-factor plans -- values and hi/lo
                             pairs) */
} hmvm_plan_opts;

typedef struct hmvm_plan_info {
  int32_t nd, nlf, n_lowrank, n_dense;
  int32_t precision, device, num_sms, _pad0;
  int64_t algorithmic_bytes; /* stored leaf elements once + x + y, as the reference stores them */
  int64_t device_bytes;      /* repacked matrix bytes resident on the GPU (incl. padding) */
  int64_t t_len;             /* length of the intermediate V x vector */
  int32_t stage1_tiles, stage2_tiles, stage1_teams, stage2_teams;
  int32_t split_rows, kernels_per_apply, stage1_cfg, stage2_cfg;  /* split_rows: rows finished by a reduction */
  int64_t flops;             /* 2 * stored elements */
  int64_t stage1_bytes;      /* algorithmic bytes of the V stage: V elements + x */
  int64_t stage2_bytes;      /* algorithmic bytes of the row stage: U + dense elements + x + y */
  int32_t kernel, ctas_per_sm;           /* ctas_per_sm: of the V stage */
  int64_t cols_fp32, cols_lr16, cols_fp8; /* HMVM_MIXED: low-rank columns per storage format */
  int32_t stage2_ctas_per_sm;             /* CTAs per SM of the row stage */
  int32_t nrhs_max;                       /* right-hand sides per multi-RHS pass (1: single-vector plan) */
} hmvm_plan_info;

void hmvm_b200_default_opts(hmvm_plan_opts *opts);

/* Build a plan from the reference's SoA structure (replaces the per-call
 * cudaMalloc/cudaMemcpy of every matrix2 array in hmvm_cuda1.cu:333-353 with a
 * one-time repack + upload).  For HMVM_FP32 from a double matrix the elements
 * are rounded to float exactly as convertD2F does. */
int hmvm_b200_plan_create_d(const hmvm_matrix2_d *mat2, const hmvm_plan_opts *opts, hmvm_plan **plan);
int hmvm_b200_plan_create_f(const hmvm_matrix2_f *mat2, const hmvm_plan_opts *opts, hmvm_plan **plan);
/* 64-bit leaf table, rowmat in double / float. */
int hmvm_b200_plan_create64_d(const hmvm_leaves64 *lv, const hmvm_plan_opts *opts, hmvm_plan **plan);
int hmvm_b200_plan_create64_f(const hmvm_leaves64 *lv, const hmvm_plan_opts *opts, hmvm_plan **plan);
void hmvm_b200_plan_destroy(hmvm_plan *plan);
int hmvm_b200_plan_get_info(const hmvm_plan *plan, hmvm_plan_info *info);

/* y = H x with x, y in device memory of the plan's device (double for FP64
 * plans, float for FP32 plans); y is overwritten, x and y must not overlap.
 * Launches asynchronously on `stream` (a cudaStream_t, NULL = legacy default
 * stream).  The kernels sum in a fixed order, so repeated calls on the same
 * inputs give bitwise-identical y.  Replaces the kernel launch of
 * hmvm_cuda{0,1,2,3} (e.g. hmvm_cuda2.cu:262-306). */
int hmvm_b200_apply(hmvm_plan *plan, const void *x_dev, void *y_dev, void *stream);
/* The same with host buffers: copies x in, runs, copies y out, and waits for
 * the stream. */
int hmvm_b200_apply_host(hmvm_plan *plan, const void *x_host, void *y_host, void *stream);
/* Records one apply (y = H x for these device buffers) into a CUDA graph the
 * plan keeps (a new capture replaces the previous one; the buffers must stay
 * valid while it is replayed; profiling must be off), and launches it with one
 * cudaGraphLaunch.  For small matrices an apply is 2-5 kernels whose host
 * launch cost exceeds their device time; a solver loop replays instead.  The
 * reference launches its kernel per call (hmvm_cuda2.cu:262-306) and has no
 * counterpart. */
int hmvm_b200_plan_capture(hmvm_plan *plan, const void *x_dev, void *y_dev);
int hmvm_b200_plan_replay(hmvm_plan *plan, void *stream);

/* Y = H X for nrhs right-hand sides: X and Y column-major in device memory
 * (column r at X + r * ldx, ldx >= N; same for Y), element type as for
 * hmvm_b200_apply.  Plans created with opts.nrhs_max > 1 run passes of up to
 * nrhs_max (8 at most) columns through the multi-RHS kernel, each pass
 * streaming the matrix once; plans with nrhs_max = 1 run nrhs single-vector
 * applies.  Each column of Y is computed in a fixed order (repeatable bit for
 * bit; it may differ in the last bits from the single-vector apply).  The
 * reference has no multi-RHS entry point: its hmvm_cuda* wrappers take one b
 * (hmvm_cuda.h:4-7). */
int hmvm_b200_apply_multi(hmvm_plan *plan, const void *X_dev, int64_t ldx, void *Y_dev, int64_t ldy, int32_t nrhs,
                          void *stream);
/* The same with host buffers (copies in, runs, copies out, waits). */
int hmvm_b200_apply_multi_host(hmvm_plan *plan, const void *X_host, int64_t ldx, void *Y_host, int64_t ldy,
                               int32_t nrhs, void *stream);
/* Kernels one hmvm_b200_apply_multi call with nrhs columns launches. */
int hmvm_b200_plan_multi_kernel_count(const hmvm_plan *plan, int32_t nrhs);

/* ---- batches of independent H-matrices -------------------------------------
 * Many H-matrices of uneven N planned together.  Instances are grouped into
 * classes by the right-hand sides they will be applied with (nrhs[m] at
 * creation; NULL = opts->nrhs_max for all): pass width 1, 2, 4 or 8 (more than
 * 8 columns run several 8-wide passes).  Each class is one block-diagonal plan
 * (instance m owns rows/columns [offset, offset + N_m) of its class's
 * concatenated index space), so each stage of a class is one persistent launch
 * over all its instances' items.  The reference has no batched entry point.
 * Instances share the plan options other than nrhs_max. */
typedef struct hmvm_batch hmvm_batch;
int hmvm_b200_batch_create64_d(const hmvm_leaves64 *mats, int32_t count, const hmvm_plan_opts *opts,
                               const int32_t *nrhs, hmvm_batch **batch);
int hmvm_b200_batch_create64_f(const hmvm_leaves64 *mats, int32_t count, const hmvm_plan_opts *opts,
                               const int32_t *nrhs, hmvm_batch **batch);
int hmvm_b200_batch_create_d(const hmvm_matrix2_d *mats, int32_t count, const hmvm_plan_opts *opts,
                             const int32_t *nrhs, hmvm_batch **batch);
void hmvm_b200_batch_destroy(hmvm_batch *batch);
/* Sums over the classes' plans (nd, leaves, bytes, tiles, ...); the other
 * fields are those of the first class. */
int hmvm_b200_batch_get_info(const hmvm_batch *batch, hmvm_plan_info *info);
int hmvm_b200_batch_instance(const hmvm_batch *batch, int32_t m, int32_t *n, int32_t *cls, int64_t *offset);
int hmvm_b200_batch_class_count(const hmvm_batch *batch);
/* Y_m = H_m X_m for every instance m < count: X[m], Y[m] device pointers to
 * column-major N_m x nrhs[m] blocks with leading dimensions ldx[m], ldy[m]
 * (arrays of `count` entries in host memory; 0 columns skips the instance; an
 * instance given more columns than its class width runs more passes). */
int hmvm_b200_batch_apply(hmvm_batch *batch, const void *const *X, const int64_t *ldx, void *const *Y,
                          const int64_t *ldy, const int32_t *nrhs, void *stream);
/* Record the launches of hmvm_b200_batch_apply for these buffers into a CUDA
 * graph kept by the batch (replacing an earlier one); hmvm_b200_batch_launch
 * replays it on `stream` with one cudaGraphLaunch. */
int hmvm_b200_batch_capture(hmvm_batch *batch, const void *const *X, const int64_t *ldx, void *const *Y,
                            const int64_t *ldy, const int32_t *nrhs);
int hmvm_b200_batch_launch(hmvm_batch *batch, void *stream);
int hmvm_b200_batch_status(hmvm_batch *batch);
/* Kernels one apply (or one graph replay) launches for the columns last given. */
int hmvm_b200_batch_kernel_count(const hmvm_batch *batch);

/* ---- Krylov solver on a resident plan ---------------------------------------
 * Solves H u = b by BiCGSTAB, restating HACApK_bicgstab_lfmtx
 * (src_lhdump/m_HACApK_solve.f90:977-1028): u_dev holds the initial guess and
 * receives the solution; at most max_steps steps, stopping when
 * ||b - H u|| / ||b|| < eps.  b and u are device vectors of the plan's x / y
 * type; two HMVMs (hmvm_b200_apply) per step, inner products summed in a fixed
 * order (repeatable).  *steps and *relres receive the steps taken and the
 * final relative residual.  Returns HMVM_EINVAL on a breakdown (a vanishing
 * BiCGSTAB scalar).  Allocates 7 work vectors for the call. */
int hmvm_b200_bicgstab(hmvm_plan *plan, const void *b_dev, void *u_dev, int32_t max_steps, double eps,
                       int32_t *steps, double *relres, void *stream);
/* Solves H u = b by GCR(m), restating HACApK_gcrm_lfmtx
 * (src_lhdump/m_HACApK_solve.f90:1277-1342; max_steps = param(83), restart =
 * m = param(87) in 1..64, eps = param(91)): one HMVM per step, each new search
 * direction A-orthogonalised against the last `restart` (stored cyclically).
 * Same conventions as hmvm_b200_bicgstab; HMVM_EINVAL on a breakdown (A p = 0).
 * Allocates 2 + 2 * restart work vectors for the call. */
int hmvm_b200_gcrm(hmvm_plan *plan, const void *b_dev, void *u_dev, int32_t max_steps, int32_t restart, double eps,
                   int32_t *steps, double *relres, void *stream);

/* ---- leaf fill on the GPU ------------------------------------------------------
 * Fills a matrix from hgen_build_tree (include/hacapk_hgen.h) on `device`: ACA
 * for its low-rank leaves (HACApK_aca, src_hdump/m_HACApK_base.f90:494-577)
 * and kernel entries for its dense leaves (HACApK_fill_leafmtx_hyp, :580-662),
 * with results bit-identical to hgen_fill_leaves (point-kernel matrices only;
 * a matrix from hgen_build_tree_mesh is refused).  Sets kt, a1, a2, len, ktmax
 * and aca_incomplete and allocates rowmat (malloc; hgen_free releases it).
 * The matrix is left unchanged on failure. */
struct hgen_hmatrix;
struct hgen_params;
typedef struct hmvm_aca_report {
  int32_t rounds;        /* capacity rounds (32, 128, 512, ... terms per leaf) */
  int32_t ktmax;
  int64_t scratch_bytes; /* device factor scratch over all rounds */
  double ms_aca;         /* device time of the ACA rounds */
  double ms_dense;       /* ... of the dense-leaf fill */
  double ms_gather_copy; /* ... of packing the factors and copying rowmat to the host */
} hmvm_aca_report;
int hmvm_b200_aca_fill(struct hgen_hmatrix *m, const struct hgen_params *p, int32_t device,
                       hmvm_aca_report *report);

/* ---- autotuner ---------------------------------------------------------------
 * Picks, per leaf shape class -- the V stage (stacked low-rank V factors) and
 * the row stage (row tiles of dense leaves and U factors) -- the kernel
 * configuration that runs fastest on the current device for this very matrix:
 * one warp per team (stream kernel) or warp groups per tile item (tile kernel),
 * their ring / buffer / group shapes, and the rows per row tile.  Every
 * candidate plan is built and timed stage by stage (reps applies, CUDA events;
 * building a plan costs about a second per million leaves); the best stage
 * configurations are combined and timed as well.  `best` receives `base` with
 * kernel, stage1_cfg, stage2_cfg and max_tile_rows of the fastest measured
 * plan; pass it to hmvm_b200_plan_create*.  Replaces the hand-tuned warp/block
 * thresholds of the reference's hmvm_cuda_hybrid kernels (hmvm_cuda1.cu). */
#define HMVM_TUNE_MAX_ENTRIES 64
typedef struct hmvm_tune_entry {
  int32_t kernel, stage1_cfg, stage2_cfg, max_tile_rows;
  int32_t ctas_per_sm, _pad0;
  double stage1_ms, stage2_ms, total_ms; /* per apply; each stage with its reduction */
} hmvm_tune_entry;
typedef struct hmvm_tune_report {
  int32_t n_entries, best_entry;
  hmvm_tune_entry entries[HMVM_TUNE_MAX_ENTRIES];
} hmvm_tune_report;
int hmvm_b200_autotune64(const hmvm_leaves64 *lv, int32_t rowmat_is_float, const hmvm_plan_opts *base, int32_t reps,
                         hmvm_plan_opts *best, hmvm_tune_report *report);
int hmvm_b200_autotune_d(const hmvm_matrix2_d *mat2, const hmvm_plan_opts *base, int32_t reps,
                         hmvm_plan_opts *best, hmvm_tune_report *report);
/* Shape classes and a persistent choice (no counterpart in the reference, which
 * re-runs its offline sweeps per matrix, src_hmvm/src_cpp/hmvm1.cpp:82-89).
 * hmvm_b200_shape_histogram64 fills hist[HMVM_SHAPE_BINS] with the fraction of
 * the matrix's stored elements in each (kind, rows, width) class: bins 0..63
 * dense leaves, 64..127 low-rank leaves; within a kind 8 row buckets (<= 8, 16,
 * ..., 512, above) times 8 width buckets (dense: columns <= 8 .. above 512;
 * low-rank: rank <= 2 .. above 128).
 * hmvm_b200_autotune_cached64 looks in the text file cache_path for a choice
 * stored for this device (name and SM count), precision and factor format
 * whose histogram lies within max_distance of this matrix's (L1 distance, in
 * [0, 2]; a negative value means 0.45, which joins generated matrices of one
 * family within 2x in size and keeps other geometries apart), and returns the
 * closest one without timing anything (*from_cache = 1; report holds that one
 * entry).  Otherwise it runs hmvm_b200_autotune64 and appends the fastest
 * measured choice, with the histogram, to the file (created if missing). */
#define HMVM_SHAPE_BINS 128
int hmvm_b200_shape_histogram64(const hmvm_leaves64 *lv, float *hist);
int hmvm_b200_autotune_cached64(const hmvm_leaves64 *lv, int32_t rowmat_is_float, const hmvm_plan_opts *base,
                                int32_t reps, const char *cache_path, double max_distance, hmvm_plan_opts *best,
                                hmvm_tune_report *report, int32_t *from_cache);

/* Capacity of the scratch array used by hmvm_b200_apply_noalloc: 16 MiB. */
#define HMVM_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)

/* y = H x exactly like hmvm_b200_apply, for callers that must not allocate GPU
 * memory while they run: a solver embedded in an application that hands out
 * all device memory from its own pool and forbids further cudaMalloc/cudaFree
 * once it is running, or code whose device-memory budget is fixed at start-up.
 * This call allocates nothing.  Its scratch -- the intermediate V x vector and
 * the partial sums of split panels -- lives in one library-wide array of
 * HMVM_NOALLOC_SCRATCH_BYTES in device memory, which every GPU that loads the
 * library holds until the process exits.  The array is reserved on a device
 * when the library's kernels are loaded there: under CUDA's default lazy module
 * loading that happens during the first plan creation on that device, not when
 * the library is loaded, so a caller with a fixed memory budget should create its
 * plans before it hands the remaining memory to its own pool.  A plan whose scratch (t_len + 16 and
 * p_len + 16 elements, each rounded up to 256 bytes; see hmvm_plan_info.t_len)
 * does not fit is rejected with HMVM_ERANGE.  The first call on each device
 * looks up that array's device address (once per device and context, with
 * that device current; a new context after cudaDeviceReset looks it up again);
 * make that first call before any stream capture.  All calls share
 * the array and it keeps the last call's contents: the call clears, on
 * `stream` and before its kernels, the part that has to start at zero.  Calls
 * whose work overlaps on the GPU (other streams, threads or plans running at
 * the same time) race on the array; order them on one stream or synchronise
 * between them.  No counterpart in the reference. */
int hmvm_b200_apply_noalloc(hmvm_plan *plan, const void *x_dev, void *y_dev, void *stream);

/* Per-stage device timing.  While enabled, every apply records CUDA events
 * around its launches on the launch stream (up to 4096 applies are kept);
 * profile_read waits for the last recorded apply, returns the summed
 * milliseconds of stage 0 (V stage), 1 (its reduction), 2 (row stage), 3 (its
 * reduction) and the number of applies, and clears the record. */
int hmvm_b200_plan_profile(hmvm_plan *plan, int enable);
int hmvm_b200_plan_profile_read(hmvm_plan *plan, double *stage_ms4, int32_t *napplies);

/* Device-side status of the plan's kernels: HMVM_OK, or HMVM_EDEVICE if a
 * kernel gave up on a bounded wait since the last call (the wait's results are
 * not valid then).  Waits for the plan's device to finish its work; clears the
 * flag. */
int hmvm_b200_plan_status(hmvm_plan *plan);

/* ---- one-shot call with the reference's shape ---------------------------- */
typedef struct hmvm_stats {
  double seconds_setup;  /* plan creation (repack + upload) */
  double seconds_apply;  /* device time of the HMVM itself (CUDA events) */
  int64_t algorithmic_bytes;
  double gbytes_per_s;   /* algorithmic bytes / seconds_apply / 1e9 */
} hmvm_stats;

/* y = H x from host arrays: plan, apply once, release (the reference's
 * hmvm_cuda<T>(mat2, b, kernel, dump, nbench) minus the dump and timing loop,
 * with an output argument the reference lacks).  stats may be NULL. */
int hmvm_cuda_d(const hmvm_matrix2_d *mat2, const double *x, double *y, int mode, hmvm_stats *stats);
int hmvm_cuda_f(const hmvm_matrix2_f *mat2, const float *x, float *y, int mode, hmvm_stats *stats);

/* ---- inspection (host only; no GPU needed) ------------------------------ */
/* Builds the repacked layout on the host exactly as plan creation does, so it
 * can be checked without a device.  Arrays stay owned by the layout. */
typedef struct hmvm_layout hmvm_layout;
typedef struct hmvm_layout_view {
  int32_t precision, vec;            /* vec = elements per 16-byte vector */
  int32_t n_tiles, n_segs;           /* all stages */
  int32_t stage1_tiles, stage2_tiles; /* tiles [0,stage1) are stage 1, then stage 2 */
  int32_t stage1_teams, stage2_teams;
  int32_t n_red1, n_red2, nd, kernel;
  int64_t data_vectors;              /* 16-byte vectors in the data stream */
  int64_t t_len, p_len;
  const void *tiles;                 /* hmvm_tile_desc[n_tiles] */
  const void *segs;                  /* hmvm_seg_desc[n_segs] */
  const int32_t *team_begin1;        /* [stage1_teams+1], indexes tiles */
  const int32_t *team_begin2;        /* [stage2_teams+1], indexes tiles */
  const int32_t *out_idx;            /* stage-1 output slots */
  const int32_t *red1;               /* [n_red1][4]: t slot, partial base, parts, 0 */
  const int32_t *red2;               /* [n_red2][4]: y row, partial base, parts, 0 */
  const void *data;                  /* data_vectors * 16 bytes */
  const double *rowscale;            /* HMVM_MIXED: [n_rowscale] s_u * s_v per V-stage output row, in
                                        stage-1 item order (tile _pad = first index of the tile) */
  int64_t n_rowscale;
  /* wide tensor-core layout (FP32 / mixed plans with nrhs_max >= 32); segment formats in the top bits of
     ncols: 0 one 16-bit value per element, 1 a 16-bit hi/lo pair, stored K-step-major */
  int32_t tcw, tcw_bf16;             /* 16-bit format: FP16 (0) or BF16 (1) */
  const float *tscale;               /* [n_tscale]: per V-stage panel row 2^-c (tile _pad = first index of the
                                        tile), from tscale_rows0 on the row scale s_i of every y row */
  int64_t n_tscale;
  int32_t tscale_rows0, _pad_view;
  const int32_t *tblocks;            /* [n_tiles]: rows of the item's row blocks 0..3, 8 bits each (block b's
                                        rows follow block b-1's); segment ncols bits 24..27 select the blocks a
                                        segment multiplies, and consecutive segments with one input range share it */
  /* the step program the kernel's producer walks: per input group 4 words (src word, 8-column vectors,
     rows per K step | MMAs << 16 | item's last group << 20, first MMA template), per MMA 2 words (first B row
     | A lo part << 12 | block << 13 | block rows * 16 << 16, tcgen05 instruction descriptor) */
  const uint32_t *tgroups;           /* [n_tgroups][4] */
  const uint32_t *tops;              /* [n_tops][2] (+ 12 zero templates) */
  const int32_t *tgfirst;            /* [n_tiles + 1]: first input group of each item */
  int64_t n_tgroups, n_tops;
} hmvm_layout_view;

/* Tile and segment records as stored in the data structures above. */
typedef struct hmvm_tile_desc {
  int64_t data_off;  /* first 16-byte vector of the tile in the data stream */
  int32_t seg_begin, nseg, nvec, out_base;
  int16_t nrows, mode; /* mode 0: y[out_base+r]; 1: t[out_idx[out_base+r]]; 2: partial[out_base+r] */
  int32_t _pad;
} hmvm_tile_desc;
typedef struct hmvm_seg_desc {
  int32_t src;   /* x index, or (t index | 0x80000000) */
  int32_t ncols; /* HMVM_MIXED: low 28 bits columns, high bits the storage type
                    (0 FP64, 1 FP32, 2 FP16, 3 FP8 E4M3, 4 BF16) */
} hmvm_seg_desc;

int hmvm_b200_layout_build_d(const hmvm_matrix2_d *mat2, const hmvm_plan_opts *opts, int32_t num_sms,
                             hmvm_layout **layout);
int hmvm_b200_layout_build64(const hmvm_leaves64 *lv, int32_t rowmat_is_float, const hmvm_plan_opts *opts,
                             int32_t num_sms, hmvm_layout **layout);
/* Bounds checks of every descriptor of a single-vector layout against the
 * buffers it indexes: each item's data-stream range, segment range, rows, the
 * x or t columns of its segments, its padded inputs against the stage kernel's
 * input buffer, the y / t / partial-sum rows it writes, its t slots and row
 * scales, every reduction entry, and the team ranges.  HMVM_OK, or HMVM_ERANGE
 * with a message naming the first failing item.  Wide tensor-core layouts
 * (view.tcw = 1) are not described by these checks and return HMVM_OK.  The
 * library built with HMVM_DEVICE_CHECKS (libhmvm_b200_checked.so) runs the same
 * checks at plan creation and on the device before every single-vector stage
 * launch: a violation sets the status word (hmvm_b200_plan_status returns
 * HMVM_EDEVICE) and the stage kernels then touch no memory.  The reference
 * checks none of its offsets (hmvm_seq.cpp, hmvm_cuda2.cu index the leaf
 * arrays directly). */
int hmvm_b200_layout_validate(const hmvm_layout *layout);
/* The device address of a plan's item descriptors (hmvm_tile_desc[n_tiles],
 * stage-1 items first), for inspection and for tests of the device checks;
 * a caller that changes them owns the consequences (the HMVM_DEVICE_CHECKS
 * build reports descriptors that leave their buffers instead of following
 * them). */
int hmvm_b200_plan_descriptors(const hmvm_plan *plan, void **tiles_dev, int32_t *n_tiles, int32_t *stage1_tiles);
int hmvm_b200_layout_view(const hmvm_layout *layout, hmvm_layout_view *view);
void hmvm_b200_layout_destroy(hmvm_layout *layout);

/* ---- misc --------------------------------------------------------------- */
const char *hmvm_b200_strerror(int status);
const char *hmvm_b200_last_error(void);
int hmvm_b200_version(void);
/* Number of kernel launches one apply issues for this plan. */
int hmvm_b200_plan_kernel_count(const hmvm_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* HMVM_B200_H */
