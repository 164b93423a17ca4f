// Host-side planner: turns a HACApK leaf list into the repacked, row-owned
// layout that the sm_100a kernels stream.  No CUDA calls here.
//
// Layout (one data stream of 16-byte vectors, T = double or float, VEC = 16/sizeof(T)):
//
//  * The HMVM is split into two block-sparse matrix-vector stages over one
//    combined input z = [x ; t]:
//      stage 1  t = V x      one "panel" per (column cluster, 32 rows): the rows
//                            of V^T of every low-rank leaf that shares the
//                            column range (nstrtt, ndt) are stacked, so a warp
//                            lane owns one (leaf, k) row and all lanes share x.
//      stage 2  y = D x + U t  one "tile" per row interval of <= 32 rows whose
//                            ends are leaf row boundaries; its segments are the
//                            dense leaves over those rows (adjacent column
//                            ranges merged) and, per row cluster, the U factors
//                            of all low-rank leaves on that cluster (their t
//                            entries are contiguous: "slots" ordered by row
//                            cluster).
//  * A tile is stored column-major in vectors: vector v of a tile with R rows
//    is R consecutive 16-byte records (lane r holds columns v*VEC..v*VEC+VEC-1
//    of row r), so one warp-wide load reads R*16 contiguous bytes and every
//    lane accumulates its own row: no shuffles and no atomics, and the
//    summation order is fixed by the layout.
//  * Tiles larger than a per-stage bound are cut into "items": contiguous
//    vector ranges (segments trimmed to the range) that write partial sums; a
//    small reduction adds the parts in order into t (stage 1) or y (stage 2).
//  * Items are assigned to persistent "teams" (a warp, or a group of warps) by
//    LPT on their byte cost and stored in team order, so a team streams one
//    contiguous region of HBM.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "hmvm_b200.h"

namespace hmvm {

struct alignas(16) Vec16 {
  uint32_t w[4];
};

// Allocator whose resize() leaves new elements uninitialised (default- rather
// than value-initialised).  The packed matrix is gigabytes and the planner's
// parallel pack writes every byte of it, so zeroing it first on one thread
// only cost time (3.3 of the 3.9 s of an FP64 layout at N = 262,144 on 8
// threads); its pages are now first touched by the packing threads.
template <class T>
struct UninitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = UninitAlloc<U>;
  };
  UninitAlloc() = default;
  template <class U>
  UninitAlloc(const UninitAlloc<U>&) noexcept {}
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    if constexpr (sizeof...(A) == 0) ::new (static_cast<void*>(p)) U;
    else ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};

// Normalised view of the caller's leaf table (64-bit offsets).
struct LeafTable {
  int32_t nd = 0, nlf = 0, ktmax = 0;
  int64_t len = 0;
  const int32_t *ltmtx = nullptr, *kt = nullptr, *ndl = nullptr, *ndt = nullptr, *nstrtl = nullptr,
                *nstrtt = nullptr;
  const int32_t *a1_32 = nullptr, *a2_32 = nullptr;  // one of the offset pairs is set
  const int64_t *a1_64 = nullptr, *a2_64 = nullptr;
  const void *rowmat = nullptr;
  bool rowmat_is_float = false;
  int64_t a1(int32_t i) const { return a1_64 ? a1_64[i] : (int64_t)a1_32[i]; }
  int64_t a2(int32_t i) const { return a2_64 ? a2_64[i] : (int64_t)a2_32[i]; }
};

// Kernel variants.
//   0: hmvm_tile_kernel   -- teams of WG warps split a tile's vectors; data
//                            streamed with 16-byte register loads.
//   1: hmvm_stream_kernel -- one warp per team; each warp streams its contiguous
//                            region through a private shared-memory ring filled
//                            by cp.async.bulk (TMA bulk copies) ahead of use.
// Configurations of variant 0: warps per team (WG) and teams per CTA (TPC).
struct KernelCfg {
  int wg, tpc;
};
constexpr int kNumCfgs = 8;
constexpr KernelCfg kCfgs[kNumCfgs] = {{1, 8}, {2, 4}, {4, 2}, {8, 1}, {2, 8}, {4, 4}, {8, 2}, {16, 1}};
// Configurations of variant 1: warps per CTA, ring slots per warp, slot bytes,
// and zcap, the x/t columns one item may read (the size of each of the warp's
// two input buffers in shared memory).
struct StreamCfg {
  int wpb, slots, chunk, zcap;
};
constexpr int kNumStreamCfgs = 8;
constexpr StreamCfg kStreamCfgs[kNumStreamCfgs] = {{8, 4, 1024, 256}, {4, 4, 2048, 512}, {8, 4, 2048, 256},
                                                   {16, 4, 1024, 128}, {4, 8, 1024, 512}, {8, 8, 512, 256},
                                                   {8, 2, 4096, 256},  {4, 4, 4096, 512}};
inline int stream_smem_bytes(const StreamCfg& c, int elem) {
  return c.wpb * (c.slots * c.chunk + 2 * c.zcap * elem + c.slots * 8);
}
inline int teams_per_cta(int kernel, int cfg) { return kernel == 0 ? kCfgs[cfg].tpc : kStreamCfgs[cfg].wpb; }
constexpr int kDefaultKernel = 1;
constexpr int kDefaultStage1Cfg = 4;  // variant 0 defaults
constexpr int kDefaultStage2Cfg = 5;
constexpr int kDefaultCtasPerSm = 2;
constexpr int kDefaultStreamCfg = 7;  // variant 1 defaults
constexpr int kDefaultStreamCtasPerSm = 2;  // plans use the occupancy the device reports
constexpr int kMaxRows = 32;
// Item split: a stage's tiles are cut so that no item exceeds
// max(kMinItemBytes, stage bytes / (teams * kItemsPerTeam)).
constexpr int64_t kMinItemBytes = 32 * 1024;
// A stage below this many bytes is cut finer (items of at least
// kSmallItemBytes, about one per team): there every team holds at most an item
// or two and the stage takes as long as its longest item.
constexpr int64_t kSmallStageBytes = 8 << 20;
constexpr int64_t kSmallItemBytes = 4 * 1024;
constexpr int64_t kItemsPerTeam = 6;
constexpr int64_t kItemOverheadBytes = 1024;

// Element type of a segment's matrix data (mixed-precision plans encode it in
// the top bits of hmvm_seg_desc.ncols; plain plans leave those bits zero).
enum SegType : int32_t { ST_F64 = 0, ST_F32 = 1, ST_F16 = 2, ST_E4M3 = 3, ST_BF16 = 4 };
constexpr int kSegTypeShift = 28;
constexpr int32_t kSegColsMask = (1 << kSegTypeShift) - 1;
inline int seg_vec(int type) {  // matrix elements per 16-byte vector
  return type == ST_F64 ? 2 : type == ST_F32 ? 4 : type == ST_E4M3 ? 16 : 8;
}
inline int seg_zbytes(int type) {  // input bytes per 16-byte vector (x in FP64 for F64, else FP32)
  return type == ST_F64 ? 16 : seg_vec(type) * 4;
}
// Mixed-precision stream kernel: segments per item (one descriptor per lane)
// and configurations: warps per CTA, ring slots, slot bytes, and the bytes of
// each of the warp's two input buffers.
constexpr int kMixedMaxSegs = 32;
struct MixedCfg {
  int wpb, slots, chunk, zbytes;
};
constexpr int kNumMixedCfgs = 11;
constexpr MixedCfg kMixedCfgs[kNumMixedCfgs] = {{8, 4, 2048, 2048}, {8, 4, 1024, 4096}, {8, 4, 2048, 4096},
                                                {4, 4, 2048, 4096}, {6, 4, 2048, 4096}, {16, 4, 1024, 2048},
                                                {8, 2, 4096, 2048}, {4, 4, 4096, 2048}, {6, 2, 4096, 4096},
                                                {4, 2, 8192, 2048}, {5, 2, 8192, 2048}};
inline int mixed_smem_bytes(const MixedCfg& c) { return c.wpb * (c.slots * c.chunk + 2 * c.zbytes + c.slots * 8); }
// Default configuration of a stage (1: V stage, 2: row stage) for a plan's
// precision and kernel variant.  Stream kernel: 4 warps x 16 KB rings for FP64
// and for the FP32 V stage; the FP32 row stage runs fastest with 4 warps x
// 4 x 2 KB (cfg 1: 0.445 against 0.454 ms at N = 262,144).
int default_stage_cfg(int precision, int kernel, int stage);
// defaults measured at N = 262,144 with each stage at its own resident CTAs
// per SM: 5 warps x (2 slots of 8 KB) for the V stage, 6 warps x (2 slots of
// 4 KB) for the row stage, 2 CTAs per SM each (0.473 ms against 0.518 ms
// with 4 x (4 slots of 4 KB) and 6 x (4 slots of 2 KB): half the bulk-copy
// issues per byte, and one more warp per CTA in the V stage)
constexpr int kDefaultMixedCfg1 = 10;
constexpr int kDefaultMixedCfg2 = 8;

// Multi-RHS kernel (hmvm_multi_kernel): rhs per pass and its input buffer.
constexpr int kMaxNrhsPass = 8;   // CUDA-core multi-RHS passes
constexpr int kTcNrhs = 16;        // tensor-core passes (mixed plans with nrhs_max = 16)
constexpr int kTcWarpsPerSm = 7;   // resident warps (teams) per SM of the tensor-core kernel
// Each warp's two input buffers of the multi-RHS kernel (an item's x/t columns
// for all of a pass's right-hand sides): 4 KiB each lets 3 CTAs of 4 warps
// share an SM (12 warps; 8 with 8 KiB: 12 % faster at 8 FP32 right-hand sides).
// FP64 plans keep 8 KiB and 8 warps: their inputs are twice as wide, and 4 KiB
// cut their items twice as often (10 % slower at 8 right-hand sides).
constexpr int kMultiZBytes = 4096;
constexpr int kMultiZBytesF64 = 8192;
constexpr int multi_zbytes(bool f64) { return f64 ? kMultiZBytesF64 : kMultiZBytes; }
// An item's inputs for the 16-wide tensor-core pass (its kernel's buffer is kTcZBytes).
constexpr int kTcItemZBytes = 8192;
struct MultiCfg {
  int wpb, slots, chunk;
};
// one shape: 4 warps per CTA, a ring of 2 x 4 KiB per warp (faster than the
// 4 x 2 KiB and 8 x 1 KiB rings it replaced)
constexpr int kNumMultiCfgs = 1;
constexpr MultiCfg kMultiCfgs[kNumMultiCfgs] = {{4, 2, 4096}};
inline int multi_smem_bytes(const MultiCfg& c, bool f64) {
  return c.wpb * (c.slots * c.chunk + 2 * multi_zbytes(f64) + c.slots * 8);
}
constexpr int kDefaultMultiCfg = 0;
constexpr int kMultiWarpsPerSm = 12;    // resident warps (teams) per SM of the multi-RHS kernel
constexpr int kMultiWarpsPerSmF64 = 8;  // the same for FP64 plans (8 KiB input buffers)

// Wide tensor-core passes (plans with nrhs_max >= kTcwMinNrhs, FP32 or mixed
// storage): 128 right-hand sides per pass, every product on tcgen05.
constexpr int kTcwRhs = 128;        // right-hand sides per pass: the MMA's M
constexpr int kTcwMinNrhs = 32;     // nrhs_max from which a plan takes this form
constexpr int kTcwTileRows = 32;    // row-stage tile rows
constexpr int kTcwTilesPerItem = 4; // row-stage tiles per item (blocks sharing their inputs)
constexpr int kTcwMaskShift = 24;   // segment ncols: bits 0..23 columns, 24..27 block mask, 28 format
// Segment formats of the wide tensor-core layout (top bits of ncols).
enum TcwFmt : int32_t { TF_HI = 0, TF_HILO = 1 };
// The step program of the wide form, per input group (consecutive segments of
// an item with one input range) a 4-word header:
//   [0] the segments' src word (bit 31: t planes, bits 0..30: first input row)
//   [1] 8-column vectors of the range
//   [2] rows streamed per K step (pairs count twice) | item's last group << 12 |
//       MMAs on row block b << (16 + 4 b)
//   [3] index of its first MMA template
// and per MMA of a K step (ordered by row block: block b's MMAs are issued by
// their own warp) a 2-word template:
//   [0] first B row (in 16-byte units of the step's vectors) | A lo part << 12 | block << 13 |
//       into the block's correction accumulator << 15 | the block's rows * 16 << 16
//   [1] instruction descriptor
// The correction products (hi x x_lo, lo x x_hi, about 2^-11 of the main ones)
// go to a second accumulator where the block has room for one, so the main
// accumulator takes one rounding per 16 columns instead of three.
constexpr int kTcwMaxOps = 12;         // MMAs of one K step at most (4 block jobs x 3 products)
constexpr uint32_t kTcwGroupLast = 1u << 12;
constexpr uint32_t kTcwCorrBit = 1u << 15;
#if defined(__CUDACC__)
#define HMVM_TCW_HD __host__ __device__
#else
#define HMVM_TCW_HD
#endif
// tcgen05 instruction descriptor, kind::f16: D FP32, A and B FP16 (bf = 0) or
// BF16 (bf = 1), A MN-major, B K-major, M = 128, N = n.
HMVM_TCW_HD constexpr uint32_t tcw_idesc(int bf, int n) {
  return (1u << 4) | ((uint32_t)bf << 7) | ((uint32_t)bf << 10) | (1u << 15) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

struct HostLayout {
  int precision = HMVM_FP64;
  int vec = 2;
  int elem_size = 8;
  int32_t nd = 0, nlf = 0, n_lowrank = 0, n_dense = 0;
  int kernel = kDefaultKernel;
  int stage1_cfg = kDefaultStreamCfg, stage2_cfg = kDefaultStreamCfg, ctas_per_sm = kDefaultStreamCtasPerSm;
  int ctas2_per_sm = kDefaultStreamCtasPerSm;  // of the row stage (ctas_per_sm: the V stage)
  int num_sms = 148;
  std::vector<hmvm_tile_desc> tiles;  // [stage1 tiles][stage2 tiles], each in team order
  std::vector<hmvm_seg_desc> segs;
  std::vector<int32_t> team_begin1, team_begin2;  // absolute tile indices
  std::vector<int32_t> out_idx;
  std::vector<int32_t> red1;  // 4 ints per entry: t slot, first partial, parts, stride between parts
  std::vector<int32_t> red2;  // 4 ints per entry: y row, first partial, parts, stride between parts
  std::vector<Vec16, UninitAlloc<Vec16>> data;  // every byte written by the pack
  int32_t stage1_tiles = 0, stage2_tiles = 0, stage1_teams = 0, stage2_teams = 0;
  int64_t t_len = 0, p_len = 0;
  int64_t stored_elems = 0;  // sum of leaf element counts (the reference's len)
  int32_t split_rows = 0;
  // mixed precision
  bool mixed = false;
  std::vector<double> rowscale;  // per V-stage panel row: s_u * s_v of its (leaf, k) column
  int64_t cols_fp32 = 0, cols_lr16 = 0, cols_fp8 = 0;
  int64_t stored_bytes = 0;      // bytes of the stored elements in their storage formats
  int64_t stored_bytes1 = 0;     // ... of the V stage
  int nrhs_max = 1;              // items fit the multi-RHS input buffer for this many rhs
  // wide tensor-core layout
  bool tcw = false;
  bool tcw_bf16 = false;          // 16-bit format of the stored pairs and the input planes
  std::vector<float> tscale;      // per V-stage panel row 2^-c, then per y row the row scale s_i
  std::vector<int32_t> tblocks;   // per item: rows of blocks 0..3, 8 bits each
  std::vector<uint32_t> tgroups;  // the step program: 4 words per input group
  std::vector<uint32_t> tops;     // ... 2 words per MMA template, then kTcwMaxOps zero templates
  std::vector<int32_t> tgfirst;   // [items + 1]: first input group of each item
  int32_t tscale_rows0 = 0;       // index of y row 0 in tscale
};

// Returns HMVM_OK or a status; msg receives a description on failure.
// ctas2_per_sm > 0 gives the row stage its own CTAs per SM (else both stages
// use opts.ctas_per_sm, or the kernel's default).
int build_layout(const LeafTable &lt, const hmvm_plan_opts &opts, int num_sms, HostLayout &out,
                 std::string &msg, int ctas2_per_sm = 0);

int validate_leaves(const LeafTable &lt, std::string &msg);

// The wide tensor-core layout (see layout_tc.cpp).
int build_tc_layout(const LeafTable &lt, const hmvm_plan_opts &opts, int num_sms, HostLayout &out,
                    std::string &msg);

}  // namespace hmvm
