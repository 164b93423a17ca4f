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
//  * Column panels wider than split_cols are cut into chunks that write
//    partial sums; a small reduction adds the chunks in chunk order.
//  * Tiles are assigned to persistent "teams" (groups of warps) by LPT on
//    their byte cost and stored in team order, so a team streams one
//    contiguous region.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "hmvm_b200.h"

namespace hmvm {

struct alignas(16) Vec16 {
  uint32_t w[4];
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

// Kernel configurations: warps per team (WG) and teams per CTA (TPC).
struct KernelCfg {
  int wg, tpc;
};
constexpr int kNumCfgs = 8;
constexpr KernelCfg kCfgs[kNumCfgs] = {{1, 8}, {2, 4}, {4, 2}, {8, 1}, {2, 8}, {4, 4}, {8, 2}, {16, 1}};
constexpr int kDefaultStage1Cfg = 4;
constexpr int kDefaultStage2Cfg = 5;
constexpr int kDefaultCtasPerSm = 2;
constexpr int kMaxRows = 32;

struct HostLayout {
  int precision = HMVM_FP64;
  int vec = 2;
  int elem_size = 8;
  int32_t nd = 0, nlf = 0, n_lowrank = 0, n_dense = 0;
  int stage1_cfg = kDefaultStage1Cfg, stage2_cfg = kDefaultStage2Cfg, ctas_per_sm = kDefaultCtasPerSm;
  int num_sms = 148;
  std::vector<hmvm_tile_desc> tiles;  // [stage1 tiles][stage2 tiles], each in team order
  std::vector<hmvm_seg_desc> segs;
  std::vector<int32_t> team_begin1, team_begin2;  // absolute tile indices
  std::vector<int32_t> out_idx;
  std::vector<int32_t> red;  // 4 ints per entry
  std::vector<Vec16> data;
  int32_t stage1_tiles = 0, stage2_tiles = 0, stage1_teams = 0, stage2_teams = 0;
  int64_t t_len = 0, p_len = 0;
  int64_t stored_elems = 0;  // sum of leaf element counts (the reference's len)
  int32_t split_rows = 0;
};

// Returns HMVM_OK or a status; msg receives a description on failure.
int build_layout(const LeafTable &lt, const hmvm_plan_opts &opts, int num_sms, HostLayout &out,
                 std::string &msg);

int validate_leaves(const LeafTable &lt, std::string &msg);

}  // namespace hmvm
