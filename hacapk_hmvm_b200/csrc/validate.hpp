// Bounds checks of a plan's descriptors, compiled for the host and the device.
//
// Every index a single-vector stage kernel derives from the layout (the data
// stream range of a tile, its segment descriptors, the x / t columns each
// segment reads, the padded inputs an item gathers, the y / t / partial-sum
// rows it writes, the t slots and row scales it looks up, and the reduction
// lists) is checked against the length of the buffer it indexes.  The host
// runs the checks through hmvm_b200_layout_validate; builds compiled with
// HMVM_DEVICE_CHECKS run them on the device before every stage launch, and the
// stage kernels then return without touching memory once the error word is
// set (they never trap).
#pragma once

#include <cstdint>

#include "hmvm_b200.h"

#ifdef __CUDACC__
#define HMVM_HD __host__ __device__
#else
#define HMVM_HD
#endif

namespace hmvm {

// Lengths of the buffers a layout indexes, in elements (data: 16-byte vectors).
struct LayoutCaps {
  int64_t data_vectors = 0, n_segs = 0, n_out_idx = 0, t_len = 0, p_len = 0, nd = 0, n_rowscale = 0;
  int32_t n_tiles = 0;
  int32_t max_rows = 32;
  int32_t max_segs = 0;  // segments per item a kernel takes (mixed kernels: 32; 0: no limit)
  int32_t mixed = 0;
};

// What a failed check names (0: none).
enum LayoutCheck : int {
  kCheckOk = 0,
  kCheckData = 1,     // the tile's vectors leave the data stream
  kCheckSegs = 2,     // its segment descriptors leave the segment table
  kCheckRows = 3,     // rows outside 1..max_rows, or negative vectors
  kCheckOut = 4,      // its output rows leave y, the t slot list or the partial sums
  kCheckSlot = 5,     // a t slot it writes is outside t
  kCheckSrc = 6,      // a segment's columns leave x or t
  kCheckInputs = 7,   // the item's padded inputs exceed the kernel's input buffer
  kCheckType = 8,     // a mixed segment's storage type is unknown
  kCheckScale = 9,    // its row scales leave the row-scale table
  kCheckReduce = 10,  // a reduction entry reads or writes outside its buffers
  kCheckTeams = 11,   // the team ranges do not cover the stage's tiles in order
};

// Elements per 16-byte vector of a segment type (mixed layouts; plain ones pass vec).
HMVM_HD inline int check_seg_vec(int type) { return type == 0 ? 2 : type == 1 ? 4 : type == 3 ? 16 : 8; }

// One tile (item) of stage 1 (V stage) or 2 (row stage).  vec: elements per
// vector of plain layouts; zcap_bytes: the input buffer of the stage's kernel
// (0: unchecked); elem: bytes per input element of plain layouts.
HMVM_HD inline int check_tile(const hmvm_tile_desc& d, const hmvm_seg_desc* segs, const int32_t* out_idx,
                              const LayoutCaps& c, int vec, int elem, int64_t zcap_bytes, bool stage1) {
  if (d.nrows < 1 || d.nrows > c.max_rows || d.nvec < 0) return kCheckRows;
  if (d.data_off < 0 || d.data_off + (int64_t)d.nvec * d.nrows > c.data_vectors) return kCheckData;
  if (d.seg_begin < 0 || d.nseg < 0 || (int64_t)d.seg_begin + d.nseg > c.n_segs) return kCheckSegs;
  if (c.max_segs > 0 && d.nseg > c.max_segs) return kCheckSegs;
  const int64_t ob = d.out_base, R = d.nrows;
  if (ob < 0) return kCheckOut;
  if (d.mode == 0) {
    if (stage1 || ob + R > c.nd) return kCheckOut;
  } else if (d.mode == 1) {
    if (!stage1 || ob + R > c.n_out_idx) return kCheckOut;
    for (int64_t r = 0; r < R; r++)
      if (out_idx[ob + r] < 0 || out_idx[ob + r] >= c.t_len) return kCheckSlot;
  } else if (d.mode == 2) {
    if (ob + R > c.p_len) return kCheckOut;
  } else {
    return kCheckOut;
  }
  if (c.mixed && stage1 && (d._pad < 0 || (int64_t)d._pad + R > c.n_rowscale)) return kCheckScale;
  int64_t zbytes = 0, vecs = 0;
  for (int32_t j = 0; j < d.nseg; j++) {
    const hmvm_seg_desc s = segs[d.seg_begin + j];
    int type = 0, nc = s.ncols, v = vec, e = elem;
    if (c.mixed) {
      type = (int)((uint32_t)s.ncols >> 28);
      nc = s.ncols & 0x0fffffff;
      if (type > 4) return kCheckType;
      v = check_seg_vec(type);
      e = type == 0 ? 8 : 4;
    }
    if (nc < 0) return kCheckSrc;
    if (s.src < 0) {
      if ((int64_t)(s.src & 0x7fffffff) + nc > c.t_len) return kCheckSrc;
    } else if ((int64_t)s.src + nc > c.nd) {
      return kCheckSrc;
    }
    const int64_t nv = (nc + v - 1) / v;
    vecs += nv;
    zbytes += nv * v * e;
  }
  if (vecs != d.nvec) return kCheckData;
  if (zcap_bytes > 0 && zbytes > zcap_bytes) return kCheckInputs;
  return kCheckOk;
}

// One reduction entry {destination, first partial, parts, stride}: stage 1
// writes t slots, stage 2 y rows.
HMVM_HD inline int check_red(const int32_t* e, const LayoutCaps& c, bool stage1) {
  const int64_t dst = e[0], p0 = e[1], parts = e[2], stride = e[3];
  if (dst < 0 || dst >= (stage1 ? c.t_len : c.nd)) return kCheckReduce;
  if (parts < 1 || p0 < 0 || stride < 0 || p0 + (parts - 1) * stride >= c.p_len) return kCheckReduce;
  return kCheckOk;
}

// The team ranges of a stage: nteams + 1 tile indices from first to end.
HMVM_HD inline int check_teams(const int32_t* tb, int32_t nteams, int32_t first, int32_t end) {
  if (nteams < 1 || tb[0] != first || tb[nteams] != end) return kCheckTeams;
  for (int32_t k = 0; k < nteams; k++)
    if (tb[k + 1] < tb[k]) return kCheckTeams;
  return kCheckOk;
}

}  // namespace hmvm
