// Host planner of the wide tensor-core form: a leaf list -> the layout that
// hmvm_tcw_kernel streams (128 right-hand sides per pass, every product on
// tcgen05 with FP32 accumulation).
//
// The GEMMs run transposed, Y^T = X^T H^T: the right-hand sides are the MMA's
// M (128), the rows of an item its N (<= 32 for a row-stage tile, <= 128 for a
// V-stage panel), and 16 matrix columns one K step.  The matrix is the B
// operand, read by the MMA straight from the kernel's shared-memory ring in the
// canonical K-major layout without swizzle -- which is what a tile of 16-byte
// vectors already is (vector v = R rows x 16 bytes, row r holding columns
// 8v..8v+7; 8-row core matrices 128 bytes apart, the next 8 columns R*16 bytes
// on).  The inputs (x, and t = V x) are the A operand: 16-bit planes gathered
// per K step by one TMA tensor copy.
//
// Storage, all in one 16-bit format (FP16, or BF16 for BF16-factor plans):
//   * HI segments: one 16-bit value per element (the 16-bit low-rank columns of
//     mixed plans, and their FP8 columns, widened);
//   * HILO segments: a pair hi + lo (hi = fmt(v), lo = fmt(v - hi)), about 22
//     significant bits with FP16: dense leaves, the leading low-rank columns of
//     mixed plans (term >= tau |block|) and every column of FP32 plans.  The
//     MMAs take hi x x_hi, hi x x_lo and lo x x_hi (lo x x_lo is dropped).
//   * A segment is stored K-step-major: per 16 columns [hi v, hi v+1] or
//     [hi v, hi v+1, lo v, lo v+1]; an odd last step holds one vector of each.
//   * Scales (powers of two, exact): V-stage row n (leaf i, term k) is stored as
//     V_n * 2^-e_n with max |V| in (2^14, 2^15]; its output t_n is written as
//     tau_n = (V_n . x / sigma_x) * 2^-c_n with 2^c_n >= sum |V_n 2^-e_n|, so
//     |tau| <= 2^15.  Row-stage row i is stored divided by s_i, the power of two
//     putting the row's largest value (dense D_ij, and U_in 2^(e_n + c_n)) in
//     (2^14, 2^15]; y_i = s_i * sigma_x * (its accumulator).  sigma_x is the
//     per-right-hand-side scale of the x planes (1 for BF16).
//   * Items: a row-stage tile is one item (no partial sums); a V-stage panel is
//     cut into K-step ranges when it is large, whose FP32 partial sums a small
//     kernel adds in part order.  Items go to one team per SM by LPT.
//
// The summation order is fixed by the layout, so results are bitwise
// repeatable.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <queue>
#include <tuple>
#include <unordered_map>
#include <utility>

#include "layout.hpp"
#include "numfmt.hpp"

namespace hmvm {

namespace {

constexpr int32_t kTFlagTc = (int32_t)0x80000000u;

inline uint64_t key2t(int32_t a, int32_t b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }

// Exponent k with 2^(k-1) < m <= 2^k (m > 0 and finite).
inline int ceil_log2(double m) {
  int e;
  const double f = std::frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
  return f == 0.5 ? e - 1 : e;
}

// The power-of-two scale that puts a largest magnitude m in (2^14, 2^15]
// (1 when m is 0 or not finite).
inline double pow2_for_max(double m) {
  if (!(m > 0.0) || !std::isfinite(m)) return 1.0;
  return std::ldexp(1.0, ceil_log2(m) - 15);
}

// A segment of an item: an input range (x columns, or t slots) multiplied by
// the blocks in its mask.  kind 0: V rows (V stage); 1: a dense leaf per block
// (row stage); 2: the low-rank columns of one format of a row group (row stage).
struct TcSeg2 {
  int32_t src = 0, ncols = 0, fmt = 0, mask = 0, kind = 0, group = -1;
  int32_t leaf[4] = {-1, -1, -1, -1};
};

struct TcItem {
  int32_t stage = 2;
  int32_t nblk = 0;
  int32_t R[4] = {0, 0, 0, 0};  // rows per block
  int32_t row0 = 0;             // row stage: first y row (blocks are consecutive rows)
  int32_t panel_row0 = 0;       // V stage: first entry in panel_rows (blocks consecutive)
  std::vector<TcSeg2> segs;
};

}  // namespace

int build_tc_layout(const LeafTable &lt, const hmvm_plan_opts &opts, int num_sms, HostLayout &L, std::string &msg) {
  int rc = validate_leaves(lt, msg);
  if (rc) return rc;
  if (opts.precision != HMVM_FP32 && opts.precision != HMVM_MIXED) {
    msg = "the tensor-core form takes FP32 or mixed plans";
    return HMVM_EINVAL;
  }
  try {
    L = HostLayout();
    L.tcw = true;
    L.precision = opts.precision;
    L.mixed = opts.precision == HMVM_MIXED;
    L.tcw_bf16 = L.mixed && opts.mixed_lr_format == HMVM_LR_BF16;
    L.elem_size = opts.precision == HMVM_FP32 ? 4 : 8;  // x and y
    L.vec = 8;
    L.nd = lt.nd;
    L.nlf = lt.nlf;
    L.num_sms = num_sms > 0 ? num_sms : 148;
    L.kernel = 4;
    L.nrhs_max = kTcwRhs;
    L.stage1_teams = L.stage2_teams = L.num_sms;
    L.ctas_per_sm = L.ctas2_per_sm = 1;
    const bool bf = L.tcw_bf16;
    auto enc = [bf](double v) { return bf ? to_bf16(v) : to_fp16(v); };
    auto dec = [bf](uint16_t h) {
      if (!bf) return from_fp16(h);
      uint32_t w = (uint32_t)h << 16;
      float f;
      std::memcpy(&f, &w, 4);
      return (double)f;
    };
    const int32_t nd = lt.nd, nlf = lt.nlf;
    const bool srcf = lt.rowmat_is_float;
    auto get = [&](int64_t idx) {
      return srcf ? (double)static_cast<const float *>(lt.rowmat)[idx] : static_cast<const double *>(lt.rowmat)[idx];
    };

    // ---- low-rank columns: format, V scale 2^-e, output scale 2^-c ------------
    std::vector<uint8_t> live_lr(nlf, 0);
    std::vector<int64_t> colbase(nlf, -1);
    int64_t ncolflat = 0;
    for (int32_t i = 0; i < nlf; i++) {
      if (lt.ltmtx[i] == 1) {
        L.n_lowrank++;
        L.stored_elems += (int64_t)lt.kt[i] * (lt.ndl[i] + (int64_t)lt.ndt[i]);
        live_lr[i] = lt.kt[i] > 0 && lt.ndl[i] > 0 && lt.ndt[i] > 0;
        if (live_lr[i]) {
          colbase[i] = ncolflat;
          ncolflat += lt.kt[i];
        }
      } else {
        L.n_dense++;
        L.stored_elems += (int64_t)lt.ndl[i] * lt.ndt[i];
      }
    }
    std::vector<uint8_t> col_fmt(ncolflat, TF_HILO);
    std::vector<double> vsc(ncolflat, 1.0), csc(ncolflat, 1.0);  // 2^e and 2^c per column
    const double tau = opts.mixed_fp32_tau >= 0.0 ? opts.mixed_fp32_tau
                       : (opts.mixed_lr_format == HMVM_LR_BF16 ? 0.05 : 0.5);
#pragma omp parallel for schedule(dynamic, 64)
    for (int32_t i = 0; i < nlf; i++) {
      if (!live_lr[i]) continue;
      const int32_t kt = lt.kt[i], ndl = lt.ndl[i], ndt = lt.ndt[i];
      std::vector<double> term(kt);
      double block = 0.0;
      for (int32_t k = 0; k < kt; k++) {
        double su = 0, sv = 0, mv = 0;
        for (int32_t r = 0; r < ndl; r++) {
          const double u = get(lt.a2(i) + (int64_t)k * ndl + r);
          su += u * u;
        }
        for (int32_t c = 0; c < ndt; c++) {
          const double v = get(lt.a1(i) + (int64_t)k * ndt + c);
          sv += v * v;
          mv = std::max(mv, std::fabs(v));
        }
        term[k] = std::sqrt(su) * std::sqrt(sv);
        block = std::max(block, term[k]);
        const int64_t f = colbase[i] + k;
        const double e = pow2_for_max(mv);
        vsc[f] = e;
        double l1 = 0.0;
        for (int32_t c = 0; c < ndt; c++) l1 += std::fabs(get(lt.a1(i) + (int64_t)k * ndt + c) / e);
        csc[f] = l1 > 0.0 ? std::ldexp(1.0, ceil_log2(l1)) : 1.0;
      }
      if (L.mixed)
        for (int32_t k = 0; k < kt; k++) col_fmt[colbase[i] + k] = term[k] >= tau * block ? TF_HILO : TF_HI;
    }
    for (int64_t f = 0; f < ncolflat; f++) (col_fmt[f] == TF_HILO ? L.cols_fp32 : L.cols_lr16)++;

    // ---- row tiles (leaf row boundaries, <= 32 rows) ------------------------------
    std::vector<int32_t> bnd;
    bnd.reserve(2 * (size_t)nlf + 2);
    bnd.push_back(0);
    bnd.push_back(nd);
    for (int32_t i = 0; i < nlf; i++) {
      if (lt.ndl[i] <= 0) continue;
      bnd.push_back(lt.nstrtl[i] - 1);
      bnd.push_back(lt.nstrtl[i] - 1 + lt.ndl[i]);
    }
    std::sort(bnd.begin(), bnd.end());
    bnd.erase(std::unique(bnd.begin(), bnd.end()), bnd.end());
    std::vector<int32_t> trow0, tnrows;
    for (size_t b = 0; b + 1 < bnd.size(); b++) {
      const int32_t a = bnd[b], n = bnd[b + 1] - a;
      const int32_t pieces = (n + kTcwTileRows - 1) / kTcwTileRows;
      for (int32_t p = 0; p < pieces; p++) {
        const int32_t s0 = a + (int32_t)((int64_t)n * p / pieces), s1 = a + (int32_t)((int64_t)n * (p + 1) / pieces);
        trow0.push_back(s0);
        tnrows.push_back(s1 - s0);
      }
    }
    const int32_t nrt = (int32_t)trow0.size();
    std::vector<int32_t> row_tile(nd > 0 ? nd : 1);
    for (int32_t ti = 0; ti < nrt; ti++)
      for (int32_t r = trow0[ti]; r < trow0[ti] + tnrows[ti]; r++) row_tile[r] = ti;

    // ---- row groups, column groups, t slots ---------------------------------------
    std::unordered_map<uint64_t, int32_t> rgmap, cgmap;
    std::vector<std::vector<int32_t>> rg_members, cg_members;
    for (int32_t i = 0; i < nlf; i++) {
      if (!live_lr[i]) continue;
      auto add = [&](std::unordered_map<uint64_t, int32_t> &m, std::vector<std::vector<int32_t>> &mem, uint64_t k) {
        auto it = m.find(k);
        int32_t g;
        if (it == m.end()) {
          g = (int32_t)mem.size();
          m.emplace(k, g);
          mem.emplace_back();
        } else {
          g = it->second;
        }
        mem[g].push_back(i);
      };
      add(rgmap, rg_members, key2t(lt.nstrtl[i], lt.ndl[i]));
      add(cgmap, cg_members, key2t(lt.nstrtt[i], lt.ndt[i]));
    }
    const int32_t nrg = (int32_t)rg_members.size();
    // slots in (row group, format) order, no padding: the kernel's input boxes
    // start at any row
    std::vector<int64_t> slot_of_col(ncolflat, -1);
    std::vector<int32_t> rg_slot((size_t)nrg * 2), rg_k((size_t)nrg * 2);
    int64_t t_len = 0;
    for (int32_t g = 0; g < nrg; g++) {
      for (int fm = TF_HILO; fm >= TF_HI; fm--) {
        rg_slot[(size_t)g * 2 + fm] = (int32_t)t_len;
        int32_t k = 0;
        for (int32_t i : rg_members[g])
          for (int32_t kk = 0; kk < lt.kt[i]; kk++) {
            const int64_t f = colbase[i] + kk;
            if (col_fmt[f] != fm) continue;
            slot_of_col[f] = t_len + k;
            k++;
          }
        rg_k[(size_t)g * 2 + fm] = k;
        t_len += k;
      }
      if (t_len > INT32_MAX / 2) {
        msg = "intermediate vector too long";
        return HMVM_ERANGE;
      }
    }
    L.t_len = t_len;

    // ---- items: row blocks sharing their input loads --------------------------------
    // An item is up to 4 row blocks (V stage: panels of one column group, the
    // pair-stored rows in a block of <= 64, the others in blocks of <= 128;
    // row stage: up to 4 consecutive row tiles of <= 32 rows).  Its segments
    // carry a block mask: a segment's K-step streams its input once and
    // multiplies every block in the mask by it (one MMA group per block), and
    // consecutive segments with the same input range share the input too.
    std::vector<TcItem> titems;
    std::vector<std::pair<int32_t, int32_t>> panel_rows;  // (leaf, k) per V-stage output row
    for (int32_t c = 0; c < (int32_t)cg_members.size(); c++) {
      const auto &mem = cg_members[c];
      const int32_t ndt = lt.ndt[mem[0]], st = lt.nstrtt[mem[0]];
      std::vector<std::pair<int32_t, int32_t>> rows[2];  // by format
      for (int32_t i : mem)
        for (int32_t k = 0; k < lt.kt[i]; k++) rows[col_fmt[colbase[i] + k]].emplace_back(i, k);
      // blocks: pair rows in blocks of <= 64 (a K step of 64 pair rows is 4 KiB), the others <= 128
      std::vector<std::pair<int, std::vector<std::pair<int32_t, int32_t>>>> blocks[2];
      for (int fm = 0; fm < 2; fm++) {
        const size_t cap = fm == TF_HILO ? 64 : 128;
        const size_t nb = (rows[fm].size() + cap - 1) / cap;
        for (size_t q = 0; q < nb; q++) {
          const size_t b0 = rows[fm].size() * q / nb, b1 = rows[fm].size() * (q + 1) / nb;
          blocks[fm].emplace_back(fm, std::vector<std::pair<int32_t, int32_t>>(rows[fm].begin() + b0,
                                                                               rows[fm].begin() + b1));
        }
      }
      // pair one block of each format per item (a K step: <= 4 + 4 KiB); the rest alone
      const size_t nit = std::max(blocks[0].size(), blocks[1].size());
      for (size_t q = 0; q < nit; q++) {
        TcItem t;
        t.stage = 1;
        t.panel_row0 = (int32_t)panel_rows.size();
        for (int fm = TF_HILO; fm >= TF_HI; fm--) {
          if (q >= blocks[fm].size()) continue;
          const auto &blk = blocks[fm][q].second;
          const int b = t.nblk++;
          t.R[b] = (int32_t)blk.size();
          for (const auto &lk : blk) {
            const int64_t f = colbase[lk.first] + lk.second;
            L.out_idx.push_back((int32_t)slot_of_col[f]);
            L.tscale.push_back((float)(1.0 / csc[f]));
            panel_rows.push_back(lk);
          }
          TcSeg2 sg;
          sg.src = st - 1;
          sg.ncols = ndt;
          sg.fmt = fm;
          sg.mask = 1 << b;
          sg.kind = 0;
          t.segs.push_back(sg);
        }
        titems.push_back(std::move(t));
      }
    }
    const int32_t n1 = (int32_t)titems.size();
    L.tscale_rows0 = (int32_t)L.tscale.size();

    // ---- row stage: items of up to 4 consecutive row tiles -------------------------------
    std::vector<int32_t> dcount(nrt + 1, 0), gcount(nrt + 1, 0);
    for (int32_t i = 0; i < nlf; i++) {
      if (lt.ltmtx[i] != 2 || lt.ndl[i] <= 0 || lt.ndt[i] <= 0) continue;
      const int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
      for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) dcount[ti + 1]++;
    }
    for (int32_t g = 0; g < nrg; g++) {
      const int32_t i = rg_members[g][0];
      const int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
      for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) gcount[ti + 1]++;
    }
    for (int32_t ti = 0; ti < nrt; ti++) {
      dcount[ti + 1] += dcount[ti];
      gcount[ti + 1] += gcount[ti];
    }
    std::vector<int32_t> dlist(dcount[nrt]), glist(gcount[nrt]);
    {
      std::vector<int32_t> dpos(dcount.begin(), dcount.end() - 1), gpos(gcount.begin(), gcount.end() - 1);
      for (int32_t i = 0; i < nlf; i++) {
        if (lt.ltmtx[i] != 2 || lt.ndl[i] <= 0 || lt.ndt[i] <= 0) continue;
        const int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
        for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) dlist[dpos[ti]++] = i;
      }
      for (int32_t g = 0; g < nrg; g++) {
        const int32_t i = rg_members[g][0];
        const int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
        for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) glist[gpos[ti]++] = g;
      }
    }
    for (int32_t t0 = 0; t0 < nrt; t0 += kTcwTilesPerItem) {
      TcItem t;
      t.stage = 2;
      t.row0 = trow0[t0];
      std::map<std::tuple<int32_t, int32_t, int32_t>, size_t> index;  // (src, ncols, fmt) -> segment
      for (int32_t ti = t0; ti < std::min(nrt, t0 + kTcwTilesPerItem); ti++) {
        const int b = t.nblk++;
        t.R[b] = tnrows[ti];
        auto add = [&](int32_t src, int32_t nc, int32_t fm, int kind, int32_t leaf, int32_t group) {
          const auto key = std::make_tuple(src, nc, fm);
          auto it = index.find(key);
          if (it == index.end()) {
            TcSeg2 sg;
            sg.src = src;
            sg.ncols = nc;
            sg.fmt = fm;
            sg.mask = 0;
            sg.kind = kind;
            sg.group = group;
            it = index.emplace(key, t.segs.size()).first;
            t.segs.push_back(sg);
          }
          TcSeg2 &sg = t.segs[it->second];
          sg.mask |= 1 << b;
          sg.leaf[b] = leaf;
        };
        for (int32_t d = dcount[ti]; d < dcount[ti + 1]; d++) {
          const int32_t i = dlist[d];
          add(lt.nstrtt[i] - 1, lt.ndt[i], TF_HILO, 1, i, -1);
        }
        for (int32_t gg = gcount[ti]; gg < gcount[ti + 1]; gg++) {
          const int32_t g = glist[gg];
          for (int fm = TF_HILO; fm >= TF_HI; fm--) {
            const int32_t k = rg_k[(size_t)g * 2 + fm];
            if (k > 0) add(kTFlagTc | rg_slot[(size_t)g * 2 + fm], k, fm, 2, -1, g);
          }
        }
      }
      // input order: x segments by column, then t segments by slot (segments with one input range adjacent)
      std::stable_sort(t.segs.begin(), t.segs.end(), [](const TcSeg2 &x, const TcSeg2 &y) {
        const uint32_t ax = (uint32_t)x.src, ay = (uint32_t)y.src;
        return ax != ay ? ax < ay : x.ncols < y.ncols;
      });
      titems.push_back(std::move(t));
    }
    const int32_t ntb = (int32_t)titems.size();

    // ---- row scales s_i: the largest stored magnitude of each row -----------------------
    std::vector<double> rowmax(nd > 0 ? nd : 1, 0.0);
    for (int32_t i = 0; i < nlf; i++) {
      if (lt.ltmtx[i] != 2 || lt.ndl[i] <= 0 || lt.ndt[i] <= 0) continue;
      const int32_t rs = lt.nstrtl[i] - 1, ndt = lt.ndt[i];
      for (int32_t r = 0; r < lt.ndl[i]; r++) {
        double m = rowmax[rs + r];
        for (int32_t c = 0; c < ndt; c++) m = std::max(m, std::fabs(get(lt.a1(i) + (int64_t)r * ndt + c)));
        rowmax[rs + r] = m;
      }
    }
    for (int32_t i = 0; i < nlf; i++) {
      if (!live_lr[i]) continue;
      const int32_t rs = lt.nstrtl[i] - 1, ndl = lt.ndl[i];
      for (int32_t kk = 0; kk < lt.kt[i]; kk++) {
        const int64_t f = colbase[i] + kk;
        const double w = vsc[f] * csc[f];
        for (int32_t r = 0; r < ndl; r++)
          rowmax[rs + r] = std::max(rowmax[rs + r], std::fabs(get(lt.a2(i) + (int64_t)kk * ndl + r) * w));
      }
    }
    std::vector<double> rowsc(nd > 0 ? nd : 1, 1.0);
    for (int32_t r = 0; r < nd; r++) {
      rowsc[r] = pow2_for_max(rowmax[r]);
      L.tscale.push_back((float)rowsc[r]);
    }

    // ---- items cut into parts (V stage, large), costs ------------------------------------
    auto item_records = [&](const TcItem &t, int32_t j0, int32_t j1) {  // 16-byte records of K steps [j0, j1)
      int64_t n = 0;
      for (const TcSeg2 &sg : t.segs) {
        const int32_t c0 = 16 * j0, nc = std::min(sg.ncols - c0, 16 * (j1 - j0));
        if (nc <= 0) continue;
        const int64_t vec = (int64_t)((nc + 7) / 8) * (sg.fmt == TF_HILO ? 2 : 1);
        for (int b = 0; b < 4; b++)
          if (sg.mask >> b & 1) n += vec * t.R[b];
      }
      return n;
    };
    auto item_nks = [&](const TcItem &t) {
      int32_t m = 0;
      for (const TcSeg2 &sg : t.segs) m = std::max(m, (sg.ncols + 15) / 16);
      return m;
    };
    int64_t stage_bytes = 0;
    for (int32_t k = 0; k < n1; k++) stage_bytes += item_records(titems[k], 0, item_nks(titems[k])) * 16;
    const int64_t cap1 = std::max<int64_t>(64 * 1024, stage_bytes / std::max<int64_t>(1, (int64_t)L.num_sms * 4));
    struct Item {
      int32_t tile, j0, j1, mode, out_base;
      int64_t cost;
    };
    std::vector<Item> items;
    std::vector<int32_t> tile_item0(ntb + 1);
    int64_t p_len = 0;
    for (int32_t k = 0; k < ntb; k++) {
      const TcItem &t = titems[k];
      tile_item0[k] = (int32_t)items.size();
      const int32_t nks = item_nks(t);
      const int64_t bytes = item_records(t, 0, nks) * 16;
      if (t.stage == 2) {
        items.push_back(Item{k, 0, nks, 0, t.row0, bytes + 4096});
        continue;
      }
      const int32_t nparts = (int32_t)std::min<int64_t>(nks, (bytes + cap1 - 1) / cap1);
      if (nparts <= 1) {
        items.push_back(Item{k, 0, nks, 1, t.panel_row0, bytes + 4096});
        continue;
      }
      int32_t rows = 0;
      for (int b = 0; b < t.nblk; b++) rows += t.R[b];
      const int64_t pb = p_len;
      p_len += (int64_t)nparts * rows;
      for (int32_t r = 0; r < rows; r++) {
        L.red1.push_back(L.out_idx[t.panel_row0 + r]);
        L.red1.push_back((int32_t)(pb + r));
        L.red1.push_back(nparts);
        L.red1.push_back(rows);
      }
      for (int32_t q = 0; q < nparts; q++) {
        const int32_t j0 = (int32_t)((int64_t)nks * q / nparts), j1 = (int32_t)((int64_t)nks * (q + 1) / nparts);
        items.push_back(Item{k, j0, j1, 2, (int32_t)(pb + (int64_t)q * rows), item_records(t, j0, j1) * 16 + 4096});
      }
    }
    tile_item0[ntb] = (int32_t)items.size();
    if (p_len > INT32_MAX / kTcwRhs) {
      msg = "partial-sum buffer too long";
      return HMVM_ERANGE;
    }
    L.p_len = p_len;
    L.split_rows = (int32_t)(L.red1.size() / 4);
    const int32_t ni1 = tile_item0[n1];
    const int32_t ni2 = (int32_t)items.size() - ni1;

    auto assign = [&](int32_t first, int32_t count, int32_t nteams, std::vector<int32_t> &order,
                      std::vector<int32_t> &team_begin) {
      std::vector<int32_t> idx(count);
      for (int32_t k = 0; k < count; k++) idx[k] = first + k;
      std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) { return items[a].cost > items[b].cost; });
      using HE = std::pair<int64_t, int32_t>;
      std::priority_queue<HE, std::vector<HE>, std::greater<HE>> heap;
      for (int32_t k = 0; k < nteams; k++) heap.emplace(0, k);
      std::vector<int32_t> team_of(count);
      for (int32_t k : idx) {
        HE h = heap.top();
        heap.pop();
        team_of[k - first] = h.second;
        heap.emplace(h.first + items[k].cost, h.second);
      }
      std::vector<int32_t> cnt(nteams + 1, 0);
      for (int32_t k = 0; k < count; k++) cnt[team_of[k] + 1]++;
      for (int32_t k = 0; k < nteams; k++) cnt[k + 1] += cnt[k];
      team_begin.assign(cnt.begin(), cnt.end());
      std::vector<int32_t> pos(cnt.begin(), cnt.end() - 1);
      order.resize(count);
      for (int32_t k = 0; k < count; k++) order[pos[team_of[k]]++] = first + k;
    };
    std::vector<int32_t> ord1, ord2, tb1, tb2;
    assign(0, ni1, L.stage1_teams, ord1, tb1);
    assign(ni1, ni2, L.stage2_teams, ord2, tb2);
    std::vector<int32_t> order(ord1);
    order.insert(order.end(), ord2.begin(), ord2.end());
    L.team_begin1 = tb1;
    L.team_begin2.resize(tb2.size());
    for (size_t k = 0; k < tb2.size(); k++) L.team_begin2[k] = tb2[k] + ni1;
    L.stage1_tiles = ni1;
    L.stage2_tiles = ni2;

    // ---- descriptors ---------------------------------------------------------------------
    const int32_t nitems = (int32_t)items.size();
    L.tiles.resize(nitems);
    L.tblocks.resize(nitems);
    L.segs.clear();
    std::vector<int64_t> item_off(nitems);  // by item index: first 16-byte record
    int64_t off = 0;
    for (int32_t k = 0; k < nitems; k++) {
      const Item &it = items[order[k]];
      const TcItem &t = titems[it.tile];
      hmvm_tile_desc &d = L.tiles[k];
      d.data_off = off;
      d.seg_begin = (int32_t)L.segs.size();
      d.out_base = it.out_base;
      int32_t rows = 0, used = 0, packed = 0;
      for (int b = 0; b < t.nblk; b++) {
        rows += t.R[b];
        packed |= t.R[b] << (8 * b);
      }
      int32_t nseg = 0;
      for (const TcSeg2 &sg : t.segs) {
        const int32_t c0 = 16 * it.j0, nc = std::min(sg.ncols - c0, 16 * (it.j1 - it.j0));
        if (nc <= 0) continue;
        if (nc >= (1 << kTcwMaskShift)) {
          msg = "a segment of 2^24 or more columns";
          return HMVM_ERANGE;
        }
        const int32_t src = sg.src < 0 ? (kTFlagTc | ((sg.src & 0x7fffffff) + c0)) : sg.src + c0;
        L.segs.push_back(hmvm_seg_desc{src, nc | (sg.mask << kTcwMaskShift) | (sg.fmt << kSegTypeShift)});
        used |= sg.mask;
        nseg++;
      }
      d.nseg = nseg;
      d.nrows = (int16_t)rows;
      d.mode = (int16_t)(it.mode | (used << 4));
      d._pad = t.stage == 1 ? t.panel_row0 : L.tscale_rows0 + t.row0;
      const int64_t nrec = item_records(t, it.j0, it.j1);
      d.nvec = (int32_t)nrec;
      L.tblocks[k] = packed;
      item_off[order[k]] = off;
      off += nrec;
    }
    L.data.resize((size_t)off);

    // ---- step program -----------------------------------------------------------------------
    // Per item, its input groups (consecutive segments with one input range) in
    // stream order; per group the MMAs of each of its K steps: per segment, per
    // block of its mask, hi x x_hi, hi x x_lo and (pairs) lo x x_hi, B at the
    // block's hi vectors (then lo vectors) of the step.
    L.tgroups.clear();
    L.tops.clear();
    L.tgfirst.assign((size_t)nitems + 1, 0);
    for (int32_t k = 0; k < nitems; k++) {
      const hmvm_tile_desc &d = L.tiles[k];
      const uint32_t R4 = (uint32_t)L.tblocks[k];
      L.tgfirst[k] = (int32_t)(L.tgroups.size() / 4);
      const int32_t se = d.seg_begin + d.nseg;
      for (int32_t s = d.seg_begin; s < se;) {
        const hmvm_seg_desc &f = L.segs[s];
        const int32_t nc = f.ncols & ((1 << kTcwMaskShift) - 1);
        int32_t s1 = s + 1;
        while (s1 < se && L.segs[s1].src == f.src && (L.segs[s1].ncols & ((1 << kTcwMaskShift) - 1)) == nc) s1++;
        const uint32_t op0 = (uint32_t)(L.tops.size() / 2);
        uint32_t pre = 0, nops = 0, counts = 0;
        std::vector<uint32_t> by_block[4];  // template words, per row block in stream order
        for (int32_t z = s; z < s1; z++) {
          const uint32_t enc = (uint32_t)L.segs[z].ncols, mask = (enc >> kTcwMaskShift) & 15u;
          const bool pair = ((enc >> kSegTypeShift) & 1u) == (uint32_t)TF_HILO;
          for (int b = 0; b < 4; b++) {
            if (!(mask >> b & 1u)) continue;
            const uint32_t R = (R4 >> (8 * b)) & 0xffu;
            const uint32_t id = tcw_idesc(L.tcw_bf16 ? 1 : 0, std::max(16, (int)((R + 15) & ~15u)));
            const uint32_t blk = ((uint32_t)b << 13) | ((R * 16u) << 16);
            // the correction products (hi x x_lo, lo x x_hi) into their own accumulator where
            // the block has room for one (every row-stage block; V-stage blocks of <= 64 rows)
            const uint32_t corr = (k >= L.stage1_tiles || R <= 64u) ? kTcwCorrBit : 0u;
            by_block[b].insert(by_block[b].end(), {pre | blk, id, pre | (1u << 12) | blk | corr, id});
            nops += 2;
            if (pair) {
              by_block[b].insert(by_block[b].end(), {(pre + R) | blk | corr, id});
              nops++;
            }
            pre += pair ? 2 * R : R;
          }
        }
        if (nops > (uint32_t)kTcwMaxOps || pre >= 4096u) {
          msg = "an input group of more than 4 block jobs";
          return HMVM_ERANGE;
        }
        for (int b = 0; b < 4; b++) {
          L.tops.insert(L.tops.end(), by_block[b].begin(), by_block[b].end());
          counts |= (uint32_t)(by_block[b].size() / 2) << (16 + 4 * b);
        }
        L.tgroups.insert(L.tgroups.end(), {(uint32_t)f.src, (uint32_t)((nc + 7) / 8),
                                           pre | (s1 == se ? kTcwGroupLast : 0u) | counts, op0});
        s = s1;
      }
    }
    L.tgfirst[nitems] = (int32_t)(L.tgroups.size() / 4);
    L.tops.insert(L.tops.end(), 2 * (size_t)kTcwMaxOps, 0u);

    // ---- pack -------------------------------------------------------------------------------
    // Per item part: per input group (consecutive segments with one input range),
    // per K step, per segment, per block in its mask: the hi vectors of the step
    // (R rows x 16 bytes each), then the lo vectors of a pair segment.
    int64_t stored_bytes = 0, stored_bytes1 = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : stored_bytes, stored_bytes1)
    for (int32_t q = 0; q < nitems; q++) {
      const Item &it = items[q];
      const TcItem &t = titems[it.tile];
      char *base = reinterpret_cast<char *>(L.data.data() + item_off[q]);
      int32_t brow[4] = {0, 0, 0, 0};  // first item row of each block
      for (int b = 1; b < t.nblk; b++) brow[b] = brow[b - 1] + t.R[b - 1];
      // the item's segments, trimmed to the part's K steps
      struct PSeg {
        const TcSeg2 *sg;
        int32_t c0, nc;
      };
      std::vector<PSeg> ps;
      for (const TcSeg2 &sg : t.segs) {
        const int32_t c0 = 16 * it.j0, nc = std::min(sg.ncols - c0, 16 * (it.j1 - it.j0));
        if (nc > 0) ps.push_back(PSeg{&sg, c0, nc});
      }
      // value of segment z, block b, block row r, (absolute) column c, scaled for 16-bit storage
      // U segments: the (leaf, k) of each of its columns, looked up once
      std::vector<std::vector<std::pair<int32_t, int32_t>>> ucols(ps.size());
      for (size_t z = 0; z < ps.size(); z++) {
        const TcSeg2 &sg = *ps[z].sg;
        if (sg.kind != 2) continue;
        for (int32_t i : rg_members[sg.group])
          for (int32_t kk = 0; kk < lt.kt[i]; kk++)
            if (col_fmt[colbase[i] + kk] == sg.fmt) ucols[z].emplace_back(i, kk);
      }
      auto val = [&](size_t z, int b, int32_t r, int32_t c) -> double {
        const TcSeg2 &sg = *ps[z].sg;
        if (sg.kind == 0) {  // V row (leaf, k) of the panel
          const auto lk = panel_rows[t.panel_row0 + brow[b] + r];
          const int64_t f = colbase[lk.first] + lk.second;
          return get(lt.a1(lk.first) + (int64_t)lk.second * lt.ndt[lk.first] + c) / vsc[f];
        }
        if (sg.kind == 1) {  // dense leaf of block b
          const int32_t i = sg.leaf[b], row = t.row0 + brow[b] + r;
          return get(lt.a1(i) + (int64_t)(row - (lt.nstrtl[i] - 1)) * lt.ndt[i] + c) / rowsc[row];
        }
        const auto lk = ucols[z][c];
        const int64_t f = colbase[lk.first] + lk.second;
        const int32_t row = t.row0 + brow[b] + r, rs = lt.nstrtl[lk.first] - 1;
        return get(lt.a2(lk.first) + (int64_t)lk.second * lt.ndl[lk.first] + (row - rs)) * vsc[f] * csc[f] /
               rowsc[row];
      };
      int64_t pos = 0;
      for (size_t g0 = 0; g0 < ps.size();) {
        // the input group [g0, g1): consecutive segments with one (trimmed) input range, as the kernel groups them
        auto same_input = [&](size_t u, size_t v) {
          return ps[u].sg->src == ps[v].sg->src && ps[u].c0 == ps[v].c0 &&
                 ps[u].nc == ps[v].nc;
        };
        size_t g1 = g0 + 1;
        while (g1 < ps.size() && same_input(g1, g0)) g1++;
        const int32_t nc = ps[g0].nc, nv = (nc + 7) / 8, nks = (nv + 1) / 2;
        for (int32_t j = 0; j < nks; j++) {
          const int32_t nvj = std::min(2, nv - 2 * j);
          for (size_t z = g0; z < g1; z++) {
            const TcSeg2 &sg = *ps[z].sg;
            for (int b = 0; b < t.nblk; b++) {
              if (!(sg.mask >> b & 1)) continue;
              const int32_t R = t.R[b];
              const int parts = sg.fmt == TF_HILO ? 2 : 1;
              std::memset(base + pos, 0, (size_t)nvj * R * 16 * parts);
              for (int32_t u = 0; u < nvj; u++)
                for (int32_t e = 0; e < 8; e++) {
                  const int32_t c = 16 * j + 8 * u + e;  // column within the part
                  if (c >= nc) continue;
                  for (int32_t r = 0; r < R; r++) {
                    const double v = val(z, b, r, ps[z].c0 + c);
                    const uint16_t hi = enc(v);
                    std::memcpy(base + pos + ((int64_t)u * R + r) * 16 + e * 2, &hi, 2);
                    if (parts == 2) {
                      const uint16_t lo = enc(v - dec(hi));
                      std::memcpy(base + pos + ((int64_t)(nvj + u) * R + r) * 16 + e * 2, &lo, 2);
                    }
                  }
                }
              pos += (int64_t)nvj * R * 16 * parts;
              const int64_t sb = (int64_t)std::min(16, nc - 16 * j) * R * 2 * parts;
              stored_bytes += sb;
              if (t.stage == 1) stored_bytes1 += sb;
            }
          }
        }
        g0 = g1;
      }
    }
    L.stored_bytes = stored_bytes;
    L.stored_bytes1 = stored_bytes1;
  } catch (const std::bad_alloc &) {
    msg = "host allocation failed while building the layout";
    return HMVM_ENOMEM;
  }
  return HMVM_OK;
}

}  // namespace hmvm
