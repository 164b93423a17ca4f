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
#include <queue>
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

struct TcPart {  // one part of a row-stage segment's columns
  int32_t leaf;   // dense leaf, or -1 for a low-rank row group
  int32_t group;  // row group when leaf < 0
  int32_t fmt;    // its columns' format (low-rank)
  int32_t ncols;
};

struct TcSeg {
  int32_t src, ncols, fmt;
  int32_t part_first, nparts;  // row stage
};

struct TcTile {
  int32_t stage = 2;
  int32_t row0 = 0, nrows = 0;  // row stage: rows; V stage: panel rows
  int32_t panel_row0 = 0;       // V stage: first entry in panel_rows
  int32_t seg_first = 0, nseg = 0;
  int64_t nvec = 0;
};

inline int64_t seg_vectors(int32_t ncols, int fmt) { return (int64_t)((ncols + 7) / 8) * (fmt == TF_HILO ? 2 : 1); }

// Byte offset, within a segment of `ncols` columns stored K-step-major for R
// rows, of element (row r, column c), hi (lo = false) or lo part.
inline int64_t tc_elem_off(int32_t ncols, int fmt, int32_t R, int32_t r, int32_t c, bool lo) {
  const int h = fmt == TF_HILO ? 2 : 1;
  const int32_t nv = (ncols + 7) / 8;
  const int32_t j = c >> 4, u = (c >> 3) & 1, e = c & 7;
  const int32_t nvj = std::min(2, nv - 2 * j);
  int64_t off = (int64_t)j * 2 * h * R * 16 + (int64_t)u * R * 16 + (int64_t)r * 16 + e * 2;
  if (lo) off += (int64_t)nvj * R * 16;
  return off;
}

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

    // ---- V stage: panels of <= 128 rows per (column group, format) -------------------
    std::vector<TcTile> tb;
    std::vector<TcSeg> sb;
    std::vector<TcPart> parts;
    std::vector<std::pair<int32_t, int32_t>> panel_rows;  // (leaf, k)
    for (int32_t c = 0; c < (int32_t)cg_members.size(); c++) {
      const auto &mem = cg_members[c];
      const int32_t ndt = lt.ndt[mem[0]], st = lt.nstrtt[mem[0]];
      for (int fm = TF_HILO; fm >= TF_HI; fm--) {
        std::vector<std::pair<int32_t, int32_t>> rows;
        for (int32_t i : mem)
          for (int32_t k = 0; k < lt.kt[i]; k++)
            if (col_fmt[colbase[i] + k] == fm) rows.emplace_back(i, k);
        const int32_t npanels = (int32_t)((rows.size() + kTcwPanelRows - 1) / kTcwPanelRows);
        for (int32_t p = 0; p < npanels; p++) {
          // even split so no panel is a sliver
          const size_t a = rows.size() * p / npanels, e = rows.size() * (p + 1) / npanels;
          TcTile t;
          t.stage = 1;
          t.nrows = (int32_t)(e - a);
          t.panel_row0 = (int32_t)panel_rows.size();
          for (size_t r = a; r < e; r++) {
            const auto lk = rows[r];
            const int64_t f = colbase[lk.first] + lk.second;
            L.out_idx.push_back((int32_t)slot_of_col[f]);
            L.tscale.push_back((float)(1.0 / csc[f]));
            panel_rows.push_back(lk);
          }
          t.seg_first = (int32_t)sb.size();
          t.nseg = 1;
          sb.push_back(TcSeg{st - 1, ndt, fm, -1, 0});
          t.nvec = seg_vectors(ndt, fm);
          tb.push_back(t);
        }
      }
    }
    const int32_t n1 = (int32_t)tb.size();
    L.tscale_rows0 = (int32_t)L.tscale.size();

    // ---- row stage: tiles with their dense and low-rank segments ---------------------
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
    for (int32_t ti = 0; ti < nrt; ti++) {
      TcTile t;
      t.stage = 2;
      t.row0 = trow0[ti];
      t.nrows = tnrows[ti];
      t.seg_first = (int32_t)sb.size();
      for (int32_t d = dcount[ti]; d < dcount[ti + 1]; d++) {
        const int32_t i = dlist[d];
        const int32_t src = lt.nstrtt[i] - 1;
        if (t.nseg > 0) {
          TcSeg &last = sb.back();
          if (last.src >= 0 && last.src + last.ncols == src) {  // column-adjacent dense leaves merge
            last.ncols += lt.ndt[i];
            last.nparts++;
            parts.push_back(TcPart{i, -1, TF_HILO, lt.ndt[i]});
            continue;
          }
        }
        sb.push_back(TcSeg{src, lt.ndt[i], TF_HILO, (int32_t)parts.size(), 1});
        parts.push_back(TcPart{i, -1, TF_HILO, lt.ndt[i]});
        t.nseg++;
      }
      for (int32_t gg = gcount[ti]; gg < gcount[ti + 1]; gg++) {
        const int32_t g = glist[gg];
        for (int fm = TF_HILO; fm >= TF_HI; fm--) {
          const int32_t k = rg_k[(size_t)g * 2 + fm];
          if (k == 0) continue;
          sb.push_back(TcSeg{kTFlagTc | rg_slot[(size_t)g * 2 + fm], k, fm, (int32_t)parts.size(), 1});
          parts.push_back(TcPart{-1, g, fm, k});
          t.nseg++;
        }
      }
      for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++) t.nvec += seg_vectors(sb[s].ncols, sb[s].fmt);
      tb.push_back(t);
    }
    const int32_t ntb = (int32_t)tb.size();

    // ---- row scales s_i: largest stored magnitude of each row -----------------------
    std::vector<double> rowmax(nd > 0 ? nd : 1, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
    for (int32_t k = n1; k < ntb; k++) {
      const TcTile &t = tb[k];
      for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++)
        for (int32_t p = sb[s].part_first; p < sb[s].part_first + sb[s].nparts; p++) {
          const TcPart &pt = parts[p];
          if (pt.leaf >= 0) {
            const int32_t i = pt.leaf, ndt = lt.ndt[i], rs = lt.nstrtl[i] - 1;
            for (int32_t r = 0; r < t.nrows; r++) {
              const int64_t src0 = lt.a1(i) + (int64_t)(t.row0 + r - rs) * ndt;
              double m = rowmax[t.row0 + r];
              for (int32_t c = 0; c < ndt; c++) m = std::max(m, std::fabs(get(src0 + c)));
              rowmax[t.row0 + r] = m;
            }
          } else {
            for (int32_t i : rg_members[pt.group]) {
              const int32_t ndl = lt.ndl[i], rs = lt.nstrtl[i] - 1;
              for (int32_t kk = 0; kk < lt.kt[i]; kk++) {
                const int64_t f = colbase[i] + kk;
                if (col_fmt[f] != pt.fmt) continue;
                const double w = vsc[f] * csc[f];
                const int64_t src0 = lt.a2(i) + (int64_t)kk * ndl + (t.row0 - rs);
                for (int32_t r = 0; r < t.nrows; r++)
                  rowmax[t.row0 + r] = std::max(rowmax[t.row0 + r], std::fabs(get(src0 + r) * w));
              }
            }
          }
        }
    }
    std::vector<double> rowsc(nd > 0 ? nd : 1, 1.0);
    for (int32_t r = 0; r < nd; r++) {
      rowsc[r] = pow2_for_max(rowmax[r]);
      L.tscale.push_back((float)rowsc[r]);
    }

    // ---- items ------------------------------------------------------------------------
    int64_t stage_bytes[2] = {0, 0};
    for (int32_t k = 0; k < ntb; k++) stage_bytes[k < n1 ? 0 : 1] += tb[k].nvec * tb[k].nrows * 16;
    const int64_t cap1 = std::max<int64_t>(64 * 1024, stage_bytes[0] / std::max<int64_t>(1, (int64_t)L.num_sms * 4));
    struct Item {
      int32_t tile, j0, j1, mode, out_base;  // V stage: K steps [j0, j1) of the panel
      int64_t cost;
    };
    std::vector<Item> items;
    std::vector<int32_t> tile_item0(ntb + 1);
    int64_t p_len = 0;
    for (int32_t k = 0; k < ntb; k++) {
      const TcTile &t = tb[k];
      tile_item0[k] = (int32_t)items.size();
      const int64_t bytes = t.nvec * t.nrows * 16;
      if (t.stage == 2) {
        items.push_back(Item{k, 0, 0, 0, t.row0, bytes + 2048});
        continue;
      }
      const TcSeg &sg = sb[t.seg_first];
      const int32_t nks = (sg.ncols + 15) / 16;
      const int32_t nparts = (int32_t)std::min<int64_t>(nks, (bytes + cap1 - 1) / cap1);
      if (nparts <= 1) {
        items.push_back(Item{k, 0, nks, 1, t.panel_row0, bytes + 2048});
        continue;
      }
      const int64_t pb = p_len;
      p_len += (int64_t)nparts * t.nrows;
      for (int32_t r = 0; r < t.nrows; r++) {
        L.red1.push_back(L.out_idx[t.panel_row0 + r]);
        L.red1.push_back((int32_t)(pb + r));
        L.red1.push_back(nparts);
        L.red1.push_back(t.nrows);
      }
      for (int32_t q = 0; q < nparts; q++) {
        const int32_t j0 = (int32_t)((int64_t)nks * q / nparts), j1 = (int32_t)((int64_t)nks * (q + 1) / nparts);
        items.push_back(Item{k, j0, j1, 2, (int32_t)(pb + (int64_t)q * t.nrows), bytes * (j1 - j0) / nks + 2048});
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

    // ---- descriptors --------------------------------------------------------------------
    const int32_t nitems = (int32_t)items.size();
    L.tiles.resize(nitems);
    L.segs.clear();
    // by item index: data offset and vectors, and the item's first vector within its tile's packing
    std::vector<int64_t> item_off(nitems), item_nvec(nitems), item_src_off(nitems);
    int64_t off = 0;
    for (int32_t k = 0; k < nitems; k++) {
      const Item &it = items[order[k]];
      const TcTile &t = tb[it.tile];
      hmvm_tile_desc &d = L.tiles[k];
      d.data_off = off;
      d.seg_begin = (int32_t)L.segs.size();
      d.out_base = it.out_base;
      d.nrows = (int16_t)t.nrows;
      d.mode = (int16_t)it.mode;
      int64_t nvec = 0, src_off = 0;
      if (t.stage == 1) {
        const TcSeg &sg = sb[t.seg_first];
        const int h = sg.fmt == TF_HILO ? 2 : 1;
        const int32_t c0 = 16 * it.j0, nc = std::min(sg.ncols - c0, 16 * (it.j1 - it.j0));
        L.segs.push_back(hmvm_seg_desc{sg.src + c0, nc | (sg.fmt << kSegTypeShift)});
        d.nseg = 1;
        nvec = (int64_t)((nc + 7) / 8) * h;
        src_off = (int64_t)it.j0 * 2 * h;  // vectors before step j0
        d._pad = t.panel_row0;             // tscale index of panel row 0
      } else {
        for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++)
          L.segs.push_back(hmvm_seg_desc{sb[s].src, sb[s].ncols | (sb[s].fmt << kSegTypeShift)});
        d.nseg = t.nseg;
        nvec = t.nvec;
        d._pad = L.tscale_rows0 + t.row0;  // tscale index of the tile's row 0
      }
      d.nvec = (int32_t)nvec;
      item_off[order[k]] = off;
      item_nvec[order[k]] = nvec;
      item_src_off[order[k]] = src_off;
      off += nvec * t.nrows;
    }
    L.data.resize((size_t)off);

    // ---- pack ---------------------------------------------------------------------------------
    int64_t stored_bytes = 0, stored_bytes1 = 0;
#pragma omp parallel reduction(+ : stored_bytes, stored_bytes1)
    {
      std::vector<Vec16> buf;
#pragma omp for schedule(dynamic, 4)
      for (int32_t k = 0; k < ntb; k++) {
        const TcTile &t = tb[k];
        const int32_t R = t.nrows;
        buf.assign((size_t)t.nvec * R, Vec16{{0, 0, 0, 0}});
        char *base = reinterpret_cast<char *>(buf.data());
        int64_t sbase = 0;  // byte offset of the current segment
        for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++) {
          const TcSeg &sg = sb[s];
          auto put = [&](int32_t r, int32_t c, double v) {
            const uint16_t hi = enc(v);
            std::memcpy(base + sbase + tc_elem_off(sg.ncols, sg.fmt, R, r, c, false), &hi, 2);
            if (sg.fmt == TF_HILO) {
              const uint16_t lo = enc(v - dec(hi));
              std::memcpy(base + sbase + tc_elem_off(sg.ncols, sg.fmt, R, r, c, true), &lo, 2);
            }
          };
          if (t.stage == 1) {
            for (int32_t r = 0; r < R; r++) {
              const auto lk = panel_rows[t.panel_row0 + r];
              const int32_t i = lk.first, kk = lk.second;
              const double inv = 1.0 / vsc[colbase[i] + kk];
              const int64_t src0 = lt.a1(i) + (int64_t)kk * lt.ndt[i];
              for (int32_t c = 0; c < sg.ncols; c++) put(r, c, get(src0 + c) * inv);
            }
          } else {
            int32_t pc = 0;
            for (int32_t p = sg.part_first; p < sg.part_first + sg.nparts; p++) {
              const TcPart &pt = parts[p];
              if (pt.leaf >= 0) {
                const int32_t i = pt.leaf, ndt = lt.ndt[i], rs = lt.nstrtl[i] - 1;
                for (int32_t r = 0; r < R; r++) {
                  const double inv = 1.0 / rowsc[t.row0 + r];
                  const int64_t src0 = lt.a1(i) + (int64_t)(t.row0 + r - rs) * ndt;
                  for (int32_t c = 0; c < ndt; c++) put(r, pc + c, get(src0 + c) * inv);
                }
                pc += ndt;
              } else {
                int32_t kc = 0;
                for (int32_t i : rg_members[pt.group]) {
                  const int32_t ndl = lt.ndl[i], rs = lt.nstrtl[i] - 1;
                  for (int32_t kk = 0; kk < lt.kt[i]; kk++) {
                    const int64_t f = colbase[i] + kk;
                    if (col_fmt[f] != pt.fmt) continue;
                    const double w = vsc[f] * csc[f];
                    const int64_t src0 = lt.a2(i) + (int64_t)kk * ndl + (t.row0 - rs);
                    for (int32_t r = 0; r < R; r++) put(r, pc + kc, get(src0 + r) * w / rowsc[t.row0 + r]);
                    kc++;
                  }
                }
                pc += kc;
              }
            }
          }
          const int64_t sb_bytes = (int64_t)sg.ncols * R * 2 * (sg.fmt == TF_HILO ? 2 : 1);
          stored_bytes += sb_bytes;
          if (t.stage == 1) stored_bytes1 += sb_bytes;
          sbase += seg_vectors(sg.ncols, sg.fmt) * R * 16;
        }
        for (int32_t q = tile_item0[k]; q < tile_item0[k + 1]; q++)
          std::memcpy(L.data.data() + item_off[q], buf.data() + (size_t)item_src_off[q] * R,
                      (size_t)item_nvec[q] * R * sizeof(Vec16));
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
