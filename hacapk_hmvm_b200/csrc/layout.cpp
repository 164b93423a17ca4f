// Host planner: leaf list -> row-owned, vector-packed tiles (see layout.hpp).

#include "layout.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <queue>
#include <unordered_map>
#include <utility>

#include "numfmt.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace hmvm {

namespace {

constexpr int32_t kTFlag = (int32_t)0x80000000u;

inline int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

inline uint64_t key2(int32_t a, int32_t b) { return ((uint64_t)(uint32_t)a << 32) | (uint32_t)b; }

// One part of a stage-2 segment's column list.
struct Part {
  int32_t leaf;   // dense leaf, or -1 for a low-rank row group
  int32_t group;  // row group index when leaf < 0
  int32_t cls;    // column class of the row group's columns
  int32_t ncols;
};

struct TileBuild {
  int32_t row0 = 0, nrows = 0;  // stage 2
  int32_t stage = 2;
  int32_t panel_row0 = 0;       // stage 1: index into panel_rows / out_idx
  int32_t scale_base = 0;       // stage 1, mixed: index into rowscale
  int32_t mode = 0, out_base = 0;
  int32_t seg_first = 0, nseg = 0, nvec = 0;
};

struct SegBuild {
  int32_t src, ncols, type;
  int32_t part_first, nparts;  // into parts (stage 2)
};

template <class S>
inline double rd(const void *base, int64_t i) {
  return (double)static_cast<const S *>(base)[i];
}

// Writes one element of `type` (value already scaled) at byte `off` of buf.
inline void store_elem(char *buf, int64_t off, int type, double v) {
  switch (type) {
    case ST_F64: std::memcpy(buf + off, &v, 8); break;
    case ST_F32: {
      float f = (float)v;
      std::memcpy(buf + off, &f, 4);
      break;
    }
    case ST_F16: {
      uint16_t h = to_fp16(v);
      std::memcpy(buf + off, &h, 2);
      break;
    }
    case ST_BF16: {
      uint16_t h = to_bf16(v);
      std::memcpy(buf + off, &h, 2);
      break;
    }
    default: {
      uint8_t b = to_e4m3(v);
      std::memcpy(buf + off, &b, 1);
    }
  }
}

inline int elem_bytes(int type) { return 16 / seg_vec(type); }

}  // namespace

int validate_leaves(const LeafTable &lt, std::string &msg) {
  auto fail = [&](int32_t i, const char *what) {
    char buf[256];
    snprintf(buf, sizeof buf, "leaf %d: %s (ltmtx=%d kt=%d ndl=%d ndt=%d nstrtl=%d nstrtt=%d)", i, what,
             lt.ltmtx[i], lt.kt[i], lt.ndl[i], lt.ndt[i], lt.nstrtl[i], lt.nstrtt[i]);
    msg = buf;
    return HMVM_EINVAL;
  };
  if (lt.nd < 0 || lt.nlf < 0 || lt.len < 0) {
    msg = "negative nd, nlf or len";
    return HMVM_EINVAL;
  }
  if (lt.nlf > 0 && (!lt.ltmtx || !lt.kt || !lt.ndl || !lt.ndt || !lt.nstrtl || !lt.nstrtt ||
                     (!lt.a1_32 && !lt.a1_64) || (!lt.a2_32 && !lt.a2_64))) {
    msg = "missing leaf array";
    return HMVM_EINVAL;
  }
  if (lt.len > 0 && !lt.rowmat) {
    msg = "missing rowmat";
    return HMVM_EINVAL;
  }
  for (int32_t i = 0; i < lt.nlf; i++) {
    int32_t ty = lt.ltmtx[i], kt = lt.kt[i], ndl = lt.ndl[i], ndt = lt.ndt[i];
    int32_t sl = lt.nstrtl[i], st = lt.nstrtt[i];
    if (ty != 1 && ty != 2) return fail(i, "ltmtx must be 1 (low-rank) or 2 (dense)");
    if (ndl < 0 || ndt < 0) return fail(i, "negative ndl/ndt");
    if (ndl > 0 && (sl < 1 || (int64_t)sl - 1 + ndl > lt.nd)) return fail(i, "row range outside 1..nd");
    if (ndt > 0 && (st < 1 || (int64_t)st - 1 + ndt > lt.nd)) return fail(i, "column range outside 1..nd");
    int64_t a1 = lt.a1(i);
    if (ty == 1) {
      if (kt < 0) return fail(i, "negative kt");
      if (kt > lt.ktmax) return fail(i, "kt > ktmax");
      int64_t a2 = lt.a2(i);
      int64_t n1 = (int64_t)kt * ndt, n2 = (int64_t)kt * ndl;
      if (n1 > 0 && (a1 < 0 || a1 + n1 > lt.len)) return fail(i, "a1 range outside rowmat");
      if (n2 > 0 && (a2 < 0 || a2 + n2 > lt.len)) return fail(i, "a2 range outside rowmat");
    } else {
      int64_t n1 = (int64_t)ndl * ndt;
      if (n1 > 0 && (a1 < 0 || a1 + n1 > lt.len)) return fail(i, "a1 range outside rowmat");
    }
  }
  return HMVM_OK;
}

int default_stage_cfg(int precision, int kernel, int stage) {
  if (precision == HMVM_MIXED) return stage == 1 ? kDefaultMixedCfg1 : kDefaultMixedCfg2;
  if (kernel == 0) return stage == 1 ? kDefaultStage1Cfg : kDefaultStage2Cfg;
  return (precision == HMVM_FP32 && stage == 2) ? 1 : kDefaultStreamCfg;
}

int build_layout(const LeafTable &lt, const hmvm_plan_opts &opts, int num_sms, HostLayout &L,
                 std::string &msg, int ctas2_per_sm) {
  int rc = validate_leaves(lt, msg);
  if (rc) return rc;
  if (opts.precision != HMVM_FP64 && opts.precision != HMVM_FP32 && opts.precision != HMVM_MIXED) {
    msg = "unsupported precision";
    return HMVM_EINVAL;
  }
  try {
    L = HostLayout();
    L.precision = opts.precision;
    L.mixed = opts.precision == HMVM_MIXED;
    L.elem_size = opts.precision == HMVM_FP32 ? 4 : 8;  // of x, y and the partial sums
    L.vec = 16 / L.elem_size;
    L.nd = lt.nd;
    L.nlf = lt.nlf;
    L.num_sms = num_sms > 0 ? num_sms : 148;
    L.kernel = (opts.kernel == 0 && !L.mixed) ? 0 : 1;
    const int ncfg = L.mixed ? kNumMixedCfgs : (L.kernel == 0 ? kNumCfgs : kNumStreamCfgs);
    const int d1 = default_stage_cfg(opts.precision, L.kernel, 1);
    const int d2 = default_stage_cfg(opts.precision, L.kernel, 2);
    L.stage1_cfg = (opts.stage1_cfg >= 0 && opts.stage1_cfg < ncfg) ? opts.stage1_cfg : d1;
    L.stage2_cfg = (opts.stage2_cfg >= 0 && opts.stage2_cfg < ncfg) ? opts.stage2_cfg : d2;
    L.ctas_per_sm = opts.ctas_per_sm > 0 ? opts.ctas_per_sm
                    : (L.kernel == 0 ? kDefaultCtasPerSm : kDefaultStreamCtasPerSm);
    L.ctas2_per_sm = ctas2_per_sm > 0 ? ctas2_per_sm : L.ctas_per_sm;
    const int VEC = L.vec;  // plain plans: elements per vector
    // 16 right-hand sides per pass run on the tensor cores (mixed plans only)
    const int nrhs_max = (L.mixed && opts.nrhs_max >= kTcNrhs) ? kTcNrhs
                                                               : std::min(std::max(opts.nrhs_max, 1), kMaxNrhsPass);
    L.nrhs_max = nrhs_max;
    const int RMAX = (opts.max_tile_rows >= 1 && opts.max_tile_rows <= kMaxRows) ? opts.max_tile_rows : kMaxRows;
    const int32_t nd = lt.nd, nlf = lt.nlf;
    const bool srcf = lt.rowmat_is_float;
    auto get = [&](int64_t idx) { return srcf ? rd<float>(lt.rowmat, idx) : rd<double>(lt.rowmat, idx); };

    // Column classes: plain plans have one (FP64 or FP32); mixed plans have
    // FP32 (leading terms), FP16/BF16 and FP8 E4M3 (terms below eps).
    const int base_type = opts.precision == HMVM_FP32 ? ST_F32 : ST_F64;
    const int lr16 = opts.mixed_lr_format == HMVM_LR_BF16 ? ST_BF16 : ST_F16;
    const int ncls = L.mixed ? 3 : 1;
    const int cls_type[3] = {L.mixed ? (int)ST_F32 : base_type, lr16, ST_E4M3};

    // ---- leaf classes ---------------------------------------------------
    std::vector<uint8_t> live_lr(nlf, 0);
    std::vector<int64_t> colbase(nlf, -1);  // first flat column (leaf, k=0) of a live low-rank leaf
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
    // Per column: class and (mixed) the scales of its U and V factors.
    std::vector<uint8_t> col_cls(ncolflat, 0);
    std::vector<float> sc_u, sc_v;
    if (L.mixed) {
      sc_u.assign(ncolflat, 1.0f);
      sc_v.assign(ncolflat, 1.0f);
      const double fp8_eps = opts.mixed_fp8_eps;
      const double tau = opts.mixed_fp32_tau >= 0.0 ? opts.mixed_fp32_tau
                         : (opts.mixed_lr_format == HMVM_LR_BF16 ? 0.05 : 0.5);
#pragma omp parallel for schedule(dynamic, 64)
      for (int32_t i = 0; i < nlf; i++) {
        if (!live_lr[i]) continue;
        const int32_t kt = lt.kt[i], ndl = lt.ndl[i], ndt = lt.ndt[i];
        std::vector<double> nu(kt), nv(kt), mu(kt), mv(kt);
        double block = 0.0;
        for (int32_t k = 0; k < kt; k++) {
          double su = 0, sv = 0, au = 0, av = 0;
          for (int32_t r = 0; r < ndl; r++) {
            double u = get(lt.a2(i) + (int64_t)k * ndl + r);
            su += u * u;
            au = std::max(au, std::fabs(u));
          }
          for (int32_t c = 0; c < ndt; c++) {
            double v = get(lt.a1(i) + (int64_t)k * ndt + c);
            sv += v * v;
            av = std::max(av, std::fabs(v));
          }
          nu[k] = std::sqrt(su);
          nv[k] = std::sqrt(sv);
          mu[k] = au;
          mv[k] = av;
          block = std::max(block, nu[k] * nv[k]);
        }
        for (int32_t k = 0; k < kt; k++) {
          const int64_t f = colbase[i] + k;
          const double term = nu[k] * nv[k];
          int cl = 1;
          if (term >= tau * block) cl = 0;
          else if (term < fp8_eps * block) cl = 2;
          col_cls[f] = (uint8_t)cl;
          if (cl == 1) {  // FP16/BF16: scale each factor to max |value| 1
            sc_u[f] = mu[k] > 0 ? (float)mu[k] : 1.0f;
            sc_v[f] = mv[k] > 0 ? (float)mv[k] : 1.0f;
          } else if (cl == 2) {  // E4M3: scale to max |value| 448
            sc_u[f] = mu[k] > 0 ? (float)(mu[k] / 448.0) : 1.0f;
            sc_v[f] = mv[k] > 0 ? (float)(mv[k] / 448.0) : 1.0f;
          }
        }
      }
      for (int64_t f = 0; f < ncolflat; f++) {
        (col_cls[f] == 0 ? L.cols_fp32 : col_cls[f] == 1 ? L.cols_lr16 : L.cols_fp8)++;
      }
    }

    // ---- row tiles: intervals between leaf row boundaries, <= RMAX rows ----
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
    std::vector<int32_t> trow0, tnrows;  // stage-2 row tiles in row order
    for (size_t b = 0; b + 1 < bnd.size(); b++) {
      int32_t a = bnd[b], e = bnd[b + 1], n = e - a;
      int32_t pieces = (n + RMAX - 1) / RMAX;
      for (int32_t p = 0; p < pieces; p++) {
        int32_t s0 = a + (int32_t)((int64_t)n * p / pieces), s1 = a + (int32_t)((int64_t)n * (p + 1) / pieces);
        trow0.push_back(s0);
        tnrows.push_back(s1 - s0);
      }
    }
    const int32_t nrt = (int32_t)trow0.size();
    std::vector<int32_t> row_tile(nd > 0 ? nd : 1);
    for (int32_t ti = 0; ti < nrt; ti++)
      for (int32_t r = trow0[ti]; r < trow0[ti] + tnrows[ti]; r++) row_tile[r] = ti;

    // ---- low-rank row groups / column groups and t slots ------------------
    std::unordered_map<uint64_t, int32_t> rgmap, cgmap;
    std::vector<std::vector<int32_t>> rg_members, cg_members;
    for (int32_t i = 0; i < nlf; i++) {
      if (!live_lr[i]) continue;
      uint64_t kr = key2(lt.nstrtl[i], lt.ndl[i]);
      auto it = rgmap.find(kr);
      int32_t g;
      if (it == rgmap.end()) {
        g = (int32_t)rg_members.size();
        rgmap.emplace(kr, g);
        rg_members.emplace_back();
      } else {
        g = it->second;
      }
      rg_members[g].push_back(i);
      uint64_t kc = key2(lt.nstrtt[i], lt.ndt[i]);
      auto jt = cgmap.find(kc);
      int32_t c;
      if (jt == cgmap.end()) {
        c = (int32_t)cg_members.size();
        cgmap.emplace(kc, c);
        cg_members.emplace_back();
      } else {
        c = jt->second;
      }
      cg_members[c].push_back(i);
    }
    const int32_t nrg = (int32_t)rg_members.size();
    // slots ordered by (row group, column class, leaf in file order, k)
    std::vector<int64_t> slot_of_col(ncolflat, -1);
    std::vector<int32_t> rg_slot((size_t)nrg * ncls), rg_k((size_t)nrg * ncls);
    int64_t t_len = 0;
    const int slot_align = L.mixed ? 4 : VEC;
    for (int32_t g = 0; g < nrg; g++) {
      for (int cl = 0; cl < ncls; cl++) {
        rg_slot[(size_t)g * ncls + cl] = (int32_t)t_len;
        int32_t k = 0;
        for (int32_t i : rg_members[g])
          for (int32_t kk = 0; kk < lt.kt[i]; kk++) {
            const int64_t f = colbase[i] + kk;
            if (col_cls[f] != cl) continue;
            slot_of_col[f] = t_len + k;
            k++;
          }
        rg_k[(size_t)g * ncls + cl] = k;
        t_len += round_up(k, slot_align);
      }
      if (t_len > INT32_MAX / 2) {
        msg = "intermediate vector too long";
        return HMVM_ERANGE;
      }
    }
    L.t_len = t_len;

    // ---- stage 1: column panels (one column class per panel) ---------------
    std::vector<TileBuild> tb;
    std::vector<SegBuild> sb;
    std::vector<Part> parts;
    std::vector<std::pair<int32_t, int32_t>> panel_rows;  // (leaf, k) per out_idx entry
    for (int32_t c = 0; c < (int32_t)cg_members.size(); c++) {
      const auto &mem = cg_members[c];
      int32_t ndt = lt.ndt[mem[0]], st = lt.nstrtt[mem[0]];
      for (int cl = 0; cl < ncls; cl++) {
        std::vector<std::pair<int32_t, int32_t>> rows;
        for (int32_t i : mem)
          for (int32_t k = 0; k < lt.kt[i]; k++)
            if (col_cls[colbase[i] + k] == cl) rows.emplace_back(i, k);
        const int type = cls_type[cl];
        for (size_t p0 = 0; p0 < rows.size(); p0 += kMaxRows) {
          int32_t R = (int32_t)std::min<size_t>(kMaxRows, rows.size() - p0);
          int32_t ob = (int32_t)L.out_idx.size();
          TileBuild t;
          t.stage = 1;
          t.nrows = R;
          t.panel_row0 = ob;
          t.scale_base = (int32_t)L.rowscale.size();
          for (int32_t r = 0; r < R; r++) {
            auto lk = rows[p0 + r];
            const int64_t f = colbase[lk.first] + lk.second;
            L.out_idx.push_back((int32_t)slot_of_col[f]);
            panel_rows.push_back(lk);
            if (L.mixed) L.rowscale.push_back((double)sc_u[f] * (double)sc_v[f]);
          }
          t.mode = 1;
          t.out_base = ob;
          t.seg_first = (int32_t)sb.size();
          t.nseg = 1;
          sb.push_back(SegBuild{st - 1, ndt, type, -1, 0});
          t.nvec = (ndt + seg_vec(type) - 1) / seg_vec(type);
          tb.push_back(t);
        }
      }
    }
    const int32_t n1 = (int32_t)tb.size();

    // ---- stage 2: row tiles ---------------------------------------------
    std::vector<int32_t> dcount(nrt + 1, 0), gcount(nrt + 1, 0);
    for (int32_t i = 0; i < nlf; i++) {
      if (lt.ltmtx[i] != 2 || lt.ndl[i] <= 0 || lt.ndt[i] <= 0) continue;
      int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
      for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) dcount[ti + 1]++;
    }
    for (int32_t g = 0; g < nrg; g++) {
      int32_t i = rg_members[g][0];
      int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
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
        int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
        for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) dlist[dpos[ti]++] = i;
      }
      for (int32_t g = 0; g < nrg; g++) {
        int32_t i = rg_members[g][0];
        int32_t r0 = lt.nstrtl[i] - 1, r1 = r0 + lt.ndl[i];
        for (int32_t ti = row_tile[r0]; ti < nrt && trow0[ti] < r1; ti++) glist[gpos[ti]++] = g;
      }
    }
    auto dense_type = [&](int32_t i) {
      if (!L.mixed) return base_type;
      // diagonal near-field blocks keep FP64
      return (lt.nstrtl[i] == lt.nstrtt[i] && lt.ndl[i] == lt.ndt[i]) ? (int)ST_F64 : (int)ST_F32;
    };
    for (int32_t ti = 0; ti < nrt; ti++) {
      TileBuild t;
      t.stage = 2;
      t.row0 = trow0[ti];
      t.nrows = tnrows[ti];
      t.mode = 0;
      t.out_base = trow0[ti];
      t.seg_first = (int32_t)sb.size();
      int32_t nvec = 0;
      // dense segments: merge leaves whose column ranges are adjacent (same type)
      for (int32_t d = dcount[ti]; d < dcount[ti + 1]; d++) {
        int32_t i = dlist[d];
        int32_t src = lt.nstrtt[i] - 1;
        const int type = dense_type(i);
        if (t.nseg > 0) {
          SegBuild &last = sb.back();
          if (last.src >= 0 && last.type == type && last.src + last.ncols == src) {
            last.ncols += lt.ndt[i];
            last.nparts++;
            parts.push_back(Part{i, -1, 0, lt.ndt[i]});
            continue;
          }
        }
        sb.push_back(SegBuild{src, lt.ndt[i], type, (int32_t)parts.size(), 1});
        parts.push_back(Part{i, -1, 0, lt.ndt[i]});
        t.nseg++;
      }
      for (int32_t gg = gcount[ti]; gg < gcount[ti + 1]; gg++) {
        int32_t g = glist[gg];
        for (int cl = 0; cl < ncls; cl++) {
          const int32_t k = rg_k[(size_t)g * ncls + cl];
          if (k == 0) continue;
          sb.push_back(SegBuild{kTFlag | rg_slot[(size_t)g * ncls + cl], k, cls_type[cl], (int32_t)parts.size(), 1});
          parts.push_back(Part{-1, g, cl, k});
          t.nseg++;
        }
      }
      if (L.mixed) {
        // segments of one storage type next to each other: the kernel runs
        // each type's vectors as one stretch
        auto rank = [](int ty) { return ty == ST_F64 ? 0 : ty == ST_F32 ? 1 : ty == ST_E4M3 ? 3 : 2; };
        std::stable_sort(sb.begin() + t.seg_first, sb.begin() + t.seg_first + t.nseg,
                         [&](const SegBuild &a, const SegBuild &b) { return rank(a.type) < rank(b.type); });
      }
      for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++)
        nvec += (sb[s].ncols + seg_vec(sb[s].type) - 1) / seg_vec(sb[s].type);
      t.nvec = nvec;
      tb.push_back(t);
    }
    const int32_t ntb = (int32_t)tb.size();

    // ---- items: tiles cut into contiguous vector ranges ----------------------
    // A tile whose bytes exceed the stage's bound, or (stream kernels) whose
    // inputs exceed the kernel's input buffer, is cut into vector ranges that
    // write partial sums; the reduction lists add them in order.
    L.stage1_teams = L.num_sms * L.ctas_per_sm *
                     (L.mixed ? kMixedCfgs[L.stage1_cfg].wpb : teams_per_cta(L.kernel, L.stage1_cfg));
    L.stage2_teams = L.num_sms * L.ctas2_per_sm *
                     (L.mixed ? kMixedCfgs[L.stage2_cfg].wpb : teams_per_cta(L.kernel, L.stage2_cfg));
    if (nrhs_max > 1) {
      // teams for the multi-RHS kernel, all resident at once (and no more than
      // the single-vector kernels launch)
      const bool f64 = !L.mixed && L.elem_size == 8;
      const int per_sm = nrhs_max == kTcNrhs ? kTcWarpsPerSm : (f64 ? kMultiWarpsPerSmF64 : kMultiWarpsPerSm);
      L.stage1_teams = std::min(L.stage1_teams, L.num_sms * per_sm);
      L.stage2_teams = std::min(L.stage2_teams, L.num_sms * per_sm);
    }
    int64_t stage_bytes[2] = {0, 0};
    for (int32_t k = 0; k < ntb; k++) stage_bytes[k < n1 ? 0 : 1] += (int64_t)tb[k].nvec * tb[k].nrows * 16;
    int64_t max_item[2];
    for (int st = 0; st < 2; st++) {
      int32_t nteams = st == 0 ? L.stage1_teams : L.stage2_teams;
      max_item[st] = stage_bytes[st] < kSmallStageBytes
                         ? std::max<int64_t>(kSmallItemBytes, stage_bytes[st] / std::max<int64_t>(1, (int64_t)nteams))
                         : std::max<int64_t>(kMinItemBytes, stage_bytes[st] / std::max<int64_t>(1, (int64_t)nteams * kItemsPerTeam));
    }
    struct Item {
      int32_t tile, va, vb, mode, out_base;
      int64_t cost;
    };
    std::vector<Item> items;
    items.reserve((size_t)ntb + ntb / 2);
    std::vector<int32_t> tile_item0(ntb + 1);
    int64_t p_len = 0;
    for (int32_t k = 0; k < ntb; k++) {
      const TileBuild &t = tb[k];
      tile_item0[k] = (int32_t)items.size();
      const int st = k < n1 ? 0 : 1;
      const int64_t bytes = (int64_t)t.nvec * t.nrows * 16;
      std::vector<int32_t> cuts;  // vector indices where items start (after 0)
      if (!L.mixed) {
        int32_t nparts = (int32_t)std::min<int64_t>(std::max<int64_t>(1, t.nvec),
                                                    (bytes + max_item[st] - 1) / max_item[st]);
        if (st == 0 && opts.split_cols > 0) {
          int32_t vmax = std::max(1, opts.split_cols / VEC);
          nparts = std::max(nparts, (t.nvec + vmax - 1) / vmax);
        }
        if (L.kernel == 1 || nrhs_max > 1) {
          // an item's x/t columns must fit the kernels' input buffers
          const int32_t cfg = st == 0 ? L.stage1_cfg : L.stage2_cfg;
          int32_t zcap = L.kernel == 1 ? kStreamCfgs[cfg].zcap : INT32_MAX;
          if (nrhs_max > 1) zcap = std::min(zcap, multi_zbytes(L.elem_size == 8) / (nrhs_max * L.elem_size));
          const int32_t vmax = std::max(1, zcap / VEC);
          nparts = std::max(nparts, (t.nvec + vmax - 1) / vmax);
        }
        for (int32_t q = 1; q < nparts; q++) cuts.push_back((int32_t)((int64_t)t.nvec * q / nparts));
      } else {
        // greedy: close an item before it exceeds the byte bound, the input
        // buffer or kMixedMaxSegs segments
        const int cfg = st == 0 ? L.stage1_cfg : L.stage2_cfg;
        const int64_t zcap = std::min<int64_t>(kMixedCfgs[cfg].zbytes,
                                               (nrhs_max == kTcNrhs ? kTcItemZBytes : kMultiZBytes) / nrhs_max);
        const int64_t bcap = std::max<int64_t>(max_item[st], (int64_t)t.nrows * 16);
        const int32_t vsplit = (st == 0 && opts.split_cols > 0) ? std::max(1, opts.split_cols / 4) : INT32_MAX;
        int64_t zb = 0, by = 0;
        int32_t nseg = 0, nv_item = 0, v = 0;
        for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++) {
          const int32_t nvs = (sb[s].ncols + seg_vec(sb[s].type) - 1) / seg_vec(sb[s].type);
          const int64_t zv = seg_zbytes(sb[s].type);
          int32_t done = 0;
          bool seg_open = false;
          while (done < nvs) {
            if (!seg_open && nseg == kMixedMaxSegs) {  // segment cap: start a new item
              cuts.push_back(v);
              zb = by = 0;
              nseg = nv_item = 0;
            }
            if (!seg_open) {
              nseg++;
              seg_open = true;
            }
            int64_t room = std::min<int64_t>((zcap - zb) / zv, (bcap - by) / ((int64_t)t.nrows * 16));
            room = std::min<int64_t>(room, (int64_t)vsplit - nv_item);
            if (room <= 0) {  // full: the rest of this segment goes to a new item
              cuts.push_back(v);
              zb = by = 0;
              nseg = 1;
              nv_item = 0;
              continue;
            }
            const int32_t take = (int32_t)std::min<int64_t>(room, nvs - done);
            done += take;
            v += take;
            nv_item += take;
            zb += take * zv;
            by += (int64_t)take * t.nrows * 16;
          }
        }
      }
      const int32_t nparts = (int32_t)cuts.size() + 1;
      if (nparts <= 1) {
        items.push_back(Item{k, 0, t.nvec, t.mode, t.out_base, bytes + kItemOverheadBytes});
        continue;
      }
      // part q of the tile writes its R partial sums at pb + q*R
      int64_t pb = p_len;
      p_len += (int64_t)nparts * t.nrows;
      std::vector<int32_t> &red = st == 0 ? L.red1 : L.red2;
      for (int32_t r = 0; r < t.nrows; r++) {
        red.push_back(st == 0 ? L.out_idx[t.panel_row0 + r] : t.row0 + r);
        red.push_back((int32_t)(pb + r));
        red.push_back(nparts);
        red.push_back(t.nrows);
      }
      for (int32_t q = 0; q < nparts; q++) {
        int32_t va = q == 0 ? 0 : cuts[q - 1], vb = q + 1 < nparts ? cuts[q] : t.nvec;
        items.push_back(Item{k, va, vb, 2, (int32_t)(pb + (int64_t)q * t.nrows),
                             (int64_t)(vb - va) * t.nrows * 16 + kItemOverheadBytes});
      }
    }
    tile_item0[ntb] = (int32_t)items.size();
    if (p_len > INT32_MAX / 2) {
      msg = "partial-sum buffer too long";
      return HMVM_ERANGE;
    }
    L.p_len = p_len;
    L.split_rows = (int32_t)((L.red1.size() + L.red2.size()) / 4);
    const int32_t ni1 = tile_item0[n1];
    const int32_t ni2 = (int32_t)items.size() - ni1;

    // ---- team assignment (LPT) and ordering --------------------------------
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
      for (int32_t k = 0; k < count; k++) order[pos[team_of[k]]++] = first + k;  // item order within team
    };
    std::vector<int32_t> ord1, ord2, tb1, tb2;
    assign(0, ni1, L.stage1_teams, ord1, tb1);
    assign(ni1, ni2, L.stage2_teams, ord2, tb2);
    std::vector<int32_t> order;
    order.reserve(items.size());
    order.insert(order.end(), ord1.begin(), ord1.end());
    order.insert(order.end(), ord2.begin(), ord2.end());
    L.team_begin1 = tb1;
    L.team_begin2.resize(tb2.size());
    for (size_t k = 0; k < tb2.size(); k++) L.team_begin2[k] = tb2[k] + ni1;
    L.stage1_tiles = ni1;
    L.stage2_tiles = ni2;

    // ---- final descriptors (segments trimmed to each item's vector range) --
    const int32_t nitems = (int32_t)items.size();
    L.tiles.resize(nitems);
    L.segs.clear();
    L.segs.reserve(sb.size() + nitems);
    std::vector<int64_t> item_off(nitems);  // by item index
    int64_t off = 0;
    for (int32_t k = 0; k < nitems; k++) {
      const Item &it = items[order[k]];
      const TileBuild &t = tb[it.tile];
      hmvm_tile_desc &d = L.tiles[k];
      d.data_off = off;
      d.seg_begin = (int32_t)L.segs.size();
      d.nvec = it.vb - it.va;
      d.out_base = it.out_base;
      d.nrows = (int16_t)t.nrows;
      d.mode = (int16_t)it.mode;
      d._pad = (L.mixed && t.stage == 1) ? t.scale_base : 0;
      int32_t nseg = 0, sv0 = 0;
      for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++) {
        const int vs = seg_vec(sb[s].type);
        int32_t nv = (sb[s].ncols + vs - 1) / vs;
        int32_t lo = std::max(sv0, it.va), hi = std::min(sv0 + nv, it.vb);
        if (lo < hi) {
          int32_t skip = (lo - sv0) * vs;  // columns of the segment before this item
          int32_t ncols = std::min(sb[s].ncols - skip, (hi - lo) * vs);
          int32_t enc = L.mixed ? (ncols | (sb[s].type << kSegTypeShift)) : ncols;
          L.segs.push_back(hmvm_seg_desc{sb[s].src + skip, enc});
          nseg++;
        }
        sv0 += nv;
      }
      d.nseg = nseg;
      item_off[order[k]] = off;
      off += (int64_t)d.nvec * t.nrows;
    }
    // Not zeroed (UninitAlloc): the items partition [0, off) and the pack
    // below copies every item's whole range from a zero-padded tile buffer.
    L.data.resize((size_t)off);

    // ---- pack: each tile into a scratch buffer, then its items' ranges -----
    int64_t stored_bytes = 0, stored_bytes1 = 0;
#pragma omp parallel reduction(+ : stored_bytes, stored_bytes1)
    {
      std::vector<Vec16> buf;
#pragma omp for schedule(dynamic, 4)
      for (int32_t k = 0; k < ntb; k++) {
        const TileBuild &t = tb[k];
        const int32_t R = t.nrows;
        buf.assign((size_t)t.nvec * R, Vec16{{0, 0, 0, 0}});
        char *base = reinterpret_cast<char *>(buf.data());
        int64_t vs0 = 0;  // first vector of the current segment
        for (int32_t s = t.seg_first; s < t.seg_first + t.nseg; s++) {
          const SegBuild &sg = sb[s];
          const int type = sg.type, vs = seg_vec(type), eb = elem_bytes(type);
          const int lg = vs == 2 ? 1 : vs == 4 ? 2 : vs == 8 ? 3 : 4;  // vs is 2, 4, 8 or 16
          auto put = [&](int64_t c, int32_t r, double v) {
            store_elem(base, ((vs0 + (c >> lg)) * R + r) * 16 + (c & (vs - 1)) * eb, type, v);
          };
          if (t.stage == 1) {
            for (int32_t r = 0; r < R; r++) {
              auto lk = panel_rows[t.panel_row0 + r];
              int32_t i = lk.first, kk = lk.second;
              const double inv = L.mixed ? 1.0 / sc_v[colbase[i] + kk] : 1.0;
              int64_t src0 = lt.a1(i) + (int64_t)kk * lt.ndt[i];
              for (int32_t c = 0; c < sg.ncols; c++) put(c, r, get(src0 + c) * inv);
            }
          } else {
            int64_t pc = 0;  // column within segment
            for (int32_t p = sg.part_first; p < sg.part_first + sg.nparts; p++) {
              const Part &pt = parts[p];
              if (pt.leaf >= 0) {
                int32_t i = pt.leaf, ndt = lt.ndt[i];
                int32_t rs = lt.nstrtl[i] - 1;
                for (int32_t r = 0; r < R; r++) {
                  int64_t src0 = lt.a1(i) + (int64_t)(t.row0 + r - rs) * ndt;
                  for (int32_t c = 0; c < ndt; c++) put(pc + c, r, get(src0 + c));
                }
                pc += ndt;
              } else {
                int64_t kc = 0;
                for (int32_t i : rg_members[pt.group]) {
                  int32_t ndl = lt.ndl[i], rs = lt.nstrtl[i] - 1;
                  for (int32_t kk = 0; kk < lt.kt[i]; kk++) {
                    const int64_t f = colbase[i] + kk;
                    if (col_cls[f] != pt.cls) continue;
                    const double inv = L.mixed ? 1.0 / sc_u[f] : 1.0;
                    int64_t src0 = lt.a2(i) + (int64_t)kk * ndl + (t.row0 - rs);
                    for (int32_t r = 0; r < R; r++) put(pc + kc, r, get(src0 + r) * inv);
                    kc++;
                  }
                }
                pc += kc;
              }
            }
          }
          stored_bytes += (int64_t)sg.ncols * R * eb;
          if (t.stage == 1) stored_bytes1 += (int64_t)sg.ncols * R * eb;
          vs0 += (sg.ncols + vs - 1) / vs;  // the next segment starts at the next vector
        }
        for (int32_t q = tile_item0[k]; q < tile_item0[k + 1]; q++) {
          const Item &it = items[q];
          std::memcpy(L.data.data() + item_off[q], buf.data() + (size_t)it.va * R,
                      (size_t)(it.vb - it.va) * R * sizeof(Vec16));
        }
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
