// The autotuner: picks, per leaf shape class, the kernel configuration that
// runs it fastest on this device, by timing candidate plans of the matrix
// itself.
//
// Shape classes: the V stage (stacked low-rank V factors, one x segment per
// panel) and the row stage (row tiles of dense leaves and U factors).  The
// choices per class: one warp per team (the TMA-ring stream kernel, 8 ring /
// input-buffer shapes) or teams of 1..16 warps per tile item (the
// register-streaming tile kernel, 8 warp-group shapes) -- the warp-versus-block
// assignment -- for plain plans; the 8 ring / input-buffer shapes of the
// mixed-precision kernel for mixed plans; and the tile shape (rows per row
// tile: 32 or 16).  Each candidate plan is timed stage by stage with CUDA
// events (hmvm_b200_plan_profile); the best configuration of each stage is
// combined and the combination is timed too, and the fastest measured plan wins.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "hmvm_b200.h"

namespace hmvm {
int set_error(int status, const std::string& msg);
}
using hmvm::set_error;

namespace {

struct Cand {
  int kernel, cfg1, cfg2, rows;
};

// Times `reps` applies of a plan for (lv, o); fills e.
int time_plan(const hmvm_leaves64* lv, bool f32, const hmvm_plan_opts& o, int reps, void* x, void* y,
              cudaStream_t st, hmvm_tune_entry* e) {
  hmvm_plan* p = nullptr;
  int rc = f32 ? hmvm_b200_plan_create64_f(lv, &o, &p) : hmvm_b200_plan_create64_d(lv, &o, &p);
  if (rc) return rc;
  for (int i = 0; i < 2 && !rc; i++) rc = hmvm_b200_apply(p, x, y, st);
  if (!rc) rc = hmvm_b200_plan_profile(p, 1);
  for (int i = 0; i < reps && !rc; i++) rc = hmvm_b200_apply(p, x, y, st);
  double ms[4] = {0, 0, 0, 0};
  int32_t n = 0;
  if (!rc) rc = hmvm_b200_plan_profile_read(p, ms, &n);
  if (!rc) rc = hmvm_b200_plan_status(p);
  hmvm_plan_info info;
  if (!rc) rc = hmvm_b200_plan_get_info(p, &info);
  hmvm_b200_plan_destroy(p);
  if (rc) return rc;
  const double k = n > 0 ? 1.0 / n : 0.0;
  e->kernel = info.kernel;
  e->stage1_cfg = info.stage1_cfg;
  e->stage2_cfg = info.stage2_cfg;
  e->max_tile_rows = o.max_tile_rows > 0 ? o.max_tile_rows : 32;
  e->ctas_per_sm = info.ctas_per_sm;
  e->stage1_ms = (ms[0] + ms[1]) * k;  // the stage and its reduction
  e->stage2_ms = (ms[2] + ms[3]) * k;
  e->total_ms = e->stage1_ms + e->stage2_ms;
  return HMVM_OK;
}

}  // namespace

extern "C" int hmvm_b200_autotune64(const hmvm_leaves64* lv, int32_t rowmat_is_float, const hmvm_plan_opts* base,
                                    int32_t reps, hmvm_plan_opts* best, hmvm_tune_report* report) {
  if (!lv || !best) return set_error(HMVM_EINVAL, "NULL argument");
  hmvm_plan_opts o0;
  hmvm_b200_default_opts(&o0);
  if (base) o0 = *base;
  if (rowmat_is_float) o0.precision = HMVM_FP32;
  if (reps <= 0) reps = 5;
  if (lv->nd <= 0) {
    *best = o0;
    if (report) std::memset(report, 0, sizeof(*report));
    return HMVM_OK;
  }
  const bool mixed = o0.precision == HMVM_MIXED;
  const size_t xb = (size_t)(lv->nd + 16) * (o0.precision == HMVM_FP32 ? 4 : 8);
  void* x = nullptr;
  void* y = nullptr;
  cudaStream_t st = nullptr;
  if (cudaMalloc(&x, xb) != cudaSuccess || cudaMalloc(&y, xb) != cudaSuccess ||
      cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    if (x) cudaFree(x);
    if (y) cudaFree(y);
    cudaGetLastError();
    return set_error(HMVM_ECUDA, "autotune: device buffers");
  }
  cudaMemset(x, 0x3f, xb);  // a normal, non-zero pattern for both FP32 and FP64

  // candidates: per tile shape, every configuration of each kernel family,
  // the same configuration for both stages (the stages are timed apart)
  std::vector<Cand> cands;
  for (int rows : {32, 16}) {
    if (mixed) {
      for (int c = 0; c < 8; c++) cands.push_back({-1, c, c, rows});  // the mixed kernel's shapes
    } else {
      for (int c = 0; c < 8; c++) cands.push_back({1, c, c, rows});  // the stream kernel's shapes
      for (int c = 0; c < 8; c++) cands.push_back({0, c, c, rows});
    }
  }
  std::vector<hmvm_tune_entry> ent;
  int rc = HMVM_OK;
  auto run = [&](const Cand& c) -> int {
    hmvm_plan_opts o = o0;
    if (c.kernel >= 0) o.kernel = c.kernel;
    o.stage1_cfg = c.cfg1;
    o.stage2_cfg = c.cfg2;
    o.max_tile_rows = c.rows;
    o.ctas_per_sm = base && base->ctas_per_sm > 0 ? base->ctas_per_sm : 0;
    hmvm_tune_entry e;
    std::memset(&e, 0, sizeof e);
    int r = time_plan(lv, rowmat_is_float != 0, o, reps, x, y, st, &e);
    if (!r) ent.push_back(e);
    return r;
  };
  for (const Cand& c : cands) {
    rc = run(c);
    if (rc) break;
  }
  // per (kernel, tile shape): the best V-stage and row-stage configurations, combined
  if (!rc) {
    const size_t nsingle = ent.size();
    for (size_t i = 0; i < nsingle && !rc; i++) {
      const hmvm_tune_entry& e = ent[i];
      bool first = true;  // one combination per (kernel, rows) group
      for (size_t j = 0; j < i; j++)
        if (ent[j].kernel == e.kernel && ent[j].max_tile_rows == e.max_tile_rows) first = false;
      if (!first) continue;
      int b1 = -1, b2 = -1;
      for (size_t j = 0; j < nsingle; j++) {
        if (ent[j].kernel != e.kernel || ent[j].max_tile_rows != e.max_tile_rows) continue;
        if (b1 < 0 || ent[j].stage1_ms < ent[b1].stage1_ms) b1 = (int)j;
        if (b2 < 0 || ent[j].stage2_ms < ent[b2].stage2_ms) b2 = (int)j;
      }
      if (ent[b1].stage1_cfg != ent[b2].stage2_cfg)
        rc = run({mixed ? -1 : e.kernel, ent[b1].stage1_cfg, ent[b2].stage2_cfg, e.max_tile_rows});
    }
  }
  cudaFree(x);
  cudaFree(y);
  cudaStreamDestroy(st);
  if (rc) return rc;
  int bi = 0;
  for (size_t i = 1; i < ent.size(); i++)
    if (ent[i].total_ms < ent[bi].total_ms) bi = (int)i;
  *best = o0;
  if (!mixed) best->kernel = ent[bi].kernel;
  best->stage1_cfg = ent[bi].stage1_cfg;
  best->stage2_cfg = ent[bi].stage2_cfg;
  best->max_tile_rows = ent[bi].max_tile_rows;
  if (report) {
    std::memset(report, 0, sizeof(*report));
    report->n_entries = (int32_t)std::min<size_t>(ent.size(), HMVM_TUNE_MAX_ENTRIES);
    report->best_entry = bi < HMVM_TUNE_MAX_ENTRIES ? bi : -1;
    for (int i = 0; i < report->n_entries; i++) report->entries[i] = ent[i];
  }
  return HMVM_OK;
}

extern "C" int hmvm_b200_autotune_d(const hmvm_matrix2_d* m, const hmvm_plan_opts* base, int32_t reps,
                                    hmvm_plan_opts* best, hmvm_tune_report* report) {
  if (!m) return set_error(HMVM_EINVAL, "matrix is NULL");
  std::vector<int64_t> a1(m->nlf), a2(m->nlf);
  for (int i = 0; i < m->nlf; i++) {
    a1[i] = m->a1[i];
    a2[i] = m->a2[i];
  }
  hmvm_leaves64 lv;
  std::memset(&lv, 0, sizeof lv);
  lv.nd = m->nd;
  lv.nlf = m->nlf;
  lv.ktmax = m->ktmax;
  lv.len = m->len;
  lv.ltmtx = m->ltmtx;
  lv.kt = m->kt;
  lv.ndl = m->ndl;
  lv.ndt = m->ndt;
  lv.nstrtl = m->nstrtl;
  lv.nstrtt = m->nstrtt;
  lv.a1 = a1.data();
  lv.a2 = a2.data();
  lv.rowmat = m->rowmat;
  return hmvm_b200_autotune64(&lv, 0, base, reps, best, report);
}
