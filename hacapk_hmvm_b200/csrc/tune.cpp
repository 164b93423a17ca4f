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
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
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

// ---- shape classes and a persistent choice ------------------------------------
// A matrix's shape-class histogram: the fraction of its stored elements in each
// (kind, rows, width) class -- kind dense or low-rank, rows = the leaf's rows,
// width = its columns (dense) or rank (low-rank), each in 8 power-of-two
// buckets.  Matrices from one family (kernel, geometry, leaf size, tolerance)
// have nearly the same histogram whatever their size, and the same kernel
// configurations win on them; the tuning cache keys a measured choice by it.
namespace {

int shape_bucket(int64_t v, int first) {  // <= 2^first, <= 2^(first+1), ..., above 2^(first+6)
  int b = 0;
  int64_t lim = (int64_t)1 << first;
  while (b < 7 && v > lim) {
    b++;
    lim <<= 1;
  }
  return b;
}

void shape_histogram(const hmvm_leaves64* lv, float* h) {
  double acc[HMVM_SHAPE_BINS] = {0};
  double tot = 0;
  for (int32_t i = 0; i < lv->nlf; i++) {
    const bool lr = lv->ltmtx[i] == 1;
    const int64_t rows = lv->ndl[i], width = lr ? lv->kt[i] : lv->ndt[i];
    const double el = lr ? (double)lv->kt[i] * (lv->ndl[i] + lv->ndt[i]) : (double)lv->ndl[i] * lv->ndt[i];
    if (el <= 0) continue;
    const int bin = (lr ? 64 : 0) + 8 * shape_bucket(rows, 3) + shape_bucket(width, lr ? 1 : 3);
    acc[bin] += el;
    tot += el;
  }
  for (int b = 0; b < HMVM_SHAPE_BINS; b++) h[b] = tot > 0 ? (float)(acc[b] / tot) : 0.f;
}

// The device part of a cache key: its name (spaces as '_') and SM count.
int device_key(const hmvm_plan_opts& o, std::string& key) {
  int dev = o.device;
  if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return set_error(HMVM_ENODEV, "autotune: no usable CUDA device");
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    return set_error(HMVM_ENODEV, "autotune: no usable CUDA device");
  }
  std::string name(prop.name);
  for (char& c : name)
    if (c == ' ' || c == '\t') c = '_';
  key = name + " " + std::to_string(prop.multiProcessorCount);
  return HMVM_OK;
}

struct CacheEntry {
  std::string dev;  // name and SM count
  int precision = 0, lr_format = 0, kernel = 0, cfg1 = 0, cfg2 = 0, rows = 32;
  double total_ms = 0;
  std::vector<float> hist;
};

// Cache lines: "hmvm_tune 1 <device name> <SMs> <precision> <lr format> <kernel> <stage1 cfg> <stage2 cfg>
// <tile rows> <ms per apply> <HMVM_SHAPE_BINS fractions>"; other lines are ignored.
std::vector<CacheEntry> read_cache(const char* path) {
  std::vector<CacheEntry> v;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string tag, name;
    int ver = 0, sms = 0;
    CacheEntry e;
    if (!(is >> tag >> ver >> name >> sms) || tag != "hmvm_tune" || ver != 1) continue;
    if (!(is >> e.precision >> e.lr_format >> e.kernel >> e.cfg1 >> e.cfg2 >> e.rows >> e.total_ms)) continue;
    e.hist.resize(HMVM_SHAPE_BINS);
    bool ok = true;
    for (int b = 0; b < HMVM_SHAPE_BINS && ok; b++) ok = (bool)(is >> e.hist[b]);
    if (!ok) continue;
    e.dev = name + " " + std::to_string(sms);
    v.push_back(e);
  }
  return v;
}

double hist_distance(const float* a, const std::vector<float>& b) {  // L1, in [0, 2]
  double d = 0;
  for (int k = 0; k < HMVM_SHAPE_BINS; k++) d += std::fabs((double)a[k] - (double)b[k]);
  return d;
}

}  // namespace

extern "C" int hmvm_b200_shape_histogram64(const hmvm_leaves64* lv, float* hist) {
  if (!lv || !hist) return set_error(HMVM_EINVAL, "NULL argument");
  shape_histogram(lv, hist);
  return HMVM_OK;
}

extern "C" int hmvm_b200_autotune_cached64(const hmvm_leaves64* lv, int32_t rowmat_is_float, const hmvm_plan_opts* base,
                                           int32_t reps, const char* cache_path, double max_distance,
                                           hmvm_plan_opts* best, hmvm_tune_report* report, int32_t* from_cache) {
  if (!lv || !best || !cache_path) return set_error(HMVM_EINVAL, "NULL argument");
  if (from_cache) *from_cache = 0;
  hmvm_plan_opts o0;
  hmvm_b200_default_opts(&o0);
  if (base) o0 = *base;
  if (rowmat_is_float) o0.precision = HMVM_FP32;
  const bool mixed = o0.precision == HMVM_MIXED;
  std::string dev;
  int rc = device_key(o0, dev);
  if (rc) return rc;
  float h[HMVM_SHAPE_BINS];
  shape_histogram(lv, h);
  if (max_distance < 0) max_distance = 0.45;
  // the closest stored choice for this device, precision and factor format
  int bi = -1;
  double bd = 0;
  const std::vector<CacheEntry> cache = read_cache(cache_path);
  for (size_t i = 0; i < cache.size(); i++) {
    const CacheEntry& e = cache[i];
    if (e.dev != dev || e.precision != o0.precision || (mixed && e.lr_format != o0.mixed_lr_format)) continue;
    const double d = hist_distance(h, e.hist);
    if (d <= max_distance && (bi < 0 || d < bd)) {
      bi = (int)i;
      bd = d;
    }
  }
  if (bi >= 0) {
    const CacheEntry& e = cache[bi];
    *best = o0;
    if (!mixed) best->kernel = e.kernel;
    best->stage1_cfg = e.cfg1;
    best->stage2_cfg = e.cfg2;
    best->max_tile_rows = e.rows;
    if (report) {
      std::memset(report, 0, sizeof(*report));
      report->n_entries = 1;
      report->best_entry = 0;
      hmvm_tune_entry& t = report->entries[0];
      t.kernel = e.kernel;
      t.stage1_cfg = e.cfg1;
      t.stage2_cfg = e.cfg2;
      t.max_tile_rows = e.rows;
      t.total_ms = e.total_ms;  // as measured on the matrix it was tuned on
    }
    if (from_cache) *from_cache = 1;
    return HMVM_OK;
  }
  hmvm_tune_report rep;
  rc = hmvm_b200_autotune64(lv, rowmat_is_float, &o0, reps, best, &rep);
  if (rc) return rc;
  if (report) *report = rep;
  if (rep.best_entry >= 0) {
    const hmvm_tune_entry& t = rep.entries[rep.best_entry];
    std::ofstream f(cache_path, std::ios::app);
    if (!f) return set_error(HMVM_EIO, std::string("autotune: cannot append to ") + cache_path);
    char head[512];
    std::snprintf(head, sizeof head, "hmvm_tune 1 %s %d %d %d %d %d %d %.6g", dev.c_str(), o0.precision,
                  o0.mixed_lr_format, mixed ? 0 : best->kernel, best->stage1_cfg, best->stage2_cfg,
                  best->max_tile_rows, t.total_ms);
    f << head;
    for (int b = 0; b < HMVM_SHAPE_BINS; b++) f << ' ' << h[b];
    f << '\n';
    if (!f) return set_error(HMVM_EIO, std::string("autotune: cannot append to ") + cache_path);
  }
  return HMVM_OK;
}
