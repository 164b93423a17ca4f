// C-ABI of the B200 HMVM library: plan creation (host planner + upload),
// kernel dispatch, host-buffer apply, the one-shot reference-shaped call, and
// the allocation-free apply.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "hmvm_b200.h"
#include "kernels_tc.cuh"
#include "kernels_tcw.cuh"
#include "layout.hpp"

namespace hmvm {

thread_local std::string g_last_error;

int set_error(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return set_error(e == cudaErrorMemoryAllocation ? HMVM_ENOMEM : HMVM_ECUDA, m);
}

#define HMVM_CUDA_TRY(call, what)                      \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

// Makes `dev` current for the scope and restores the caller's device after.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) return;
    ok = (prev == dev) || (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DeviceGuard() {
    int cur;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// A CUDA driver-API function by name, through the runtime (so the library
// needs no link-time dependency on libcuda), or nullptr.
void* driver_fn(const char* name) {
  void* f = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPointByVersion(name, &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return f;
}

// The calling thread's current CUDA context (nullptr if none or unknown).
CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = reinterpret_cast<Fn>(driver_fn("cuCtxGetCurrent"));
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

using KernelFn = void (*)(TileArgs);

// Launches a kernel of an apply; every kernel after the apply's first one is a
// programmatic dependent of its predecessor (it may start, and prefetch plan
// data, while the predecessor drains; it waits for it before reading its
// outputs -- griddep_wait in the kernels).
template <typename... P, typename... A>
cudaError_t launch_in_apply(bool& first, void (*fn)(P...), unsigned grid, unsigned block, size_t smem,
                            cudaStream_t st, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = first ? nullptr : attr;
  cfg.numAttrs = first ? 0 : 1;
  first = false;
  return cudaLaunchKernelEx(&cfg, fn, args...);
}
using MultiFn = void (*)(MultiArgs);

// The kernel instance of configuration `cfg` of a table in layout.hpp: the
// template arguments are read from the table itself, so the launch shape the
// host sizes shared memory for (stream_smem_bytes, mixed_smem_bytes) and the
// kernel's own layout cannot disagree.  An index outside the table picks its
// last entry.
template <typename T, int... I>
KernelFn tile_kernel_pick(int cfg, std::integer_sequence<int, I...>) {
  KernelFn fn = nullptr;
  ((fn = (cfg == I ? hmvm_tile_kernel<T, kCfgs[I].wg, kCfgs[I].tpc> : fn)), ...);
  return fn;
}
template <typename T>
KernelFn tile_kernel_for(int cfg) {
  if (cfg < 0 || cfg >= kNumCfgs) cfg = kNumCfgs - 1;
  return tile_kernel_pick<T>(cfg, std::make_integer_sequence<int, kNumCfgs>{});
}

template <typename T, int... I>
KernelFn stream_kernel_pick(int cfg, std::integer_sequence<int, I...>) {
  KernelFn fn = nullptr;
  ((fn = (cfg == I ? hmvm_stream_kernel<T, kStreamCfgs[I].wpb, kStreamCfgs[I].slots, kStreamCfgs[I].chunk,
                                        kStreamCfgs[I].zcap>
                   : fn)),
   ...);
  return fn;
}
template <typename T>
KernelFn stream_kernel_for(int cfg) {
  if (cfg < 0 || cfg >= kNumStreamCfgs) cfg = kNumStreamCfgs - 1;
  return stream_kernel_pick<T>(cfg, std::make_integer_sequence<int, kNumStreamCfgs>{});
}

template <int LR16, bool VST, int... I>
KernelFn mixed_kernel_pick(int cfg, std::integer_sequence<int, I...>) {
  KernelFn fn = nullptr;
  ((fn = (cfg == I ? hmvm_mixed_kernel<kMixedCfgs[I].wpb, kMixedCfgs[I].slots, kMixedCfgs[I].chunk,
                                       kMixedCfgs[I].zbytes, LR16, VST>
                   : fn)),
   ...);
  return fn;
}
template <int LR16, bool VST>
KernelFn mixed_kernel_lr(int cfg) {
  if (cfg < 0 || cfg >= kNumMixedCfgs) cfg = kNumMixedCfgs - 1;
  return mixed_kernel_pick<LR16, VST>(cfg, std::make_integer_sequence<int, kNumMixedCfgs>{});
}
inline KernelFn mixed_kernel_for(int cfg, bool bf16, int stage) {
  if (stage == 1) return bf16 ? mixed_kernel_lr<kBF16, true>(cfg) : mixed_kernel_lr<kF16, true>(cfg);
  return bf16 ? mixed_kernel_lr<kBF16, false>(cfg) : mixed_kernel_lr<kF16, false>(cfg);
}

struct Launch {
  KernelFn fn;
  int threads, smem;
};

// kernel: 0 tile kernel, 1 stream kernel, 2 / 3 mixed-precision kernel with FP16 / BF16 factors;
// stage: 1 (V stage) or 2 (row stage)
template <typename T>
Launch stage_launch(int kernel, int cfg, int stage) {
  if (kernel == 0) return Launch{tile_kernel_for<T>(cfg), 32 * kCfgs[cfg].wg * kCfgs[cfg].tpc, 0};
  if (kernel >= 2)
    return Launch{mixed_kernel_for(cfg, kernel == 3, stage), 32 * kMixedCfgs[cfg].wpb,
                  mixed_smem_bytes(kMixedCfgs[cfg])};
  const StreamCfg& c = kStreamCfgs[cfg];
  return Launch{stream_kernel_for<T>(cfg), 32 * c.wpb, stream_smem_bytes(c, (int)sizeof(T))};
}

}  // namespace hmvm

using namespace hmvm;

struct hmvm_plan {
  int device = 0;
  int precision = HMVM_FP64;
  int elem = 8;
  int32_t nd = 0, nlf = 0, n_lowrank = 0, n_dense = 0;
  int num_sms = 0, kernel = 1, ctas_per_sm = 3, ctas2_per_sm = 3, stage1_cfg = 0, stage2_cfg = 0;
  int32_t stage1_tiles = 0, stage2_tiles = 0, stage1_teams = 0, stage2_teams = 0, n_red1 = 0, n_red2 = 0;
  int64_t stored_elems = 0, device_bytes = 0, t_len = 0, p_len = 0;
  // device buffers
  void* d_data = nullptr;
  hmvm_tile_desc* d_tiles = nullptr;
  hmvm_seg_desc* d_segs = nullptr;
  int32_t* d_tb1 = nullptr;
  int32_t* d_tb2 = nullptr;
  int32_t* d_out_idx = nullptr;
  int4* d_red1 = nullptr;
  int4* d_red2 = nullptr;
  void* d_t = nullptr;
  void* d_p = nullptr;
  int* d_err = nullptr;
  void* d_x = nullptr;  // staging for apply_host
  void* d_y = nullptr;
  // mixed precision
  bool mixed = false;
  int mixed_kcode = 2;  // stage_launch code: 2 FP16 factors, 3 BF16 factors
  float* d_x32 = nullptr;
  double* d_scale = nullptr;
  int64_t cols_fp32 = 0, cols_lr16 = 0, cols_fp8 = 0, stored_bytes = 0;
  int t_elem = 8, p_elem = 8;  // bytes per t slot and per partial sum
  // device bounds checks (HMVM_DEVICE_CHECKS builds): buffer lengths, elements per
  // vector of plain layouts, and each stage kernel's input buffer in bytes
  LayoutCaps caps;
  int vec = 2;
  int64_t zcap1 = 0, zcap2 = 0;
  int64_t stage1_bytes = 0, stage2_bytes = 0;
  // multi-RHS (nrhs_max > 1): packed inputs, t and partial sums for up to nrhs_max rhs
  int nrhs_max = 1;
  double* d_xm64 = nullptr;
  float* d_xm32 = nullptr;
  void* d_tm = nullptr;
  void* d_pm = nullptr;
  // tensor-core passes (mixed plans with nrhs_max = 16)
  bool tc = false;
  uint16_t* d_xplanes = nullptr;
  uint16_t* d_tplanes = nullptr;
  float* d_scal = nullptr;
  unsigned* d_amax = nullptr;
  // wide tensor-core passes (FP32 and mixed plans made with nrhs_max >= 32):
  // 128 right-hand sides per pass, hmvm_tcw_kernel
  bool tcw = false, tcw_bf = false;
  uint16_t* d_xpl = nullptr;  // x input chunks [4][nd][64]
  uint16_t* d_tpl = nullptr;  // t input chunks [4][tpl_rows][64]
  int64_t tpl_rows = 0;
  float* d_tscale = nullptr;  // V-stage 2^-c per panel row, then the row scale s_i per y row
  float* d_xscale = nullptr;  // sigma_x per right-hand side of the current pass
  unsigned* d_amax128 = nullptr;
  float* d_part = nullptr;    // split V-stage panels' partial sums [p_len][128]
  int32_t* d_tblocks = nullptr;  // per item: rows of its row blocks, 8 bits each
  uint32_t* d_tgroups = nullptr;  // the step program: input group headers, MMA templates
  uint32_t* d_tops = nullptr;
  int32_t* d_tgfirst = nullptr;
  int tcw_ngops = 0;            // templates in d_tops, the zero ones included
  CUtensorMap xmap, tmap;     // the planes as 3-D tensors {8, rows, 32}
  void* d_xh = nullptr;  // staging for apply_multi_host
  void* d_yh = nullptr;
  size_t xh_bytes = 0;
  cudaStream_t cs_in = nullptr, cs_out = nullptr;  // apply_multi_host: copy streams
  std::vector<cudaEvent_t> pass_events;            // apply_multi_host: per-pass ordering
  // profiling: kEventsPerApply events per recorded apply
  bool profiling = false;
  cudaGraph_t graph = nullptr;       // hmvm_b200_plan_capture: one apply
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<cudaEvent_t> prof_events;
  int prof_count = 0;
};

struct hmvm_layout {
  HostLayout L;
};

namespace {

constexpr int kMaxProfiled = 4096;
constexpr int kEventsPerApply = 5;

void free_plan_buffers(hmvm_plan* p) {
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->graph_exec = nullptr;
  p->graph = nullptr;
  for (cudaEvent_t e : p->prof_events) cudaEventDestroy(e);
  for (cudaEvent_t e : p->pass_events) cudaEventDestroy(e);
  p->pass_events.clear();
  if (p->cs_in) cudaStreamDestroy(p->cs_in);
  if (p->cs_out) cudaStreamDestroy(p->cs_out);
  p->cs_in = p->cs_out = nullptr;
  p->prof_events.clear();
  void* bufs[] = {p->d_data, p->d_tiles, p->d_segs, p->d_tb1, p->d_tb2,  p->d_out_idx, p->d_red1,
                  p->d_red2, p->d_t,     p->d_p,    p->d_err, p->d_x,    p->d_y,       p->d_x32,
                  p->d_scale, p->d_xm64, p->d_xm32, p->d_tm,  p->d_pm,   p->d_xh,      p->d_yh,
                  p->d_xplanes, p->d_tplanes, p->d_scal, p->d_amax, p->d_xpl, p->d_tpl,
                  p->d_tscale, p->d_xscale, p->d_amax128, p->d_part, p->d_tblocks, p->d_tgroups,
                  p->d_tops, p->d_tgfirst};
  for (void* b : bufs)
    if (b) cudaFree(b);
}

int check_device(int want, int* dev_out, int* sms_out) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return set_error(HMVM_ENODEV, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  }
  int dev = want;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(HMVM_ENODEV, "cudaGetDevice failed");
  }
  if (dev >= n) return set_error(HMVM_EINVAL, "device ordinal out of range");
  cudaDeviceProp prop;
  HMVM_CUDA_TRY(cudaGetDeviceProperties(&prop, dev), "cudaGetDeviceProperties");
  if (prop.major < 10) {
    return set_error(HMVM_ENODEV, std::string("device ") + prop.name +
                                      " is not sm_100-class; this library is built for sm_100a only");
  }
  *dev_out = dev;
  *sms_out = prop.multiProcessorCount;
  return HMVM_OK;
}

template <typename Buf>
int upload(Buf** dst, const void* src, size_t bytes, int64_t* total) {
  size_t nb = bytes > 0 ? bytes : 16;
  HMVM_CUDA_TRY(cudaMalloc((void**)dst, nb), "cudaMalloc");
  if (bytes) HMVM_CUDA_TRY(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  if (total) *total += (int64_t)bytes;
  return HMVM_OK;
}

int plan_mode(const hmvm_plan* p);
template <bool VST>
MultiFn multi_kernel_for(int mode, int nr, int cfg);
int tc_prepare(const hmvm_plan* p);

// Dynamic shared memory beyond 48 KB must be enabled per kernel.
int tcw_prepare(const hmvm_plan* p);

template <typename T>
int prepare_kernels(const hmvm_plan* p) {
  if (p->tcw) return tcw_prepare(p);
  if (p->tc) {
    int rc = tc_prepare(p);
    if (rc) return rc;
  } else if (p->nrhs_max > 1) {
    const int smem = multi_smem_bytes(kMultiCfgs[kDefaultMultiCfg], plan_mode(p) == kModePlain64);
    for (int nr : {2, 4, 8})
      for (MultiFn f : {multi_kernel_for<true>(plan_mode(p), nr, kDefaultMultiCfg),
                        multi_kernel_for<false>(plan_mode(p), nr, kDefaultMultiCfg)})
        HMVM_CUDA_TRY(cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                      "cudaFuncSetAttribute");
  }
  for (int st = 1; st <= 2; st++) {
    Launch l = stage_launch<T>(p->mixed ? p->mixed_kcode : p->kernel, st == 1 ? p->stage1_cfg : p->stage2_cfg, st);
    if (l.smem > 0)
      HMVM_CUDA_TRY(cudaFuncSetAttribute((const void*)l.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, l.smem),
                    "cudaFuncSetAttribute");
  }
  return HMVM_OK;
}

// CTAs per SM that stay resident, per stage kernel of the configuration `o`
// selects (its defaults resolved as the planner resolves them): out[0] the V
// stage's, out[1] the row stage's.
template <typename T>
int resident_ctas_t(int kernel, int cfg1, int cfg2, int* out) {
  for (int st = 1; st <= 2; st++) {
    const Launch l = stage_launch<T>(kernel, st == 1 ? cfg1 : cfg2, st);
    if (l.smem > 0)
      HMVM_CUDA_TRY(cudaFuncSetAttribute((const void*)l.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, l.smem),
                    "cudaFuncSetAttribute");
    int nb = 0;
    HMVM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)l.fn, l.threads, l.smem),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    out[st - 1] = std::max(nb, 1);
  }
  return HMVM_OK;
}

int resident_ctas(const hmvm_plan_opts& o, int dev, int* out) {
  DeviceGuard g(dev);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  const bool mixed = o.precision == HMVM_MIXED;
  const int kernel = mixed ? (o.mixed_lr_format == HMVM_LR_BF16 ? 3 : 2) : (o.kernel == 0 ? 0 : 1);
  const int ncfg = mixed ? kNumMixedCfgs : (kernel == 0 ? kNumCfgs : kNumStreamCfgs);
  const int d1 = default_stage_cfg(o.precision, mixed ? 1 : kernel, 1);
  const int d2 = default_stage_cfg(o.precision, mixed ? 1 : kernel, 2);
  const int c1 = (o.stage1_cfg >= 0 && o.stage1_cfg < ncfg) ? o.stage1_cfg : d1;
  const int c2 = (o.stage2_cfg >= 0 && o.stage2_cfg < ncfg) ? o.stage2_cfg : d2;
  return o.precision == HMVM_FP32 ? resident_ctas_t<float>(kernel, c1, c2, out)
                                  : resident_ctas_t<double>(kernel, c1, c2, out);
}

// Plans of FP32 or mixed storage made for 32 or more right-hand sides take the
// wide tensor-core form.
bool tcw_wanted(const hmvm_plan_opts& o) {
  return (o.precision == HMVM_FP32 || o.precision == HMVM_MIXED) && o.nrhs_max >= kTcwMinNrhs;
}

// An input buffer [4][rows][64] of 16-bit values (four chunks: hi and lo parts
// of right-hand sides 0..63 and 64..127) as a 3-D tensor {64, rows, 4} with
// boxes {64, 16, 4} and 128-byte swizzle: one K step of the 128 right-hand
// sides' hi and lo parts per TMA copy, in the MMA's swizzled MN-major layout.
// Rows past the end read as zero.
int encode_planes_map(CUtensorMap* map, void* base, int64_t rows) {
  using Fn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                          const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                          CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static Fn fn = reinterpret_cast<Fn>(driver_fn("cuTensorMapEncodeTiled"));
  if (!fn) return set_error(HMVM_ECUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[3] = {64, (cuuint64_t)rows, 4};
  const cuuint64_t strides[2] = {128, (cuuint64_t)rows * 128};
  const cuuint32_t box[3] = {64, (cuuint32_t)kTcwStepCols, 4};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(HMVM_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return HMVM_OK;
}

// Device buffers and tensor maps of a wide tensor-core plan.
int tcw_buffers(hmvm_plan* p, const HostLayout& L) {
  p->tpl_rows = std::max<int64_t>(L.t_len, 1);
  const int64_t xrows = std::max<int32_t>(L.nd, 1);
  HMVM_CUDA_TRY(cudaMalloc(&p->d_xpl, (size_t)xrows * 512), "x planes");
  HMVM_CUDA_TRY(cudaMalloc(&p->d_tpl, (size_t)p->tpl_rows * 512), "t planes");
  HMVM_CUDA_TRY(cudaMemset(p->d_tpl, 0, (size_t)p->tpl_rows * 512), "t planes");
  HMVM_CUDA_TRY(cudaMalloc(&p->d_xscale, kTcwRhs * sizeof(float)), "x scales");
  HMVM_CUDA_TRY(cudaMalloc(&p->d_amax128, kTcwRhs * sizeof(unsigned)), "x maxima");
  HMVM_CUDA_TRY(cudaMalloc(&p->d_part, (size_t)(L.p_len + 1) * kTcwRhs * sizeof(float)), "partial sums");
  int rc = upload(&p->d_tscale, L.tscale.data(), L.tscale.size() * sizeof(float), nullptr);
  if (!rc) rc = upload(&p->d_tblocks, L.tblocks.data(), L.tblocks.size() * sizeof(int32_t), nullptr);
  if (!rc) rc = upload(&p->d_tgroups, L.tgroups.data(), L.tgroups.size() * sizeof(uint32_t), nullptr);
  if (!rc) rc = upload(&p->d_tops, L.tops.data(), L.tops.size() * sizeof(uint32_t), nullptr);
  p->tcw_ngops = (int)(L.tops.size() / 2);
  if (!rc) rc = upload(&p->d_tgfirst, L.tgfirst.data(), L.tgfirst.size() * sizeof(int32_t), nullptr);
  if (!rc) rc = encode_planes_map(&p->xmap, p->d_xpl, xrows);
  if (!rc) rc = encode_planes_map(&p->tmap, p->d_tpl, p->tpl_rows);
  return rc;
}

// sms_cap > 0: plan the layout's teams for that many SMs (a batch class shares the GPU
// with the other classes of its batch, which run in the same launches).
// The input buffer of a stage's kernel for a layout's shapes, in bytes, as the
// planner bounds items by it (0: the kernel has none, or the layout is the
// wide tensor-core one, whose items these checks do not describe).
int64_t stage_zcap_bytes(const HostLayout& L, int stage) {
  if (L.tcw) return 0;
  const int cfg = stage == 1 ? L.stage1_cfg : L.stage2_cfg;
  if (L.mixed)
    return std::min<int64_t>(kMixedCfgs[cfg].zbytes,
                             (L.nrhs_max == kTcNrhs ? kTcItemZBytes : kMultiZBytes) / L.nrhs_max);
  int64_t zcap = L.kernel == 1 ? (int64_t)kStreamCfgs[cfg].zcap : -1;
  if (L.nrhs_max > 1) {
    const int64_t zm = multi_zbytes(L.elem_size == 8) / ((int64_t)L.nrhs_max * L.elem_size);
    zcap = zcap < 0 ? zm : std::min(zcap, zm);
  }
  return zcap < 0 ? 0 : zcap * L.elem_size;
}

LayoutCaps caps_of(const HostLayout& L) {
  LayoutCaps c;
  c.data_vectors = (int64_t)L.data.size();
  c.n_segs = (int64_t)L.segs.size();
  c.n_out_idx = (int64_t)L.out_idx.size();
  c.t_len = L.t_len;
  c.p_len = L.p_len;
  c.nd = L.nd;
  c.n_rowscale = (int64_t)L.rowscale.size();
  c.n_tiles = (int32_t)L.tiles.size();
  c.max_rows = kMaxRows;
  c.max_segs = L.mixed ? kMixedMaxSegs : 0;
  c.mixed = L.mixed ? 1 : 0;
  return c;
}

const char* check_name(int rc) {
  switch (rc) {
    case kCheckData: return "its vectors leave the data stream";
    case kCheckSegs: return "its segment descriptors leave the segment table";
    case kCheckRows: return "its rows are outside 1..32 or its vectors negative";
    case kCheckOut: return "its output rows leave their buffer";
    case kCheckSlot: return "a t slot it writes is outside t";
    case kCheckSrc: return "a segment's columns leave x or t";
    case kCheckInputs: return "its inputs exceed the kernel's input buffer";
    case kCheckType: return "a segment's storage type is unknown";
    case kCheckScale: return "its row scales leave the row-scale table";
    default: return "bounds check failed";
  }
}

// Every descriptor of a single-vector layout against the buffers it indexes
// (validate.hpp); wide tensor-core layouts are not described by these checks.
int validate_layout(const HostLayout& L, std::string& msg) {
  if (L.tcw) return HMVM_OK;
  const LayoutCaps c = caps_of(L);
  const int64_t z1 = stage_zcap_bytes(L, 1), z2 = stage_zcap_bytes(L, 2);
  for (int32_t k = 0; k < (int32_t)L.tiles.size(); k++) {
    const bool st1 = k < L.stage1_tiles;
    const int rc = check_tile(L.tiles[k], L.segs.data(), L.out_idx.data(), c, L.vec, L.elem_size, st1 ? z1 : z2, st1);
    if (rc) {
      msg = "item " + std::to_string(k) + " (stage " + (st1 ? "1" : "2") + "): " + check_name(rc);
      return HMVM_ERANGE;
    }
  }
  for (int st = 1; st <= 2; st++) {
    const std::vector<int32_t>& red = st == 1 ? L.red1 : L.red2;
    for (size_t e = 0; e + 4 <= red.size(); e += 4)
      if (check_red(&red[e], c, st == 1)) {
        msg = "reduction entry " + std::to_string(e / 4) + " of stage " + std::to_string(st) +
              " reads or writes outside its buffers";
        return HMVM_ERANGE;
      }
    const std::vector<int32_t>& tb = st == 1 ? L.team_begin1 : L.team_begin2;
    const int32_t nt = st == 1 ? L.stage1_teams : L.stage2_teams;
    const int32_t first = st == 1 ? 0 : L.stage1_tiles, end = st == 1 ? L.stage1_tiles : (int32_t)L.tiles.size();
    if ((int64_t)tb.size() != (int64_t)nt + 1 || check_teams(tb.data(), nt, first, end)) {
      msg = "the team ranges of stage " + std::to_string(st) + " do not cover its items in order";
      return HMVM_ERANGE;
    }
  }
  return HMVM_OK;
}

int create_plan(const LeafTable& lt, const hmvm_plan_opts* opts_in, hmvm_plan** out, int sms_cap = 0) {
  if (!out) return set_error(HMVM_EINVAL, "plan output pointer is NULL");
  *out = nullptr;
  hmvm_plan_opts opts;
  hmvm_b200_default_opts(&opts);
  if (opts_in) opts = *opts_in;
  int dev = 0, sms = 0;
  int rc = check_device(opts.device, &dev, &sms);
  if (rc) return rc;
  int ctas2 = opts.ctas_per_sm;
  const bool want_tcw = tcw_wanted(opts);
  if (opts.ctas_per_sm <= 0 && !want_tcw) {
    // Persistent grids: per stage, as many CTAs per SM as can be resident at
    // once, so no CTA waits for another to finish.
    int r[2] = {1, 1};
    rc = resident_ctas(opts, dev, r);
    if (rc) return rc;
    opts.ctas_per_sm = r[0];
    ctas2 = r[1];
  }
  HostLayout* L = new (std::nothrow) HostLayout();
  if (!L) return set_error(HMVM_ENOMEM, "host allocation failed");
  std::string msg;
  const int lsms = sms_cap > 0 ? std::min(sms, sms_cap) : sms;
  rc = want_tcw ? build_tc_layout(lt, opts, lsms, *L, msg) : build_layout(lt, opts, lsms, *L, msg, ctas2);
  if (rc) {
    delete L;
    return set_error(rc, msg);
  }
  hmvm_plan* p = new (std::nothrow) hmvm_plan();
  if (!p) {
    delete L;
    return set_error(HMVM_ENOMEM, "host allocation failed");
  }
  p->device = dev;
  p->precision = L->precision;
  p->elem = L->elem_size;
  p->nd = L->nd;
  p->nlf = L->nlf;
  p->n_lowrank = L->n_lowrank;
  p->n_dense = L->n_dense;
  p->num_sms = lsms;  // the SMs its layout's teams were planned for
  p->kernel = L->kernel;
  p->ctas_per_sm = L->ctas_per_sm;
  p->ctas2_per_sm = L->ctas2_per_sm;
  p->stage1_cfg = L->stage1_cfg;
  p->stage2_cfg = L->stage2_cfg;
  p->stage1_tiles = L->stage1_tiles;
  p->stage2_tiles = L->stage2_tiles;
  p->stage1_teams = L->stage1_teams;
  p->stage2_teams = L->stage2_teams;
  p->n_red1 = (int32_t)(L->red1.size() / 4);
  p->n_red2 = (int32_t)(L->red2.size() / 4);
  p->stored_elems = L->stored_elems;
  p->t_len = L->t_len;
  p->p_len = L->p_len;
  p->mixed = L->mixed;
  p->nrhs_max = L->nrhs_max;
  p->tc = !L->tcw && L->mixed && L->nrhs_max == kTcNrhs;
  p->tcw = L->tcw;
  p->tcw_bf = L->tcw_bf16;
  p->mixed_kcode = opts.mixed_lr_format == HMVM_LR_BF16 ? 3 : 2;
  p->cols_fp32 = L->cols_fp32;
  p->cols_lr16 = L->cols_lr16;
  p->cols_fp8 = L->cols_fp8;
  p->t_elem = L->mixed ? 4 : L->elem_size;
  p->p_elem = L->elem_size;
  p->caps = caps_of(*L);
  p->vec = L->vec;
  p->zcap1 = stage_zcap_bytes(*L, 1);
  p->zcap2 = stage_zcap_bytes(*L, 2);
  if (kDeviceChecks) {  // checked builds also check the layout on the host
    std::string vmsg;
    rc = validate_layout(*L, vmsg);
    if (rc) {
      delete L;
      delete p;
      return set_error(rc, "layout check: " + vmsg);
    }
  }
  if (L->tcw) {
    // Algorithmic bytes per pass: the stored elements in their storage formats
    // (pairs count 4 bytes) and scales; per stage kernel also the 16-bit planes
    // it reads and writes and, for the row stage, Y (128 columns).
    const int64_t planes = 512 * ((int64_t)lt.nd + L->t_len);
    p->stored_bytes = L->stored_bytes + 4 * (int64_t)L->tscale.size();
    p->stage1_bytes = L->stored_bytes1 + 4 * (int64_t)L->tscale_rows0 + planes;
    p->stage2_bytes = L->stored_bytes - L->stored_bytes1 + 4 * (int64_t)lt.nd + planes +
                      (int64_t)lt.nd * kTcwRhs * L->elem_size;
  } else if (L->mixed) {
    // Algorithmic bytes: the stored elements in their storage formats, the
    // per-column scales, x and y once.
    p->stored_bytes = L->stored_bytes + 8 * (int64_t)L->rowscale.size();
    p->stage1_bytes = L->stored_bytes1 + 8 * (int64_t)L->rowscale.size() + 8 * (int64_t)lt.nd;
    p->stage2_bytes = L->stored_bytes - L->stored_bytes1 + 16 * (int64_t)lt.nd;
  } else {
    // Algorithmic bytes per stage: stored elements of the stage once, plus the
    // vectors it reads/writes once (the intermediate t is not counted).
    int64_t v_elems = 0;
    for (int32_t i = 0; i < lt.nlf; i++)
      if (lt.ltmtx[i] == 1) v_elems += (int64_t)lt.kt[i] * lt.ndt[i];
    p->stored_bytes = L->stored_elems * L->elem_size;
    p->stage1_bytes = (v_elems + (int64_t)lt.nd) * L->elem_size;
    p->stage2_bytes = (L->stored_elems - v_elems + 2 * (int64_t)lt.nd) * L->elem_size;
  }
  {
    DeviceGuard g(dev);
    if (!g.ok) rc = set_error(HMVM_ECUDA, "cannot select the plan's device");
    int64_t dbytes = 0;
    if (!rc) rc = upload(&p->d_data, L->data.data(), L->data.size() * sizeof(Vec16), &dbytes);
    p->device_bytes = dbytes;
    if (!rc) rc = upload(&p->d_tiles, L->tiles.data(), L->tiles.size() * sizeof(hmvm_tile_desc), nullptr);
    if (!rc) rc = upload(&p->d_segs, L->segs.data(), L->segs.size() * sizeof(hmvm_seg_desc), nullptr);
    if (!rc) rc = upload(&p->d_tb1, L->team_begin1.data(), L->team_begin1.size() * 4, nullptr);
    if (!rc) rc = upload(&p->d_tb2, L->team_begin2.data(), L->team_begin2.size() * 4, nullptr);
    if (!rc) rc = upload(&p->d_out_idx, L->out_idx.data(), L->out_idx.size() * 4, nullptr);
    if (!rc) rc = upload(&p->d_red1, L->red1.data(), L->red1.size() * 4, nullptr);
    if (!rc) rc = upload(&p->d_red2, L->red2.data(), L->red2.size() * 4, nullptr);
    // t: the padding slots of every row group must read as zero; stage 1 only
    // ever writes real slots, so one clear at creation keeps them zero.
    size_t tbytes = (size_t)(L->t_len + 16) * p->t_elem;
    if (!rc) {
      cudaError_t e = cudaMalloc(&p->d_t, tbytes);
      if (e == cudaSuccess) e = cudaMemset(p->d_t, 0, tbytes);
      if (e != cudaSuccess) rc = cuda_fail(e, "t buffer");
    }
    if (!rc) {
      cudaError_t e = cudaMalloc(&p->d_p, (size_t)(L->p_len + 16) * p->p_elem);
      if (e != cudaSuccess) rc = cuda_fail(e, "partial buffer");
    }
    if (!rc && L->mixed) {
      cudaError_t e = cudaMalloc(&p->d_x32, (size_t)(L->nd + 16) * sizeof(float));
      if (e != cudaSuccess) rc = cuda_fail(e, "x32 buffer");
      if (!rc) rc = upload(&p->d_scale, L->rowscale.data(), L->rowscale.size() * sizeof(double), nullptr);
    }
    if (!rc && p->tcw) rc = tcw_buffers(p, *L);
    if (!rc && p->nrhs_max > 1 && !p->tcw) {
      const size_t nr = (size_t)p->nrhs_max;
      cudaError_t e = cudaSuccess;
      if (p->precision != HMVM_FP32) e = cudaMalloc(&p->d_xm64, (size_t)(L->nd + 16) * nr * sizeof(double));
      if (e == cudaSuccess && p->precision != HMVM_FP64)
        e = cudaMalloc(&p->d_xm32, (size_t)(L->nd + 16) * nr * sizeof(float));
      if (e == cudaSuccess) e = cudaMalloc(&p->d_tm, (size_t)(L->t_len + 16) * nr * p->t_elem);
      if (e == cudaSuccess) e = cudaMalloc(&p->d_pm, (size_t)(L->p_len + 16) * nr * p->p_elem);
      // t padding slots must read as zero (the tensor-core pass scales by max |t|)
      if (e == cudaSuccess) e = cudaMemset(p->d_tm, 0, (size_t)(L->t_len + 16) * nr * p->t_elem);
      if (e == cudaSuccess && p->tc) {
        e = cudaMalloc(&p->d_xplanes, (size_t)4 * (L->nd + 16) * 16);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_tplanes, (size_t)4 * (L->t_len + 16) * 16);
        if (e == cudaSuccess) e = cudaMalloc(&p->d_scal, 64 * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&p->d_amax, 32 * sizeof(unsigned));
      }
      if (e != cudaSuccess) rc = cuda_fail(e, "multi-RHS buffers");
    }
    if (!rc) {
      cudaError_t e = cudaMalloc(&p->d_err, sizeof(int));
      if (e == cudaSuccess) e = cudaMemset(p->d_err, 0, sizeof(int));
      if (e != cudaSuccess) rc = cuda_fail(e, "status word");
    }
    if (!rc) rc = p->precision == HMVM_FP32 ? prepare_kernels<float>(p) : prepare_kernels<double>(p);
    if (!rc) {
      cudaError_t e = cudaDeviceSynchronize();
      if (e != cudaSuccess) rc = cuda_fail(e, "plan upload");
    }
    if (rc) free_plan_buffers(p);
  }
  delete L;
  if (rc) {
    delete p;
    return rc;
  }
  *out = p;
  return HMVM_OK;
}

// HMVM_DEVICE_CHECKS builds: the stage's descriptors checked on the device
// (hmvm_validate_kernel) before it runs; other builds launch nothing.
int launch_validate(bool& first, hmvm_plan* p, int stage, cudaStream_t st) {
  if (!kDeviceChecks) return HMVM_OK;
  ValidateArgs v;
  v.tiles = p->d_tiles;
  v.segs = p->d_segs;
  v.out_idx = p->d_out_idx;
  v.team_begin = stage == 1 ? p->d_tb1 : p->d_tb2;
  v.red = stage == 1 ? p->d_red1 : p->d_red2;
  v.nteams = stage == 1 ? p->stage1_teams : p->stage2_teams;
  v.first = stage == 1 ? 0 : p->stage1_tiles;
  v.end = stage == 1 ? p->stage1_tiles : p->stage1_tiles + p->stage2_tiles;
  v.n_red = stage == 1 ? p->n_red1 : p->n_red2;
  v.caps = p->caps;
  v.vec = p->vec;
  v.elem = p->elem;
  v.stage1 = stage == 1 ? 1 : 0;
  v.zcap = stage == 1 ? p->zcap1 : p->zcap2;
  v.err = p->d_err;
  const int64_t n = std::max<int64_t>(v.end - v.first, v.n_red);
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)p->num_sms * 4));
  HMVM_CUDA_TRY(launch_in_apply(first, hmvm_validate_kernel, grid, 256, 0, st, v), "validation launch");
  return HMVM_OK;
}

// Mixed plans: x rounded to FP32, V stage (scaled t in FP32), its reduction,
// row stage, its reduction into y (partials in FP64).
int launch_stages_mixed(hmvm_plan* p, const void* x, void* y, void* tbuf, void* pbuf, float* x32, cudaStream_t st) {
  TileArgs a;
  a.err = p->d_err;
  a.tiles = p->d_tiles;
  a.segs = p->d_segs;
  a.data = p->d_data;
  a.x = x;
  a.t = tbuf;
  a.y = y;
  a.p = pbuf;
  a.out_idx = p->d_out_idx;
  a.x32 = x32;
  const int ctas = p->num_sms * p->ctas_per_sm, ctas2 = p->num_sms * p->ctas2_per_sm;
  cudaEvent_t* ev = nullptr;
  if (p->profiling && p->prof_count < kMaxProfiled) {
    ev = &p->prof_events[kEventsPerApply * (size_t)p->prof_count];
    p->prof_count++;
  }
  if (ev) cudaEventRecord(ev[0], st);
  bool first = true;
  HMVM_CUDA_TRY(launch_in_apply(first, hmvm_round_f32_kernel, (unsigned)std::min((p->nd + 255) / 256, p->num_sms * 8),
                                256, 0, st, static_cast<const double*>(x), x32, p->nd),
                "x rounding launch");
  if (p->stage1_tiles > 0) {
    int vrc = launch_validate(first, p, 1, st);
    if (vrc) return vrc;
    const Launch l = stage_launch<double>(p->mixed_kcode, p->stage1_cfg, 1);
    a.team_begin = p->d_tb1;
    a.nteams = p->stage1_teams;
    a.scale = p->d_scale;
    HMVM_CUDA_TRY(launch_in_apply(first, l.fn, ctas, l.threads, l.smem, st, a), "V-stage launch");
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (p->n_red1 > 0) {
    HMVM_CUDA_TRY(launch_in_apply(first, hmvm_reduce_kernel<double, float>, (unsigned)((p->n_red1 + 255) / 256), 256,
                                  0, st, (const int4*)p->d_red1, p->n_red1, static_cast<const double*>(pbuf),
                                  static_cast<float*>(tbuf), (const int*)p->d_err),
                  "V-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[2], st);
  {
    int vrc = launch_validate(first, p, 2, st);
    if (vrc) return vrc;
    const Launch l = stage_launch<double>(p->mixed_kcode, p->stage2_cfg, 2);
    a.team_begin = p->d_tb2;
    a.nteams = p->stage2_teams;
    a.scale = nullptr;
    HMVM_CUDA_TRY(launch_in_apply(first, l.fn, ctas2, l.threads, l.smem, st, a), "row-stage launch");
  }
  if (ev) cudaEventRecord(ev[3], st);
  if (p->n_red2 > 0) {
    HMVM_CUDA_TRY(launch_in_apply(first, hmvm_reduce_kernel<double, double>, (unsigned)((p->n_red2 + 255) / 256), 256,
                                  0, st, (const int4*)p->d_red2, p->n_red2, static_cast<const double*>(pbuf),
                                  static_cast<double*>(y), (const int*)p->d_err),
                  "row-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[4], st);
  return HMVM_OK;
}

// The launches of one HMVM: V stage, its reduction into t, row stage, its
// reduction into y.  t and the partial sums live in tbuf / pbuf.
template <typename T>
int launch_stages(hmvm_plan* p, const void* x, void* y, void* tbuf, void* pbuf, cudaStream_t st) {
  TileArgs a;
  a.err = p->d_err;
  a.tiles = p->d_tiles;
  a.segs = p->d_segs;
  a.data = p->d_data;
  a.x = x;
  a.t = tbuf;
  a.y = y;
  a.p = pbuf;
  a.out_idx = p->d_out_idx;
  a.x32 = nullptr;
  a.scale = nullptr;
  const int ctas = p->num_sms * p->ctas_per_sm, ctas2 = p->num_sms * p->ctas2_per_sm;
  cudaEvent_t* ev = nullptr;
  if (p->profiling && p->prof_count < kMaxProfiled) {
    ev = &p->prof_events[kEventsPerApply * (size_t)p->prof_count];
    p->prof_count++;
  }
  bool first = true;
  if (ev) cudaEventRecord(ev[0], st);
  if (p->stage1_tiles > 0) {
    int vrc = launch_validate(first, p, 1, st);
    if (vrc) return vrc;
    const Launch l = stage_launch<T>(p->kernel, p->stage1_cfg, 1);
    a.team_begin = p->d_tb1;
    a.nteams = p->stage1_teams;
    HMVM_CUDA_TRY(launch_in_apply(first, l.fn, ctas, l.threads, l.smem, st, a), "V-stage launch");
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (p->n_red1 > 0) {
    HMVM_CUDA_TRY(launch_in_apply(first, hmvm_reduce_kernel<T, T>, (unsigned)((p->n_red1 + 255) / 256), 256, 0, st,
                                  (const int4*)p->d_red1, p->n_red1, static_cast<const T*>(pbuf),
                                  static_cast<T*>(tbuf), (const int*)p->d_err),
                  "V-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[2], st);
  {
    int vrc = launch_validate(first, p, 2, st);
    if (vrc) return vrc;
    const Launch l = stage_launch<T>(p->kernel, p->stage2_cfg, 2);
    a.team_begin = p->d_tb2;
    a.nteams = p->stage2_teams;
    HMVM_CUDA_TRY(launch_in_apply(first, l.fn, ctas2, l.threads, l.smem, st, a), "row-stage launch");
  }
  if (ev) cudaEventRecord(ev[3], st);
  if (p->n_red2 > 0) {
    HMVM_CUDA_TRY(launch_in_apply(first, hmvm_reduce_kernel<T, T>, (unsigned)((p->n_red2 + 255) / 256), 256, 0, st,
                                  (const int4*)p->d_red2, p->n_red2, static_cast<const T*>(pbuf), static_cast<T*>(y),
                                  (const int*)p->d_err),
                  "row-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[4], st);
  return HMVM_OK;
}

int apply_impl(hmvm_plan* p, const void* x, void* y, cudaStream_t st);
inline int apply_impl_fwd(hmvm_plan* p, const void* x, void* y, cudaStream_t st) { return apply_impl(p, x, y, st); }

// ---- multi-RHS ---------------------------------------------------------------
// The multi-RHS kernel's launch shape is read from kMultiCfgs (layout.hpp),
// like the single-vector kernels' (see tile_kernel_pick).
template <int NR, int MODE, bool VST>
MultiFn multi_kernel_cfg(int cfg) {
  static_assert(kNumMultiCfgs == 1 && kDefaultMultiCfg == 0, "one multi-RHS shape is instantiated");
  (void)cfg;
  constexpr MultiCfg c = kMultiCfgs[kDefaultMultiCfg];
  return hmvm_multi_kernel<c.wpb, c.slots, c.chunk, NR, MODE, VST>;
}
template <int MODE, bool VST>
MultiFn multi_kernel_nr(int nr, int cfg) {
  switch (nr) {
    case 2: return multi_kernel_cfg<2, MODE, VST>(cfg);
    case 4: return multi_kernel_cfg<4, MODE, VST>(cfg);
    default: return multi_kernel_cfg<8, MODE, VST>(cfg);
  }
}
template <bool VST>
MultiFn multi_kernel_for(int mode, int nr, int cfg) {
  switch (mode) {
    case kModePlain64: return multi_kernel_nr<kModePlain64, VST>(nr, cfg);
    case kModePlain32: return multi_kernel_nr<kModePlain32, VST>(nr, cfg);
    case kModeMixed16: return multi_kernel_nr<kModeMixed16, VST>(nr, cfg);
    default: return multi_kernel_nr<kModeMixedBF16, VST>(nr, cfg);
  }
}
int plan_mode(const hmvm_plan* p) {
  if (p->mixed) return p->mixed_kcode == 3 ? kModeMixedBF16 : kModeMixed16;
  return p->precision == HMVM_FP64 ? kModePlain64 : kModePlain32;
}

template <typename TP, typename TD, bool VST>
void launch_reduce_multi(int nr_inst, const int4* red, int n, const void* pbuf, void* dst, int64_t ldy, int nr,
                         cudaStream_t st) {
  const int64_t work = (int64_t)n * nr_inst;
  const int blocks = (int)std::min<int64_t>((work + 255) / 256, 65535);
  const TP* pp = static_cast<const TP*>(pbuf);
  TD* dd = static_cast<TD*>(dst);
  switch (nr_inst) {
    case 16: hmvm_reduce_multi_kernel<TP, TD, 16, VST><<<blocks, 256, 0, st>>>(red, n, pp, dd, ldy, nr); break;
    case 2: hmvm_reduce_multi_kernel<TP, TD, 2, VST><<<blocks, 256, 0, st>>>(red, n, pp, dd, ldy, nr); break;
    case 4: hmvm_reduce_multi_kernel<TP, TD, 4, VST><<<blocks, 256, 0, st>>>(red, n, pp, dd, ldy, nr); break;
    default: hmvm_reduce_multi_kernel<TP, TD, 8, VST><<<blocks, 256, 0, st>>>(red, n, pp, dd, ldy, nr); break;
  }
}

template <int NR>
void launch_pack(const hmvm_plan* p, const void* X, int64_t ldx, int nr, cudaStream_t st) {
  const int64_t work = (int64_t)(p->nd + 16) * NR;
  const int blocks = (int)std::min<int64_t>((work + 255) / 256, (int64_t)p->num_sms * 8);
  double* x64 = p->precision != HMVM_FP32 ? p->d_xm64 : nullptr;
  float* x32 = p->precision != HMVM_FP64 ? p->d_xm32 : nullptr;
  if (p->precision == HMVM_FP32)
    hmvm_pack_x_kernel<float, NR><<<blocks, 256, 0, st>>>(static_cast<const float*>(X), ldx, p->nd, 16, nr, x64, x32);
  else
    hmvm_pack_x_kernel<double, NR><<<blocks, 256, 0, st>>>(static_cast<const double*>(X), ldx, p->nd, 16, nr, x64,
                                                           x32);
}

// One pass: nr (<= nr_inst) right-hand sides X[:, 0:nr] -> Y[:, 0:nr].
int launch_multi_stages(hmvm_plan* p, void* Y, int64_t ldy, int nr, int nr_inst, cudaStream_t st);

int launch_multi_pass(hmvm_plan* p, const void* X, int64_t ldx, void* Y, int64_t ldy, int nr, int nr_inst,
                      cudaStream_t st) {
  switch (nr_inst) {
    case 2: launch_pack<2>(p, X, ldx, nr, st); break;
    case 4: launch_pack<4>(p, X, ldx, nr, st); break;
    default: launch_pack<8>(p, X, ldx, nr, st); break;
  }
  HMVM_CUDA_TRY(cudaGetLastError(), "input packing launch");
  return launch_multi_stages(p, Y, ldy, nr, nr_inst, st);
}

// The stages of one pass, the packed inputs already in place.
int launch_multi_stages(hmvm_plan* p, void* Y, int64_t ldy, int nr, int nr_inst, cudaStream_t st) {
  MultiArgs a;
  a.err = p->d_err;
  a.tiles = p->d_tiles;
  a.segs = p->d_segs;
  a.data = p->d_data;
  a.x64 = p->d_xm64;
  a.x32 = p->d_xm32;
  a.t = p->d_tm;
  a.y = Y;
  a.ldy = ldy;
  a.nr = nr;
  a.p = p->d_pm;
  a.out_idx = p->d_out_idx;
  a.scale = p->d_scale;
  const int mode = plan_mode(p);
  const MultiCfg& c = kMultiCfgs[kDefaultMultiCfg];
  const int threads = 32 * c.wpb, smem = multi_smem_bytes(c, mode == kModePlain64);
  cudaEvent_t* ev = nullptr;
  if (p->profiling && p->prof_count < kMaxProfiled) {
    ev = &p->prof_events[kEventsPerApply * (size_t)p->prof_count];
    p->prof_count++;
  }
  if (ev) cudaEventRecord(ev[0], st);
  if (p->stage1_tiles > 0) {
    a.team_begin = p->d_tb1;
    a.nteams = p->stage1_teams;
    const int ctas = (p->stage1_teams + c.wpb - 1) / c.wpb;
    multi_kernel_for<true>(mode, nr_inst, kDefaultMultiCfg)<<<ctas, threads, smem, st>>>(a);
    HMVM_CUDA_TRY(cudaGetLastError(), "multi-RHS V-stage launch");
  }
  if (ev) cudaEventRecord(ev[1], st);
  const bool f32 = p->precision == HMVM_FP32;
  if (p->n_red1 > 0) {
    if (mode == kModePlain64) launch_reduce_multi<double, double, true>(nr_inst, p->d_red1, p->n_red1, p->d_pm, p->d_tm, 0, nr, st);
    else if (f32) launch_reduce_multi<float, float, true>(nr_inst, p->d_red1, p->n_red1, p->d_pm, p->d_tm, 0, nr, st);
    else launch_reduce_multi<double, float, true>(nr_inst, p->d_red1, p->n_red1, p->d_pm, p->d_tm, 0, nr, st);
    HMVM_CUDA_TRY(cudaGetLastError(), "multi-RHS V-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[2], st);
  {
    a.team_begin = p->d_tb2;
    a.nteams = p->stage2_teams;
    const int ctas = (p->stage2_teams + c.wpb - 1) / c.wpb;
    multi_kernel_for<false>(mode, nr_inst, kDefaultMultiCfg)<<<ctas, threads, smem, st>>>(a);
    HMVM_CUDA_TRY(cudaGetLastError(), "multi-RHS row-stage launch");
  }
  if (ev) cudaEventRecord(ev[3], st);
  if (p->n_red2 > 0) {
    if (f32) launch_reduce_multi<float, float, false>(nr_inst, p->d_red2, p->n_red2, p->d_pm, Y, ldy, nr, st);
    else launch_reduce_multi<double, double, false>(nr_inst, p->d_red2, p->n_red2, p->d_pm, Y, ldy, nr, st);
    HMVM_CUDA_TRY(cudaGetLastError(), "multi-RHS row-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[4], st);
  return HMVM_OK;
}

// ---- tensor-core passes ------------------------------------------------------------
constexpr int kTcWpb = kTcWarpsPerSm;  // one CTA of 6 warps per SM
using TcFn = void (*)(TcArgs);
template <bool VST>
TcFn tc_kernel_for(bool bf16) {
  return bf16 ? hmvm_tc_kernel<kTcWpb, 2, 4096, kModeMixedBF16, VST> : hmvm_tc_kernel<kTcWpb, 2, 4096, kModeMixed16, VST>;
}
constexpr int tc_smem() { return tc_smem_bytes<kTcWpb, 2, 4096>(); }

int tc_prepare(const hmvm_plan* p) {
  const bool bf = p->mixed_kcode == 3;
  for (TcFn f : {tc_kernel_for<true>(bf), tc_kernel_for<false>(bf)})
    HMVM_CUDA_TRY(cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem()),
                  "cudaFuncSetAttribute");
  return HMVM_OK;
}

// One 16-column pass: pack X, scale and split it into 16-bit planes, V stage,
// its reduction, t into planes, row stage, its reduction into Y.
int launch_tc_pass(hmvm_plan* p, const void* X, int64_t ldx, void* Y, int64_t ldy, int nr, cudaStream_t st) {
  const bool bf = p->mixed_kcode == 3;
  const int gsm = p->num_sms * 8;  // grid stride (x 256 threads) is a multiple of 16, as the plane kernels need
  HMVM_CUDA_TRY(cudaMemsetAsync(p->d_amax, 0, 32 * sizeof(unsigned), st), "scale reset");
  launch_pack<kTcNrhs>(p, X, ldx, nr, st);
  const int64_t nx = (int64_t)(p->nd + 16) * kTcNrhs, nt = (int64_t)(p->t_len + 16) * kTcNrhs;
  hmvm_absmax_kernel<<<gsm, 256, 0, st>>>(p->d_xm32, nx, p->d_amax);
  if (bf) hmvm_tc_planes_kernel<true><<<gsm, 256, 0, st>>>(p->d_xm32, p->nd, 16, p->d_amax, p->d_xplanes, p->d_scal);
  else hmvm_tc_planes_kernel<false><<<gsm, 256, 0, st>>>(p->d_xm32, p->nd, 16, p->d_amax, p->d_xplanes, p->d_scal);
  HMVM_CUDA_TRY(cudaGetLastError(), "input planes launch");
  TcArgs ta;
  MultiArgs& a = ta.m;
  a.err = p->d_err;
  a.tiles = p->d_tiles;
  a.segs = p->d_segs;
  a.data = p->d_data;
  a.x64 = p->d_xm64;
  a.x32 = p->d_xm32;
  a.t = p->d_tm;
  a.y = Y;
  a.ldy = ldy;
  a.nr = nr;
  a.p = p->d_pm;
  a.out_idx = p->d_out_idx;
  a.scale = p->d_scale;
  ta.xplanes = p->d_xplanes;
  ta.tplanes = p->d_tplanes;
  ta.xrows = p->nd + 16;
  ta.trows = p->t_len + 16;
  ta.scal = p->d_scal;
  cudaEvent_t* ev = nullptr;
  if (p->profiling && p->prof_count < kMaxProfiled) {
    ev = &p->prof_events[kEventsPerApply * (size_t)p->prof_count];
    p->prof_count++;
  }
  if (ev) cudaEventRecord(ev[0], st);
  if (p->stage1_tiles > 0) {
    a.team_begin = p->d_tb1;
    a.nteams = p->stage1_teams;
    tc_kernel_for<true>(bf)<<<(p->stage1_teams + kTcWpb - 1) / kTcWpb, 32 * kTcWpb, tc_smem(), st>>>(ta);
    HMVM_CUDA_TRY(cudaGetLastError(), "tensor-core V-stage launch");
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (p->n_red1 > 0)
    launch_reduce_multi<double, float, true>(kTcNrhs, p->d_red1, p->n_red1, p->d_pm, p->d_tm, 0, nr, st);
  hmvm_absmax_kernel<<<gsm, 256, 0, st>>>(static_cast<const float*>(p->d_tm), nt, p->d_amax + 16);
  if (bf)
    hmvm_tc_planes_kernel<true><<<gsm, 256, 0, st>>>(static_cast<const float*>(p->d_tm), (int)p->t_len, 16,
                                                    p->d_amax + 16, p->d_tplanes, p->d_scal + 32);
  else
    hmvm_tc_planes_kernel<false><<<gsm, 256, 0, st>>>(static_cast<const float*>(p->d_tm), (int)p->t_len, 16,
                                                     p->d_amax + 16, p->d_tplanes, p->d_scal + 32);
  HMVM_CUDA_TRY(cudaGetLastError(), "t planes launch");
  if (ev) cudaEventRecord(ev[2], st);
  a.team_begin = p->d_tb2;
  a.nteams = p->stage2_teams;
  tc_kernel_for<false>(bf)<<<(p->stage2_teams + kTcWpb - 1) / kTcWpb, 32 * kTcWpb, tc_smem(), st>>>(ta);
  HMVM_CUDA_TRY(cudaGetLastError(), "tensor-core row-stage launch");
  if (ev) cudaEventRecord(ev[3], st);
  if (p->n_red2 > 0)
    launch_reduce_multi<double, double, false>(kTcNrhs, p->d_red2, p->n_red2, p->d_pm, Y, ldy, nr, st);
  HMVM_CUDA_TRY(cudaGetLastError(), "tensor-core reductions");
  if (ev) cudaEventRecord(ev[4], st);
  return HMVM_OK;
}

// ---- wide tensor-core passes ---------------------------------------------------------
template <bool VST, bool BF>
void tcw_fn_attr(int* rc) {
  if (*rc) return;
  const cudaError_t e = cudaFuncSetAttribute((const void*)hmvm_tcw_kernel<VST, BF>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kTcwSmem);
  if (e != cudaSuccess) *rc = cuda_fail(e, "cudaFuncSetAttribute");
}
int tcw_prepare(const hmvm_plan* p) {
  int rc = HMVM_OK;
  if (p->tcw_bf) {
    tcw_fn_attr<true, true>(&rc);
    tcw_fn_attr<false, true>(&rc);
  } else {
    tcw_fn_attr<true, false>(&rc);
    tcw_fn_attr<false, false>(&rc);
  }
  return rc;
}

// One pass of up to 128 right-hand sides: (FP16) per-column maxima, the x
// planes, V stage into the t planes, the split panels' reduction, row stage
// into Y.
int launch_tcw_pass(hmvm_plan* p, const void* X, int64_t ldx, void* Y, int64_t ldy, int nr, cudaStream_t st) {
  const bool f32 = p->precision == HMVM_FP32;
  const int gx = (int)std::min<int64_t>(((int64_t)p->nd + 31) / 32, (int64_t)p->num_sms * 16);
  if (!p->tcw_bf) {
    HMVM_CUDA_TRY(cudaMemsetAsync(p->d_amax128, 0, kTcwRhs * sizeof(unsigned), st), "scale reset");
    // per column at most 32 blocks of at least 16 elements per thread
    const int per_col = std::max(1, std::min(32, p->nd / (kTcwAbsmaxThreads * 16)));
    const dim3 g((unsigned)per_col, (unsigned)nr);
    if (f32)
      hmvm_tcw_absmax_kernel<float><<<g, kTcwAbsmaxThreads, 0, st>>>(static_cast<const float*>(X), ldx, p->nd,
                                                                     p->d_amax128);
    else
      hmvm_tcw_absmax_kernel<double><<<g, kTcwAbsmaxThreads, 0, st>>>(static_cast<const double*>(X), ldx, p->nd,
                                                                      p->d_amax128);
  }
  if (f32) {
    if (p->tcw_bf) hmvm_tcw_xplanes_kernel<float, true><<<gx, 256, 0, st>>>(static_cast<const float*>(X), ldx, p->nd, nr, p->d_amax128, p->d_xscale, p->d_xpl);
    else hmvm_tcw_xplanes_kernel<float, false><<<gx, 256, 0, st>>>(static_cast<const float*>(X), ldx, p->nd, nr, p->d_amax128, p->d_xscale, p->d_xpl);
  } else {
    if (p->tcw_bf) hmvm_tcw_xplanes_kernel<double, true><<<gx, 256, 0, st>>>(static_cast<const double*>(X), ldx, p->nd, nr, p->d_amax128, p->d_xscale, p->d_xpl);
    else hmvm_tcw_xplanes_kernel<double, false><<<gx, 256, 0, st>>>(static_cast<const double*>(X), ldx, p->nd, nr, p->d_amax128, p->d_xscale, p->d_xpl);
  }
  HMVM_CUDA_TRY(cudaGetLastError(), "input planes launch");
  TcwArgs a;
  a.tiles = p->d_tiles;
  a.segs = p->d_segs;
  a.blocks = p->d_tblocks;
  a.groups = reinterpret_cast<const uint4*>(p->d_tgroups);
  a.gops = reinterpret_cast<const uint2*>(p->d_tops);
  a.gfirst = p->d_tgfirst;
  a.n_gops = p->tcw_ngops;
  a.data = static_cast<const char*>(p->d_data);
  a.out_idx = p->d_out_idx;
  a.tscale = p->d_tscale;
  a.xscale = p->d_xscale;
  a.tplanes = p->d_tpl;
  a.trows = p->tpl_rows;
  a.part = p->d_part;
  a.y = Y;
  a.ldy = ldy;
  a.nr = nr;
  a.y32 = f32 ? 1 : 0;
  a.err = p->d_err;
  cudaEvent_t* ev = nullptr;
  if (p->profiling && p->prof_count < kMaxProfiled) {
    ev = &p->prof_events[kEventsPerApply * (size_t)p->prof_count];
    p->prof_count++;
  }
  if (ev) cudaEventRecord(ev[0], st);
  if (p->stage1_tiles > 0) {
    a.team_begin = p->d_tb1;
    a.nteams = p->stage1_teams;
    if (p->tcw_bf) hmvm_tcw_kernel<true, true><<<p->stage1_teams, kTcwThreads, kTcwSmem, st>>>(p->xmap, p->tmap, a);
    else hmvm_tcw_kernel<true, false><<<p->stage1_teams, kTcwThreads, kTcwSmem, st>>>(p->xmap, p->tmap, a);
    HMVM_CUDA_TRY(cudaGetLastError(), "tensor-core V-stage launch");
  }
  if (ev) cudaEventRecord(ev[1], st);
  if (p->n_red1 > 0) {
    const int blocks = (int)std::min<int64_t>(((int64_t)p->n_red1 * kTcwRhs + 255) / 256, (int64_t)p->num_sms * 8);
    if (p->tcw_bf) hmvm_tcw_reduce_kernel<true><<<blocks, 256, 0, st>>>(p->d_red1, p->n_red1, p->d_part, p->d_tpl, p->tpl_rows);
    else hmvm_tcw_reduce_kernel<false><<<blocks, 256, 0, st>>>(p->d_red1, p->n_red1, p->d_part, p->d_tpl, p->tpl_rows);
    HMVM_CUDA_TRY(cudaGetLastError(), "tensor-core V-stage reduction launch");
  }
  if (ev) cudaEventRecord(ev[2], st);
  a.team_begin = p->d_tb2;
  a.nteams = p->stage2_teams;
  if (p->tcw_bf) hmvm_tcw_kernel<false, true><<<p->stage2_teams, kTcwThreads, kTcwSmem, st>>>(p->xmap, p->tmap, a);
  else hmvm_tcw_kernel<false, false><<<p->stage2_teams, kTcwThreads, kTcwSmem, st>>>(p->xmap, p->tmap, a);
  HMVM_CUDA_TRY(cudaGetLastError(), "tensor-core row-stage launch");
  if (ev) cudaEventRecord(ev[3], st);
  if (ev) cudaEventRecord(ev[4], st);
  return HMVM_OK;
}
int tcw_kernels_per_pass(const hmvm_plan* p) {
  return (p->tcw_bf ? 1 : 2) + (p->stage1_tiles > 0) + (p->n_red1 > 0) + 1;
}

// Right-hand sides per pass: the largest of 8, 4, 2 that is <= nrhs_max and
// not above what is left (a last single column runs in a 2-wide pass).
int multi_pass_width(int nrhs_max, int left) {
  for (int w : {8, 4, 2})
    if (w <= nrhs_max && w <= std::max(left, 2)) return w;
  return 2;
}

// The passes of a multi-RHS apply: {first column, columns, pass width}.
struct Pass {
  int r0, nr, w;
};
std::vector<Pass> multi_passes(const hmvm_plan* p, int nrhs) {
  std::vector<Pass> v;
  for (int r0 = 0; r0 < nrhs;) {
    const int w = p->tcw ? kTcwRhs : p->nrhs_max <= 1 ? 1 : p->tc ? kTcNrhs : multi_pass_width(p->nrhs_max, nrhs - r0);
    const int nr = std::min(w, nrhs - r0);
    v.push_back(Pass{r0, nr, w});
    r0 += nr;
  }
  return v;
}
// One pass; X and Y point at the pass's first column.
int run_pass(hmvm_plan* p, const Pass& q, const void* X, int64_t ldx, void* Y, int64_t ldy, cudaStream_t st) {
  if (p->tcw) return launch_tcw_pass(p, X, ldx, Y, ldy, q.nr, st);
  if (p->nrhs_max <= 1) return apply_impl_fwd(p, X, Y, st);  // single-vector passes
  if (p->tc) return launch_tc_pass(p, X, ldx, Y, ldy, q.nr, st);
  return launch_multi_pass(p, X, ldx, Y, ldy, q.nr, q.w, st);
}

int apply_multi_impl(hmvm_plan* p, const void* X, int64_t ldx, void* Y, int64_t ldy, int nrhs, cudaStream_t st) {
  if (p->nd == 0 || nrhs == 0) return HMVM_OK;
  const size_t ex = (size_t)p->elem;
  for (const Pass& q : multi_passes(p, nrhs)) {
    int rc = run_pass(p, q, static_cast<const char*>(X) + (size_t)q.r0 * ldx * ex, ldx,
                      static_cast<char*>(Y) + (size_t)q.r0 * ldy * ex, ldy, st);
    if (rc) return rc;
  }
  return HMVM_OK;
}

int check_multi(const hmvm_plan* p, const void* X, int64_t ldx, const void* Y, int64_t ldy, int32_t nrhs) {
  if (!p) return set_error(HMVM_EINVAL, "plan is NULL");
  if (nrhs < 0) return set_error(HMVM_EINVAL, "nrhs < 0");
  if (p->nd == 0 || nrhs == 0) return HMVM_OK;
  if (!X || !Y) return set_error(HMVM_EINVAL, "X or Y is NULL");
  if (ldx < p->nd || ldy < p->nd) return set_error(HMVM_EINVAL, "ldx and ldy must be >= N");
  const char* xb = static_cast<const char*>(X);
  const char* yb = static_cast<const char*>(Y);
  const size_t xe = ((size_t)(nrhs - 1) * ldx + p->nd) * p->elem, ye = ((size_t)(nrhs - 1) * ldy + p->nd) * p->elem;
  if (xb < yb + ye && yb < xb + xe) return set_error(HMVM_EINVAL, "X and Y overlap");
  return HMVM_OK;
}

int apply_impl(hmvm_plan* p, const void* x, void* y, cudaStream_t st) {
  if (p->nd == 0) return HMVM_OK;
  if (p->tcw) return launch_tcw_pass(p, x, p->nd, y, p->nd, 1, st);  // one right-hand side in a pass
  if (p->mixed) return launch_stages_mixed(p, x, y, p->d_t, p->d_p, p->d_x32, st);
  if (p->precision == HMVM_FP64) return launch_stages<double>(p, x, y, p->d_t, p->d_p, st);
  return launch_stages<float>(p, x, y, p->d_t, p->d_p, st);
}

int check_xy(const hmvm_plan* p, const void* x, const void* y) {
  if (!p) return set_error(HMVM_EINVAL, "plan is NULL");
  if (p->nd > 0 && (!x || !y)) return set_error(HMVM_EINVAL, "x or y is NULL");
  const char* xb = static_cast<const char*>(x);
  const char* yb = static_cast<const char*>(y);
  const size_t nb = (size_t)p->nd * p->elem;
  if (p->nd > 0 && xb < yb + nb && yb < xb + nb) return set_error(HMVM_EINVAL, "x and y overlap");
  return HMVM_OK;
}

void make_table_from_matrix2(int nd, int nlf, int ktmax, int len, const int* ltmtx, const int* kt, const int* ndl,
                             const int* ndt, const int* nstrtl, const int* nstrtt, const int* a1, const int* a2,
                             const void* rowmat, bool is_float, LeafTable& lt) {
  lt.nd = nd;
  lt.nlf = nlf;
  lt.ktmax = ktmax;
  lt.len = len;
  lt.ltmtx = ltmtx;
  lt.kt = kt;
  lt.ndl = ndl;
  lt.ndt = ndt;
  lt.nstrtl = nstrtl;
  lt.nstrtt = nstrtt;
  lt.a1_32 = a1;
  lt.a2_32 = a2;
  lt.rowmat = rowmat;
  lt.rowmat_is_float = is_float;
}

void table_from_leaves64(const hmvm_leaves64* lv, bool is_float, LeafTable& lt) {
  lt.nd = lv->nd;
  lt.nlf = lv->nlf;
  lt.ktmax = lv->ktmax;
  lt.len = lv->len;
  lt.ltmtx = lv->ltmtx;
  lt.kt = lv->kt;
  lt.ndl = lv->ndl;
  lt.ndt = lv->ndt;
  lt.nstrtl = lv->nstrtl;
  lt.nstrtt = lv->nstrtt;
  lt.a1_64 = lv->a1;
  lt.a2_64 = lv->a2;
  lt.rowmat = lv->rowmat;
  lt.rowmat_is_float = is_float;
}

}  // namespace

extern "C" {

void hmvm_b200_default_opts(hmvm_plan_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = HMVM_FP64;
  o->device = -1;
  o->max_tile_rows = 32;
  o->split_cols = 0;
  o->stage1_cfg = -1;
  o->stage2_cfg = -1;
  o->ctas_per_sm = 0;
  o->kernel = -1;
  o->mixed_fp8_eps = 1e-4;
  o->mixed_fp32_tau = -1.0;
  o->mixed_lr_format = HMVM_LR_FP16;
  o->nrhs_max = 1;
}

int hmvm_b200_plan_create_d(const hmvm_matrix2_d* m, const hmvm_plan_opts* opts, hmvm_plan** plan) {
  if (!m) return set_error(HMVM_EINVAL, "matrix is NULL");
  LeafTable lt;
  make_table_from_matrix2(m->nd, m->nlf, m->ktmax, m->len, m->ltmtx, m->kt, m->ndl, m->ndt, m->nstrtl, m->nstrtt,
                          m->a1, m->a2, m->rowmat, false, lt);
  return create_plan(lt, opts, plan);
}

int hmvm_b200_plan_create_f(const hmvm_matrix2_f* m, const hmvm_plan_opts* opts, hmvm_plan** plan) {
  if (!m) return set_error(HMVM_EINVAL, "matrix is NULL");
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  if (opts) o = *opts;
  o.precision = HMVM_FP32;
  LeafTable lt;
  make_table_from_matrix2(m->nd, m->nlf, m->ktmax, m->len, m->ltmtx, m->kt, m->ndl, m->ndt, m->nstrtl, m->nstrtt,
                          m->a1, m->a2, m->rowmat, true, lt);
  return create_plan(lt, &o, plan);
}

int hmvm_b200_plan_create64_d(const hmvm_leaves64* lv, const hmvm_plan_opts* opts, hmvm_plan** plan) {
  if (!lv) return set_error(HMVM_EINVAL, "leaf table is NULL");
  LeafTable lt;
  table_from_leaves64(lv, false, lt);
  return create_plan(lt, opts, plan);
}

int hmvm_b200_plan_create64_f(const hmvm_leaves64* lv, const hmvm_plan_opts* opts, hmvm_plan** plan) {
  if (!lv) return set_error(HMVM_EINVAL, "leaf table is NULL");
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  if (opts) o = *opts;
  o.precision = HMVM_FP32;
  LeafTable lt;
  table_from_leaves64(lv, true, lt);
  return create_plan(lt, &o, plan);
}

void hmvm_b200_plan_destroy(hmvm_plan* p) {
  if (!p) return;
  {
    DeviceGuard g(p->device);
    free_plan_buffers(p);
  }
  delete p;
}

int hmvm_b200_plan_get_info(const hmvm_plan* p, hmvm_plan_info* info) {
  if (!p || !info) return set_error(HMVM_EINVAL, "NULL argument");
  std::memset(info, 0, sizeof(*info));
  info->nd = p->nd;
  info->nlf = p->nlf;
  info->n_lowrank = p->n_lowrank;
  info->n_dense = p->n_dense;
  info->precision = p->precision;
  info->device = p->device;
  info->num_sms = p->num_sms;
  info->algorithmic_bytes = p->stored_bytes + 2 * (int64_t)p->nd * p->elem;
  info->device_bytes = p->device_bytes;
  info->t_len = p->t_len;
  info->stage1_tiles = p->stage1_tiles;
  info->stage2_tiles = p->stage2_tiles;
  info->stage1_teams = p->stage1_teams;
  info->stage2_teams = p->stage2_teams;
  info->split_rows = p->n_red1 + p->n_red2;
  info->kernels_per_apply = hmvm_b200_plan_kernel_count(p);
  info->stage1_cfg = p->stage1_cfg;
  info->stage2_cfg = p->stage2_cfg;
  info->flops = 2 * p->stored_elems;
  info->stage1_bytes = p->stage1_bytes;
  info->stage2_bytes = p->stage2_bytes;
  info->kernel = p->tcw ? 4 : p->mixed ? 2 : p->kernel;
  info->ctas_per_sm = p->ctas_per_sm;
  info->stage2_ctas_per_sm = p->ctas2_per_sm;
  info->cols_fp32 = p->cols_fp32;
  info->cols_lr16 = p->cols_lr16;
  info->cols_fp8 = p->cols_fp8;
  info->nrhs_max = p->tcw ? kTcwRhs : p->nrhs_max;
  return HMVM_OK;
}

int hmvm_b200_plan_profile(hmvm_plan* p, int enable) {
  if (!p) return set_error(HMVM_EINVAL, "plan is NULL");
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  if (enable && p->prof_events.empty()) {
    p->prof_events.resize(kEventsPerApply * (size_t)kMaxProfiled);
    for (auto& e : p->prof_events) HMVM_CUDA_TRY(cudaEventCreate(&e), "cudaEventCreate");
  }
  p->profiling = enable != 0;
  p->prof_count = 0;
  return HMVM_OK;
}

int hmvm_b200_plan_profile_read(hmvm_plan* p, double* ms4, int32_t* napplies) {
  if (!p || !ms4) return set_error(HMVM_EINVAL, "NULL argument");
  DeviceGuard g(p->device);
  for (int s = 0; s < 4; s++) ms4[s] = 0.0;
  const int n = p->prof_count;
  if (n > 0)
    HMVM_CUDA_TRY(cudaEventSynchronize(p->prof_events[kEventsPerApply * (size_t)(n - 1) + kEventsPerApply - 1]),
                  "event sync");
  for (int k = 0; k < n; k++) {
    for (int s = 0; s < kEventsPerApply - 1; s++) {
      float ms = 0.f;
      HMVM_CUDA_TRY(cudaEventElapsedTime(&ms, p->prof_events[kEventsPerApply * (size_t)k + s],
                                         p->prof_events[kEventsPerApply * (size_t)k + s + 1]),
                    "cudaEventElapsedTime");
      ms4[s] += ms;
    }
  }
  if (napplies) *napplies = n;
  p->prof_count = 0;
  return HMVM_OK;
}

int hmvm_b200_plan_status(hmvm_plan* p) {
  if (!p) return set_error(HMVM_EINVAL, "plan is NULL");
  DeviceGuard g(p->device);
  int h = 0;
  HMVM_CUDA_TRY(cudaMemcpy(&h, p->d_err, sizeof(int), cudaMemcpyDeviceToHost), "read status word");
  if (h == 0) return HMVM_OK;
  HMVM_CUDA_TRY(cudaMemset(p->d_err, 0, sizeof(int)), "clear status word");
  return set_error(HMVM_EDEVICE, h == 1   ? "a kernel gave up waiting for its bulk copies"
                                 : h == 2 ? "a kernel found a stream region too large"
                                 : h == 3 ? "a kernel found an index outside its buffers"
                                          : "device bounds check: a plan descriptor points outside its buffer");
}

int hmvm_b200_plan_kernel_count(const hmvm_plan* p) {
  if (!p || p->nd == 0) return 0;
  if (p->tcw) return tcw_kernels_per_pass(p);
  return (p->stage1_tiles > 0) + (p->n_red1 > 0) + 1 + (p->n_red2 > 0) + (p->mixed ? 1 : 0) +
         (kDeviceChecks ? (p->stage1_tiles > 0) + 1 : 0);  // checked builds: a validation per stage
}

int hmvm_b200_apply(hmvm_plan* p, const void* x, void* y, void* stream) {
  int rc = check_xy(p, x, y);
  if (rc) return rc;
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  return apply_impl(p, x, y, static_cast<cudaStream_t>(stream));
}

int hmvm_b200_plan_capture(hmvm_plan* p, const void* x, void* y) {
  int rc = check_xy(p, x, y);
  if (rc) return rc;
  if (p->profiling) return set_error(HMVM_EINVAL, "profiling is on; a captured apply cannot record events");
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->graph_exec = nullptr;
  p->graph = nullptr;
  cudaStream_t cs;
  HMVM_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaStreamDestroy(cs);
    return cuda_fail(e, "cudaStreamBeginCapture");
  }
  rc = apply_impl(p, x, y, cs);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(cs, &graph);  // always end the capture
  cudaStreamDestroy(cs);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&p->graph_exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_fail(e, "cudaGraphInstantiate");
  }
  p->graph = graph;
  return HMVM_OK;
}

int hmvm_b200_plan_replay(hmvm_plan* p, void* stream) {
  if (!p) return set_error(HMVM_EINVAL, "plan is NULL");
  if (p->nd == 0) return HMVM_OK;
  if (!p->graph_exec) return set_error(HMVM_EINVAL, "nothing captured: call hmvm_b200_plan_capture first");
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  HMVM_CUDA_TRY(cudaGraphLaunch(p->graph_exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch");
  return HMVM_OK;
}

int hmvm_b200_apply_host(hmvm_plan* p, const void* x_host, void* y_host, void* stream) {
  if (!p) return set_error(HMVM_EINVAL, "plan is NULL");
  if (p->nd > 0 && (!x_host || !y_host)) return set_error(HMVM_EINVAL, "x or y is NULL");
  if (p->nd == 0) return HMVM_OK;
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  size_t nb = (size_t)p->nd * p->elem;
  if (!p->d_x) HMVM_CUDA_TRY(cudaMalloc(&p->d_x, nb), "cudaMalloc x staging");
  if (!p->d_y) HMVM_CUDA_TRY(cudaMalloc(&p->d_y, nb), "cudaMalloc y staging");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HMVM_CUDA_TRY(cudaMemcpyAsync(p->d_x, x_host, nb, cudaMemcpyHostToDevice, st), "copy x to device");
  int rc = apply_impl(p, p->d_x, p->d_y, st);
  if (rc) return rc;
  HMVM_CUDA_TRY(cudaMemcpyAsync(y_host, p->d_y, nb, cudaMemcpyDeviceToHost, st), "copy y to host");
  HMVM_CUDA_TRY(cudaStreamSynchronize(st), "stream synchronize");
  return HMVM_OK;
}

int hmvm_b200_apply_multi(hmvm_plan* p, const void* X, int64_t ldx, void* Y, int64_t ldy, int32_t nrhs,
                          void* stream) {
  int rc = check_multi(p, X, ldx, Y, ldy, nrhs);
  if (rc) return rc;
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  return apply_multi_impl(p, X, ldx, Y, ldy, nrhs, static_cast<cudaStream_t>(stream));
}

int hmvm_b200_apply_multi_host(hmvm_plan* p, const void* X_host, int64_t ldx, void* Y_host, int64_t ldy,
                               int32_t nrhs, void* stream) {
  int rc = check_multi(p, X_host, ldx, Y_host, ldy, nrhs);
  if (rc) return rc;
  if (p->nd == 0 || nrhs == 0) return HMVM_OK;
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  // device copies with leading dimension N, grown on demand
  const size_t col = (size_t)p->nd * p->elem, nb = col * (size_t)nrhs;
  if (nb > p->xh_bytes) {
    if (p->d_xh) cudaFree(p->d_xh);
    if (p->d_yh) cudaFree(p->d_yh);
    p->d_xh = p->d_yh = nullptr;
    p->xh_bytes = 0;
    HMVM_CUDA_TRY(cudaMalloc(&p->d_xh, nb), "cudaMalloc X staging");
    HMVM_CUDA_TRY(cudaMalloc(&p->d_yh, nb), "cudaMalloc Y staging");
    p->xh_bytes = nb;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // Pass by pass: X columns in on cs_in, the pass on st, its Y columns out on
  // cs_out, ordered by events, so a pass's compute overlaps the next pass's
  // upload and the previous pass's download (each pass has its own slice of
  // the staging buffers).
  const std::vector<Pass> passes = multi_passes(p, nrhs);
  if (!p->cs_in) HMVM_CUDA_TRY(cudaStreamCreateWithFlags(&p->cs_in, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!p->cs_out) HMVM_CUDA_TRY(cudaStreamCreateWithFlags(&p->cs_out, cudaStreamNonBlocking), "cudaStreamCreate");
  while (p->pass_events.size() < 2 * passes.size() + 1) {
    cudaEvent_t e;
    HMVM_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    p->pass_events.push_back(e);
  }
  cudaEvent_t* ev = p->pass_events.data();
  cudaError_t e = cudaEventRecord(ev[0], st);  // after the caller's earlier work on st
  if (e == cudaSuccess) e = cudaStreamWaitEvent(p->cs_in, ev[0], 0);
  const size_t ex = (size_t)p->elem;
  for (size_t k = 0; k < passes.size() && e == cudaSuccess && !rc; k++) {
    const Pass& q = passes[k];
    char* dx = static_cast<char*>(p->d_xh) + (size_t)q.r0 * col;
    char* dy = static_cast<char*>(p->d_yh) + (size_t)q.r0 * col;
    const char* hx = static_cast<const char*>(X_host) + (size_t)q.r0 * ldx * ex;
    char* hy = static_cast<char*>(Y_host) + (size_t)q.r0 * ldy * ex;
    e = ldx == p->nd ? cudaMemcpyAsync(dx, hx, col * q.nr, cudaMemcpyHostToDevice, p->cs_in)
                     : cudaMemcpy2DAsync(dx, col, hx, (size_t)ldx * ex, col, (size_t)q.nr, cudaMemcpyHostToDevice,
                                         p->cs_in);
    if (e == cudaSuccess) e = cudaEventRecord(ev[1 + 2 * k], p->cs_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev[1 + 2 * k], 0);
    if (e != cudaSuccess) break;
    rc = run_pass(p, q, dx, p->nd, dy, p->nd, st);
    if (rc) break;
    e = cudaEventRecord(ev[2 + 2 * k], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->cs_out, ev[2 + 2 * k], 0);
    if (e == cudaSuccess)
      e = ldy == p->nd ? cudaMemcpyAsync(hy, dy, col * q.nr, cudaMemcpyDeviceToHost, p->cs_out)
                       : cudaMemcpy2DAsync(hy, (size_t)ldy * ex, dy, col, col, (size_t)q.nr, cudaMemcpyDeviceToHost,
                                           p->cs_out);
  }
  // drain every stream before returning (the staging buffers may be in use)
  const cudaError_t e1 = cudaStreamSynchronize(p->cs_in);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  const cudaError_t e3 = cudaStreamSynchronize(p->cs_out);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "apply_multi_host: copies");
  if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess)
    return cuda_fail(e1 != cudaSuccess ? e1 : e2 != cudaSuccess ? e2 : e3, "stream synchronize");
  return HMVM_OK;
}

int hmvm_b200_plan_multi_kernel_count(const hmvm_plan* p, int32_t nrhs) {
  if (!p || p->nd == 0 || nrhs <= 0) return 0;
  if (p->tcw) return (nrhs + kTcwRhs - 1) / kTcwRhs * tcw_kernels_per_pass(p);
  if (p->nrhs_max <= 1) return nrhs * hmvm_b200_plan_kernel_count(p);
  if (p->tc)  // per pass: pack, 2 x (max, planes), the stages and their reductions
    return (nrhs + kTcNrhs - 1) / kTcNrhs * (5 + (p->stage1_tiles > 0) + (p->n_red1 > 0) + 1 + (p->n_red2 > 0));
  int passes = 0;
  for (int r0 = 0; r0 < nrhs; passes++) r0 += std::min(multi_pass_width(p->nrhs_max, nrhs - r0), nrhs - r0);
  return passes * (1 + (p->stage1_tiles > 0) + (p->n_red1 > 0) + 1 + (p->n_red2 > 0));
}

static int one_shot(hmvm_plan* plan, const void* x, void* y, hmvm_stats* stats, double setup_s) {
  cudaEvent_t e0, e1;
  HMVM_CUDA_TRY(cudaEventCreate(&e0), "cudaEventCreate");
  HMVM_CUDA_TRY(cudaEventCreate(&e1), "cudaEventCreate");
  size_t nb = (size_t)plan->nd * plan->elem;
  int rc = HMVM_OK;
  if (plan->nd > 0) {
    if (!plan->d_x && cudaMalloc(&plan->d_x, nb) != cudaSuccess) rc = set_error(HMVM_ENOMEM, "x staging");
    if (!rc && !plan->d_y && cudaMalloc(&plan->d_y, nb) != cudaSuccess) rc = set_error(HMVM_ENOMEM, "y staging");
    if (!rc && cudaMemcpy(plan->d_x, x, nb, cudaMemcpyHostToDevice) != cudaSuccess) rc = set_error(HMVM_ECUDA, "copy x");
    if (!rc) {
      cudaEventRecord(e0, 0);
      rc = apply_impl(plan, plan->d_x, plan->d_y, 0);
      cudaEventRecord(e1, 0);
    }
    if (!rc) {
      cudaError_t e = cudaMemcpy(y, plan->d_y, nb, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = cuda_fail(e, "copy y");
    }
    if (!rc) rc = hmvm_b200_plan_status(plan);
  }
  float ms = 0.f;
  if (!rc && plan->nd > 0) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc && stats) {
    stats->seconds_setup = setup_s;
    stats->seconds_apply = ms * 1e-3;
    stats->algorithmic_bytes = plan->stored_bytes + 2 * (int64_t)plan->nd * plan->elem;
    stats->gbytes_per_s = ms > 0 ? stats->algorithmic_bytes / (ms * 1e-3) / 1e9 : 0.0;
  }
  return rc;
}

int hmvm_cuda_d(const hmvm_matrix2_d* mat2, const double* x, double* y, int mode, hmvm_stats* stats) {
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  o.precision = HMVM_FP64;
  (void)mode;
  auto t0 = std::chrono::steady_clock::now();
  hmvm_plan* plan = nullptr;
  int rc = hmvm_b200_plan_create_d(mat2, &o, &plan);
  if (rc) return rc;
  double setup = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  {
    DeviceGuard g(plan->device);
    rc = one_shot(plan, x, y, stats, setup);
  }
  hmvm_b200_plan_destroy(plan);
  return rc;
}

int hmvm_cuda_f(const hmvm_matrix2_f* mat2, const float* x, float* y, int mode, hmvm_stats* stats) {
  (void)mode;
  auto t0 = std::chrono::steady_clock::now();
  hmvm_plan* plan = nullptr;
  int rc = hmvm_b200_plan_create_f(mat2, nullptr, &plan);
  if (rc) return rc;
  double setup = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  {
    DeviceGuard g(plan->device);
    rc = one_shot(plan, x, y, stats, setup);
  }
  hmvm_b200_plan_destroy(plan);
  return rc;
}

}  // extern "C"

// ---- apply without allocation ----------------------------------------------
// The scratch of hmvm_b200_apply_noalloc: a file-scope device array, reserved
// on every GPU that loads the library until the process exits.  Host code must
// not pass its name to a kernel: on the host it only stands in for the symbol,
// so its device address is looked up with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[HMVM_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoallocMaxDevices] = {};
CUcontext g_noalloc_ctx[kNoallocMaxDevices] = {};

// Device address of the scratch array on `dev`, which must be the current
// device; looked up once per device and context and cached.  A new context on
// the device (after cudaDeviceReset, say) holds a new copy of the array, so a
// change of context makes the lookup run again.
int noalloc_scratch(int dev, void** out) {
  if (dev < 0 || dev >= kNoallocMaxDevices) return set_error(HMVM_EINVAL, "device ordinal beyond the scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  const CUcontext ctx = current_context();
  if (!g_noalloc_addr[dev] || !ctx || ctx != g_noalloc_ctx[dev]) {
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the no-alloc scratch");
    g_noalloc_addr[dev] = addr;
    g_noalloc_ctx[dev] = ctx;
  }
  *out = g_noalloc_addr[dev];
  return HMVM_OK;
}

}  // namespace

extern "C" {

int hmvm_b200_apply_noalloc(hmvm_plan* p, const void* x, void* y, void* stream) {
  int rc = check_xy(p, x, y);
  if (rc) return rc;
  if (p->tcw) return set_error(HMVM_EINVAL, "tensor-core multi-RHS plans keep their scratch in the plan; use hmvm_b200_apply");
  auto round256 = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t tbytes = round256((size_t)(p->t_len + 16) * p->t_elem);
  const size_t pbytes = round256((size_t)(p->p_len + 16) * p->p_elem);
  const size_t xbytes = p->mixed ? round256((size_t)(p->nd + 16) * sizeof(float)) : 0;
  if (tbytes + pbytes + xbytes > (size_t)HMVM_NOALLOC_SCRATCH_BYTES)
    return set_error(HMVM_ERANGE, "this plan needs " + std::to_string(tbytes + pbytes + xbytes) +
                                      " bytes of scratch but hmvm_b200_apply_noalloc has " +
                                      std::to_string((size_t)HMVM_NOALLOC_SCRATCH_BYTES) +
                                      "; use hmvm_b200_apply");
  if (p->nd == 0) return HMVM_OK;
  DeviceGuard g(p->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the plan's device");
  void* base = nullptr;
  rc = noalloc_scratch(p->device, &base);
  if (rc) return rc;
  char* tbuf = static_cast<char*>(base);
  char* pbuf = tbuf + tbytes;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // t's padding slots must read as zero, and earlier calls (of any plan) left
  // other values there; the partial sums are written in full before they are read.
  HMVM_CUDA_TRY(cudaMemsetAsync(tbuf, 0, tbytes, st), "clear the no-alloc scratch");
  if (p->mixed) return launch_stages_mixed(p, x, y, tbuf, pbuf, reinterpret_cast<float*>(pbuf + pbytes), st);
  if (p->precision == HMVM_FP64) return launch_stages<double>(p, x, y, tbuf, pbuf, st);
  return launch_stages<float>(p, x, y, tbuf, pbuf, st);
}

// ---- inspection --------------------------------------------------------
int hmvm_b200_layout_build_d(const hmvm_matrix2_d* m, const hmvm_plan_opts* opts, int32_t num_sms,
                             hmvm_layout** out) {
  if (!m || !out) return set_error(HMVM_EINVAL, "NULL argument");
  *out = nullptr;
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  if (opts) o = *opts;
  LeafTable lt;
  make_table_from_matrix2(m->nd, m->nlf, m->ktmax, m->len, m->ltmtx, m->kt, m->ndl, m->ndt, m->nstrtl, m->nstrtt,
                          m->a1, m->a2, m->rowmat, false, lt);
  hmvm_layout* h = new (std::nothrow) hmvm_layout();
  if (!h) return set_error(HMVM_ENOMEM, "host allocation failed");
  std::string msg;
  int rc = tcw_wanted(o) ? build_tc_layout(lt, o, num_sms, h->L, msg) : build_layout(lt, o, num_sms, h->L, msg);
  if (rc) {
    delete h;
    return set_error(rc, msg);
  }
  *out = h;
  return HMVM_OK;
}

int hmvm_b200_layout_build64(const hmvm_leaves64* lv, int32_t rowmat_is_float, const hmvm_plan_opts* opts,
                             int32_t num_sms, hmvm_layout** out) {
  if (!lv || !out) return set_error(HMVM_EINVAL, "NULL argument");
  *out = nullptr;
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  if (opts) o = *opts;
  LeafTable lt;
  table_from_leaves64(lv, rowmat_is_float != 0, lt);
  hmvm_layout* h = new (std::nothrow) hmvm_layout();
  if (!h) return set_error(HMVM_ENOMEM, "host allocation failed");
  std::string msg;
  int rc = tcw_wanted(o) ? build_tc_layout(lt, o, num_sms, h->L, msg) : build_layout(lt, o, num_sms, h->L, msg);
  if (rc) {
    delete h;
    return set_error(rc, msg);
  }
  *out = h;
  return HMVM_OK;
}

int hmvm_b200_plan_descriptors(const hmvm_plan* p, void** tiles_dev, int32_t* n_tiles, int32_t* stage1_tiles) {
  if (!p || !tiles_dev || !n_tiles || !stage1_tiles) return set_error(HMVM_EINVAL, "NULL argument");
  *tiles_dev = p->d_tiles;
  *n_tiles = p->stage1_tiles + p->stage2_tiles;
  *stage1_tiles = p->stage1_tiles;
  return HMVM_OK;
}

int hmvm_b200_layout_validate(const hmvm_layout* h) {
  if (!h) return set_error(HMVM_EINVAL, "NULL argument");
  std::string msg;
  const int rc = validate_layout(h->L, msg);
  return rc ? set_error(rc, "layout check: " + msg) : HMVM_OK;
}

int hmvm_b200_layout_view(const hmvm_layout* h, hmvm_layout_view* v) {
  if (!h || !v) return set_error(HMVM_EINVAL, "NULL argument");
  const HostLayout& L = h->L;
  std::memset(v, 0, sizeof(*v));
  v->precision = L.precision;
  v->vec = L.vec;
  v->n_tiles = (int32_t)L.tiles.size();
  v->n_segs = (int32_t)L.segs.size();
  v->stage1_tiles = L.stage1_tiles;
  v->stage2_tiles = L.stage2_tiles;
  v->stage1_teams = L.stage1_teams;
  v->stage2_teams = L.stage2_teams;
  v->n_red1 = (int32_t)(L.red1.size() / 4);
  v->n_red2 = (int32_t)(L.red2.size() / 4);
  v->nd = L.nd;
  v->kernel = L.kernel;
  v->data_vectors = (int64_t)L.data.size();
  v->t_len = L.t_len;
  v->p_len = L.p_len;
  v->rowscale = L.rowscale.empty() ? nullptr : L.rowscale.data();
  v->n_rowscale = (int64_t)L.rowscale.size();
  v->tiles = L.tiles.data();
  v->segs = L.segs.data();
  v->team_begin1 = L.team_begin1.data();
  v->team_begin2 = L.team_begin2.data();
  v->out_idx = L.out_idx.data();
  v->red1 = L.red1.data();
  v->red2 = L.red2.data();
  v->data = L.data.data();
  v->tcw = L.tcw ? 1 : 0;
  v->tcw_bf16 = L.tcw_bf16 ? 1 : 0;
  v->tscale = L.tscale.empty() ? nullptr : L.tscale.data();
  v->n_tscale = (int64_t)L.tscale.size();
  v->tscale_rows0 = L.tscale_rows0;
  v->tblocks = L.tblocks.empty() ? nullptr : L.tblocks.data();
  v->tgroups = L.tgroups.empty() ? nullptr : L.tgroups.data();
  v->tops = L.tops.empty() ? nullptr : L.tops.data();
  v->tgfirst = L.tgfirst.empty() ? nullptr : L.tgfirst.data();
  v->n_tgroups = (int64_t)(L.tgroups.size() / 4);
  v->n_tops = L.tops.empty() ? 0 : (int64_t)(L.tops.size() / 2) - kTcwMaxOps;
  return HMVM_OK;
}

void hmvm_b200_layout_destroy(hmvm_layout* h) { delete h; }

const char* hmvm_b200_strerror(int s) {
  switch (s) {
    case HMVM_OK: return "success";
    case HMVM_EINVAL: return "invalid argument or leaf table";
    case HMVM_ENOMEM: return "out of memory";
    case HMVM_ECUDA: return "CUDA runtime error";
    case HMVM_EIO: return "file could not be opened or read";
    case HMVM_EFORMAT: return "malformed H-matrix file";
    case HMVM_ERANGE: return "count exceeds the structure or format";
    case HMVM_ENODEV: return "no usable CUDA device";
    case HMVM_EDEVICE: return "kernel reported an error";
    default: return "unknown status";
  }
}

const char* hmvm_b200_last_error(void) { return g_last_error.c_str(); }

int hmvm_b200_version(void) { return 2; }

}  // extern "C"

// ---- batches of independent H-matrices ----------------------------------------
// Instances are grouped into classes by the pass width their right-hand sides
// need (2, 4 or 8 columns; a single column runs in a 2-wide pass) and by their
// number of passes (above 8 columns: ceil(k / 8) passes of 8).  Each class is
// planned as ONE block-diagonal H-matrix: instance m's leaves are shifted by
// its offset in rows and columns, and the class's layout is planned for its
// share of the SMs: every pass of every class runs at once, so a class gets
// the SMs in proportion to its stored elements among all passes' elements.  An apply runs every
// (class, pass) -- a part, with its own packed inputs, t, partial sums and
// concatenated outputs -- at once: one packing launch, one launch per stage
// (hmvm_batch_multi_kernel, each block running its part's body), one per
// reduction, one unpacking launch.

struct PassBufs {  // a class's buffers for one pass (pass 0: its plan's own)
  double* xm64 = nullptr;
  float* xm32 = nullptr;
  void* tm = nullptr;
  void* pm = nullptr;
  void* ycat = nullptr;
  bool owned = false;  // allocated by the batch (passes >= 1)
};

struct BatchClass {
  hmvm_plan* plan = nullptr;
  int width = 2;                 // rhs per pass (the plan's nrhs_max)
  int npass = 1;                 // passes it was grouped by (the columns given may differ)
  std::vector<int32_t> members;  // instance ids
  std::vector<int32_t> n;
  std::vector<int64_t> off;
  int64_t ntot = 0;
  int32_t nmax = 0;
  int passes = 0;                // passes of the columns last given
  std::vector<PassBufs> pass;    // buffers per pass (grown on demand, kept)
};

struct hmvm_batch {
  int32_t count = 0;
  std::vector<int32_t> cls_of;  // class of each instance
  std::vector<int32_t> pos_of;  // position within its class
  std::vector<BatchClass> cls;
  // the part tables of the columns last given
  std::vector<BatchIO> io;      // per instance
  std::vector<BatchPack> pack;  // per (instance, pass)
  std::vector<BatchPart> parts;        // the V-stage parts, then the row-stage parts
  int n1 = 0;                          // V-stage parts
  std::vector<BatchRedPart> reds;      // the V-stage reductions, then the row-stage ones
  int nr1 = 0;
  int64_t red_total[2] = {0, 0};       // work items of each reduction launch
  BatchIO* d_io = nullptr;
  BatchPack* d_pack = nullptr;
  BatchPart* d_parts = nullptr;
  BatchRedPart* d_reds = nullptr;
  size_t cap_io = 0, cap_pack = 0, cap_parts = 0, cap_reds = 0;
  int64_t nmax_rows = 0;        // the largest instance (pack / unpack grids)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

namespace {

// Pass width of an instance applied with k right-hand sides (k > 8: ceil(k / 8)
// passes of 8).
int batch_width(int32_t k) {
  if (k <= 2) return 2;
  if (k <= 4) return 4;
  return 8;
}

void free_batch(hmvm_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  for (void* q : {(void*)b->d_io, (void*)b->d_pack, (void*)b->d_parts, (void*)b->d_reds})
    if (q) cudaFree(q);
  b->d_io = nullptr;
  b->d_pack = nullptr;
  b->d_parts = nullptr;
  b->d_reds = nullptr;
  for (BatchClass& c : b->cls) {
    for (PassBufs& q : c.pass) {
      if (q.owned)
        for (void* v : {(void*)q.xm64, (void*)q.xm32, q.tm, q.pm})
          if (v) cudaFree(v);
      if (q.ycat) cudaFree(q.ycat);
    }
    c.pass.clear();
    if (c.plan) hmvm_b200_plan_destroy(c.plan);
    c.plan = nullptr;
  }
}

// Buffers of pass q of class c (pass 0 uses the plan's packed inputs, t and partials).
int class_pass_buffers(BatchClass& c, int q) {
  hmvm_plan* p = c.plan;
  while ((int)c.pass.size() <= q) {
    const int k = (int)c.pass.size();
    const size_t nr = (size_t)c.width;
    PassBufs b;
    cudaError_t e = cudaSuccess;
    if (k == 0) {
      b.xm64 = p->d_xm64;
      b.xm32 = p->d_xm32;
      b.tm = p->d_tm;
      b.pm = p->d_pm;
    } else {
      b.owned = true;
      if (p->d_xm64) e = cudaMalloc(&b.xm64, (size_t)(c.ntot + 16) * nr * sizeof(double));
      if (e == cudaSuccess && b.xm64) e = cudaMemset(b.xm64, 0, (size_t)(c.ntot + 16) * nr * sizeof(double));
      if (e == cudaSuccess && p->d_xm32) e = cudaMalloc(&b.xm32, (size_t)(c.ntot + 16) * nr * sizeof(float));
      if (e == cudaSuccess && b.xm32) e = cudaMemset(b.xm32, 0, (size_t)(c.ntot + 16) * nr * sizeof(float));
      if (e == cudaSuccess) e = cudaMalloc(&b.tm, (size_t)(p->t_len + 16) * nr * p->t_elem);
      if (e == cudaSuccess) e = cudaMemset(b.tm, 0, (size_t)(p->t_len + 16) * nr * p->t_elem);
      if (e == cudaSuccess) e = cudaMalloc(&b.pm, (size_t)(p->p_len + 16) * nr * p->p_elem);
    }
    if (e == cudaSuccess) e = cudaMalloc(&b.ycat, (size_t)(c.ntot + 16) * nr * p->elem);
    if (e != cudaSuccess) {
      if (b.owned)
        for (void* v : {(void*)b.xm64, (void*)b.xm32, b.tm, b.pm})
          if (v) cudaFree(v);
      if (b.ycat) cudaFree(b.ycat);
      return cuda_fail(e, "batch pass buffers");
    }
    c.pass.push_back(b);
  }
  return HMVM_OK;
}

int class_create(BatchClass& c, const std::vector<LeafTable>& tabs, bool is_float, hmvm_plan_opts o, int sms) {
  int64_t ntot = 0, nlf = 0, len = 0;
  int32_t ktmax = 0, nmax = 0;
  for (int32_t m : c.members) {
    const LeafTable& t = tabs[m];
    ntot += t.nd;
    nlf += t.nlf;
    len += t.len;
    ktmax = std::max(ktmax, t.ktmax);
    nmax = std::max(nmax, t.nd);
  }
  if (ntot > INT32_MAX - 64 || nlf > INT32_MAX) return set_error(HMVM_ERANGE, "batch class too large for one plan");
  std::vector<int32_t> ltmtx, kt, ndl, ndt, sl, st;
  std::vector<int64_t> a1, a2;
  std::vector<unsigned char> rowmat;
  const size_t esz = is_float ? 4 : 8;
  try {
    for (auto* v : {&ltmtx, &kt, &ndl, &ndt, &sl, &st}) v->reserve((size_t)nlf);
    a1.reserve((size_t)nlf);
    a2.reserve((size_t)nlf);
    rowmat.resize((size_t)len * esz);
  } catch (const std::bad_alloc&) {
    return set_error(HMVM_ENOMEM, "host allocation failed while merging the batch");
  }
  int64_t roff = 0, loff = 0;
  for (int32_t m : c.members) {
    const LeafTable& t = tabs[m];
    c.n.push_back(t.nd);
    c.off.push_back(roff);
    for (int32_t i = 0; i < t.nlf; i++) {
      ltmtx.push_back(t.ltmtx[i]);
      kt.push_back(t.kt[i]);
      ndl.push_back(t.ndl[i]);
      ndt.push_back(t.ndt[i]);
      sl.push_back(t.nstrtl[i] + (int32_t)roff);
      st.push_back(t.nstrtt[i] + (int32_t)roff);
      a1.push_back(t.a1(i) + loff);
      a2.push_back(t.a2(i) + loff);
    }
    if (t.len > 0) std::memcpy(rowmat.data() + (size_t)loff * esz, t.rowmat, (size_t)t.len * esz);
    roff += t.nd;
    loff += t.len;
  }
  c.ntot = ntot;
  c.nmax = nmax;
  LeafTable mt;
  mt.nd = (int32_t)ntot;
  mt.nlf = (int32_t)nlf;
  mt.ktmax = ktmax;
  mt.len = len;
  mt.ltmtx = ltmtx.data();
  mt.kt = kt.data();
  mt.ndl = ndl.data();
  mt.ndt = ndt.data();
  mt.nstrtl = sl.data();
  mt.nstrtt = st.data();
  mt.a1_64 = a1.data();
  mt.a2_64 = a2.data();
  mt.rowmat = rowmat.data();
  mt.rowmat_is_float = is_float;
  o.nrhs_max = c.width;
  int rc = create_plan(mt, &o, &c.plan, sms);
  if (rc) return rc;
  DeviceGuard g(c.plan->device);
  // the packed inputs' pad rows are never written: zero them once
  hmvm_plan* p = c.plan;
  cudaError_t e = cudaSuccess;
  if (p->d_xm64) e = cudaMemset(p->d_xm64, 0, (size_t)(ntot + 16) * c.width * sizeof(double));
  if (e == cudaSuccess && p->d_xm32) e = cudaMemset(p->d_xm32, 0, (size_t)(ntot + 16) * c.width * sizeof(float));
  if (e != cudaSuccess) return cuda_fail(e, "batch buffers");
  rc = class_pass_buffers(c, 0);
  if (rc) return rc;
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "batch buffers");
  return HMVM_OK;
}

int batch_mode(const hmvm_batch* b) { return plan_mode(b->cls.front().plan); }

template <int MODE, bool VST>
const void* batch_stage_kernel() {
  constexpr MultiCfg c = kMultiCfgs[kDefaultMultiCfg];
  return (const void*)hmvm_batch_multi_kernel<c.wpb, c.slots, c.chunk, MODE, VST>;
}
const void* batch_stage_kernel_for(int mode, bool vst) {
  switch (mode) {
    case kModePlain64: return vst ? batch_stage_kernel<kModePlain64, true>() : batch_stage_kernel<kModePlain64, false>();
    case kModePlain32: return vst ? batch_stage_kernel<kModePlain32, true>() : batch_stage_kernel<kModePlain32, false>();
    case kModeMixed16: return vst ? batch_stage_kernel<kModeMixed16, true>() : batch_stage_kernel<kModeMixed16, false>();
    default: return vst ? batch_stage_kernel<kModeMixedBF16, true>() : batch_stage_kernel<kModeMixedBF16, false>();
  }
}

int batch_create(const std::vector<LeafTable>& tabs, bool is_float, const hmvm_plan_opts* opts,
                 const int32_t* nrhs, hmvm_batch** out) {
  if (!out) return set_error(HMVM_EINVAL, "output handle is NULL");
  *out = nullptr;
  const int32_t count = (int32_t)tabs.size();
  if (count <= 0) return set_error(HMVM_EINVAL, "a batch needs at least one matrix");
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  if (opts) o = *opts;
  for (int32_t m = 0; m < count; m++) {
    std::string msg;
    int rc = validate_leaves(tabs[m], msg);
    if (rc) return set_error(rc, "batch instance " + std::to_string(m) + ": " + msg);
    if (nrhs && nrhs[m] < 0) return set_error(HMVM_EINVAL, "nrhs < 0");
  }
  int dev = 0, sms = 0;
  {
    int rc = check_device(o.device, &dev, &sms);
    if (rc) return rc;
  }
  hmvm_batch* b = new (std::nothrow) hmvm_batch();
  if (!b) return set_error(HMVM_ENOMEM, "host allocation failed");
  b->count = count;
  b->cls_of.assign(count, -1);
  b->pos_of.assign(count, -1);
  // classes in the order of their widths (2, 4, 8) and passes; each planned for its
  // share of the SMs: its stored elements among the elements of all passes
  const int32_t kdef = std::min(std::max(o.nrhs_max, 1), kMaxNrhsPass);
  std::vector<int> keys;  // width * 1024 + passes
  for (int32_t m = 0; m < count; m++) {
    const int32_t k = nrhs ? nrhs[m] : kdef;
    const int w = batch_width(k), np = std::max(1, (k + w - 1) / w);
    keys.push_back(w * 1024 + np);
  }
  std::vector<int> order(keys);
  std::sort(order.begin(), order.end());
  order.erase(std::unique(order.begin(), order.end()), order.end());
  std::vector<double> elems;
  double wsum = 0;
  for (int key : order) {
    BatchClass c;
    c.width = key / 1024;
    c.npass = key % 1024;
    double el = 0;
    for (int32_t m = 0; m < count; m++) {
      if (keys[m] != key) continue;
      b->cls_of[m] = (int32_t)b->cls.size();
      b->pos_of[m] = (int32_t)c.members.size();
      c.members.push_back(m);
      el += (double)std::max<int64_t>(tabs[m].len, 1);
    }
    wsum += el * c.npass;
    b->cls.push_back(std::move(c));
    elems.push_back(el);
  }
  for (size_t k = 0; k < b->cls.size(); k++) {
    const int share = std::max(1, (int)std::lround(sms * elems[k] / std::max(wsum, 1.0)));
    int rc = class_create(b->cls[k], tabs, is_float, o, std::min(share, sms));
    if (rc) {
      {
        DeviceGuard g(dev);
        free_batch(b);
      }
      delete b;
      return rc;
    }
  }
  b->device = b->cls.front().plan->device;
  {
    DeviceGuard g(b->device);
    const int smem = multi_smem_bytes(kMultiCfgs[kDefaultMultiCfg], batch_mode(b) == kModePlain64);
    for (bool vst : {true, false}) {
      cudaError_t e = cudaFuncSetAttribute(batch_stage_kernel_for(batch_mode(b), vst),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (e != cudaSuccess) {
        free_batch(b);
        delete b;
        return cuda_fail(e, "cudaFuncSetAttribute");
      }
    }
  }
  *out = b;
  return HMVM_OK;
}

MultiArgs part_args(const hmvm_plan* p, const PassBufs& q, bool vst, int64_t ldy) {
  MultiArgs a;
  const int64_t w = p->nrhs_max;
  a.xcap = (int64_t)(p->nd + 16) * w;
  a.tcap = (int64_t)(p->t_len + 16) * w;
  a.pcap = (int64_t)(p->p_len + 16) * w;
  a.ycap = (int64_t)(p->nd + 16) * w;
  a.err = p->d_err;
  a.tiles = p->d_tiles;
  a.segs = p->d_segs;
  a.team_begin = vst ? p->d_tb1 : p->d_tb2;
  a.nteams = vst ? p->stage1_teams : p->stage2_teams;
  a.data = p->d_data;
  a.x64 = q.xm64;
  a.x32 = q.xm32;
  a.t = q.tm;
  a.y = q.ycat;
  a.ldy = ldy;
  a.nr = p->nrhs_max;
  a.p = q.pm;
  a.out_idx = p->d_out_idx;
  a.scale = p->d_scale;
  return a;
}

// The part tables for these columns: per class its passes (the widest instance
// sets them), per (class, pass) a part of each stage and reduction, per
// (instance, pass) a row of the pack / unpack grids.
int batch_set_io(hmvm_batch* b, const void* const* X, const int64_t* ldx, void* const* Y, const int64_t* ldy,
                 const int32_t* nrhs) {
  if (!b) return set_error(HMVM_EINVAL, "batch is NULL");
  if (!X || !ldx || !Y || !ldy || !nrhs) return set_error(HMVM_EINVAL, "NULL argument array");
  std::vector<BatchIO> io(b->count);
  for (int32_t m = 0; m < b->count; m++) {
    const BatchClass& c = b->cls[b->cls_of[m]];
    BatchIO& q = io[m];
    q.X = X[m];
    q.ldx = ldx[m];
    q.Y = Y[m];
    q.ldy = ldy[m];
    q.off = c.off[b->pos_of[m]];
    q.n = c.n[b->pos_of[m]];
    q.nrhs = nrhs[m];
    if (q.nrhs < 0) return set_error(HMVM_EINVAL, "instance " + std::to_string(m) + ": nrhs < 0");
    if (q.n == 0 || q.nrhs == 0) continue;
    if (!q.X || !q.Y) return set_error(HMVM_EINVAL, "instance " + std::to_string(m) + ": X or Y is NULL");
    if (q.ldx < q.n || q.ldy < q.n) return set_error(HMVM_EINVAL, "instance " + std::to_string(m) + ": ld < N");
  }
  DeviceGuard g(b->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the batch's device");
  std::vector<BatchPack> pack;
  std::vector<BatchPart> p1, p2;
  std::vector<BatchRedPart> r1, r2;
  int64_t nmax_rows = 0;
  auto stage_add = [](std::vector<BatchPart>& v, const MultiArgs& a, int nr) {
    const int ctas = (a.nteams + kMultiCfgs[kDefaultMultiCfg].wpb - 1) / kMultiCfgs[kDefaultMultiCfg].wpb;
    if (ctas <= 0) return;
    BatchPart q;
    q.a = a;
    q.cta0 = v.empty() ? 0 : v.back().cta0 + (v.back().a.nteams + kMultiCfgs[kDefaultMultiCfg].wpb - 1) /
                                                  kMultiCfgs[kDefaultMultiCfg].wpb;
    q.nr = nr;
    v.push_back(q);
  };
  auto red_add = [](std::vector<BatchRedPart>& v, const int4* red, int n, const void* pp, int64_t pcap, void* dst,
                    int64_t dcap, int64_t ld, int nr) {
    if (n <= 0) return;
    BatchRedPart q;
    q.red = red;
    q.p = pp;
    q.dst = dst;
    q.ldy = ld;
    q.w0 = v.empty() ? 0 : v.back().w0 + (int64_t)v.back().n * v.back().nr;
    q.pcap = pcap;
    q.dcap = dcap;
    q.n = n;
    q.nr = nr;
    v.push_back(q);
  };
  for (BatchClass& c : b->cls) {
    int mx = 0;
    for (size_t i = 0; i < c.members.size(); i++) mx = std::max(mx, (int)io[c.members[i]].nrhs);
    c.passes = (mx + c.width - 1) / c.width;
    if (c.passes > 0) {
      int rc = class_pass_buffers(c, c.passes - 1);
      if (rc) return rc;
    }
    const hmvm_plan* p = c.plan;
    const int64_t w = c.width;
    const int64_t xcap = (c.ntot + 16) * w, tcap = (p->t_len + 16) * w, pcap = (p->p_len + 16) * w;
    for (int q = 0; q < c.passes; q++) {
      const PassBufs& pb = c.pass[q];
      if (p->stage1_tiles > 0) stage_add(p1, part_args(p, pb, true, c.ntot), c.width);
      stage_add(p2, part_args(p, pb, false, c.ntot), c.width);
      red_add(r1, (const int4*)p->d_red1, p->n_red1, pb.pm, pcap, pb.tm, tcap, 0, c.width);
      red_add(r2, (const int4*)p->d_red2, p->n_red2, pb.pm, pcap, pb.ycat, xcap, c.ntot, c.width);
      for (size_t i = 0; i < c.members.size(); i++) {
        const int32_t m = c.members[i];
        if (io[m].n == 0 || io[m].nrhs <= q * c.width) continue;  // no columns in this pass
        BatchPack e;
        e.io = m;
        e.c0 = q * c.width;
        e.nr = c.width;
        e._pad = 0;
        e.x64 = pb.xm64;
        e.x32 = pb.xm32;
        e.ycat = pb.ycat;
        e.ldc = c.ntot;
        e.xcap = xcap;
        e.ycap = xcap;
        pack.push_back(e);
        nmax_rows = std::max<int64_t>(nmax_rows, io[m].n);
      }
    }
  }
  const int n1 = (int)p1.size(), nr1 = (int)r1.size();
  const int64_t tot1 = r1.empty() ? 0 : r1.back().w0 + (int64_t)r1.back().n * r1.back().nr;
  const int64_t tot2 = r2.empty() ? 0 : r2.back().w0 + (int64_t)r2.back().n * r2.back().nr;
  p1.insert(p1.end(), p2.begin(), p2.end());
  r1.insert(r1.end(), r2.begin(), r2.end());
  // device copies of the tables (grown on demand)
  auto grow = [](auto*& d, size_t& cap, size_t need, const char* what) -> int {
    if (need <= cap) return HMVM_OK;
    if (d) cudaFree(d);
    d = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&d, need * sizeof(*d));
    if (e != cudaSuccess) return cuda_fail(e, what);
    cap = need;
    return HMVM_OK;
  };
  int rc = grow(b->d_io, b->cap_io, io.size(), "batch table");
  if (!rc) rc = grow(b->d_pack, b->cap_pack, std::max<size_t>(pack.size(), 1), "batch table");
  if (!rc) rc = grow(b->d_parts, b->cap_parts, std::max<size_t>(p1.size(), 1), "batch table");
  if (!rc) rc = grow(b->d_reds, b->cap_reds, std::max<size_t>(r1.size(), 1), "batch table");
  if (rc) return rc;
  b->io.swap(io);
  b->pack.swap(pack);
  b->parts.swap(p1);
  b->n1 = n1;
  b->reds.swap(r1);
  b->nr1 = nr1;
  b->red_total[0] = tot1;
  b->red_total[1] = tot2;
  b->nmax_rows = nmax_rows;
  return HMVM_OK;
}

template <typename T>
int batch_run_t(hmvm_batch* b, cudaStream_t st) {
  if (b->pack.empty()) return HMVM_OK;
  const int mode = batch_mode(b);
  int* err = b->cls.front().plan->d_err;
  const MultiCfg& mc = kMultiCfgs[kDefaultMultiCfg];
  const int threads = 32 * mc.wpb, smem = multi_smem_bytes(mc, mode == kModePlain64);
  const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>((b->nmax_rows * 8 + 255) / 256, 64));
  const dim3 pgrid(gx, (unsigned)b->pack.size());
  const int nio = (int)b->io.size();
  hmvm_batch_pack_kernel<T><<<pgrid, 256, 0, st>>>(b->d_io, nio, b->d_pack, err);
  HMVM_CUDA_TRY(cudaGetLastError(), "batch packing launch");
  const bool f32 = b->cls.front().plan->precision == HMVM_FP32;  // partial sums in FP32
  auto run_reduce = [&](const BatchRedPart* parts, int n, int64_t total, bool vst) -> int {
    if (n == 0 || total == 0) return HMVM_OK;
    const int blocks = (int)std::min<int64_t>((total + 255) / 256, 65535);
    if (vst) {
      if (mode == kModePlain64) hmvm_batch_reduce_kernel<double, double, true><<<blocks, 256, 0, st>>>(parts, n, total, err);
      else if (f32) hmvm_batch_reduce_kernel<float, float, true><<<blocks, 256, 0, st>>>(parts, n, total, err);
      else hmvm_batch_reduce_kernel<double, float, true><<<blocks, 256, 0, st>>>(parts, n, total, err);
    } else {
      if (f32) hmvm_batch_reduce_kernel<float, float, false><<<blocks, 256, 0, st>>>(parts, n, total, err);
      else hmvm_batch_reduce_kernel<double, double, false><<<blocks, 256, 0, st>>>(parts, n, total, err);
    }
    HMVM_CUDA_TRY(cudaGetLastError(), "batch reduction launch");
    return HMVM_OK;
  };
  auto run_stage = [&](int k0, int n, bool vst) -> int {
    if (n == 0) return HMVM_OK;
    const BatchPart& last = b->parts[k0 + n - 1];
    const unsigned grid = (unsigned)(last.cta0 + (last.a.nteams + mc.wpb - 1) / mc.wpb);
    const BatchPart* dp = b->d_parts + k0;
    void* args[] = {(void*)&dp, (void*)&n};
    HMVM_CUDA_TRY(cudaLaunchKernel(batch_stage_kernel_for(mode, vst), dim3(grid), dim3((unsigned)threads), args,
                                   (size_t)smem, st),
                  vst ? "batch V-stage launch" : "batch row-stage launch");
    return HMVM_OK;
  };
  const int np = (int)b->parts.size(), nrd = (int)b->reds.size();
  int rc = run_stage(0, b->n1, true);
  if (!rc) rc = run_reduce(b->d_reds, b->nr1, b->red_total[0], true);
  if (!rc) rc = run_stage(b->n1, np - b->n1, false);
  if (!rc) rc = run_reduce(b->d_reds + b->nr1, nrd - b->nr1, b->red_total[1], false);
  if (rc) return rc;
  hmvm_batch_unpack_parts_kernel<T><<<pgrid, 256, 0, st>>>(b->d_io, nio, b->d_pack, err);
  HMVM_CUDA_TRY(cudaGetLastError(), "batch unpacking launch");
  return HMVM_OK;
}

int batch_run(hmvm_batch* b, cudaStream_t st) {
  HMVM_CUDA_TRY(cudaMemcpyAsync(b->d_io, b->io.data(), sizeof(BatchIO) * b->io.size(), cudaMemcpyHostToDevice, st),
                "batch table upload");
  if (!b->pack.empty())
    HMVM_CUDA_TRY(cudaMemcpyAsync(b->d_pack, b->pack.data(), sizeof(BatchPack) * b->pack.size(),
                                  cudaMemcpyHostToDevice, st),
                  "batch table upload");
  if (!b->parts.empty())
    HMVM_CUDA_TRY(cudaMemcpyAsync(b->d_parts, b->parts.data(), sizeof(BatchPart) * b->parts.size(),
                                  cudaMemcpyHostToDevice, st),
                  "batch table upload");
  if (!b->reds.empty())
    HMVM_CUDA_TRY(cudaMemcpyAsync(b->d_reds, b->reds.data(), sizeof(BatchRedPart) * b->reds.size(),
                                  cudaMemcpyHostToDevice, st),
                  "batch table upload");
  // X and Y: FP32 for FP32 plans, FP64 otherwise (whatever the stored elements were)
  return b->cls.front().plan->precision == HMVM_FP32 ? batch_run_t<float>(b, st) : batch_run_t<double>(b, st);
}

int batch_create_tables(std::vector<LeafTable>& t, bool is_float, const hmvm_plan_opts* opts, const int32_t* nrhs,
                        hmvm_batch** out) {
  return batch_create(t, is_float, opts, nrhs, out);
}

}  // namespace

extern "C" {

int hmvm_b200_batch_create64_d(const hmvm_leaves64* mats, int32_t count, const hmvm_plan_opts* opts,
                               const int32_t* nrhs, hmvm_batch** out) {
  if (!mats || count <= 0) return set_error(HMVM_EINVAL, "no matrices");
  std::vector<LeafTable> t((size_t)count);
  for (int32_t m = 0; m < count; m++) table_from_leaves64(&mats[m], false, t[m]);
  return batch_create_tables(t, false, opts, nrhs, out);
}

int hmvm_b200_batch_create64_f(const hmvm_leaves64* mats, int32_t count, const hmvm_plan_opts* opts,
                               const int32_t* nrhs, hmvm_batch** out) {
  if (!mats || count <= 0) return set_error(HMVM_EINVAL, "no matrices");
  hmvm_plan_opts o;
  hmvm_b200_default_opts(&o);
  if (opts) o = *opts;
  o.precision = HMVM_FP32;
  std::vector<LeafTable> t((size_t)count);
  for (int32_t m = 0; m < count; m++) table_from_leaves64(&mats[m], true, t[m]);
  return batch_create_tables(t, true, &o, nrhs, out);
}

int hmvm_b200_batch_create_d(const hmvm_matrix2_d* mats, int32_t count, const hmvm_plan_opts* opts,
                             const int32_t* nrhs, hmvm_batch** out) {
  if (!mats || count <= 0) return set_error(HMVM_EINVAL, "no matrices");
  std::vector<LeafTable> t((size_t)count);
  for (int32_t m = 0; m < count; m++) {
    const hmvm_matrix2_d* q = &mats[m];
    make_table_from_matrix2(q->nd, q->nlf, q->ktmax, q->len, q->ltmtx, q->kt, q->ndl, q->ndt, q->nstrtl, q->nstrtt,
                            q->a1, q->a2, q->rowmat, false, t[m]);
  }
  return batch_create_tables(t, false, opts, nrhs, out);
}

void hmvm_b200_batch_destroy(hmvm_batch* b) {
  if (!b) return;
  {
    DeviceGuard g(b->device);
    free_batch(b);
  }
  delete b;
}

int hmvm_b200_batch_get_info(const hmvm_batch* b, hmvm_plan_info* info) {
  if (!b || !info) return set_error(HMVM_EINVAL, "NULL argument");
  int rc = hmvm_b200_plan_get_info(b->cls.front().plan, info);
  if (rc) return rc;
  // sums over the classes
  for (size_t k = 1; k < b->cls.size(); k++) {
    hmvm_plan_info q;
    rc = hmvm_b200_plan_get_info(b->cls[k].plan, &q);
    if (rc) return rc;
    info->nd += q.nd;
    info->nlf += q.nlf;
    info->n_lowrank += q.n_lowrank;
    info->n_dense += q.n_dense;
    info->algorithmic_bytes += q.algorithmic_bytes;
    info->device_bytes += q.device_bytes;
    info->t_len += q.t_len;
    info->stage1_tiles += q.stage1_tiles;
    info->stage2_tiles += q.stage2_tiles;
    info->split_rows += q.split_rows;
    info->kernels_per_apply += q.kernels_per_apply;
    info->flops += q.flops;
    info->stage1_bytes += q.stage1_bytes;
    info->stage2_bytes += q.stage2_bytes;
    info->cols_fp32 += q.cols_fp32;
    info->cols_lr16 += q.cols_lr16;
    info->cols_fp8 += q.cols_fp8;
  }
  return HMVM_OK;
}

int hmvm_b200_batch_instance(const hmvm_batch* b, int32_t m, int32_t* n, int32_t* cls, int64_t* offset) {
  if (!b || m < 0 || m >= b->count) return set_error(HMVM_EINVAL, "no such instance");
  const BatchClass& c = b->cls[b->cls_of[m]];
  if (n) *n = c.n[b->pos_of[m]];
  if (cls) *cls = b->cls_of[m];
  if (offset) *offset = c.off[b->pos_of[m]];
  return HMVM_OK;
}

int hmvm_b200_batch_class_count(const hmvm_batch* b) { return b ? (int)b->cls.size() : 0; }

int hmvm_b200_batch_apply(hmvm_batch* b, const void* const* X, const int64_t* ldx, void* const* Y,
                          const int64_t* ldy, const int32_t* nrhs, void* stream) {
  int rc = batch_set_io(b, X, ldx, Y, ldy, nrhs);
  if (rc) return rc;
  DeviceGuard g(b->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the batch's device");
  return batch_run(b, static_cast<cudaStream_t>(stream));
}

int hmvm_b200_batch_capture(hmvm_batch* b, const void* const* X, const int64_t* ldx, void* const* Y,
                            const int64_t* ldy, const int32_t* nrhs) {
  int rc = batch_set_io(b, X, ldx, Y, ldy, nrhs);
  if (rc) return rc;
  DeviceGuard g(b->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the batch's device");
  for (const BatchClass& c : b->cls)
    if (c.plan->profiling) return set_error(HMVM_EINVAL, "profiling is on; a captured batch cannot record events");
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  cudaStream_t cs;
  HMVM_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate");
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaStreamDestroy(cs);
    return cuda_fail(e, "cudaStreamBeginCapture");
  }
  rc = batch_run(b, cs);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(cs, &graph);  // always end the capture
  cudaStreamDestroy(cs);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&b->exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return cuda_fail(e, "cudaGraphInstantiate");
  }
  b->graph = graph;
  return HMVM_OK;
}

int hmvm_b200_batch_launch(hmvm_batch* b, void* stream) {
  if (!b) return set_error(HMVM_EINVAL, "batch is NULL");
  if (!b->exec) return set_error(HMVM_EINVAL, "nothing captured: call hmvm_b200_batch_capture first");
  DeviceGuard g(b->device);
  if (!g.ok) return set_error(HMVM_ECUDA, "cannot select the batch's device");
  HMVM_CUDA_TRY(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)), "cudaGraphLaunch");
  return HMVM_OK;
}

int hmvm_b200_batch_status(hmvm_batch* b) {
  if (!b) return set_error(HMVM_EINVAL, "batch is NULL");
  for (BatchClass& c : b->cls) {
    int rc = hmvm_b200_plan_status(c.plan);
    if (rc) return rc;
  }
  return HMVM_OK;
}

int hmvm_b200_batch_kernel_count(const hmvm_batch* b) {
  if (!b || b->pack.empty()) return 0;
  // pack, one launch per stage and per reduction that has work, unpack
  const int np = (int)b->parts.size(), nrd = (int)b->reds.size();
  return 2 + (b->n1 > 0) + (np > b->n1) + (b->nr1 > 0 && b->red_total[0] > 0) + (nrd > b->nr1 && b->red_total[1] > 0);
}

}  // extern "C"
