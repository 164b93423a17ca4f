// Leaf fill on the GPU: the step before the HMVM (HACApK_fill_leafmtx_hyp,
// src_hdump/m_HACApK_base.f90:580-662, an OpenMP loop over leaves in the
// reference) for the generator's point kernel K(i,j) = 1/(4*pi*|p_i - p_j|).
//
// Low-rank leaves: partially pivoted ACA (HACApK_aca, m_HACApK_base.f90:
// 494-577, with the generator's parameters), one CTA per leaf, largest leaves
// first.  Within a term the residual row / column is computed element-parallel
// (each element's sum over earlier terms in term order), the pivot search is an
// argmax whose ties go to the lowest index, and the scaled 2-norms of the
// stopping test (HACApK_unrm_d, HACApK_lib.f90:31-46) run sequentially, one
// thread per vector, in the reference's order.  Every floating-point operation
// is an explicitly rounded one (__dadd_rn, __dmul_rn, __ddiv_rn, __dsqrt_rn:
// no contraction into FMAs), so the factors equal the host generator's
// (csrc/hgen.cpp) bit for bit.
//
// A leaf's rank is unknown until its ACA stops, so leaves run in rounds of
// growing capacity (32, 128, 512, ... terms, capped at min(kmax, ndl, ndt));
// a leaf that would need more terms than its round's capacity stops, is marked,
// and reruns from the start in the next round.  Factors stay in their round's
// scratch until every rank is known; then the file-order offsets are computed
// on the host, a gather kernel packs the factors and a fill kernel evaluates the
// dense leaves into one device rowmat, which is copied to the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hacapk_hgen.h"
#include "hmvm_b200.h"

namespace hmvm {
int set_error(int status, const std::string& msg);
}
using hmvm::set_error;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kAcaThreads = 256;
constexpr int kAcaThreadsSmall = 64;  // leaves with max(ndl, ndt) <= 64
constexpr int kFirstCap = 32;
static_assert(kAcaThreadsSmall >= 64, "the two norm threads are 0 and 32");

struct AcaLeaf {
  int32_t ndl, ndt, nstrtl, nstrtt;
  int32_t cap, kstop;  // terms this round can hold; min(kmax, ndl, ndt)
  int64_t off;         // first double of the leaf's scratch: V [cap][ndt], U [cap][ndl], masks
};

struct AcaArgs {
  const double* xyz;  // original points, xyz interleaved
  const int32_t* lod;  // 1-based point id at each 1-based position
  const AcaLeaf* leaves;
  double* scratch;
  int32_t* kt;     // per leaf: the rank, or 0 when the round's capacity was too small
  uint8_t* flags;  // per leaf: 1 = needs more than cap terms, 2 = incomplete (zeps > eps, k < rank)
  double eps, aca_eps;
};

// Entry of the permuted matrix at 1-based positions, as hgen.cpp's kernel_entry.
__device__ __forceinline__ double aca_entry(const double* __restrict__ xyz, const int32_t* __restrict__ lod,
                                            int32_t ill, int32_t itt) {
  const int32_t i = lod[ill - 1] - 1, j = lod[itt - 1] - 1;
  if (i == j) return 1.0;
  const double dx = __dsub_rn(xyz[3 * i], xyz[3 * j]);
  const double dy = __dsub_rn(xyz[3 * i + 1], xyz[3 * j + 1]);
  const double dz = __dsub_rn(xyz[3 * i + 2], xyz[3 * j + 2]);
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  return __ddiv_rn(1.0, __dmul_rn(4.0 * kPi, __dsqrt_rn(s)));
}

// HACApK_unrm_d: the scaled 2-norm, entries below 1e-30 skipped, in order.
__device__ double aca_unrm(const double* __restrict__ za, int32_t n) {
  double zscl = 0.0, zzz = 1.0;
  for (int32_t i = 0; i < n; i++) {
    const double zza = fabs(za[i]);
    if (zza < 1.0e-30) continue;
    if (zscl < zza) {
      const double q = __ddiv_rn(zscl, zza);
      zzz = __dadd_rn(1.0, __dmul_rn(__dmul_rn(zzz, q), q));
      zscl = zza;
    } else {
      const double q = __ddiv_rn(zza, zscl);
      zzz = __dadd_rn(zzz, __dmul_rn(q, q));
    }
  }
  return __dmul_rn(zscl, __dsqrt_rn(zzz));
}

// Block-wide argmax of |value| keeping the lowest 1-based index among equal
// maxima (index 0: none above 0) -- the result of a sequential strict-greater scan.
template <int NT>
__device__ void block_argmax(double v, int32_t i, double* sv, int32_t* si, double* out_v, int32_t* out_i) {
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, v, o);
    const int32_t i2 = __shfl_down_sync(0xffffffffu, i, o);
    if (v2 > v || (v2 == v && i2 != 0 && (i == 0 || i2 < i))) {
      v = v2;
      i = i2;
    }
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sv[w] = v;
    si[w] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = sv[0];
    int32_t bi = si[0];
    for (int k = 1; k < NT / 32; k++)
      if (sv[k] > bv || (sv[k] == bv && si[k] != 0 && (bi == 0 || si[k] < bi))) {
        bv = sv[k];
        bi = si[k];
      }
    *out_v = bv;
    *out_i = bi;
  }
  __syncthreads();
}

// One leaf per CTA: HACApK_aca with the host generator's handling of a zero
// residual row (hgen.cpp: aca).
template <int NT>
__global__ void __launch_bounds__(NT) hmvm_aca_kernel(AcaArgs a, int32_t first) {
  const int32_t li = first + (int32_t)blockIdx.x;
  const AcaLeaf L = a.leaves[li];
  const int32_t ndl = L.ndl, ndt = L.ndt, nstrtl = L.nstrtl, nstrtt = L.nstrtt;
  const int tid = threadIdx.x;
  double* V = a.scratch + L.off;               // row-direction factors, [cap][ndt]
  double* U = V + (int64_t)L.cap * ndt;        // column-direction factors, [cap][ndl]
  uint8_t* rmsk = reinterpret_cast<uint8_t*>(U + (int64_t)L.cap * ndl);
  uint8_t* cmsk = rmsk + ndl;
  for (int32_t i = tid; i < ndl + ndt; i += NT) rmsk[i] = 0;

  __shared__ double sv[NT / 32];
  __shared__ int32_t si[NT / 32];
  __shared__ double s_row_max, s_col_max, s_nrm_col, s_nrm_row, s_zdltinv;
  __shared__ int32_t s_jst, s_istn;
  int32_t ist = (nstrtl > nstrtt) ? 1 : ndl;
  int32_t k = 1;
  double znrm = 0.0, zeps = 0.0;
  int32_t kt = 0;
  bool overflow = false;
  __syncthreads();
  for (;;) {
    double* prow = V + (int64_t)(k - 1) * ndt;
    double* pcol = U + (int64_t)(k - 1) * ndl;
    // residual row ist over unmasked columns; masked entries 0
    double bv = 0.0;
    int32_t bi = 0;
    for (int32_t ii = tid; ii < ndt; ii += NT) {
      double v = 0.0;
      if (!cmsk[ii]) {
        v = aca_entry(a.xyz, a.lod, ist + nstrtl - 1, ii + nstrtt);
        if (k > 1) {
          double z = 0.0;
          for (int32_t j = 0; j < k - 1; j++)
            z = __dadd_rn(z, __dmul_rn(V[(int64_t)j * ndt + ii], U[(int64_t)j * ndl + (ist - 1)]));
          v = __dsub_rn(v, z);
        }
        if (fabs(v) > bv) {
          bv = fabs(v);
          bi = ii + 1;
        }
      }
      prow[ii] = v;
    }
    block_argmax<NT>(bv, bi, sv, si, &s_row_max, &s_jst);
    const int32_t jst = s_jst;
    if (jst == 0) {
      // zero residual row: keep k-1 terms (one zero term if k == 1)
      if (k == 1) {
        for (int32_t ii = tid; ii < ndt; ii += NT) prow[ii] = 0.0;
        for (int32_t ii = tid; ii < ndl; ii += NT) pcol[ii] = 0.0;
        kt = 1;
      } else {
        kt = k - 1;
      }
      zeps = 0.0;
      break;
    }
    if (tid == 0) s_zdltinv = __ddiv_rn(1.0, prow[jst - 1]);
    __syncthreads();
    const double zdltinv = s_zdltinv;
    for (int32_t ii = tid; ii < ndt; ii += NT) prow[ii] = __dmul_rn(prow[ii], zdltinv);
    __syncthreads();
    // residual column jst over unmasked rows; the argmax also skips row ist,
    // which is masked before the search
    bv = 0.0;
    bi = 0;
    for (int32_t ii = tid; ii < ndl; ii += NT) {
      double v = 0.0;
      if (!rmsk[ii]) {
        v = aca_entry(a.xyz, a.lod, ii + nstrtl, jst + nstrtt - 1);
        if (k > 1) {
          double z = 0.0;
          for (int32_t j = 0; j < k - 1; j++)
            z = __dadd_rn(z, __dmul_rn(U[(int64_t)j * ndl + ii], V[(int64_t)j * ndt + (jst - 1)]));
          v = __dsub_rn(v, z);
        }
        if (ii != ist - 1 && fabs(v) > bv) {
          bv = fabs(v);
          bi = ii + 1;
        }
      }
      pcol[ii] = v;
    }
    block_argmax<NT>(bv, bi, sv, si, &s_col_max, &s_istn);
    const int32_t istn = s_istn;
    if (tid == 0) {
      rmsk[ist - 1] = 1;
      cmsk[jst - 1] = 1;
    }
    const int32_t ist_next = istn > 0 ? istn : ist;
    if (fabs(s_row_max) < a.aca_eps && fabs(s_col_max) < a.aca_eps) {
      kt = k;
      break;
    }
    // zeps = unrm(pcol) * unrm(prow): two threads, each sequential
    if (tid == 0) s_nrm_col = aca_unrm(pcol, ndl);
    if (tid == 32) s_nrm_row = aca_unrm(prow, ndt);  // NT >= 64
    __syncthreads();
    zeps = __dmul_rn(s_nrm_col, s_nrm_row);
    if (k == 1) znrm = zeps;
    zeps = znrm > 0.0 ? __ddiv_rn(zeps, znrm) : 0.0;
    if (zeps < a.eps || k == L.kstop || istn == 0) {
      kt = k;
      break;
    }
    if (k == L.cap) {
      overflow = true;
      break;
    }
    k++;
    ist = ist_next;
    __syncthreads();  // masks and factors of this term before the next
  }
  if (tid == 0) {
    a.kt[li] = overflow ? 0 : kt;
    const int32_t krank = ndl < ndt ? ndl : ndt;
    a.flags[li] = overflow ? 1 : ((zeps > a.eps && kt < krank) ? 2 : 0);
  }
}

struct GatherItem {
  const double* src;  // the leaf's V rows; its U rows start cap * ndt later
  int64_t dst_v, dst_u;
  int32_t kt, ndt, ndl, cap;
};

__global__ void hmvm_aca_gather_kernel(const GatherItem* __restrict__ items, double* __restrict__ rowmat) {
  const GatherItem g = items[blockIdx.x];
  const int64_t nv = (int64_t)g.kt * g.ndt, nu = (int64_t)g.kt * g.ndl;
  const double* su = g.src + (int64_t)g.cap * g.ndt;
  for (int64_t e = threadIdx.x; e < nv; e += blockDim.x) rowmat[g.dst_v + e] = g.src[e];
  for (int64_t e = threadIdx.x; e < nu; e += blockDim.x) rowmat[g.dst_u + e] = su[e];
}

struct DenseItem {
  int64_t dst;
  int32_t ndl, ndt, nstrtl, nstrtt;
};

// a1(it + il * ndt) = K(row il, column it) (m_HACApK_base.f90:637-649)
__global__ void hmvm_dense_fill_kernel(const DenseItem* __restrict__ items, const double* __restrict__ xyz,
                                       const int32_t* __restrict__ lod, double* __restrict__ rowmat) {
  const DenseItem d = items[blockIdx.x];
  const int64_t n = (int64_t)d.ndl * d.ndt;
  for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int32_t il = (int32_t)(e / d.ndt), it = (int32_t)(e % d.ndt);
    rowmat[d.dst + e] = aca_entry(xyz, lod, il + d.nstrtl, it + d.nstrtt);
  }
}

// Device buffers released on every exit path.
struct DevBufs {
  std::vector<void*> p;
  ~DevBufs() {
    for (void* b : p) cudaFree(b);
  }
  template <typename T>
  int alloc(T** out, size_t bytes, const char* what) {
    void* q = nullptr;
    if (cudaMalloc(&q, bytes > 0 ? bytes : 16) != cudaSuccess) {
      cudaGetLastError();
      return set_error(HMVM_ENOMEM, std::string("aca fill: device allocation for ") + what);
    }
    p.push_back(q);
    *out = static_cast<T*>(q);
    return HMVM_OK;
  }
};

// dst (pageable) = src (device), n doubles: chunks go through two pinned
// staging buffers; while chunk c transfers, all host threads copy chunk c-1 out
// (which also spreads the first-touch page faults of dst over the threads).
int copy_to_host(double* dst, const double* src, int64_t n, cudaStream_t st) {
  constexpr int64_t kChunk = (32 << 20) / sizeof(double);
  const int64_t nchunks = (n + kChunk - 1) / kChunk;
  if (nchunks == 0) return HMVM_OK;
  double* stage[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  int rc = HMVM_OK;
  for (int b = 0; b < 2 && !rc; b++)
    if (cudaMallocHost(&stage[b], sizeof(double) * kChunk) != cudaSuccess ||
        cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming) != cudaSuccess)
      rc = set_error(HMVM_ENOMEM, "aca fill: pinned staging");
  auto issue = [&](int64_t c) {
    const int64_t m = std::min(kChunk, n - c * kChunk);
    cudaError_t e = cudaMemcpyAsync(stage[c & 1], src + c * kChunk, sizeof(double) * m, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(done[c & 1], st);
    return e;
  };
  if (!rc && issue(0) != cudaSuccess) rc = set_error(HMVM_ECUDA, "aca fill: rowmat D2H");
  for (int64_t c = 1; c <= nchunks && !rc; c++) {
    // stage[c & 1] last held chunk c-2, copied out in the previous iteration
    if (c < nchunks && issue(c) != cudaSuccess) {
      rc = set_error(HMVM_ECUDA, "aca fill: rowmat D2H");
      break;
    }
    const int64_t p = c - 1, m = std::min(kChunk, n - p * kChunk);
    if (cudaEventSynchronize(done[p & 1]) != cudaSuccess) {
      rc = set_error(HMVM_ECUDA, "aca fill: rowmat D2H");
      break;
    }
    const double* s = stage[p & 1];
    double* d = dst + p * kChunk;
    constexpr int64_t kPiece = (1 << 20) / sizeof(double);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < (m + kPiece - 1) / kPiece; q++)
      std::memcpy(d + q * kPiece, s + q * kPiece, sizeof(double) * std::min(kPiece, m - q * kPiece));
  }
  cudaStreamSynchronize(st);
  for (int b = 0; b < 2; b++) {
    if (stage[b]) cudaFreeHost(stage[b]);
    if (done[b]) cudaEventDestroy(done[b]);
  }
  cudaGetLastError();
  return rc;
}

#define ACA_TRY(call, what)                                                          \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      cudaGetLastError();                                                            \
      return set_error(HMVM_ECUDA, std::string("aca fill: ") + (what) + ": " +       \
                                       cudaGetErrorString(e_));                      \
    }                                                                                \
  } while (0)

int aca_fill(hgen_hmatrix* m, const hgen_params* p, cudaStream_t st, hmvm_aca_report* rep) {
  const int32_t nlf = m->nlf, nd = m->nd;
  const double aca_eps = p->aca_eps_factor * p->eps;
  DevBufs B;
  double* d_xyz = nullptr;
  int32_t* d_lod = nullptr;
  int rc;
  if ((rc = B.alloc(&d_xyz, sizeof(double) * 3 * (size_t)nd, "points"))) return rc;
  if ((rc = B.alloc(&d_lod, sizeof(int32_t) * (size_t)nd, "permutation"))) return rc;
  ACA_TRY(cudaMemcpyAsync(d_xyz, m->coords, sizeof(double) * 3 * (size_t)nd, cudaMemcpyHostToDevice, st), "H2D");
  ACA_TRY(cudaMemcpyAsync(d_lod, m->lod, sizeof(int32_t) * (size_t)nd, cudaMemcpyHostToDevice, st), "H2D");

  // low-rank leaves, largest first (ties by file order)
  std::vector<int32_t> pending;
  for (int32_t i = 0; i < nlf; i++)
    if (m->ltmtx[i] == 1) pending.push_back(i);
  std::sort(pending.begin(), pending.end(), [&](int32_t x, int32_t y) {
    const int64_t cx = (int64_t)m->ndl[x] + m->ndt[x], cy = (int64_t)m->ndl[y] + m->ndt[y];
    return cx != cy ? cx > cy : x < y;
  });
  std::vector<GatherItem> gather;  // src filled per round
  std::vector<int32_t> gather_leaf;
  std::vector<int32_t> kt_of(nlf, 0);
  int64_t incomplete = 0;
  cudaEvent_t ev[4];
  for (auto& e : ev) ACA_TRY(cudaEventCreate(&e), "event");
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() {
      for (int i = 0; i < 4; i++) cudaEventDestroy(e[i]);
    }
  } evfree{ev};
  ACA_TRY(cudaEventRecord(ev[0], st), "event");
  int64_t base_cap = kFirstCap;
  int rounds = 0;
  int64_t scratch_total = 0;
  while (!pending.empty()) {
    rounds++;
    std::vector<AcaLeaf> lv(pending.size());
    int64_t off = 0;
    int32_t n_small = 0;  // trailing leaves handled by the 64-thread kernel
    for (size_t q = 0; q < pending.size(); q++) {
      const int32_t i = pending[q];
      AcaLeaf& L = lv[q];
      L.ndl = m->ndl[i];
      L.ndt = m->ndt[i];
      L.nstrtl = m->nstrtl[i];
      L.nstrtt = m->nstrtt[i];
      L.kstop = std::min<int32_t>(p->kmax, std::min(L.ndl, L.ndt));
      L.cap = (int32_t)std::min<int64_t>(L.kstop, base_cap);
      L.off = off;
      off += (int64_t)L.cap * (L.ndl + L.ndt) + ((int64_t)L.ndl + L.ndt + 7) / 8;
      if (std::max(L.ndl, L.ndt) <= kAcaThreadsSmall) n_small++;
    }
    const int32_t nl = (int32_t)lv.size();
    AcaLeaf* d_lv = nullptr;
    double* d_scr = nullptr;
    int32_t* d_kt = nullptr;
    uint8_t* d_fl = nullptr;
    if ((rc = B.alloc(&d_lv, sizeof(AcaLeaf) * (size_t)nl, "leaf table"))) return rc;
    if ((rc = B.alloc(&d_scr, sizeof(double) * (size_t)off, "factor scratch"))) return rc;
    if ((rc = B.alloc(&d_kt, sizeof(int32_t) * (size_t)nl, "ranks"))) return rc;
    if ((rc = B.alloc(&d_fl, (size_t)nl, "flags"))) return rc;
    scratch_total += (int64_t)sizeof(double) * off;
    ACA_TRY(cudaMemcpyAsync(d_lv, lv.data(), sizeof(AcaLeaf) * (size_t)nl, cudaMemcpyHostToDevice, st), "H2D");
    AcaArgs a{d_xyz, d_lod, d_lv, d_scr, d_kt, d_fl, p->eps, aca_eps};
    const int32_t n_big = nl - n_small;  // leaves sorted by size: the small ones are last
    if (n_big > 0) hmvm_aca_kernel<kAcaThreads><<<n_big, kAcaThreads, 0, st>>>(a, 0);
    if (n_small > 0) hmvm_aca_kernel<kAcaThreadsSmall><<<n_small, kAcaThreadsSmall, 0, st>>>(a, n_big);
    ACA_TRY(cudaGetLastError(), "ACA launch");
    std::vector<int32_t> kt(nl);
    std::vector<uint8_t> fl(nl);
    ACA_TRY(cudaMemcpyAsync(kt.data(), d_kt, sizeof(int32_t) * (size_t)nl, cudaMemcpyDeviceToHost, st), "D2H");
    ACA_TRY(cudaMemcpyAsync(fl.data(), d_fl, (size_t)nl, cudaMemcpyDeviceToHost, st), "D2H");
    ACA_TRY(cudaStreamSynchronize(st), "ACA kernels");
    std::vector<int32_t> next;
    for (int32_t q = 0; q < nl; q++) {
      const int32_t i = pending[q];
      if (fl[q] & 1) {
        next.push_back(i);
        continue;
      }
      kt_of[i] = kt[q];
      if (fl[q] & 2) incomplete++;
      GatherItem g;
      g.src = d_scr + lv[q].off;
      g.dst_v = g.dst_u = 0;
      g.kt = kt[q];
      g.ndt = lv[q].ndt;
      g.ndl = lv[q].ndl;
      g.cap = lv[q].cap;
      gather.push_back(g);
      gather_leaf.push_back(i);
    }
    pending.swap(next);
    base_cap *= 4;
  }
  ACA_TRY(cudaEventRecord(ev[1], st), "event");

  // file-order offsets (as the host generator lays them out)
  std::vector<int64_t> a1(nlf), a2(nlf);
  int64_t len = 0;
  int32_t ktmax = 0;
  std::vector<DenseItem> dense;
  for (int32_t i = 0; i < nlf; i++) {
    if (m->ltmtx[i] == 1) {
      a1[i] = len;
      len += (int64_t)kt_of[i] * m->ndt[i];
      a2[i] = len;
      len += (int64_t)kt_of[i] * m->ndl[i];
      ktmax = std::max(ktmax, kt_of[i]);
    } else {
      a1[i] = len;
      a2[i] = 0;
      dense.push_back(DenseItem{len, m->ndl[i], m->ndt[i], m->nstrtl[i], m->nstrtt[i]});
      len += (int64_t)m->ndl[i] * m->ndt[i];
    }
  }
  for (size_t g = 0; g < gather.size(); g++) {
    gather[g].dst_v = a1[gather_leaf[g]];
    gather[g].dst_u = a2[gather_leaf[g]];
  }
  double* d_rowmat = nullptr;
  GatherItem* d_g = nullptr;
  DenseItem* d_d = nullptr;
  if ((rc = B.alloc(&d_rowmat, sizeof(double) * (size_t)len, "rowmat"))) return rc;
  if ((rc = B.alloc(&d_g, sizeof(GatherItem) * gather.size(), "gather list"))) return rc;
  if ((rc = B.alloc(&d_d, sizeof(DenseItem) * dense.size(), "dense list"))) return rc;
  ACA_TRY(cudaMemcpyAsync(d_g, gather.data(), sizeof(GatherItem) * gather.size(), cudaMemcpyHostToDevice, st), "H2D");
  ACA_TRY(cudaMemcpyAsync(d_d, dense.data(), sizeof(DenseItem) * dense.size(), cudaMemcpyHostToDevice, st), "H2D");
  if (!dense.empty()) hmvm_dense_fill_kernel<<<(unsigned)dense.size(), 256, 0, st>>>(d_d, d_xyz, d_lod, d_rowmat);
  ACA_TRY(cudaGetLastError(), "dense fill launch");
  ACA_TRY(cudaEventRecord(ev[2], st), "event");
  if (!gather.empty()) hmvm_aca_gather_kernel<<<(unsigned)gather.size(), 256, 0, st>>>(d_g, d_rowmat);
  ACA_TRY(cudaGetLastError(), "gather launch");
  double* rowmat = static_cast<double*>(malloc(sizeof(double) * (size_t)(len > 0 ? len : 1)));
  if (!rowmat) return set_error(HMVM_ENOMEM, "aca fill: host rowmat");
  rc = copy_to_host(rowmat, d_rowmat, len, st);
  if (!rc && (cudaEventRecord(ev[3], st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess))
    rc = set_error(HMVM_ECUDA, "aca fill: rowmat D2H");
  if (rc) {
    free(rowmat);
    return rc;
  }
  for (int32_t i = 0; i < nlf; i++) {
    m->kt[i] = m->ltmtx[i] == 1 ? kt_of[i] : 0;
    m->a1[i] = a1[i];
    m->a2[i] = a2[i];
  }
  m->rowmat = rowmat;
  m->len = len;
  m->ktmax = ktmax;
  m->aca_incomplete = incomplete;
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->rounds = rounds;
    rep->ktmax = ktmax;
    rep->scratch_bytes = scratch_total;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    rep->ms_aca = ms;
    cudaEventElapsedTime(&ms, ev[1], ev[2]);
    rep->ms_dense = ms;
    cudaEventElapsedTime(&ms, ev[2], ev[3]);
    rep->ms_gather_copy = ms;
  }
  return HMVM_OK;
}

}  // namespace

extern "C" int hmvm_b200_aca_fill(hgen_hmatrix* m, const hgen_params* p, int32_t device, hmvm_aca_report* report) {
  if (!m || !p) return set_error(HMVM_EINVAL, "NULL argument");
  if (m->rowmat) return set_error(HMVM_EINVAL, "aca fill: the matrix already holds leaf data");
  if (m->mesh) return set_error(HMVM_EINVAL, "aca fill: the GPU fill evaluates the point kernel only (not a mesh)");
  if (!(p->eps > 0.0) || p->kmax < 1) return set_error(HMVM_EINVAL, "aca fill: eps must be > 0 and kmax >= 1");
  if (m->nlf > 0 && (!m->ltmtx || !m->ndl || !m->ndt || !m->nstrtl || !m->nstrtt || !m->kt || !m->a1 || !m->a2))
    return set_error(HMVM_EINVAL, "aca fill: missing leaf array");
  if (m->nd > 0 && (!m->coords || !m->lod)) return set_error(HMVM_EINVAL, "aca fill: missing points");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return set_error(HMVM_ENODEV, "no CUDA device available");
  }
  if (device < 0 || device >= n) return set_error(HMVM_EINVAL, "device ordinal out of range");
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10)
    return set_error(HMVM_ENODEV, "aca fill: the device is not sm_100-class");
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return set_error(HMVM_ECUDA, "cannot select the device");
  cudaStream_t st = nullptr;
  int rc = HMVM_OK;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    rc = set_error(HMVM_ECUDA, "aca fill: stream");
  } else {
    rc = aca_fill(m, p, st, report);
    cudaStreamDestroy(st);
  }
  cudaSetDevice(prev);
  return rc;
}
