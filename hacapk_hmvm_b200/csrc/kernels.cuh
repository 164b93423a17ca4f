// sm_100a kernels for the row-owned HMVM layout built by layout.cpp.
//
// hmvm_tile_kernel<T, WG, TPC>: persistent; each CTA holds TPC teams of WG
// warps and each team walks its own contiguous list of tiles.  For one tile
// (R <= 32 rows, nvec 16-byte column vectors):
//   * lane r of every warp owns row r; warp w of the team takes the w-th of WG
//     equal contiguous slices of the tile's vectors;
//   * each vector is one coalesced 16-byte-per-lane streaming load (R*16
//     contiguous bytes per warp), times VEC input values that every lane of
//     the warp reads at the same address (x for dense segments, t for
//     low-rank U segments);
//   * the WG per-lane partial sums are added in warp order through shared
//     memory after a per-team named barrier, and lane r writes its row once.
// No global atomics; the summation order is fixed by the layout, so results
// are bitwise reproducible.
//
// hmvm_stream_kernel<T, WPB, S, CHUNK, ZCAP>: persistent; every warp is a team
// and owns one contiguous region of the data stream (its items in order).
//   * Matrix bytes: lane 0 keeps S chunks of CHUNK bytes in flight into the
//     warp's shared-memory ring with cp.async.bulk (TMA bulk copies, completion
//     counted on one mbarrier per slot), refilling a slot as soon as the warp
//     has moved past it, so loads run ahead across item boundaries.
//   * Inputs: the x / t columns an item reads (<= ZCAP) are gathered into one of
//     two shared-memory buffers with cp.async while the previous item runs;
//     item descriptors are loaded two items ahead.
//   * The inner loop then only reads shared memory: lane r takes its row's
//     16-byte vector from the ring and the vector's VEC input values from the
//     buffer (a broadcast), and accumulates as in hmvm_tile_kernel.
// Every wait on an mbarrier is bounded by time; a warp that gives up sets
// *err, waits (bounded) for its copies in flight and stops.
//
// hmvm_reduce_kernel<T>: for tiles that were cut into parts, adds the parts'
// partial sums in part order and writes the t slot or y row.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include "hmvm_b200.h"
#include "validate.hpp"

namespace hmvm {

template <typename T>
struct VecT;
template <>
struct VecT<double> {
  using V = double2;
  static constexpr int N = 2;
};
template <>
struct VecT<float> {
  using V = float4;
  static constexpr int N = 4;
};

struct TileArgs {
  int* err;                   // device status word (0 = ok)
  const hmvm_tile_desc* tiles;
  const hmvm_seg_desc* segs;
  const int32_t* team_begin;  // [nteams+1] absolute tile indices
  int32_t nteams;
  const void* data;           // 16-byte vectors
  const void* x;              // input vector (T)
  void* t;                    // V x slots (T), zero padded per row group
  void* y;                    // output (T)
  void* p;                    // partial sums of split panels (T)
  const int32_t* out_idx;     // stage-1 output slots
  const float* x32;           // mixed: x rounded to FP32
  const double* scale;        // mixed, V stage: per panel-row column scale (NULL in the row stage)
};

__device__ __forceinline__ void fma_vec(double& a0, double& a1, const double2& m, const double2& z) {
  a0 = fma(m.x, z.x, a0);
  a1 = fma(m.y, z.y, a1);
}
__device__ __forceinline__ void fma_vec(float& a0, float& a1, const float4& m, const float4& z) {
  a0 = fmaf(m.x, z.x, a0);
  a1 = fmaf(m.y, z.y, a1);
  a0 = fmaf(m.z, z.z, a0);
  a1 = fmaf(m.w, z.w, a1);
}

// Programmatic dependent launch (sm_90+): a kernel lets the next kernel of the
// apply be scheduled as soon as every CTA has started (launch_dependents), and
// a kernel launched as a dependent waits for its predecessors' completion and
// memory (wait) before it reads their outputs; launched normally, wait returns
// at once.
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Device bounds checks (builds compiled with HMVM_DEVICE_CHECKS): before every
// stage launch hmvm_validate_kernel checks the stage's descriptors against the
// lengths of the buffers they index and sets the error word to
// kErrDeviceCheck on a violation; each stage kernel first waits for its
// predecessors and returns, touching nothing, while the error word is set.
// Other builds compile none of it.
#ifdef HMVM_DEVICE_CHECKS
constexpr bool kDeviceChecks = true;
#else
constexpr bool kDeviceChecks = false;
#endif
constexpr int kErrDeviceCheck = 4;
__device__ __forceinline__ bool checks_failed(const int* err) {
  if constexpr (kDeviceChecks) {
    griddep_wait();
    return *reinterpret_cast<const volatile int*>(err) != 0;
  }
  return false;
}

template <typename T>
__device__ __forceinline__ typename VecT<T>::V zero_vec() {
  typename VecT<T>::V v;
  T* e = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int i = 0; i < VecT<T>::N; i++) e[i] = T(0);
  return v;
}

// Streaming (evict-first) 16-byte load of matrix data that is read once.
template <typename V>
__device__ __forceinline__ V ld_stream(const V* p) {
  return __ldcs(p);
}

// Input values for columns [c, c+N) of an x segment whose valid columns end
// at climit (relative to zp); columns past the end read as zero.
template <typename T>
__device__ __forceinline__ typename VecT<T>::V ld_x(const T* __restrict__ zp, int c, int climit) {
  typename VecT<T>::V v;
  T* e = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int i = 0; i < VecT<T>::N; i++) e[i] = (c + i < climit) ? __ldg(zp + c + i) : T(0);
  return v;
}

template <typename T, int WG, int TPC>
__global__ void __launch_bounds__(32 * WG * TPC) hmvm_tile_kernel(TileArgs a) {
  using V = typename VecT<T>::V;
  constexpr int VN = VecT<T>::N;
  __shared__ T red[TPC][2][WG > 1 ? WG : 1][32];
  griddep_launch_dependents();
  griddep_wait();
  if (checks_failed(a.err)) return;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int tic = warp / WG;
  const int wt = warp - tic * WG;
  const int team = blockIdx.x * TPC + tic;
  if (team >= a.nteams) return;  // whole teams only (uniform per team)

  const T* __restrict__ x = static_cast<const T*>(a.x);
  const T* __restrict__ tv = static_cast<const T*>(a.t);
  const V* __restrict__ data = static_cast<const V*>(a.data);
  int parity = 0;
  const int tb = a.team_begin[team], te = a.team_begin[team + 1];
  for (int ti = tb; ti < te; ++ti) {
    const hmvm_tile_desc td = a.tiles[ti];
    const int R = td.nrows;
    const bool act = lane < R;
    const int nvt = td.nvec;
    int v = (int)(((long long)nvt * wt) / WG);
    const int vw_end = (int)(((long long)nvt * (wt + 1)) / WG);
    T acc0 = T(0), acc1 = T(0);
    const V* __restrict__ dp = data + td.data_off + lane;
    int s = td.seg_begin;
    int segv0 = 0;
    while (v < vw_end) {
      const hmvm_seg_desc sd = a.segs[s];
      const int nv = (sd.ncols + VN - 1) / VN;
      if (v >= segv0 + nv) {
        segv0 += nv;
        ++s;
        continue;
      }
      const int ve = min(vw_end, segv0 + nv);
      if (sd.src < 0) {
        // U segment: t slots are VEC-aligned and zero padded -> vector loads.
        const V* __restrict__ zv = reinterpret_cast<const V*>(tv + (sd.src & 0x7fffffff)) - segv0;
        for (; v + 4 <= ve; v += 4) {
          V m0 = act ? ld_stream(dp + (size_t)(v + 0) * R) : zero_vec<T>();
          V m1 = act ? ld_stream(dp + (size_t)(v + 1) * R) : zero_vec<T>();
          V m2 = act ? ld_stream(dp + (size_t)(v + 2) * R) : zero_vec<T>();
          V m3 = act ? ld_stream(dp + (size_t)(v + 3) * R) : zero_vec<T>();
          V z0 = __ldg(zv + v + 0), z1 = __ldg(zv + v + 1), z2 = __ldg(zv + v + 2), z3 = __ldg(zv + v + 3);
          fma_vec(acc0, acc1, m0, z0);
          fma_vec(acc0, acc1, m1, z1);
          fma_vec(acc0, acc1, m2, z2);
          fma_vec(acc0, acc1, m3, z3);
        }
        for (; v < ve; ++v) {
          V m0 = act ? ld_stream(dp + (size_t)v * R) : zero_vec<T>();
          fma_vec(acc0, acc1, m0, __ldg(zv + v));
        }
      } else {
        // Dense / V segment over x: scalar broadcast loads, columns past the
        // segment end read as zero (their matrix entries are zero padding).
        const T* __restrict__ zp = x + sd.src - (ptrdiff_t)segv0 * VN;
        const int climit = segv0 * VN + sd.ncols;
        for (; v + 4 <= ve; v += 4) {
          V m0 = act ? ld_stream(dp + (size_t)(v + 0) * R) : zero_vec<T>();
          V m1 = act ? ld_stream(dp + (size_t)(v + 1) * R) : zero_vec<T>();
          V m2 = act ? ld_stream(dp + (size_t)(v + 2) * R) : zero_vec<T>();
          V m3 = act ? ld_stream(dp + (size_t)(v + 3) * R) : zero_vec<T>();
          V z0 = ld_x<T>(zp, (v + 0) * VN, climit);
          V z1 = ld_x<T>(zp, (v + 1) * VN, climit);
          V z2 = ld_x<T>(zp, (v + 2) * VN, climit);
          V z3 = ld_x<T>(zp, (v + 3) * VN, climit);
          fma_vec(acc0, acc1, m0, z0);
          fma_vec(acc0, acc1, m1, z1);
          fma_vec(acc0, acc1, m2, z2);
          fma_vec(acc0, acc1, m3, z3);
        }
        for (; v < ve; ++v) {
          V m0 = act ? ld_stream(dp + (size_t)v * R) : zero_vec<T>();
          fma_vec(acc0, acc1, m0, ld_x<T>(zp, v * VN, climit));
        }
      }
    }
    T acc = acc0 + acc1;
    if constexpr (WG > 1) {
      red[tic][parity][wt][lane] = acc;
      asm volatile("bar.sync %0, %1;" ::"r"(1 + tic), "r"(32 * WG) : "memory");
      if (wt == 0) {
        acc = red[tic][parity][0][lane];
#pragma unroll
        for (int w = 1; w < WG; w++) acc += red[tic][parity][w][lane];
      }
      parity ^= 1;
    }
    if (wt == 0 && act) {
      if (td.mode == 0) static_cast<T*>(a.y)[td.out_base + lane] = acc;
      else if (td.mode == 1) static_cast<T*>(a.t)[a.out_idx[td.out_base + lane]] = acc;
      else static_cast<T*>(a.p)[td.out_base + lane] = acc;
    }
  }
}

// ---- TMA bulk-copy ring -------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Global -> shared bulk copy (no multicast); completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Give up on an mbarrier after this long (the copies it waits for take
// microseconds; only a broken copy would get near this).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

// Warp-uniform bounded wait for the phase with parity `parity` of `bar`.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity) {
  if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;  // usually already landed
  const uint64_t t0 = global_ns();
  for (;;) {
    bool ok = mbar_try_wait(bar, parity);
    if (__all_sync(0xffffffffu, ok)) return true;
    if (global_ns() - t0 > kWaitLimitNs) return false;
  }
}

// Asynchronous 4/8/16-byte global -> shared copy (completion by group).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copy the x / t columns item `d` reads into zb (one column per element, each
// segment padded with zeros to whole vectors), with cp.async; `sreg` holds the
// item's first 32 segment descriptors (lane j: segment j).
template <typename T>
__device__ __forceinline__ void gather_inputs(const hmvm_tile_desc& d, const hmvm_seg_desc& sreg,
                                              const hmvm_seg_desc* __restrict__ segs, const T* __restrict__ x,
                                              const T* __restrict__ tv, T* zb, int lane) {
  constexpr int VN = VecT<T>::N;
  int col0 = 0;
  for (int base = 0; base < d.nseg; base += 32) {
    hmvm_seg_desc my = sreg;
    if (base > 0) my = (base + lane < d.nseg) ? segs[d.seg_begin + base + lane] : hmvm_seg_desc{0, 0};
    const int cnt = min(32, d.nseg - base);
    for (int j = 0; j < cnt; j++) {
      const int src = __shfl_sync(0xffffffffu, my.src, j);
      const int nc = __shfl_sync(0xffffffffu, my.ncols, j);
      const int ncp = (nc + VN - 1) / VN * VN;
      const T* zs = src < 0 ? tv + (src & 0x7fffffff) : x + src;
      for (int c = lane; c < ncp; c += 32) {
        if (c < nc) cp_async<sizeof(T)>(zb + col0 + c, zs + c);
        else zb[col0 + c] = T(0);
      }
      col0 += ncp;
    }
  }
}

// CTAs of a configuration that fit one SM's 227 KB of shared memory (at most
// 24 warps): the register budget the kernel is compiled for.
template <typename T, int WPB, int S, int CHUNK, int ZCAP>
constexpr int stream_min_blocks() {
  constexpr int smem = WPB * (S * CHUNK + 2 * ZCAP * (int)sizeof(T) + S * 8);
  constexpr int by_smem = (227 * 1024) / smem;
  constexpr int by_warps = 24 / WPB;
  constexpr int m = by_smem < by_warps ? by_smem : by_warps;
  return m > 0 ? m : 1;
}

template <typename T, int WPB, int S, int CHUNK, int ZCAP>
__global__ void __launch_bounds__(32 * WPB, (stream_min_blocks<T, WPB, S, CHUNK, ZCAP>()))
    hmvm_stream_kernel(TileArgs a) {
  using V = typename VecT<T>::V;
  constexpr uint32_t RING = (uint32_t)S * CHUNK;
  // vectors per batch: 8 when the ring has room for them (see the assert below)
  constexpr int B = ((S - 1) * CHUNK / (32 * 16) >= 8) ? 8 : 4;
  static_assert((RING & (RING - 1)) == 0, "ring size must be a power of two");
  static_assert(CHUNK % 16 == 0 && CHUNK >= 512, "bulk copies move multiples of 16 bytes");
  // A batch (B vectors of <= 32 rows x 16 bytes) must fit in the S-1 slots
  // after the first one it touches, or its wait could need an unissued chunk.
  static_assert(B * 32 * 16 <= (S - 1) * CHUNK, "ring too small for one batch");
  static_assert(ZCAP % 4 == 0, "input buffers hold whole vectors");
  extern __shared__ __align__(128) unsigned char smem[];
  griddep_launch_dependents();
  if (checks_failed(a.err)) return;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int team = blockIdx.x * WPB + warp;
  if (team >= a.nteams) return;
  const int tb = a.team_begin[team], te = a.team_begin[team + 1];
  if (tb >= te) return;
  unsigned char* ring = smem + (size_t)warp * RING;
  T* zbase = reinterpret_cast<T*>(smem + (size_t)WPB * RING) + (size_t)warp * 2 * ZCAP;
  uint64_t* bars =
      reinterpret_cast<uint64_t*>(smem + (size_t)WPB * RING + (size_t)WPB * 2 * ZCAP * sizeof(T)) + warp * S;

  const hmvm_tile_desc* __restrict__ tiles = a.tiles;
  const hmvm_seg_desc* __restrict__ segs = a.segs;
  const T* __restrict__ x = static_cast<const T*>(a.x);
  const T* __restrict__ tv = static_cast<const T*>(a.t);
  const hmvm_tile_desc dzero = {0, 0, 0, 0, 0, 1, 0, 0};
  const hmvm_seg_desc szero = {0, 0};

  // ---- the matrix stream: this warp's items are one contiguous region ----
  hmvm_tile_desc cur = tiles[tb];
  const int64_t vbase = cur.data_off;
  const hmvm_tile_desc tl = tiles[te - 1];
  const int64_t total64 = (tl.data_off + (int64_t)tl.nvec * tl.nrows - vbase) * 16;
  if (total64 >= (int64_t)1 << 31) {  // the planner keeps regions far below this
    if (lane == 0) atomicExch(a.err, 2);
    return;
  }
  const uint32_t total = (uint32_t)total64;
  const char* gsrc = static_cast<const char*>(a.data) + vbase * 16;
  const uint32_t nchunks = (total + CHUNK - 1) / CHUNK;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < S; s++) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  // Lane 0 only: start the copy of chunk q into slot q % S.
  auto issue = [&](uint32_t q) {
    const uint32_t off = q * (uint32_t)CHUNK;
    const uint32_t bytes = min((uint32_t)CHUNK, total - off);
    uint64_t* bar = &bars[q % S];
    mbar_expect_tx(bar, bytes);
    bulk_g2s(ring + (q % S) * CHUNK, gsrc + off, bytes, bar);
  };
  if (lane == 0)
    for (uint32_t q = 0; q < min((uint32_t)S, nchunks); q++) issue(q);

  // ---- descriptor pipeline: item i+1's inputs are gathered during item i ----
  hmvm_seg_desc cur_seg = lane < cur.nseg ? segs[cur.seg_begin + lane] : szero;
  // the ring's first chunks (plan data) are in flight; x / t and the outputs
  // wait for the preceding kernels of the apply
  griddep_wait();
  gather_inputs<T>(cur, cur_seg, segs, x, tv, zbase, lane);
  cp_async_commit();
  hmvm_tile_desc nxt = tb + 1 < te ? tiles[tb + 1] : dzero;
  hmvm_seg_desc nxt_seg = (tb + 1 < te && lane < nxt.nseg) ? segs[nxt.seg_begin + lane] : szero;
  int nxt_oidx = (tb + 1 < te && nxt.mode == 1 && lane < nxt.nrows) ? a.out_idx[nxt.out_base + lane] : 0;
  int cur_oidx = (cur.mode == 1 && lane < cur.nrows) ? a.out_idx[cur.out_base + lane] : 0;
  hmvm_tile_desc nn = tb + 2 < te ? tiles[tb + 2] : dzero;

  uint32_t q_ready = 0, q_rel = 0;  // chunks < q_ready have landed; chunks < q_rel are released
  bool failed = false;
  for (int ti = tb, k = 0; ti < te; ++ti, ++k) {
    T* zcur = zbase + (k & 1) * ZCAP;
    __syncwarp();  // every lane is done with the buffer the next gather overwrites
    if (ti + 1 < te) gather_inputs<T>(nxt, nxt_seg, segs, x, tv, zbase + ((k + 1) & 1) * ZCAP, lane);
    cp_async_commit();
    // loads for two items ahead; they land while this item runs
    const hmvm_seg_desc nn_seg = (ti + 2 < te && lane < nn.nseg) ? segs[nn.seg_begin + lane] : szero;
    const int nn_oidx = (ti + 2 < te && nn.mode == 1 && lane < nn.nrows) ? a.out_idx[nn.out_base + lane] : 0;
    const hmvm_tile_desc nnn = ti + 3 < te ? tiles[ti + 3] : dzero;
    cp_async_wait<1>();
    __syncwarp();  // this item's inputs are in zcur

    const int R = cur.nrows;
    const bool act = lane < R;
    const uint32_t rstride = (uint32_t)R * 16;
    const int nvt = cur.nvec;
    // Lanes >= R read ring bytes of other rows (always inside the ring); their
    // sums are never written, so the loop needs no per-lane predicate.
    uint32_t o = (uint32_t)((cur.data_off - vbase) * 16);  // byte offset of vector v in the region
    const unsigned char* zc = reinterpret_cast<const unsigned char*>(zcur);
    T acc0 = T(0), acc1 = T(0), acc2 = T(0), acc3 = T(0);
    for (int v = 0; v < nvt; v += B) {
      const int nb = min(B, nvt - v);
      const uint32_t o_end = o + (uint32_t)nb * rstride;
      // Release the slots the warp has moved past, then wait for the batch's chunks.
      if (o >= (q_rel + 1) * (uint32_t)CHUNK) {
        const uint32_t qf = o / CHUNK;
        __syncwarp();
        if (lane == 0) {
          fence_proxy_async();
          for (uint32_t q = q_rel; q < qf; q++)
            if (q + S < nchunks) issue(q + S);
        }
        q_rel = qf;
      }
      if (o_end > q_ready * (uint32_t)CHUNK) {
        const uint32_t ql = (o_end - 1) / CHUNK;
        while (q_ready <= ql) {
          if (!warp_wait(&bars[q_ready % S], (q_ready / S) & 1)) {
            failed = true;
            break;
          }
          q_ready++;
        }
        if (failed) break;
      }
      const uint32_t ol = o + (uint32_t)lane * 16;
      if (nb == B) {
        V m[B], z[B];
#pragma unroll
        for (int u = 0; u < B; u++) {
          m[u] = *reinterpret_cast<const V*>(ring + ((ol + (uint32_t)u * rstride) & (RING - 1)));
          z[u] = *reinterpret_cast<const V*>(zc + (size_t)(v + u) * 16);
        }
#pragma unroll
        for (int u = 0; u < B; u += 2) {
          fma_vec(acc0, acc1, m[u], z[u]);
          fma_vec(acc2, acc3, m[u + 1], z[u + 1]);
        }
      } else {
        for (int u = 0; u < nb; u++) {
          const V m = *reinterpret_cast<const V*>(ring + ((ol + (uint32_t)u * rstride) & (RING - 1)));
          const V z = *reinterpret_cast<const V*>(zc + (size_t)(v + u) * 16);
          fma_vec(acc0, acc1, m, z);
        }
      }
      o = o_end;
    }
    if (failed) break;
    const T acc = (acc0 + acc1) + (acc2 + acc3);
    if (act) {
      if (cur.mode == 0) static_cast<T*>(a.y)[cur.out_base + lane] = acc;
      else if (cur.mode == 1) static_cast<T*>(a.t)[cur_oidx] = acc;
      else static_cast<T*>(a.p)[cur.out_base + lane] = acc;
    }
    cur = nxt;
    cur_oidx = nxt_oidx;
    nxt = nn;
    nxt_seg = nn_seg;
    nxt_oidx = nn_oidx;
    nn = nnn;
  }
  cp_async_wait<0>();
  if (failed) {
    // Let every copy still in flight land before the CTA's shared memory goes away.
    const uint32_t issued = min(nchunks, q_rel + (uint32_t)S);
    for (uint32_t q = q_ready; q < issued; q++) warp_wait(&bars[q % S], (q / S) & 1);
    if (lane == 0) atomicExch(a.err, 1);
  }
}

template <typename TP, typename TD>
__global__ void hmvm_reduce_kernel(const int4* __restrict__ red, int n, const TP* __restrict__ p,
                                   TD* __restrict__ dst, const int* __restrict__ err) {
  griddep_launch_dependents();
  griddep_wait();
  if (checks_failed(err)) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int4 e = red[i];  // destination, first partial, parts, stride
    TP s = p[e.y];
    for (int c = 1; c < e.z; c++) s += p[e.y + c * e.w];
    dst[e.x] = (TD)s;
  }
}

// One stage's descriptors (HMVM_DEVICE_CHECKS builds): tiles [first, end)
// with their segments, output slots and row scales, the stage's reduction
// entries and its team ranges, checked against the lengths of the buffers they
// index (validate.hpp).  The kernel waits for its predecessors before it ends,
// so the stage launched after it stays ordered after them.
struct ValidateArgs {
  const hmvm_tile_desc* tiles;
  const hmvm_seg_desc* segs;
  const int32_t* out_idx;
  const int32_t* team_begin;
  const int4* red;
  int32_t nteams, first, end, n_red;
  LayoutCaps caps;
  int32_t vec, elem, stage1;
  int64_t zcap;
  int* err;
};
__global__ void hmvm_validate_kernel(ValidateArgs v) {
  griddep_launch_dependents();
  const int i = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  int rc = kCheckOk;
  for (int k = v.first + i; k < v.end && rc == kCheckOk; k += stride)
    rc = check_tile(v.tiles[k], v.segs, v.out_idx, v.caps, v.vec, v.elem, v.zcap, v.stage1 != 0);
  for (int k = i; k < v.n_red && rc == kCheckOk; k += stride)
    rc = check_red(reinterpret_cast<const int32_t*>(v.red + k), v.caps, v.stage1 != 0);
  if (i == 0 && rc == kCheckOk) rc = check_teams(v.team_begin, v.nteams, v.first, v.end);
  if (rc != kCheckOk) atomicCAS(v.err, 0, kErrDeviceCheck);
  griddep_wait();
}

// x rounded to FP32 once per HMVM (the inputs of the FP32 / FP16 / FP8 segments).
__global__ void hmvm_round_f32_kernel(const double* __restrict__ x, float* __restrict__ x32, int n) {
  griddep_launch_dependents();
  griddep_wait();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x32[i] = (float)x[i];
}

// ---- mixed precision ---------------------------------------------------------
// Segment element types (the top 4 bits of hmvm_seg_desc.ncols in mixed plans).
enum : int { kF64 = 0, kF32 = 1, kF16 = 2, kE4M3 = 3, kBF16 = 4 };
// log2 of a type's elements per 16-byte vector (2 FP64, 4 FP32, 8 FP16/BF16,
// 16 E4M3): whole vectors of a segment by shifts, not a division by a value
// the compiler cannot see is a power of two
__device__ __forceinline__ int mixed_vec_log2(int type) {
  return type == kF64 ? 1 : type == kF32 ? 2 : type == kE4M3 ? 4 : 3;
}

// Copy the inputs item `d` reads into zb: FP64 segments take x (8-byte
// elements), the others x rounded to FP32 or t (4-byte elements); every
// segment is padded with zeros to whole vectors.  d has at most 32 segments.
__device__ __forceinline__ void gather_inputs_mixed(const hmvm_tile_desc& d, const hmvm_seg_desc& sreg,
                                                    const double* __restrict__ x, const float* __restrict__ x32,
                                                    const float* __restrict__ tv, unsigned char* zb, int lane) {
  int zoff = 0;
  for (int j = 0; j < d.nseg; j++) {
    const int src = __shfl_sync(0xffffffffu, sreg.src, j);
    const int enc = __shfl_sync(0xffffffffu, sreg.ncols, j);
    const int type = enc >> 28, nc = enc & 0x0fffffff;
    const int lg = mixed_vec_log2(type);
    const int ncp = ((nc + (1 << lg) - 1) >> lg) << lg;
    if (type == kF64) {
      double* z = reinterpret_cast<double*>(zb + zoff);
      for (int c = lane; c < ncp; c += 32) {
        if (c < nc) cp_async<8>(z + c, x + src + c);
        else z[c] = 0.0;
      }
      zoff += ncp * 8;
    } else {
      float* z = reinterpret_cast<float*>(zb + zoff);
      const float* zs = src < 0 ? tv + (src & 0x7fffffff) : x32 + src;
      for (int c = lane; c < ncp; c += 32) {
        if (c < nc) cp_async<4>(z + c, zs + c);
        else z[c] = 0.0f;
      }
      zoff += ncp * 4;
    }
  }
}

__device__ __forceinline__ float2 h2f(uint32_t w) {
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
__device__ __forceinline__ float2 bf2f(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}
__device__ __forceinline__ float2 e4m3x2f(uint16_t w) {
  __half2_raw h = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)w, __NV_E4M3);
  return __half22float2(*reinterpret_cast<const __half2*>(&h));
}

template <int V>
struct TypeTag {
  static constexpr int value = V;
};
// Input bytes per 16-byte matrix vector: FP64 segments read x in FP64, the
// others x rounded to FP32 or t (FP32), one per stored element.
template <int TY>
struct MixedZ {
  static constexpr int bytes = TY == kF64 ? 16 : TY == kF32 ? 16 : TY == kE4M3 ? 64 : 32;
};
// Vectors per batch: 4 (2 for FP8, whose vectors carry 16 products), twice
// that when the launch leaves at least 216 registers per thread (WIDE: the
// 8-vector instances use up to 211); fewer
// when the ring cannot hold a batch of 32-row vectors beside the chunk being
// refilled.
template <int TY, int S, int CHUNK, bool VST, bool WIDE>
__host__ __device__ constexpr int mixed_batch() {
  constexpr int want = TY == kE4M3 ? (WIDE ? 4 : 2) : (WIDE ? 8 : 4);
  constexpr int room = (S - 1) * CHUNK / (32 * 16);
  return want <= room ? want : (room >= 4 ? 4 : (room >= 2 ? 2 : 1));
}

// acc += the products of one matrix vector m (element type TY) with its
// inputs at z.  Each of a vector's products goes to its own accumulator of
// acc[8] (FP32 vectors use half of them: the caller passes acc or acc + 4 by
// vector parity); FP64 vectors add to e[2].
// Two independent FP32 FMAs as one packed sm_100 instruction (fma.rn.f32x2):
// each lane rounds exactly as fmaf.
__device__ __forceinline__ void fma2(float& a0, float& a1, const float2 m, const float2 z) {
  const float2 r = __ffma2_rn(m, z, make_float2(a0, a1));
  a0 = r.x;
  a1 = r.y;
}
template <int TY>
__device__ __forceinline__ void mixed_fma(const uint4 m, const unsigned char* z, float* acc, double* e) {
  if constexpr (TY == kF64) {
    const double2 zz = *reinterpret_cast<const double2*>(z);
    e[0] = fma(__hiloint2double(m.y, m.x), zz.x, e[0]);
    e[1] = fma(__hiloint2double(m.w, m.z), zz.y, e[1]);
  } else if constexpr (TY == kF32) {
    const float4 zz = *reinterpret_cast<const float4*>(z);
    fma2(acc[0], acc[1], make_float2(__uint_as_float(m.x), __uint_as_float(m.y)), make_float2(zz.x, zz.y));
    fma2(acc[2], acc[3], make_float2(__uint_as_float(m.z), __uint_as_float(m.w)), make_float2(zz.z, zz.w));
  } else if constexpr (TY == kE4M3) {
    const float4* zz = reinterpret_cast<const float4*>(z);
    const uint32_t w[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float4 zi = zz[i];
      fma2(acc[2 * i], acc[2 * i + 1], e4m3x2f((uint16_t)w[i]), make_float2(zi.x, zi.y));
      fma2(acc[(2 * i + 4) & 7], acc[(2 * i + 5) & 7], e4m3x2f((uint16_t)(w[i] >> 16)), make_float2(zi.z, zi.w));
    }
  } else {
    const float4* zz = reinterpret_cast<const float4*>(z);
    const uint32_t w[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float4 zi = zz[i >> 1];
      const float2 zp = (i & 1) ? make_float2(zi.z, zi.w) : make_float2(zi.x, zi.y);
      fma2(acc[2 * i], acc[2 * i + 1], TY == kBF16 ? bf2f(w[i]) : h2f(w[i]), zp);
    }
  }
}

// hmvm_mixed_kernel<WPB, S, CHUNK, ZBYTES, LR16, VST>: the stream kernel's pipeline (TMA
// bulk ring for the matrix, cp.async-gathered inputs one item ahead) for
// mixed-precision plans, whose items hold segments of different element types
// (FP64, FP32, FP8 E4M3 and LR16 = the plan's 16-bit format, kF16 or kBF16).
// Each run of same-type segments is summed in FP32 (FP64 for FP64 segments)
// and added to the row's FP64 total.  VST: the V-stage instance, which
// multiplies a row's total by its column scale before storing t (FP32); the
// row-stage instance carries neither scales nor t slots.
template <int WPB, int S, int CHUNK, int ZBYTES>
__host__ __device__ constexpr int mixed_min_blocks() {
  constexpr int smem = WPB * (S * CHUNK + 2 * ZBYTES + S * 8);
  constexpr int by_smem = (227 * 1024) / smem;
  constexpr int by_warps = 24 / WPB;
  constexpr int m = by_smem < by_warps ? by_smem : by_warps;
  return m > 0 ? m : 1;
}

template <int WPB, int S, int CHUNK, int ZBYTES, int LR16, bool VST>
__global__ void __launch_bounds__(32 * WPB, (mixed_min_blocks<WPB, S, CHUNK, ZBYTES>()))
    hmvm_mixed_kernel(TileArgs a) {
  constexpr uint32_t RING = (uint32_t)S * CHUNK;
  static_assert((RING & (RING - 1)) == 0, "ring size must be a power of two");
  static_assert(CHUNK % 16 == 0 && CHUNK >= 512, "bulk copies move multiples of 16 bytes");
  constexpr bool WIDE = 65536 / (32 * WPB * mixed_min_blocks<WPB, S, CHUNK, ZBYTES>()) >= 216;
  static_assert(mixed_batch<kF32, S, CHUNK, VST, WIDE>() * 32 * 16 <= (S - 1) * CHUNK, "ring too small for one batch");
  extern __shared__ __align__(128) unsigned char smem[];
  griddep_launch_dependents();
  if (checks_failed(a.err)) return;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int team = blockIdx.x * WPB + warp;
  if (team >= a.nteams) return;
  const int tb = a.team_begin[team], te = a.team_begin[team + 1];
  if (tb >= te) return;
  unsigned char* ring = smem + (size_t)warp * RING;
  unsigned char* zbase = smem + (size_t)WPB * RING + (size_t)warp * 2 * ZBYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)WPB * RING + (size_t)WPB * 2 * ZBYTES) + warp * S;

  const hmvm_tile_desc* __restrict__ tiles = a.tiles;
  const hmvm_seg_desc* __restrict__ segs = a.segs;
  const double* __restrict__ x = static_cast<const double*>(a.x);
  const float* __restrict__ x32 = a.x32;
  const float* __restrict__ tv = static_cast<const float*>(a.t);
  const double* __restrict__ scl = a.scale;
  const hmvm_tile_desc dzero = {0, 0, 0, 0, 0, 1, 0, 0};
  const hmvm_seg_desc szero = {0, 0};

  hmvm_tile_desc cur = tiles[tb];
  const int64_t vbase = cur.data_off;
  const hmvm_tile_desc tl = tiles[te - 1];
  const int64_t total64 = (tl.data_off + (int64_t)tl.nvec * tl.nrows - vbase) * 16;
  if (total64 >= (int64_t)1 << 31) {
    if (lane == 0) atomicExch(a.err, 2);
    return;
  }
  const uint32_t total = (uint32_t)total64;
  const char* gsrc = static_cast<const char*>(a.data) + vbase * 16;
  const uint32_t nchunks = (total + CHUNK - 1) / CHUNK;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < S; s++) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  auto issue = [&](uint32_t q) {
    const uint32_t off = q * (uint32_t)CHUNK;
    const uint32_t bytes = min((uint32_t)CHUNK, total - off);
    uint64_t* bar = &bars[q % S];
    mbar_expect_tx(bar, bytes);
    bulk_g2s(ring + (q % S) * CHUNK, gsrc + off, bytes, bar);
  };
  if (lane == 0)
    for (uint32_t q = 0; q < min((uint32_t)S, nchunks); q++) issue(q);

  auto row_scale = [&](const hmvm_tile_desc& d) {
    if constexpr (VST) return lane < d.nrows ? scl[d._pad + lane] : 1.0;
    else return 1.0;
  };
  auto out_slot = [&](const hmvm_tile_desc& d) {
    if constexpr (VST) return (d.mode == 1 && lane < d.nrows) ? a.out_idx[d.out_base + lane] : 0;
    else return 0;
  };
  hmvm_seg_desc cur_seg = lane < cur.nseg ? segs[cur.seg_begin + lane] : szero;
  griddep_wait();  // as in hmvm_stream_kernel
  gather_inputs_mixed(cur, cur_seg, x, x32, tv, zbase, lane);
  cp_async_commit();
  int cur_oidx = out_slot(cur);
  double cur_scale = row_scale(cur);
  hmvm_tile_desc nxt = tb + 1 < te ? tiles[tb + 1] : dzero;
  hmvm_seg_desc nxt_seg = (tb + 1 < te && lane < nxt.nseg) ? segs[nxt.seg_begin + lane] : szero;
  int nxt_oidx = tb + 1 < te ? out_slot(nxt) : 0;
  double nxt_scale = tb + 1 < te ? row_scale(nxt) : 1.0;
  hmvm_tile_desc nn = tb + 2 < te ? tiles[tb + 2] : dzero;

  uint32_t q_ready = 0, q_rel = 0;
  bool failed = false;
  for (int ti = tb, k = 0; ti < te; ++ti, ++k) {
    unsigned char* zcur = zbase + (k & 1) * ZBYTES;
    __syncwarp();
    if (ti + 1 < te) gather_inputs_mixed(nxt, nxt_seg, x, x32, tv, zbase + ((k + 1) & 1) * ZBYTES, lane);
    cp_async_commit();
    const bool has_nn = ti + 2 < te;
    const hmvm_seg_desc nn_seg = (has_nn && lane < nn.nseg) ? segs[nn.seg_begin + lane] : szero;
    const int nn_oidx = has_nn ? out_slot(nn) : 0;
    const double nn_scale = has_nn ? row_scale(nn) : 1.0;
    const hmvm_tile_desc nnn = ti + 3 < te ? tiles[ti + 3] : dzero;
    cp_async_wait<1>();
    __syncwarp();

    const int R = cur.nrows;
    const uint32_t rstride = (uint32_t)R * 16;
    uint32_t o = (uint32_t)((cur.data_off - vbase) * 16);
    const uint32_t ol_lane = (uint32_t)lane * 16;
    double row = 0.0;
    int zoff = 0;
    // One segment of element type TY: batches of B vectors whose matrix and
    // input loads are issued together; FP32 (FP64) partial sums per segment.
    auto run_seg = [&](auto tag, const unsigned char* zs, int nv) -> bool {
      constexpr int TY = decltype(tag)::value;
      constexpr int B = mixed_batch<TY, S, CHUNK, VST, WIDE>();
      float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      double e[4] = {0.0, 0.0, 0.0, 0.0};
      for (int v = 0; v < nv; v += B) {
        const int nb = min(B, nv - v);
        const uint32_t o_end = o + (uint32_t)nb * rstride;
        if (o >= (q_rel + 1) * (uint32_t)CHUNK) {  // release the slots the warp has moved past
          const uint32_t qf = o / CHUNK;
          __syncwarp();
          if (lane == 0) {
            fence_proxy_async();
            for (uint32_t q = q_rel; q < qf; q++)
              if (q + S < nchunks) issue(q + S);
          }
          q_rel = qf;
        }
        if (o_end > q_ready * (uint32_t)CHUNK) {  // wait for the batch's chunks
          const uint32_t ql = (o_end - 1) / CHUNK;
          while (q_ready <= ql) {
            if (!warp_wait(&bars[q_ready % S], (q_ready / S) & 1)) return false;
            q_ready++;
          }
        }
        const uint32_t ol = o + ol_lane;
        const unsigned char* zv = zs + (size_t)v * MixedZ<TY>::bytes;
        // the last batch of a stretch is predicated (vectors past nb are
        // neither loaded nor used)
        uint4 m[B];
        if (nb == B) {  // a full batch: no predicates
#pragma unroll
          for (int u = 0; u < B; u++)
            m[u] = *reinterpret_cast<const uint4*>(ring + ((ol + (uint32_t)u * rstride) & (RING - 1)));
#pragma unroll
          for (int u = 0; u < B; u++)
            mixed_fma<TY>(m[u], zv + u * MixedZ<TY>::bytes, acc + (TY == kF32 ? (u & 1) * 4 : 0), e + (u & 1) * 2);
        } else {
#pragma unroll
          for (int u = 0; u < B; u++)
            if (u < nb) m[u] = *reinterpret_cast<const uint4*>(ring + ((ol + (uint32_t)u * rstride) & (RING - 1)));
#pragma unroll
          for (int u = 0; u < B; u++) {
            if (u < nb)
              mixed_fma<TY>(m[u], zv + u * MixedZ<TY>::bytes, acc + (TY == kF32 ? (u & 1) * 4 : 0), e + (u & 1) * 2);
          }
        }
        o = o_end;
      }
      row += ((e[0] + e[1]) + (e[2] + e[3])) +
             (double)(((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7])));
      return true;
    };
    // Segments come sorted by type: each run of one type is one stretch of
    // vectors (matrix and inputs both contiguous).  V-stage items are one
    // segment.
    int j = 0;
    while (j < (VST ? 1 : cur.nseg)) {
      const int type = __shfl_sync(0xffffffffu, cur_seg.ncols, j) >> 28;
      const int lg = mixed_vec_log2(type);
      const unsigned char* zs = zcur + zoff;
      int nv = 0;
      if constexpr (VST) {
        nv = cur.nvec;
        j = 1;
      } else {
        for (; j < cur.nseg; j++) {
          const int enc = __shfl_sync(0xffffffffu, cur_seg.ncols, j);
          if ((enc >> 28) != type) break;
          nv += ((enc & 0x0fffffff) + (1 << lg) - 1) >> lg;
        }
      }
      zoff += (nv << lg) * (type == kF64 ? 8 : 4);
      bool ok;
      switch (type) {
        case kF64: ok = run_seg(TypeTag<kF64>{}, zs, nv); break;
        case kF32: ok = run_seg(TypeTag<kF32>{}, zs, nv); break;
        case kE4M3: ok = run_seg(TypeTag<kE4M3>{}, zs, nv); break;
        default: ok = run_seg(TypeTag<LR16>{}, zs, nv); break;
      }
      if (!ok) {
        failed = true;
        break;
      }
    }
    if (failed) break;
    if (lane < R) {
      if constexpr (VST) {
        const double val = row * cur_scale;
        if (cur.mode == 1) const_cast<float*>(tv)[cur_oidx] = (float)val;
        else static_cast<double*>(a.p)[cur.out_base + lane] = val;
      } else {
        if (cur.mode == 0) static_cast<double*>(a.y)[cur.out_base + lane] = row;
        else static_cast<double*>(a.p)[cur.out_base + lane] = row;
      }
    }
    cur = nxt;
    cur_seg = nxt_seg;
    cur_oidx = nxt_oidx;
    cur_scale = nxt_scale;
    nxt = nn;
    nxt_seg = nn_seg;
    nxt_oidx = nn_oidx;
    nxt_scale = nn_scale;
    nn = nnn;
  }
  cp_async_wait<0>();
  if (failed) {
    const uint32_t issued = min(nchunks, q_rel + (uint32_t)S);
    for (uint32_t q = q_ready; q < issued; q++) warp_wait(&bars[q % S], (q / S) & 1);
    if (lane == 0) atomicExch(a.err, 1);
  }
}

}  // namespace hmvm
