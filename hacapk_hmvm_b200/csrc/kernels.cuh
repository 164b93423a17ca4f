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
// hmvm_reduce_kernel<T>: for column panels that were split into chunks, adds
// the chunk partial sums in chunk order and writes the t slot.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hmvm_b200.h"

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

template <typename T>
__global__ void hmvm_reduce_kernel(const int4* __restrict__ red, int n, const T* __restrict__ p,
                                   T* __restrict__ t) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int4 e = red[i];
    T s = p[e.y];
    for (int c = 1; c < e.z; c++) s += p[e.y + c * 32];
    t[e.x] = s;
  }
}

}  // namespace hmvm
