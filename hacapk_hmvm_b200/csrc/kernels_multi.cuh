// Multi-RHS HMVM on the CUDA cores: Y = H X for NR right-hand sides per pass
// (NR in {1, 2, 4, 8}), over the same planner layout as the single-vector
// kernels (hmvm_reduce_kernel / hmvm_stream_kernel / hmvm_mixed_kernel).
//
//   hmvm_pack_x_kernel      X (column-major, leading dimension ldx) -> the
//                           row-interleaved input xpk[i * NR + r] (FP64 and/or
//                           FP32 copies, zero rows past N), so that every
//                           segment's inputs are one contiguous block.
//   hmvm_multi_kernel       one warp per team, lane = row; the matrix streams
//                           through the warp's TMA ring exactly as in the
//                           single-vector kernels; each stored element is
//                           multiplied by its column's NR inputs.  V stage:
//                           t[slot * NR + r]; row stage: Y[row + r * ldy] or
//                           partial sums p[(base + lane) * NR + r].
//   hmvm_reduce_multi_kernel adds the partial sums of split tiles in part
//                           order, per right-hand side.
//
// MODE: kModePlain64 (FP64 plan), kModePlain32 (FP32 plan), kModeMixed16 /
// kModeMixedBF16 (mixed plan with FP16 / BF16 factors).  Element types per
// segment follow the plan: FP64 plans store FP64 only, FP32 plans FP32 only,
// mixed plans carry the type in the segment descriptor.  Inputs: FP64
// segments read the FP64 copy of x (or the FP64 t of FP64 plans), all others
// FP32 values.  Sums: FP32 per run of same-type segments (FP64 for FP64
// segments), FP64 per row.
#pragma once

#include "kernels.cuh"
#include "layout.hpp"

namespace hmvm {

enum : int { kModePlain64 = 0, kModePlain32 = 1, kModeMixed16 = 2, kModeMixedBF16 = 3 };

struct MultiArgs {
  int* err;
  const hmvm_tile_desc* tiles;
  const hmvm_seg_desc* segs;
  const int32_t* team_begin;
  int32_t nteams;
  const void* data;
  const double* x64;       // packed FP64 inputs [(N + pad) * NR]
  const float* x32;        // packed FP32 inputs [(N + pad) * NR]
  void* t;                 // [t_len * NR]: double (FP64 plans) or float
  void* y;                 // Y column r at y + r * ldy: double (FP64, mixed) or float (FP32)
  int64_t ldy;
  int32_t nr;              // columns of Y written (<= NR; inputs r >= nr are zero)
  void* p;                 // partial sums [(p_len) * NR]: double, or float for FP32 plans
  const int32_t* out_idx;  // V-stage output slots
  const double* scale;     // mixed, V stage: per panel-row column scale
  // elements of x64 / x32, t, p and y (checked by the batch instances only)
  int64_t xcap = 0, tcap = 0, pcap = 0, ycap = 0;
};

// X[i + r * ldx] -> xpk[i * NR + r] for i < n, r < nr; zeros for r >= nr and
// for the pad rows [n, n + pad).  Writes the FP64 copy if x64 != NULL and
// the FP32 copy if x32 != NULL.
template <typename TI, int NR>
__global__ void hmvm_pack_x_kernel(const TI* __restrict__ X, int64_t ldx, int n, int pad, int nr,
                                   double* __restrict__ x64, float* __restrict__ x32) {
  const int64_t total = (int64_t)(n + pad) * NR;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k / NR;
    const int r = (int)(k % NR);
    const double v = (i < n && r < nr) ? (double)X[i + r * ldx] : 0.0;
    if (x64) x64[k] = v;
    if (x32) x32[k] = (float)v;
  }
}

// red entries {dst, first partial, parts, stride}: for every rhs r < nr,
// dst[...] = sum over parts q of p[(first + q * stride) * NR + r].
// VST: dst is t (index dst * NR + r); else Y (index dst + r * ldy).
template <typename TP, typename TD, int NR, bool VST>
__global__ void hmvm_reduce_multi_kernel(const int4* __restrict__ red, int n, const TP* __restrict__ p,
                                         TD* __restrict__ dst, int64_t ldy, int nr) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)n * NR;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / NR), r = (int)(k % NR);
    const int4 e = red[i];
    TP s = TP(0);
    for (int q = 0; q < e.z; q++) s += p[(int64_t)(e.y + q * e.w) * NR + r];
    if (VST) dst[(int64_t)e.x * NR + r] = (TD)s;
    else if (r < nr) dst[e.x + r * ldy] = (TD)s;
  }
}

template <int MODE>
struct MultiMode {
  static constexpr bool mixed = MODE >= kModeMixed16;
  static constexpr int lr16 = MODE == kModeMixedBF16 ? kBF16 : kF16;
  using TT = typename std::conditional<MODE == kModePlain64, double, float>::type;  // t element
  using TY = typename std::conditional<MODE == kModePlain32, float, double>::type;  // y / p element
};

// Copy the inputs item `d` reads into zb: for each segment, ncp columns of
// NR values (ncp = columns rounded up to whole vectors; the padding is zero).
// FP64 segments take 8-byte values, the others 4-byte values.
template <int MODE, int NR, bool CHECK = false>
__device__ __forceinline__ void gather_multi(const hmvm_tile_desc& d, const hmvm_seg_desc& sreg, const MultiArgs& a,
                                             unsigned char* zb, int lane) {
  using TT = typename MultiMode<MODE>::TT;
  int zoff = 0;
  for (int j = 0; j < d.nseg; j++) {
    const int src = __shfl_sync(0xffffffffu, sreg.src, j);
    const int enc = __shfl_sync(0xffffffffu, sreg.ncols, j);
    const int type = MultiMode<MODE>::mixed ? (enc >> 28) : (MODE == kModePlain64 ? kF64 : kF32);
    const int nc = MultiMode<MODE>::mixed ? (enc & 0x0fffffff) : enc;
    const int lg = mixed_vec_log2(type);
    const int ncp = ((nc + (1 << lg) - 1) >> lg) << lg;
    const bool from_t = src < 0;
    const int64_t base = (int64_t)(from_t ? (src & 0x7fffffff) : src) * NR;
    if constexpr (CHECK) {  // a range outside its buffer: record it and read nothing
      if (base + (int64_t)ncp * NR > (from_t ? a.tcap : a.xcap)) {
        if (lane == 0) atomicExch(a.err, 3);
        for (int c = lane; c < ncp * NR * (type == kF64 ? 2 : 1); c += 32) reinterpret_cast<float*>(zb + zoff)[c] = 0.f;
        zoff += ncp * NR * (type == kF64 ? 8 : 4);
        continue;
      }
    }
    if (type == kF64) {
      const double* s = from_t ? reinterpret_cast<const double*>(static_cast<const TT*>(a.t)) + base : a.x64 + base;
      double* z = reinterpret_cast<double*>(zb + zoff);
      if constexpr (NR % 2 == 0) {  // 16-byte copies: (src * NR) is even
        for (int c = lane; c < ncp * NR / 2; c += 32) {
          if (c < nc * NR / 2) cp_async<16>(z + 2 * c, s + 2 * c);
          else *reinterpret_cast<double2*>(z + 2 * c) = make_double2(0.0, 0.0);
        }
      } else {
        for (int c = lane; c < ncp; c += 32) {
          if (c < nc) cp_async<8>(z + c, s + c);
          else z[c] = 0.0;
        }
      }
      zoff += ncp * NR * 8;
    } else {
      const float* s = from_t ? reinterpret_cast<const float*>(static_cast<const TT*>(a.t)) + base : a.x32 + base;
      float* z = reinterpret_cast<float*>(zb + zoff);
      if constexpr (NR % 4 == 0) {
        for (int c = lane; c < ncp * NR / 4; c += 32) {
          if (c < nc * NR / 4) cp_async<16>(z + 4 * c, s + 4 * c);
          else *reinterpret_cast<float4*>(z + 4 * c) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      } else if constexpr (NR == 2) {
        for (int c = lane; c < ncp; c += 32) {
          if (c < nc) cp_async<8>(z + 2 * c, s + 2 * c);
          else *reinterpret_cast<float2*>(z + 2 * c) = make_float2(0.f, 0.f);
        }
      } else {
        for (int c = lane; c < ncp; c += 32) {
          if (c < nc) cp_async<4>(z + c, s + c);
          else z[c] = 0.f;
        }
      }
      zoff += ncp * NR * 4;
    }
  }
}

// acc[r] += a * z[r] for the NR inputs of one column (FP32 z); pairs of
// right-hand sides as packed FP32 FMAs (fma2).
template <int NR>
__device__ __forceinline__ void axpy_f(float* acc, float a, const float* z) {
  const float2 aa = make_float2(a, a);
  if constexpr (NR >= 4) {
#pragma unroll
    for (int q = 0; q < NR / 4; q++) {
      const float4 zz = reinterpret_cast<const float4*>(z)[q];
      fma2(acc[4 * q + 0], acc[4 * q + 1], aa, make_float2(zz.x, zz.y));
      fma2(acc[4 * q + 2], acc[4 * q + 3], aa, make_float2(zz.z, zz.w));
    }
  } else if constexpr (NR == 2) {
    const float2 zz = *reinterpret_cast<const float2*>(z);
    fma2(acc[0], acc[1], aa, zz);
  } else {
    acc[0] = fmaf(a, z[0], acc[0]);
  }
}
template <int NR>
__device__ __forceinline__ void axpy_d(double* acc, double a, const double* z) {
  if constexpr (NR >= 2) {
#pragma unroll
    for (int q = 0; q < NR / 2; q++) {
      const double2 zz = reinterpret_cast<const double2*>(z)[q];
      acc[2 * q + 0] = fma(a, zz.x, acc[2 * q + 0]);
      acc[2 * q + 1] = fma(a, zz.y, acc[2 * q + 1]);
    }
  } else {
    acc[0] = fma(a, z[0], acc[0]);
  }
}

// The products of one 16-byte matrix vector m of type TY with its columns'
// inputs z (vs columns of NR values).
template <int TY, int NR>
__device__ __forceinline__ void multi_vec(const uint4 m, const unsigned char* z, float* fa, double* da) {
  if constexpr (TY == kF64) {
    const double* zz = reinterpret_cast<const double*>(z);
    axpy_d<NR>(da, __hiloint2double(m.y, m.x), zz);
    axpy_d<NR>(da, __hiloint2double(m.w, m.z), zz + NR);
  } else if constexpr (TY == kF32) {
    const float* zz = reinterpret_cast<const float*>(z);
    axpy_f<NR>(fa, __uint_as_float(m.x), zz);
    axpy_f<NR>(fa, __uint_as_float(m.y), zz + NR);
    axpy_f<NR>(fa, __uint_as_float(m.z), zz + 2 * NR);
    axpy_f<NR>(fa, __uint_as_float(m.w), zz + 3 * NR);
  } else if constexpr (TY == kE4M3) {
    const float* zz = reinterpret_cast<const float*>(z);
    const uint32_t w[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float2 lo = e4m3x2f((uint16_t)w[i]), hi = e4m3x2f((uint16_t)(w[i] >> 16));
      axpy_f<NR>(fa, lo.x, zz + (4 * i + 0) * NR);
      axpy_f<NR>(fa, lo.y, zz + (4 * i + 1) * NR);
      axpy_f<NR>(fa, hi.x, zz + (4 * i + 2) * NR);
      axpy_f<NR>(fa, hi.y, zz + (4 * i + 3) * NR);
    }
  } else {
    const float* zz = reinterpret_cast<const float*>(z);
    const uint32_t w[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const float2 v = TY == kBF16 ? bf2f(w[i]) : h2f(w[i]);
      axpy_f<NR>(fa, v.x, zz + (2 * i + 0) * NR);
      axpy_f<NR>(fa, v.y, zz + (2 * i + 1) * NR);
    }
  }
}

template <int WPB, int S, int CHUNK, int ZB>
constexpr int multi_min_blocks() {
  constexpr int smem = WPB * (S * CHUNK + 2 * ZB + S * 8);
  constexpr int by_smem = (227 * 1024) / smem;
  constexpr int by_warps = 16 / WPB;
  constexpr int m = by_smem < by_warps ? by_smem : by_warps;
  return m > 0 ? m : 1;
}

// The body of hmvm_multi_kernel for block bid of the launch (a batch launch
// runs several plans' bodies, each over its own range of blocks).
template <int WPB, int S, int CHUNK, int NR, int MODE, bool VST, bool CHECK = false>
__device__ __forceinline__ void multi_body(const MultiArgs& a, int bid) {
  using MM = MultiMode<MODE>;
  using TT = typename MM::TT;
  using TYO = typename MM::TY;
  constexpr uint32_t RING = (uint32_t)S * CHUNK;
  constexpr int ZB = MODE == kModePlain64 ? kMultiZBytesF64 : kMultiZBytes;  // each of the two input buffers
  constexpr int B = 2;  // vectors per batch: each carries 2..16 columns of NR products
  static_assert((RING & (RING - 1)) == 0, "ring size must be a power of two");
  static_assert(CHUNK % 16 == 0 && CHUNK >= 512, "bulk copies move multiples of 16 bytes");
  static_assert(B * 32 * 16 <= (S - 1) * CHUNK, "ring too small for one batch");
  extern __shared__ __align__(128) unsigned char smem[];

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int team = bid * WPB + warp;
  if (team >= a.nteams) return;
  const int tb = a.team_begin[team], te = a.team_begin[team + 1];
  if (tb >= te) return;
  unsigned char* ring = smem + (size_t)warp * RING;
  unsigned char* zbase = smem + (size_t)WPB * RING + (size_t)warp * 2 * ZB;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)WPB * RING + (size_t)WPB * 2 * ZB) + warp * S;

  const hmvm_tile_desc* __restrict__ tiles = a.tiles;
  const hmvm_seg_desc* __restrict__ segs = a.segs;
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
    if constexpr (VST && MM::mixed) return lane < d.nrows ? a.scale[d._pad + lane] : 1.0;
    else return 1.0;
  };
  auto out_slot = [&](const hmvm_tile_desc& d) {
    if constexpr (VST) return (d.mode == 1 && lane < d.nrows) ? a.out_idx[d.out_base + lane] : 0;
    else return 0;
  };
  hmvm_seg_desc cur_seg = lane < cur.nseg ? segs[cur.seg_begin + lane] : szero;
  gather_multi<MODE, NR, CHECK>(cur, cur_seg, a, zbase, lane);
  cp_async_commit();
  int cur_oidx = out_slot(cur);
  double cur_scale = row_scale(cur);
  hmvm_tile_desc nxt = tb + 1 < te ? tiles[tb + 1] : dzero;
  hmvm_seg_desc nxt_seg = (tb + 1 < te && lane < nxt.nseg) ? segs[nxt.seg_begin + lane] : szero;

  uint32_t q_ready = 0, q_rel = 0;
  bool failed = false;
  for (int ti = tb, k = 0; ti < te; ++ti, ++k) {
    unsigned char* zcur = zbase + (k & 1) * ZB;
    __syncwarp();
    if (ti + 1 < te) gather_multi<MODE, NR, CHECK>(nxt, nxt_seg, a, zbase + ((k + 1) & 1) * ZB, lane);
    cp_async_commit();
    const bool has_nn = ti + 2 < te;
    const hmvm_tile_desc nn = has_nn ? tiles[ti + 2] : dzero;
    const int nxt_oidx = ti + 1 < te ? out_slot(nxt) : 0;
    const double nxt_scale = ti + 1 < te ? row_scale(nxt) : 1.0;
    cp_async_wait<1>();
    __syncwarp();

    const int R = cur.nrows;
    const uint32_t rstride = (uint32_t)R * 16;
    uint32_t o = (uint32_t)((cur.data_off - vbase) * 16);
    const uint32_t ol_lane = (uint32_t)lane * 16;
    double row[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) row[r] = 0.0;
    int zoff = 0;
    auto run_seg = [&](auto tag, const unsigned char* zs, int nv) -> bool {
      constexpr int TY = decltype(tag)::value;
      constexpr int VS = TY == kF64 ? 2 : TY == kF32 ? 4 : TY == kE4M3 ? 16 : 8;
      constexpr int ZV = VS * NR * (TY == kF64 ? 8 : 4);  // input bytes per vector
      float fa[NR];
      double da[NR];
#pragma unroll
      for (int r = 0; r < NR; r++) {
        fa[r] = 0.f;
        da[r] = 0.0;
      }
      for (int v = 0; v < nv; v += B) {
        const int nb = min(B, nv - v);
        const uint32_t o_end = o + (uint32_t)nb * rstride;
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
            if (!warp_wait(&bars[q_ready % S], (q_ready / S) & 1)) return false;
            q_ready++;
          }
        }
        const uint32_t ol = o + ol_lane;
        uint4 m[B];
#pragma unroll
        for (int u = 0; u < B; u++)
          if (u < nb) m[u] = *reinterpret_cast<const uint4*>(ring + ((ol + (uint32_t)u * rstride) & (RING - 1)));
#pragma unroll
        for (int u = 0; u < B; u++)
          if (u < nb) multi_vec<TY, NR>(m[u], zs + (size_t)(v + u) * ZV, fa, da);
        o = o_end;
      }
#pragma unroll
      for (int r = 0; r < NR; r++) row[r] += da[r] + (double)fa[r];
      return true;
    };
    int j = 0;
    while (j < (VST ? 1 : cur.nseg)) {
      const int enc0 = __shfl_sync(0xffffffffu, cur_seg.ncols, j);
      const int type = MM::mixed ? (enc0 >> 28) : (MODE == kModePlain64 ? kF64 : kF32);
      const int lg = mixed_vec_log2(type);
      const unsigned char* zs = zcur + zoff;
      int nv = 0;
      if (VST) {
        nv = cur.nvec;
        j = 1;
      } else {
        for (; j < cur.nseg; j++) {
          const int enc = __shfl_sync(0xffffffffu, cur_seg.ncols, j);
          if (MM::mixed && (enc >> 28) != type) break;
          nv += ((MM::mixed ? (enc & 0x0fffffff) : enc) + (1 << lg) - 1) >> lg;
        }
      }
      zoff += (nv << lg) * NR * (type == kF64 ? 8 : 4);
      bool ok;
      if constexpr (MODE == kModePlain64) {
        ok = run_seg(TypeTag<kF64>{}, zs, nv);
      } else if constexpr (MODE == kModePlain32) {
        ok = run_seg(TypeTag<kF32>{}, zs, nv);
      } else {
        switch (type) {
          case kF64: ok = run_seg(TypeTag<kF64>{}, zs, nv); break;
          case kF32: ok = run_seg(TypeTag<kF32>{}, zs, nv); break;
          case kE4M3: ok = run_seg(TypeTag<kE4M3>{}, zs, nv); break;
          default: ok = run_seg(TypeTag<MM::lr16>{}, zs, nv); break;
        }
      }
      if (!ok) {
        failed = true;
        break;
      }
    }
    if (failed) break;
    bool store_ok = true;
    if constexpr (CHECK) {  // an output outside its buffer: record it and write nothing
      const int64_t hi = VST ? (cur.mode == 1 ? ((int64_t)cur_oidx + 1) * NR : ((int64_t)cur.out_base + R) * NR)
                             : (cur.mode == 0 ? (int64_t)cur.out_base + R + (int64_t)(NR - 1) * a.ldy
                                              : ((int64_t)cur.out_base + R) * NR);
      const int64_t cap = VST ? (cur.mode == 1 ? a.tcap : a.pcap) : (cur.mode == 0 ? a.ycap : a.pcap);
      store_ok = cur_oidx >= 0 && cur.out_base >= 0 && hi <= cap;
      if (!store_ok && lane == 0) atomicExch(a.err, 3);
    }
    if (lane < R && store_ok) {
      if constexpr (VST) {
        if (cur.mode == 1) {
#pragma unroll
          for (int r = 0; r < NR; r++)
            static_cast<TT*>(a.t)[(int64_t)cur_oidx * NR + r] = (TT)(row[r] * cur_scale);
        } else {
#pragma unroll
          for (int r = 0; r < NR; r++)
            static_cast<TYO*>(a.p)[(int64_t)(cur.out_base + lane) * NR + r] = (TYO)(row[r] * cur_scale);
        }
      } else {
        if (cur.mode == 0) {
#pragma unroll
          for (int r = 0; r < NR; r++)
            if (r < a.nr) static_cast<TYO*>(a.y)[cur.out_base + lane + r * a.ldy] = (TYO)row[r];
        } else {
#pragma unroll
          for (int r = 0; r < NR; r++)
            static_cast<TYO*>(a.p)[(int64_t)(cur.out_base + lane) * NR + r] = (TYO)row[r];
        }
      }
    }
    cur = nxt;
    cur_seg = nxt_seg;
    cur_oidx = nxt_oidx;
    cur_scale = nxt_scale;
    nxt = nn;
    nxt_seg = (has_nn && lane < nn.nseg) ? segs[nn.seg_begin + lane] : szero;
  }
  cp_async_wait<0>();
  if (failed) {
    const uint32_t issued = min(nchunks, q_rel + (uint32_t)S);
    for (uint32_t q = q_ready; q < issued; q++) warp_wait(&bars[q % S], (q / S) & 1);
    if (lane == 0) atomicExch(a.err, 1);
  }
}

template <int WPB, int S, int CHUNK, int NR, int MODE, bool VST>
__global__ void __launch_bounds__(
    32 * WPB, (multi_min_blocks<WPB, S, CHUNK, (MODE == kModePlain64 ? kMultiZBytesF64 : kMultiZBytes)>()))
    hmvm_multi_kernel(MultiArgs a) {
  multi_body<WPB, S, CHUNK, NR, MODE, VST>(a, (int)blockIdx.x);
}

// ---- batches of independent H-matrices ----------------------------------------
// A batch runs as one block-diagonal H-matrix over the concatenated index
// space; instance m owns rows [off, off + n).  These kernels move each
// instance's vectors between its own buffers and the concatenated ones
// (blockIdx.y = instance).
struct BatchIO {
  const void* X;  // column c at X + c * ldx
  int64_t ldx;
  void* Y;
  int64_t ldy;
  int64_t off;
  int32_t n, nrhs;
};

// Column c of every instance -> xcat[off + i] (zero where c >= nrhs).
template <typename T>
__global__ void hmvm_batch_pack1_kernel(const BatchIO* __restrict__ io, int c, T* __restrict__ xcat) {
  const BatchIO b = io[blockIdx.y];
  const T* X = static_cast<const T*>(b.X);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x)
    xcat[b.off + i] = c < b.nrhs ? X[i + c * b.ldx] : T(0);
}
// Columns [c0, c0 + NR) -> the row-interleaved packed inputs (zero past nrhs).
template <typename TI, int NR>
__global__ void hmvm_batch_packm_kernel(const BatchIO* __restrict__ io, int c0, double* __restrict__ x64,
                                        float* __restrict__ x32) {
  const BatchIO b = io[blockIdx.y];
  const TI* X = static_cast<const TI*>(b.X);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)b.n * NR;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k / NR;
    const int r = (int)(k % NR);
    const double v = c0 + r < b.nrhs ? (double)X[i + (int64_t)(c0 + r) * b.ldx] : 0.0;
    const int64_t dst = (b.off + i) * NR + r;
    if (x64) x64[dst] = v;
    if (x32) x32[dst] = (float)v;
  }
}
// ycat (column r at ycat + r * ldc) -> Y[:, c0 + r] for r < w, c0 + r < nrhs.
template <typename T>
__global__ void hmvm_batch_unpack_kernel(const BatchIO* __restrict__ io, int c0, int w, const T* __restrict__ ycat,
                                         int64_t ldc) {
  const BatchIO b = io[blockIdx.y];
  T* Y = static_cast<T*>(b.Y);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)b.n * w;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / b.n);
    const int64_t i = k % b.n;
    if (c0 + r < b.nrhs) Y[i + (int64_t)(c0 + r) * b.ldy] = ycat[b.off + i + r * ldc];
  }
}

// ---- a whole batch in one launch per stage --------------------------------------
// A batch is planned as block-diagonal classes (one plan per pass width), and an
// apply runs each class's passes; every (class, pass) -- a "part" -- has its own
// packed inputs, t, partial sums and concatenated outputs, so all parts run at
// once: each of these kernels reads the batch's part table (global memory) and
// cuts its blocks (or work items) into per-part ranges.  Every buffer access of
// a part is checked against the part's capacities (a miss records error 3 and
// is skipped).
struct BatchPart {
  MultiArgs a;
  int32_t cta0;  // first block of the part in its stage launch
  int32_t nr;    // pass width: 2, 4 or 8
};
template <int WPB, int S, int CHUNK, int MODE, bool VST>
__global__ void __launch_bounds__(
    32 * WPB, (multi_min_blocks<WPB, S, CHUNK, (MODE == kModePlain64 ? kMultiZBytesF64 : kMultiZBytes)>()))
    hmvm_batch_multi_kernel(const BatchPart* __restrict__ parts, int nparts) {
  int k = 0;
  while (k + 1 < nparts && (int)blockIdx.x >= parts[k + 1].cta0) k++;
  const MultiArgs a = parts[k].a;
  const int bid = (int)blockIdx.x - parts[k].cta0;
  switch (parts[k].nr) {
    case 2: multi_body<WPB, S, CHUNK, 2, MODE, VST, true>(a, bid); break;
    case 4: multi_body<WPB, S, CHUNK, 4, MODE, VST, true>(a, bid); break;
    default: multi_body<WPB, S, CHUNK, 8, MODE, VST, true>(a, bid); break;
  }
}

// The split-tile reductions of every part (hmvm_reduce_multi_kernel's sums, with
// each part's width): work items [w0, w0 + n * nr) are the part's.
struct BatchRedPart {
  const int4* red;
  const void* p;
  void* dst;
  int64_t ldy;
  int64_t w0;
  int64_t pcap, dcap;  // elements of p and dst
  int32_t n, nr;
};
template <typename TP, typename TD, bool VST>
__global__ void hmvm_batch_reduce_kernel(const BatchRedPart* __restrict__ parts, int nparts, int64_t total,
                                         int* err) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    int q = 0;
    while (q + 1 < nparts && k >= parts[q + 1].w0) q++;
    const BatchRedPart& P = parts[q];
    const int NR = P.nr;
    const int64_t l = k - P.w0;
    const int i = (int)(l / NR), r = (int)(l % NR);
    const int4 e = P.red[i];
    const int64_t last = (int64_t)(e.y + (e.z - 1) * e.w) * NR + r;
    const int64_t d = VST ? (int64_t)e.x * NR + r : (int64_t)e.x + (int64_t)r * P.ldy;
    if (e.y < 0 || e.z < 0 || last >= P.pcap || d < 0 || d >= P.dcap) {
      atomicExch(err, 3);
      continue;
    }
    const TP* p = static_cast<const TP*>(P.p);
    TP sum = TP(0);
    for (int u = 0; u < e.z; u++) sum += p[(int64_t)(e.y + u * e.w) * NR + r];
    static_cast<TD*>(P.dst)[d] = (TD)sum;
  }
}

// One row of the pack / unpack grids (blockIdx.y): an instance in one part.
struct BatchPack {
  int32_t io;       // the instance (index into the batch's BatchIO table)
  int32_t c0;       // first column of the part's pass
  int32_t nr;       // pass width
  int32_t _pad;
  double* x64;      // the part's packed inputs (row-interleaved, nr per row)
  float* x32;
  void* ycat;       // the part's concatenated outputs, column r at ycat + r * ldc
  int64_t ldc;
  int64_t xcap, ycap;  // elements of the packed inputs and of ycat
};
// Columns [c0, c0 + nr) of each instance -> its part's packed inputs (zero past nrhs).
template <typename TI>
__global__ void hmvm_batch_pack_kernel(const BatchIO* __restrict__ io, int nio, const BatchPack* __restrict__ e,
                                       int* err) {
  const BatchPack q = e[blockIdx.y];
  if (q.io < 0 || q.io >= nio) {
    if (threadIdx.x == 0) atomicExch(err, 3);
    return;
  }
  const BatchIO b = io[q.io];
  if (b.off < 0 || (b.off + b.n) * q.nr > q.xcap) {
    if (threadIdx.x == 0) atomicExch(err, 3);
    return;
  }
  const TI* X = static_cast<const TI*>(b.X);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)b.n * q.nr;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k / q.nr;
    const int r = (int)(k % q.nr);
    const double v = q.c0 + r < b.nrhs ? (double)X[i + (int64_t)(q.c0 + r) * b.ldx] : 0.0;
    const int64_t dst = (b.off + i) * q.nr + r;
    if (q.x64) q.x64[dst] = v;
    if (q.x32) q.x32[dst] = (float)v;
  }
}
// Each instance's columns of its part's concatenated outputs -> its own Y.
template <typename T>
__global__ void hmvm_batch_unpack_parts_kernel(const BatchIO* __restrict__ io, int nio,
                                               const BatchPack* __restrict__ e, int* err) {
  const BatchPack q = e[blockIdx.y];
  if (q.io < 0 || q.io >= nio) {
    if (threadIdx.x == 0) atomicExch(err, 3);
    return;
  }
  const BatchIO b = io[q.io];
  if (b.off < 0 || b.off + b.n + (int64_t)(q.nr - 1) * q.ldc > q.ycap) {
    if (threadIdx.x == 0) atomicExch(err, 3);
    return;
  }
  T* Y = static_cast<T*>(b.Y);
  const T* yc = static_cast<const T*>(q.ycat);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)b.n * q.nr;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k / b.n);
    const int64_t i = k % b.n;
    if (q.c0 + r < b.nrhs) Y[i + (int64_t)(q.c0 + r) * b.ldy] = yc[b.off + i + r * q.ldc];
  }
}

}  // namespace hmvm
