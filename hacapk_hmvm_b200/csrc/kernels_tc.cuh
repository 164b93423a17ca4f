// Multi-RHS HMVM with the 16-bit low-rank factor runs on the 5th-generation
// tensor cores (tcgen05), 16 right-hand sides per pass, for mixed-precision
// plans (FP16 or BF16 factors).
//
// Per item (one warp, lane = row, the matrix streaming through the warp's TMA
// ring exactly as in the other kernels):
//   * FP64 / FP32 / FP8 runs: CUDA cores, 16 FP32 (FP64) accumulators per lane.
//   * the FP16/BF16 run (segments are sorted by type, so an item has at most
//     one): each lane copies its row's 16-byte vectors from the ring into a
//     linear staging tile (K-major canonical layout: 8 rows x 16 B core
//     matrices, 512 B per 16-byte column chunk), then lane 0 issues
//     tcgen05.mma.cta_group::1.kind::f16 with M = 128, N = 32, K = 16:
//       A = the staging tile (the warp's 32 rows sit at M rows 32q..32q+31,
//           q = warp % 4, so that the accumulator rows land in the TMEM lanes
//           this warp may read),
//       B = the run's inputs as 16-bit hi/lo pairs (N = 16 hi + 16 lo
//           columns) in MN-major canonical layout, gathered from planes made
//           once per pass (hmvm_tc_planes_kernel), each right-hand side scaled
//           by its own power of two,
//       D = FP32 in the warp's own 32 TMEM columns, accumulated over the run;
//     tcgen05.commit signals an mbarrier; at the end of the item the warp reads
//     its rows with tcgen05.ld.32x32b.x32 and adds (hi + lo) * 2^e_r per rhs r.
//   Every wait (ring, MMA commit) is bounded; a warp that gives up records
//   the error, and the CTA frees its TMEM before it exits.
#pragma once

#include <cuda_bf16.h>

#include "kernels_multi.cuh"

namespace hmvm {

constexpr int kTcNr = 16;             // right-hand sides per tensor-core pass
constexpr int kTcN = 2 * kTcNr;       // MMA N: hi and lo parts
constexpr int kTcPiece = 8;           // 16-byte column chunks staged per MMA batch (4 K-steps)
// input buffer per item (x2, double-buffered): the planner's budget for 16
// right-hand sides (8 KiB) plus the 16-bit planes' padding to 16 rows (< 1 KiB)
constexpr int kTcZBytes = 9216;
constexpr int kTcStageBytes = kTcPiece * 32 * 16;  // 4 KiB A staging per warp
constexpr int kTcPad = 2048;          // slack before the staging tiles (M rows below 32q)

// ---- global inputs as 16-bit hi/lo planes -----------------------------------
// amax[r] = max |v| of right-hand side r (values v[i * 16 + r]) as float bits
// (atomicMax on the non-negative bit pattern).  The grid stride is a multiple
// of 16, so each thread always reads the same column r = threadIdx.x % 16.
__global__ void hmvm_absmax_kernel(const float* __restrict__ v, int64_t n, unsigned* __restrict__ amax) {
  float m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(v[i]));
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));  // lanes l and l + 16 hold the same column
  if ((threadIdx.x & 31) < 16 && m > 0.f) atomicMax(amax + (threadIdx.x & 15), __float_as_uint(m));
}

// A power-of-two scale s = 2^-e with max |v| * s in [2^13, 2^14) (1 if max = 0
// or not finite), and its inverse.
__device__ __forceinline__ void tc_scale(unsigned amax_bits, float* s, float* inv) {
  const float m = __uint_as_float(amax_bits);
  if (!(m > 0.f) || !isfinite(m)) {
    *s = 1.f;
    *inv = 1.f;
    return;
  }
  int e;
  frexpf(m, &e);  // m = f * 2^e, f in [0.5, 1)
  *s = ldexpf(1.f, 14 - e);
  *inv = ldexpf(1.f, e - 14);
}

// src: rows [0, n) of 16 FP32 values (row-interleaved, src[i * 16 + r]);
// planes: 4 planes of (n + pad) rows x 8 16-bit values: plane g, row i holds
// hi (g < 2) or lo (g >= 2) parts of rhs 8 * (g % 2) .. + 7, each column r
// scaled by its own power of two s_r (from amax[r]).  Rows [n, n + pad) are
// zero.  scal[r] = s_r, scal[16 + r] = 1 / s_r.
template <bool BF>
__global__ void hmvm_tc_planes_kernel(const float* __restrict__ src, int n, int pad, const unsigned* __restrict__ amax,
                                      uint16_t* __restrict__ planes, float* __restrict__ scal) {
  const int r = threadIdx.x & 15;  // the grid stride is a multiple of 16: a fixed column per thread
  float s, inv;
  tc_scale(amax[r], &s, &inv);
  if (blockIdx.x == 0 && threadIdx.x < 16) {
    scal[r] = s;
    scal[16 + r] = inv;
  }
  const int64_t rows = (int64_t)n + pad;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < rows * kTcNr;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = k / kTcNr;
    const float v = i < n ? src[k] * s : 0.f;
    uint16_t hi, lo;
    if (BF) {
      const __nv_bfloat16 h = __float2bfloat16_rn(v);
      const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
      hi = *reinterpret_cast<const uint16_t*>(&h);
      lo = *reinterpret_cast<const uint16_t*>(&l);
    } else {
      const __half h = __float2half_rn(v);
      const __half l = __float2half_rn(v - __half2float(h));
      hi = *reinterpret_cast<const uint16_t*>(&h);
      lo = *reinterpret_cast<const uint16_t*>(&l);
    }
    const int g = r >> 3, j = r & 7;
    planes[((int64_t)g * rows + i) * 8 + j] = hi;
    planes[((int64_t)(g + 2) * rows + i) * 8 + j] = lo;
  }
}

// ---- tcgen05 helpers -----------------------------------------------------------
// Shared-memory matrix descriptor, no swizzle (canonical INTERLEAVE layouts):
// start address, leading-dimension and stride-dimension byte offsets (all
// multiples of 16), descriptor version 1.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor, kind::f16: D FP32, A and B both FP16 (bf = 0) or
// both BF16 (bf = 1), A K-major, B MN-major, N and M as given.
__host__ __device__ constexpr uint32_t tc_idesc(int bf, int m, int n) {
  return (1u << 4) | ((uint32_t)bf << 7) | ((uint32_t)bf << 10) | (0u << 15) | (1u << 16) |
         ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

struct TcArgs {
  MultiArgs m;               // NR = 16 buffers (x64, x32, t, y, p, ...)
  const uint16_t* xplanes;   // 4 planes of (N + 16) rows (stage 1 inputs of 16-bit runs)
  const uint16_t* tplanes;   // 4 planes of (t_len + 16) rows (stage 2 inputs of 16-bit runs)
  int64_t xrows, trows;      // rows per plane
  const float* scal;         // [16..31] x column scales' inverses, [48..63] t column scales' inverses
};

__device__ __forceinline__ int tc_seg_type(int enc) { return enc >> 28; }

template <int WPB, int S, int CHUNK>
constexpr int tc_smem_bytes() {
  return WPB * (S * CHUNK + 2 * kTcZBytes + kTcStageBytes) + kTcPad + 2048 + WPB * (S + 3) * 8 + 16;
}

template <int WPB, int S, int CHUNK, int MODE, bool VST>
__global__ void __launch_bounds__(32 * WPB, 1) hmvm_tc_kernel(TcArgs ta) {
  using MM = MultiMode<MODE>;
  constexpr int NR = kTcNr;
  constexpr uint32_t RING = (uint32_t)S * CHUNK;
  constexpr int B = 2;
  constexpr int LR = MM::lr16;
  constexpr uint32_t IDESC = tc_idesc(MODE == kModeMixedBF16 ? 1 : 0, 128, kTcN);
  static_assert(MM::mixed, "tensor-core passes serve mixed plans");
  static_assert((RING & (RING - 1)) == 0, "ring size must be a power of two");
  static_assert(B * 32 * 16 <= (S - 1) * CHUNK, "ring too small for one batch");
  constexpr int TMEM_COLS = WPB * kTcN <= 32 ? 32 : WPB * kTcN <= 64 ? 64 : WPB * kTcN <= 128 ? 128 : 256;
  static_assert(WPB * kTcN <= 256, "TMEM columns");
  extern __shared__ __align__(1024) unsigned char tc_smem_base[];
  unsigned char* smem = tc_smem_base;
  const MultiArgs& a = ta.m;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int team = blockIdx.x * WPB + warp;
  // layout: [kTcPad][staging x WPB][rings x WPB][z x 2 x WPB][2048 tail][bars][tmem addr]
  unsigned char* stage = smem + kTcPad + (size_t)warp * kTcStageBytes;
  unsigned char* ring = smem + kTcPad + (size_t)WPB * kTcStageBytes + (size_t)warp * RING;
  unsigned char* zbase = smem + kTcPad + (size_t)WPB * (kTcStageBytes + RING) + (size_t)warp * 2 * kTcZBytes;
  uint64_t* bars_all =
      reinterpret_cast<uint64_t*>(smem + kTcPad + (size_t)WPB * (kTcStageBytes + RING + 2 * kTcZBytes) + 2048);
  uint64_t* bars = bars_all + warp * (S + 3);
  uint64_t* mbar = bars + S;      // MMA completion
  uint64_t* zbars = bars + S + 1;  // input buffers 0 and 1 (bulk-copy completion)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars_all + WPB * (S + 3));

  // TMEM: warp 0 allocates for the CTA
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int quad = warp & 3;
  const uint32_t dcol = tmem_base + (uint32_t)(warp * kTcN);   // this warp's D columns (lane field 0)
  const uint32_t dread = dcol + ((uint32_t)(32 * quad) << 16);  // its lanes 32q..32q+31

  bool failed = false;
  const bool active = team < a.nteams && a.team_begin[team] < a.team_begin[team + 1];
  uint32_t q_ready = 0, q_rel = 0, nchunks = 0, mma_phase = 0;
  bool mma_open = false;  // a commit not yet waited for
  if (active) {
    const int tb = a.team_begin[team], te = a.team_begin[team + 1];
    const hmvm_tile_desc* __restrict__ tiles = a.tiles;
    const hmvm_seg_desc* __restrict__ segs = a.segs;
    const hmvm_tile_desc dzero = {0, 0, 0, 0, 0, 1, 0, 0};
    const hmvm_seg_desc szero = {0, 0};
    const uint16_t* __restrict__ planes = VST ? ta.xplanes : ta.tplanes;
    const int64_t prows = VST ? ta.xrows : ta.trows;
    const float* pscale_inv = ta.scal + (VST ? 16 : 48);

    hmvm_tile_desc cur = tiles[tb];
    const int64_t vbase = cur.data_off;
    const hmvm_tile_desc tl = tiles[te - 1];
    const int64_t total64 = (tl.data_off + (int64_t)tl.nvec * tl.nrows - vbase) * 16;
    if (total64 >= (int64_t)1 << 31) {
      if (lane == 0) atomicExch(a.err, 2);
      failed = true;
    }
    const uint32_t total = (uint32_t)total64;
    const char* gsrc = static_cast<const char*>(a.data) + vbase * 16;
    nchunks = failed ? 0 : (total + CHUNK - 1) / CHUNK;
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < S + 3; s++) mbar_init(&bars[s], 1);
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

    // inputs of one item: 16-bit segments go to the front of the buffer as
    // four planes of K16 rows (K16 = the run's columns, rounded up to 16);
    // the other segments follow, in order, as ncp columns x 16 values.  Lane j
    // takes segment j: its rows (plane slices, or input rows of 16 values) are
    // contiguous in global memory, so each is one TMA bulk copy completing on
    // the buffer's mbarrier (lane 0 posts the item's byte count); the padding
    // is written with plain stores.
    auto gather = [&](const hmvm_tile_desc& d, const hmvm_seg_desc& sreg, unsigned char* zb, uint64_t* zbar,
                      int* k16_out) {
      const bool has = lane < d.nseg;
      const int type = has ? tc_seg_type(sreg.ncols) : -1;
      const int nc = has ? (sreg.ncols & 0x0fffffff) : 0;
      const int lg = has ? mixed_vec_log2(type) : 0;
      const int ncp = ((nc + (1 << lg) - 1) >> lg) << lg;
      const bool lr = has && type == LR;
      const int es = type == kF64 ? 8 : 4;
      const int lr_rows = lr ? ncp : 0;
      const int zb_bytes = (has && !lr) ? ncp * NR * es : 0;
      int koff = lr_rows, zo = zb_bytes;  // inclusive scans, then made exclusive
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int k2 = __shfl_up_sync(0xffffffffu, koff, o), z2 = __shfl_up_sync(0xffffffffu, zo, o);
        if (lane >= o) {
          koff += k2;
          zo += z2;
        }
      }
      const int k16 = __shfl_sync(0xffffffffu, koff, 31);
      koff -= lr_rows;
      zo -= zb_bytes;
      const int k16p = (k16 + 15) / 16 * 16;
      *k16_out = k16p;
      const int zoff = 4 * k16p * 16 + zo;
      const uint32_t tx = lr ? 4u * nc * 16 : (has ? (uint32_t)nc * NR * es : 0u);
      uint32_t tx_all = tx;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tx_all += __shfl_xor_sync(0xffffffffu, tx_all, o);
      fence_proxy_async();  // this buffer's earlier generic reads and stores before the async writes
      __syncwarp();
      if (lane == 0) mbar_expect_tx(zbar, tx_all);
      __syncwarp();
      const int64_t row0 = sreg.src < 0 ? (sreg.src & 0x7fffffff) : sreg.src;
      if (lr) {
        for (int g = 0; g < 4; g++) {
          unsigned char* dst = zb + ((size_t)g * k16p + koff) * 16;
          if (nc > 0) bulk_g2s(dst, planes + ((int64_t)g * prows + row0) * 8, (uint32_t)nc * 16, zbar);
          for (int r = nc; r < ncp; r++) *reinterpret_cast<uint4*>(dst + (size_t)r * 16) = make_uint4(0, 0, 0, 0);
        }
      } else if (has) {
        const void* src = type == kF64 ? static_cast<const void*>(a.x64 + row0 * NR)
                                       : static_cast<const void*>((sreg.src < 0 ? static_cast<const float*>(a.t)
                                                                                : a.x32) + row0 * NR);
        if (nc > 0) bulk_g2s(zb + zoff, src, (uint32_t)nc * NR * es, zbar);
        for (int b = nc * NR * es; b < zb_bytes; b += 16)
          *reinterpret_cast<uint4*>(zb + zoff + b) = make_uint4(0, 0, 0, 0);
      }
      // zero rows [k16, k16p) of the 16-bit planes
      for (int c = lane; c < 4 * (k16p - k16); c += 32) {
        const int g = c / (k16p - k16), r = c % (k16p - k16);
        *reinterpret_cast<uint4*>(zb + ((size_t)g * k16p + k16 + r) * 16) = make_uint4(0, 0, 0, 0);
      }
    };

    auto row_scale = [&](const hmvm_tile_desc& d) {
      if constexpr (VST) return lane < d.nrows ? a.scale[d._pad + lane] : 1.0;
      else return 1.0;
    };
    auto out_slot = [&](const hmvm_tile_desc& d) {
      if constexpr (VST) return (d.mode == 1 && lane < d.nrows) ? a.out_idx[d.out_base + lane] : 0;
      else return 0;
    };
    hmvm_seg_desc cur_seg = (!failed && lane < cur.nseg) ? segs[cur.seg_begin + lane] : szero;
    int cur_k16 = 0, nxt_k16 = 0;
    uint32_t zpar[2] = {0, 0};
    bool zpend[2] = {false, false};
    if (!failed) {
      gather(cur, cur_seg, zbase, &zbars[0], &cur_k16);
      zpend[0] = true;
    }
    int cur_oidx = out_slot(cur);
    double cur_scale = row_scale(cur);
    hmvm_tile_desc nxt = tb + 1 < te ? tiles[tb + 1] : dzero;
    hmvm_seg_desc nxt_seg = (tb + 1 < te && lane < nxt.nseg) ? segs[nxt.seg_begin + lane] : szero;

    for (int ti = tb, k = 0; ti < te && !failed; ++ti, ++k) {
      unsigned char* zcur = zbase + (k & 1) * kTcZBytes;
      __syncwarp();
      if (ti + 1 < te) {
        gather(nxt, nxt_seg, zbase + ((k + 1) & 1) * kTcZBytes, &zbars[(k + 1) & 1], &nxt_k16);
        zpend[(k + 1) & 1] = true;
      }
      const bool has_nn = ti + 2 < te;
      const hmvm_tile_desc nn = has_nn ? tiles[ti + 2] : dzero;
      const int nxt_oidx = ti + 1 < te ? out_slot(nxt) : 0;
      const double nxt_scale = ti + 1 < te ? row_scale(nxt) : 1.0;
      if (!warp_wait(&zbars[k & 1], zpar[k & 1])) {
        failed = true;
        break;
      }
      zpar[k & 1] ^= 1;
      zpend[k & 1] = false;

      const int R = cur.nrows;
      const uint32_t rstride = (uint32_t)R * 16;
      uint32_t o = (uint32_t)((cur.data_off - vbase) * 16);
      const uint32_t ol_lane = (uint32_t)lane * 16;
      double row[NR];
#pragma unroll
      for (int r = 0; r < NR; r++) row[r] = 0.0;
      int zoff = 4 * cur_k16 * 16;
      bool mma_issued = false;

      // ring: release what the warp has passed, wait for [o, o_end)
      auto ensure = [&](uint32_t o_end) -> bool {
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
        return true;
      };

      // CUDA-core run of type TY (not the 16-bit type)
      auto run_cc = [&](auto tag, const unsigned char* zs, int nv) -> bool {
        constexpr int TY = decltype(tag)::value;
        constexpr int VS = TY == kF64 ? 2 : TY == kF32 ? 4 : 16;
        constexpr int ZV = VS * NR * (TY == kF64 ? 8 : 4);
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
          if (!ensure(o_end)) return false;
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

      // the 16-bit run on the tensor cores: pieces of up to kTcPiece chunks
      auto run_tc = [&](int nv) -> bool {
        const uint32_t zb_addr = smem_u32(zcur);
        const uint32_t st_addr = smem_u32(stage);
        for (int v0 = 0; v0 < nv; v0 += kTcPiece) {
          const int np = min(kTcPiece, nv - v0);
          if (mma_issued) {  // the previous piece's MMAs read the staging tile
            if (!warp_wait(mbar, mma_phase)) return false;
            mma_phase ^= 1;
            mma_open = false;
            tc_fence_after();
          }
          for (int v = 0; v < np; v += B) {
            const int nb = min(B, np - v);
            const uint32_t o_end = o + (uint32_t)nb * rstride;
            if (!ensure(o_end)) return false;
#pragma unroll
            for (int u = 0; u < B; u++) {
              if (u < nb) {
                uint4 m = *reinterpret_cast<const uint4*>(ring + ((o + ol_lane + (uint32_t)u * rstride) & (RING - 1)));
                if (lane >= R) m = make_uint4(0, 0, 0, 0);
                *reinterpret_cast<uint4*>(stage + (size_t)(v + u) * 512 + lane * 16) = m;
              }
            }
            o = o_end;
          }
          if (np & 1)  // an odd piece ends with a zero chunk (its K rows of B are zero too)
            *reinterpret_cast<uint4*>(stage + (size_t)np * 512 + lane * 16) = make_uint4(0, 0, 0, 0);
          fence_proxy_async();
          __syncwarp();
          if (lane == 0) {
            tc_fence_after();
            for (int s = 0; s < (np + 1) / 2; s++) {
              // A: chunks 2s, 2s+1 of the staging tile, M row 32q = tile row 0
              const uint64_t ad = tc_desc(st_addr + (uint32_t)(s * 1024) - (uint32_t)(512 * quad), 512, 128);
              // B: K rows (v0 * 8 + 16 s) .. + 15 of the four planes
              const uint64_t bd = tc_desc(zb_addr + (uint32_t)((v0 * 8 + 16 * s) * 16), 128,
                                          (uint32_t)(cur_k16 * 16));
              tc_mma(dcol, ad, bd, IDESC, (mma_issued || s > 0) ? 1 : 0);
            }
            tc_commit(mbar);
          }
          __syncwarp();
          mma_issued = true;
          mma_open = true;
        }
        return true;
      };

      int j = 0;
      while (j < (VST ? 1 : cur.nseg)) {
        const int type = tc_seg_type(__shfl_sync(0xffffffffu, cur_seg.ncols, j));
        const int lg = mixed_vec_log2(type);
        int nv = 0;
        if (VST) {
          nv = cur.nvec;
          j = 1;
        } else {
          for (; j < cur.nseg; j++) {
            const int enc = __shfl_sync(0xffffffffu, cur_seg.ncols, j);
            if (tc_seg_type(enc) != type) break;
            nv += ((enc & 0x0fffffff) + (1 << lg) - 1) >> lg;
          }
        }
        bool ok;
        if (type == LR) {
          ok = run_tc(nv);
        } else {
          const unsigned char* zs = zcur + zoff;
          zoff += (nv << lg) * NR * (type == kF64 ? 8 : 4);
          switch (type) {
            case kF64: ok = run_cc(TypeTag<kF64>{}, zs, nv); break;
            case kF32: ok = run_cc(TypeTag<kF32>{}, zs, nv); break;
            default: ok = run_cc(TypeTag<kE4M3>{}, zs, nv); break;
          }
        }
        if (!ok) {
          failed = true;
          break;
        }
      }
      if (!failed && mma_issued) {
        if (!warp_wait(mbar, mma_phase)) {
          failed = true;
        } else {
          mma_phase ^= 1;
          mma_open = false;
          tc_fence_after();
          float d[kTcN];
          tc_ld32(dread, d);
#pragma unroll
          for (int r = 0; r < NR; r++) row[r] += ((double)d[r] + (double)d[NR + r]) * (double)pscale_inv[r];
          tc_fence_before();
        }
      }
      if (failed) break;
      if (lane < R) {
        if constexpr (VST) {
          if (cur.mode == 1) {
#pragma unroll
            for (int r = 0; r < NR; r++)
              static_cast<float*>(a.t)[(int64_t)cur_oidx * NR + r] = (float)(row[r] * cur_scale);
          } else {
#pragma unroll
            for (int r = 0; r < NR; r++)
              static_cast<double*>(a.p)[(int64_t)(cur.out_base + lane) * NR + r] = row[r] * cur_scale;
          }
        } else {
          if (cur.mode == 0) {
#pragma unroll
            for (int r = 0; r < NR; r++)
              if (r < a.nr) static_cast<double*>(a.y)[cur.out_base + lane + r * a.ldy] = row[r];
          } else {
#pragma unroll
            for (int r = 0; r < NR; r++) static_cast<double*>(a.p)[(int64_t)(cur.out_base + lane) * NR + r] = row[r];
          }
        }
      }
      cur = nxt;
      cur_seg = nxt_seg;
      cur_k16 = nxt_k16;
      cur_oidx = nxt_oidx;
      cur_scale = nxt_scale;
      nxt = nn;
      nxt_seg = (has_nn && lane < nn.nseg) ? segs[nn.seg_begin + lane] : szero;
    }
    if (failed) {
      // let the copies and MMAs in flight finish (bounded) before the shared
      // memory and TMEM go away
      const uint32_t issued = min(nchunks, q_rel + (uint32_t)S);
      for (uint32_t q = q_ready; q < issued; q++) warp_wait(&bars[q % S], (q / S) & 1);
      for (int b = 0; b < 2; b++)
        if (zpend[b]) warp_wait(&zbars[b], zpar[b]);
      if (mma_open) warp_wait(mbar, mma_phase);
      if (lane == 0) atomicExch(a.err, 1);
    }
  }
  // the CTA's MMAs are complete (every warp waited for its last commit, or gave up
  // after a bounded wait): free the TMEM
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace hmvm
