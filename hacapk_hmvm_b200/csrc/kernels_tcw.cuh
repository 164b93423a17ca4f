// Wide tensor-core multi-RHS HMVM: 128 right-hand sides per pass, every
// product on the 5th-generation tensor cores (tcgen05, FP32 accumulation in
// TMEM), the matrix streamed from HBM once per pass.  The layout it walks is
// built by build_tc_layout (layout_tc.cpp).
//
// GEMM orientation: Y^T = X^T H^T, so the MMA (kind::f16, cta_group::1) has
//   M = 128 right-hand sides (TMEM lanes),
//   N = the item's rows rounded up to 16 (<= 32 row-stage, <= 128 V-stage),
//   K = 16 matrix columns (a K step of the pipeline is 32: two MMA "halves"),
//   A = the inputs, 16-bit hi and lo parts of 128 right-hand sides, held in
//       four "chunk" arrays [4][rows][64] (chunk 0/1: hi of right-hand sides
//       0..63 / 64..127, chunk 2/3: their lo parts); one TMA tensor copy per K
//       step (a 3-D box {64, 32, 4}, 128-byte rows, SWIZZLE_128B) lands as the
//       canonical 128-byte-swizzled MN-major layout: per chunk 32 K rows of
//       128 bytes, 8-row atoms 1 KiB apart, the second half 2 KiB on, the next
//       64 right-hand sides 4 KiB on;
//   B = the matrix, K-major without swizzle, read by the MMA straight from the
//       ring the bulk copies fill (8-row core matrices 128 B apart, the second
//       8 columns R*16 B on; the missing half of an odd last step points at a
//       zero block);
//   D = FP32 in TMEM, 2 accumulator buffers of 256 columns: V stage row block b
//       at column 128 b, row stage at 32 b; the correction products (hi x x_lo,
//       lo x x_hi) in a second accumulator where the block has room (row stage
//       at 128 + 32 b, V-stage blocks of <= 64 rows at 128 b + 64), added to
//       the main one in the epilogue: each addition into a TMEM accumulator
//       rounds, and the main one then takes one per 16 columns, not three.
// An item is up to 4 row blocks; a segment multiplies the blocks in its mask
// by one input range, and consecutive segments with the same range form an
// input group: per K step of a group one TMA copy of the inputs, then for each
// segment and each of its blocks hi x x_hi and hi x x_lo, plus lo x x_hi for
// pair-stored segments (the stream holds, per K step, per segment, per block,
// the hi vectors and then the lo vectors).
//
// One CTA of 14 warps per SM, warp-specialised:
//   warp 13              matrix producer of the row stage (the whole warp; lane 0 issues the
//                        copies): per K step a bulk copy of its matrix bytes
//                        into the current 16 KiB slot of a 6-slot ring (a slot
//                        -- "chunk" -- takes whole K steps, at most 6, across
//                        segments and items; each copy adds its bytes with
//                        mbarrier.expect_tx and the chunk is closed by one
//                        arrive);
//   warp 0               input producer (the whole warp; in the V stage also
//                        the matrix producer, warp 13 idle): per K step a TMA
//                        tensor copy of its inputs into a 7 x 16 KiB ring and,
//                        beside the input slot, the step's MMAs fully formed
//                        (16 bytes each, lane q the q-th) from the host-built
//                        step program; it repeats the matrix producer's chunk
//                        arithmetic to know where each step's matrix bytes lie;
//   warps 1..4           MMA issue, one thread each: warp 1 + b issues row
//                        block b's MMAs into its own TMEM columns (a thread
//                        that issues MMAs whose operands it loads sustains
//                        about one per 100 cycles; four of them keep the
//                        tensor core busy), and commits each input slot,
//                        matrix chunk and finished accumulator to its
//                        mbarrier, which counts the issuing warps (warp 1 also
//                        allocates the TMEM);
//   warps 5..12          epilogue: tcgen05.ld the accumulators (warp w reads
//                        lanes 32 (w % 4) ..), scale, and store t (16-bit
//                        hi/lo chunks) or y (each thread 32 consecutive rows of
//                        its right-hand side); in the V stage, whose bound is
//                        converting and storing t, warps 5..8 take an item's
//                        even 32-row chunks and warps 9..12 its odd ones; in
//                        the row stage warps 5..8 take all and 9..12 idle.
// The matrix producer waits only for the chunk 6 back, the input producer only
// for the input slot 7 back, and the MMAs of a chunk need only that chunk and
// its input slots: no wait can close a cycle.  Where one warp holds both roles,
// a chunk holds fewer K steps than the input ring has slots, so it always
// reaches the K step that closes a chunk before it needs an input slot the
// MMAs of that chunk would free.
// Every mbarrier wait is bounded (kWaitLimitNs); a role that gives up records
// the error and stops; before the CTA exits, the copies still in flight and
// the MMAs issued are waited for (bounded) and the TMEM is freed.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "kernels_tc.cuh"
#include "layout.hpp"

namespace hmvm {

// A K step covers 32 matrix columns: two 16-column MMA steps ("halves").
constexpr int kTcwStepCols = 32;
constexpr int kTcwSlotM = 16384;  // matrix ring chunk: whole K steps (one K step of an item is <= 16 KiB)
constexpr int kTcwSlotsM = 6;
constexpr int kTcwChunkSteps = 6; // K steps per chunk at most (< kTcwSlotsA)
constexpr int kTcwSlotA = 16384;  // one K step of inputs: 4 chunks x 32 rows x 128 B
constexpr int kTcwSlotsA = 7;
static_assert(kTcwChunkSteps < kTcwSlotsA, "a chunk must hold fewer K steps than the input ring has slots");
constexpr int kTcwEpiWarps = 8;   // two per TMEM lane quadrant
constexpr int kTcwThreads = 32 * (6 + kTcwEpiWarps);  // input producer, 4 MMA-issue warps, epilogue, matrix producer
constexpr int kTcwBoth = 0, kTcwInputs = 1, kTcwMatrix = 2;  // producer roles
// Zeros: the B operand of the per-item MMA that clears the accumulators (256
// rows x 16 columns, the second 8 columns 4 KiB on; its first 4 KiB also serve
// as that MMA's A operand) and of an odd last K step's missing 8 columns.
constexpr int kTcwZeroBytes = 8192;
constexpr int kTcwOffA = kTcwSlotsM * kTcwSlotM;
constexpr int kTcwOffZero = kTcwOffA + kTcwSlotsA * kTcwSlotA;
// Per input slot, the MMAs of its K step as the producer formed them, per half
// at most kTcwMaxOps ordered by row block, 16 bytes each, and a header word
// (per row block its MMA count per half in 4 bits, flags).
constexpr uint32_t kTcwNewChunk = 1u << 16, kTcwLastStep = 1u << 17, kTcwTwoHalves = 1u << 18;  // header flags
constexpr int kTcwOpsPerSlot = 2 * kTcwMaxOps;
constexpr int kTcwOffOps = kTcwOffZero + kTcwZeroBytes;
constexpr int kTcwOffHdr = kTcwOffOps + kTcwSlotsA * kTcwOpsPerSlot * 16;
constexpr int kTcwOffBar = kTcwOffHdr + ((kTcwSlotsA * 4 + 15) & ~15);
constexpr int kTcwNumBars = 2 * kTcwSlotsM + 2 * kTcwSlotsA + 2 * 4 + 1;
constexpr int kTcwOffMisc = kTcwOffBar + kTcwNumBars * 8;
// per epilogue warp: the current 32-row chunk's row scales and t slots (V stage)
constexpr int kTcwOffRows = kTcwOffMisc + 32;
constexpr int kTcwSmem = kTcwOffRows + kTcwEpiWarps * 32 * 8 + 1024;  // + room to align the base to 1 KiB
static_assert(kTcwSmem <= 227 * 1024, "shared memory");
// TMEM geometry per stage: accumulator buffers x columns, and the column stride of a row block
// (a block's correction accumulator is corr columns after its main one: row
// stage at 128 + 32 b, V stage at 128 b + 64 for blocks of <= 64 rows)
template <bool VST>
struct TcwGeom {
  static constexpr int bufs = 2;
  static constexpr int cols = 256;
  static constexpr int bstride = VST ? 128 : 32;
  static constexpr int corr = VST ? 64 : 128;
  static constexpr int issuers = VST ? 2 : 4;  // row blocks: one MMA-issue warp each
  static constexpr int cpb = VST ? 4 : 1;      // 32-row chunks of a row block at most
  static constexpr int chunks = issuers * cpb; // 32-row chunks of an item at most
  // epilogue warps: V stage two per TMEM lane quadrant (converting and storing t
  // bounds it), row stage one (more warps polling beside the producers slow it)
  static constexpr int epi = VST ? kTcwEpiWarps : 4;
  static_assert(bufs * cols == 512, "the CTA owns the SM's 512 TMEM columns");
};

struct TcwArgs {
  const hmvm_tile_desc* tiles;
  const hmvm_seg_desc* segs;
  const int32_t* blocks;      // per item: rows of its row blocks 0..3, 8 bits each
  const uint4* groups;        // the step program: per input group its header ...
  const uint2* gops;          // ... and its MMA templates (kTcwMaxOps zero templates after the last)
  const int32_t* gfirst;      // [items + 1]: first input group of each item
  int n_gops;                 // templates in gops, the zero ones included
  const int32_t* team_begin;  // [nteams + 1]
  int nteams;
  const char* data;           // the 16-byte vectors of the stream
  const int32_t* out_idx;     // V stage: t slot per panel row
  const float* tscale;        // V stage: 2^-c per panel row; row stage: s_i per row (tile _pad indexes it)
  const float* xscale;        // sigma_x per right-hand side [128]
  uint16_t* tplanes;          // V stage output: 4 chunks x trows x 64
  int64_t trows;
  float* part;                // V-stage split panels: FP32 partial sums [row][128]
  void* y;                    // row-stage output, column-major, leading dimension ldy
  int64_t ldy;
  int nr;                     // right-hand sides of this pass (<= 128)
  int y32;                    // y is FP32 (FP32 plans), else FP64
  int* err;
};

// Shared-memory matrix descriptor of a 128-byte-swizzled layout (tcgen05
// layout type 2): start address, leading- and stride-dimension byte offsets.
__device__ __forceinline__ uint64_t tc_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return tc_desc(saddr, lbo, sbo) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
// Adds `bytes` to the transaction count of the current phase without arriving.
__device__ __forceinline__ void mbar_expect_tx_only(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Single-thread bounded wait for the phase with parity `parity`.
__device__ __forceinline__ bool thread_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity))
    if (global_ns() - t0 > kWaitLimitNs) return false;
  return true;
}

template <bool BF>
__device__ __forceinline__ void tcw_split(float v, uint16_t& hi, uint16_t& lo) {
  if (BF) {
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
  } else {
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    hi = __half_as_ushort(h);
    lo = __half_as_ushort(l);
  }
}

// Row-stage output: rows 0..31 of a 32-row chunk for this lane's right-hand
// side, y[o + i] = v[i] * ts_i * sx (ts_i from lane i), rows >= nrow skipped.
// W consecutive rows go out as one 16-byte store (W = 2 doubles or 4 floats;
// W = 1: single stores) from row P on, P chosen by the caller so that o + P is
// a multiple of W (the same on every lane when the leading dimension is);
// the rows before P and after the last whole group go out singly.
template <typename T, int W, int P>
__device__ __forceinline__ void tcw_store_rows(T* __restrict__ y, int64_t o, int nrow, bool act, const float* v,
                                               float ts_l, double sx) {
  auto val = [&](int i, float ts) { return (T)((double)v[i] * (double)ts * sx); };
#pragma unroll
  for (int i = 0; i < P; i++) {
    const float ts = __shfl_sync(0xffffffffu, ts_l, i);
    if (act && i < nrow) y[o + i] = val(i, ts);
  }
  constexpr int kEnd = P + ((32 - P) / W) * W;
#pragma unroll
  for (int i = P; i < kEnd; i += W) {
    float ts[W];
#pragma unroll
    for (int k = 0; k < W; k++) ts[k] = __shfl_sync(0xffffffffu, ts_l, i + k);
    if (act) {
      if (W > 1 && i + W <= nrow) {
        if constexpr (W == 2) {
          *reinterpret_cast<double2*>(y + o + i) = make_double2(val(i, ts[0]), val(i + 1, ts[1]));
        } else if constexpr (W == 4) {
          *reinterpret_cast<float4*>(y + o + i) =
              make_float4(val(i, ts[0]), val(i + 1, ts[1]), val(i + 2, ts[2]), val(i + 3, ts[3]));
        }
      } else {
#pragma unroll
        for (int k = 0; k < W; k++)
          if (i + k < nrow) y[o + i + k] = val(i + k, ts[k]);
      }
    }
  }
#pragma unroll
  for (int i = kEnd; i < 32; i++) {
    const float ts = __shfl_sync(0xffffffffu, ts_l, i);
    if (act && i < nrow) y[o + i] = val(i, ts);
  }
}

template <bool VST, bool BF>
__global__ void __launch_bounds__(kTcwThreads, 1)
    hmvm_tcw_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap tmap,
                    const TcwArgs a) {
  using G = TcwGeom<VST>;
  extern __shared__ __align__(1024) unsigned char tcw_smem_raw[];
  // the swizzled input slots need 1 KiB alignment
  unsigned char* tcw_smem = tcw_smem_raw + ((1024u - (smem_u32(tcw_smem_raw) & 1023u)) & 1023u);
  unsigned char* ringM = tcw_smem;
  unsigned char* ringA = tcw_smem + kTcwOffA;
  unsigned char* zero = tcw_smem + kTcwOffZero;
  uint64_t* bars = reinterpret_cast<uint64_t*>(tcw_smem + kTcwOffBar);
  uint64_t* mfull = bars;
  uint64_t* mempty = mfull + kTcwSlotsM;
  uint64_t* afull = mempty + kTcwSlotsM;
  uint64_t* aempty = afull + kTcwSlotsA;
  uint64_t* accfull = aempty + kTcwSlotsA;
  uint64_t* accempty = accfull + 4;
  uint64_t* done = accempty + 4;
  uint32_t* misc = reinterpret_cast<uint32_t*>(tcw_smem + kTcwOffMisc);
  // misc: [0] TMEM base, [1] matrix chunks opened, [2] input steps issued,
  //       [3] matrix chunks consumed, [4] input steps consumed (least over the issuers)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < kTcwSlotsM; s++) {
      mbar_init(&mfull[s], 1);
      mbar_init(&mempty[s], G::issuers);
    }
    for (int s = 0; s < kTcwSlotsA; s++) {
      mbar_init(&afull[s], 1);
      mbar_init(&aempty[s], G::issuers);
    }
    for (int s = 0; s < G::bufs; s++) {
      mbar_init(&accfull[s], G::issuers);
      mbar_init(&accempty[s], G::epi);
    }
    mbar_init(done, G::issuers);
    misc[1] = misc[2] = 0;
    misc[3] = misc[4] = 0xffffffffu;  // the issuers' least progress
    fence_mbar_init();
  }
  for (int k = tid; k < kTcwZeroBytes / 16; k += kTcwThreads)
    reinterpret_cast<uint4*>(zero)[k] = make_uint4(0, 0, 0, 0);
  fence_proxy_async();  // the zeros, before the tensor cores read them
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(misc))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = misc[0];
  const int team = blockIdx.x;
  const int tb = team < a.nteams ? a.team_begin[team] : 0;
  const int te = team < a.nteams ? a.team_begin[team + 1] : 0;

  // ---- producers (two whole warps, one role each) ----
  // Each walks the team's step program: per input group its header (and, for
  // the inputs, its MMA templates: lane q gets template q), read by shuffles
  // from two 32-entry windows that the warp loads coalesced one window ahead,
  // so no global load latency lands on a K step.  Both run the same chunk
  // arithmetic.  The matrix role (warp 13) copies each K step's matrix bytes
  // into the current chunk (lane 0: the chunk's mbarriers and bulk copies).
  // The input role (warp 0) forms the step's MMAs from the templates (lane q
  // writes MMA q: low words of the A and B descriptors, block, instruction
  // descriptor), a header word (counts, starts a chunk, the item's last step)
  // and the input slot's TMA copy (lane 0), whose arrive publishes the MMAs.
  // Every lane keeps the same counters; lane 0's waits decide for all.  The
  // row stage splits the roles (its producer bounds it); the V stage, bound by
  // its epilogue, runs both in warp 0 (measured faster there).
  auto produce = [&](auto role) {
    constexpr int R = decltype(role)::value;  // kTcwBoth, kTcwInputs or kTcwMatrix
    constexpr bool MAT = R != kTcwInputs, INP = R != kTcwMatrix;
    if (tb >= te) return;
    uint4* ops = reinterpret_cast<uint4*>(tcw_smem + kTcwOffOps);
    uint32_t* hdr = reinterpret_cast<uint32_t*>(tcw_smem + kTcwOffHdr);
    const uint32_t zaddr = smem_u32(zero);
    // A: input slot 0's first half, hi part (the two 64-rhs chunks 4 KiB apart); slot s is
    // (16 KiB * s) >> 4 further on, the second half 2 KiB on, the lo part 8 KiB on
    const uint32_t alo0 = (uint32_t)tc_desc_sw128(smem_u32(ringA), 4096, 1024);
    const int g0 = a.gfirst[tb], gend = a.gfirst[te];
    const int glast = max(gend - 1, 0);  // window loads past the team's groups read its last one
    const int tlast = a.n_gops - 1;
    int hb = g0;  // group of lane 0 of the header window H0; H1 holds the next 32
    uint4 H0 = a.groups[min(hb + lane, glast)], H1 = a.groups[min(hb + 32 + lane, glast)];
    uint32_t tc = __shfl_sync(0xffffffffu, H0.w, 0);  // this group's first template
    uint32_t tw = tc;                                  // template of lane 0 of window T0; T1 the next 32
    uint2 T0 = make_uint2(0, 0), T1 = make_uint2(0, 0);
    if constexpr (INP) {
      T0 = a.gops[min((int)tw + lane, tlast)];
      T1 = a.gops[min((int)tw + 32 + lane, tlast)];
    }
    uint32_t mI = 0, aI = 0, used = 0, cnt = 0, cbase = 0;
    int ms = 0;
    bool ok = true, open = false;
    const char* g = a.data + a.tiles[tb].data_off * 16;  // the team's items are contiguous in the stream
    for (int gi = g0; gi < gend && ok; gi++) {
      if (gi - hb == 32) {
        hb += 32;
        H0 = H1;
        H1 = a.groups[min(hb + 32 + lane, glast)];
      }
      const int hl = gi - hb;
      uint4 gh;
      gh.x = __shfl_sync(0xffffffffu, H0.x, hl);
      gh.y = __shfl_sync(0xffffffffu, H0.y, hl);
      gh.z = __shfl_sync(0xffffffffu, H0.z, hl);
      const uint32_t counts = gh.z >> 16, hrows = gh.z & 0xfffu;
      const uint32_t nops = (counts & 15u) + ((counts >> 4) & 15u) + ((counts >> 8) & 15u) + (counts >> 12);
      const int hq = lane >= kTcwMaxOps ? 1 : 0, q = lane - hq * kTcwMaxOps;  // lane: half hq, MMA q
      uint2 tp = make_uint2(0, 0);
      if constexpr (INP) {
        if (tc - tw >= 32u) {  // a group's templates (<= kTcwMaxOps) span at most the two windows
          tw += 32;
          T0 = T1;
          T1 = a.gops[min((int)tw + 32 + lane, tlast)];
        }
        const uint32_t ti = tc - tw + (uint32_t)min(q, kTcwMaxOps - 1);
        const uint32_t t0x = __shfl_sync(0xffffffffu, T0.x, (int)(ti & 31u));
        const uint32_t t0y = __shfl_sync(0xffffffffu, T0.y, (int)(ti & 31u));
        const uint32_t t1x = __shfl_sync(0xffffffffu, T1.x, (int)(ti & 31u));
        const uint32_t t1y = __shfl_sync(0xffffffffu, T1.y, (int)(ti & 31u));
        tp = ti < 32u ? make_uint2(t0x, t0y) : make_uint2(t1x, t1y);
        tc += nops;
      }
      const CUtensorMap* map = (gh.x >> 31) ? &tmap : &xmap;
      const int row0 = (int)(gh.x & 0x7fffffffu), nv = (int)gh.y, nks = (nv + 3) >> 2;
      const uint32_t prow = tp.x & 0xfffu, alo = (tp.x >> 12) & 1u, blk = (tp.x >> 13) & 3u, rb16 = tp.x >> 16;
      const uint32_t dcol = blk * (uint32_t)G::bstride + ((tp.x & kTcwCorrBit) ? (uint32_t)G::corr : 0u);
      for (int j = 0; j < nks; j++) {
        // 8-column vectors of the two halves (an odd last one: 1; a missing second half: 0)
        const uint32_t nvj0 = (uint32_t)min(2, nv - 4 * j), nvj1 = (uint32_t)max(0, min(2, nv - 4 * j - 2));
        const uint32_t kb0 = nvj0 * 16u * hrows, kb = kb0 + nvj1 * 16u * hrows;
        uint32_t flags = 0;
        if (!open || used + kb > (uint32_t)kTcwSlotM || cnt == kTcwChunkSteps) {
          ms = mI % kTcwSlotsM;
          if constexpr (MAT) {
            bool okw = true;
            if (lane == 0) {
              if (open) mbar_arrive(&mfull[(mI + kTcwSlotsM - 1) % kTcwSlotsM]);  // close the chunk
              okw = mI < kTcwSlotsM || thread_wait(&mempty[ms], ((mI / kTcwSlotsM) - 1) & 1);
            }
            if (!__shfl_sync(0xffffffffu, okw, 0)) {
              ok = false;
              open = false;
              break;
            }
          }
          mI++;
          open = true;
          used = cnt = 0;
          cbase = smem_u32(ringM + ms * kTcwSlotM);
          flags |= kTcwNewChunk;
        }
        if constexpr (MAT) {
          if (lane == 0) {
            mbar_expect_tx_only(&mfull[ms], kb);
            bulk_g2s(ringM + ms * kTcwSlotM + used, g, kb, &mfull[ms]);
          }
        }
        if constexpr (INP) {
          const int as = aI % kTcwSlotsA;
          bool okw = true;
          if (lane == 0) okw = aI < kTcwSlotsA || thread_wait(&aempty[as], ((aI / kTcwSlotsA) - 1) & 1);
          if (!__shfl_sync(0xffffffffu, okw, 0)) {
            ok = false;
            break;
          }
          if ((gh.z & kTcwGroupLast) && j + 1 == nks) flags |= kTcwLastStep;
          const uint32_t nvjh = hq ? nvj1 : nvj0;
          if ((uint32_t)q < nops && nvjh > 0) {
            // B: the block's rows from prow on in the half's vectors, K-major core matrices; an odd
            // last half's second 8 columns read the zero block
            const uint32_t start = cbase + used + (hq ? kb0 : 0u) + nvjh * 16u * prow;
            const uint32_t lbo = nvjh == 2 ? rb16 : zaddr - start;
            ops[as * kTcwOpsPerSlot + hq * (int)nops + q] =
                make_uint4(alo0 + (uint32_t)as * (uint32_t)(kTcwSlotA >> 4) + (uint32_t)hq * (2048u >> 4) +
                               alo * (8192u >> 4),
                           ((start >> 4) & 0x3fffu) | (((lbo >> 4) & 0x3fffu) << 16), dcol, tp.y);
          }
          __syncwarp();
          if (lane == 0) {
            hdr[as] = counts | flags | (nvj1 > 0 ? kTcwTwoHalves : 0u);
            mbar_expect_tx(&afull[as], kTcwSlotA);
            tma_load_3d(ringA + as * kTcwSlotA, map, 0, row0 + kTcwStepCols * j, 0, &afull[as]);
          }
          aI++;
        }
        g += kb;
        used += kb;
        cnt++;
      }
    }
    if (lane == 0) {
      if constexpr (MAT) {
        if (open) mbar_arrive(&mfull[ms]);  // close the last chunk (also after a failure, so it can drain)
        misc[1] = mI;
      }
      if constexpr (INP) misc[2] = aI;
      if (!ok) atomicExch(a.err, 1);
    }
  };
  if (warp == 0) {
    if constexpr (VST) produce(std::integral_constant<int, kTcwBoth>{});
    else produce(std::integral_constant<int, kTcwInputs>{});
  } else if (warp == kTcwThreads / 32 - 1) {
    if constexpr (!VST) produce(std::integral_constant<int, kTcwMatrix>{});
  } else if (warp <= 4) {
    // ---- MMA issue: warp 1 + b, one thread, row block b ----
    // Per item one MMA that clears the block's accumulator, then per K step
    // the block's part of the producer's MMA list.  Every issuer waits for and
    // commits every step, chunk and item (the barriers count the issuers).
    const int b = warp - 1;
    if (b < G::issuers && lane == 0) {
      const uint4* ops = reinterpret_cast<const uint4*>(tcw_smem + kTcwOffOps);
      const uint32_t* hdr = reinterpret_cast<const uint32_t*>(tcw_smem + kTcwOffHdr);
      // descriptor high words: stride byte offset, version, layout (128-byte swizzle for A)
      const uint64_t ahi = tc_desc_sw128(0, 0, 1024) & 0xffffffff00000000ull;
      const uint64_t bhi = tc_desc(0, 0, 128) & 0xffffffff00000000ull;
      // the clearing MMA: zeros x zeros over the block's columns (V stage: its main and
      // correction accumulators; row stage: the main one, and a second for the correction one)
      const uint32_t zaddr = smem_u32(zero);
      const uint64_t zadesc = tc_desc_sw128(zaddr, 2048, 1024);
      const uint64_t zbdesc = tc_desc(zaddr, 4096, 128);
      const uint32_t zidesc = tcw_idesc(BF ? 1 : 0, G::bstride);
      uint32_t mC = 0, aC = 0, ic = 0;
      int ms = 0;
      bool ok = true, open = false;
      int nseg_next = tb < te ? a.tiles[tb].nseg : 0;
      for (int it = tb; it < te && ok; it++, ic++) {
        const int nseg = nseg_next;
        nseg_next = it + 1 < te ? a.tiles[it + 1].nseg : 0;
        const int buf = ic % G::bufs;
        if (ic >= G::bufs && !thread_wait(&accempty[buf], ((ic / G::bufs) - 1) & 1)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t dbase = tmem_base + (uint32_t)(buf * G::cols);
        if (nseg > 0) {
          tc_mma(dbase + (uint32_t)(b * G::bstride), zadesc, zbdesc, zidesc, 0);
          if (!VST) tc_mma(dbase + (uint32_t)(b * G::bstride + G::corr), zadesc, zbdesc, zidesc, 0);
        }
        bool last = nseg == 0;
        while (!last) {
          const int as = aC % kTcwSlotsA;
          if (!thread_wait(&afull[as], (aC / kTcwSlotsA) & 1)) {
            ok = false;
            break;
          }
          aC++;
          const uint32_t h = hdr[as];
          last = (h & kTcwLastStep) != 0;
          if (h & kTcwNewChunk) {
            if (open) tc_commit(&mempty[ms]);  // the previous chunk's MMAs done: it can be refilled
            ms = mC % kTcwSlotsM;
            if (!thread_wait(&mfull[ms], (mC / kTcwSlotsM) & 1)) {
              ok = false;
              open = false;
              break;
            }
            mC++;
            open = true;
          }
          tc_fence_after();  // the MMAs below are ordered after the waits that saw their operands land
          uint32_t off = 0;  // this block's first MMA in a half's list: the counts of the blocks before it
#pragma unroll
          for (int c = 0; c < 3; c++)
            if (c < b) off += (h >> (4 * c)) & 15u;
          const uint32_t n = (h >> (4 * b)) & 15u;
          const uint32_t nall = (h & 15u) + ((h >> 4) & 15u) + ((h >> 8) & 15u) + ((h >> 12) & 15u);
          const uint4* o = ops + as * kTcwOpsPerSlot + off;
          // this block's MMAs of each half: the half's list holds nall; the loop is compact (an
          // unrolled one measured slower), the next record loaded ahead (past the last it reads a
          // later record or the header words: inside shared memory)
          for (int half = 0; half < ((h & kTcwTwoHalves) ? 2 : 1); half++, o += nall) {
            uint4 r = o[0];
#pragma unroll 1
            for (uint32_t k = 0; k < n; k++) {
              const uint4 nx = o[k + 1];
              tc_mma(dbase + r.z, ahi | r.x, bhi | r.y, r.w, 1);
              r = nx;
            }
          }
          tc_commit(&aempty[as]);
        }
        if (ok) tc_commit(&accfull[buf]);
      }
      if (open) tc_commit(&mempty[ms]);
      atomicMin(&misc[3], mC);
      atomicMin(&misc[4], aC);
      // every MMA issued has completed before the CTA goes on (bounded)
      tc_commit(done);
      if (!thread_wait(done, 0)) ok = false;
      if (!ok) atomicExch(a.err, 1);
    }
  } else if (warp < 5 + G::epi) {
    // ---- epilogue ----
    // Warps 5..4+G::epi: warp w reads TMEM lanes 32 (w % 4) .. (the right-hand
    // sides 32 (w % 4) + lane); with 8 of them, of each item's 32-row chunks in
    // order the even ones (w <= 8) or the odd ones.
    const int q = warp & 3;
    const int half = G::epi == 8 ? (warp - 5) >> 2 : 0;
    const int r = 32 * q + lane;  // this thread's right-hand side
    const double sx = a.xscale[r];
    // V stage: this right-hand side's element of t slot 0 in the hi chunk and in
    // the lo chunk (slot s is s * 64 elements on); per row of a chunk its scale
    // and slot by one broadcast shared-memory load
    uint16_t* const thi = VST ? a.tplanes + (int64_t)(r >> 6) * a.trows * 64 + (r & 63) : nullptr;
    uint16_t* const tlo = VST ? thi + (int64_t)2 * a.trows * 64 : nullptr;
    uint2* const rows_sm = reinterpret_cast<uint2*>(tcw_smem + kTcwOffRows) + (warp - 5) * 32;
    // row stage: 16-byte stores of consecutive rows where y's base is 16-byte aligned and its
    // leading dimension a multiple of the rows per store (then every lane's rows align alike)
    const bool vec_y = !VST && (reinterpret_cast<uintptr_t>(a.y) & 15) == 0 && (a.ldy & (a.y32 ? 3 : 1)) == 0;
    // The scale (and t slot) of row 32 k + lane of an item's chunk k (chunk k = 32-row
    // piece k % cpb of row block k / cpb), loaded a whole item ahead; the descriptors
    // two items ahead; a chunk's values are then taken by shuffles.
    struct Rows {
      float ts[G::chunks];
      int32_t sl[G::chunks];
    };
    auto load_rows = [&](const hmvm_tile_desc& d, uint32_t R4, Rows& rw) {
      const int mode = d.mode & 3;
      int rb = 0;
#pragma unroll
      for (int b = 0; b < G::issuers; b++) {
        const int Rb = (int)((R4 >> (8 * b)) & 0xffu);
#pragma unroll
        for (int c = 0; c < G::cpb; c++) {
          const bool in = lane < Rb - 32 * c;
          const int row = rb + 32 * c + lane;
          rw.ts[b * G::cpb + c] = in ? a.tscale[d._pad + row] : 0.f;
          rw.sl[b * G::cpb + c] = (VST && in && mode == 1) ? a.out_idx[d.out_base + row] : 0;
        }
        rb += Rb;
      }
    };
    hmvm_tile_desc dc, dn;
    uint32_t Rc = 0, Rn = 0;
    Rows rc, rn;
    if (tb < te) {
      dc = a.tiles[tb];
      Rc = (uint32_t)a.blocks[tb];
      load_rows(dc, Rc, rc);
    }
    if (tb + 1 < te) {
      dn = a.tiles[tb + 1];
      Rn = (uint32_t)a.blocks[tb + 1];
    }
    uint32_t ic = 0;
    for (int it = tb; it < te; it++, ic++) {
      const hmvm_tile_desc d = dc;
      const uint32_t R4 = Rc;
      if (it + 1 < te) load_rows(dn, Rn, rn);  // the next item's rows, in flight during this one
      hmvm_tile_desc dnn = dn;
      uint32_t Rnn = 0;
      if (it + 2 < te) {
        dnn = a.tiles[it + 2];
        Rnn = (uint32_t)a.blocks[it + 2];
      }
      const int buf = ic % G::bufs;
      const int mode = d.mode & 3, has = (d.mode >> 4) & 15;
      if (!warp_wait(&accfull[buf], (ic / G::bufs) & 1)) {
        if (lane == 0) atomicExch(a.err, 1);
        break;
      }
      tc_fence_after();
      int rb = 0;  // the block's first item row
      int seq = 0;  // the item's chunks in order: this warp takes every other one
      for (int b = 0; b < G::issuers; b++) {
        const int Rb = (int)((R4 >> (8 * b)) & 0xffu);
        if (!Rb) break;  // blocks after the last are empty
        for (int c0 = 0; c0 < Rb; c0 += 32) {
          if (G::epi == 8 && (seq++ & 1) != half) continue;
          const int k = b * G::cpb + (c0 >> 5), nrow = min(32, Rb - c0), row = rb + c0;
          float ts_l = rc.ts[0];
          int32_t slot_l = rc.sl[0];
#pragma unroll
          for (int j = 1; j < G::chunks; j++) {
            ts_l = k == j ? rc.ts[j] : ts_l;
            slot_l = k == j ? rc.sl[j] : slot_l;
          }
          float v[32];
          if (has >> b & 1) {
            const uint32_t ta = tmem_base + ((uint32_t)(32 * q) << 16) + (uint32_t)(buf * G::cols + b * G::bstride + c0);
            tc_ld32(ta, v);
            if (!VST || Rb <= 64) {  // plus the correction accumulator
              float w[32];
              tc_ld32(ta + (uint32_t)G::corr, w);
#pragma unroll
              for (int i = 0; i < 32; i++) v[i] += w[i];
            }
          } else {
#pragma unroll
            for (int i = 0; i < 32; i++) v[i] = 0.f;
          }
          if constexpr (VST) {
            rows_sm[lane] = make_uint2(__float_as_uint(ts_l), (uint32_t)slot_l);
            __syncwarp();
            if (mode == 1) {
#pragma unroll
              for (int i = 0; i < 32; i++) {
                const uint2 e = rows_sm[i];
                if (i < nrow) {
                  uint16_t hi, lo;
                  tcw_split<BF>(v[i] * __uint_as_float(e.x), hi, lo);
                  const int64_t so = (int64_t)(int32_t)e.y * 64;
                  thi[so] = hi;
                  tlo[so] = lo;
                }
              }
            } else {
              float* const pp = a.part + (int64_t)(d.out_base + row) * 128 + r;
#pragma unroll
              for (int i = 0; i < 32; i++) {
                const uint2 e = rows_sm[i];
                if (i < nrow) pp[(int64_t)i * 128] = v[i] * __uint_as_float(e.x);
              }
            }
            __syncwarp();  // the chunk's rows are read before the next chunk writes them
          } else {
            const int64_t o = (int64_t)d.out_base + row + (int64_t)r * a.ldy;
            const bool act = r < a.nr;
            const int m = (int)(((int64_t)d.out_base + row) & 3);  // o's offset from a 4-element boundary (vec_y)
            if (a.y32) {
              float* const y = static_cast<float*>(a.y);
              if (!vec_y) tcw_store_rows<float, 1, 0>(y, o, nrow, act, v, ts_l, sx);
              else if (m == 0) tcw_store_rows<float, 4, 0>(y, o, nrow, act, v, ts_l, sx);
              else if (m == 1) tcw_store_rows<float, 4, 3>(y, o, nrow, act, v, ts_l, sx);
              else if (m == 2) tcw_store_rows<float, 4, 2>(y, o, nrow, act, v, ts_l, sx);
              else tcw_store_rows<float, 4, 1>(y, o, nrow, act, v, ts_l, sx);
            } else {
              double* const y = static_cast<double*>(a.y);
              if (!vec_y) tcw_store_rows<double, 1, 0>(y, o, nrow, act, v, ts_l, sx);
              else if ((m & 1) == 0) tcw_store_rows<double, 2, 0>(y, o, nrow, act, v, ts_l, sx);
              else tcw_store_rows<double, 2, 1>(y, o, nrow, act, v, ts_l, sx);
            }
          }
        }
        rb += Rb;
      }
      dc = dn;
      Rc = Rn;
      rc = rn;
      dn = dnn;
      Rn = Rnn;
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&accempty[buf]);
    }
  }

  __syncthreads();
  if (tid == 0) {
    // copies issued but never consumed (a role gave up): let them land (bounded)
    // before the shared memory is released
    for (uint32_t c = misc[3]; c < misc[1]; c++) thread_wait(&mfull[c % kTcwSlotsM], (c / kTcwSlotsM) & 1);
    for (uint32_t c = misc[4]; c < misc[2]; c++) thread_wait(&afull[c % kTcwSlotsA], (c / kTcwSlotsA) & 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem_base) : "memory");
  }
}

// ---- per-pass input planes -------------------------------------------------------
// amax[r] = max |X[:, r]| as float bits (FP16 plans scale each right-hand side).
// Grid (blocks per column, columns) with 256 threads: each block reduces its
// share of column r in shared memory and makes one atomic (same-address
// atomics from every warp of many small blocks measured slower than reading X).
constexpr int kTcwAbsmaxThreads = 256;
template <typename TX>
__global__ void __launch_bounds__(kTcwAbsmaxThreads) hmvm_tcw_absmax_kernel(const TX* __restrict__ X, int64_t ldx,
                                                                           int n, unsigned* __restrict__ amax) {
  __shared__ float wm[kTcwAbsmaxThreads / 32];
  const int r = blockIdx.y;
  const TX* __restrict__ col = X + (int64_t)r * ldx;
  const int64_t step = (int64_t)gridDim.x * kTcwAbsmaxThreads;
  float m0 = 0.f, m1 = 0.f, m2 = 0.f, m3 = 0.f;
  int64_t i = blockIdx.x * (int64_t)kTcwAbsmaxThreads + threadIdx.x;
  for (; i + 3 * step < n; i += 4 * step) {  // four independent loads in flight
    m0 = fmaxf(m0, fabsf((float)col[i]));
    m1 = fmaxf(m1, fabsf((float)col[i + step]));
    m2 = fmaxf(m2, fabsf((float)col[i + 2 * step]));
    m3 = fmaxf(m3, fabsf((float)col[i + 3 * step]));
  }
  for (; i < n; i += step) m0 = fmaxf(m0, fabsf((float)col[i]));
  float m = fmaxf(fmaxf(m0, m1), fmaxf(m2, m3));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = wm[0];
#pragma unroll
    for (int w = 1; w < kTcwAbsmaxThreads / 32; w++) b = fmaxf(b, wm[w]);
    if (b > 0.f) atomicMax(amax + r, __float_as_uint(b));
  }
}

// sigma = 2^(ceil(log2 m) - 15), so |x| / sigma <= 2^15; 1 for m = 0, not finite, or BF16.
template <bool BF>
__device__ __forceinline__ float tcw_sigma(unsigned amax_bits) {
  if (BF) return 1.f;
  const float m = __uint_as_float(amax_bits);
  if (!(m > 0.f) || !isfinite(m)) return 1.f;
  int e;
  const float f = frexpf(m, &e);
  return ldexpf(1.f, (f == 0.5f ? e - 1 : e) - 15);
}

// X (column-major, nr <= 128 columns) -> chunks[4][n][64]: chunk c < 2 holds
// the hi parts of right-hand sides 64c..64c+63 (scaled by 1 / sigma_r), chunk
// 2 + c their lo parts; columns nr..127 are zero.  xscale[r] = sigma_r.  A
// block of 256 threads takes 32 rows: each warp reads whole columns of them
// (coalesced), the hi/lo values meet in shared memory, and the block writes
// the 4 x 32 chunk rows of 128 bytes.
template <typename TX, bool BF>
__global__ void __launch_bounds__(256) hmvm_tcw_xplanes_kernel(const TX* __restrict__ X, int64_t ldx, int n, int nr,
                                                               const unsigned* __restrict__ amax,
                                                               float* __restrict__ xscale,
                                                               uint16_t* __restrict__ planes) {
  __shared__ float inv[128];
  __shared__ __align__(16) uint16_t sh[4][32][72];  // chunk, row, right-hand side (+8 to spread the banks)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 128) {
    const float sg = tid < nr ? tcw_sigma<BF>(amax[tid]) : 1.f;
    inv[tid] = 1.f / sg;  // a power of two: exact
    if (blockIdx.x == 0) xscale[tid] = sg;
  }
  __syncthreads();
  for (int64_t i0 = (int64_t)blockIdx.x * 32; i0 < n; i0 += (int64_t)gridDim.x * 32) {
    const int64_t i = i0 + lane;
    for (int c = warp; c < 128; c += 8) {
      const float v = (c < nr && i < n) ? (float)X[i + c * ldx] * inv[c] : 0.f;
      uint16_t hi, lo;
      tcw_split<BF>(v, hi, lo);
      sh[c >> 6][lane][c & 63] = hi;
      sh[2 + (c >> 6)][lane][c & 63] = lo;
    }
    __syncthreads();
    for (int u = tid; u < 4 * 32 * 8; u += 256) {
      const int ch = u >> 8, row = (u >> 3) & 31, part = u & 7;
      if (i0 + row < n)
        reinterpret_cast<uint4*>(planes)[((int64_t)ch * n + i0 + row) * 8 + part] =
            *reinterpret_cast<const uint4*>(&sh[ch][row][part * 8]);
    }
    __syncthreads();
  }
}

// V-stage panels cut into parts: add each t slot's parts in part order and
// write the sum as hi/lo planes.  red[e] = {slot, first partial row, parts, stride}.
template <bool BF>
__global__ void hmvm_tcw_reduce_kernel(const int4* __restrict__ red, int n, const float* __restrict__ part,
                                       uint16_t* __restrict__ tplanes, int64_t trows) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (int64_t)n * 128;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(k >> 7), r = (int)(k & 127);
    const int4 rd = red[e];
    float s = 0.f;
    for (int q = 0; q < rd.z; q++) s += part[(int64_t)(rd.y + q * rd.w) * 128 + r];
    uint16_t hi, lo;
    tcw_split<BF>(s, hi, lo);
    tplanes[((int64_t)(r >> 6) * trows + rd.x) * 64 + (r & 63)] = hi;
    tplanes[((int64_t)(2 + (r >> 6)) * trows + rd.x) * 64 + (r & 63)] = lo;
  }
}

}  // namespace hmvm
