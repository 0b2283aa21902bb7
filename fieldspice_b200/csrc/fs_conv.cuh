// 3x3x3 convolution on 5th-generation tensor cores (tcgen05, sm_100a).
//
// Activations are BF16, channels-last, on a zero halo of one voxel:
//   x[b][i][j][k][c], i in [0, X+2), j in [0, Y+2), k in [0, Z+2),
// flattened to rows r = ((b*Xp + i)*Yp + j)*Zp + k of C_total channels.
// In that layout the input row of tap (dx, dy, dz) for output row r is
// r + dx*Yp*Zp + dy*Zp + dz, so the convolution is an implicit GEMM
//   D[r][co] = sum_taps sum_ci X[r + off_t][ci] * W[t][co][ci]
// whose A operand for a tap is a contiguous window of rows shifted by off_t.
//
// One CTA computes T tiles of 128 consecutive output rows.  Per x-offset dx
// it stages, with 2-D TMA tensor loads (no multicast), the window of rows
// [m0 + dx*S - Zp - 1, m0 + 128T + dx*S + Zp + 1) of the C_in channels,
// 8 channels (16 B) per column, so every (dy, dz) tap of that dx is the same
// window at a row offset: a descriptor start address +16 B per row.  Weights
// arrive pre-packed in their shared-memory image with one bulk copy.  One
// thread issues tcgen05.mma (M = 128, N = C_out, K = 16, BF16 x BF16 -> FP32)
// into tensor memory, commits to an mbarrier, and the four warps read the
// accumulators back (tcgen05.ld), add the bias, apply ReLU and/or a ReLU
// mask, zero the halo rows and store BF16.  Output halo rows are always
// written as zeros, which keeps the zero-halo invariant for the next layer.
//
// Small layers keep all 27 taps' operands resident (one phase); large ones
// run three phases, one per dx, reusing the shared memory.  Every wait is
// bounded; on a timeout the CTA records an error, waits again (bounded) for
// its own transfers, frees its tensor memory and returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fs_tc.cuh"
#include "fs_tma.cuh"

namespace fs {

struct ConvGeom {
  int X, Y, Z;          // interior voxels per batch element
  int Xp, Yp, Zp;       // padded (X + 2, ...)
  long long S;          // Yp * Zp (row distance of dx = 1)
  long long V;          // Xp * Yp * Zp (rows per batch element)
  long long R;          // batch * V
};

struct ConvArgs {
  ConvGeom g;
  int cin, cin_off;     // channels read from the input buffer
  int cout;             // output channels (multiple of 16, <= 128)
  const uint16_t* wpack;  // BF16 image [27][cin/8][cout][8]
  const float* bias;      // [cout] or null
  __nv_bfloat16* out;
  int out_stride, out_off;
  const __nv_bfloat16* mask;  // optional: result *= (mask > 0)
  int mask_stride, mask_off;
  int relu;
  int accumulate;       // out += result
  int T;                // 128-row tiles per CTA
  int W;                // staged window rows (a multiple of BR)
  int BR;               // rows per TMA box (<= 256, multiple of 8)
  int phases;           // 1: all taps resident; 3: one dx per phase
  int nst;              // window ring stages of the persistent kernel (2..4)
  int* error;
};

constexpr long long kConvBudget = 4000000000LL;  // ~2 s of SM clocks

__device__ __forceinline__ uint32_t tmem_cols(int n) {
  uint32_t c = 32;
  while ((int)c < n) c <<= 1;
  return c;
}

// The kernels are defined in exactly one translation unit (fs_net.cu).
#ifdef FS_CONV_DEFINE_KERNELS
__global__ void __launch_bounds__(128)
    k_conv3d_tc(const __grid_constant__ CUtensorMap xmap, ConvArgs a) {
  extern __shared__ uint8_t conv_smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)conv_smem_raw + 1023) & ~(uintptr_t)1023);
  const int nch = a.cin >> 3;
  const int ndx = a.phases == 1 ? 3 : 1;  // windows resident per phase
  const uint32_t colb = (uint32_t)a.W * 16u;
  uint8_t* A = smem;
  uint8_t* Bw = A + (size_t)ndx * nch * colb;
  const uint32_t wtap = (uint32_t)nch * a.cout * 16u;  // one tap's weights
  const int ntap_res = a.phases == 1 ? 27 : 9;
  uint64_t* bars = (uint64_t*)(Bw + (size_t)ntap_res * wtap);
  uint32_t* tslot = (uint32_t*)(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.x * 128LL * a.T;
  const uint32_t ncols = tmem_cols(a.T * a.cout);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tc_alloc(tslot, ncols);
    tc_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t idesc = umma_idesc_bf16(128, a.cout);
  const int nseg = a.W / a.BR;
  bool ok = true;
  int issued = 0;  // phases whose loads were issued (thread 0)
  int mmas = 0;    // phases whose MMAs were committed (thread 0)
  for (int ph = 0; ph < a.phases && ok; ++ph) {
    if (tid == 0) {
      const int dx0 = a.phases == 1 ? 0 : ph;
      mbar_arrive_expect_tx(&bars[0], (uint32_t)ndx * nch * colb + ntap_res * wtap);
      bulk_load(Bw, a.wpack + (size_t)(a.phases == 1 ? 0 : ph * 9) * (wtap / 2),
                ntap_res * wtap, &bars[0]);
      for (int w = 0; w < ndx; ++w) {
        const long long r0 = m0 + (long long)(dx0 + w - 1) * a.g.S - a.g.Zp - 1;
        for (int c = 0; c < nch; ++c)
          for (int sg = 0; sg < nseg; ++sg)
            tma_load_2d(A + (size_t)(w * nch + c) * colb + (size_t)sg * a.BR * 16, &xmap,
                        &bars[0], a.cin_off + 8 * c, (int)(r0 + (long long)sg * a.BR));
      }
      issued = ph + 1;
    }
    ok = mbar_wait_bounded(&bars[0], ph & 1, kConvBudget);
    ok = __syncthreads_and(ok);
    if (!ok) break;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t abase = smem_u32(A), bbase = smem_u32(Bw);
      for (int j = 0; j < a.T; ++j) {
        for (int tl = 0; tl < ntap_res; ++tl) {
          const int t = a.phases == 1 ? tl : ph * 9 + tl;
          const int w = a.phases == 1 ? t / 9 : 0;
          const int dy = (t / 3) % 3, dz = t % 3;
          const uint32_t rowoff = (uint32_t)(j * 128 + dy * a.g.Zp + dz) * 16u;
          for (int s = 0; s < (a.cin >> 4); ++s) {
            const uint64_t ad =
                umma_desc(abase + (uint32_t)(w * nch + 2 * s) * colb + rowoff, colb, 128);
            const uint64_t bd =
                umma_desc(bbase + (uint32_t)tl * wtap + (uint32_t)(2 * s * a.cout) * 16u,
                          (uint32_t)a.cout * 16u, 128);
            const uint32_t acc = (ph > 0 || tl > 0 || s > 0) ? 1u : 0u;
            tc_mma_bf16(tbase + (uint32_t)(j * a.cout), ad, bd, idesc, acc);
          }
        }
      }
      tc_commit(&bars[1]);
      mmas = ph + 1;
    }
    // the operands of this phase stay in use until its MMAs complete
    ok = mbar_wait_bounded(&bars[1], ph & 1, kConvBudget);
    ok = __syncthreads_and(ok);
    tc_fence_after();
  }
  if (ok) {
    for (int j = 0; j < a.T; ++j) {
      const long long row = m0 + (long long)j * 128 + warp * 32 + lane;
      bool interior = false;
      if (row < a.g.R) {
        const long long rr = row % a.g.V;
        const int k = (int)(rr % a.g.Zp);
        const int jj = (int)((rr / a.g.Zp) % a.g.Yp);
        const int i = (int)(rr / a.g.S);
        interior = k >= 1 && k <= a.g.Z && jj >= 1 && jj <= a.g.Y && i >= 1 && i <= a.g.X;
      }
      for (int q = 0; q < (a.cout >> 4); ++q) {
        float v[16];
        tc_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * a.cout + q * 16), v);
        if (row >= a.g.R) continue;
        __nv_bfloat16* dst = a.out + row * a.out_stride + a.out_off + q * 16;
        if (!interior) {
          if (!a.accumulate) {
            uint4 z = make_uint4(0, 0, 0, 0);
            ((uint4*)dst)[0] = z;
            ((uint4*)dst)[1] = z;
          }
          continue;
        }
        if (a.bias) {
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] += __ldg(a.bias + q * 16 + e);
        }
        if (a.relu) {
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] = fmaxf(v[e], 0.0f);
        }
        if (a.mask) {
          const __nv_bfloat16* mp = a.mask + row * a.mask_stride + a.mask_off + q * 16;
          uint4 mraw[2];
          mraw[0] = ((const uint4*)mp)[0];
          mraw[1] = ((const uint4*)mp)[1];
          const __nv_bfloat16* mv = (const __nv_bfloat16*)mraw;
#pragma unroll
          for (int e = 0; e < 16; ++e)
            if (!(__bfloat162float(mv[e]) > 0.0f)) v[e] = 0.0f;
        }
        if (a.accumulate) {
          uint4 oraw[2];
          oraw[0] = ((const uint4*)dst)[0];
          oraw[1] = ((const uint4*)dst)[1];
          const __nv_bfloat16* ov = (const __nv_bfloat16*)oraw;
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] += __bfloat162float(ov[e]);
        }
        uint4 packed[2];
        __nv_bfloat16* pv = (__nv_bfloat16*)packed;
#pragma unroll
        for (int e = 0; e < 16; ++e) pv[e] = __float2bfloat16_rn(v[e]);
        ((uint4*)dst)[0] = packed[0];
        ((uint4*)dst)[1] = packed[1];
      }
    }
  } else {
    // bounded second wait for this CTA's own transfers and MMAs in flight
    if (tid == 0) {
      if (issued > 0) (void)mbar_wait_bounded(&bars[0], (issued - 1) & 1, kConvBudget);
      if (mmas > 0) (void)mbar_wait_bounded(&bars[1], (mmas - 1) & 1, kConvBudget);
    }
    if (tid == 0 && a.error) atomicExch(a.error, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tc_dealloc(tbase, ncols);
}

// ---- persistent, warp-specialised variant ----------------------------------------
// Same implicit GEMM as k_conv3d_tc, for layers whose weights and two window
// stages fit in shared memory.  One CTA per SM loops over 128-row tiles
// (tile = blockIdx.x + i * gridDim.x) with three roles:
//   warp 4 (one thread): TMA producer, fills a 2-stage ring of 3-window tiles;
//   warp 5 (one thread): MMA issuer, 27 x (C_in/16) MMAs per tile into one of
//                        two TMEM accumulators, commits to "stage empty" and
//                        "accumulator full";
//   warps 0-3: epilogue, drain an accumulator (tcgen05.ld), store, release it.
// So the loads of tile i+1, the MMAs of tile i and the epilogue of tile i-1
// overlap.  Weights are loaded once per CTA.  Every wait is bounded; on a
// timeout the thread records an error and stops its role, the others time
// out in turn, and the CTA drains its own transfers before freeing TMEM.
struct Conv2Cfg {
  int W, BR;          // window rows (multiple of BR) and TMA box rows
  size_t smem;
};

constexpr int kConv2Threads = 192;

#ifdef FS_CONV_DEFINE_KERNELS
__global__ void __launch_bounds__(kConv2Threads, 1)
    k_conv3d_tc2(const __grid_constant__ CUtensorMap xmap, ConvArgs a, long long ntiles) {
  extern __shared__ uint8_t conv2_smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)conv2_smem_raw + 1023) & ~(uintptr_t)1023);
  const int nch = a.cin >> 3;
  const uint32_t colb = (uint32_t)a.W * 16u;
  const uint32_t stage_bytes = 3u * nch * colb;
  const int nst = a.nst;
  uint8_t* Aring = smem;                            // nst stages
  uint8_t* Bw = Aring + (size_t)nst * stage_bytes;  // 27 taps
  const uint32_t wtap = (uint32_t)nch * a.cout * 16u;
  uint64_t* bars = (uint64_t*)(Bw + (size_t)27 * wtap);
  uint64_t* full = bars;           // [4] TMA -> MMA
  uint64_t* empty = bars + 4;      // [4] MMA done reading a stage -> TMA
  uint64_t* accfull = bars + 8;    // [2] MMA -> epilogue
  uint64_t* accempty = bars + 10;  // [2] epilogue -> MMA (4 warp arrivals)
  uint64_t* wbar = bars + 12;      // weights
  uint32_t* tslot = (uint32_t*)(bars + 13);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = tmem_cols(2 * a.cout);
  if (tid == 0) {
    for (int i = 0; i < 8; ++i) mbar_init(&bars[i], 1);
    mbar_init(&accfull[0], 1);
    mbar_init(&accfull[1], 1);
    mbar_init(&accempty[0], 4);
    mbar_init(&accempty[1], 4);
    mbar_init(wbar, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tc_alloc(tslot, ncols);
    tc_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const int nseg = a.W / a.BR;
  const long long my_tiles =
      blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  bool ok = true;
  if (warp == 4) {
    // ---- producer -----------------------------------------------------------------
    if (lane == 0) {
      mbar_arrive_expect_tx(wbar, 27u * wtap);
      bulk_load(Bw, a.wpack, 27u * wtap, wbar);
      long long issued = 0;
      for (long long i = 0; i < my_tiles && ok; ++i) {
        const int st = (int)(i % nst);
        if (i >= nst)
          ok = mbar_wait_bounded(&empty[st], (uint32_t)((i / nst - 1) & 1), kConvBudget);
        if (!ok) break;
        const long long m0 = (blockIdx.x + i * gridDim.x) * 128LL;
        mbar_arrive_expect_tx(&full[st], stage_bytes);
        uint8_t* A = Aring + (size_t)st * stage_bytes;
        for (int w = 0; w < 3; ++w) {
          const long long r0 = m0 + (long long)(w - 1) * a.g.S - a.g.Zp - 1;
          for (int c = 0; c < nch; ++c)
            for (int sg = 0; sg < nseg; ++sg)
              tma_load_2d(A + (size_t)(w * nch + c) * colb + (size_t)sg * a.BR * 16, &xmap,
                          &full[st], a.cin_off + 8 * c, (int)(r0 + (long long)sg * a.BR));
        }
        issued = i + 1;
      }
      // drain: the last stages' loads must land before the CTA exits
      for (long long i = (issued > nst ? issued - nst : 0); i < issued; ++i)
        (void)mbar_wait_bounded(&full[i % nst], (uint32_t)((i / nst) & 1), kConvBudget);
      (void)mbar_wait_bounded(wbar, 0, kConvBudget);
      if (!ok && a.error) atomicExch(a.error, 1);
    }
  } else if (warp == 5) {
    // ---- MMA issuer -----------------------------------------------------------------
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_bf16(128, a.cout);
      ok = mbar_wait_bounded(wbar, 0, kConvBudget);
      long long committed = 0;
      for (long long i = 0; i < my_tiles && ok; ++i) {
        const int st = (int)(i % nst), ac = (int)(i & 1);
        ok = mbar_wait_bounded(&full[st], (uint32_t)((i / nst) & 1), kConvBudget);
        if (ok && i >= 2)
          ok = mbar_wait_bounded(&accempty[ac], (uint32_t)(((i >> 1) - 1) & 1), kConvBudget);
        if (!ok) break;
        tc_fence_after();
        const uint32_t abase = smem_u32(Aring + (size_t)st * stage_bytes), bbase = smem_u32(Bw);
        for (int t = 0; t < 27; ++t) {
          const int w = t / 9, dy = (t / 3) % 3, dz = t % 3;
          const uint32_t rowoff = (uint32_t)(dy * a.g.Zp + dz) * 16u;
          for (int s = 0; s < (a.cin >> 4); ++s) {
            const uint64_t ad = umma_desc(abase + (uint32_t)(w * nch + 2 * s) * colb + rowoff, colb, 128);
            const uint64_t bd = umma_desc(bbase + (uint32_t)t * wtap + (uint32_t)(2 * s * a.cout) * 16u,
                                          (uint32_t)a.cout * 16u, 128);
            tc_mma_bf16(tbase + (uint32_t)(ac * a.cout), ad, bd, idesc, (t > 0 || s > 0) ? 1u : 0u);
          }
        }
        tc_commit(&empty[st]);
        tc_commit(&accfull[ac]);
        committed = i + 1;
      }
      // drain: the last MMAs must complete before TMEM is freed
      if (committed > 0)
        (void)mbar_wait_bounded(&accfull[(committed - 1) & 1], (uint32_t)(((committed - 1) >> 1) & 1),
                                kConvBudget);
      if (!ok && a.error) atomicExch(a.error, 1);
    }
  } else {
    // ---- epilogue (warps 0-3, TMEM lanes 32 w .. 32 w + 31) ---------------------------
    for (long long i = 0; i < my_tiles && ok; ++i) {
      const int ac = (int)(i & 1);
      ok = mbar_wait_bounded(&accfull[ac], (uint32_t)((i >> 1) & 1), kConvBudget);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      tc_fence_after();
      const long long row = (blockIdx.x + i * gridDim.x) * 128LL + warp * 32 + lane;
      bool interior = false;
      if (row < a.g.R) {
        const long long rr = row % a.g.V;
        const int k = (int)(rr % a.g.Zp);
        const int jj = (int)((rr / a.g.Zp) % a.g.Yp);
        const int ii = (int)(rr / a.g.S);
        interior = k >= 1 && k <= a.g.Z && jj >= 1 && jj <= a.g.Y && ii >= 1 && ii <= a.g.X;
      }
      for (int q = 0; q < (a.cout >> 4); ++q) {
        float v[16];
        tc_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(ac * a.cout + q * 16), v);
        if (row >= a.g.R) continue;
        __nv_bfloat16* dst = a.out + row * a.out_stride + a.out_off + q * 16;
        if (!interior) {
          if (!a.accumulate) {
            uint4 z = make_uint4(0, 0, 0, 0);
            ((uint4*)dst)[0] = z;
            ((uint4*)dst)[1] = z;
          }
          continue;
        }
        if (a.bias) {
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] += __ldg(a.bias + q * 16 + e);
        }
        if (a.relu) {
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] = fmaxf(v[e], 0.0f);
        }
        if (a.mask) {
          const __nv_bfloat16* mp = a.mask + row * a.mask_stride + a.mask_off + q * 16;
          uint4 mraw[2];
          mraw[0] = ((const uint4*)mp)[0];
          mraw[1] = ((const uint4*)mp)[1];
          const __nv_bfloat16* mv = (const __nv_bfloat16*)mraw;
#pragma unroll
          for (int e = 0; e < 16; ++e)
            if (!(__bfloat162float(mv[e]) > 0.0f)) v[e] = 0.0f;
        }
        if (a.accumulate) {
          uint4 oraw[2];
          oraw[0] = ((const uint4*)dst)[0];
          oraw[1] = ((const uint4*)dst)[1];
          const __nv_bfloat16* ov = (const __nv_bfloat16*)oraw;
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] += __bfloat162float(ov[e]);
        }
        uint4 packed[2];
        __nv_bfloat16* pv = (__nv_bfloat16*)packed;
#pragma unroll
        for (int e = 0; e < 16; ++e) pv[e] = __float2bfloat16_rn(v[e]);
        ((uint4*)dst)[0] = packed[0];
        ((uint4*)dst)[1] = packed[1];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&accempty[ac]);
    }
    if (!ok && lane == 0 && a.error) atomicExch(a.error, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tc_dealloc(tbase, ncols);
}
#endif  // FS_CONV_DEFINE_KERNELS

// Pack FP32 weights w[27][cout][cin] into the BF16 shared-memory image
// [27][cin/8][cout][8]; flip != 0 packs the data-gradient operator instead:
// taps reversed and the channel roles swapped (image [27][cout/8][cin][8]).
__global__ void k_pack_weights(const float* __restrict__ w, int cin, int cout, int flip,
                               uint16_t* __restrict__ out) {
  const long long n = 27LL * cin * cout;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(idx / ((long long)cin * cout));
    const int rem = (int)(idx % ((long long)cin * cout));
    const int co = rem / cin, ci = rem % cin;
    const float v = w[idx];
    long long dst;
    if (!flip) {
      dst = (((long long)t * (cin / 8) + ci / 8) * cout + co) * 8 + (ci & 7);
    } else {
      // operator with K = cout_f channels, N = cin_f rows, tap 26 - t
      dst = (((long long)(26 - t) * (cout / 8) + co / 8) * cin + ci) * 8 + (co & 7);
    }
    __nv_bfloat16 b = __float2bfloat16_rn(v);
    out[dst] = *(uint16_t*)&b;
  }
}
#endif  // FS_CONV_DEFINE_KERNELS

// ---- weight gradient on tensor cores ----------------------------------------------
//   dW[t][co][ci] = sum_r dY[r][co] * X[r + off_t][ci]
// is, per tap, a GEMM whose reduction index is the voxel row r: D[co][ci] +=
// A B^T with A = dY (M = co, K = r) and B = the tap-shifted X (N = ci, K = r).
// In the activation layout a row holds 8 channels per 16 bytes, so both
// operands are MN-major (channels contiguous) and a one-row shift of the tap
// window is +16 bytes of descriptor start address, as in the forward pass.
// A CTA owns `rows_per` rows (a multiple of 128) and a group of taps with the
// same dx (all 9 when 9 * cin columns fit in tensor memory, else the 3 taps of
// one (dx, dy)); per 128-row subtile it stages dY (16 channel groups; groups
// past cout stay zero, so M = 128 always) and the X window covering its taps
// with 2-D TMA loads into a two-stage ring, one thread issues
// ntap * 8 MMAs (M = 128, N = cin, K = 16) accumulating in tensor memory, and
// at the end four warps drain D (lane = co) into the CTA's partial
// pw[blockIdx.x][t][co][ci].  Waits are bounded: on a timeout the CTA records
// an error, waits (bounded) for its own copies and MMAs, frees tensor memory
// and returns.
struct WgradArgs {
  ConvGeom g;
  int cin, cin_off, cout, cout_off;
  int ntap;             // 9 (one dx) or 3 (one dx, dy) per blockIdx.y
  long long rows_per;   // rows per blockIdx.x, a multiple of 128
  int W, BR;            // X window rows (multiple of BR) and TMA box rows
  float* pw;            // [gridDim.x][27][cout][cin]
  int* error;
};

constexpr int kWgradThreads = 128;

#ifdef FS_CONV_DEFINE_KERNELS
__global__ void __launch_bounds__(kWgradThreads, 1)
    k_conv_wgrad_tc(const __grid_constant__ CUtensorMap xmap,
                    const __grid_constant__ CUtensorMap ymap, WgradArgs a) {
  extern __shared__ uint8_t wg_smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)wg_smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr uint32_t kAgrp = 128u * 16u;           // one 8-channel group of 128 rows
  const uint32_t abytes = 16u * kAgrp;             // dY stage: 16 groups (M = 128)
  const int ncx = a.cin >> 3, ncy = a.cout >> 3;
  const uint32_t colb = (uint32_t)a.W * 16u;       // one 8-channel group of the window
  const uint32_t stage = abytes + (uint32_t)ncx * colb;
  uint64_t* full = (uint64_t*)(smem + 2 * stage);  // [2] TMA -> MMA
  uint64_t* done = full + 2;                       // [2] MMA -> stage free
  uint32_t* tslot = (uint32_t*)(done + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long r_begin = (long long)blockIdx.x * a.rows_per;
  const long long r_end = min(a.g.R, r_begin + a.rows_per);
  const int nsub = r_end > r_begin ? (int)((r_end - r_begin + 127) / 128) : 0;
  // taps of this CTA: t = dx*9 + dy*3 + dz; ntap = 9: dx = y; ntap = 3: (dx, dy)
  const int t0 = blockIdx.y * a.ntap;
  const int dx = t0 / 9;
  const uint32_t ncols = tmem_cols(a.ntap * a.cin);
  // zero the dY channel groups past cout in both stages (M is always 128)
  for (uint32_t e = tid; e < (uint32_t)(16 - ncy) * kAgrp / 16u; e += blockDim.x) {
    const uint32_t off = (uint32_t)ncy * kAgrp + e * 16u;
    *(uint4*)(smem + off) = make_uint4(0, 0, 0, 0);
    *(uint4*)(smem + stage + off) = make_uint4(0, 0, 0, 0);
  }
  fence_proxy_async_smem();
  if (tid == 0) {
    for (int i = 0; i < 4; ++i) mbar_init(&full[i], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tc_alloc(tslot, ncols);
    tc_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  bool ok = true;
  int loaded = 0, mma_done = 0;  // subtiles whose loads / MMAs were issued (thread 0)
  if (tid == 0) {
    const uint32_t idesc = umma_idesc_bf16_mn(128, a.cin);
    const int nseg = a.W / a.BR;
    auto issue = [&](int i) {
      uint8_t* st = smem + (size_t)(i & 1) * stage;
      const long long m0 = r_begin + 128LL * i;
      mbar_arrive_expect_tx(&full[i & 1], (uint32_t)ncy * kAgrp + (uint32_t)ncx * colb);
      for (int c = 0; c < ncy; ++c)
        tma_load_2d(st + (size_t)c * kAgrp, &ymap, &full[i & 1], a.cout_off + 8 * c, (int)m0);
      const long long r0 = m0 + (long long)(dx - 1) * a.g.S - a.g.Zp - 1;
      for (int c = 0; c < ncx; ++c)
        for (int sg = 0; sg < nseg; ++sg)
          tma_load_2d(st + abytes + (size_t)c * colb + (size_t)sg * a.BR * 16, &xmap,
                      &full[i & 1], a.cin_off + 8 * c, (int)(r0 + (long long)sg * a.BR));
      loaded = i + 1;
    };
    if (nsub > 0) issue(0);
    for (int i = 0; i < nsub && ok; ++i) {
      if (i + 1 < nsub) {
        // the other stage is free once the MMAs of subtile i - 1 completed
        if (i >= 1) ok = mbar_wait_bounded(&done[(i - 1) & 1], (uint32_t)(((i - 1) >> 1) & 1),
                                           kConvBudget);
        if (!ok) break;
        issue(i + 1);
      }
      ok = mbar_wait_bounded(&full[i & 1], (uint32_t)((i >> 1) & 1), kConvBudget);
      if (!ok) break;
      tc_fence_after();
      const uint32_t sa = smem_u32(smem + (size_t)(i & 1) * stage);
      const uint32_t sb = sa + abytes;
      for (int tl = 0; tl < a.ntap; ++tl) {
        const int t = t0 + tl;
        const int dy = (t / 3) % 3, dz = t % 3;
        const uint32_t woff = (uint32_t)(dy * a.g.Zp + dz) * 16u;
        for (int kk = 0; kk < 8; ++kk) {  // 16 rows per MMA
          const uint64_t ad = umma_desc(sa + (uint32_t)kk * 256u, 128u, kAgrp);
          const uint64_t bd = umma_desc(sb + woff + (uint32_t)kk * 256u, 128u, colb);
          tc_mma_bf16(tbase + (uint32_t)(tl * a.cin), ad, bd, idesc,
                      (i > 0 || kk > 0) ? 1u : 0u);
        }
      }
      tc_commit(&done[i & 1]);
      mma_done = i + 1;
    }
    if (ok && nsub > 0)
      ok = mbar_wait_bounded(&done[(nsub - 1) & 1], (uint32_t)(((nsub - 1) >> 1) & 1),
                             kConvBudget);
    if (!ok) {
      // bounded wait for this CTA's own transfers and MMAs still in flight
      if (loaded > 0)
        (void)mbar_wait_bounded(&full[(loaded - 1) & 1], (uint32_t)(((loaded - 1) >> 1) & 1),
                                kConvBudget);
      if (mma_done > 0)
        (void)mbar_wait_bounded(&done[(mma_done - 1) & 1],
                                (uint32_t)(((mma_done - 1) >> 1) & 1), kConvBudget);
      if (a.error) atomicExch(a.error, 1);
    }
  }
  ok = __syncthreads_and(ok);
  tc_fence_after();
  if (ok) {
    // lane = co; columns tl * cin + ci
    const int co = warp * 32 + lane;
    for (int tl = 0; tl < a.ntap; ++tl) {
      for (int q = 0; q < (a.cin >> 4); ++q) {
        float v[16];
        if (nsub > 0) {
          tc_ld16(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(tl * a.cin + q * 16), v);
        } else {
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] = 0.0f;
        }
        if (co >= a.cout) continue;
        float* dst = a.pw + (((size_t)blockIdx.x * 27 + t0 + tl) * a.cout + co) * a.cin + q * 16;
#pragma unroll
        for (int e = 0; e < 16; e += 4) *(float4*)(dst + e) = make_float4(v[e], v[e + 1], v[e + 2], v[e + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tc_dealloc(tbase, ncols);
}

// Bias gradient partials: pb[blockIdx.x][co] = sum of dY[r][co] over the rows
// of group blockIdx.x (the same row groups as the weight gradient).
__global__ void __launch_bounds__(256)
    k_conv_bgrad(ConvGeom g, const __nv_bfloat16* __restrict__ dy, int ctot, int off, int cout,
                 long long rows_per, float* __restrict__ pb) {
  __shared__ float red[256];
  const long long r_begin = (long long)blockIdx.x * rows_per;
  const long long r_end = min(g.R, r_begin + rows_per);
  const int per = 256 / cout;  // rows handled side by side (cout divides 256 or not: rest idle)
  const int c = threadIdx.x % cout, lane_r = threadIdx.x / cout;
  float acc = 0.0f;
  if (lane_r < per)
    for (long long r = r_begin + lane_r; r < r_end; r += per)
      acc += __bfloat162float(dy[r * ctot + off + c]);
  red[threadIdx.x] = lane_r < per ? acc : 0.0f;
  __syncthreads();
  if (threadIdx.x < cout) {
    float s = 0.0f;
    for (int k = 0; k < per; ++k) s += red[k * cout + threadIdx.x];
    pb[(size_t)blockIdx.x * cout + threadIdx.x] = s;
  }
}
#endif  // FS_CONV_DEFINE_KERNELS

}  // namespace fs
