// CUDA-core kernels of the learned preconditioner's U-Net: input packing,
// output head, average pooling / nearest upsampling and their adjoints, the
// training loss, weight gradients of the 3x3x3 convolutions (FP32
// accumulation), deterministic reductions and Adam.  The convolutions
// themselves run on tensor cores (fs_conv.cuh).
//
// Volumes are BF16 channels-last on a one-voxel zero halo (see fs_conv.cuh);
// a "slice" is channels [off, off + c) of a volume with ctot channels.
// Every kernel here writes interior voxels only, so halos stay zero.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fs_common.cuh"
#include "fs_conv.cuh"

namespace fs {

__device__ __forceinline__ long long vol_row(const ConvGeom& g, int b, int i, int j, int k) {
  return (long long)b * g.V + ((long long)(i + 1) * g.Yp + (j + 1)) * g.Zp + (k + 1);
}

__device__ __forceinline__ void load8(const __nv_bfloat16* p, float (&v)[8]) {
  uint4 raw = *(const uint4*)p;
  const __nv_bfloat16* h = (const __nv_bfloat16*)&raw;
#pragma unroll
  for (int e = 0; e < 8; ++e) v[e] = __bfloat162float(h[e]);
}

__device__ __forceinline__ void store8(__nv_bfloat16* p, const float (&v)[8]) {
  uint4 raw;
  __nv_bfloat16* h = (__nv_bfloat16*)&raw;
#pragma unroll
  for (int e = 0; e < 8; ++e) h[e] = __float2bfloat16_rn(v[e]);
  *(uint4*)p = raw;
}

// Network input: channel 0 = rhs / scale, 1..3 = equilibrated masses of the
// +x, +y, +z edges, 4 = 1 on fixed (non-free) nodes, 5..15 = 0.
// rhs[b, n] at rhs + b*rhs_sb + n*rhs_sn; the +x, +y, +z masses of sample b
// at emx/emy/emz + b*em_sb + n; label at lab + b*lab_sb + n.
__global__ void k_unet_pack(ConvGeom g, int batch, const float* __restrict__ rhs,
                            long long rhs_sn, long long rhs_sb, const float* __restrict__ emx,
                            const float* __restrict__ emy, const float* __restrict__ emz,
                            long long em_sb, const uint8_t* __restrict__ lab, long long lab_sb,
                            const float* __restrict__ inv_scale, __nv_bfloat16* __restrict__ in0) {
  const long long N = (long long)g.X * g.Y * g.Z;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N * batch;
       idx += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(idx / N);
    const long long n = idx % N;
    const int k = (int)(n % g.Z), j = (int)((n / g.Z) % g.Y), i = (int)(n / ((long long)g.Y * g.Z));
    const bool fixed = lab[b * lab_sb + n] != FS_LABEL_FREE;
    float v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    v[0] = fixed ? 0.0f : rhs[b * rhs_sb + n * rhs_sn] * inv_scale[b];
    v[1] = emx[b * em_sb + n];
    v[2] = emy[b * em_sb + n];
    v[3] = emz[b * em_sb + n];
    v[4] = fixed ? 1.0f : 0.0f;
    __nv_bfloat16* dst = in0 + vol_row(g, b, i, j, k) * 16;
    store8(dst, v);
    const float z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    store8(dst + 8, z);
  }
}

// Output head (1x1 convolution 16 -> 1, FP32): out[b, n] = mult[b] *
// (bias + sum_c w[c] d0[c]) on free nodes, 0 on fixed ones.
__global__ void k_unet_head(ConvGeom g, int batch, const __nv_bfloat16* __restrict__ d0,
                            const float* __restrict__ w, const uint8_t* __restrict__ lab,
                            long long lab_sb, const float* __restrict__ mult,
                            float* __restrict__ out, long long out_sn, long long out_sb) {
  const long long N = (long long)g.X * g.Y * g.Z;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N * batch;
       idx += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(idx / N);
    const long long n = idx % N;
    const int k = (int)(n % g.Z), j = (int)((n / g.Z) % g.Y), i = (int)(n / ((long long)g.Y * g.Z));
    float a[8], c[8];
    const __nv_bfloat16* src = d0 + vol_row(g, b, i, j, k) * 16;
    load8(src, a);
    load8(src + 8, c);
    float s = w[16];
#pragma unroll
    for (int e = 0; e < 8; ++e) s += w[e] * a[e] + w[8 + e] * c[e];
    const bool fixed = lab[b * lab_sb + n] != FS_LABEL_FREE;
    out[b * out_sb + n * out_sn] = fixed ? 0.0f : s * mult[b];
  }
}

// Per-sample sums of squares, stage 1: partial[blk][b] over a node range.
__global__ void k_unet_sumsq(long long N, int batch, const float* __restrict__ x, long long sn,
                             long long sb, const uint8_t* __restrict__ lab, long long lab_sb,
                             float* __restrict__ partial) {
  __shared__ float red[256];
  for (int b = 0; b < batch; ++b) {
    float s = 0.0f;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
         n += (long long)gridDim.x * blockDim.x) {
      if (lab && lab[b * lab_sb + n] != FS_LABEL_FREE) continue;
      const float v = x[b * sb + n * sn];
      s += v * v;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * batch + b] = red[0];
    __syncthreads();
  }
}

// Stage 2 (one block): scale[b] = sqrt(sum / N), inv[b] = 1/scale (0 if 0).
// With tnorm != NULL instead: tnorm[b] = sum * inv[b]^2 (normalised target).
__global__ void k_unet_scale(int nblk, int batch, long long N, const float* __restrict__ partial,
                             float* __restrict__ scale, float* __restrict__ inv,
                             float* __restrict__ tnorm) {
  for (int b = threadIdx.x; b < batch; b += blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < nblk; ++k) s += partial[(size_t)k * batch + b];
    if (tnorm) {
      tnorm[b] = (float)(s * (double)inv[b] * (double)inv[b]);
      continue;
    }
    const double r = sqrt(s / (double)N);
    scale[b] = (float)r;
    inv[b] = r > 0.0 ? (float)(1.0 / r) : 0.0f;
  }
}

// Average pooling 2x2x2 (ceil): dst (coarse) = mean of the existing children.
__global__ void k_unet_pool(ConvGeom gf, ConvGeom gc, int batch, const __nv_bfloat16* __restrict__ src,
                            int ctot_s, int off_s, __nv_bfloat16* __restrict__ dst, int ctot_d,
                            int off_d, int c) {
  const int c8 = c / 8;
  const long long Nc = (long long)gc.X * gc.Y * gc.Z;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < Nc * batch * c8;
       idx += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(idx % c8);
    const long long t = idx / c8;
    const int b = (int)(t / Nc);
    const long long n = t % Nc;
    const int K = (int)(n % gc.Z), J = (int)((n / gc.Z) % gc.Y), I = (int)(n / ((long long)gc.Y * gc.Z));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int cnt = 0;
    for (int a = 0; a < 2; ++a)
      for (int bb = 0; bb < 2; ++bb)
        for (int e = 0; e < 2; ++e) {
          const int i = 2 * I + a, j = 2 * J + bb, k = 2 * K + e;
          if (i >= gf.X || j >= gf.Y || k >= gf.Z) continue;
          float v[8];
          load8(src + vol_row(gf, b, i, j, k) * ctot_s + off_s + 8 * q, v);
#pragma unroll
          for (int z = 0; z < 8; ++z) acc[z] += v[z];
          ++cnt;
        }
    const float r = 1.0f / (float)cnt;
#pragma unroll
    for (int z = 0; z < 8; ++z) acc[z] *= r;
    store8(dst + vol_row(gc, b, I, J, K) * ctot_d + off_d + 8 * q, acc);
  }
}

// Adjoint of the pooling, accumulated through a ReLU mask:
// dst_f[child] += src_c[parent] / count(parent) * (act_f[child] > 0).
__global__ void k_unet_pool_bwd(ConvGeom gf, ConvGeom gc, int batch,
                                const __nv_bfloat16* __restrict__ src, int ctot_s, int off_s,
                                const __nv_bfloat16* __restrict__ act, int ctot_a, int off_a,
                                __nv_bfloat16* __restrict__ dst, int ctot_d, int off_d, int c) {
  const int c8 = c / 8;
  const long long Nf = (long long)gf.X * gf.Y * gf.Z;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < Nf * batch * c8;
       idx += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(idx % c8);
    const long long t = idx / c8;
    const int b = (int)(t / Nf);
    const long long n = t % Nf;
    const int k = (int)(n % gf.Z), j = (int)((n / gf.Z) % gf.Y), i = (int)(n / ((long long)gf.Y * gf.Z));
    const int I = i / 2, J = j / 2, K = k / 2;
    const int cnt = (2 * I + 1 < gf.X ? 2 : 1) * (2 * J + 1 < gf.Y ? 2 : 1) * (2 * K + 1 < gf.Z ? 2 : 1);
    float g[8], m[8], o[8];
    load8(src + vol_row(gc, b, I, J, K) * ctot_s + off_s + 8 * q, g);
    const long long row = vol_row(gf, b, i, j, k);
    load8(act + row * ctot_a + off_a + 8 * q, m);
    __nv_bfloat16* dp = dst + row * ctot_d + off_d + 8 * q;
    load8(dp, o);
    const float r = 1.0f / (float)cnt;
#pragma unroll
    for (int z = 0; z < 8; ++z) o[z] += m[z] > 0.0f ? g[z] * r : 0.0f;
    store8(dp, o);
  }
}

// Nearest upsampling: dst_f[i, j, k] = src_c[i/2, j/2, k/2].
__global__ void k_unet_up(ConvGeom gf, ConvGeom gc, int batch, const __nv_bfloat16* __restrict__ src,
                          int ctot_s, int off_s, __nv_bfloat16* __restrict__ dst, int ctot_d,
                          int off_d, int c) {
  const int c8 = c / 8;
  const long long Nf = (long long)gf.X * gf.Y * gf.Z;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < Nf * batch * c8;
       idx += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(idx % c8);
    const long long t = idx / c8;
    const int b = (int)(t / Nf);
    const long long n = t % Nf;
    const int k = (int)(n % gf.Z), j = (int)((n / gf.Z) % gf.Y), i = (int)(n / ((long long)gf.Y * gf.Z));
    float v[8];
    load8(src + vol_row(gc, b, i / 2, j / 2, k / 2) * ctot_s + off_s + 8 * q, v);
    store8(dst + vol_row(gf, b, i, j, k) * ctot_d + off_d + 8 * q, v);
  }
}

// Adjoint of the upsampling: dst_c[I, J, K] = sum of the children's src_f.
__global__ void k_unet_up_bwd(ConvGeom gf, ConvGeom gc, int batch,
                              const __nv_bfloat16* __restrict__ src, int ctot_s, int off_s,
                              __nv_bfloat16* __restrict__ dst, int ctot_d, int off_d, int c) {
  const int c8 = c / 8;
  const long long Nc = (long long)gc.X * gc.Y * gc.Z;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < Nc * batch * c8;
       idx += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(idx % c8);
    const long long t = idx / c8;
    const int b = (int)(t / Nc);
    const long long n = t % Nc;
    const int K = (int)(n % gc.Z), J = (int)((n / gc.Z) % gc.Y), I = (int)(n / ((long long)gc.Y * gc.Z));
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int a = 0; a < 2; ++a)
      for (int bb = 0; bb < 2; ++bb)
        for (int e = 0; e < 2; ++e) {
          const int i = 2 * I + a, j = 2 * J + bb, k = 2 * K + e;
          if (i >= gf.X || j >= gf.Y || k >= gf.Z) continue;
          float v[8];
          load8(src + vol_row(gf, b, i, j, k) * ctot_s + off_s + 8 * q, v);
#pragma unroll
          for (int z = 0; z < 8; ++z) acc[z] += v[z];
        }
    store8(dst + vol_row(gc, b, I, J, K) * ctot_d + off_d + 8 * q, acc);
  }
}

// Training loss stage 1: out in normalised units, tgt in original units
// (normalised by inv[b]), planar [b][n]; per sample sum (out - tgt*inv)^2
// on free nodes -> partial[blk][b].
__global__ void k_unet_loss_partial(long long N, int batch, const float* __restrict__ out,
                                    const float* __restrict__ tgt, const float* __restrict__ inv,
                                    const uint8_t* __restrict__ lab,
                                    float* __restrict__ partial) {
  __shared__ float red[256];
  for (int b = 0; b < batch; ++b) {
    float s = 0.0f;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
         n += (long long)gridDim.x * blockDim.x) {
      if (lab[b * N + n] != FS_LABEL_FREE) continue;
      const float d = out[b * N + n] - tgt[b * N + n] * inv[b];
      s += d * d;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * batch + b] = red[0];
    __syncthreads();
  }
}

// Loss stage 2 (one block): loss = mean_b sum_b / tnorm_b (tnorm = sum tgt^2).
__global__ void k_unet_loss_final(int nblk, int batch, const float* __restrict__ partial,
                                  const float* __restrict__ tnorm, float* __restrict__ loss) {
  if (threadIdx.x == 0) {
    double l = 0.0;
    for (int b = 0; b < batch; ++b) {
      double s = 0.0;
      for (int k = 0; k < nblk; ++k) s += partial[(size_t)k * batch + b];
      l += tnorm[b] > 0.0f ? s / tnorm[b] : 0.0;
    }
    *loss = (float)(l / batch);
  }
}

// dL/d(head output) = 2 (out - tgt) / (batch * tnorm_b) on free nodes, then
// back through the head: g_d0[c] = w[c] dout (d0 > 0), and the head's own
// weight gradient partials (16 weights + bias) per block.
__global__ void k_unet_head_bwd(ConvGeom g, int batch, const float* __restrict__ out,
                                const float* __restrict__ tgt, const float* __restrict__ inv,
                                const uint8_t* __restrict__ lab,
                                const float* __restrict__ tnorm, const __nv_bfloat16* __restrict__ d0,
                                const float* __restrict__ w, __nv_bfloat16* __restrict__ gd0,
                                float* __restrict__ partial /* [blk][17] */) {
  const long long N = (long long)g.X * g.Y * g.Z;
  float acc[17];
#pragma unroll
  for (int e = 0; e < 17; ++e) acc[e] = 0.0f;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N * batch;
       idx += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(idx / N);
    const long long n = idx % N;
    const int k = (int)(n % g.Z), j = (int)((n / g.Z) % g.Y), i = (int)(n / ((long long)g.Y * g.Z));
    const long long row = vol_row(g, b, i, j, k);
    float dout = 0.0f;
    if (lab[b * N + n] == FS_LABEL_FREE && tnorm[b] > 0.0f)
      dout = 2.0f * (out[b * N + n] - tgt[b * N + n] * inv[b]) / ((float)batch * tnorm[b]);
    float a[8], c[8];
    load8(d0 + row * 16, a);
    load8(d0 + row * 16 + 8, c);
    float ga[8], gc[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      acc[e] += dout * a[e];
      acc[8 + e] += dout * c[e];
      ga[e] = a[e] > 0.0f ? w[e] * dout : 0.0f;
      gc[e] = c[e] > 0.0f ? w[8 + e] * dout : 0.0f;
    }
    acc[16] += dout;
    store8(gd0 + row * 16, ga);
    store8(gd0 + row * 16 + 8, gc);
  }
  __shared__ float red[256];
  for (int e = 0; e < 17; ++e) {
    red[threadIdx.x] = acc[e];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * 17 + e] = red[0];
    __syncthreads();
  }
}

// Weight gradient of one 3x3x3 convolution (FP32 accumulation on CUDA cores):
//   dW[t][co][ci] = sum_rows dY[r][co] X[r + off_t][ci],  db[co] = sum_rows dY[r][co]
// Block (tap t = blockIdx.y, row group blockIdx.x), 256 threads as 16 x 16
// (co lane, ci lane), each thread a CO x CI register block.  Per-group
// partials, summed in a fixed order by k_sum_groups.
constexpr int kWgRows = 32;

template <int CO, int CI>
__global__ void __launch_bounds__(256)
    k_conv_wgrad(ConvGeom g, const __nv_bfloat16* __restrict__ x, int ctot_x, int off_x,
                 const __nv_bfloat16* __restrict__ dy, int ctot_y, int off_y, long long rows_per,
                 float* __restrict__ pw /* [G][27][cout][cin] */,
                 float* __restrict__ pb /* [G][cout] */) {
  constexpr int cout = CO * 16, cin = CI * 16;
  __shared__ float sy[kWgRows][cout];
  __shared__ float sx[kWgRows][cin];
  const int t = blockIdx.y;
  const long long off = (long long)(t / 9 - 1) * g.S + (long long)((t / 3) % 3 - 1) * g.Zp + (t % 3 - 1);
  const int tco = threadIdx.x / 16, tci = threadIdx.x % 16;
  float acc[CO][CI];
  float bacc[CO];
#pragma unroll
  for (int a = 0; a < CO; ++a) {
    bacc[a] = 0.0f;
#pragma unroll
    for (int b = 0; b < CI; ++b) acc[a][b] = 0.0f;
  }
  const long long r_begin = (long long)blockIdx.x * rows_per;
  const long long r_end = min(g.R, r_begin + rows_per);
  for (long long r0 = r_begin; r0 < r_end; r0 += kWgRows) {
    // stage kWgRows rows of dY and the tap-shifted rows of X (as FP32)
    for (int e = threadIdx.x; e < kWgRows * cout; e += 256) {
      const int rr = e / cout, c = e % cout;
      const long long r = r0 + rr;
      float v = 0.0f;
      if (r < r_end) v = __bfloat162float(dy[r * ctot_y + off_y + c]);
      sy[rr][c] = v;
    }
    for (int e = threadIdx.x; e < kWgRows * cin; e += 256) {
      const int rr = e / cin, c = e % cin;
      const long long r = r0 + rr + off;
      float v = 0.0f;
      if (r0 + rr < r_end && r >= 0 && r < g.R) v = __bfloat162float(x[r * ctot_x + off_x + c]);
      sx[rr][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < kWgRows; ++rr) {
      float yv[CO], xv[CI];
#pragma unroll
      for (int a = 0; a < CO; ++a) yv[a] = sy[rr][tco + 16 * a];
#pragma unroll
      for (int b = 0; b < CI; ++b) xv[b] = sx[rr][tci + 16 * b];
#pragma unroll
      for (int a = 0; a < CO; ++a) {
        bacc[a] += yv[a];
#pragma unroll
        for (int b = 0; b < CI; ++b) acc[a][b] += yv[a] * xv[b];
      }
    }
    __syncthreads();
  }
  float* dst = pw + ((size_t)blockIdx.x * 27 + t) * cout * cin;
#pragma unroll
  for (int a = 0; a < CO; ++a)
#pragma unroll
    for (int b = 0; b < CI; ++b) dst[(tco + 16 * a) * cin + tci + 16 * b] = acc[a][b];
  if (t == 13 && tci == 0) {
#pragma unroll
    for (int a = 0; a < CO; ++a) pb[(size_t)blockIdx.x * cout + tco + 16 * a] = bacc[a];
  }
}

// out[e] = sum_g part[g * n + e] (fixed order).
__global__ void k_sum_groups(long long n, int groups, const float* __restrict__ part,
                             float* __restrict__ out) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int gi = 0; gi < groups; ++gi) s += part[(size_t)gi * n + e];
    out[e] = s;
  }
}

// Adam on FP32 master parameters; c1 = 1 / (1 - b1^t), c2 = 1 / (1 - b2^t).
__global__ void k_adam(long long n, float* __restrict__ w, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.0f - b1) * gg;
    const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    w[e] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
  }
}

}  // namespace fs
