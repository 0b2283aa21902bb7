// The learned preconditioner's network: a 4-level BF16 3-D U-Net
// (channels 16/32/48/64, two 3x3x3 convolutions per level and side, ReLU,
// 2x2x2 average pooling, nearest upsampling with skip concatenation, a 1x1
// output head), evaluated and trained with this library's kernels: the
// fourteen 3x3x3 convolutions and their data gradients on tcgen05 tensor
// cores (fs_conv.cuh), everything else on CUDA cores (fs_unet_kernels.cuh).
//
// Input (per sample): a residual on the free nodes of one grid level plus the
// level's equilibrated edge masses and fixed-node flags; output: the error
// estimate on that level (0 on fixed nodes).  The residual is normalised by
// its RMS and the output scaled back, so the network sees unit-size inputs
// at every CG iteration.
//
// Parameters: one FP32 vector theta = [W_0 b_0 W_1 b_1 ... W_13 b_13 head],
// W_l[27][cout][cin] (taps (dx, dy, dz), z fastest), b_l[cout], head = 16
// weights + 1 bias.  Training keeps FP32 gradients and Adam moments of theta
// and re-packs the BF16 tensor-core images after every step.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include "fieldspice_b200.h"
#include "fs_common.cuh"
#include "fs_conv.cuh"
#include "fs_net.cuh"
#include "fs_unet_kernels.cuh"

namespace {

constexpr int kNConv = 14;
constexpr int kCin[kNConv] = {16, 16, 16, 32, 32, 48, 48, 64, 112, 48, 80, 32, 48, 16};
constexpr int kCout[kNConv] = {16, 16, 32, 32, 48, 48, 64, 64, 48, 48, 32, 32, 16, 16};
constexpr int kRedBlocks = 256;   // blocks of the per-sample reductions
constexpr int kWgGroups = 24;     // row groups of the weight gradients

long long conv_woff(int l) {
  long long o = 0;
  for (int i = 0; i < l; ++i) o += 27LL * kCin[i] * kCout[i] + kCout[i];
  return o;
}
long long conv_boff(int l) { return conv_woff(l) + 27LL * kCin[l] * kCout[l]; }
long long head_off() { return conv_woff(kNConv); }
long long theta_size() { return head_off() + 17; }
long long max_wgrad_elems() {
  long long m = 0;
  for (int l = 0; l < kNConv; ++l) m = m > 27LL * kCin[l] * kCout[l] ? m : 27LL * kCin[l] * kCout[l];
  return m;
}

struct Vol {
  __nv_bfloat16* p = nullptr;
  int ctot = 0;
  int lev = 0;
};

// Bump allocator over the caller's workspace (256-byte aligned pieces).
struct Bump {
  uint8_t* base;
  size_t off, cap;
  void* take(size_t bytes) {
    off = (off + 255) & ~(size_t)255;
    void* p = base ? base + off : nullptr;
    off += bytes;
    return p;
  }
};

}  // namespace

struct fs_unet {
  int batch = 0, train = 0;
  fs::ConvGeom g[4];
  Vol in0, e0a, cat0, d0a, d0, p1, e1a, cat1, d1a, d1, p2, e2a, cat2, d2a, d2, p3, e3a, e3;
  Vol g_e0a, g_cat0, g_d0a, g_d0, g_p1, g_e1a, g_cat1, g_d1a, g_d1, g_p2, g_e2a, g_cat2, g_d2a,
      g_d2, g_p3, g_e3a, g_e3;
  float* theta = nullptr;  // caller-owned master parameters
  uint16_t* wfwd[kNConv] = {};
  uint16_t* wbwd[kNConv] = {};
  float *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  float *red = nullptr, *pw = nullptr, *pb = nullptr, *ph = nullptr;
  float *scale = nullptr, *inv = nullptr, *tnorm = nullptr, *ones = nullptr, *loss = nullptr;
  float* out_n = nullptr;
  int* err = nullptr;
  long long step = 0;
};

namespace {

fs::ConvGeom level_geom(int batch, int X, int Y, int Z, int l) {
  for (int i = 0; i < l; ++i) {
    X = (X + 1) / 2;
    Y = (Y + 1) / 2;
    Z = (Z + 1) / 2;
  }
  return fs::conv_geom(batch, X, Y, Z);
}

size_t vol_bytes(const fs::ConvGeom& g, int c) { return (size_t)g.R * c * 2; }

// Lay out every buffer; with base == nullptr only the size is computed.
size_t layout(fs_unet* U, uint8_t* base, int X, int Y, int Z, int batch, int train) {
  Bump a{base, 0, 0};
  for (int l = 0; l < 4; ++l) U->g[l] = level_geom(batch, X, Y, Z, l);
  auto vol = [&](Vol& v, int lev, int c) {
    v.ctot = c;
    v.lev = lev;
    v.p = (__nv_bfloat16*)a.take(vol_bytes(U->g[lev], c));
  };
  vol(U->in0, 0, 16);
  vol(U->e0a, 0, 16);
  vol(U->cat0, 0, 48);
  vol(U->d0a, 0, 16);
  vol(U->d0, 0, 16);
  vol(U->p1, 1, 16);
  vol(U->e1a, 1, 32);
  vol(U->cat1, 1, 80);
  vol(U->d1a, 1, 32);
  vol(U->d1, 1, 32);
  vol(U->p2, 2, 32);
  vol(U->e2a, 2, 48);
  vol(U->cat2, 2, 112);
  vol(U->d2a, 2, 48);
  vol(U->d2, 2, 48);
  vol(U->p3, 3, 48);
  vol(U->e3a, 3, 64);
  vol(U->e3, 3, 64);
  for (int l = 0; l < kNConv; ++l) U->wfwd[l] = (uint16_t*)a.take(27LL * kCin[l] * kCout[l] * 2);
  const long long N0 = (long long)U->g[0].X * U->g[0].Y * U->g[0].Z;
  U->red = (float*)a.take(sizeof(float) * (size_t)kRedBlocks * (batch > 17 ? batch : 17));
  U->scale = (float*)a.take(sizeof(float) * batch);
  U->inv = (float*)a.take(sizeof(float) * batch);
  U->tnorm = (float*)a.take(sizeof(float) * batch);
  U->ones = (float*)a.take(sizeof(float) * batch);
  U->loss = (float*)a.take(sizeof(float) * 4);
  U->err = (int*)a.take(sizeof(int) * 4);
  if (train) {
    vol(U->g_e0a, 0, 16);
    vol(U->g_cat0, 0, 48);
    vol(U->g_d0a, 0, 16);
    vol(U->g_d0, 0, 16);
    vol(U->g_p1, 1, 16);
    vol(U->g_e1a, 1, 32);
    vol(U->g_cat1, 1, 80);
    vol(U->g_d1a, 1, 32);
    vol(U->g_d1, 1, 32);
    vol(U->g_p2, 2, 32);
    vol(U->g_e2a, 2, 48);
    vol(U->g_cat2, 2, 112);
    vol(U->g_d2a, 2, 48);
    vol(U->g_d2, 2, 48);
    vol(U->g_p3, 3, 48);
    vol(U->g_e3a, 3, 64);
    vol(U->g_e3, 3, 64);
    for (int l = 0; l < kNConv; ++l) U->wbwd[l] = (uint16_t*)a.take(27LL * kCin[l] * kCout[l] * 2);
    const long long nt = theta_size();
    U->grad = (float*)a.take(sizeof(float) * nt);
    U->adam_m = (float*)a.take(sizeof(float) * nt);
    U->adam_v = (float*)a.take(sizeof(float) * nt);
    U->pw = (float*)a.take(sizeof(float) * (size_t)kWgGroups * max_wgrad_elems());
    U->pb = (float*)a.take(sizeof(float) * (size_t)kWgGroups * 64);
    U->ph = (float*)a.take(sizeof(float) * (size_t)kRedBlocks * 17);
    U->out_n = (float*)a.take(sizeof(float) * (size_t)N0 * batch);
  }
  return a.off + 256;
}

int blocks_for(long long n) {
  long long b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 16) b = 148 * 16;
  return (int)b;
}

int pack_all(fs_unet* U, cudaStream_t s) {
  int st;
  for (int l = 0; l < kNConv; ++l) {
    if ((st = fs::pack_weights(U->theta + conv_woff(l), kCin[l], kCout[l], 0, U->wfwd[l], s)) != FS_OK)
      return st;
    if (U->train &&
        (st = fs::pack_weights(U->theta + conv_woff(l), kCin[l], kCout[l], 1, U->wbwd[l], s)) != FS_OK)
      return st;
  }
  return FS_OK;
}

int conv(fs_unet* U, int l, const Vol& x, int xoff, const Vol& y, int yoff, cudaStream_t s) {
  fs::ConvIO io;
  io.x = x.p;
  io.ctot_in = x.ctot;
  io.cin_off = xoff;
  io.cin = kCin[l];
  io.wpack = U->wfwd[l];
  io.bias = U->theta + conv_boff(l);
  io.out = y.p;
  io.ctot_out = y.ctot;
  io.out_off = yoff;
  io.cout = kCout[l];
  io.relu = 1;
  io.error = U->err;
  return fs::conv_launch(U->g[x.lev], io, s);
}

// Data gradient of conv l: dx[xoff..] = W^T dy[yoff..] (times mask > 0).
int conv_dgrad(fs_unet* U, int l, const Vol& dy, int yoff, const Vol& dx, int xoff,
               const Vol* mask, int moff, cudaStream_t s) {
  fs::ConvIO io;
  io.x = dy.p;
  io.ctot_in = dy.ctot;
  io.cin_off = yoff;
  io.cin = kCout[l];
  io.wpack = U->wbwd[l];
  io.bias = nullptr;
  io.out = dx.p;
  io.ctot_out = dx.ctot;
  io.out_off = xoff;
  io.cout = kCin[l];
  if (mask) {
    io.mask = mask->p;
    io.ctot_mask = mask->ctot;
    io.mask_off = moff;
  }
  io.relu = 0;
  io.error = U->err;
  return fs::conv_launch(U->g[dy.lev], io, s);
}

template <int CO, int CI>
void wgrad_launch(const fs::ConvGeom& g, const Vol& x, int xoff, const Vol& dy, int yoff,
                  long long rows_per, float* pw, float* pb, cudaStream_t s) {
  dim3 grid(kWgGroups, 27);
  fs::k_conv_wgrad<CO, CI><<<grid, 256, 0, s>>>(g, x.p, x.ctot, xoff, dy.p, dy.ctot, yoff,
                                                rows_per, pw, pb);
}

// The weight gradient of training: on tensor cores unless FS_WGRAD=cuda
// selects the CUDA-core kernel.
bool wgrad_on_cuda_cores() {
  const char* sel = getenv("FS_WGRAD");
  return sel && strcmp(sel, "cuda") == 0;
}

// Weight and bias gradient of conv l into U->grad.
int conv_wgrad(fs_unet* U, int l, const Vol& x, int xoff, const Vol& dy, int yoff,
               cudaStream_t s) {
  const fs::ConvGeom& g = U->g[x.lev];
  float* pw = U->pw;
  float* pb = U->pb;
  if (!wgrad_on_cuda_cores()) {
    // tensor cores: row groups of whole 128-row subtiles
    long long rows_per = (g.R + kWgGroups - 1) / kWgGroups;
    rows_per = (rows_per + 127) / 128 * 128;
    const int st = fs::wgrad_tc_launch(g, x.p, x.ctot, xoff, kCin[l], dy.p, dy.ctot, yoff,
                                       kCout[l], kWgGroups, rows_per, pw, pb, U->err, s);
    if (st != FS_OK) return st;
  } else {
    long long rows_per = (g.R + kWgGroups - 1) / kWgGroups;
    rows_per = (rows_per + fs::kWgRows - 1) / fs::kWgRows * fs::kWgRows;
    const int CO = kCout[l] / 16, CI = kCin[l] / 16;
#define FS_WG(a, b) \
  if (CO == a && CI == b) wgrad_launch<a, b>(g, x, xoff, dy, yoff, rows_per, pw, pb, s); else
    FS_WG(1, 1) FS_WG(2, 1) FS_WG(2, 2) FS_WG(3, 2) FS_WG(3, 3) FS_WG(4, 3) FS_WG(4, 4)
    FS_WG(3, 7) FS_WG(2, 5) FS_WG(1, 3) {
      fs_set_error_msg("unet: no weight-gradient kernel for this layer shape");
      return FS_BAD_ARG;
    }
#undef FS_WG
    FS_CHECK_LAUNCH("k_conv_wgrad");
  }
  const long long nw = 27LL * kCin[l] * kCout[l];
  fs::k_sum_groups<<<blocks_for(nw), 256, 0, s>>>(nw, kWgGroups, pw, U->grad + conv_woff(l));
  fs::k_sum_groups<<<1, 256, 0, s>>>(kCout[l], kWgGroups, pb, U->grad + conv_boff(l));
  FS_CHECK_LAUNCH("k_sum_groups");
  return FS_OK;
}

int pool(fs_unet* U, const Vol& src, int soff, const Vol& dst, int doff, int c, cudaStream_t s) {
  const fs::ConvGeom &gf = U->g[src.lev], &gc = U->g[dst.lev];
  const long long n = (long long)gc.X * gc.Y * gc.Z * U->batch * (c / 8);
  fs::k_unet_pool<<<blocks_for(n), 256, 0, s>>>(gf, gc, U->batch, src.p, src.ctot, soff, dst.p,
                                                 dst.ctot, doff, c);
  FS_CHECK_LAUNCH("k_unet_pool");
  return FS_OK;
}

int up(fs_unet* U, const Vol& src, int soff, const Vol& dst, int doff, int c, cudaStream_t s) {
  const fs::ConvGeom &gc = U->g[src.lev], &gf = U->g[dst.lev];
  const long long n = (long long)gf.X * gf.Y * gf.Z * U->batch * (c / 8);
  fs::k_unet_up<<<blocks_for(n), 256, 0, s>>>(gf, gc, U->batch, src.p, src.ctot, soff, dst.p,
                                               dst.ctot, doff, c);
  FS_CHECK_LAUNCH("k_unet_up");
  return FS_OK;
}

int up_bwd(fs_unet* U, const Vol& gsrc, int soff, const Vol& gdst, int doff, int c,
           cudaStream_t s) {
  const fs::ConvGeom &gf = U->g[gsrc.lev], &gc = U->g[gdst.lev];
  const long long n = (long long)gc.X * gc.Y * gc.Z * U->batch * (c / 8);
  fs::k_unet_up_bwd<<<blocks_for(n), 256, 0, s>>>(gf, gc, U->batch, gsrc.p, gsrc.ctot, soff,
                                                   gdst.p, gdst.ctot, doff, c);
  FS_CHECK_LAUNCH("k_unet_up_bwd");
  return FS_OK;
}

int pool_bwd(fs_unet* U, const Vol& gsrc, const Vol& act, int aoff, const Vol& gdst, int doff,
             int c, cudaStream_t s) {
  const fs::ConvGeom &gc = U->g[gsrc.lev], &gf = U->g[gdst.lev];
  const long long n = (long long)gf.X * gf.Y * gf.Z * U->batch * (c / 8);
  fs::k_unet_pool_bwd<<<blocks_for(n), 256, 0, s>>>(gf, gc, U->batch, gsrc.p, gsrc.ctot, 0, act.p,
                                                     act.ctot, aoff, gdst.p, gdst.ctot, doff, c);
  FS_CHECK_LAUNCH("k_unet_pool_bwd");
  return FS_OK;
}

#define FS_TRY(x)                  \
  do {                             \
    const int _st = (x);           \
    if (_st != FS_OK) return _st;  \
  } while (0)

// Everything from the packed input to d0 (the head's input).
int body_forward(fs_unet* U, cudaStream_t s) {
  FS_TRY(conv(U, 0, U->in0, 0, U->e0a, 0, s));
  FS_TRY(conv(U, 1, U->e0a, 0, U->cat0, 32, s));
  FS_TRY(pool(U, U->cat0, 32, U->p1, 0, 16, s));
  FS_TRY(conv(U, 2, U->p1, 0, U->e1a, 0, s));
  FS_TRY(conv(U, 3, U->e1a, 0, U->cat1, 48, s));
  FS_TRY(pool(U, U->cat1, 48, U->p2, 0, 32, s));
  FS_TRY(conv(U, 4, U->p2, 0, U->e2a, 0, s));
  FS_TRY(conv(U, 5, U->e2a, 0, U->cat2, 64, s));
  FS_TRY(pool(U, U->cat2, 64, U->p3, 0, 48, s));
  FS_TRY(conv(U, 6, U->p3, 0, U->e3a, 0, s));
  FS_TRY(conv(U, 7, U->e3a, 0, U->e3, 0, s));
  FS_TRY(up(U, U->e3, 0, U->cat2, 0, 64, s));
  FS_TRY(conv(U, 8, U->cat2, 0, U->d2a, 0, s));
  FS_TRY(conv(U, 9, U->d2a, 0, U->d2, 0, s));
  FS_TRY(up(U, U->d2, 0, U->cat1, 0, 48, s));
  FS_TRY(conv(U, 10, U->cat1, 0, U->d1a, 0, s));
  FS_TRY(conv(U, 11, U->d1a, 0, U->d1, 0, s));
  FS_TRY(up(U, U->d1, 0, U->cat0, 0, 32, s));
  FS_TRY(conv(U, 12, U->cat0, 0, U->d0a, 0, s));
  FS_TRY(conv(U, 13, U->d0a, 0, U->d0, 0, s));
  return FS_OK;
}

// From g_d0 (gradient at the head's input, ReLU-masked) back to every weight.
int body_backward(fs_unet* U, cudaStream_t s) {
  FS_TRY(conv_wgrad(U, 13, U->d0a, 0, U->g_d0, 0, s));
  FS_TRY(conv_dgrad(U, 13, U->g_d0, 0, U->g_d0a, 0, &U->d0a, 0, s));
  FS_TRY(conv_wgrad(U, 12, U->cat0, 0, U->g_d0a, 0, s));
  FS_TRY(conv_dgrad(U, 12, U->g_d0a, 0, U->g_cat0, 0, &U->cat0, 0, s));
  FS_TRY(up_bwd(U, U->g_cat0, 0, U->g_d1, 0, 32, s));
  FS_TRY(conv_wgrad(U, 11, U->d1a, 0, U->g_d1, 0, s));
  FS_TRY(conv_dgrad(U, 11, U->g_d1, 0, U->g_d1a, 0, &U->d1a, 0, s));
  FS_TRY(conv_wgrad(U, 10, U->cat1, 0, U->g_d1a, 0, s));
  FS_TRY(conv_dgrad(U, 10, U->g_d1a, 0, U->g_cat1, 0, &U->cat1, 0, s));
  FS_TRY(up_bwd(U, U->g_cat1, 0, U->g_d2, 0, 48, s));
  FS_TRY(conv_wgrad(U, 9, U->d2a, 0, U->g_d2, 0, s));
  FS_TRY(conv_dgrad(U, 9, U->g_d2, 0, U->g_d2a, 0, &U->d2a, 0, s));
  FS_TRY(conv_wgrad(U, 8, U->cat2, 0, U->g_d2a, 0, s));
  FS_TRY(conv_dgrad(U, 8, U->g_d2a, 0, U->g_cat2, 0, &U->cat2, 0, s));
  FS_TRY(up_bwd(U, U->g_cat2, 0, U->g_e3, 0, 64, s));
  FS_TRY(conv_wgrad(U, 7, U->e3a, 0, U->g_e3, 0, s));
  FS_TRY(conv_dgrad(U, 7, U->g_e3, 0, U->g_e3a, 0, &U->e3a, 0, s));
  FS_TRY(conv_wgrad(U, 6, U->p3, 0, U->g_e3a, 0, s));
  FS_TRY(conv_dgrad(U, 6, U->g_e3a, 0, U->g_p3, 0, nullptr, 0, s));
  FS_TRY(pool_bwd(U, U->g_p3, U->cat2, 64, U->g_cat2, 64, 48, s));
  FS_TRY(conv_wgrad(U, 5, U->e2a, 0, U->g_cat2, 64, s));
  FS_TRY(conv_dgrad(U, 5, U->g_cat2, 64, U->g_e2a, 0, &U->e2a, 0, s));
  FS_TRY(conv_wgrad(U, 4, U->p2, 0, U->g_e2a, 0, s));
  FS_TRY(conv_dgrad(U, 4, U->g_e2a, 0, U->g_p2, 0, nullptr, 0, s));
  FS_TRY(pool_bwd(U, U->g_p2, U->cat1, 48, U->g_cat1, 48, 32, s));
  FS_TRY(conv_wgrad(U, 3, U->e1a, 0, U->g_cat1, 48, s));
  FS_TRY(conv_dgrad(U, 3, U->g_cat1, 48, U->g_e1a, 0, &U->e1a, 0, s));
  FS_TRY(conv_wgrad(U, 2, U->p1, 0, U->g_e1a, 0, s));
  FS_TRY(conv_dgrad(U, 2, U->g_e1a, 0, U->g_p1, 0, nullptr, 0, s));
  FS_TRY(pool_bwd(U, U->g_p1, U->cat0, 32, U->g_cat0, 32, 16, s));
  FS_TRY(conv_wgrad(U, 1, U->e0a, 0, U->g_cat0, 32, s));
  FS_TRY(conv_dgrad(U, 1, U->g_cat0, 32, U->g_e0a, 0, &U->e0a, 0, s));
  FS_TRY(conv_wgrad(U, 0, U->in0, 0, U->g_e0a, 0, s));
  return FS_OK;
}

int scale_inputs(fs_unet* U, const float* rhs, long long sn, long long sb, const uint8_t* lab,
                 long long lab_sb, cudaStream_t s) {
  const long long N = (long long)U->g[0].X * U->g[0].Y * U->g[0].Z;
  fs::k_unet_sumsq<<<kRedBlocks, 256, 0, s>>>(N, U->batch, rhs, sn, sb, lab, lab_sb, U->red);
  fs::k_unet_scale<<<1, 64, 0, s>>>(kRedBlocks, U->batch, N, U->red, U->scale, U->inv, nullptr);
  FS_CHECK_LAUNCH("k_unet_scale");
  return FS_OK;
}

// One Adam step of theta on gradient g (device, theta-sized; the net's own
// gradient buffer, or a caller's, e.g. averaged over data-parallel ranks),
// then the tensor-core weight images re-packed from the new theta.
int adam_update(fs_unet* U, const float* g, float lr, cudaStream_t s) {
  U->step += 1;
  const double b1 = 0.9, b2 = 0.999;
  const float c1 = (float)(1.0 / (1.0 - pow(b1, (double)U->step)));
  const float c2 = (float)(1.0 / (1.0 - pow(b2, (double)U->step)));
  const long long nt = theta_size();
  fs::k_adam<<<blocks_for(nt), 256, 0, s>>>(nt, U->theta, g, U->adam_m, U->adam_v, lr,
                                             (float)b1, (float)b2, 1e-8f, c1, c2);
  FS_CHECK_LAUNCH("k_adam");
  return pack_all(U, s);
}

}  // namespace

int unet_forward(fs_unet* U, const float* rhs, long long rhs_sn, long long rhs_sb,
                 const float* emx, const float* emy, const float* emz, long long em_sb,
                 const uint8_t* lab, long long lab_sb, float* out, long long out_sn,
                 long long out_sb, bool normalised, cudaStream_t s) {
  const long long N = (long long)U->g[0].X * U->g[0].Y * U->g[0].Z;
  FS_TRY(scale_inputs(U, rhs, rhs_sn, rhs_sb, lab, lab_sb, s));
  fs::k_unet_pack<<<blocks_for(N * U->batch), 256, 0, s>>>(U->g[0], U->batch, rhs, rhs_sn, rhs_sb,
                                                           emx, emy, emz, em_sb, lab, lab_sb,
                                                           U->inv, U->in0.p);
  FS_CHECK_LAUNCH("k_unet_pack");
  FS_TRY(body_forward(U, s));
  fs::k_unet_head<<<blocks_for(N * U->batch), 256, 0, s>>>(
      U->g[0], U->batch, U->d0.p, U->theta + head_off(), lab, lab_sb,
      normalised ? U->ones : U->scale, out, out_sn, out_sb);
  FS_CHECK_LAUNCH("k_unet_head");
  return FS_OK;
}

// Kernel launches of one forward pass (for the launch accounting of plans).
long long unet_forward_launches() { return 2 + 1 + kNConv + 3 + 3 + 1; }

size_t unet_bytes(int X, int Y, int Z, int batch, int train) {
  fs_unet tmp;
  return layout(&tmp, nullptr, X, Y, Z, batch, train);
}

int unet_init(fs_unet* U, int X, int Y, int Z, int batch, int train, float* theta, void* ws,
              size_t bytes, cudaStream_t s) {
  const size_t need = layout(U, nullptr, X, Y, Z, batch, train);
  if (!ws || bytes < need || ((uintptr_t)ws & 255)) {
    fs_set_error_msg("unet: workspace missing, too small or not 256-byte aligned");
    return FS_BAD_ARG;
  }
  U->batch = batch;
  U->train = train;
  U->theta = theta;
  layout(U, (uint8_t*)ws, X, Y, Z, batch, train);
  FS_CHECK(cudaMemsetAsync(ws, 0, need - 256, s));  // zero halos and moments
  float ones[64];
  for (int i = 0; i < 64; ++i) ones[i] = 1.0f;
  for (int b0 = 0; b0 < batch; b0 += 64) {
    const int nb = batch - b0 < 64 ? batch - b0 : 64;
    FS_CHECK(cudaMemcpyAsync(U->ones + b0, ones, sizeof(float) * nb, cudaMemcpyHostToDevice, s));
  }
  FS_CHECK(cudaStreamSynchronize(s));  // `ones` is a host stack array
  return pack_all(U, s);
}

extern "C" {

int fs_conv3d_wgrad_workspace_bytes(int cin, int cout, size_t* bytes) {
  if (cin < 16 || cout < 16 || !bytes) return FS_BAD_ARG;
  *bytes = sizeof(float) * (size_t)kWgGroups * (27ull * cin * cout + cout) + 256;
  return FS_OK;
}

int fs_conv3d_wgrad_bf16(const void* x, int ctot_in, int cin_off, int cin, const void* dy,
                         int ctot_out, int cout_off, int cout, int batch, int X, int Y, int Z,
                         float* dw, float* db, void* workspace, size_t workspace_bytes,
                         int* error, void* stream) {
  size_t need = 0;
  if (fs_conv3d_wgrad_workspace_bytes(cin, cout, &need) != FS_OK || !dw || !workspace ||
      workspace_bytes < need || ((uintptr_t)workspace & 255) || batch < 1 || X < 1 || Y < 1 ||
      Z < 1)
    return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const fs::ConvGeom g = fs::conv_geom(batch, X, Y, Z);
  long long rows_per = (g.R + kWgGroups - 1) / kWgGroups;
  rows_per = (rows_per + 127) / 128 * 128;
  float* pw = (float*)workspace;
  float* pb = pw + (size_t)kWgGroups * 27 * cin * cout;
  int st = fs::wgrad_tc_launch(g, x, ctot_in, cin_off, cin, dy, ctot_out, cout_off, cout,
                               kWgGroups, rows_per, pw, db ? pb : nullptr, error, s);
  if (st != FS_OK) return st;
  const long long nw = 27LL * cin * cout;
  fs::k_sum_groups<<<blocks_for(nw), 256, 0, s>>>(nw, kWgGroups, pw, dw);
  if (db) fs::k_sum_groups<<<1, 256, 0, s>>>(cout, kWgGroups, pb, db);
  FS_CHECK_LAUNCH("k_sum_groups");
  return FS_OK;
}

int fs_unet_param_count(long long* n) {
  if (!n) return FS_BAD_ARG;
  *n = theta_size();
  return FS_OK;
}

int fs_unet_layer(int l, int* cin, int* cout, long long* woff, long long* boff) {
  if (l < 0 || l > kNConv || !cin || !cout || !woff || !boff) return FS_BAD_ARG;
  if (l == kNConv) {  // the 1x1 head: 16 weights then the bias
    *cin = 16;
    *cout = 1;
    *woff = head_off();
    *boff = head_off() + 16;
    return FS_OK;
  }
  *cin = kCin[l];
  *cout = kCout[l];
  *woff = conv_woff(l);
  *boff = conv_boff(l);
  return FS_OK;
}

int fs_unet_workspace_bytes(int X, int Y, int Z, int batch, int train, size_t* bytes) {
  if (!bytes || X < 1 || Y < 1 || Z < 1 || batch < 1 || batch > 64) return FS_BAD_ARG;
  *bytes = unet_bytes(X, Y, Z, batch, train);
  return FS_OK;
}

int fs_unet_create(int X, int Y, int Z, int batch, int train, float* theta, void* workspace,
                   size_t workspace_bytes, fs_unet** net, void* stream) {
  if (!net || !theta || X < 1 || Y < 1 || Z < 1 || batch < 1 || batch > 64) return FS_BAD_ARG;
  *net = nullptr;
  fs_unet* U = new (std::nothrow) fs_unet();
  if (!U) return FS_CUDA_ERROR;
  const int st = unet_init(U, X, Y, Z, batch, train, theta, workspace, workspace_bytes,
                           (cudaStream_t)stream);
  if (st != FS_OK) {
    delete U;
    return st;
  }
  *net = U;
  return FS_OK;
}

int fs_unet_sync(fs_unet* net, void* stream) {
  if (!net) return FS_BAD_ARG;
  return pack_all(net, (cudaStream_t)stream);
}

int fs_unet_forward(fs_unet* net, const float* rhs, long long rhs_sn, long long rhs_sb,
                    const float* em, long long em_sb, const uint8_t* label, long long label_sb,
                    float* out, long long out_sn, long long out_sb, void* stream) {
  if (!net || !rhs || !em || !label || !out) return FS_BAD_ARG;
  const long long N = (long long)net->g[0].X * net->g[0].Y * net->g[0].Z;
  return unet_forward(net, rhs, rhs_sn, rhs_sb, em, em + N, em + 2 * N, em_sb, label, label_sb,
                      out, out_sn, out_sb, false, (cudaStream_t)stream);
}

int fs_unet_train_step(fs_unet* net, const float* rhs, const float* em, const uint8_t* label,
                       const float* target, float lr, float* loss, void* stream) {
  if (!net || !net->train || !rhs || !em || !label || !target || !(lr >= 0.0f)) return FS_BAD_ARG;
  fs_unet* U = net;
  cudaStream_t s = (cudaStream_t)stream;
  const long long N = (long long)U->g[0].X * U->g[0].Y * U->g[0].Z;
  const int B = U->batch;
  FS_TRY(unet_forward(U, rhs, 1, N, em, em + N, em + 2 * N, 3 * N, label, N, U->out_n, 1, N,
                      true, s));
  // normalised target norms, loss and dL/d(out) through the head
  fs::k_unet_sumsq<<<kRedBlocks, 256, 0, s>>>(N, B, target, 1, N, label, N, U->red);
  fs::k_unet_scale<<<1, 64, 0, s>>>(kRedBlocks, B, N, U->red, nullptr, U->inv, U->tnorm);
  fs::k_unet_loss_partial<<<kRedBlocks, 256, 0, s>>>(N, B, U->out_n, target, U->inv, label, U->red);
  fs::k_unet_loss_final<<<1, 32, 0, s>>>(kRedBlocks, B, U->red, U->tnorm, U->loss);
  fs::k_unet_head_bwd<<<kRedBlocks, 256, 0, s>>>(U->g[0], B, U->out_n, target, U->inv, label,
                                                  U->tnorm, U->d0.p, U->theta + head_off(),
                                                  U->g_d0.p, U->ph);
  fs::k_sum_groups<<<1, 32, 0, s>>>(17, kRedBlocks, U->ph, U->grad + head_off());
  FS_CHECK_LAUNCH("unet loss");
  FS_TRY(body_backward(U, s));
  FS_TRY(adam_update(U, U->grad, lr, s));
  if (loss) FS_CHECK(cudaMemcpyAsync(loss, U->loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
  return FS_OK;
}

int fs_unet_adam_step(fs_unet* net, const float* grad, float lr, void* stream) {
  if (!net || !net->train || !grad || !(lr >= 0.0f)) return FS_BAD_ARG;
  return adam_update(net, grad, lr, (cudaStream_t)stream);
}

int fs_unet_gradient(fs_unet* net, const float* rhs, const float* em, const uint8_t* label,
                     const float* target, float* grad, float* loss, void* stream) {
  // One forward and backward without an update: the loss and dL/dtheta
  // (used to check the gradient against a CPU reference).
  if (!net || !net->train || !rhs || !em || !label || !target || !grad) return FS_BAD_ARG;
  fs_unet* U = net;
  cudaStream_t s = (cudaStream_t)stream;
  const long long N = (long long)U->g[0].X * U->g[0].Y * U->g[0].Z;
  const int B = U->batch;
  FS_TRY(unet_forward(U, rhs, 1, N, em, em + N, em + 2 * N, 3 * N, label, N, U->out_n, 1, N,
                      true, s));
  fs::k_unet_sumsq<<<kRedBlocks, 256, 0, s>>>(N, B, target, 1, N, label, N, U->red);
  fs::k_unet_scale<<<1, 64, 0, s>>>(kRedBlocks, B, N, U->red, nullptr, U->inv, U->tnorm);
  fs::k_unet_loss_partial<<<kRedBlocks, 256, 0, s>>>(N, B, U->out_n, target, U->inv, label, U->red);
  fs::k_unet_loss_final<<<1, 32, 0, s>>>(kRedBlocks, B, U->red, U->tnorm, U->loss);
  fs::k_unet_head_bwd<<<kRedBlocks, 256, 0, s>>>(U->g[0], B, U->out_n, target, U->inv, label,
                                                  U->tnorm, U->d0.p, U->theta + head_off(),
                                                  U->g_d0.p, U->ph);
  fs::k_sum_groups<<<1, 32, 0, s>>>(17, kRedBlocks, U->ph, U->grad + head_off());
  FS_CHECK_LAUNCH("unet loss");
  FS_TRY(body_backward(U, s));
  FS_CHECK(cudaMemcpyAsync(grad, U->grad, sizeof(float) * theta_size(), cudaMemcpyDeviceToDevice, s));
  if (loss) FS_CHECK(cudaMemcpyAsync(loss, U->loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
  return FS_OK;
}

int fs_unet_error(const fs_unet* net, int* flag, void* stream) {
  if (!net || !flag) return FS_BAD_ARG;
  FS_CHECK(cudaMemcpyAsync(flag, net->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  FS_CHECK(cudaStreamSynchronize((cudaStream_t)stream));
  return FS_OK;
}

int fs_unet_destroy(fs_unet* net) {
  delete net;
  return FS_OK;
}

}  // extern "C"
