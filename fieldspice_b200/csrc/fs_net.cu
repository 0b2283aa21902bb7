// Learned coarse-level preconditioner: a small BF16 3-D U-Net on tcgen05.
//
// This file holds the host side of the tensor-core convolution (fs_conv.cuh)
// -- launch planning, TMA tensor maps -- and the C-ABI entry points that run
// one convolution on caller buffers (used by the tests and by the network).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fieldspice_b200.h"
#include "fs_common.cuh"
#define FS_CONV_DEFINE_KERNELS
#include "fs_conv.cuh"
#include "fs_net.cuh"

namespace fs {

PFN_cuTensorMapEncodeTiled_v12000 net_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      (void)cudaGetLastError();
  }
  return fn;
}

ConvGeom conv_geom(int batch, int X, int Y, int Z) {
  ConvGeom g;
  g.X = X;
  g.Y = Y;
  g.Z = Z;
  g.Xp = X + 2;
  g.Yp = Y + 2;
  g.Zp = Z + 2;
  g.S = (long long)g.Yp * g.Zp;
  g.V = (long long)g.Xp * g.S;
  g.R = (long long)batch * g.V;
  return g;
}

bool conv_config(const ConvGeom& g, int cin, int cout, ConvCfg* c) {
  const int nch = cin / 8;
  const int phase_opts[2] = {1, 3};
  const int t_opts[3] = {4, 2, 1};
  for (int pi = 0; pi < 2; ++pi) {
    for (int ti = 0; ti < 3; ++ti) {
      const int phases = phase_opts[pi], T = t_opts[ti];
      if (T * cout > 256) continue;
      const long long need = 128LL * T + 2LL * g.Zp + 2;
      const int nseg = (int)((need + 255) / 256);
      const int BR = (int)(((need + nseg - 1) / nseg + 7) / 8 * 8);
      const int W = nseg * BR;
      const int ndx = phases == 1 ? 3 : 1, ntap = phases == 1 ? 27 : 9;
      const size_t smem = 1024 + (size_t)ndx * nch * W * 16 + (size_t)ntap * nch * cout * 16 + 64;
      if (smem <= 227u * 1024u) {
        c->T = T;
        c->W = W;
        c->BR = BR;
        c->phases = phases;
        c->smem = smem;
        return true;
      }
    }
  }
  return false;
}

int act_map(CUtensorMap* map, const void* base, int ctot, long long rows, int box_rows) {
  auto encode = net_encode_fn();
  if (!encode) {
    fs_set_error_msg("cuTensorMapEncodeTiled is unavailable from the driver");
    return FS_CUDA_ERROR;
  }
  cuuint64_t dims[2] = {(cuuint64_t)ctot, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ctot * 2};
  cuuint32_t box[2] = {8, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims,
                      strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    fs_set_error_msg("cuTensorMapEncodeTiled rejected an activation tensor map");
    return FS_CUDA_ERROR;
  }
  return FS_OK;
}

int wgrad_tc_launch(const ConvGeom& g, const void* x, int ctot_x, int xoff, int cin,
                    const void* dy, int ctot_y, int yoff, int cout, int groups,
                    long long rows_per, float* pw, float* pb, int* error, cudaStream_t s) {
  if (cin < 16 || cin % 16 || cin > 160 || cout < 16 || cout % 16 || cout > 128 ||
      xoff % 8 || yoff % 8 || ctot_x % 8 || ctot_y % 8 || xoff + cin > ctot_x ||
      yoff + cout > ctot_y || !x || !dy || !pw || ((uintptr_t)x & 15) || ((uintptr_t)dy & 15) ||
      groups < 1 || rows_per < 128 || rows_per % 128 || g.R <= 0 ||
      (long long)groups * rows_per < g.R) {
    fs_set_error_msg("conv3d wgrad: bad channel counts, offsets, alignment or row groups");
    return FS_BAD_ARG;
  }
  WgradArgs a;
  a.g = g;
  a.cin = cin;
  a.cin_off = xoff;
  a.cout = cout;
  a.cout_off = yoff;
  a.ntap = 9 * cin <= 512 ? 9 : 3;  // tensor-memory columns ntap * cin <= 512
  a.rows_per = rows_per;
  const long long need = 128 + 2LL * g.Zp + 2;
  const int nseg = (int)((need + 255) / 256);
  a.BR = (int)(((need + nseg - 1) / nseg + 7) / 8 * 8);
  a.W = nseg * a.BR;
  a.pw = pw;
  a.error = error;
  const size_t stage = 16u * 128u * 16u + (size_t)(cin / 8) * a.W * 16u;
  const size_t smem = 1024 + 2 * stage + 64;
  if (smem > 227u * 1024u) {
    fs_set_error_msg("conv3d wgrad: window does not fit in shared memory");
    return FS_BAD_ARG;
  }
  CUtensorMap xmap, ymap;
  int st = act_map(&xmap, x, ctot_x, g.R, a.BR);
  if (st != FS_OK) return st;
  st = act_map(&ymap, dy, ctot_y, g.R, 128);
  if (st != FS_OK) return st;
  static bool attr[fs::kMaxDevices] = {};
  if (!attr[fs::current_device_slot()]) {
    cudaError_t e = cudaFuncSetAttribute(k_conv_wgrad_tc,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         227 * 1024);
    if (e != cudaSuccess) return fs_cuda_status("cudaFuncSetAttribute(wgrad)", e);
    attr[fs::current_device_slot()] = true;
  }
  dim3 grid((unsigned)groups, (unsigned)(27 / a.ntap));
  k_conv_wgrad_tc<<<grid, kWgradThreads, smem, s>>>(xmap, ymap, a);
  FS_CHECK_LAUNCH("k_conv_wgrad_tc");
  if (pb) {
    k_conv_bgrad<<<groups, 256, 0, s>>>(g, (const __nv_bfloat16*)dy, ctot_y, yoff, cout,
                                        rows_per, pb);
    FS_CHECK_LAUNCH("k_conv_bgrad");
  }
  return FS_OK;
}

int conv_launch(const ConvGeom& g, const ConvIO& io, cudaStream_t s) {
  if (io.cin < 16 || io.cin % 16 || io.cout < 16 || io.cout % 16 || io.cout > 128 ||
      io.cin_off % 8 || io.ctot_in % 8 || io.out_off % 8 || io.ctot_out % 8 ||
      io.cin_off + io.cin > io.ctot_in || io.out_off + io.cout > io.ctot_out || !io.x ||
      !io.out || !io.wpack || ((uintptr_t)io.x & 15) || ((uintptr_t)io.out & 15) ||
      ((uintptr_t)io.wpack & 15) || g.X < 1 || g.Y < 1 || g.Z < 1 || g.R <= 0) {
    fs_set_error_msg("conv3d: bad channel counts, offsets, alignment or dims");
    return FS_BAD_ARG;
  }
  if (io.mask && (io.mask_off % 8 || io.ctot_mask % 8 || ((uintptr_t)io.mask & 15) ||
                  io.mask_off + io.cout > io.ctot_mask)) {
    fs_set_error_msg("conv3d: bad mask layout");
    return FS_BAD_ARG;
  }
  ConvCfg c;
  if (!conv_config(g, io.cin, io.cout, &c)) {
    fs_set_error_msg("conv3d: layer does not fit in shared memory");
    return FS_BAD_ARG;
  }
  // The one-tile-per-CTA kernel is the default: measured over a U-Net
  // forward at 64x64x32x8 it takes 1.51 ms against 1.77 ms for the
  // persistent, warp-specialised kernel, which FS_CONV=v2 selects where its
  // window ring and all weights fit.
  {
    const char* sel = getenv("FS_CONV");
    const bool v1 = !(sel && strcmp(sel, "v2") == 0);
    const int nch = io.cin / 8;
    const long long need = 128LL + 2LL * g.Zp + 2;
    const int nseg = (int)((need + 255) / 256);
    const int BR = (int)(((need + nseg - 1) / nseg + 7) / 8 * 8);
    const int W = nseg * BR;
    // deepest ring (up to 4 tile stages) that fits; prefer two CTAs per SM
    int nst = 0;
    size_t smem2 = 0;
    for (int cand = 4; cand >= 2 && !nst; --cand) {
      const size_t b = 1024 + (size_t)cand * 3 * nch * W * 16 + (size_t)27 * nch * io.cout * 16 + 160;
      if (b <= 113u * 1024u) {
        nst = cand;
        smem2 = b;
      }
    }
    for (int cand = 4; cand >= 2 && !nst; --cand) {
      const size_t b = 1024 + (size_t)cand * 3 * nch * W * 16 + (size_t)27 * nch * io.cout * 16 + 160;
      if (b <= 227u * 1024u) {
        nst = cand;
        smem2 = b;
      }
    }
    if (!v1 && nst && !io.accumulate) {
      CUtensorMap map2;
      int st2 = act_map(&map2, io.x, io.ctot_in, g.R, BR);
      if (st2 != FS_OK) return st2;
      ConvArgs a2;
      a2.g = g;
      a2.cin = io.cin;
      a2.cin_off = io.cin_off;
      a2.cout = io.cout;
      a2.wpack = (const uint16_t*)io.wpack;
      a2.bias = io.bias;
      a2.out = (__nv_bfloat16*)io.out;
      a2.out_stride = io.ctot_out;
      a2.out_off = io.out_off;
      a2.mask = (const __nv_bfloat16*)io.mask;
      a2.mask_stride = io.ctot_mask;
      a2.mask_off = io.mask_off;
      a2.relu = io.relu;
      a2.accumulate = 0;
      a2.T = 1;
      a2.W = W;
      a2.BR = BR;
      a2.phases = 1;
      a2.nst = nst;
      a2.error = io.error;
      static bool attr2[fs::kMaxDevices] = {};
      if (!attr2[fs::current_device_slot()]) {
        cudaError_t e = cudaFuncSetAttribute(k_conv3d_tc2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             227 * 1024);
        if (e != cudaSuccess) return fs_cuda_status("cudaFuncSetAttribute(conv2)", e);
        attr2[fs::current_device_slot()] = true;
      }
      const long long ntiles = (g.R + 127) / 128;
      int per_sm = 1, dev = 0, sms = 148;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv3d_tc2, kConv2Threads,
                                                        smem2) != cudaSuccess || per_sm < 1)
        per_sm = 1;
      if (per_sm > 2) per_sm = 2;  // TMEM: two accumulators of <= 128 columns per CTA
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      long long grid = (long long)sms * per_sm;
      if (grid > ntiles) grid = ntiles;
      k_conv3d_tc2<<<(unsigned)grid, kConv2Threads, smem2, s>>>(map2, a2, ntiles);
      FS_CHECK_LAUNCH("k_conv3d_tc2");
      return FS_OK;
    }
  }
  CUtensorMap map;
  int st = act_map(&map, io.x, io.ctot_in, g.R, c.BR);
  if (st != FS_OK) return st;
  ConvArgs a;
  a.g = g;
  a.cin = io.cin;
  a.cin_off = io.cin_off;
  a.cout = io.cout;
  a.wpack = (const uint16_t*)io.wpack;
  a.bias = io.bias;
  a.out = (__nv_bfloat16*)io.out;
  a.out_stride = io.ctot_out;
  a.out_off = io.out_off;
  a.mask = (const __nv_bfloat16*)io.mask;
  a.mask_stride = io.ctot_mask;
  a.mask_off = io.mask_off;
  a.relu = io.relu;
  a.accumulate = io.accumulate;
  a.T = c.T;
  a.W = c.W;
  a.BR = c.BR;
  a.phases = c.phases;
  a.nst = 0;
  a.error = io.error;
  static bool attr_set[fs::kMaxDevices] = {};
  if (!attr_set[fs::current_device_slot()]) {
    cudaError_t e = cudaFuncSetAttribute(k_conv3d_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         227 * 1024);
    if (e != cudaSuccess) return fs_cuda_status("cudaFuncSetAttribute(conv)", e);
    attr_set[fs::current_device_slot()] = true;
  }
  const long long tiles = (g.R + 128LL * c.T - 1) / (128LL * c.T);
  if (tiles > 0x7fffffffLL) {
    fs_set_error_msg("conv3d: volume too large");
    return FS_BAD_ARG;
  }
  k_conv3d_tc<<<(unsigned)tiles, 128, c.smem, s>>>(map, a);
  FS_CHECK_LAUNCH("k_conv3d_tc");
  return FS_OK;
}

int pack_weights(const float* w, int cin, int cout, int flip, void* out, cudaStream_t s) {
  if (!w || !out || cin < 16 || cin % 16 || cout < 16 || cout % 16) {
    fs_set_error_msg("pack_weights: channel counts must be multiples of 16");
    return FS_BAD_ARG;
  }
  const long long n = 27LL * cin * cout;
  const int blocks = (int)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
  k_pack_weights<<<blocks, 256, 0, s>>>(w, cin, cout, flip, (uint16_t*)out);
  FS_CHECK_LAUNCH("k_pack_weights");
  return FS_OK;
}

}  // namespace fs

extern "C" {

int fs_conv3d_pack_weights(const float* w, int cin, int cout, int flip, void* wpack,
                           void* stream) {
  return fs::pack_weights(w, cin, cout, flip, wpack, (cudaStream_t)stream);
}

int fs_conv3d_bf16(const void* x, int ctot_in, int cin_off, int cin, const void* wpack,
                   const float* bias, void* y, int ctot_out, int cout_off, int cout,
                   const void* mask, int ctot_mask, int mask_off, int batch, int X, int Y,
                   int Z, int relu, int accumulate, int* error, void* stream) {
  if (batch < 1) return FS_BAD_ARG;
  fs::ConvIO io;
  io.x = x;
  io.ctot_in = ctot_in;
  io.cin_off = cin_off;
  io.cin = cin;
  io.wpack = wpack;
  io.bias = bias;
  io.out = y;
  io.ctot_out = ctot_out;
  io.out_off = cout_off;
  io.cout = cout;
  io.mask = mask;
  io.ctot_mask = ctot_mask;
  io.mask_off = mask_off;
  io.relu = relu;
  io.accumulate = accumulate;
  io.error = error;
  return fs::conv_launch(fs::conv_geom(batch, X, Y, Z), io, (cudaStream_t)stream);
}

}  // extern "C"
