// Host-side declarations shared by the network sources.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>

#include <stdint.h>

#include "fieldspice_b200.h"
#include "fs_conv.cuh"

namespace fs {

struct ConvCfg {
  int T, W, BR, phases;
  size_t smem;
};

// One convolution's buffers: input channels [cin_off, cin_off + cin) of a
// ctot_in-channel volume, output channels [out_off, out_off + cout) of a
// ctot_out-channel volume, optional ReLU mask channels of a third volume.
struct ConvIO {
  const void* x = nullptr;
  int ctot_in = 0, cin_off = 0, cin = 0;
  const void* wpack = nullptr;
  const float* bias = nullptr;
  void* out = nullptr;
  int ctot_out = 0, out_off = 0, cout = 0;
  const void* mask = nullptr;
  int ctot_mask = 0, mask_off = 0;
  int relu = 0, accumulate = 0;
  int* error = nullptr;
};

ConvGeom conv_geom(int batch, int X, int Y, int Z);
bool conv_config(const ConvGeom& g, int cin, int cout, ConvCfg* c);
int conv_launch(const ConvGeom& g, const ConvIO& io, cudaStream_t s);
int pack_weights(const float* w, int cin, int cout, int flip, void* out, cudaStream_t s);
// Weight-gradient partials of one convolution on tensor cores:
// pw[G][27][cout][cin] (and pb[G][cout] when pb is not NULL) over G row
// groups of rows_per rows (a multiple of 128) each.
int wgrad_tc_launch(const ConvGeom& g, const void* x, int ctot_x, int xoff, int cin,
                    const void* dy, int ctot_y, int yoff, int cout, int groups,
                    long long rows_per, float* pw, float* pb, int* error, cudaStream_t s);

}  // namespace fs

// The U-Net forward pass on caller buffers (defined in fs_unet.cu): rhs and
// out in any (node, sample) strides, the level's three mass arrays and
// labels with a per-sample stride (0: shared by every sample).
int unet_forward(fs_unet* U, const float* rhs, long long rhs_sn, long long rhs_sb,
                 const float* emx, const float* emy, const float* emz, long long em_sb,
                 const uint8_t* lab, long long lab_sb, float* out, long long out_sn,
                 long long out_sb, bool normalised, cudaStream_t s);
long long unet_forward_launches();
