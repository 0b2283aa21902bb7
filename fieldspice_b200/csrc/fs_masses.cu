// Edge masses (material averaging + metric), Dirichlet excitations and the
// library's bookkeeping entry points.
//
// fs_build_masses restates fieldspice/operators.py:144-237 (cell_to_edge)
// and operators.py:302-315 (edge_mass) as one pass over the node grid.  The
// floating-point operations are issued with explicit round-to-nearest
// intrinsics in the order NumPy evaluates them, so no multiply-add is fused
// and the FP64 masses are bit-identical to the reference's:
//   w_m   = wa * wb                        (broadcast product, y|x then z|y)
//   wsum  = ((w0 + w1) + w2) + w3          (reduction over the quadrant axis)
//   num   = ((q0*w0 + q1*w1) + q2*w2) + q3*w3
//   prop  = num / (wsum > 0 ? wsum : 1)    (parallel)
//         = safe / (((w0/q0 + w1/q1) + w2/q2) + w3/q3)   (harmonic)
//   mass  = (prop * (hda*hdb)) / h
#include <stdio.h>
#include <string.h>

#include "fs_common.cuh"

using fs::Dims;

namespace {

__device__ __forceinline__ double half_lo(const double* h, int idx) {
  // Half width of the cell below node plane idx (0 at the lower wall).
  return idx == 0 ? 0.0 : __dmul_rn(0.5, h[idx - 1]);
}
__device__ __forceinline__ double half_hi(const double* h, int idx, int ncell) {
  // Half width of the cell above node plane idx (0 at the upper wall).
  return idx == ncell ? 0.0 : __dmul_rn(0.5, h[idx]);
}
__device__ __forceinline__ int clampi(int v, int lo, int hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// Combine four quadrant values q with weights w in the reference's order.
__device__ __forceinline__ double combine4(const double (&q)[4],
                                           const double (&w)[4], int mode) {
  double wsum = __dadd_rn(__dadd_rn(__dadd_rn(w[0], w[1]), w[2]), w[3]);
  double safe = wsum > 0.0 ? wsum : 1.0;
  if (mode == FS_AVERAGE_HARMONIC) {
    const double tiny = 2.2250738585072014e-308;  // np.finfo(float).tiny
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      double qq = q[m] > 0.0 ? q[m] : tiny;
      double t = __ddiv_rn(w[m], qq);
      s = (m == 0) ? t : __dadd_rn(s, t);
    }
    return __ddiv_rn(safe, s);
  }
  double num = __dmul_rn(q[0], w[0]);
#pragma unroll
  for (int m = 1; m < 4; ++m) num = __dadd_rn(num, __dmul_rn(q[m], w[m]));
  return __ddiv_rn(num, safe);
}

// One thread per node; writes the three edges leaving the node in +x/+y/+z.
__global__ void k_build_masses(Dims d, const double* __restrict__ prop,
                               const double* __restrict__ hx,
                               const double* __restrict__ hy,
                               const double* __restrict__ hz,
                               const double* __restrict__ hxd,
                               const double* __restrict__ hyd,
                               const double* __restrict__ hzd, int mode,
                               double* __restrict__ mx, double* __restrict__ my,
                               double* __restrict__ mz) {
  const int cx = d.nx - 1, cy = d.ny - 1, cz = d.nz - 1;  // cells per axis
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    auto cell = [&](int a, int b, int c) -> double {
      return prop[((long long)clampi(a, 0, cx - 1) * cy + clampi(b, 0, cy - 1)) *
                      cz +
                  clampi(c, 0, cz - 1)];
    };
    // x-edge (i,j,k): quadrants (dj,dk) in (0,0),(0,1),(1,0),(1,1)
    if (i < cx) {
      double q[4], w[4];
      const double wy[2] = {half_lo(hy, j), half_hi(hy, j, cy)};
      const double wz[2] = {half_lo(hz, k), half_hi(hz, k, cz)};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        int dj = m >> 1, dk = m & 1;
        q[m] = cell(i, j + dj - 1, k + dk - 1);
        w[m] = __dmul_rn(wy[dj], wz[dk]);
      }
      double pe = combine4(q, w, mode);
      mx[n] = __ddiv_rn(__dmul_rn(pe, __dmul_rn(hyd[j], hzd[k])), hx[i]);
    } else {
      mx[n] = 0.0;
    }
    // y-edge (i,j,k): quadrants (di,dk)
    if (j < cy) {
      double q[4], w[4];
      const double wx[2] = {half_lo(hx, i), half_hi(hx, i, cx)};
      const double wz[2] = {half_lo(hz, k), half_hi(hz, k, cz)};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        int di = m >> 1, dk = m & 1;
        q[m] = cell(i + di - 1, j, k + dk - 1);
        w[m] = __dmul_rn(wx[di], wz[dk]);
      }
      double pe = combine4(q, w, mode);
      my[n] = __ddiv_rn(__dmul_rn(pe, __dmul_rn(hxd[i], hzd[k])), hy[j]);
    } else {
      my[n] = 0.0;
    }
    // z-edge (i,j,k): quadrants (di,dj)
    if (k < cz) {
      double q[4], w[4];
      const double wx[2] = {half_lo(hx, i), half_hi(hx, i, cx)};
      const double wy[2] = {half_lo(hy, j), half_hi(hy, j, cy)};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        int di = m >> 1, dj = m & 1;
        q[m] = cell(i + di - 1, j + dj - 1, k);
        w[m] = __dmul_rn(wx[di], wy[dj]);
      }
      double pe = combine4(q, w, mode);
      mz[n] = __ddiv_rn(__dmul_rn(pe, __dmul_rn(hxd[i], hyd[j])), hz[k]);
    } else {
      mz[n] = 0.0;
    }
  }
}

__global__ void k_combine(const double* __restrict__ m1,
                          const double* __restrict__ m2, double a, double b,
                          double* __restrict__ out, long long n) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    out[t] = __dadd_rn(__dmul_rn(a, m1[t]), __dmul_rn(b, m2[t]));
}

__global__ void k_unit_excitation(long long N, int nrhs,
                                  const int16_t* __restrict__ group,
                                  const uint8_t* __restrict__ label,
                                  double* __restrict__ phi) {
  // pairs of values as 16-byte stores where the width and the base allow it,
  // one thread per pair (consecutive threads write consecutive 16 bytes)
  const bool pairs = (nrhs & 1) == 0 && (reinterpret_cast<uintptr_t>(phi) & 15) == 0;
  if (pairs) {
    const int np = nrhs / 2;
    const long long total = N * np;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
      long long n;
      int c;
      if (total <= 0x7fffffffLL) {
        n = (unsigned)t / (unsigned)np;
        c = (int)((unsigned)t - (unsigned)n * (unsigned)np);
      } else {
        n = t / np;
        c = (int)(t - n * np);
      }
      const int g = label[n] == FS_LABEL_FIXED ? group[n] : -1;
      reinterpret_cast<double2*>(phi)[t] =
          make_double2(g == 2 * c ? 1.0 : 0.0, g == 2 * c + 1 ? 1.0 : 0.0);
    }
    return;
  }
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    const bool fixed = label[n] == FS_LABEL_FIXED;
    const int g = fixed ? group[n] : -1;
    for (int r = 0; r < nrhs; ++r) phi[n * nrhs + r] = g == r ? 1.0 : 0.0;
  }
}

__global__ void k_set_dirichlet(long long N, const int16_t* __restrict__ group,
                                const uint8_t* __restrict__ label,
                                const double* __restrict__ values,
                                double* __restrict__ phi) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    const int g = group[n];
    if (g >= 0 && label[n] == FS_LABEL_FIXED) phi[n] = values[g];
  }
}

thread_local char g_last_error[512] = "";

}  // namespace

// ---- bookkeeping -------------------------------------------------------------
void fs_set_error(const char* where, cudaError_t err) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s)", where,
           cudaGetErrorString(err), cudaGetErrorName(err));
}

void fs_set_error_msg(const char* msg) {
  snprintf(g_last_error, sizeof(g_last_error), "%s", msg);
}

int fs_cuda_status(const char* where, cudaError_t err) {
  fs_set_error(where, err);
  return FS_CUDA_ERROR;
}

int fs_grid_blocks(const void* kernel, long long work_items) {
  static int sm_counts[fs::kMaxDevices] = {};
  int& sm_count = sm_counts[fs::current_device_slot()];
  if (sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    sm_count = n > 0 ? n : 148;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, fs::kBlock,
                                                    0) != cudaSuccess ||
      per_sm <= 0)
    per_sm = 4;
  long long want = (work_items + fs::kBlock - 1) / fs::kBlock;
  long long cap = (long long)sm_count * per_sm;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (int)want;
}

// Masses of the reduced (wrap-around) grid: every reduced node sums the
// masses of the full-grid nodes merged into it (the first plane of a periodic
// axis absorbs the last), component by component.  On a periodic axis the
// own-direction mass of the last reduced plane is the full grid's edge into
// the dropped plane, i.e. the wrap edge.
__global__ void k_periodic_masses(fs::Dims f, fs::Dims r, const double* __restrict__ mf,
                                  double* __restrict__ mr) {
  const bool px = r.per & 1, py = (r.per >> 1) & 1, pz = (r.per >> 2) & 1;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < r.N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(r, n, i, j, k);
    const int ni = (px && i == 0) ? 2 : 1, nj = (py && j == 0) ? 2 : 1,
              nk = (pz && k == 0) ? 2 : 1;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b)
        for (int c = 0; c < nk; ++c) {
          const int fi = a ? f.nx - 1 : i, fj = b ? f.ny - 1 : j, fk = c ? f.nz - 1 : k;
          const long long fn = ((long long)fi * f.ny + fj) * f.nz + fk;
          for (int m = 0; m < 3; ++m) acc[m] += mf[m * f.N + fn];
        }
    for (int m = 0; m < 3; ++m) mr[m * r.N + n] = acc[m];
  }
}

extern "C" {

const char* fs_version(void) { return "fieldspice_b200 0.1.0 sm_100a"; }

int fs_periodic_masses(const double* m_full, int nx, int ny, int nz, int periodic,
                       double* m_reduced, void* stream) {
  if (!m_full || !m_reduced || periodic < 1 || periodic > 7) return FS_BAD_ARG;
  const int rx = nx - (periodic & 1), ry = ny - ((periodic >> 1) & 1),
            rz = nz - ((periodic >> 2) & 1);
  if (rx < 2 || ry < 2 || rz < 2) return FS_BAD_ARG;
  const fs::Dims f = fs::make_dims(nx, ny, nz);
  const fs::Dims r = fs::make_dims(rx, ry, rz, periodic);
  int g = fs_grid_blocks((const void*)k_periodic_masses, r.N);
  k_periodic_masses<<<g, fs::kBlock, 0, (cudaStream_t)stream>>>(f, r, m_full, m_reduced);
  FS_CHECK_LAUNCH("k_periodic_masses");
  return FS_OK;
}

const char* fs_status_string(int status) {
  switch (status) {
    case FS_OK: return "ok";
    case FS_NOT_CONVERGED: return "not converged";
    case FS_TIMEOUT: return "device did not report completion";
    case FS_BAD_ARG: return "bad argument";
    case FS_NAN: return "residual became NaN or Inf";
    case FS_CUDA_ERROR: return "CUDA error";
    case FS_STALLED: return "mixed-precision iterations stalled";
    default: return "unknown status";
  }
}

const char* fs_last_error(void) { return g_last_error; }

int fs_build_masses(const double* prop_cell, const double* hx, const double* hy,
                    const double* hz, const double* hxd, const double* hyd,
                    const double* hzd, int nx, int ny, int nz, int mode,
                    double* mx, double* my, double* mz, void* stream) {
  if (nx < 2 || ny < 2 || nz < 2 || !prop_cell || !hx || !hy || !hz || !hxd ||
      !hyd || !hzd || !mx || !my || !mz)
    return FS_BAD_ARG;
  if (mode != FS_AVERAGE_PARALLEL && mode != FS_AVERAGE_HARMONIC)
    return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  int g = fs_grid_blocks((const void*)k_build_masses, d.N);
  k_build_masses<<<g, fs::kBlock, 0, (cudaStream_t)stream>>>(
      d, prop_cell, hx, hy, hz, hxd, hyd, hzd, mode, mx, my, mz);
  FS_CHECK_LAUNCH("k_build_masses");
  return FS_OK;
}

int fs_combine_masses(const double* m1, const double* m2, double a, double b,
                      double* out, long long n, void* stream) {
  if (!m1 || !m2 || !out || n < 0) return FS_BAD_ARG;
  if (n == 0) return FS_OK;
  int g = fs_grid_blocks((const void*)k_combine, n);
  k_combine<<<g, fs::kBlock, 0, (cudaStream_t)stream>>>(m1, m2, a, b, out, n);
  FS_CHECK_LAUNCH("k_combine");
  return FS_OK;
}

int fs_fill_unit_excitation(const int16_t* group, const uint8_t* label,
                            double* phi, int nx, int ny, int nz, int nrhs,
                            void* stream) {
  if (!group || !label || !phi || nx < 1 || ny < 1 || nz < 1 || nrhs < 1)
    return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  int g = fs_grid_blocks((const void*)k_unit_excitation, d.N * (nrhs > 1 ? nrhs / 2 : 1));
  k_unit_excitation<<<g, fs::kBlock, 0, (cudaStream_t)stream>>>(d.N, nrhs,
                                                                group, label, phi);
  FS_CHECK_LAUNCH("k_unit_excitation");
  return FS_OK;
}

int fs_set_dirichlet(const int16_t* group, const uint8_t* label,
                     const double* values, double* phi, int nx, int ny, int nz,
                     void* stream) {
  if (!group || !label || !values || !phi || nx < 1 || ny < 1 || nz < 1)
    return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  int g = fs_grid_blocks((const void*)k_set_dirichlet, d.N);
  k_set_dirichlet<<<g, fs::kBlock, 0, (cudaStream_t)stream>>>(d.N, group, label,
                                                              values, phi);
  FS_CHECK_LAUNCH("k_set_dirichlet");
  return FS_OK;
}

}  // extern "C"
