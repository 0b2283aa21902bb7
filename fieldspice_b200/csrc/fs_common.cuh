// Shared device helpers: grid indexing, RHS-interleaved vector access,
// deterministic block/grid reductions and error bookkeeping.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "fieldspice_b200.h"

namespace fs {

constexpr int kBlock = 256;  // threads per block for every grid-stride kernel
constexpr int kMaxRhs = 16;
// Per-device caches (kernel attributes, occupancy, SM counts) are indexed by
// the current device ordinal; ordinals at or beyond this bound share slot 0.
constexpr int kMaxDevices = 64;
inline int current_device_slot() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) d = 0;
  return d;
}

struct Dims {
  int nx, ny, nz;
  long long N;   // nodes
  long long sx;  // stride of i (ny*nz)
  int sy;        // stride of j (nz)
  // Periodic axes (bit 0 x, 1 y, 2 z): the last and first planes of such an
  // axis are joined by a wrap edge whose mass sits on the last plane; wx, wy,
  // wz are the index distances from the first to the last plane.
  int per;
  long long wx;
  int wy, wz;
  // x-marching kernels: 0 = every CTA takes an even contiguous share of the
  // column-planes (column after column); > 0 = CTA b takes x-planes
  // [c * xc, (c + 1) * xc) of column (b mod ncols), c = b / ncols, so CTAs
  // running at the same time march neighbouring columns over the same
  // x-planes and re-read each other's halo rows from L2, not DRAM.
  int xc;
};

inline Dims make_dims(int nx, int ny, int nz, int per = 0) {
  Dims d;
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.sy = nz;
  d.sx = (long long)ny * nz;
  d.N = (long long)nx * d.sx;
  d.per = per;
  d.wx = (long long)(nx - 1) * d.sx;
  d.wy = (ny - 1) * nz;
  d.wz = nz - 1;
  d.xc = 0;
  return d;
}

// The column-planes (u = column * nx + x) of this CTA in an x-marching
// kernel over ncols (z, y) tile columns; see Dims::xc.
template <typename I>
__device__ __forceinline__ void march_range(const Dims& d, I ncols, I& u, I& u_end) {
  const I total = ncols * (I)d.nx;
  if (d.xc > 0) {
    const I col = (I)blockIdx.x % ncols, chunk = (I)blockIdx.x / ncols;
    const I xa = min((I)d.nx, chunk * (I)d.xc), xb = min((I)d.nx, xa + (I)d.xc);
    u = col * (I)d.nx + xa;
    u_end = col * (I)d.nx + xb;
  } else {
    const I per = (total + (I)gridDim.x - 1) / (I)gridDim.x;
    u = (I)blockIdx.x * per;
    u_end = min(u + per, total);
  }
}

// Grid of an x-marching kernel with `resident` CTAs resident at once: the
// lockstep assignment (d->xc > 0, chunks of at least 16 planes) when a
// level's vectors are larger than `l2_bytes` (halo re-reads would go to DRAM),
// else an even contiguous split (d->xc = 0) over at most `resident` CTAs.
inline long long march_grid(Dims* d, long long ncols, long long resident,
                            long long vector_bytes, long long l2_bytes) {
  d->xc = 0;
  const long long cols = ncols * d->nx;
  if (vector_bytes > l2_bytes && ncols <= resident) {
    long long chunks = resident / ncols;
    if (chunks > d->nx / 16) chunks = d->nx / 16 > 0 ? d->nx / 16 : 1;
    const int xc = (int)((d->nx + chunks - 1) / chunks);
    d->xc = xc;
    return ncols * ((d->nx + xc - 1) / xc);
  }
  return resident < cols ? resident : cols;
}

// The six edges of node n = (i, j, k) as edge(present, mass, neighbour).  On
// a periodic axis the first and last planes are neighbours through the wrap
// edge, whose mass is stored on the last plane; otherwise the missing edges
// of boundary nodes are reported as absent (and their neighbour not read).
template <typename M, typename E>
__device__ __forceinline__ void edge6(const Dims& d, const M* __restrict__ mx,
                                      const M* __restrict__ my, const M* __restrict__ mz,
                                      long long n, int i, int j, int k, E&& edge) {
  const bool px = d.per & 1, py = (d.per >> 1) & 1, pz = (d.per >> 2) & 1;
  if (i > 0) edge(true, mx[n - d.sx], n - d.sx);
  else edge(px, px ? mx[n + d.wx] : (M)0, n + d.wx);
  if (i < d.nx - 1) edge(true, mx[n], n + d.sx);
  else edge(px, mx[n], n - d.wx);
  if (j > 0) edge(true, my[n - d.sy], n - d.sy);
  else edge(py, py ? my[n + d.wy] : (M)0, n + d.wy);
  if (j < d.ny - 1) edge(true, my[n], n + d.sy);
  else edge(py, my[n], n - d.wy);
  if (k > 0) edge(true, mz[n - 1], n - 1);
  else edge(pz, pz ? mz[n + d.wz] : (M)0, n + d.wz);
  if (k < d.nz - 1) edge(true, mz[n], n + 1);
  else edge(pz, mz[n], n - d.wz);
}

__device__ __forceinline__ void node_ijk(const Dims& d, long long n, int& i,
                                         int& j, int& k) {
  if (n <= 0x7fffffffLL) {  // 32-bit divisions while the index fits
    const unsigned u = (unsigned)n, nz = (unsigned)d.nz, ny = (unsigned)d.ny;
    const unsigned t = u / nz;
    k = (int)(u - t * nz);
    i = (int)(t / ny);
    j = (int)(t - (unsigned)i * ny);
    return;
  }
  long long t = n / d.nz;
  k = (int)(n - t * d.nz);
  i = (int)(t / d.ny);
  j = (int)(t - (long long)i * d.ny);
}

// ---- RHS-interleaved vector loads/stores -----------------------------------
// 128-bit accesses by default.  `Wide` selects sm_100's 256-bit accesses
// (ld/st.global.v8.f32, .v4.f64) for nodes of 8 FP32 or 4 FP64 values: one
// instruction per 32-byte node, so a warp request covers whole sectors.
// Measured on the 256x256x128 extraction, they speed up the streaming CG
// kernels (p update 0.138 -> 0.120 ms, x/r update 0.285 -> 0.264 ms) but
// slow the neighbour-gathering smoother and stencil kernels (the degree-2
// post-smoother 0.193 -> 0.258 ms), so only the streaming kernels ask for
// them.  The 256-bit form needs a 32-byte aligned node; nodes are n*32 bytes
// apart, so only the base pointer is checked (a uniform branch) and a base
// that is only 16-byte aligned takes 128-bit accesses.  Every pointer given
// to these helpers is global memory.
__device__ __forceinline__ bool aligned32(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & 31) == 0;
}

template <bool NC>
__device__ __forceinline__ void ld256(const float* p, float& a0, float& a1, float& a2, float& a3,
                                      float& a4, float& a5, float& a6, float& a7) {
  if constexpr (NC)  // read-only data: the compiler may schedule it freely
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(a4), "=f"(a5), "=f"(a6),
                   "=f"(a7)
                 : "l"(p));
  else
    asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a0), "=f"(a1), "=f"(a2), "=f"(a3), "=f"(a4), "=f"(a5), "=f"(a6),
                   "=f"(a7)
                 : "l"(p)
                 : "memory");
}

template <bool NC>
__device__ __forceinline__ void ld256(const double* p, double& a0, double& a1, double& a2,
                                      double& a3) {
  if constexpr (NC)
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3)
                 : "l"(p));
  else
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(a0), "=d"(a1), "=d"(a2), "=d"(a3)
                 : "l"(p)
                 : "memory");
}

__device__ __forceinline__ void st256(float* p, float a0, float a1, float a2, float a3, float a4,
                                      float a5, float a6, float a7) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a0),
               "f"(a1), "f"(a2), "f"(a3), "f"(a4), "f"(a5), "f"(a6), "f"(a7)
               : "memory");
}

__device__ __forceinline__ void st256(double* p, double a0, double a1, double a2, double a3) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a0), "d"(a1), "d"(a2),
               "d"(a3)
               : "memory");
}

// Whole 32-byte chunks of a node, one 256-bit access each (p 32-byte aligned).
template <bool NC, typename T, int K>
__device__ __forceinline__ void ld_chunks32(const T* p, T (&v)[K]) {
  if constexpr (std::is_same<T, float>::value) {
#pragma unroll
    for (int c = 0; c < K / 8; ++c)
      ld256<NC>(p + 8 * c, v[8 * c], v[8 * c + 1], v[8 * c + 2], v[8 * c + 3], v[8 * c + 4],
                v[8 * c + 5], v[8 * c + 6], v[8 * c + 7]);
  } else {
#pragma unroll
    for (int c = 0; c < K / 4; ++c)
      ld256<NC>(p + 4 * c, v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
  }
}

template <typename T, int K>
__device__ __forceinline__ void st_chunks32(T* p, const T (&v)[K]) {
  if constexpr (std::is_same<T, float>::value) {
#pragma unroll
    for (int c = 0; c < K / 8; ++c)
      st256(p + 8 * c, v[8 * c], v[8 * c + 1], v[8 * c + 2], v[8 * c + 3], v[8 * c + 4],
            v[8 * c + 5], v[8 * c + 6], v[8 * c + 7]);
  } else {
#pragma unroll
    for (int c = 0; c < K / 4; ++c) st256(p + 4 * c, v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
  }
}

// K values of T fill whole 32-byte chunks
template <typename T, int K>
constexpr bool node_is_32b() {
  return (K * (int)sizeof(T)) % 32 == 0 &&
         (std::is_same<T, float>::value || std::is_same<T, double>::value);
}

template <typename T, int K, bool Wide = false>
__device__ __forceinline__ void ldv(const T* __restrict__ base, long long n,
                                    T (&v)[K]) {
  const T* p = base + n * K;
  if constexpr (Wide && node_is_32b<T, K>()) {
    if (aligned32(base)) {
      ld_chunks32<false, T, K>(p, v);
      return;
    }
  }
  if constexpr (std::is_same<T, float>::value && K % 4 == 0) {
#pragma unroll
    for (int c = 0; c < K / 4; ++c) {
      float4 t = reinterpret_cast<const float4*>(p)[c];
      v[4 * c] = t.x;
      v[4 * c + 1] = t.y;
      v[4 * c + 2] = t.z;
      v[4 * c + 3] = t.w;
    }
  } else if constexpr (std::is_same<T, float>::value && K == 2) {
    float2 t = reinterpret_cast<const float2*>(p)[0];
    v[0] = t.x;
    v[1] = t.y;
  } else if constexpr (std::is_same<T, double>::value && K % 2 == 0) {
#pragma unroll
    for (int c = 0; c < K / 2; ++c) {
      double2 t = reinterpret_cast<const double2*>(p)[c];
      v[2 * c] = t.x;
      v[2 * c + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < K; ++c) v[c] = p[c];
  }
}

// Read-only-path variant for arrays that no thread writes during the kernel.
template <typename T, int K, bool Wide = false>
__device__ __forceinline__ void ldv_ro(const T* __restrict__ base, long long n,
                                       T (&v)[K]) {
  const T* p = base + n * K;
  if constexpr (Wide && node_is_32b<T, K>()) {
    if (aligned32(base)) {
      ld_chunks32<true, T, K>(p, v);
      return;
    }
  }
  if constexpr (std::is_same<T, float>::value && K % 4 == 0) {
#pragma unroll
    for (int c = 0; c < K / 4; ++c) {
      float4 t = __ldg(reinterpret_cast<const float4*>(p) + c);
      v[4 * c] = t.x;
      v[4 * c + 1] = t.y;
      v[4 * c + 2] = t.z;
      v[4 * c + 3] = t.w;
    }
  } else if constexpr (std::is_same<T, float>::value && K == 2) {
    float2 t = __ldg(reinterpret_cast<const float2*>(p));
    v[0] = t.x;
    v[1] = t.y;
  } else if constexpr (std::is_same<T, double>::value && K % 2 == 0) {
#pragma unroll
    for (int c = 0; c < K / 2; ++c) {
      double2 t = __ldg(reinterpret_cast<const double2*>(p) + c);
      v[2 * c] = t.x;
      v[2 * c + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < K; ++c) v[c] = __ldg(p + c);
  }
}

template <typename T, int K, bool Wide = false>
__device__ __forceinline__ void stv(T* __restrict__ base, long long n,
                                    const T (&v)[K]) {
  T* p = base + n * K;
  if constexpr (Wide && node_is_32b<T, K>()) {
    if (aligned32(base)) {
      st_chunks32<T, K>(p, v);
      return;
    }
  }
  if constexpr (std::is_same<T, float>::value && K % 4 == 0) {
#pragma unroll
    for (int c = 0; c < K / 4; ++c)
      reinterpret_cast<float4*>(p)[c] =
          make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
  } else if constexpr (std::is_same<T, float>::value && K == 2) {
    reinterpret_cast<float2*>(p)[0] = make_float2(v[0], v[1]);
  } else if constexpr (std::is_same<T, double>::value && K % 2 == 0) {
#pragma unroll
    for (int c = 0; c < K / 2; ++c)
      reinterpret_cast<double2*>(p)[c] = make_double2(v[2 * c], v[2 * c + 1]);
  } else {
#pragma unroll
    for (int c = 0; c < K; ++c) p[c] = v[c];
  }
}

// ---- nodes split into FP64 chunks --------------------------------------------
// The streaming per-node kernels that touch the FP64 solution (K doubles per
// node, 64 bytes for 8 RHS) run one thread per 16-byte chunk of it:
// Chunks<K>::NCH threads per node, W = 2 right-hand sides each (1 when
// K == 1), so a warp request covers whole sectors instead of four 16-byte
// pieces 64 bytes apart.  The grid-stride step is a multiple of NCH, so a
// thread keeps its chunk h = threadIdx.x % NCH for the whole loop.
template <int K>
struct Chunks {
  static constexpr int W = K >= 2 ? 2 : 1;  // right-hand sides per thread
  static constexpr int NCH = K / W;         // threads per node
  static_assert(NCH * W == K && (NCH & (NCH - 1)) == 0, "K must be a power of two");
};

// W consecutive values of T at p (8- or 16-byte aligned for W == 2)
template <typename T, int W>
__device__ __forceinline__ void ldw(const T* p, T (&v)[W]) {
  if constexpr (W == 2 && std::is_same<T, float>::value) {
    const float2 t = *reinterpret_cast<const float2*>(p);
    v[0] = t.x;
    v[1] = t.y;
  } else if constexpr (W == 2) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    v[0] = t.x;
    v[1] = t.y;
  } else {
#pragma unroll
    for (int t = 0; t < W; ++t) v[t] = p[t];
  }
}

template <typename T, int W>
__device__ __forceinline__ void stw(T* p, const T (&v)[W]) {
  if constexpr (W == 2 && std::is_same<T, float>::value) {
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
  } else if constexpr (W == 2) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  } else {
#pragma unroll
    for (int t = 0; t < W; ++t) p[t] = v[t];
  }
}

// ---- deterministic reductions ---------------------------------------------
// Each block reduces its per-thread FP64 accumulators in a fixed order
// (warp shuffle tree, then warps in index order) and writes one partial per
// value.  The last block to finish (atomic ticket) sums the partials over
// blocks, again in a fixed order, so results do not depend on scheduling.
// scratch: NT / 32 * M doubles of shared memory (a kernel whose dynamic
// shared memory is free by then passes part of it: no static array that would
// lower its occupancy).
template <int M, int NT>
__device__ __forceinline__ void block_partials_to(double (&acc)[M],
                                                  double* __restrict__ partials,
                                                  double* scratch) {
  static_assert(NT % 32 == 0 && NT >= 32, "block size must be whole warps");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double v = acc[m];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
      v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) scratch[warp * M + m] = v;
  }
  __syncthreads();
  if (threadIdx.x < M) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) s += scratch[w * M + threadIdx.x];
    partials[(size_t)blockIdx.x * M + threadIdx.x] = s;
  }
}

template <int M, int NT = kBlock>
__device__ __forceinline__ void block_partials(double (&acc)[M],
                                               double* __restrict__ partials) {
  __shared__ double sm[NT / 32 * M];
  block_partials_to<M, NT>(acc, partials, sm);
}

// Returns true in exactly one block: the last one to arrive.  That block
// also resets the ticket so the next launch starts from zero.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == gridDim.x - 1);
    if (is_last) *ticket = 0u;
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// Sum partials[b*M + m] over b in a fixed order; call from the last block
// (NT threads).  Result is valid in out[m] for all threads after the call.
// scratch: NT doubles of shared memory.
template <int M, int NT>
__device__ __forceinline__ void grid_total_to(const double* partials, int nblocks,
                                              double (&out)[M], double* scratch) {
  static_assert((NT & (NT - 1)) == 0, "block size must be a power of two");
  for (int m = 0; m < M; ++m) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += NT)
      s += __ldcg(partials + (size_t)b * M + m);
    scratch[threadIdx.x] = s;
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) scratch[threadIdx.x] += scratch[threadIdx.x + w];
      __syncthreads();
    }
    out[m] = scratch[0];
    __syncthreads();
  }
}

template <int M, int NT = kBlock>
__device__ __forceinline__ void grid_total(const double* partials, int nblocks,
                                           double (&out)[M]) {
  __shared__ double red[NT];
  grid_total_to<M, NT>(partials, nblocks, out, red);
}

}  // namespace fs

// ---- host-side error bookkeeping --------------------------------------------
void fs_set_error(const char* where, cudaError_t err);
void fs_set_error_msg(const char* msg);
int fs_cuda_status(const char* where, cudaError_t err);
int fs_grid_blocks(const void* kernel, long long work_items);

#define FS_CHECK(call)                                        \
  do {                                                        \
    cudaError_t _e = (call);                                  \
    if (_e != cudaSuccess) return fs_cuda_status(#call, _e);  \
  } while (0)

#define FS_CHECK_LAUNCH(name)                                     \
  do {                                                            \
    cudaError_t _e = cudaGetLastError();                          \
    if (_e != cudaSuccess) return fs_cuda_status(name, _e);       \
  } while (0)
