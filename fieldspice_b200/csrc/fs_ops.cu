// Stand-alone FP64/FP32 stencil applies and the FP64 post-processing
// reductions: terminal charge / current integration and edge energies.
#include <mutex>
#include <stdio.h>

#include "fs_common.cuh"
#include "fs_tma.cuh"

using fs::Dims;

namespace {

// y = L x (optionally the eliminated operator: x read as 0 and y written 0
// on non-free nodes).  Thread per node, all RHS per thread.
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_stencil(Dims d, const T* __restrict__ x, T* __restrict__ y,
              const T* __restrict__ mx, const T* __restrict__ my,
              const T* __restrict__ mz, const uint8_t* __restrict__ label,
              const T* __restrict__ add) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T out[K];
    if (label && label[n] != FS_LABEL_FREE) {
#pragma unroll
      for (int t = 0; t < K; ++t) out[t] = (T)0;
      fs::stv<T, K>(y, n, out);
      continue;
    }
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    T xc[K];
    fs::ldv_ro<T, K>(x, n, xc);
#pragma unroll
    for (int t = 0; t < K; ++t) out[t] = (T)0;
    auto nbr = [&](T m, long long nb) {
      T xn[K];
      const bool zero = label && label[nb] != FS_LABEL_FREE;
      if (zero) {
#pragma unroll
        for (int t = 0; t < K; ++t) xn[t] = (T)0;
      } else {
        fs::ldv_ro<T, K>(x, nb, xn);
      }
#pragma unroll
      for (int t = 0; t < K; ++t) out[t] += m * (xc[t] - xn[t]);
    };
    if (i > 0) nbr(mx[n - d.sx], n - d.sx);
    if (i < d.nx - 1) nbr(mx[n], n + d.sx);
    if (j > 0) nbr(my[n - d.sy], n - d.sy);
    if (j < d.ny - 1) nbr(my[n], n + d.sy);
    if (k > 0) nbr(mz[n - 1], n - 1);
    if (k < d.nz - 1) nbr(mz[n], n + 1);
    if (add) {
      T a[K];
      fs::ldv_ro<T, K>(add, n, a);
#pragma unroll
      for (int t = 0; t < K; ++t) out[t] += a[t];
    }
    fs::stv<T, K>(y, n, out);
  }
}

template <typename T>
int launch_stencil(const Dims& d, int nrhs, const T* x, T* y, const T* mx,
                   const T* my, const T* mz, const uint8_t* label, const T* add,
                   cudaStream_t s) {
#define FS_ST(KK)                                                           \
  case KK: {                                                                \
    int g = fs_grid_blocks((const void*)k_stencil<T, KK>, d.N);             \
    k_stencil<T, KK><<<g, fs::kBlock, 0, s>>>(d, x, y, mx, my, mz, label,   \
                                              add);                         \
    FS_CHECK_LAUNCH("k_stencil");                                           \
    return FS_OK;                                                           \
  }
  switch (nrhs) {
    FS_ST(1)
    FS_ST(2)
    FS_ST(4)
    FS_ST(8)
    FS_ST(16)
    default: return FS_BAD_ARG;
  }
#undef FS_ST
}

// Per-group sums of (L_A u - L_B w) over explicit node lists.  Grid: one row
// of `chunks` blocks per group; each block reduces its slice of the group's
// nodes, the last block sums the partials in a fixed order.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_group_apply(Dims d, const double* __restrict__ ax,
                  const double* __restrict__ ay, const double* __restrict__ az,
                  const double* __restrict__ u, const double* __restrict__ bx,
                  const double* __restrict__ by, const double* __restrict__ bz,
                  const double* __restrict__ w,
                  const long long* __restrict__ nodes,
                  const long long* __restrict__ offsets, int ngroups,
                  int chunks, double* __restrict__ partials,
                  double* __restrict__ out, unsigned int* ticket) {
  const int g = blockIdx.x / chunks, c = blockIdx.x % chunks;
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  const long long lo = offsets[g], hi = offsets[g + 1];
  for (long long e = lo + (long long)c * blockDim.x + threadIdx.x; e < hi;
       e += (long long)chunks * blockDim.x) {
    const long long n = nodes[e];
    if (n < 0 || n >= d.N) continue;  // host validates; never index out of range
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    auto apply = [&](const double* mx, const double* my, const double* mz,
                     const double* v, double sign) {
      double vc[K];
#pragma unroll
      for (int t = 0; t < K; ++t) vc[t] = v[n * K + t];
      auto edge = [&](bool ok, double m, long long nb) {
        if (!ok || m == 0.0) return;
#pragma unroll
        for (int t = 0; t < K; ++t) acc[t] += sign * m * (vc[t] - v[nb * K + t]);
      };
      edge(i > 0, i > 0 ? mx[n - d.sx] : 0.0, n - d.sx);
      edge(i < d.nx - 1, mx[n], n + d.sx);
      edge(j > 0, j > 0 ? my[n - d.sy] : 0.0, n - d.sy);
      edge(j < d.ny - 1, my[n], n + d.sy);
      edge(k > 0, k > 0 ? mz[n - 1] : 0.0, n - 1);
      edge(k < d.nz - 1, mz[n], n + 1);
    };
    apply(ax, ay, az, u, 1.0);
    if (bx) apply(bx, by, bz, w, -1.0);
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(ticket)) {
    // out[g][t] = sum over that group's chunks, in chunk order.
    const int total = ngroups * K;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      const int gg = idx / K, t = idx % K;
      double s = 0.0;
      for (int cc = 0; cc < chunks; ++cc)
        s += __ldcg(partials + ((size_t)gg * chunks + cc) * K + t);
      out[idx] = s;
    }
  }
}

// out[t] = sum_e m_e (u_head - u_tail)^2 per RHS.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_quadform(Dims d, const double* __restrict__ mx,
               const double* __restrict__ my, const double* __restrict__ mz,
               const double* __restrict__ u, double* __restrict__ partials,
               double* __restrict__ out, unsigned int* ticket) {
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    auto edge = [&](bool ok, double m, long long nb) {
      if (!ok) return;
#pragma unroll
      for (int t = 0; t < K; ++t) {
        const double df = u[nb * K + t] - u[n * K + t];
        acc[t] += m * df * df;
      }
    };
    edge(i < d.nx - 1, mx[n], n + d.sx);
    edge(j < d.ny - 1, my[n], n + d.sy);
    edge(k < d.nz - 1, mz[n], n + 1);
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(ticket)) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) out[threadIdx.x] = tot[threadIdx.x];
  }
}

constexpr int kGroupChunks = 32;
constexpr int kQuadMaxBlocks = 4096;

// ---- static scratch of fs_group_apply_noalloc ---------------------------------
// One 256-byte slot for the completion ticket, then the per-block partial
// sums: ngroups * kGroupChunks * nrhs doubles.  Every GPU that loads this
// library holds one copy (512 KiB + 256 B) until the process exits.
constexpr int kNoAllocMaxGroupRhs = 2048;  // limit on ngroups * nrhs
constexpr size_t kNoAllocScratchBytes =
    256 + (size_t)kNoAllocMaxGroupRhs * kGroupChunks * sizeof(double);
static __device__ __align__(256) unsigned char
    g_group_scratch[kNoAllocScratchBytes];

// Host code may not pass `g_group_scratch` itself to a kernel: in host code
// that name is a stand-in, not a device address.  The device address is
// looked up once per device (with that device current) and cached.
constexpr int kMaxDevices = fs::kMaxDevices;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

int group_scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fs_cuda_status("cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) {
    fs_set_error_msg("fs_group_apply_noalloc: device ordinal beyond 64");
    return FS_BAD_ARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_group_scratch);
    if (e != cudaSuccess) return fs_cuda_status("cudaGetSymbolAddress", e);
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return FS_OK;
}

size_t group_ws(int ngroups, int nrhs) {
  return 256 + (size_t)ngroups * kGroupChunks * nrhs * 8;
}

}  // namespace

extern "C" {

int fs_stencil_apply(const void* x, void* y, const void* mx, const void* my,
                     const void* mz, const uint8_t* label, int nx, int ny,
                     int nz, int nrhs, int dtype, void* stream) {
  if (!x || !y || !mx || !my || !mz || nx < 2 || ny < 2 || nz < 2)
    return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == FS_DTYPE_F64)
    return launch_stencil<double>(d, nrhs, (const double*)x, (double*)y,
                                  (const double*)mx, (const double*)my,
                                  (const double*)mz, label, nullptr, s);
  if (dtype == FS_DTYPE_F32)
    return launch_stencil<float>(d, nrhs, (const float*)x, (float*)y,
                                 (const float*)mx, (const float*)my,
                                 (const float*)mz, label, nullptr, s);
  return FS_BAD_ARG;
}

int fs_apply_laplacian(const double* mx, const double* my, const double* mz,
                       const double* u, const double* add, double* out, int nx,
                       int ny, int nz, int nrhs, void* stream) {
  if (!mx || !my || !mz || !u || !out || nx < 2 || ny < 2 || nz < 2)
    return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  return launch_stencil<double>(d, nrhs, u, out, mx, my, mz, nullptr, add,
                                (cudaStream_t)stream);
}

int fs_group_apply_workspace_bytes(int ngroups, int nrhs, size_t* bytes) {
  if (ngroups < 1 || nrhs < 1 || nrhs > fs::kMaxRhs || !bytes) return FS_BAD_ARG;
  *bytes = group_ws(ngroups, nrhs);
  return FS_OK;
}

int fs_group_apply(const double* mAx, const double* mAy, const double* mAz,
                   const double* u, const double* mBx, const double* mBy,
                   const double* mBz, const double* w, const long long* nodes,
                   const long long* offsets, int ngroups, int nx, int ny,
                   int nz, int nrhs, double* out, void* workspace,
                   size_t workspace_bytes, void* stream) {
  if (!mAx || !mAy || !mAz || !u || !nodes || !offsets || !out || !workspace ||
      ngroups < 1 || nx < 2 || ny < 2 || nz < 2)
    return FS_BAD_ARG;
  if (mBx && (!mBy || !mBz || !w)) return FS_BAD_ARG;
  if (workspace_bytes < group_ws(ngroups, nrhs) || ((uintptr_t)workspace & 255))
    return FS_BAD_ARG;
  if ((long long)ngroups * kGroupChunks > 65535LL * 1024) return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* ticket = (unsigned int*)workspace;
  double* partials = (double*)((char*)workspace + 256);
  FS_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s));
  const int grid = ngroups * kGroupChunks;
#define FS_GA(KK)                                                            \
  case KK:                                                                   \
    k_group_apply<KK><<<grid, fs::kBlock, 0, s>>>(                           \
        d, mAx, mAy, mAz, u, mBx, mBy, mBz, w, nodes, offsets, ngroups,      \
        kGroupChunks, partials, out, ticket);                                \
    FS_CHECK_LAUNCH("k_group_apply");                                        \
    return FS_OK;
  switch (nrhs) {
    FS_GA(1)
    FS_GA(2)
    FS_GA(4)
    FS_GA(8)
    FS_GA(16)
    default: return FS_BAD_ARG;
  }
#undef FS_GA
}

int fs_quadform_workspace_bytes(int nrhs, size_t* bytes) {
  if (nrhs < 1 || nrhs > fs::kMaxRhs || !bytes) return FS_BAD_ARG;
  *bytes = 256 + (size_t)kQuadMaxBlocks * nrhs * 8;
  return FS_OK;
}

int fs_quadform(const double* mx, const double* my, const double* mz,
                const double* u, int nx, int ny, int nz, int nrhs, double* out,
                void* workspace, size_t workspace_bytes, void* stream) {
  size_t need = 0;
  if (fs_quadform_workspace_bytes(nrhs, &need) != FS_OK) return FS_BAD_ARG;
  if (!mx || !my || !mz || !u || !out || !workspace || workspace_bytes < need ||
      nx < 2 || ny < 2 || nz < 2 || ((uintptr_t)workspace & 255))
    return FS_BAD_ARG;
  Dims d = fs::make_dims(nx, ny, nz);
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* ticket = (unsigned int*)workspace;
  double* partials = (double*)((char*)workspace + 256);
  FS_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s));
#define FS_QF(KK)                                                             \
  case KK: {                                                                  \
    int g = fs_grid_blocks((const void*)k_quadform<KK>, d.N);                 \
    if (g > kQuadMaxBlocks) g = kQuadMaxBlocks;                               \
    k_quadform<KK><<<g, fs::kBlock, 0, s>>>(d, mx, my, mz, u, partials, out,  \
                                            ticket);                          \
    FS_CHECK_LAUNCH("k_quadform");                                            \
    return FS_OK;                                                             \
  }
  switch (nrhs) {
    FS_QF(1)
    FS_QF(2)
    FS_QF(4)
    FS_QF(8)
    FS_QF(16)
    default: return FS_BAD_ARG;
  }
#undef FS_QF
}

int fs_group_apply_noalloc(const double* mAx, const double* mAy,
                           const double* mAz, const double* u,
                           const double* mBx, const double* mBy,
                           const double* mBz, const double* w,
                           const long long* nodes, const long long* offsets,
                           int ngroups, int nx, int ny, int nz, int nrhs,
                           double* out, void* stream) {
  if (!mAx || !mAy || !mAz || !u || !nodes || !offsets || !out ||
      ngroups < 1 || nx < 2 || ny < 2 || nz < 2 || nrhs < 1)
    return FS_BAD_ARG;
  if (mBx && (!mBy || !mBz || !w)) return FS_BAD_ARG;
  // every argument is checked before the shared array is touched
  if (nrhs != 1 && nrhs != 2 && nrhs != 4 && nrhs != 8 && nrhs != 16) {
    char msg[128];
    snprintf(msg, sizeof(msg),
             "fs_group_apply_noalloc: nrhs = %d; it must be 1, 2, 4, 8 or 16", nrhs);
    fs_set_error_msg(msg);
    return FS_BAD_ARG;
  }
  if ((long long)ngroups * nrhs > kNoAllocMaxGroupRhs) {
    char msg[160];
    snprintf(msg, sizeof(msg),
             "fs_group_apply_noalloc: ngroups*nrhs = %lld exceeds the static "
             "scratch limit of %d",
             (long long)ngroups * nrhs, kNoAllocMaxGroupRhs);
    fs_set_error_msg(msg);
    return FS_BAD_ARG;
  }
  void* scratch = nullptr;
  int st = group_scratch_address(&scratch);
  if (st != FS_OK) return st;
  Dims d = fs::make_dims(nx, ny, nz);
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* ticket = (unsigned int*)scratch;
  double* partials = (double*)((char*)scratch + 256);
  // The array keeps whatever the previous call left; the ticket must start
  // at zero (the partials are written before they are read).
  FS_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s));
  const int grid = ngroups * kGroupChunks;
#define FS_GA(KK)                                                            \
  case KK:                                                                   \
    k_group_apply<KK><<<grid, fs::kBlock, 0, s>>>(                           \
        d, mAx, mAy, mAz, u, mBx, mBy, mBz, w, nodes, offsets, ngroups,      \
        kGroupChunks, partials, out, ticket);                                \
    FS_CHECK_LAUNCH("k_group_apply");                                        \
    return FS_OK;
  switch (nrhs) {
    FS_GA(1)
    FS_GA(2)
    FS_GA(4)
    FS_GA(8)
    FS_GA(16)
    default: return FS_BAD_ARG;
  }
#undef FS_GA
}

}  // extern "C"

// ---- bounded-wait self test ---------------------------------------------------------
// One thread waits on an mbarrier that nothing will ever complete, with a
// clock budget; when the budget runs out it records FS_TIMEOUT and returns.
// This exercises, on the device, the path every TMA/tcgen05 wait of the
// library takes on a timeout, without a hang and without a fault.
namespace {
__global__ void k_selftest_wait(long long budget, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    fs::mbar_init(&bar, 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const bool ok = fs::mbar_wait_bounded(&bar, 0, budget);
    *status = ok ? FS_OK : FS_TIMEOUT;
  }
}
}  // namespace

extern "C" int fs_selftest_wait_timeout(long long budget_cycles, int* status_host, void* stream) {
  if (budget_cycles < 1 || budget_cycles > 4000000000LL || !status_host) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int* d = nullptr;
  FS_CHECK(cudaMallocAsync((void**)&d, sizeof(int), s));
  FS_CHECK(cudaMemsetAsync(d, 0xff, sizeof(int), s));
  k_selftest_wait<<<1, 32, 0, s>>>(budget_cycles, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(status_host, d, sizeof(int), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(d, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fs_cuda_status("fs_selftest_wait_timeout", e);
  return FS_OK;
}

// ---- input validation on the device ---------------------------------------------------
// min, max and the count of non-finite values of an FP64 array, in one pass
// (the reference's eager checks of a cell property, poisson.py:733-742,
// 872-877, without a host pass over the array).  Per-block partials, the
// last block folds them in a fixed order.
namespace {
__global__ void k_prop_stats(const double* __restrict__ p, long long n, double* __restrict__ part,
                             unsigned int* ticket, double* __restrict__ out) {
  double mn = INFINITY, mx = -INFINITY, bad = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = p[i];
    if (!isfinite(v)) {
      bad += 1.0;
    } else {
      mn = fmin(mn, v);
      mx = fmax(mx, v);
    }
  }
  __shared__ double smn[fs::kBlock], smx[fs::kBlock], sbd[fs::kBlock];
  smn[threadIdx.x] = mn;
  smx[threadIdx.x] = mx;
  sbd[threadIdx.x] = bad;
  __syncthreads();
  for (int w = fs::kBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      smn[threadIdx.x] = fmin(smn[threadIdx.x], smn[threadIdx.x + w]);
      smx[threadIdx.x] = fmax(smx[threadIdx.x], smx[threadIdx.x + w]);
      sbd[threadIdx.x] += sbd[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = smn[0];
    part[3 * blockIdx.x + 1] = smx[0];
    part[3 * blockIdx.x + 2] = sbd[0];
  }
  if (fs::last_block(ticket) && threadIdx.x == 0) {
    double a = INFINITY, b = -INFINITY, c = 0.0;
    for (unsigned int k = 0; k < gridDim.x; ++k) {
      a = fmin(a, __ldcg(part + 3 * k));
      b = fmax(b, __ldcg(part + 3 * k + 1));
      c += __ldcg(part + 3 * k + 2);
    }
    out[0] = a;
    out[1] = b;
    out[2] = c;
  }
}
}  // namespace

// The partials, result and ticket live in the caller's workspace: a
// stream-ordered allocation here returned its memory to the driver at the
// synchronisation below, which waited for the work of every stream (measured:
// 0.4 s of a 64-geometry batch whose builds overlap other plans' solves).
extern "C" int fs_prop_stats_enqueue(const double* p, long long n, void* workspace,
                                     size_t workspace_bytes, void* stream) {
  constexpr int g = 592;
  static_assert(sizeof(double) * (3 * g + 3) + sizeof(unsigned int) <=
                    FS_PROP_STATS_WORKSPACE_BYTES, "workspace constant too small");
  static_assert(sizeof(double) * 3 * g == FS_PROP_STATS_RESULT_OFFSET,
                "result offset constant out of date");
  if (!p || n < 1 || !workspace || workspace_bytes < FS_PROP_STATS_WORKSPACE_BYTES ||
      ((uintptr_t)workspace & 15))
    return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  double* buf = (double*)workspace;
  unsigned int* ticket = (unsigned int*)(buf + 3 * g + 3);
  FS_CHECK(cudaMemsetAsync(ticket, 0, sizeof(unsigned int), s));
  k_prop_stats<<<g, fs::kBlock, 0, s>>>(p, n, buf, ticket, buf + 3 * g);
  FS_CHECK_LAUNCH("k_prop_stats");
  return FS_OK;
}

extern "C" int fs_prop_stats(const double* p, long long n, double* stats_host, void* workspace,
                             size_t workspace_bytes, void* stream) {
  if (!stats_host) return FS_BAD_ARG;
  const int st = fs_prop_stats_enqueue(p, n, workspace, workspace_bytes, stream);
  if (st != FS_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(stats_host, (const char*)workspace + FS_PROP_STATS_RESULT_OFFSET,
                                  3 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fs_cuda_status("fs_prop_stats", e);
  return FS_OK;
}

namespace {
struct SuperposeCoef {
  double c[16];
};

// out[n] = base[n] + sum_c coef[c] * phi[n*k + c0 + c]: the back-substitution
// of a field region as a superposition of its unit-excitation solutions.
__global__ void __launch_bounds__(fs::kBlock)
    k_rhs_superpose(const double* __restrict__ phi, int k, int c0, int ncols,
                    SuperposeCoef coef, const double* __restrict__ base,
                    double* __restrict__ out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double acc = base ? base[i] : 0.0;
    const double* row = phi + i * k + c0;
    for (int c = 0; c < ncols; ++c) acc = fma(coef.c[c], row[c], acc);
    out[i] = acc;
  }
}
}  // namespace

extern "C" int fs_rhs_superpose(const double* phi, int k, int c0, int ncols,
                                const double* coef_host, const double* base,
                                double* out, long long n, void* stream) {
  if (!phi || !out || !coef_host || n < 0 || k < 1 || c0 < 0 || ncols < 0 ||
      ncols > 16 || c0 + ncols > k)
    return FS_BAD_ARG;
  if (n == 0) return FS_OK;
  SuperposeCoef cf{};
  for (int c = 0; c < ncols; ++c) cf.c[c] = coef_host[c];
  int g = fs_grid_blocks((const void*)k_rhs_superpose, n);
  k_rhs_superpose<<<g, fs::kBlock, 0, (cudaStream_t)stream>>>(phi, k, c0, ncols, cf,
                                                               base, out, n);
  FS_CHECK_LAUNCH("k_rhs_superpose");
  return FS_OK;
}
