// Geometric multigrid V-cycle for the equilibrated, Dirichlet-eliminated
// system  A~ = S A S  (S = diag(A)^-1/2 on free nodes, 0 on fixed nodes).
//
// Levels.  Vertex-centred coarsening: coarse node I sits on fine node 2I, so
// n_c = (n + 1) / 2 per axis.  An axis too short to coarsen (the two node
// planes of a 2-D cross-section, say) is kept as it is (n_c = n, coarse node I
// on fine node I): semi-coarsening, recognised by every kernel below from
// f.n == c.n on that axis.  The coarse operator is a rediscretisation of
// the original Laplacian A: a coarse x-edge joins fine nodes 2I -> 2I+2, i.e.
// two fine x-edges in series, and collects the 3 x 3 fine edge rows around
// it with lateral weights (1/2, 1, 1/2) per direction, which reproduces the
// coarse edge mass 2m of a uniform medium (twice the dual area over twice
// the length) and the half dual areas at the walls.  A coarse node is fixed
// when its fine node is.  Every level is then equilibrated the same way, so
// every level's operator has unit diagonal and one stencil form
//     (A~ u)_i = u_i - sum_e m~_e u_nbr(e).
//
// Transfers.  With trilinear P (weights 1, 1/2, 1/2 per axis; a last fine
// node with no coarse partner takes weight 1 from its lower neighbour), the
// equilibrated prolongation is P~ = S_f^-1 P S_c and restriction R~ = P~^T,
// so that P~^T A~_f P~ = S_c (P^T A_f P) S_c ~ A~_c.  S^-1 is stored as
// `sd` (sqrt(diag), 0 on fixed nodes) and S as `s`.
//
// Smoothing.  Chebyshev polynomials of A~ on [lo, 2]: 2 bounds the spectrum
// of A~ (it is similar to D^-1 A, whose Gershgorin discs lie in [0, 2]).
// Pre- and post-smoothing use the same polynomial and the coarsest level a
// fixed higher-degree one, so the V-cycle is a symmetric linear operator and
// plain PCG applies.
#pragma once

#include "fs_common.cuh"

namespace fs {

// Coarsening ratio of one axis: 2, or 1 where the axis is kept.
__device__ __forceinline__ int ratio(int nf, int nc) { return nf == nc ? 1 : 2; }

// ---- setup (FP64, original scale) ---------------------------------------------
__device__ __forceinline__ double series2(double a, double b) {
  return (a > 0.0 && b > 0.0) ? 1.0 / (1.0 / a + 1.0 / b) : 0.0;
}

// Coarse masses (padded node layout) and coarse "fixed" labels.
__global__ void k_mg_coarsen(Dims f, Dims c, const double* __restrict__ fmx,
                             const double* __restrict__ fmy,
                             const double* __restrict__ fmz,
                             const uint8_t* __restrict__ flabel,
                             double* __restrict__ cmx, double* __restrict__ cmy,
                             double* __restrict__ cmz,
                             uint8_t* __restrict__ clabel) {
  const double lat[3] = {0.5, 1.0, 0.5};
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.N;
       n += (long long)gridDim.x * blockDim.x) {
    int I, J, Kc;
    node_ijk(c, n, I, J, Kc);
    const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
    const int i = rx * I, j = ry * J, k = rz * Kc;
    const long long fn = ((long long)i * f.ny + j) * f.nz + k;
    clabel[n] = flabel[fn] == FS_LABEL_FREE ? FS_LABEL_FREE : FS_LABEL_FIXED;
    // lateral weight of offset a on an axis of ratio r: (1/2, 1, 1/2) when
    // coarsened, the single fine row otherwise
    auto lw = [&](int a, int r) { return r == 2 ? lat[a + 1] : 1.0; };
    // x-edge I -> I+1: fine x-edges i -> i+1 -> i+2 in series (one fine edge
    // on an uncoarsened axis), lateral j, k
    double sx = 0.0, sy = 0.0, sz = 0.0;
    if (I + 1 < c.nx) {
      for (int a = 1 - ry; a <= ry - 1; ++a)
        for (int b = 1 - rz; b <= rz - 1; ++b) {
          const int jj = j + a, kk = k + b;
          if (jj < 0 || jj >= f.ny || kk < 0 || kk >= f.nz) continue;
          const long long m0 = ((long long)i * f.ny + jj) * f.nz + kk;
          sx += lw(a, ry) * lw(b, rz) *
                (rx == 2 ? series2(fmx[m0], fmx[m0 + f.sx]) : fmx[m0]);
        }
    }
    if (J + 1 < c.ny) {
      for (int a = 1 - rx; a <= rx - 1; ++a)
        for (int b = 1 - rz; b <= rz - 1; ++b) {
          const int ii = i + a, kk = k + b;
          if (ii < 0 || ii >= f.nx || kk < 0 || kk >= f.nz) continue;
          const long long m0 = ((long long)ii * f.ny + j) * f.nz + kk;
          sy += lw(a, rx) * lw(b, rz) *
                (ry == 2 ? series2(fmy[m0], fmy[m0 + f.sy]) : fmy[m0]);
        }
    }
    if (Kc + 1 < c.nz) {
      for (int a = 1 - rx; a <= rx - 1; ++a)
        for (int b = 1 - ry; b <= ry - 1; ++b) {
          const int ii = i + a, jj = j + b;
          if (ii < 0 || ii >= f.nx || jj < 0 || jj >= f.ny) continue;
          const long long m0 = ((long long)ii * f.ny + jj) * f.nz + k;
          sz += lw(a, rx) * lw(b, ry) *
                (rz == 2 ? series2(fmz[m0], fmz[m0 + 1]) : fmz[m0]);
        }
    }
    cmx[n] = sx;
    cmy[n] = sy;
    cmz[n] = sz;
  }
}

// s = diag^-1/2 and sd = diag^1/2 in T (both 0 on non-free nodes).
template <typename T>
__global__ void k_mg_scales(long long N, const double* __restrict__ s64,
                            T* __restrict__ s, T* __restrict__ sd) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    const double v = s64[n];
    s[n] = (T)v;
    sd[n] = (T)(v > 0.0 ? 1.0 / v : 0.0);
  }
}

// ---- V-cycle kernels (T, K RHS interleaved) ---------------------------------------
// Three resident blocks per SM where the per-node state is small enough to
// keep in registers (FP32, up to 8 RHS); wider nodes keep the register room.
template <typename T, int K>
constexpr int mg_min_blocks() {
  return sizeof(T) * K <= 32 ? 3 : 1;
}

template <typename T, int K>
__device__ __forceinline__ void apply_eq(const Dims& d, const T* __restrict__ ex,
                                         const T* __restrict__ ey,
                                         const T* __restrict__ ez,
                                         const T* __restrict__ x, long long n,
                                         T (&ax)[K]) {
  int i, j, k;
  node_ijk(d, n, i, j, k);
  ldv_ro<T, K>(x, n, ax);
  auto nbr = [&](T m, long long nb) {
    T v[K];
    ldv_ro<T, K>(x, nb, v);
#pragma unroll
    for (int t = 0; t < K; ++t) ax[t] -= m * v[t];
  };
  if (d.per) {  // a periodic level (aggregation hierarchy): wrap edges
    edge6(d, ex, ey, ez, n, i, j, k, [&](bool ok, T m, long long nb) {
      if (ok) nbr(m, nb);
    });
    return;
  }
  if (i > 0) nbr(__ldg(ex + n - d.sx), n - d.sx);
  if (i < d.nx - 1) nbr(__ldg(ex + n), n + d.sx);
  if (j > 0) nbr(__ldg(ey + n - d.sy), n - d.sy);
  if (j < d.ny - 1) nbr(__ldg(ey + n), n + d.sy);
  if (k > 0) nbr(__ldg(ez + n - 1), n - 1);
  if (k < d.nz - 1) nbr(__ldg(ez + n), n + 1);
}

// One Chebyshev step: d = cd*d + cr*(b - A~ x_in), x_out = x_in + d.
// x_zero: x_in is identically zero (first pre-smoothing step); store_d = 0
// on the last step of a sequence, whose d nobody reads.
template <typename T, int K>
__global__ void __launch_bounds__(kBlock, mg_min_blocks<T, K>())
    k_mg_cheb(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
              const T* __restrict__ ez, const T* __restrict__ xin,
              T* __restrict__ xout, T* __restrict__ dv,
              const T* __restrict__ b, T cd, T cr, int x_zero, int store_d,
              const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T r[K], bv[K], dd[K], xo[K];
    ldv_ro<T, K>(b, n, bv);
    if (x_zero) {
#pragma unroll
      for (int t = 0; t < K; ++t) {
        r[t] = bv[t];
        xo[t] = (T)0;
      }
    } else {
      T ax[K];
      apply_eq<T, K>(d, ex, ey, ez, xin, n, ax);
      ldv_ro<T, K>(xin, n, xo);
#pragma unroll
      for (int t = 0; t < K; ++t) r[t] = bv[t] - ax[t];
    }
    if (cd != (T)0) {
      ldv<T, K>(dv, n, dd);
#pragma unroll
      for (int t = 0; t < K; ++t) dd[t] = cd * dd[t] + cr * r[t];
    } else {
#pragma unroll
      for (int t = 0; t < K; ++t) dd[t] = cr * r[t];
    }
#pragma unroll
    for (int t = 0; t < K; ++t) xo[t] += dd[t];
    if (store_d) stv<T, K>(dv, n, dd);
    stv<T, K>(xout, n, xo);
  }
}

// ---- coarsest level: the whole Chebyshev solve in one launch -----------------
// The coarsest level is small (a few thousand nodes), so its degree-32
// Chebyshev solve is launch-bound as 32 grid-wide steps.  Here one block per
// right-hand side runs every step: the level's iterate lives in shared memory
// (its neighbours are other threads' nodes), b and the step direction d of a
// thread's own nodes in registers, the equilibrated masses in shared memory.
// Each step computes d = cd d + cr (b - A~ x), x += d for all nodes into
// registers, then a barrier, the writes of x, another barrier; the arithmetic
// and its order are k_mg_cheb's, so the result is the same.
constexpr int kCoarseThreads = 1024;
constexpr int kCoarseMaxDeg = 64;
// nodes per thread (registers: b, d and the new x of each): levels up to 8192
// nodes in FP32, 4096 in FP64
template <typename T>
constexpr int coarse_npt() {
  return sizeof(T) == 4 ? 8 : 4;
}

template <typename T>
struct CoarseCoef {
  T cd[kCoarseMaxDeg], cr[kCoarseMaxDeg];
};

// Shared memory of k_mg_coarse for a level of n nodes (x and three mass arrays).
template <typename T>
constexpr size_t coarse_smem(long long n) {
  return (size_t)n * sizeof(T) * 4;
}

constexpr size_t kCoarseSmemCap = 160 * 1024;

// Whether a coarsest level of n nodes and a degree fit k_mg_coarse.
template <typename T>
constexpr bool coarse_fits(long long n, int deg) {
  return n >= 1 && n <= (long long)kCoarseThreads * coarse_npt<T>() && deg >= 1 &&
         deg <= kCoarseMaxDeg && coarse_smem<T>(n) <= kCoarseSmemCap;
}

template <typename T, int K>
__global__ void __launch_bounds__(kCoarseThreads)
    k_mg_coarse(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
                const T* __restrict__ ez, const T* __restrict__ b, T* __restrict__ xout,
                const CoarseCoef<T> coef, int deg, const int* __restrict__ done) {
  if (*done) return;
  extern __shared__ unsigned char smem_raw[];
  const int N = (int)d.N;
  T* xs = reinterpret_cast<T*>(smem_raw);
  T* mx = xs + N;
  T* my = mx + N;
  T* mz = my + N;
  const int col = blockIdx.x;  // right-hand side
  for (int n = threadIdx.x; n < N; n += kCoarseThreads) {
    mx[n] = ex[n];
    my[n] = ey[n];
    mz[n] = ez[n];
  }
  // own nodes n = threadIdx.x + e * kCoarseThreads: b, d and the valid-neighbour mask
  constexpr int NPT = coarse_npt<T>();
  T bv[NPT], dv[NPT], xn[NPT];
  int nb[NPT];
#pragma unroll
  for (int e = 0; e < NPT; ++e) {
    const int n = threadIdx.x + e * kCoarseThreads;
    bv[e] = (T)0;
    dv[e] = (T)0;
    nb[e] = 0;
    if (n < N) {
      bv[e] = b[(long long)n * K + col];
      int i, j, k;
      node_ijk(d, n, i, j, k);
      nb[e] = (i > 0) | ((i < d.nx - 1) << 1) | ((j > 0) << 2) | ((j < d.ny - 1) << 3) |
              ((k > 0) << 4) | ((k < d.nz - 1) << 5);
    }
  }
  const int sx = (int)d.sx, sy = (int)d.sy;
  for (int step = 0; step < deg; ++step) {
    const T cd = coef.cd[step], cr = coef.cr[step];
#pragma unroll
    for (int e = 0; e < NPT; ++e) {
      const int n = threadIdx.x + e * kCoarseThreads;
      if (n >= N) continue;
      T r, xo;
      if (step == 0) {  // x_in = 0
        r = bv[e];
        xo = (T)0;
      } else {
        const int m = nb[e];
        T ax = xs[n];
        if (m & 1) ax -= mx[n - sx] * xs[n - sx];
        if (m & 2) ax -= mx[n] * xs[n + sx];
        if (m & 4) ax -= my[n - sy] * xs[n - sy];
        if (m & 8) ax -= my[n] * xs[n + sy];
        if (m & 16) ax -= mz[n - 1] * xs[n - 1];
        if (m & 32) ax -= mz[n] * xs[n + 1];
        xo = xs[n];
        r = bv[e] - ax;
      }
      dv[e] = cd != (T)0 ? cd * dv[e] + cr * r : cr * r;
      xn[e] = xo + dv[e];
    }
    __syncthreads();  // every read of x (and, first time, of the masses) done
#pragma unroll
    for (int e = 0; e < NPT; ++e) {
      const int n = threadIdx.x + e * kCoarseThreads;
      if (n < N) xs[n] = xn[e];
    }
    __syncthreads();
  }
#pragma unroll
  for (int e = 0; e < NPT; ++e) {
    const int n = threadIdx.x + e * kCoarseThreads;
    if (n < N) xout[(long long)n * K + col] = xn[e];
  }
}

// res = b - A~ x
template <typename T, int K>
__global__ void __launch_bounds__(kBlock, mg_min_blocks<T, K>())
    k_mg_residual(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
                  const T* __restrict__ ez, const T* __restrict__ x,
                  const T* __restrict__ b, T* __restrict__ res,
                  const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T ax[K], bv[K];
    apply_eq<T, K>(d, ex, ey, ez, x, n, ax);
    ldv_ro<T, K>(b, n, bv);
#pragma unroll
    for (int t = 0; t < K; ++t) bv[t] -= ax[t];
    stv<T, K>(res, n, bv);
  }
}

// Degree-2 pre-smoothing from x = 0 in residual form.  The Chebyshev steps
//   x1 = c0 b,  d1 = cd1 x1 + cr1 (b - A~ x1),  x2 = x1 + d1
// need r1 = b - A~ x1 and r2 = r1 - A~ d1 for the restriction; carrying the
// residual along saves the separate residual pass over x2.
// pre0: x1 = c0 b, r1 = b - c0 A~ b.
template <typename T, int K>
__global__ void __launch_bounds__(kBlock, mg_min_blocks<T, K>())
    k_mg_pre0(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
              const T* __restrict__ ez, const T* __restrict__ b,
              T* __restrict__ x1, T* __restrict__ r1, T c0,
              const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T ab[K], bv[K], xo[K];
    apply_eq<T, K>(d, ex, ey, ez, b, n, ab);
    ldv_ro<T, K>(b, n, bv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      xo[t] = c0 * bv[t];
      ab[t] = bv[t] - c0 * ab[t];
    }
    stv<T, K>(x1, n, xo);
    stv<T, K>(r1, n, ab);
  }
}

// pre1: d1 = cd x1 + cr r1 (formed at the node and its six neighbours),
// x2 = x1 + d1, r2 = r1 - A~ d1.
template <typename T, int K>
__global__ void __launch_bounds__(kBlock, mg_min_blocks<T, K>())
    k_mg_pre1(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
              const T* __restrict__ ez, const T* __restrict__ x1,
              const T* __restrict__ r1, T* __restrict__ x2, T* __restrict__ r2,
              T cd, T cr, const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    node_ijk(d, n, i, j, k);
    T xv[K], rv[K], dc[K], ad[K];
    ldv_ro<T, K>(x1, n, xv);
    ldv_ro<T, K>(r1, n, rv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      dc[t] = cd * xv[t] + cr * rv[t];
      ad[t] = dc[t];
    }
    auto nbr = [&](T m, long long nb) {
      T a[K], c[K];
      ldv_ro<T, K>(x1, nb, a);
      ldv_ro<T, K>(r1, nb, c);
#pragma unroll
      for (int t = 0; t < K; ++t) ad[t] -= m * (cd * a[t] + cr * c[t]);
    };
    if (d.per) {  // periodic level: wrap edges
      edge6(d, ex, ey, ez, n, i, j, k, [&](bool ok, T m, long long nb) {
        if (ok) nbr(m, nb);
      });
    } else {
      if (i > 0) nbr(__ldg(ex + n - d.sx), n - d.sx);
      if (i < d.nx - 1) nbr(__ldg(ex + n), n + d.sx);
      if (j > 0) nbr(__ldg(ey + n - d.sy), n - d.sy);
      if (j < d.ny - 1) nbr(__ldg(ey + n), n + d.sy);
      if (k > 0) nbr(__ldg(ez + n - 1), n - 1);
      if (k < d.nz - 1) nbr(__ldg(ez + n), n + 1);
    }
#pragma unroll
    for (int t = 0; t < K; ++t) {
      xv[t] += dc[t];
      rv[t] -= ad[t];
    }
    stv<T, K>(x2, n, xv);
    stv<T, K>(r2, n, rv);
  }
}

// x += u (the learned level's guess added to the V-cycle's correction).
template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    k_mg_add(Dims d, T* __restrict__ x, const T* __restrict__ u, const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T xv[K], uv[K];
    ldv<T, K>(x, n, xv);
    ldv_ro<T, K>(u, n, uv);
#pragma unroll
    for (int t = 0; t < K; ++t) xv[t] += uv[t];
    stv<T, K>(x, n, xv);
  }
}

// Degree-2 post-smoothing in two passes.  With r0 = b - A~ x (a residual
// pass), the two Chebyshev steps d1 = c0 r0, d2 = cd1 d1 + cr1 (r0 - A~ d1)
// collapse to x2 = x + alpha r0 + beta A~ r0, alpha = c0 (1 + cd1) + cr1,
// beta = -cr1 c0: 6 vector passes instead of 8.
template <typename T, int K>
__global__ void __launch_bounds__(kBlock, mg_min_blocks<T, K>())
    k_mg_post2(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
               const T* __restrict__ ez, const T* __restrict__ x, const T* __restrict__ r0,
               T* __restrict__ xout, T alpha, T beta, const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T ar[K], rv[K], xv[K];
    apply_eq<T, K>(d, ex, ey, ez, r0, n, ar);
    ldv_ro<T, K>(r0, n, rv);
    ldv_ro<T, K>(x, n, xv);
#pragma unroll
    for (int t = 0; t < K; ++t) xv[t] += alpha * rv[t] + beta * ar[t];
    stv<T, K>(xout, n, xv);
  }
}

// Per-axis trilinear weights of fine index i onto coarse index I (0 if none);
// the identity on an uncoarsened axis.
__device__ __forceinline__ float pw(int i, int I, int nf, int nc) {
  if (nf == nc) return i == I ? 1.0f : 0.0f;
  const int dlt = i - 2 * I;
  if (dlt == 0) return 1.0f;
  if (dlt == 1) return (I + 1 < nc) ? 0.5f : 1.0f;  // last fine node: weight 1
  if (dlt == -1) return 0.5f;
  return 0.0f;
}

// Coarse node diagonal term (heat capacity / dt, convection): the row-sum
// lumping of P^T D_f P, i.e. d_c(I) = sum_f P(f, I) d_f(f) (P 1 = 1).
__global__ void k_mg_coarsen_diag(Dims f, Dims c, const double* __restrict__ fd,
                                  double* __restrict__ cd) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.N;
       n += (long long)gridDim.x * blockDim.x) {
    int I, J, Kc;
    node_ijk(c, n, I, J, Kc);
    const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
    double acc = 0.0;
    for (int a = 1 - rx; a <= rx - 1; ++a) {
      const int i = rx * I + a;
      if (i < 0 || i >= f.nx) continue;
      const double wa = pw(i, I, f.nx, c.nx);
      for (int b = 1 - ry; b <= ry - 1; ++b) {
        const int j = ry * J + b;
        if (j < 0 || j >= f.ny) continue;
        const double wb = wa * pw(j, J, f.ny, c.ny);
        for (int e = 1 - rz; e <= rz - 1; ++e) {
          const int k = rz * Kc + e;
          if (k < 0 || k >= f.nz) continue;
          const double w = wb * pw(k, Kc, f.nz, c.nz);
          if (w != 0.0) acc += w * fd[((long long)i * f.ny + j) * f.nz + k];
        }
      }
    }
    cd[n] = acc;
  }
}

// b_c(I) = s_c(I) * sum_f P(f,I) sd(f) res(f)   (coarse-centric gather)
template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    k_mg_restrict(Dims f, Dims c, const T* __restrict__ res,
                  const T* __restrict__ sdf, const T* __restrict__ sc,
                  T* __restrict__ bc, const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.N;
       n += (long long)gridDim.x * blockDim.x) {
    const T scale = sc[n];
    T acc[K];
#pragma unroll
    for (int t = 0; t < K; ++t) acc[t] = (T)0;
    if (scale != (T)0) {
      int I, J, Kc;
      node_ijk(c, n, I, J, Kc);
      const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
      for (int a = 1 - rx; a <= rx - 1; ++a) {
        const int i = rx * I + a;
        if (i < 0 || i >= f.nx) continue;
        const float wa = pw(i, I, f.nx, c.nx);
        for (int b = 1 - ry; b <= ry - 1; ++b) {
          const int j = ry * J + b;
          if (j < 0 || j >= f.ny) continue;
          const float wb = wa * pw(j, J, f.ny, c.ny);
          for (int e = 1 - rz; e <= rz - 1; ++e) {
            const int k = rz * Kc + e;
            if (k < 0 || k >= f.nz) continue;
            const long long fn = ((long long)i * f.ny + j) * f.nz + k;
            const T w = (T)(wb * pw(k, Kc, f.nz, c.nz)) * __ldg(sdf + fn);
            if (w == (T)0) continue;
            T v[K];
            ldv_ro<T, K>(res, fn, v);
#pragma unroll
            for (int t = 0; t < K; ++t) acc[t] += w * v[t];
          }
        }
      }
#pragma unroll
      for (int t = 0; t < K; ++t) acc[t] *= scale;
    }
    stv<T, K>(bc, n, acc);
  }
}

// Prolongation, coarse-cell-centric: the thread of coarse node (I, J, Kc)
// writes the fine nodes 2I+a, 2J+b, 2Kc+c (a, b, c in {0, 1}; only offset 0,
// fine node I, on an uncoarsened axis) that it owns,
// interpolating from the up to 8 coarse corners it loads once:
//   x_f += sd(f) * sum_I P(f, I) s_c(I) x_c(I).
template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    k_mg_prolong_cell(Dims f, Dims c, const T* __restrict__ xc,
                      const T* __restrict__ sc, const T* __restrict__ sdf,
                      T* __restrict__ xf, const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.N;
       n += (long long)gridDim.x * blockDim.x) {
    int I, J, Kc;
    node_ijk(c, n, I, J, Kc);
    const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
    // an upper coarse partner exists (and is used) only on coarsened axes
    const bool hx = rx == 2 && I + 1 < c.nx, hy = ry == 2 && J + 1 < c.ny,
               hz = rz == 2 && Kc + 1 < c.nz;
    // corner values v[a][b][e] = s_c x_c at (I+a, J+b, Kc+e); absent -> 0
    T v[2][2][2][K];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const bool ok = (a == 0 || hx) && (b == 0 || hy) && (e == 0 || hz);
          if (ok) {
            const long long cn = n + a * c.sx + b * c.sy + e;
            const T w = __ldg(sc + cn);
            ldv_ro<T, K>(xc, cn, v[a][b][e]);
#pragma unroll
            for (int t = 0; t < K; ++t) v[a][b][e][t] *= w;
          } else {
#pragma unroll
            for (int t = 0; t < K; ++t) v[a][b][e][t] = (T)0;
          }
        }
    // per-axis weights for fine offset 0 (coarse node itself) and 1 (midpoint
    // or, on a last fine node with no upper partner, weight 1 from below)
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int i = rx * I + a;
      if (a >= rx || i >= f.nx) continue;
      const T wa0 = a == 0 ? (T)1 : (hx ? (T)0.5 : (T)1), wa1 = a == 0 ? (T)0 : (hx ? (T)0.5 : (T)0);
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const int j = ry * J + b;
        if (b >= ry || j >= f.ny) continue;
        const T wb0 = b == 0 ? (T)1 : (hy ? (T)0.5 : (T)1), wb1 = b == 0 ? (T)0 : (hy ? (T)0.5 : (T)0);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int k = rz * Kc + e;
          if (e >= rz || k >= f.nz) continue;
          const T we0 = e == 0 ? (T)1 : (hz ? (T)0.5 : (T)1), we1 = e == 0 ? (T)0 : (hz ? (T)0.5 : (T)0);
          const long long fn = ((long long)i * f.ny + j) * f.nz + k;
          const T scale = __ldg(sdf + fn);
          if (scale == (T)0) continue;
          T xv[K];
          ldv<T, K>(xf, fn, xv);
#pragma unroll
          for (int t = 0; t < K; ++t) {
            const T y0 = wb0 * (we0 * v[0][0][0][t] + we1 * v[0][0][1][t]) +
                         wb1 * (we0 * v[0][1][0][t] + we1 * v[0][1][1][t]);
            const T y1 = wb0 * (we0 * v[1][0][0][t] + we1 * v[1][0][1][t]) +
                         wb1 * (we0 * v[1][1][0][t] + we1 * v[1][1][1][t]);
            xv[t] += scale * (wa0 * y0 + wa1 * y1);
          }
          stv<T, K>(xf, fn, xv);
        }
      }
    }
  }
}

// ---- aggregation hierarchy: Galerkin coarse operators --------------------------
// The alternative hierarchy (FS_PRECOND_MG_AGG) for strongly discontinuous
// coefficients (copper in oxide: edge masses 1e6 apart), where rediscretised
// coarse operators and trilinear transfers smear a conductor over its
// surroundings.  Coarse node I is the aggregate of the fine nodes
// r*I .. r*I + r - 1 on each axis (r = 2 where the axis is coarsened, 1 where
// it is kept; the last aggregate of an odd axis holds one node), so the level
// sizes are those of the vertex-centred hierarchy.  P is 1 from an aggregate
// to each of its FREE fine nodes and 0 on fixed ones; the coarse operator is
// exactly P^T A P, which keeps the 7-point form:
//   coarse edge mass I -> I+1 = the sum of the free-free fine edges crossing
//     from aggregate I to aggregate I+1;
//   coarse node term d_c(I) = sum over the aggregate's free nodes of their
//     own term plus the masses of their edges to fixed nodes (the part of
//     the diagonal the coarse edges do not carry); edges inside an aggregate
//     cancel.
// An aggregate with no free node is fixed.  A conductor region therefore
// stays one strongly coupled block on every level, and its near-constant
// modes (a floating copper box) have an exact coarse representation.

__global__ void k_agg_coarsen(Dims f, Dims c, const double* __restrict__ fmx,
                              const double* __restrict__ fmy,
                              const double* __restrict__ fmz,
                              const double* __restrict__ fdg,
                              const uint8_t* __restrict__ flabel,
                              double* __restrict__ cmx, double* __restrict__ cmy,
                              double* __restrict__ cmz, double* __restrict__ cdg,
                              uint8_t* __restrict__ clabel) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.N;
       n += (long long)gridDim.x * blockDim.x) {
    int I, J, Kc;
    node_ijk(c, n, I, J, Kc);
    const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
    const int i0 = rx * I, j0 = ry * J, k0 = rz * Kc;
    const int i1 = min(i0 + rx, f.nx) - 1, j1 = min(j0 + ry, f.ny) - 1,
              k1 = min(k0 + rz, f.nz) - 1;
    bool any_free = false;
    double dg = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int i = i0; i <= i1; ++i)
      for (int j = j0; j <= j1; ++j)
        for (int k = k0; k <= k1; ++k) {
          const long long fn = ((long long)i * f.ny + j) * f.nz + k;
          if (flabel[fn] != FS_LABEL_FREE) continue;
          any_free = true;
          if (fdg) dg += fdg[fn];
          // one fine edge of this free node: to a fixed node it stays on the
          // diagonal; to a free node of the next aggregate up it is part of
          // the coarse edge; inside the aggregate or towards the aggregate
          // below (counted there) it adds nothing here
          auto edge = [&](bool exists, double m, long long nb, bool up_cross, double& acc) {
            if (!exists || m == 0.0) return;
            if (flabel[nb] != FS_LABEL_FREE)
              dg += m;
            else if (up_cross)
              acc += m;
          };
          // on a periodic axis the last plane's +edge is the wrap edge to the
          // first plane (its mass stored on the last plane): the last
          // aggregate's crossing to aggregate 0, kept on the last coarse plane
          double none = 0.0;
          const bool px = f.per & 1, py = (f.per >> 1) & 1, pz = (f.per >> 2) & 1;
          edge(i > 0 || px, i > 0 ? fmx[fn - f.sx] : fmx[fn + f.wx],
               i > 0 ? fn - f.sx : fn + f.wx, false, none);
          edge(i + 1 < f.nx || px, fmx[fn], i + 1 < f.nx ? fn + f.sx : fn - f.wx, i == i1, sx);
          edge(j > 0 || py, j > 0 ? fmy[fn - f.sy] : fmy[fn + f.wy],
               j > 0 ? fn - f.sy : fn + f.wy, false, none);
          edge(j + 1 < f.ny || py, fmy[fn], j + 1 < f.ny ? fn + f.sy : fn - f.wy, j == j1, sy);
          edge(k > 0 || pz, k > 0 ? fmz[fn - 1] : fmz[fn + f.wz],
               k > 0 ? fn - 1 : fn + f.wz, false, none);
          edge(k + 1 < f.nz || pz, fmz[fn], k + 1 < f.nz ? fn + 1 : fn - f.wz, k == k1, sz);
        }
    clabel[n] = any_free ? FS_LABEL_FREE : FS_LABEL_FIXED;
    cdg[n] = any_free ? dg : 0.0;
    cmx[n] = (I + 1 < c.nx || (c.per & 1)) ? sx : 0.0;
    cmy[n] = (J + 1 < c.ny || (c.per & 2)) ? sy : 0.0;
    cmz[n] = (Kc + 1 < c.nz || (c.per & 4)) ? sz : 0.0;
  }
}

// b_c(I) = s_c(I) * sum over the aggregate of sd_f(i) res(i)
template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    k_agg_restrict(Dims f, Dims c, const T* __restrict__ res, const T* __restrict__ sdf,
                   const T* __restrict__ sc, T* __restrict__ bc,
                   const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < c.N;
       n += (long long)gridDim.x * blockDim.x) {
    const T scale = sc[n];
    T acc[K];
#pragma unroll
    for (int t = 0; t < K; ++t) acc[t] = (T)0;
    if (scale != (T)0) {
      int I, J, Kc;
      node_ijk(c, n, I, J, Kc);
      const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
      const int i1 = min(rx * I + rx, f.nx), j1 = min(ry * J + ry, f.ny),
                k1 = min(rz * Kc + rz, f.nz);
      for (int i = rx * I; i < i1; ++i)
        for (int j = ry * J; j < j1; ++j)
          for (int k = rz * Kc; k < k1; ++k) {
            const long long fn = ((long long)i * f.ny + j) * f.nz + k;
            const T w = __ldg(sdf + fn);
            if (w == (T)0) continue;
            T v[K];
            ldv_ro<T, K>(res, fn, v);
#pragma unroll
            for (int t = 0; t < K; ++t) acc[t] += w * v[t];
          }
#pragma unroll
      for (int t = 0; t < K; ++t) acc[t] *= scale;
    }
    stv<T, K>(bc, n, acc);
  }
}

// x_f(i) += alpha * sd_f(i) * s_c(I) * x_c(I), I the aggregate of fine node i
// (one thread per fine node: coalesced fine accesses, coarse values from
// cache).  alpha over-corrects: the piecewise-constant coarse space of
// unsmoothed aggregation captures the error's coarse component with too little
// energy, and a fixed factor in (1, 2) restores most of what smoothed
// transfers would (the V-cycle stays symmetric, and positive definite for
// alpha < 2).
template <typename T, int K>
__global__ void __launch_bounds__(kBlock)
    k_agg_prolong(Dims f, Dims c, const T* __restrict__ xc, const T* __restrict__ sc,
                  const T* __restrict__ sdf, T* __restrict__ xf, T alpha,
                  const int* __restrict__ done) {
  if (*done) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < f.N;
       n += (long long)gridDim.x * blockDim.x) {
    const T sf = __ldg(sdf + n);
    if (sf == (T)0) continue;
    int i, j, k;
    node_ijk(f, n, i, j, k);
    const int rx = ratio(f.nx, c.nx), ry = ratio(f.ny, c.ny), rz = ratio(f.nz, c.nz);
    const long long cn = ((long long)(i / rx) * c.ny + j / ry) * c.nz + k / rz;
    const T w = sf * __ldg(sc + cn) * alpha;
    T v[K], xv[K];
    ldv_ro<T, K>(xc, cn, v);
    ldv<T, K>(xf, n, xv);
#pragma unroll
    for (int t = 0; t < K; ++t) xv[t] += w * v[t];
    stv<T, K>(xf, n, xv);
  }
}

}  // namespace fs
