// Harmonic (phasor) EQS solve: the complex-symmetric system
//   K phi = 0,  K = A + jB  (A = L_sigma - w L_eps'', B = w L_eps'),
// phi fixed on the Dirichlet (terminal) nodes; fieldspice/solvers/ac.py:69-145.
//
// Method: conjugate-orthogonal CG (COCG: CG with the unconjugated bilinear form
// x^T y, valid for complex-symmetric K) on the eliminated system, equilibrated
// with the real scaling S = diag(P)^-1/2 of the SPD companion P = |A| + |B|,
// and preconditioned by the multigrid V-cycle of S P S applied to the real and
// imaginary parts separately.  With A, B >= 0 the preconditioned spectrum lies
// near the segment from 1 to j, so the iteration count stays that of the real
// multigrid PCG.  The V-cycle comes from an FP64 multigrid plan built on P
// (fs_pcg_plan_precondition); everything here is FP64.
//
// Vector layout: N x K values, K = 2H in {2, 4, 8, 16}; column c < H holds the
// real part and column H + c the imaginary part of right-hand side c.
#include <stdio.h>

#include "fs_common.cuh"

using fs::Dims;

namespace {

struct AcState {
  double rho_re, rho_im;      // r~^T z (unconjugated)
  double alpha_re, alpha_im;
  double beta_re, beta_im;
  double rr;                  // ||r~||^2 (conjugated norm)
  double bb;                  // ||b~||^2
  double tol2;                // tol^2
  int active, iters, status, fresh;
};

enum { kTkApply = 0, kTkUpdate = 1, kTkRz = 2, kTkRhs = 3, kTkRes = 4, kTickets = 8 };

__device__ __forceinline__ void cdiv(double ar, double ai, double br, double bi, double& qr,
                                     double& qi) {
  // (ar + j ai) / (br + j bi), scaled to avoid overflow (Smith's method)
  if (fabs(br) >= fabs(bi)) {
    const double t = bi / br, den = br + bi * t;
    qr = (ar + ai * t) / den;
    qi = (ai - ar * t) / den;
  } else {
    const double t = br / bi, den = br * t + bi;
    qr = (ar * t + ai) / den;
    qi = (ai * t - ar) / den;
  }
}

// Equilibrated masses and diagonals of A and B: e = m s_i s_j (0 where an end
// is not free), d = s^2 * (sum of the node's incident masses).
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_setup(Dims d, const double* __restrict__ mA, const double* __restrict__ mB,
               const double* __restrict__ s64, double* __restrict__ eA,
               double* __restrict__ eB, double* __restrict__ dA, double* __restrict__ dB) {
  const long long N = d.N;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    const double s = s64[n];
    eA[n] = i < d.nx - 1 ? mA[n] * s * s64[n + d.sx] : 0.0;
    eA[N + n] = j < d.ny - 1 ? mA[N + n] * s * s64[n + d.sy] : 0.0;
    eA[2 * N + n] = k < d.nz - 1 ? mA[2 * N + n] * s * s64[n + 1] : 0.0;
    eB[n] = i < d.nx - 1 ? mB[n] * s * s64[n + d.sx] : 0.0;
    eB[N + n] = j < d.ny - 1 ? mB[N + n] * s * s64[n + d.sy] : 0.0;
    eB[2 * N + n] = k < d.nz - 1 ? mB[2 * N + n] * s * s64[n + 1] : 0.0;
    double sa = 0.0, sb = 0.0;
    if (i > 0) { sa += mA[n - d.sx]; sb += mB[n - d.sx]; }
    if (i < d.nx - 1) { sa += mA[n]; sb += mB[n]; }
    if (j > 0) { sa += mA[N + n - d.sy]; sb += mB[N + n - d.sy]; }
    if (j < d.ny - 1) { sa += mA[N + n]; sb += mB[N + n]; }
    if (k > 0) { sa += mA[2 * N + n - 1]; sb += mB[2 * N + n - 1]; }
    if (k < d.nz - 1) { sa += mA[2 * N + n]; sb += mB[2 * N + n]; }
    dA[n] = s * s * sa;
    dB[n] = s * s * sb;
  }
}

// Sum over the six edges of node n of (mA + j mB)_e * phi(nbr) restricted to
// neighbours that satisfy `use(nbr)`; all H complex right-hand sides.
template <int K, typename Use>
__device__ __forceinline__ void coupled_sum(const Dims& d, const double* __restrict__ mA,
                                            const double* __restrict__ mB,
                                            const double* __restrict__ phi, long long n,
                                            Use use, double (&re)[K / 2],
                                            double (&im)[K / 2], double& da, double& db) {
  constexpr int H = K / 2;
  const long long N = d.N;
  int i, j, k;
  fs::node_ijk(d, n, i, j, k);
#pragma unroll
  for (int c = 0; c < H; ++c) re[c] = im[c] = 0.0;
  da = db = 0.0;
  auto edge = [&](double a, double b, long long nb) {
    da += a;
    db += b;
    if (!use(nb)) return;
    double v[K];
    fs::ldv<double, K>(phi, nb, v);
#pragma unroll
    for (int c = 0; c < H; ++c) {
      re[c] += a * v[c] - b * v[H + c];
      im[c] += a * v[H + c] + b * v[c];
    }
  };
  if (i > 0) edge(mA[n - d.sx], mB[n - d.sx], n - d.sx);
  if (i < d.nx - 1) edge(mA[n], mB[n], n + d.sx);
  if (j > 0) edge(mA[N + n - d.sy], mB[N + n - d.sy], n - d.sy);
  if (j < d.ny - 1) edge(mA[N + n], mB[N + n], n + d.sy);
  if (k > 0) edge(mA[2 * N + n - 1], mB[2 * N + n - 1], n - 1);
  if (k < d.nz - 1) edge(mA[2 * N + n], mB[2 * N + n], n + 1);
}

// b~ = S (sum over fixed neighbours of (mA + j mB) phi_D) on free nodes, the
// eliminated right-hand side of K phi = 0 (the complex apply_dirichlet of
// ac.py:166-181); x~ = 0, r~ = b~; ||b~||^2 per RHS.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_rhs(Dims d, const double* __restrict__ mA, const double* __restrict__ mB,
             const double* __restrict__ s64, const uint8_t* __restrict__ label,
             const double* __restrict__ phi, double* __restrict__ x, double* __restrict__ r,
             double* __restrict__ partials, AcState* st, unsigned int* tickets) {
  constexpr int H = K / 2;
  double acc[H];
#pragma unroll
  for (int c = 0; c < H; ++c) acc[c] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    double out[K];
#pragma unroll
    for (int c = 0; c < K; ++c) out[c] = 0.0;
    if (label[n] == FS_LABEL_FREE) {
      double re[H], im[H], da, db;
      coupled_sum<K>(d, mA, mB, phi, n, [&](long long nb) { return label[nb] == FS_LABEL_FIXED; },
                     re, im, da, db);
      const double s = s64[n];
#pragma unroll
      for (int c = 0; c < H; ++c) {
        out[c] = s * re[c];
        out[H + c] = s * im[c];
        acc[c] += out[c] * out[c] + out[H + c] * out[H + c];
      }
    }
    fs::stv<double, K>(r, n, out);
#pragma unroll
    for (int c = 0; c < K; ++c) out[c] = 0.0;
    fs::stv<double, K>(x, n, out);
  }
  fs::block_partials<H>(acc, partials);
  if (fs::last_block(&tickets[kTkRhs])) {
    double tot[H];
    fs::grid_total<H>(partials, gridDim.x, tot);
    if (threadIdx.x < H) {
      AcState& a = st[threadIdx.x];
      a.bb = tot[threadIdx.x];
      a.rr = a.bb;
      a.iters = 0;
      a.fresh = 1;
      a.alpha_re = a.alpha_im = a.beta_re = a.beta_im = 0.0;
      a.rho_re = a.rho_im = 0.0;
      a.status = FS_NOT_CONVERGED;
      a.active = a.bb > 0.0 ? 1 : 0;
      if (!a.active) a.status = FS_OK;  // zero right-hand side: x = 0
    }
  }
}

// q = K~ p and the unconjugated p^T q; the last block forms alpha = rho / p^T q.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_apply(Dims d, const double* __restrict__ eA, const double* __restrict__ eB,
               const double* __restrict__ dA, const double* __restrict__ dB,
               const double* __restrict__ p, double* __restrict__ q,
               double* __restrict__ partials, AcState* st, unsigned int* tickets) {
  constexpr int H = K / 2;
  const long long N = d.N;
  double acc[K];
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    double pc[K], qv[K];
    fs::ldv<double, K>(p, n, pc);
    const double a0 = dA[n], b0 = dB[n];
#pragma unroll
    for (int c = 0; c < H; ++c) {
      qv[c] = a0 * pc[c] - b0 * pc[H + c];
      qv[H + c] = a0 * pc[H + c] + b0 * pc[c];
    }
    auto nbr = [&](double a, double b, long long nb) {
      if (a == 0.0 && b == 0.0) return;
      double v[K];
      fs::ldv<double, K>(p, nb, v);
#pragma unroll
      for (int c = 0; c < H; ++c) {
        qv[c] -= a * v[c] - b * v[H + c];
        qv[H + c] -= a * v[H + c] + b * v[c];
      }
    };
    if (i > 0) nbr(eA[n - d.sx], eB[n - d.sx], n - d.sx);
    if (i < d.nx - 1) nbr(eA[n], eB[n], n + d.sx);
    if (j > 0) nbr(eA[N + n - d.sy], eB[N + n - d.sy], n - d.sy);
    if (j < d.ny - 1) nbr(eA[N + n], eB[N + n], n + d.sy);
    if (k > 0) nbr(eA[2 * N + n - 1], eB[2 * N + n - 1], n - 1);
    if (k < d.nz - 1) nbr(eA[2 * N + n], eB[2 * N + n], n + 1);
    fs::stv<double, K>(q, n, qv);
#pragma unroll
    for (int c = 0; c < H; ++c) {
      acc[c] += pc[c] * qv[c] - pc[H + c] * qv[H + c];
      acc[H + c] += pc[c] * qv[H + c] + pc[H + c] * qv[c];
    }
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(&tickets[kTkApply])) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    if (threadIdx.x < H) {
      AcState& a = st[threadIdx.x];
      const double sr = tot[threadIdx.x], si = tot[H + threadIdx.x];
      a.alpha_re = a.alpha_im = 0.0;
      if (a.active) {
        if (!isfinite(sr) || !isfinite(si)) {
          a.active = 0;
          a.status = FS_NAN;
        } else if (sr == 0.0 && si == 0.0) {
          a.active = 0;  // breakdown of the bilinear form
          a.status = FS_STALLED;
        } else {
          cdiv(a.rho_re, a.rho_im, sr, si, a.alpha_re, a.alpha_im);
        }
      }
    }
  }
}

// x~ += alpha p, r~ -= alpha q, ||r~||^2; the last block counts the
// iteration and retires the right-hand sides that reached the tolerance.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_update(Dims d, const double* __restrict__ p, const double* __restrict__ q,
                double* __restrict__ x, double* __restrict__ r, double* __restrict__ partials,
                AcState* st, unsigned int* tickets) {
  constexpr int H = K / 2;
  __shared__ double al[2 * H];
  if (threadIdx.x < H) {
    al[threadIdx.x] = st[threadIdx.x].alpha_re;
    al[H + threadIdx.x] = st[threadIdx.x].alpha_im;
  }
  __syncthreads();
  double acc[H];
#pragma unroll
  for (int c = 0; c < H; ++c) acc[c] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    double pv[K], qv[K], xv[K], rv[K];
    fs::ldv<double, K>(p, n, pv);
    fs::ldv<double, K>(q, n, qv);
    fs::ldv<double, K>(x, n, xv);
    fs::ldv<double, K>(r, n, rv);
#pragma unroll
    for (int c = 0; c < H; ++c) {
      const double ar = al[c], ai = al[H + c];
      xv[c] += ar * pv[c] - ai * pv[H + c];
      xv[H + c] += ar * pv[H + c] + ai * pv[c];
      rv[c] -= ar * qv[c] - ai * qv[H + c];
      rv[H + c] -= ar * qv[H + c] + ai * qv[c];
      acc[c] += rv[c] * rv[c] + rv[H + c] * rv[H + c];
    }
    fs::stv<double, K>(x, n, xv);
    fs::stv<double, K>(r, n, rv);
  }
  fs::block_partials<H>(acc, partials);
  if (fs::last_block(&tickets[kTkUpdate])) {
    double tot[H];
    fs::grid_total<H>(partials, gridDim.x, tot);
    if (threadIdx.x < H) {
      AcState& a = st[threadIdx.x];
      if (a.active) {
        a.iters += 1;
        a.rr = tot[threadIdx.x];
        if (!isfinite(a.rr)) {
          a.active = 0;
          a.status = FS_NAN;
        } else if (a.rr <= a.tol2 * a.bb) {
          a.active = 0;
          a.status = FS_OK;
        }
      }
    }
  }
}

// rho' = r~^T z (unconjugated), beta = rho' / rho.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_rz(Dims d, const double* __restrict__ r, const double* __restrict__ z,
            double* __restrict__ partials, AcState* st, unsigned int* tickets) {
  constexpr int H = K / 2;
  double acc[K];
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    double rv[K], zv[K];
    fs::ldv<double, K>(r, n, rv);
    fs::ldv<double, K>(z, n, zv);
#pragma unroll
    for (int c = 0; c < H; ++c) {
      acc[c] += rv[c] * zv[c] - rv[H + c] * zv[H + c];
      acc[H + c] += rv[c] * zv[H + c] + rv[H + c] * zv[c];
    }
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(&tickets[kTkRz])) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    if (threadIdx.x < H) {
      AcState& a = st[threadIdx.x];
      const double gr = tot[threadIdx.x], gi = tot[H + threadIdx.x];
      a.beta_re = a.beta_im = 0.0;
      if (a.active) {
        if (!isfinite(gr) || !isfinite(gi)) {
          a.active = 0;
          a.status = FS_NAN;
        } else if (gr == 0.0 && gi == 0.0) {
          a.active = 0;
          a.status = FS_STALLED;
        } else {
          if (!a.fresh) cdiv(gr, gi, a.rho_re, a.rho_im, a.beta_re, a.beta_im);
          a.fresh = 0;
          a.rho_re = gr;
          a.rho_im = gi;
        }
      }
    }
  }
}

// p = z + beta p
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_pnew(Dims d, const double* __restrict__ z, double* __restrict__ p, const AcState* st) {
  constexpr int H = K / 2;
  __shared__ double be[2 * H];
  if (threadIdx.x < H) {
    be[threadIdx.x] = st[threadIdx.x].beta_re;
    be[H + threadIdx.x] = st[threadIdx.x].beta_im;
  }
  __syncthreads();
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    double zv[K], pv[K];
    fs::ldv<double, K>(z, n, zv);
    fs::ldv<double, K>(p, n, pv);
#pragma unroll
    for (int c = 0; c < H; ++c) {
      const double br = be[c], bi = be[H + c];
      const double pr = pv[c], pi = pv[H + c];
      pv[c] = zv[c] + br * pr - bi * pi;
      pv[H + c] = zv[H + c] + br * pi + bi * pr;
    }
    fs::stv<double, K>(p, n, pv);
  }
}

// phi on free nodes = S x~; on solo nodes (every neighbour fixed) the 1x1
// complex solve b / d; pinned nodes 0; fixed nodes keep their values.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_finalize(Dims d, const double* __restrict__ mA, const double* __restrict__ mB,
                  const double* __restrict__ s64, const uint8_t* __restrict__ label,
                  const double* __restrict__ x, double* __restrict__ phi) {
  constexpr int H = K / 2;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    const uint8_t lab = label[n];
    if (lab == FS_LABEL_FIXED) continue;
    double out[K];
    if (lab == FS_LABEL_FREE) {
      fs::ldv<double, K>(x, n, out);
      const double s = s64[n];
#pragma unroll
      for (int c = 0; c < K; ++c) out[c] *= s;
    } else if (lab == FS_LABEL_SOLO) {
      double re[H], im[H], da, db;
      coupled_sum<K>(d, mA, mB, phi, n, [&](long long nb) { return label[nb] == FS_LABEL_FIXED; },
                     re, im, da, db);
#pragma unroll
      for (int c = 0; c < H; ++c) cdiv(re[c], im[c], da, db, out[c], out[H + c]);
    } else {
#pragma unroll
      for (int c = 0; c < K; ++c) out[c] = 0.0;
    }
    fs::stv<double, K>(phi, n, out);
  }
}

// True residual of the final phi on the free nodes, equilibrated like b~:
// r~ = S (b - K phi)|_free = -S (K phi)|_free (K phi = 0 is the equation);
// writes r~ (for a restart) and ||r~||^2 per RHS into st.rr.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_ac_true_res(Dims d, const double* __restrict__ mA, const double* __restrict__ mB,
                  const double* __restrict__ s64, const uint8_t* __restrict__ label,
                  const double* __restrict__ phi, double* __restrict__ r,
                  double* __restrict__ partials, AcState* st, unsigned int* tickets) {
  constexpr int H = K / 2;
  double acc[H];
#pragma unroll
  for (int c = 0; c < H; ++c) acc[c] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    double out[K];
#pragma unroll
    for (int c = 0; c < K; ++c) out[c] = 0.0;
    if (label[n] == FS_LABEL_FREE) {
      double re[H], im[H], da, db;
      coupled_sum<K>(d, mA, mB, phi, n, [](long long) { return true; }, re, im, da, db);
      double v[K];
      fs::ldv<double, K>(phi, n, v);
      const double s = s64[n];
#pragma unroll
      for (int c = 0; c < H; ++c) {
        // (K phi)_n = d phi_n - sum_e m_e phi_nbr; residual = -(K phi)_n
        const double kr = da * v[c] - db * v[H + c] - re[c];
        const double ki = da * v[H + c] + db * v[c] - im[c];
        out[c] = -s * kr;
        out[H + c] = -s * ki;
        acc[c] += out[c] * out[c] + out[H + c] * out[H + c];
      }
    }
    fs::stv<double, K>(r, n, out);
  }
  fs::block_partials<H>(acc, partials);
  if (fs::last_block(&tickets[kTkRes])) {
    double tot[H];
    fs::grid_total<H>(partials, gridDim.x, tot);
    if (threadIdx.x < H) st[threadIdx.x].rr = tot[threadIdx.x];
  }
}

// P = |A| + |B| edge by edge: the real SPD companion whose multigrid plan
// equilibrates and preconditions the complex system.
__global__ void k_ac_companion(const double* __restrict__ mA, const double* __restrict__ mB,
                               double* __restrict__ mP, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    mP[i] = fabs(mA[i]) + fabs(mB[i]);
}

struct AcLayout {
  size_t plan, mP, eA, eB, dA, dB, x, r, z, p, q, partials, st, tickets, total;
};

constexpr int kAcMaxBlocks = 4096;

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

int ac_layout(int nx, int ny, int nz, int K, int precond, AcLayout* L) {
  size_t plan_bytes = 0;
  const int st = fs_pcg_workspace_bytes(nx, ny, nz, K, FS_PRECISION_FP64, precond, &plan_bytes);
  if (st != FS_OK) return st;
  const size_t N = (size_t)nx * ny * nz;
  size_t o = 0;
  auto take = [&](size_t bytes) {
    const size_t at = o;
    o += up256(bytes);
    return at;
  };
  L->plan = take(plan_bytes);
  L->mP = take(3 * N * sizeof(double));
  L->eA = take(3 * N * sizeof(double));
  L->eB = take(3 * N * sizeof(double));
  L->dA = take(N * sizeof(double));
  L->dB = take(N * sizeof(double));
  L->x = take(N * K * sizeof(double));
  L->r = take(N * K * sizeof(double));
  L->z = take(N * K * sizeof(double));
  L->p = take(N * K * sizeof(double));
  L->q = take(N * K * sizeof(double));
  L->partials = take((size_t)kAcMaxBlocks * K * sizeof(double));
  L->st = take(8 * sizeof(AcState));
  L->tickets = take(kTickets * sizeof(unsigned int));
  L->total = o;
  return FS_OK;
}

int grid_for(const void* kernel, long long n) {
  int g = fs_grid_blocks(kernel, n);
  return g > kAcMaxBlocks ? kAcMaxBlocks : g;
}

template <int K>
int ac_run(const Dims& d, fs_pcg_plan* plan, const double* mA, const double* mB,
           const double* s64, const uint8_t* label, double* phi, double tol, int maxiter,
           unsigned char* ws, const AcLayout& L, fs_rhs_stats* stats, int ncplx,
           cudaStream_t s) {
  constexpr int H = K / 2;
  double* eA = (double*)(ws + L.eA);
  double* eB = (double*)(ws + L.eB);
  double* dA = (double*)(ws + L.dA);
  double* dB = (double*)(ws + L.dB);
  double* x = (double*)(ws + L.x);
  double* r = (double*)(ws + L.r);
  double* z = (double*)(ws + L.z);
  double* p = (double*)(ws + L.p);
  double* q = (double*)(ws + L.q);
  double* part = (double*)(ws + L.partials);
  AcState* st = (AcState*)(ws + L.st);
  unsigned int* tk = (unsigned int*)(ws + L.tickets);
  FS_CHECK(cudaMemsetAsync(tk, 0, kTickets * sizeof(unsigned int), s));
  k_ac_setup<<<grid_for((const void*)k_ac_setup, d.N), fs::kBlock, 0, s>>>(d, mA, mB, s64, eA,
                                                                           eB, dA, dB);
  FS_CHECK_LAUNCH("k_ac_setup");
  k_ac_rhs<K><<<grid_for((const void*)k_ac_rhs<K>, d.N), fs::kBlock, 0, s>>>(
      d, mA, mB, s64, label, phi, x, r, part, st, tk);
  FS_CHECK_LAUNCH("k_ac_rhs");
  AcState h[H];
  FS_CHECK(cudaMemcpyAsync(h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
  FS_CHECK(cudaStreamSynchronize(s));
  for (int c = 0; c < H; ++c) h[c].tol2 = tol * tol;
  for (int c = ncplx; c < H; ++c) {  // padding columns: nothing to solve
    h[c].active = 0;
    h[c].status = FS_OK;
  }
  FS_CHECK(cudaMemcpyAsync(st, h, sizeof(h), cudaMemcpyHostToDevice, s));
  const int g_apply = grid_for((const void*)k_ac_apply<K>, d.N);
  const int g_upd = grid_for((const void*)k_ac_update<K>, d.N);
  const int g_rz = grid_for((const void*)k_ac_rz<K>, d.N);
  const int g_pn = grid_for((const void*)k_ac_pnew<K>, d.N);
  const size_t vbytes = (size_t)d.N * K * sizeof(double);
  int total_iters = 0;
  int restarts = 0;
  for (;;) {
    // z = M r, rho = r^T z, p = z (beta = 0 on a fresh start)
    int rc = fs_pcg_plan_precondition(plan, r, z, s);
    if (rc != FS_OK) return rc;
    k_ac_rz<K><<<g_rz, fs::kBlock, 0, s>>>(d, r, z, part, st, tk);
    FS_CHECK(cudaMemcpyAsync(p, z, vbytes, cudaMemcpyDeviceToDevice, s));
    bool any = true;
    while (any && total_iters < maxiter) {
      k_ac_apply<K><<<g_apply, fs::kBlock, 0, s>>>(d, eA, eB, dA, dB, p, q, part, st, tk);
      k_ac_update<K><<<g_upd, fs::kBlock, 0, s>>>(d, p, q, x, r, part, st, tk);
      FS_CHECK_LAUNCH("k_ac_update");
      ++total_iters;
      FS_CHECK(cudaMemcpyAsync(h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
      FS_CHECK(cudaStreamSynchronize(s));
      any = false;
      for (int c = 0; c < H; ++c) any = any || h[c].active;
      if (!any) break;
      rc = fs_pcg_plan_precondition(plan, r, z, s);
      if (rc != FS_OK) return rc;
      k_ac_rz<K><<<g_rz, fs::kBlock, 0, s>>>(d, r, z, part, st, tk);
      k_ac_pnew<K><<<g_pn, fs::kBlock, 0, s>>>(d, z, p, st);
      FS_CHECK_LAUNCH("k_ac_pnew");
    }
    // back to phi, then the true residual
    k_ac_finalize<K><<<grid_for((const void*)k_ac_finalize<K>, d.N), fs::kBlock, 0, s>>>(
        d, mA, mB, s64, label, x, phi);
    k_ac_true_res<K><<<grid_for((const void*)k_ac_true_res<K>, d.N), fs::kBlock, 0, s>>>(
        d, mA, mB, s64, label, phi, r, part, st, tk);
    FS_CHECK_LAUNCH("k_ac_true_res");
    FS_CHECK(cudaMemcpyAsync(h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
    FS_CHECK(cudaStreamSynchronize(s));
    // one restart from the current iterate when the recursive residual ran
    // ahead of the true one (r~ now holds the true residual, x~ the iterate)
    bool redo = false;
    for (int c = 0; c < ncplx; ++c)
      if (h[c].bb > 0.0 && h[c].rr > h[c].tol2 * h[c].bb && h[c].status != FS_NAN)
        redo = true;
    if (!redo || restarts >= 2 || total_iters >= maxiter) break;
    ++restarts;
    for (int c = 0; c < H; ++c) {
      const bool want = c < ncplx && h[c].bb > 0.0 && h[c].rr > h[c].tol2 * h[c].bb;
      h[c].active = want ? 1 : 0;
      h[c].fresh = 1;
      if (want) h[c].status = FS_NOT_CONVERGED;
    }
    FS_CHECK(cudaMemcpyAsync(st, h, sizeof(h), cudaMemcpyHostToDevice, s));
  }
  for (int c = 0; c < ncplx; ++c) {
    fs_rhs_stats& o = stats[c];
    o.iterations = h[c].iters;
    o.bnorm = sqrt(h[c].bb);
    o.relres = h[c].bb > 0.0 ? sqrt(h[c].rr / h[c].bb) : 0.0;
    o.reliable_updates = restarts;
    o.reserved = 0;
    if (h[c].status == FS_NAN || h[c].status == FS_STALLED)
      o.status = h[c].status;
    else
      o.status = (o.relres <= tol || h[c].bb == 0.0) ? FS_OK : FS_NOT_CONVERGED;
  }
  return FS_OK;
}

}  // namespace

extern "C" int fs_ac_workspace_bytes(int nx, int ny, int nz, int ncplx, int precond,
                                     size_t* bytes) {
  if (nx < 2 || ny < 2 || nz < 2 || ncplx < 1 || ncplx > 8 || !bytes) return FS_BAD_ARG;
  if (precond != FS_PRECOND_JACOBI && precond != FS_PRECOND_MG) return FS_BAD_ARG;
  int K = 2;
  while (K < 2 * ncplx) K *= 2;
  AcLayout L;
  const int st = ac_layout(nx, ny, nz, K, precond, &L);
  if (st != FS_OK) return st;
  *bytes = L.total;
  return FS_OK;
}

extern "C" int fs_ac_solve(int nx, int ny, int nz, int ncplx, int precond, const double* mA,
                           const double* mB, const uint8_t* label_in, double* phi, double tol,
                           int maxiter, void* workspace, size_t workspace_bytes,
                           fs_rhs_stats* stats, void* stream) {
  if (nx < 2 || ny < 2 || nz < 2 || ncplx < 1 || ncplx > 8 || !mA || !mB || !label_in ||
      !phi || !workspace || !stats || !(tol > 0.0) || maxiter < 1)
    return FS_BAD_ARG;
  if (precond != FS_PRECOND_JACOBI && precond != FS_PRECOND_MG) return FS_BAD_ARG;
  if ((uintptr_t)workspace & 255) return FS_BAD_ARG;
  int K = 2;
  while (K < 2 * ncplx) K *= 2;
  AcLayout L;
  int st = ac_layout(nx, ny, nz, K, precond, &L);
  if (st != FS_OK) return st;
  if (workspace_bytes < L.total) {
    fs_set_error_msg("fs_ac_solve: workspace too small");
    return FS_BAD_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* ws = (unsigned char*)workspace;
  const Dims d = fs::make_dims(nx, ny, nz);
  double* mP = (double*)(ws + L.mP);
  k_ac_companion<<<grid_for((const void*)k_ac_companion, 3 * d.N), fs::kBlock, 0, s>>>(
      mA, mB, mP, 3 * d.N);
  FS_CHECK_LAUNCH("k_ac_companion");
  size_t plan_bytes = 0;
  st = fs_pcg_workspace_bytes(nx, ny, nz, K, FS_PRECISION_FP64, precond, &plan_bytes);
  if (st != FS_OK) return st;
  fs_pcg_plan* plan = nullptr;
  st = fs_pcg_plan_create(nx, ny, nz, K, FS_PRECISION_FP64, precond, mP, mP + d.N,
                          mP + 2 * d.N, label_in, phi, nullptr, ws + L.plan, plan_bytes, &plan,
                          stream);
  if (st != FS_OK) return st;
  const double* s64 = nullptr;
  const uint8_t* label = nullptr;
  st = fs_pcg_plan_scale(plan, &s64, &label);
  if (st == FS_OK) {
    switch (K) {
      case 2: st = ac_run<2>(d, plan, mA, mB, s64, label, phi, tol, maxiter, ws, L, stats, ncplx, s); break;
      case 4: st = ac_run<4>(d, plan, mA, mB, s64, label, phi, tol, maxiter, ws, L, stats, ncplx, s); break;
      case 8: st = ac_run<8>(d, plan, mA, mB, s64, label, phi, tol, maxiter, ws, L, stats, ncplx, s); break;
      case 16: st = ac_run<16>(d, plan, mA, mB, s64, label, phi, tol, maxiter, ws, L, stats, ncplx, s); break;
      default: st = FS_BAD_ARG;
    }
  }
  const int st2 = fs_pcg_plan_destroy(plan);
  return st != FS_OK ? st : st2;
}
