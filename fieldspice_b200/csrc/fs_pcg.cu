// Matrix-free conjugate gradients on the Dirichlet-eliminated, Jacobi-
// equilibrated system  D^-1/2 A_ff D^-1/2 x~ = D^-1/2 b_f.
//
// This is the system the reference hands to SciPy's CG
// (fieldspice/solvers/poisson.py:364-377 builds S A S with S = diag(A)^-1/2,
// :533-552 runs cg(rtol=tol, atol=0) with a Jacobi preconditioner on it), so
// the stopping rule ||r~|| < tol*||b~|| is the reference's rule.  Here the
// scaled operator is never assembled: the setup pass stores equilibrated
// edge masses  m~_e = m_e * s_head * s_tail  (s = diag^-1/2 on free nodes,
// 0 elsewhere), so an edge that touches a Dirichlet node carries 0 and the
// inner stencil needs neither a mask nor a diagonal:
//     (A~ p)_i = p_i - sum_e m~_e p_nbr(e).
//
// Precision.  The inner CG runs in T (double, or float in mixed mode) with
// FP64 inner products and FP64 alpha/beta.  The solution is kept in FP64 in
// phi; the inner iterate x~ is a correction accumulated since the last
// "reliable update" (Sleijpen & van der Vorst residual replacement).  A
// reliable update folds x~ into phi and recomputes the TRUE residual
// f - L phi with the FP64 masses, so convergence is always decided on an FP64
// residual.  Updates trigger when the iterated residual falls below
// tol*||b~|| (to verify convergence), at the iteration cap, and in mixed mode
// whenever it has dropped by `delta` since the previous update.
//
// Each CG iteration is four kernels captured once in a CUDA graph:
//   K0 p = r + beta p  (and, after a reliable update, phi += s x~, x~ = 0)
//   K1 q = A~ p, partial p.q -> alpha           (stencil, FP64 dot)
//   K2 x~ += alpha p, r -= alpha q, r.r -> beta (FP64 dot)
//   K3 reliable update when flagged (FP64 true residual)
// Scalars live on the device; the host only polls an "all done" flag between
// graph launches.  Reductions are deterministic (fixed-order block partials,
// reduced by the last block to finish).  No kernel waits on another block.
#include <math.h>
#include <string.h>

#include <new>

#include "fs_common.cuh"

using fs::Dims;

namespace {

struct RhsState {
  double gamma;      // r~.r~ of the current residual
  double gamma_old;  // previous gamma
  double pq;
  double alpha, beta;
  double bnorm;      // ||b~||
  double rmax;       // residual norm at the last reliable update
  double relres;     // last FP64 true relative residual
  int iters;
  int active;
  int ru;            // reliable update requested
  int fold;          // x~ must be folded into phi
  int zero;          // b == 0: the solution on free nodes is 0 (SciPy)
  int status;
  int nru;
  int pad;
};

enum { kTicketP = 0, kTicketApply, kTicketUpdate, kTicketRel, kTicketInit,
       kTicketFin, kTickets };

struct Control {
  double tol;
  double delta;
  int maxiter;
  int all_done;
  int any_ru;
  int any_fold;
  unsigned int tickets[kTickets];
  unsigned int pad[2];
};

__device__ void refresh_done(RhsState* st, Control* ctl, int nrhs) {
  // Called by thread 0 of a last block after the per-RHS updates.
  int done = 1, ru = 0;
  for (int t = 0; t < nrhs; ++t) {
    done &= !st[t].active;
    ru |= st[t].ru;
  }
  ctl->all_done = done;
  ctl->any_ru = ru;
}

// ---- setup --------------------------------------------------------------------
__global__ void k_classify(Dims d, const double* __restrict__ mx,
                           const double* __restrict__ my,
                           const double* __restrict__ mz,
                           const uint8_t* __restrict__ label_in,
                           uint8_t* __restrict__ label,
                           double* __restrict__ s64) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    uint8_t lab = label_in[n] == FS_LABEL_FREE ? FS_LABEL_FREE : FS_LABEL_FIXED;
    double s = 0.0;
    if (lab == FS_LABEL_FREE) {
      int i, j, k;
      fs::node_ijk(d, n, i, j, k);
      double dg = 0.0, sfree = 0.0;
      auto edge = [&](bool ok, double m, long long nb) {
        if (!ok) return;
        dg += m;
        if (label_in[nb] == FS_LABEL_FREE) sfree += m;
      };
      edge(i > 0, i > 0 ? mx[n - d.sx] : 0.0, n - d.sx);
      edge(i < d.nx - 1, mx[n], n + d.sx);
      edge(j > 0, j > 0 ? my[n - d.sy] : 0.0, n - d.sy);
      edge(j < d.ny - 1, my[n], n + d.sy);
      edge(k > 0, k > 0 ? mz[n - 1] : 0.0, n - 1);
      edge(k < d.nz - 1, mz[n], n + 1);
      if (dg == 0.0)
        lab = FS_LABEL_PINNED;  // coupled to nothing: pinned to 0
      else if (sfree == 0.0)
        lab = FS_LABEL_SOLO;  // decoupled row: x = b / diag
      else
        s = 1.0 / sqrt(dg);
    }
    label[n] = lab;
    s64[n] = s;
  }
}

template <typename T>
__global__ void k_eq_masses(Dims d, const double* __restrict__ mx,
                            const double* __restrict__ my,
                            const double* __restrict__ mz,
                            const double* __restrict__ s64, T* __restrict__ ex,
                            T* __restrict__ ey, T* __restrict__ ez) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    const double s = s64[n];
    ex[n] = (T)(i < d.nx - 1 ? mx[n] * s * s64[n + d.sx] : 0.0);
    ey[n] = (T)(j < d.ny - 1 ? my[n] * s * s64[n + d.sy] : 0.0);
    ez[n] = (T)(k < d.nz - 1 ? mz[n] * s * s64[n + 1] : 0.0);
  }
}

// ---- per-solve initialisation -------------------------------------------------
// r~ = s (f - L phi0) on free nodes, b~ = s (f - L phi_D) for ||b~||, solo
// and pinned nodes solved directly, inner vectors zeroed everywhere.
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_init(Dims d, const double* __restrict__ mx, const double* __restrict__ my,
           const double* __restrict__ mz, const uint8_t* __restrict__ label,
           const double* __restrict__ s64, double* __restrict__ phi,
           const double* __restrict__ f, int warm, T* __restrict__ x,
           T* __restrict__ r, T* __restrict__ p, double* __restrict__ partials,
           RhsState* st, Control* ctl, double tol, int maxiter, double delta) {
  double acc[2 * K];
#pragma unroll
  for (int t = 0; t < 2 * K; ++t) acc[t] = 0.0;
  T zero[K];
#pragma unroll
  for (int t = 0; t < K; ++t) zero[t] = (T)0;

  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    const uint8_t lab = label[n];
    fs::stv<T, K>(x, n, zero);
    fs::stv<T, K>(p, n, zero);
    if (lab == FS_LABEL_FIXED) {
      fs::stv<T, K>(r, n, zero);
      continue;
    }
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    double res[K], bres[K], c[K];
#pragma unroll
    for (int t = 0; t < K; ++t) {
      res[t] = f ? f[n * K + t] : 0.0;
      bres[t] = res[t];
      c[t] = (lab == FS_LABEL_FREE && warm) ? phi[n * K + t] : 0.0;
    }
    double dg = 0.0;
    auto edge = [&](bool ok, double m, long long nb) {
      if (!ok || m == 0.0) return;
      dg += m;
      const bool nb_free = label[nb] == FS_LABEL_FREE;
#pragma unroll
      for (int t = 0; t < K; ++t) {
        double v = nb_free ? (warm ? phi[nb * K + t] : 0.0) : phi[nb * K + t];
        res[t] -= m * (c[t] - v);
        if (!nb_free) bres[t] += m * v;
      }
    };
    edge(i > 0, i > 0 ? mx[n - d.sx] : 0.0, n - d.sx);
    edge(i < d.nx - 1, mx[n], n + d.sx);
    edge(j > 0, j > 0 ? my[n - d.sy] : 0.0, n - d.sy);
    edge(j < d.ny - 1, my[n], n + d.sy);
    edge(k > 0, k > 0 ? mz[n - 1] : 0.0, n - 1);
    edge(k < d.nz - 1, mz[n], n + 1);

    if (lab == FS_LABEL_FREE) {
      const double s = s64[n];
      T rv[K];
#pragma unroll
      for (int t = 0; t < K; ++t) {
        double rs = res[t] * s, bs = bres[t] * s;
        rv[t] = (T)rs;
        acc[t] += rs * rs;
        acc[K + t] += bs * bs;
        if (!warm) phi[n * K + t] = 0.0;
      }
      fs::stv<T, K>(r, n, rv);
    } else {
      // Solo: every coupled neighbour is fixed, so x = b / diag exactly
      // (poisson.py:559-564).  Pinned: coupled to nothing, x = 0 (:522).
#pragma unroll
      for (int t = 0; t < K; ++t)
        phi[n * K + t] = (lab == FS_LABEL_SOLO) ? bres[t] / dg : 0.0;
      fs::stv<T, K>(r, n, zero);
    }
  }
  fs::block_partials<2 * K>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketInit])) {
    double tot[2 * K];
    fs::grid_total<2 * K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
      RhsState& s = st[threadIdx.x];
      const double g = tot[threadIdx.x];
      const double bn = sqrt(tot[K + threadIdx.x]);
      s.gamma = g;
      s.gamma_old = g;
      s.pq = 0.0;
      s.alpha = 0.0;
      s.beta = 0.0;
      s.bnorm = bn;
      s.rmax = sqrt(g);
      s.iters = 0;
      s.ru = 0;
      s.fold = 0;
      s.nru = 0;
      s.zero = 0;
      s.status = FS_OK;
      s.relres = bn > 0.0 ? sqrt(g) / bn : 0.0;
      if (!isfinite(g) || !isfinite(bn)) {
        s.active = 0;
        s.status = FS_NAN;
      } else if (bn == 0.0) {
        s.active = 0;  // SciPy returns x = b = 0 for a zero right-hand side
        s.zero = 1;
      } else {
        s.active = sqrt(g) < tol * bn ? 0 : 1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      ctl->tol = tol;
      ctl->maxiter = maxiter;
      ctl->delta = delta;
      ctl->any_fold = 0;
      refresh_done(st, ctl, K);
    }
  }
}

// ---- K0: fold pending corrections, p = r + beta p -----------------------------
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_pupdate(Dims d, const double* __restrict__ s64, double* __restrict__ phi,
              T* __restrict__ x, const T* __restrict__ r, T* __restrict__ p,
              RhsState* st, Control* ctl) {
  __shared__ T beta[K];
  __shared__ int fold[K], act[K];
  __shared__ int any_fold, done;
  if (threadIdx.x == 0) {
    any_fold = ctl->any_fold;
    done = ctl->all_done;
  }
  if (threadIdx.x < K) {
    beta[threadIdx.x] = (T)st[threadIdx.x].beta;
    fold[threadIdx.x] = st[threadIdx.x].fold;
    act[threadIdx.x] = st[threadIdx.x].active;
  }
  __syncthreads();
  if (done && !any_fold) return;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    if (any_fold) {
      const double s = s64[n];
      if (s != 0.0) {
        T xv[K];
        fs::ldv<T, K>(x, n, xv);
        bool touched = false;
#pragma unroll
        for (int t = 0; t < K; ++t)
          if (fold[t]) {
            phi[n * K + t] += (double)xv[t] * s;
            xv[t] = (T)0;
            touched = true;
          }
        if (touched) fs::stv<T, K>(x, n, xv);
      }
    }
    if (!done) {
      T rv[K], pv[K];
      fs::ldv<T, K>(r, n, rv);
      fs::ldv<T, K>(p, n, pv);
#pragma unroll
      for (int t = 0; t < K; ++t)
        if (act[t]) pv[t] = rv[t] + beta[t] * pv[t];
      fs::stv<T, K>(p, n, pv);
    }
  }
  if (any_fold && fs::last_block(&ctl->tickets[kTicketP])) {
    if (threadIdx.x < K) st[threadIdx.x].fold = 0;
    if (threadIdx.x == 0) ctl->any_fold = 0;
  }
}

// ---- K1: q = A~ p and p.q -------------------------------------------------------
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_apply_pq(Dims d, const T* __restrict__ ex, const T* __restrict__ ey,
               const T* __restrict__ ez, const T* __restrict__ p,
               T* __restrict__ q, double* __restrict__ partials, RhsState* st,
               Control* ctl) {
  if (ctl->all_done) return;
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    T pc[K], qv[K];
    fs::ldv_ro<T, K>(p, n, pc);
#pragma unroll
    for (int t = 0; t < K; ++t) qv[t] = pc[t];
    auto nbr = [&](T m, long long nb) {
      T pn[K];
      fs::ldv_ro<T, K>(p, nb, pn);
#pragma unroll
      for (int t = 0; t < K; ++t) qv[t] -= m * pn[t];
    };
    if (i > 0) nbr(__ldg(ex + n - d.sx), n - d.sx);
    if (i < d.nx - 1) nbr(__ldg(ex + n), n + d.sx);
    if (j > 0) nbr(__ldg(ey + n - d.sy), n - d.sy);
    if (j < d.ny - 1) nbr(__ldg(ey + n), n + d.sy);
    if (k > 0) nbr(__ldg(ez + n - 1), n - 1);
    if (k < d.nz - 1) nbr(__ldg(ez + n), n + 1);
    fs::stv<T, K>(q, n, qv);
#pragma unroll
    for (int t = 0; t < K; ++t) acc[t] += (double)pc[t] * (double)qv[t];
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketApply])) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
      RhsState& s = st[threadIdx.x];
      s.pq = tot[threadIdx.x];
      if (s.active) {
        if (tot[threadIdx.x] > 0.0 && isfinite(tot[threadIdx.x])) {
          s.alpha = s.gamma / tot[threadIdx.x];
        } else {
          s.alpha = 0.0;  // breakdown: A~ is SPD, so p.q <= 0 means NaN/Inf
          s.active = 0;
          s.status = FS_NAN;
        }
      } else {
        s.alpha = 0.0;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) refresh_done(st, ctl, K);
  }
}

// ---- K2: x~ += alpha p, r~ -= alpha q, r~.r~ ------------------------------------
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_update(Dims d, const T* __restrict__ p, const T* __restrict__ q,
             T* __restrict__ x, T* __restrict__ r, double* __restrict__ partials,
             RhsState* st, Control* ctl) {
  if (ctl->all_done) return;
  __shared__ T alpha[K];
  if (threadIdx.x < K) alpha[threadIdx.x] = (T)st[threadIdx.x].alpha;
  __syncthreads();
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T pv[K], qv[K], xv[K], rv[K];
    fs::ldv_ro<T, K>(p, n, pv);
    fs::ldv_ro<T, K>(q, n, qv);
    fs::ldv<T, K>(x, n, xv);
    fs::ldv<T, K>(r, n, rv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      xv[t] += alpha[t] * pv[t];
      rv[t] -= alpha[t] * qv[t];
      acc[t] += (double)rv[t] * (double)rv[t];
    }
    fs::stv<T, K>(x, n, xv);
    fs::stv<T, K>(r, n, rv);
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketUpdate])) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
      RhsState& s = st[threadIdx.x];
      if (s.active) {
        const double g = tot[threadIdx.x];
        s.iters += 1;
        if (!isfinite(g)) {
          s.active = 0;
          s.status = FS_NAN;
        } else {
          s.gamma_old = s.gamma;
          s.gamma = g;
          s.beta = g / s.gamma_old;
          const double rn = sqrt(g);
          if (rn < ctl->tol * s.bnorm || s.iters >= ctl->maxiter ||
              (ctl->delta > 0.0 && rn < ctl->delta * s.rmax))
            s.ru = 1;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) refresh_done(st, ctl, K);
  }
}

// ---- K3: reliable update: true FP64 residual of phi + s x~ -----------------------
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_reliable(Dims d, const double* __restrict__ mx,
               const double* __restrict__ my, const double* __restrict__ mz,
               const uint8_t* __restrict__ label,
               const double* __restrict__ s64, const double* __restrict__ phi,
               const double* __restrict__ f, const T* __restrict__ x,
               T* __restrict__ r, double* __restrict__ partials, RhsState* st,
               Control* ctl) {
  if (!ctl->any_ru) return;
  __shared__ int ru[K];
  if (threadIdx.x < K) ru[threadIdx.x] = st[threadIdx.x].ru;
  __syncthreads();
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    if (label[n] != FS_LABEL_FREE) continue;
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    const double sc = s64[n];
    double c[K], res[K];
    {
      T xv[K];
      fs::ldv_ro<T, K>(x, n, xv);
#pragma unroll
      for (int t = 0; t < K; ++t) {
        c[t] = phi[n * K + t] + (double)xv[t] * sc;
        res[t] = f ? f[n * K + t] : 0.0;
      }
    }
    auto edge = [&](bool ok, double m, long long nb) {
      if (!ok || m == 0.0) return;
      const double snb = s64[nb];
      T xv[K];
      fs::ldv_ro<T, K>(x, nb, xv);
#pragma unroll
      for (int t = 0; t < K; ++t)
        res[t] -= m * (c[t] - (phi[nb * K + t] + (double)xv[t] * snb));
    };
    edge(i > 0, i > 0 ? mx[n - d.sx] : 0.0, n - d.sx);
    edge(i < d.nx - 1, mx[n], n + d.sx);
    edge(j > 0, j > 0 ? my[n - d.sy] : 0.0, n - d.sy);
    edge(j < d.ny - 1, my[n], n + d.sy);
    edge(k > 0, k > 0 ? mz[n - 1] : 0.0, n - 1);
    edge(k < d.nz - 1, mz[n], n + 1);
    T rv[K];
    fs::ldv<T, K>(r, n, rv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      if (ru[t]) {
        const double rs = res[t] * sc;
        rv[t] = (T)rs;
        acc[t] += rs * rs;
      }
    }
    fs::stv<T, K>(r, n, rv);
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketRel])) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
      RhsState& s = st[threadIdx.x];
      if (s.ru) {
        const double g = tot[threadIdx.x];
        const double rn = sqrt(g);
        s.nru += 1;
        s.fold = 1;
        s.ru = 0;
        s.relres = rn / s.bnorm;
        if (!isfinite(g)) {
          s.active = 0;
          s.status = FS_NAN;
        } else if (rn < ctl->tol * s.bnorm) {
          s.active = 0;
          s.status = FS_OK;
        } else if (s.iters >= ctl->maxiter) {
          s.active = 0;
          s.status = FS_NOT_CONVERGED;
        } else {
          s.gamma = g;
          s.beta = g / s.gamma_old;
          s.rmax = rn;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      ctl->any_fold = 1;
      refresh_done(st, ctl, K);
    }
  }
}

// ---- after the loop: fold what is pending, zero RHS with b == 0 ------------------
template <typename T, int K>
__global__ void k_finalize(Dims d, const uint8_t* __restrict__ label,
                           const double* __restrict__ s64,
                           double* __restrict__ phi, T* __restrict__ x,
                           RhsState* st, Control* ctl) {
  __shared__ int fold[K], zero[K];
  if (threadIdx.x < K) {
    fold[threadIdx.x] = st[threadIdx.x].fold;
    zero[threadIdx.x] = st[threadIdx.x].zero;
  }
  __syncthreads();
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    if (label[n] != FS_LABEL_FREE) continue;
    const double s = s64[n];
    T xv[K];
    fs::ldv<T, K>(x, n, xv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      if (fold[t]) {
        phi[n * K + t] += (double)xv[t] * s;
        xv[t] = (T)0;
      }
      if (zero[t]) phi[n * K + t] = 0.0;
    }
    fs::stv<T, K>(x, n, xv);
  }
  if (fs::last_block(&ctl->tickets[kTicketFin])) {
    if (threadIdx.x < K) {
      st[threadIdx.x].fold = 0;
      st[threadIdx.x].zero = 0;
    }
    if (threadIdx.x == 0) ctl->any_fold = 0;
  }
}

size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

struct Layout {
  size_t label, s64, ex, ey, ez, x, r, p, q, partials, st, ctl, total;
};

constexpr int kMaxBlocks = 4096;

Layout make_layout(const Dims& d, int nrhs, int precision) {
  const size_t tb = precision == FS_PRECISION_MIXED ? 4 : 8;
  const size_t N = (size_t)d.N;
  Layout L;
  size_t o = 0;
  L.label = o; o = align_up(o + N);
  L.s64 = o; o = align_up(o + N * 8);
  L.ex = o; o = align_up(o + N * tb);
  L.ey = o; o = align_up(o + N * tb);
  L.ez = o; o = align_up(o + N * tb);
  L.x = o; o = align_up(o + N * nrhs * tb);
  L.r = o; o = align_up(o + N * nrhs * tb);
  L.p = o; o = align_up(o + N * nrhs * tb);
  L.q = o; o = align_up(o + N * nrhs * tb);
  L.partials = o; o = align_up(o + (size_t)kMaxBlocks * 2 * fs::kMaxRhs * 8);
  L.st = o; o = align_up(o + sizeof(RhsState) * fs::kMaxRhs);
  L.ctl = o; o = align_up(o + sizeof(Control));
  L.total = o;
  return L;
}

bool valid_nrhs(int k) { return k == 1 || k == 2 || k == 4 || k == 8 || k == 16; }

}  // namespace

struct fs_pcg_plan {
  Dims d;
  int nrhs, precision;
  const double *mx, *my, *mz;
  double* phi;
  const double* f;
  uint8_t* label;
  double* s64;
  void *ex, *ey, *ez, *x, *r, *p, *q;
  double* partials;
  RhsState* st;
  Control* ctl;
  int g_init, g_p, g_apply, g_update, g_rel, g_fin;
  int chunk;
  cudaGraphExec_t exec;
  cudaStream_t cap;
  int* h_flag;
  RhsState* h_st;
  long long launches;
  // Event samples around K0, K1, K2 of the first iteration of every graph
  // launch: live per-kernel durations for the roofline figures.
  cudaEvent_t ev[4];
  double kernel_ms[3];
  long long kernel_samples;
};

namespace {

template <typename T, int K>
struct Impl {
  static void grids(fs_pcg_plan* P) {
    const long long N = P->d.N;
    P->g_init = fs_grid_blocks((const void*)k_init<T, K>, N);
    P->g_p = fs_grid_blocks((const void*)k_pupdate<T, K>, N);
    P->g_apply = fs_grid_blocks((const void*)k_apply_pq<T, K>, N);
    P->g_update = fs_grid_blocks((const void*)k_update<T, K>, N);
    P->g_rel = fs_grid_blocks((const void*)k_reliable<T, K>, N);
    P->g_fin = fs_grid_blocks((const void*)k_finalize<T, K>, N);
  }
  static void setup_masses(fs_pcg_plan* P, cudaStream_t s) {
    int g = fs_grid_blocks((const void*)k_eq_masses<T>, P->d.N);
    k_eq_masses<T><<<g, fs::kBlock, 0, s>>>(P->d, P->mx, P->my, P->mz, P->s64,
                                            (T*)P->ex, (T*)P->ey, (T*)P->ez);
  }
  static void init(fs_pcg_plan* P, int warm, double tol, int maxiter,
                   double delta, cudaStream_t s) {
    k_init<T, K><<<P->g_init, fs::kBlock, 0, s>>>(
        P->d, P->mx, P->my, P->mz, P->label, P->s64, P->phi, P->f, warm,
        (T*)P->x, (T*)P->r, (T*)P->p, P->partials, P->st, P->ctl, tol, maxiter,
        delta);
  }
  static void iteration(fs_pcg_plan* P, cudaStream_t s) {
    for (int w = 0; w < 4; ++w) kernel(P, w, s);
  }
  static void kernel(fs_pcg_plan* P, int which, cudaStream_t s) {
    switch (which) {
      case 0:
        k_pupdate<T, K><<<P->g_p, fs::kBlock, 0, s>>>(
            P->d, P->s64, P->phi, (T*)P->x, (const T*)P->r, (T*)P->p, P->st,
            P->ctl);
        break;
      case 1:
        k_apply_pq<T, K><<<P->g_apply, fs::kBlock, 0, s>>>(
            P->d, (const T*)P->ex, (const T*)P->ey, (const T*)P->ez,
            (const T*)P->p, (T*)P->q, P->partials, P->st, P->ctl);
        break;
      case 2:
        k_update<T, K><<<P->g_update, fs::kBlock, 0, s>>>(
            P->d, (const T*)P->p, (const T*)P->q, (T*)P->x, (T*)P->r,
            P->partials, P->st, P->ctl);
        break;
      default:
        k_reliable<T, K><<<P->g_rel, fs::kBlock, 0, s>>>(
            P->d, P->mx, P->my, P->mz, P->label, P->s64, P->phi, P->f,
            (const T*)P->x, (T*)P->r, P->partials, P->st, P->ctl);
        break;
    }
  }
  static void finalize(fs_pcg_plan* P, cudaStream_t s) {
    k_finalize<T, K><<<P->g_fin, fs::kBlock, 0, s>>>(P->d, P->label, P->s64,
                                                     P->phi, (T*)P->x, P->st,
                                                     P->ctl);
  }
};

template <typename T>
bool dispatch_k(int k, fs_pcg_plan* P, int op, cudaStream_t s, int warm = 0,
                double tol = 0, int maxiter = 0, double delta = 0) {
#define FS_OP(KK)                                                   \
  case KK:                                                          \
    if (op == 0) Impl<T, KK>::grids(P);                             \
    if (op == 1) Impl<T, KK>::setup_masses(P, s);                   \
    if (op == 2) Impl<T, KK>::init(P, warm, tol, maxiter, delta, s); \
    if (op == 3) Impl<T, KK>::iteration(P, s);                      \
    if (op == 4) Impl<T, KK>::finalize(P, s);                       \
    if (op >= 5 && op <= 8) Impl<T, KK>::kernel(P, op - 5, s);      \
    return true;
  switch (k) {
    FS_OP(1)
    FS_OP(2)
    FS_OP(4)
    FS_OP(8)
    FS_OP(16)
    default: return false;
  }
#undef FS_OP
}

bool dispatch(fs_pcg_plan* P, int op, cudaStream_t s, int warm = 0,
              double tol = 0, int maxiter = 0, double delta = 0) {
  if (P->precision == FS_PRECISION_MIXED)
    return dispatch_k<float>(P->nrhs, P, op, s, warm, tol, maxiter, delta);
  return dispatch_k<double>(P->nrhs, P, op, s, warm, tol, maxiter, delta);
}

// One CG iteration with event records between its kernels (captured into
// the graph as event nodes).
// A plain cudaEventRecord inside a capture only orders streams; the
// External flag makes it an event-record node that executes with the graph.
void dispatch_first(fs_pcg_plan* P, cudaStream_t s) {
  cudaEventRecordWithFlags(P->ev[0], s, cudaEventRecordExternal);
  dispatch(P, 5, s);  // K0
  cudaEventRecordWithFlags(P->ev[1], s, cudaEventRecordExternal);
  dispatch(P, 6, s);  // K1
  cudaEventRecordWithFlags(P->ev[2], s, cudaEventRecordExternal);
  dispatch(P, 7, s);  // K2
  cudaEventRecordWithFlags(P->ev[3], s, cudaEventRecordExternal);
  dispatch(P, 8, s);  // K3
}

}  // namespace

extern "C" {

int fs_pcg_workspace_bytes(int nx, int ny, int nz, int nrhs, int precision,
                           size_t* bytes) {
  if (nx < 2 || ny < 2 || nz < 2 || !valid_nrhs(nrhs) || !bytes) return FS_BAD_ARG;
  if (precision != FS_PRECISION_FP64 && precision != FS_PRECISION_MIXED)
    return FS_BAD_ARG;
  *bytes = make_layout(fs::make_dims(nx, ny, nz), nrhs, precision).total;
  return FS_OK;
}

int fs_pcg_plan_create(int nx, int ny, int nz, int nrhs, int precision,
                       const double* mx, const double* my, const double* mz,
                       const uint8_t* label_in, double* phi, const double* f,
                       void* workspace, size_t workspace_bytes,
                       fs_pcg_plan** plan, void* stream) {
  if (!plan) return FS_BAD_ARG;
  *plan = nullptr;
  size_t need = 0;
  int st = fs_pcg_workspace_bytes(nx, ny, nz, nrhs, precision, &need);
  if (st != FS_OK) return st;
  if (!mx || !my || !mz || !label_in || !phi || !workspace ||
      workspace_bytes < need)
    return FS_BAD_ARG;
  if (((uintptr_t)workspace & 255) != 0 || ((uintptr_t)phi & 15) != 0 ||
      ((uintptr_t)f & 15) != 0)
    return FS_BAD_ARG;
  fs_pcg_plan* P = new (std::nothrow) fs_pcg_plan();
  if (!P) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  P->d = fs::make_dims(nx, ny, nz);
  P->nrhs = nrhs;
  P->precision = precision;
  P->mx = mx;
  P->my = my;
  P->mz = mz;
  P->phi = phi;
  P->f = f;
  Layout L = make_layout(P->d, nrhs, precision);
  char* w = (char*)workspace;
  P->label = (uint8_t*)(w + L.label);
  P->s64 = (double*)(w + L.s64);
  P->ex = w + L.ex;
  P->ey = w + L.ey;
  P->ez = w + L.ez;
  P->x = w + L.x;
  P->r = w + L.r;
  P->p = w + L.p;
  P->q = w + L.q;
  P->partials = (double*)(w + L.partials);
  P->st = (RhsState*)(w + L.st);
  P->ctl = (Control*)(w + L.ctl);
  P->exec = nullptr;
  P->cap = nullptr;
  P->h_flag = nullptr;
  P->h_st = nullptr;
  P->launches = 0;
  dispatch(P, 0, s);
  const int gmax = P->g_init > P->g_apply ? P->g_init : P->g_apply;
  if (gmax > kMaxBlocks || P->g_p > kMaxBlocks || P->g_update > kMaxBlocks ||
      P->g_rel > kMaxBlocks || P->g_fin > kMaxBlocks) {
    delete P;
    return FS_BAD_ARG;
  }
  for (int t = 0; t < 4; ++t) P->ev[t] = nullptr;
  P->kernel_ms[0] = P->kernel_ms[1] = P->kernel_ms[2] = 0.0;
  P->kernel_samples = 0;
  auto fail = [&](const char* where, cudaError_t e) {
    fs_pcg_plan_destroy(P);
    return fs_cuda_status(where, e);
  };
  cudaError_t e;
  if ((e = cudaMemsetAsync(w + L.st, 0, L.total - L.st, s)) != cudaSuccess)
    return fail("memset state", e);
  int g = fs_grid_blocks((const void*)k_classify, P->d.N);
  k_classify<<<g, fs::kBlock, 0, s>>>(P->d, mx, my, mz, label_in, P->label,
                                      P->s64);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail("k_classify", e);
  dispatch(P, 1, s);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail("k_eq_masses", e);
  if ((e = cudaMallocHost((void**)&P->h_flag, sizeof(int))) != cudaSuccess)
    return fail("cudaMallocHost", e);
  if ((e = cudaMallocHost((void**)&P->h_st, sizeof(RhsState) * fs::kMaxRhs)) !=
      cudaSuccess)
    return fail("cudaMallocHost", e);

  // Capture `chunk` CG iterations once; the graph is replayed until the
  // device reports that every RHS has finished.
  P->chunk = 16;
  if ((e = cudaStreamCreateWithFlags(&P->cap, cudaStreamNonBlocking)) !=
      cudaSuccess)
    return fail("cudaStreamCreate", e);
  for (int t = 0; t < 4; ++t)
    if ((e = cudaEventCreate(&P->ev[t])) != cudaSuccess)
      return fail("cudaEventCreate", e);
  cudaGraph_t graph = nullptr;
  if ((e = cudaStreamBeginCapture(P->cap, cudaStreamCaptureModeThreadLocal)) !=
      cudaSuccess)
    return fail("cudaStreamBeginCapture", e);
  for (int it = 0; it < P->chunk; ++it) {
    if (it == 0) {
      dispatch_first(P, P->cap);
    } else {
      dispatch(P, 3, P->cap);
    }
  }
  e = cudaStreamEndCapture(P->cap, &graph);
  if (e != cudaSuccess) return fail("cudaStreamEndCapture", e);
  e = cudaGraphInstantiate(&P->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail("cudaGraphInstantiate", e);
  *plan = P;
  return FS_OK;
}

int fs_pcg_plan_solve(fs_pcg_plan* P, int warm_start, double tol, int maxiter,
                      fs_rhs_stats* stats, void* stream) {
  if (!P || !(tol > 0.0) || maxiter < 1) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const double delta = P->precision == FS_PRECISION_MIXED ? 0.1 : 0.0;
  cudaError_t e;
  dispatch(P, 2, s, warm_start ? 1 : 0, tol, maxiter, delta);
  FS_CHECK_LAUNCH("k_init");
  long long launches = 1;
  P->kernel_ms[0] = P->kernel_ms[1] = P->kernel_ms[2] = 0.0;
  P->kernel_samples = 0;
  const long long max_chunks = (long long)maxiter / P->chunk + 4;
  int timed_out = 1;
  for (long long c = 0; c < max_chunks; ++c) {
    if ((e = cudaGraphLaunch(P->exec, s)) != cudaSuccess)
      return fs_cuda_status("cudaGraphLaunch", e);
    launches += 4LL * P->chunk;
    if ((e = cudaMemcpyAsync(P->h_flag, &P->ctl->all_done, sizeof(int),
                             cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return fs_cuda_status("cudaMemcpyAsync", e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
      return fs_cuda_status("cudaStreamSynchronize", e);
    float ms[3];
    if (cudaEventElapsedTime(&ms[0], P->ev[0], P->ev[1]) == cudaSuccess &&
        cudaEventElapsedTime(&ms[1], P->ev[1], P->ev[2]) == cudaSuccess &&
        cudaEventElapsedTime(&ms[2], P->ev[2], P->ev[3]) == cudaSuccess) {
      for (int t = 0; t < 3; ++t) P->kernel_ms[t] += ms[t];
      P->kernel_samples += 1;
    } else {
      (void)cudaGetLastError();  // timing unavailable: not a solve failure
    }
    if (*P->h_flag) {
      timed_out = 0;
      break;
    }
  }
  dispatch(P, 4, s);
  FS_CHECK_LAUNCH("k_finalize");
  launches += 1;
  if ((e = cudaMemcpyAsync(P->h_st, P->st, sizeof(RhsState) * P->nrhs,
                           cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fs_cuda_status("cudaMemcpyAsync", e);
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fs_cuda_status("cudaStreamSynchronize", e);
  P->launches = launches;
  int worst = FS_OK;
  for (int t = 0; t < P->nrhs; ++t) {
    const RhsState& h = P->h_st[t];
    if (stats) {
      stats[t].iterations = h.iters;
      stats[t].status = h.status;
      stats[t].relres = h.relres;
      stats[t].bnorm = h.bnorm;
      stats[t].reliable_updates = h.nru;
      stats[t].reserved = 0;
    }
    if (h.status == FS_NAN) worst = FS_NAN;
    else if (h.status == FS_NOT_CONVERGED && worst == FS_OK) worst = FS_NOT_CONVERGED;
  }
  if (timed_out) return FS_TIMEOUT;
  return worst;
}

const uint8_t* fs_pcg_plan_labels(const fs_pcg_plan* P) {
  return P ? P->label : nullptr;
}

long long fs_pcg_plan_launches(const fs_pcg_plan* P) {
  return P ? P->launches : 0;
}

int fs_pcg_plan_kernel_times(const fs_pcg_plan* P, double* ms,
                             long long* samples) {
  if (!P || !ms || !samples) return FS_BAD_ARG;
  for (int t = 0; t < 3; ++t) ms[t] = P->kernel_ms[t];
  *samples = P->kernel_samples;
  return FS_OK;
}

int fs_pcg_plan_destroy(fs_pcg_plan* P) {
  if (!P) return FS_OK;
  for (int t = 0; t < 4; ++t)
    if (P->ev[t]) cudaEventDestroy(P->ev[t]);
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->cap) cudaStreamDestroy(P->cap);
  if (P->h_flag) cudaFreeHost(P->h_flag);
  if (P->h_st) cudaFreeHost(P->h_st);
  delete P;
  return FS_OK;
}

}  // extern "C"
