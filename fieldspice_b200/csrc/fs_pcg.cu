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
// whenever it has dropped by a factor `delta` since the previous update (and
// every kRefreshEvery iterations, which also feeds the stall detector).
//
// Each CG iteration is four kernels captured once in a CUDA graph:
//   K0 p = r + beta p_old                          (streaming, p double-buffered)
//   K1 q = A~ p, p.q -> alpha                      (TMA-staged stencil, FP64 dot)
//   K2 (phi += s x~, x~ = 0 after a reliable update) x~ += alpha p,
//      r -= alpha q, r.r -> beta                    (FP64 dot)
//   K3 reliable update when flagged (FP64 true residual)
// Scalars live on the device; the host only polls an "all done" flag between
// graph launches.  Reductions are deterministic (fixed-order block partials,
// reduced by the last block to finish).  No kernel waits on another block.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "fs_common.cuh"
#include "fs_tma.cuh"
#include "fs_mg.cuh"
#include "fs_net.cuh"

#include <cudaTypedefs.h>

using fs::Dims;

namespace {

struct RhsState {
  double rr;         // r~.r~ of the current residual (convergence test)
  double gamma;      // r~.z of the current residual (= rr without precond)
  double gamma_old;  // previous gamma
  double pq;
  double alpha, beta;
  double bnorm;      // ||b~||
  double rmax;       // residual norm at the last reliable update
  double relres;     // last FP64 true relative residual
  int iters;
  int active;
  int ru;            // reliable update requested
  int zero;          // b == 0: the solution on free nodes is 0 (SciPy)
  int status;
  int nru;
  int nstall;        // reliable updates since the true residual last halved
  int fresh;         // preconditioned: next r.z starts the recurrence (beta 0)
  int cand;          // iteration at which a deferred convergence check was asked
  double best;       // best true residual norm so far
};

constexpr int kStallUpdates = 6;
constexpr int kRefreshEvery = 64;
constexpr int kConvWait = 3;  // iterations a deferred convergence check may wait

enum { kTicketApply = 0, kTicketUpdate, kTicketRel, kTicketInit,
       kTicketFin, kTicketRz, kTickets };

struct Control {
  double tol;
  double delta;
  int maxiter;
  int all_done;
  int any_ru;
  int error;    // a bounded wait expired (TMA stage never landed)
  int precond;  // 0: CG on A~ (Jacobi), 1: multigrid-preconditioned CG
  int flexible; // 1: nonlinear preconditioner (flexible CG): restart at updates
  unsigned int tickets[kTickets];
  unsigned int pad[2];
  unsigned long long label_counts[4];  // free, fixed, solo, pinned nodes (level 0)
};

__device__ void refresh_done(RhsState* st, Control* ctl, int nrhs) {
  // Called by thread 0 of a last block after the per-RHS updates.  A
  // reliable update streams every RHS column anyway (the vectors are
  // interleaved), so when one RHS asks for it every active RHS takes it:
  // the RHS stay in step and the update passes happen once, not once per
  // RHS at scattered iterations.  A mixed-precision RHS whose recursive
  // residual reached the tolerance (ru = 3) keeps iterating with the others
  // (free: the block streams every column anyway) until every active RHS has
  // got there, another RHS asks, or it has waited kConvWait iterations; then
  // one FP64 check serves them all instead of one per convergence iteration.
  int done = 1, ask = 0, cand_all = 1, any = 0, waited = 0;
  for (int t = 0; t < nrhs; ++t) {
    done &= !st[t].active;
    if (!st[t].active) continue;
    any = 1;
    ask |= st[t].ru == 1;
    cand_all &= st[t].ru == 3;
    waited |= st[t].ru == 3 && st[t].iters - st[t].cand >= kConvWait;
  }
  const int ru = ask || (any && cand_all) || waited;
  if (ru)
    for (int t = 0; t < nrhs; ++t)
      if (st[t].active && !st[t].ru) st[t].ru = 2;  // 2: taken along, not asked
  ctl->all_done = done;
  ctl->any_ru = ru;
}

// ---- setup --------------------------------------------------------------------
__global__ void k_classify(Dims d, const double* __restrict__ mx,
                           const double* __restrict__ my,
                           const double* __restrict__ mz,
                           const double* __restrict__ dgn,
                           const uint8_t* __restrict__ label_in,
                           uint8_t* __restrict__ label,
                           double* __restrict__ s64,
                           unsigned long long* __restrict__ counts) {
  __shared__ unsigned int cnt[4];
  if (threadIdx.x < 4) cnt[threadIdx.x] = 0u;
  __syncthreads();
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    uint8_t lab = label_in[n] == FS_LABEL_FREE ? FS_LABEL_FREE : FS_LABEL_FIXED;
    double s = 0.0;
    if (lab == FS_LABEL_FREE) {
      int i, j, k;
      fs::node_ijk(d, n, i, j, k);
      // diagonal = sum of incident masses + the node's own term (heat
      // capacity / dt, convection), if any
      double dg = dgn ? dgn[n] : 0.0, sfree = 0.0;
      auto edge = [&](bool ok, double m, long long nb) {
        if (!ok) return;
        dg += m;
        if (label_in[nb] == FS_LABEL_FREE) sfree += m;
      };
      edge6(d, mx, my, mz, n, i, j, k, edge);
      if (dg == 0.0)
        lab = FS_LABEL_PINNED;  // coupled to nothing: pinned to 0
      else if (sfree == 0.0)
        lab = FS_LABEL_SOLO;  // decoupled row: x = b / diag
      else
        s = 1.0 / sqrt(dg);
    }
    label[n] = lab;
    s64[n] = s;
    if (counts) atomicAdd(&cnt[lab], 1u);
  }
  if (counts) {  // per-block counts, one global add per label
    __syncthreads();
    if (threadIdx.x < 4 && cnt[threadIdx.x])
      atomicAdd(&counts[threadIdx.x], (unsigned long long)cnt[threadIdx.x]);
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
    // the +x/+y/+z edge of the node; on a periodic axis the last plane's edge
    // is the wrap edge to the first plane
    const bool px = d.per & 1, py = (d.per >> 1) & 1, pz = (d.per >> 2) & 1;
    ex[n] = (T)(i < d.nx - 1 ? mx[n] * s * s64[n + d.sx] : (px ? mx[n] * s * s64[n - d.wx] : 0.0));
    ey[n] = (T)(j < d.ny - 1 ? my[n] * s * s64[n + d.sy] : (py ? my[n] * s * s64[n - d.wy] : 0.0));
    ez[n] = (T)(k < d.nz - 1 ? mz[n] * s * s64[n + 1] : (pz ? mz[n] * s * s64[n - d.wz] : 0.0));
  }
}

// ---- per-solve initialisation -------------------------------------------------
// r~ = s (f - L phi0) on free nodes, b~ = s (f - L phi_D) for ||b~||, solo
// and pinned nodes solved directly, inner vectors zeroed everywhere.
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_init(Dims d, const double* __restrict__ mx, const double* __restrict__ my,
           const double* __restrict__ mz, const double* __restrict__ dgn,
           const uint8_t* __restrict__ label,
           const double* __restrict__ s64, double* __restrict__ phi,
           const double* __restrict__ f, int warm, T* __restrict__ x,
           T* __restrict__ r, T* __restrict__ p, double* __restrict__ partials,
           RhsState* st, Control* ctl, double tol, int maxiter, double delta,
           int precond) {
  double acc[2 * K];
#pragma unroll
  for (int t = 0; t < 2 * K; ++t) acc[t] = 0.0;
  T zero[K];
#pragma unroll
  for (int t = 0; t < K; ++t) zero[t] = (T)0;

  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    const uint8_t lab = label[n];
    fs::stv<T, K, true>(x, n, zero);
    fs::stv<T, K, true>(p, n, zero);
    if (lab == FS_LABEL_FIXED) {
      fs::stv<T, K, true>(r, n, zero);
      continue;
    }
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    // whole-node vector accesses to the FP64 solution and source (no thread
    // reads a node that another thread of this kernel writes: free nodes are
    // zeroed only when no neighbour reads them, solo and pinned nodes have
    // no free neighbours that read them)
    double res[K], bres[K], c[K];
    if (f) {
      fs::ldv<double, K, true>(f, n, res);
    } else {
#pragma unroll
      for (int t = 0; t < K; ++t) res[t] = 0.0;
    }
    if (lab == FS_LABEL_FREE && warm) {
      fs::ldv<double, K, true>(phi, n, c);
    } else {
#pragma unroll
      for (int t = 0; t < K; ++t) c[t] = 0.0;
    }
#pragma unroll
    for (int t = 0; t < K; ++t) bres[t] = res[t];
    double dg = 0.0;
    auto edge = [&](bool ok, double m, long long nb) {
      if (!ok || m == 0.0) return;
      dg += m;
      const bool nb_free = label[nb] == FS_LABEL_FREE;
      double v[K];
      if (nb_free && !warm) {
#pragma unroll
        for (int t = 0; t < K; ++t) v[t] = 0.0;
      } else {
        fs::ldv<double, K, true>(phi, nb, v);
      }
#pragma unroll
      for (int t = 0; t < K; ++t) {
        res[t] -= m * (c[t] - v[t]);
        if (!nb_free) bres[t] += m * v[t];
      }
    };
    edge6(d, mx, my, mz, n, i, j, k, edge);
    if (dgn) {
      const double dd = dgn[n];
      dg += dd;
#pragma unroll
      for (int t = 0; t < K; ++t) res[t] -= dd * c[t];
    }

    if (lab == FS_LABEL_FREE) {
      const double s = s64[n];
      T rv[K];
#pragma unroll
      for (int t = 0; t < K; ++t) {
        double rs = res[t] * s, bs = bres[t] * s;
        rv[t] = (T)rs;
        acc[t] += rs * rs;
        acc[K + t] += bs * bs;
        c[t] = 0.0;
      }
      if (!warm) fs::stv<double, K, true>(phi, n, c);
      fs::stv<T, K, true>(r, n, rv);
    } else {
      // Solo: every coupled neighbour is fixed, so x = b / diag exactly
      // (poisson.py:559-564).  Pinned: coupled to nothing, x = 0 (:522).
#pragma unroll
      for (int t = 0; t < K; ++t) c[t] = (lab == FS_LABEL_SOLO) ? bres[t] / dg : 0.0;
      fs::stv<double, K, true>(phi, n, c);
      fs::stv<T, K, true>(r, n, zero);
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
      s.rr = g;
      s.gamma = g;
      s.gamma_old = g;
      s.fresh = 1;
      s.pq = 0.0;
      s.alpha = 0.0;
      s.beta = 0.0;
      s.bnorm = bn;
      s.rmax = sqrt(g);
      s.best = sqrt(g);
      s.nstall = 0;
      s.iters = 0;
      s.ru = 0;
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
      // maxiter <= 0: the reference's cap max(500, 10 sqrt(n_free))
      // (poisson.py:535-536) from this plan's own classification
      ctl->maxiter = maxiter > 0 ? maxiter
                                 : max(500, (int)(10.0 * sqrt((double)ctl->label_counts[0])));
      ctl->delta = delta;
      ctl->precond = precond > 0 ? 1 : 0;
      ctl->flexible = precond > 1 ? 1 : 0;
      ctl->error = 0;
      refresh_done(st, ctl, K);
    }
  }
}

// ---- K1: q = A~ p and p.q (TMA-staged, 2.5-D tiled, persistent) --------------
// The (z, y) plane is cut into TZ x TY tiles ("columns" along x).  The
// column-planes are dealt out evenly to a persistent grid: each block gets
// one contiguous run of x-planes, which spans at most a few columns.  Along
// a run one thread issues a TMA tensor load per x-plane of the p tile plus
// a one-node halo in y and z into an NS-deep ring of shared-memory stages
// (mbarrier completion, two planes in flight); out-of-range halo nodes
// arrive as zeros, which is the boundary of the eliminated operator.  The
// stencil of plane x reads planes x-1, x, x+1 from the ring.
constexpr long long kWaitBudget = 2000000000LL;  // ~1 s of SM clocks

template <typename T, int K>
struct TmaTile {
  static constexpr int B = K * (int)sizeof(T);       // bytes per node
  static constexpr int TZ = 32;
  static constexpr int TY = B <= 32 ? 16 : (B <= 64 ? 8 : 4);
  static constexpr int NS = 5;                       // ring of x-planes
  static constexpr int HY = TY + 2, HZ = TZ + 2;
  static constexpr int BOX = HY * HZ * B;            // bytes of one plane
  static constexpr int BOXP = (BOX + 127) / 128 * 128;
  static constexpr int THREADS = TZ * TY;
  static constexpr size_t SMEM = (size_t)NS * BOXP + NS * 8 + 128;
  static constexpr bool OK = B >= 16;                // TMA row >= 16 B
};

// A node's K values are NC 16-byte chunks.  A quarter-warp's 16-byte accesses
// are served together; eight consecutive lanes that read chunk c of their
// nodes, NC*16 bytes apart, span 8*NC*16 bytes and so meet each bank NC times
// (with 32-byte nodes lanes 0 and 4 share banks).  Each lane therefore walks its node's chunks
// in rotated order, (c + r) mod NC with r = (lane mod 8) * NC / 8, which puts
// a quarter-warp's eight reads on all 32 banks.  The registers then hold the
// chunks rotated: the per-node arithmetic does not care (the masses are the
// same for every RHS), stores put each chunk back in its place, and the
// per-RHS dot accumulators are un-rotated once at the end (`unrotate`).
template <typename T, int K>
struct NodeChunks {
  static constexpr int B = K * (int)sizeof(T);
  static constexpr bool VEC = B % 16 == 0;
  static constexpr int NC = VEC ? B / 16 : 1;             // 1, 2, 4 or 8
  static constexpr int W = VEC ? 16 / (int)sizeof(T) : K;  // values per chunk
};

template <typename T, int K>
__device__ __forceinline__ int chunk_rot() {
  constexpr int NC = NodeChunks<T, K>::NC;
  return NC > 1 ? (((int)(threadIdx.x & 7) * NC / 8) & (NC - 1)) : 0;
}

template <typename T, int K>
__device__ __forceinline__ void ld_rot(const T* p, T (&v)[K], int r) {
  using NCh = NodeChunks<T, K>;
  if constexpr (NCh::VEC && std::is_same<T, float>::value) {
#pragma unroll
    for (int c = 0; c < NCh::NC; ++c) {
      const float4 t = reinterpret_cast<const float4*>(p)[(c + r) & (NCh::NC - 1)];
      v[4 * c] = t.x; v[4 * c + 1] = t.y; v[4 * c + 2] = t.z; v[4 * c + 3] = t.w;
    }
  } else if constexpr (NCh::VEC && std::is_same<T, double>::value) {
#pragma unroll
    for (int c = 0; c < NCh::NC; ++c) {
      const double2 t = reinterpret_cast<const double2*>(p)[(c + r) & (NCh::NC - 1)];
      v[2 * c] = t.x; v[2 * c + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int c = 0; c < K; ++c) v[c] = p[c];
  }
}

// Load (ld_rot) or store (st_rot) a node's values in rotated chunk order, from
// or to shared or global memory (generic addressing).
template <typename T, int K>
__device__ __forceinline__ void st_rot(T* p, const T (&v)[K], int r) {
  using NCh = NodeChunks<T, K>;
  if constexpr (NCh::VEC && std::is_same<T, float>::value) {
#pragma unroll
    for (int c = 0; c < NCh::NC; ++c)
      reinterpret_cast<float4*>(p)[(c + r) & (NCh::NC - 1)] =
          make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
  } else if constexpr (NCh::VEC && std::is_same<T, double>::value) {
#pragma unroll
    for (int c = 0; c < NCh::NC; ++c)
      reinterpret_cast<double2*>(p)[(c + r) & (NCh::NC - 1)] =
          make_double2(v[2 * c], v[2 * c + 1]);
  } else {
#pragma unroll
    for (int c = 0; c < K; ++c) p[c] = v[c];
  }
}

// Per-node values or per-RHS accumulators held in rotated chunk order, back in
// RHS order.
template <typename T, int K, typename V>
__device__ __forceinline__ void unrotate(V (&a)[K], int r) {
  using NCh = NodeChunks<T, K>;
  if constexpr (NCh::NC > 1) {
    V o[K];
#pragma unroll
    for (int c = 0; c < NCh::NC; ++c) {
#pragma unroll
      for (int tc = 0; tc < NCh::NC; ++tc) {
        if (((c + r) & (NCh::NC - 1)) == tc) {
#pragma unroll
          for (int e = 0; e < NCh::W; ++e) o[tc * NCh::W + e] = a[c * NCh::W + e];
        }
      }
    }
#pragma unroll
    for (int t = 0; t < K; ++t) a[t] = o[t];
  }
}

template <typename T, int K, int NT>
__device__ void finish_pq(double (&acc)[K], double* partials, RhsState* st,
                          Control* ctl) {
  fs::block_partials<K, NT>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketApply])) {
    double tot[K];
    fs::grid_total<K, NT>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
      RhsState& s = st[threadIdx.x];
      s.pq = tot[threadIdx.x];
      if (ctl->error) {
        s.alpha = 0.0;
        if (s.active) s.status = FS_TIMEOUT;
        s.active = 0;
      } else if (s.active) {
        if (tot[threadIdx.x] > 0.0 && isfinite(tot[threadIdx.x])) {
          s.alpha = s.gamma / tot[threadIdx.x];
        } else {
          // A~ is SPD: a finite p.q <= 0 is round-off of a low-precision
          // direction (a stall); NaN/Inf is a breakdown.
          s.alpha = 0.0;
          s.active = 0;
          s.status = isfinite(tot[threadIdx.x]) ? FS_STALLED : FS_NAN;
        }
      } else {
        s.alpha = 0.0;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) refresh_done(st, ctl, K);
  }
}

template <typename T, int K>
__global__ void __launch_bounds__(TmaTile<T, K>::THREADS)
    k_stencil_tma(Dims d, const __grid_constant__ CUtensorMap tm_p,
                  const T* __restrict__ ex, const T* __restrict__ ey,
                  const T* __restrict__ ez, const T* __restrict__ p,
                  T* __restrict__ q, double* __restrict__ partials,
                  RhsState* st, Control* ctl) {
  using C = TmaTile<T, K>;
  if (ctl->all_done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  T* ring = reinterpret_cast<T*>(base);                    // [NS][BOXP]
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::NS * C::BOXP);
  constexpr int BOXT = C::BOXP / (int)sizeof(T);

  const int tid = threadIdx.x;
  const int tz = tid % C::TZ, ty = tid / C::TZ;
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  long long u = 0, u_end = 0;  // column-planes
  fs::march_range<long long>(d, (long long)nbz * nby, u, u_end);

  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();

  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  const int cpos = (ty + 1) * C::HZ + (tz + 1);
  const int rot = chunk_rot<T, K>();
  long long ticket = 0;  // planes issued so far by this block (ring position)
  bool failed = false;
  bool bad = false;

  while (u < u_end && !failed) {
    const long long col = u / d.nx;
    const int xa = (int)(u % d.nx);
    const int xb = (int)min((long long)d.nx, xa + (u_end - u));
    const int bz = (int)(col % nbz), by = (int)(col / nbz);
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nplanes = (xb - xa) + 2;   // planes xa-1 .. xb
    // The six masses of the next plane's node are loaded one plane ahead,
    // so their latency hides behind this plane's arithmetic.
    T nm0 = 0, nm1 = 0, nm2 = 0, nm3 = 0, nm4 = 0, nm5 = 0;
#define FS_LOAD_MASSES(xx)                                       \
  do {                                                          \
    const long long nn = ((long long)(xx) * d.ny + y) * d.nz + z; \
    nm0 = (xx) > 0 ? __ldg(ex + nn - d.sx) : (T)0;              \
    nm1 = __ldg(ex + nn); /* 0 on the last plane (padded) */    \
    nm2 = y > 0 ? __ldg(ey + nn - d.sy) : (T)0;                 \
    nm3 = __ldg(ey + nn);                                       \
    nm4 = z > 0 ? __ldg(ez + nn - 1) : (T)0;                    \
    nm5 = __ldg(ez + nn);                                       \
  } while (0)
    if (inb) FS_LOAD_MASSES(xa);
    auto issue = [&](int j) {
      const int s = (int)((ticket + j) % C::NS);
      fs::mbar_arrive_expect_tx(&bar[s], C::BOX);
      fs::tma_load_4d(ring + s * BOXT, &tm_p, &bar[s], 0, z0 - 1, y0 - 1,
                      xa - 1 + j);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nplanes; ++j) issue(j);
    for (int j = 0; j < nplanes; ++j) {
      const long long tk = ticket + j;
      const int s = (int)(tk % C::NS);
      // One CTA barrier per plane: a wait that ran out is carried to it
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j >= 2) {
        if (inb && !bad) {
          const int x = xa - 2 + j;
          const long long n = ((long long)x * d.ny + y) * d.nz + z;
          const T* pm = ring + (int)((tk - 2) % C::NS) * BOXT;
          const T* pc = ring + (int)((tk - 1) % C::NS) * BOXT;
          const T* pp = ring + s * BOXT;
          const T mxm = nm0, mxp = nm1, mym = nm2, myp = nm3, mzm = nm4, mzp = nm5;
          if (x + 1 < xb) FS_LOAD_MASSES(x + 1);
          T c[K], v[K], qv[K];
          ld_rot<T, K>(pc + cpos * K, c, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] = c[t];
          ld_rot<T, K>(pm + cpos * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxm * v[t];
          ld_rot<T, K>(pp + cpos * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxp * v[t];
          ld_rot<T, K>(pc + (cpos - C::HZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mym * v[t];
          ld_rot<T, K>(pc + (cpos + C::HZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= myp * v[t];
          ld_rot<T, K>(pc + (cpos - 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mzm * v[t];
          ld_rot<T, K>(pc + (cpos + 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) {
            qv[t] -= mzp * v[t];
            acc[t] += (double)c[t] * (double)qv[t];
          }
          st_rot<T, K>(q + n * K, qv, rot);
        }
        // plane j-2 no longer read: its stage may refill
        if (__syncthreads_or(bad)) {
          failed = true;
          break;
        }
        if (tid == 0 && j - 2 + C::NS < nplanes) issue(j - 2 + C::NS);
      }
    }
    ticket += nplanes;
    u += (xb - xa);
  }
#undef FS_LOAD_MASSES
  if (failed) {
    // A staged load did not land in time.  Give copies still in flight a
    // bounded chance to finish before the block exits, then report.
    if (tid == 0) {
      ctl->error = 1;
      for (int s = 0; s < C::NS; ++s)
        (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
  (void)p;
  unrotate<T, K>(acc, rot);
  finish_pq<T, K, TmaTile<T, K>::THREADS>(acc, partials, st, ctl);
}

// ---- K1 with the masses staged too ------------------------------------------------
// Same arithmetic as k_stencil_tma, but each ring stage holds, besides the
// p tile with its halo, the plane's three mass tiles loaded by TMA:
//   ex: (z0.., y0..)        -> m(x), and m(x-1) from the previous stage;
//   ey: (z0.., y0-1..)      -> m(y-1) and m(y);
//   ez: (z0-ZP.., y0..)     -> m(z-1) and m(z) (ZP keeps the innermost
//                              coordinate 16-byte aligned).
// Out-of-range boxes read zero, which is exactly the missing edge at a wall,
// so the inner loop has no global loads and no boundary branches.  Smaller
// tiles (TY = 8) keep three CTAs per SM with two planes in flight each.
// TYO > 0 overrides the tile height (the tile shapes the stencil autotuner
// tries for the fused direction-update stencil).
template <typename T, int K, int TYO = 0>
struct TmaTileM {
  static constexpr int B = K * (int)sizeof(T);
  static constexpr int MB = (int)sizeof(T);
  static constexpr int TZ = 32;
  static constexpr int TY = TYO > 0 ? TYO : (B <= 32 ? 8 : 4);
  static constexpr int NS = 5;
  static constexpr int ZP = 16 / MB;
  static constexpr int HY = TY + 2, HZ = TZ + 2;
  static constexpr int BOX = HY * HZ * B;
  static constexpr int EXB = TZ * TY * MB;
  static constexpr int EYB = TZ * (TY + 1) * MB;
  static constexpr int EZB = (TZ + ZP) * TY * MB;
  static constexpr int O_EX = (BOX + 127) / 128 * 128;
  static constexpr int O_EY = O_EX + (EXB + 127) / 128 * 128;
  static constexpr int O_EZ = O_EY + (EYB + 127) / 128 * 128;
  static constexpr int SLOT = O_EZ + (EZB + 127) / 128 * 128;
  static constexpr uint32_t TX = (uint32_t)(BOX + EXB + EYB + EZB);  // bytes per stage
  static constexpr int THREADS = TZ * TY;
  static constexpr size_t SMEM = (size_t)NS * SLOT + NS * 8 + 128;
  static constexpr bool OK = B >= 16;
};

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::"
      "bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(fs::smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(fs::smem_u32(bar))
      : "memory");
}

template <typename T, int K>
__global__ void __launch_bounds__(TmaTileM<T, K>::THREADS, (TmaTileM<T, K>::B <= 32 ? 3 : 1))
    k_stencil_tma_m(Dims d, const __grid_constant__ CUtensorMap tm_p,
                    const __grid_constant__ CUtensorMap tm_ex,
                    const __grid_constant__ CUtensorMap tm_ey,
                    const __grid_constant__ CUtensorMap tm_ez, T* __restrict__ q,
                    double* __restrict__ partials, RhsState* st, Control* ctl) {
  using C = TmaTileM<T, K>;
  if (ctl->all_done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::NS * C::SLOT);
  const int tid = threadIdx.x;
  const int tz = tid % C::TZ, ty = tid / C::TZ;
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  // column-planes in 32-bit: N / (TZ * TY) of them (the launch checks the bound)
  int u = 0, u_end = 0;
  fs::march_range<int>(d, nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  const int cpos = (ty + 1) * C::HZ + (tz + 1);
  const int rot = chunk_rot<T, K>();
  int ticket = 0;
  bool failed = false;
  bool bad = false;
  while (u < u_end && !failed) {
    const int col = u / d.nx;
    const int xa = u - col * d.nx;
    const int xb = min(d.nx, xa + (u_end - u));
    const int by = col / nbz, bz = col - by * nbz;
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nplanes = (xb - xa) + 2;  // planes xa-1 .. xb
    auto issue = [&](int j) {
      const int s = (ticket + j) % C::NS;
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 1 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      fs::tma_load_4d(slot, &tm_p, &bar[s], 0, z0 - 1, y0 - 1, x);
      tma_load_3d(slot + C::O_EX, &tm_ex, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_EY, &tm_ey, &bar[s], z0, y0 - 1, x);
      tma_load_3d(slot + C::O_EZ, &tm_ez, &bar[s], z0 - C::ZP, y0, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nplanes; ++j) issue(j);
    for (int j = 0; j < nplanes; ++j) {
      const int tk = ticket + j;
      const int s = tk % C::NS;
      // One CTA barrier per plane: a wait that ran out is carried to it
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j >= 2) {
        if (inb && !bad) {
          const int x = xa - 2 + j;
          const long long n = ((long long)x * d.ny + y) * d.nz + z;
          const unsigned char* sm = base + ((tk - 2) % C::NS) * C::SLOT;  // plane x-1
          const unsigned char* sc = base + ((tk - 1) % C::NS) * C::SLOT;  // plane x
          const unsigned char* sp = base + s * C::SLOT;                        // plane x+1
          const T* pm = reinterpret_cast<const T*>(sm);
          const T* pc = reinterpret_cast<const T*>(sc);
          const T* pp = reinterpret_cast<const T*>(sp);
          const T* exm = reinterpret_cast<const T*>(sm + C::O_EX);
          const T* exc = reinterpret_cast<const T*>(sc + C::O_EX);
          const T* eyc = reinterpret_cast<const T*>(sc + C::O_EY);
          const T* ezc = reinterpret_cast<const T*>(sc + C::O_EZ);
          const T mxm = exm[ty * C::TZ + tz], mxp = exc[ty * C::TZ + tz];
          const T mym = eyc[ty * C::TZ + tz], myp = eyc[(ty + 1) * C::TZ + tz];
          const T mzm = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP - 1];
          const T mzp = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP];
          T c[K], v[K], qv[K];
          ld_rot<T, K>(pc + cpos * K, c, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] = c[t];
          ld_rot<T, K>(pm + cpos * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxm * v[t];
          ld_rot<T, K>(pp + cpos * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxp * v[t];
          ld_rot<T, K>(pc + (cpos - C::HZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mym * v[t];
          ld_rot<T, K>(pc + (cpos + C::HZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= myp * v[t];
          ld_rot<T, K>(pc + (cpos - 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mzm * v[t];
          ld_rot<T, K>(pc + (cpos + 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) {
            qv[t] -= mzp * v[t];
            acc[t] += (double)c[t] * (double)qv[t];
          }
          st_rot<T, K>(q + n * K, qv, rot);
        }
        // plane j-2 no longer read: its stage may refill
        if (__syncthreads_or(bad)) {
          failed = true;
          break;
        }
        if (tid == 0 && j - 2 + C::NS < nplanes) issue(j - 2 + C::NS);
      }
    }
    ticket += nplanes;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      ctl->error = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
  unrotate<T, K>(acc, rot);
  finish_pq<T, K, TmaTileM<T, K>::THREADS>(acc, partials, st, ctl);
}

// ---- K1 with the direction update fused in ----------------------------------------
// The CG direction p = z + beta p_old (k_pnew) formed inside the stencil: each
// ring stage holds the z tile and the p_old tile (both with the one-node halo)
// next to the plane's three mass tiles, every stencil point forms its p value
// from the two, and the thread of a node writes its p (the new direction, for
// the update kernel and the next iteration) and q = A~p, with p.q reduced as
// in k_stencil_tma_m.  Every right-hand side takes p = z + beta p_old (one
// FMA, k_pnew's arithmetic for an active one); an inactive one's direction is
// never read again (its step length is 0 and a solve restarts from k_init),
// so it needs no exception.  Per node: z and p_old read, p and q written
// (4 vectors) instead of the 5 of k_pnew followed by the stencil.
// a * b + c with one rounding (k_pnew's contracted r + beta * p_old)
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }

template <typename T, int K, int TYO = 0>
struct TmaTilePZ {
  using M = TmaTileM<T, K, TYO>;
  static constexpr int B = M::B, MB = M::MB, TZ = M::TZ, TY = M::TY, HY = M::HY,
                       HZ = M::HZ, ZP = M::ZP;
  static constexpr int NS = 4;
  static constexpr int BOX = M::BOX;
  static constexpr int EXB = M::EXB, EYB = M::EYB, EZB = M::EZB;
  static constexpr int O_P = (BOX + 127) / 128 * 128;          // p_old tile
  static constexpr int O_EX = O_P + (BOX + 127) / 128 * 128;
  static constexpr int O_EY = O_EX + (EXB + 127) / 128 * 128;
  static constexpr int O_EZ = O_EY + (EYB + 127) / 128 * 128;
  static constexpr int SLOT = O_EZ + (EZB + 127) / 128 * 128;
  static constexpr uint32_t TX = (uint32_t)(2 * BOX + EXB + EYB + EZB);
  static constexpr int THREADS = TZ * TY;
  static constexpr size_t SMEM = (size_t)NS * SLOT + NS * 8 + K * sizeof(T) + 256;
  static constexpr bool OK = M::OK;
};

template <typename T, int K, int TYO = 0>
__global__ void __launch_bounds__(TmaTilePZ<T, K, TYO>::THREADS,
                                  TmaTilePZ<T, K, TYO>::THREADS >= 512 ? 1 : 2)
    k_stencil_pz(Dims d, const __grid_constant__ CUtensorMap tm_z,
                 const __grid_constant__ CUtensorMap tm_pold,
                 const __grid_constant__ CUtensorMap tm_ex,
                 const __grid_constant__ CUtensorMap tm_ey,
                 const __grid_constant__ CUtensorMap tm_ez, T* __restrict__ pnew,
                 T* __restrict__ q, double* __restrict__ partials, RhsState* st,
                 Control* ctl) {
  using C = TmaTilePZ<T, K, TYO>;
  if (ctl->all_done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::NS * C::SLOT);
  T* beta_s = reinterpret_cast<T*>(bar + C::NS);  // per RHS: p = z + beta p_old
  const int tid = threadIdx.x;
  const int tz = tid % C::TZ, ty = tid / C::TZ;
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  int u = 0, u_end = 0;  // column-planes
  fs::march_range<int>(d, nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  if (tid < K) beta_s[tid] = (T)st[tid].beta;
  __syncthreads();
  const int rot = chunk_rot<T, K>();
  // the two coefficients in this thread's rotated chunk order
  T cp[K];
  {
    // ld_rot's register order: slot (c, e) holds RHS ((c + rot) mod NC) * W + e
    using NCh = NodeChunks<T, K>;
#pragma unroll
    for (int c = 0; c < NCh::NC; ++c)
#pragma unroll
      for (int e = 0; e < NCh::W; ++e)
        cp[c * NCh::W + e] = beta_s[((c + rot) & (NCh::NC - 1)) * NCh::W + e];
  }
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  const int cpos = (ty + 1) * C::HZ + (tz + 1);
  int ticket = 0;
  bool failed = false;
  bool bad = false;
  while (u < u_end && !failed) {
    const int col = u / d.nx;
    const int xa = u - col * d.nx;
    const int xb = min(d.nx, xa + (u_end - u));
    const int by = col / nbz, bz = col - by * nbz;
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nplanes = (xb - xa) + 2;  // planes xa-1 .. xb
    auto issue = [&](int j) {
      const int s = (ticket + j) % C::NS;
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 1 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      fs::tma_load_4d(slot, &tm_z, &bar[s], 0, z0 - 1, y0 - 1, x);
      fs::tma_load_4d(slot + C::O_P, &tm_pold, &bar[s], 0, z0 - 1, y0 - 1, x);
      tma_load_3d(slot + C::O_EX, &tm_ex, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_EY, &tm_ey, &bar[s], z0, y0 - 1, x);
      tma_load_3d(slot + C::O_EZ, &tm_ez, &bar[s], z0 - C::ZP, y0, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nplanes; ++j) issue(j);
    for (int j = 0; j < nplanes; ++j) {
      const int tk = ticket + j;
      const int s = tk % C::NS;
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j >= 2) {
        if (inb && !bad) {
          const int x = xa - 2 + j;
          const long long n = ((long long)x * d.ny + y) * d.nz + z;
          const unsigned char* sm = base + ((tk - 2) % C::NS) * C::SLOT;  // plane x-1
          const unsigned char* sc = base + ((tk - 1) % C::NS) * C::SLOT;  // plane x
          const unsigned char* sp = base + s * C::SLOT;                   // plane x+1
          const T* exm = reinterpret_cast<const T*>(sm + C::O_EX);
          const T* exc = reinterpret_cast<const T*>(sc + C::O_EX);
          const T* eyc = reinterpret_cast<const T*>(sc + C::O_EY);
          const T* ezc = reinterpret_cast<const T*>(sc + C::O_EZ);
          const T mxm = exm[ty * C::TZ + tz], mxp = exc[ty * C::TZ + tz];
          const T mym = eyc[ty * C::TZ + tz], myp = eyc[(ty + 1) * C::TZ + tz];
          const T mzm = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP - 1];
          const T mzp = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP];
          // p at tile node i of a plane: z + beta * p_old
          auto pval = [&](const unsigned char* pl, int i, T (&v)[K]) {
            T zv[K];
            ld_rot<T, K>(reinterpret_cast<const T*>(pl) + i * K, zv, rot);
            ld_rot<T, K>(reinterpret_cast<const T*>(pl + C::O_P) + i * K, v, rot);
#pragma unroll
            for (int t = 0; t < K; ++t) v[t] = fma_t(cp[t], v[t], zv[t]);
          };
          T c[K], v[K], qv[K];
          pval(sc, cpos, c);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] = c[t];
          pval(sm, cpos, v);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxm * v[t];
          pval(sp, cpos, v);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxp * v[t];
          pval(sc, cpos - C::HZ, v);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mym * v[t];
          pval(sc, cpos + C::HZ, v);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= myp * v[t];
          pval(sc, cpos - 1, v);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mzm * v[t];
          pval(sc, cpos + 1, v);
#pragma unroll
          for (int t = 0; t < K; ++t) {
            qv[t] -= mzp * v[t];
            acc[t] += (double)c[t] * (double)qv[t];
          }
          st_rot<T, K>(pnew + n * K, c, rot);
          st_rot<T, K>(q + n * K, qv, rot);
        }
        if (__syncthreads_or(bad)) {
          failed = true;
          break;
        }
        if (tid == 0 && j - 2 + C::NS < nplanes) issue(j - 2 + C::NS);
      }
    }
    ticket += nplanes;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      ctl->error = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
  unrotate<T, K>(acc, rot);
  finish_pq<T, K, TmaTilePZ<T, K, TYO>::THREADS>(acc, partials, st, ctl);
}

// ---- K1 variant: q written through shared memory by TMA stores -------------------
// The same computation as k_stencil_tma_m (p and the three mass tiles staged by
// TMA, one thread per node of a TZ x TY column marching along x), but each
// plane's q tile goes to shared memory and leaves with one bulk tensor store
// instead of two 16-byte global stores per thread.  Two q buffers alternate;
// the store of a buffer must have finished reading it before the buffer is
// written again two planes later (bulk_group read wait by the issuing thread,
// then the CTA barrier).  Four p stages keep three CTAs per SM resident.
template <typename T, int K>
struct TmaTileS {
  using M = TmaTileM<T, K>;
  static constexpr int B = M::B, TZ = M::TZ, TY = M::TY, HY = M::HY, HZ = M::HZ, ZP = M::ZP;
  static constexpr int NS = 4;
  static constexpr int SLOT = M::SLOT, O_EX = M::O_EX, O_EY = M::O_EY, O_EZ = M::O_EZ;
  static constexpr uint32_t TX = M::TX;
  static constexpr int QB = TZ * TY * B;  // one q tile, [TY][TZ][K]
  static constexpr int O_Q = NS * SLOT;
  static constexpr int THREADS = M::THREADS;
  static constexpr size_t SMEM = (size_t)NS * SLOT + 2 * (size_t)QB + NS * 8 + 128;
  static constexpr bool OK = M::OK;
};

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, const void* src, int c0,
                                             int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
          (uint64_t)map),
      "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(fs::smem_u32(src))
      : "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// at most one committed store group may still be reading shared memory
__device__ __forceinline__ void bulk_wait_read_1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

template <typename T, int K>
__global__ void __launch_bounds__(TmaTileS<T, K>::THREADS, (TmaTileS<T, K>::B <= 32 ? 3 : 1))
    k_stencil_tma_s(Dims d, const __grid_constant__ CUtensorMap tm_p,
                    const __grid_constant__ CUtensorMap tm_ex,
                    const __grid_constant__ CUtensorMap tm_ey,
                    const __grid_constant__ CUtensorMap tm_ez,
                    const __grid_constant__ CUtensorMap tm_q,
                    double* __restrict__ partials, RhsState* st, Control* ctl) {
  using C = TmaTileS<T, K>;
  if (ctl->all_done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::O_Q + 2 * C::QB);
  const int tid = threadIdx.x;
  const int tz = tid % C::TZ, ty = tid / C::TZ;
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  long long u = 0, u_end = 0;  // column-planes
  fs::march_range<long long>(d, (long long)nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  const int cpos = (ty + 1) * C::HZ + (tz + 1);
  const int rot = chunk_rot<T, K>();
  long long ticket = 0, qc = 0;
  bool failed = false;
  while (u < u_end && !failed) {
    const long long col = u / d.nx;
    const int xa = (int)(u % d.nx);
    const int xb = (int)min((long long)d.nx, xa + (u_end - u));
    const int bz = (int)(col % nbz), by = (int)(col / nbz);
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nplanes = (xb - xa) + 2;  // planes xa-1 .. xb
    auto issue = [&](int j) {
      const int s = (int)((ticket + j) % C::NS);
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 1 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      fs::tma_load_4d(slot, &tm_p, &bar[s], 0, z0 - 1, y0 - 1, x);
      tma_load_3d(slot + C::O_EX, &tm_ex, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_EY, &tm_ey, &bar[s], z0, y0 - 1, x);
      tma_load_3d(slot + C::O_EZ, &tm_ez, &bar[s], z0 - C::ZP, y0, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nplanes; ++j) issue(j);
    for (int j = 0; j < nplanes; ++j) {
      const long long tk = ticket + j;
      const int s = (int)(tk % C::NS);
      // the q buffer written this plane was last stored two planes ago
      if (tid == 0 && j >= 2) bulk_wait_read_1();
      const bool ok = fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      if (j >= 2) {
        const int x = xa - 2 + j;
        T* qt = reinterpret_cast<T*>(base + C::O_Q + (int)(qc & 1) * C::QB);
        if (inb) {
          const unsigned char* sm = base + (int)((tk - 2) % C::NS) * C::SLOT;  // plane x-1
          const unsigned char* sc = base + (int)((tk - 1) % C::NS) * C::SLOT;  // plane x
          const unsigned char* sp = base + s * C::SLOT;                        // plane x+1
          const T* pm = reinterpret_cast<const T*>(sm);
          const T* pc = reinterpret_cast<const T*>(sc);
          const T* pp = reinterpret_cast<const T*>(sp);
          const T* exm = reinterpret_cast<const T*>(sm + C::O_EX);
          const T* exc = reinterpret_cast<const T*>(sc + C::O_EX);
          const T* eyc = reinterpret_cast<const T*>(sc + C::O_EY);
          const T* ezc = reinterpret_cast<const T*>(sc + C::O_EZ);
          const T mxm = exm[ty * C::TZ + tz], mxp = exc[ty * C::TZ + tz];
          const T mym = eyc[ty * C::TZ + tz], myp = eyc[(ty + 1) * C::TZ + tz];
          const T mzm = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP - 1];
          const T mzp = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP];
          T c[K], v[K], qv[K];
          ld_rot<T, K>(pc + cpos * K, c, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] = c[t];
          ld_rot<T, K>(pm + cpos * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxm * v[t];
          ld_rot<T, K>(pp + cpos * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mxp * v[t];
          ld_rot<T, K>(pc + (cpos - C::HZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mym * v[t];
          ld_rot<T, K>(pc + (cpos + C::HZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= myp * v[t];
          ld_rot<T, K>(pc + (cpos - 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) qv[t] -= mzm * v[t];
          ld_rot<T, K>(pc + (cpos + 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) {
            qv[t] -= mzp * v[t];
            acc[t] += (double)c[t] * (double)qv[t];
          }
          st_rot<T, K>(qt + (ty * C::TZ + tz) * K, qv, rot);
        }
        fence_proxy_async_smem();  // q tile writes -> visible to the bulk store
        __syncthreads();           // plane j-2 no longer read; q tile complete
        if (tid == 0) {
          tma_store_4d(&tm_q, qt, 0, z0, y0, x);  // out-of-range rows are clipped
          bulk_commit();
          if (j - 2 + C::NS < nplanes) issue(j - 2 + C::NS);
        }
        ++qc;
      }
    }
    ticket += nplanes;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      ctl->error = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
  if (tid == 0) bulk_wait_all();  // q written out before the CTA's shared memory goes
  unrotate<T, K>(acc, rot);
  finish_pq<T, K, TmaTileS<T, K>::THREADS>(acc, partials, st, ctl);
}

// ---- multigrid: degree-2 pre-smoothing from 0 in one pass over b ------------------
// k_mg_pre0 then k_mg_pre1 compute, from b alone,
//   x1 = c0 b,  r1 = b - c0 A~b,  d1 = cd x1 + cr r1,  x2 = x1 + d1,  r2 = r1 - A~d1,
// writing x1 and r1 (2 vectors) and reading them back at every node and its six
// neighbours.  Here one x-march does both stencils: per x-plane one thread issues
// TMA loads (no multicast) of the b tile with a two-node halo in y and z and of the
// three equilibrated mass tiles into an NS-deep ring; stage 1 forms d1 on the tile
// plus a one-node halo (the thread of each interior node, and one more node for 84
// of the threads on the halo ring) into a three-plane ring of d1 tiles; stage 2,
// one plane behind, forms A~d1 at the interior from that ring and from the d1, r1,
// x1 and masses of its own node kept in registers.  b is read once and only x2,
// r2 are written: 3 vectors + the masses per node instead of 7 + twice the masses.
// The arithmetic, and its order, is that of the two kernels.  Out-of-range boxes
// read zero, which is the wall (missing edges) and a zero right-hand side.
// One CTA barrier per plane: the d1 ring has three slots, so stage 1 of plane q+1
// writes the slot that stage 2 of plane q-2 read before the previous barrier.
template <typename T, int K>
struct SmoothTile {
  static constexpr int B = K * (int)sizeof(T);
  static constexpr int MB = (int)sizeof(T);
  static constexpr int TZ = 32, TY = 8;
  static constexpr int NS = 4;                      // input planes in the ring
  static constexpr int IZ = TZ + 4, IY = TY + 4;    // b tile: two-node halo
  static constexpr int RZ = TZ + 2, RY = TY + 2;    // d1 tile: one-node halo
  static constexpr int ZP = 16 / MB;                // mass boxes start at z0 - ZP
  static constexpr int WZ = TZ + 2 * ZP;            // mass box width (16-byte rows)
  static constexpr int WY = TY + 3;                 // mass box rows from y0 - 2
  static constexpr int BOXB = IZ * IY * B;
  static constexpr int MBOX = WZ * WY * MB;
  static constexpr int O_M0 = (BOXB + 127) / 128 * 128;
  static constexpr int MBOXP = (MBOX + 127) / 128 * 128;
  static constexpr int SLOT = O_M0 + 3 * MBOXP;
  static constexpr uint32_t TX = (uint32_t)(BOXB + 3 * MBOX);  // bytes per plane
  static constexpr int UPL = RZ * RY * B;           // one d1 plane
  static constexpr int UPLP = (UPL + 127) / 128 * 128;
  static constexpr int O_U = NS * SLOT;
  static constexpr int O_BAR = O_U + 3 * UPLP;
  static constexpr int THREADS = TZ * TY;
  static constexpr int NHALO = 2 * RZ + 2 * (RY - 2);
  static constexpr size_t SMEM = (size_t)O_BAR + NS * 8 + 128;
  // 8..32-byte nodes, two CTAs per SM.  16- and 32-byte nodes are staged by a
  // 4-D map {K, z, y, x}; 8-byte nodes (one FP64 RHS, two FP32) by a 3-D map
  // whose innermost dimension merges K and z (rows of IZ*K values from
  // (z0 - 2)*K, 16-byte aligned because z0 is a multiple of 32).
  static constexpr bool OK = B >= 8 && B <= 32 && B % 8 == 0 && NHALO <= THREADS;
  static constexpr bool MERGED = B < 16;
};

// The vector tile of plane x for a fused smoothing pass (see SmoothTile).
template <typename T, int K>
__device__ __forceinline__ void smooth_tile_load(void* slot, const CUtensorMap* map,
                                                 uint64_t* bar, int z0, int y0, int x) {
  if constexpr (SmoothTile<T, K>::MERGED)
    tma_load_3d(slot, map, bar, (z0 - 2) * K, y0 - 2, x);
  else
    fs::tma_load_4d(slot, map, bar, 0, z0 - 2, y0 - 2, x);
}

template <typename T, int K>
__global__ void __launch_bounds__(SmoothTile<T, K>::THREADS, 2)
    k_mg_pre_fused(Dims d, const __grid_constant__ CUtensorMap tm_b,
                   const __grid_constant__ CUtensorMap tm_ex,
                   const __grid_constant__ CUtensorMap tm_ey,
                   const __grid_constant__ CUtensorMap tm_ez, T* __restrict__ x2,
                   T* __restrict__ r2, T c0, T cd, T cr, const int* __restrict__ done,
                   int* __restrict__ err) {
  using C = SmoothTile<T, K>;
  if (*done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::O_BAR);
  const int tid = threadIdx.x;
  const int tz = tid % C::TZ, ty = tid / C::TZ;
  const int rot = chunk_rot<T, K>();
  // the halo-ring node of this thread (tid < NHALO), in d1-tile coordinates
  int hz = 0, hy = 0;
  if (tid < 2 * C::RZ) {
    hz = tid % C::RZ;
    hy = tid < C::RZ ? 0 : C::RY - 1;
  } else if (tid < C::NHALO) {
    const int k2 = tid - 2 * C::RZ;
    hy = 1 + k2 / 2;
    hz = (k2 & 1) ? C::RZ - 1 : 0;
  }
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  // column-planes in 32-bit: N / (TZ * TY) of them (the launch checks the bound)
  int u = 0, u_end = 0;
  fs::march_range<int>(d, nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  int ticket = 0, uc = 0;
  bool failed = false, bad = false;
  while (u < u_end && !failed) {
    const int col = u / d.nx;
    const int xa = u - col * d.nx;
    const int xb = min(d.nx, xa + (u_end - u));
    const int by = col / nbz, bz = col - by * nbz;
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nin = (xb - xa) + 4;  // input planes xa-2 .. xb+1
    auto issue = [&](int j) {
      const int s = (ticket + j) % C::NS;
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 2 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      smooth_tile_load<T, K>(slot, &tm_b, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_M0, &tm_ex, &bar[s], z0 - C::ZP, y0 - 2, x);
      tma_load_3d(slot + C::O_M0 + C::MBOXP, &tm_ey, &bar[s], z0 - C::ZP, y0 - 2, x);
      tma_load_3d(slot + C::O_M0 + 2 * C::MBOXP, &tm_ez, &bar[s], z0 - C::ZP, y0 - 2, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nin; ++j) issue(j);
    // own interior node: d1 of planes q-2 (dA), q-1 (dB), q (dC); r1, x1 and the
    // six masses of planes q-1 (B) and q (C)
    T dA[K], dB[K], dC[K], r1B[K], r1C[K], x1B[K], x1C[K];
    T mB[6], mC[6];
    for (int j = 0; j < nin; ++j) {
      const int tk = ticket + j;
      const int s = tk % C::NS;
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j < 2) continue;
      // ---- stage 1: d1 on plane q = xa - 3 + j (input planes q-1, q, q+1)
      const unsigned char* sm = base + ((tk - 2) % C::NS) * C::SLOT;
      const unsigned char* sc = base + ((tk - 1) % C::NS) * C::SLOT;
      const unsigned char* sp = base + s * C::SLOT;
      T* up = reinterpret_cast<T*>(base + C::O_U + (uc % 3) * C::UPLP);
      if (!bad) {
        const T* bm = reinterpret_cast<const T*>(sm);
        const T* bc = reinterpret_cast<const T*>(sc);
        const T* bp = reinterpret_cast<const T*>(sp);
        const T* exm = reinterpret_cast<const T*>(sm + C::O_M0);
        const T* exc = reinterpret_cast<const T*>(sc + C::O_M0);
        const T* eyc = reinterpret_cast<const T*>(sc + C::O_M0 + C::MBOXP);
        const T* ezc = reinterpret_cast<const T*>(sc + C::O_M0 + 2 * C::MBOXP);
        // d1 at d1-tile node (rz, ry); the interior node also keeps r1, x1, masses
        auto stage1 = [&](int rz, int ry, bool own) {
          const int bi = (ry + 1) * C::IZ + (rz + 1);        // b tile
          const int mi = (ry + 1) * C::WZ + (rz - 1 + C::ZP);  // mass tiles
          const T mxm = exm[mi], mxp = exc[mi];
          const T mym = eyc[mi - C::WZ], myp = eyc[mi];
          const T mzm = ezc[mi - 1], mzp = ezc[mi];
          T bv[K], ab[K], v[K];
          ld_rot<T, K>(bc + bi * K, bv, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] = bv[t];
          ld_rot<T, K>(bm + bi * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] -= mxm * v[t];
          ld_rot<T, K>(bp + bi * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] -= mxp * v[t];
          ld_rot<T, K>(bc + (bi - C::IZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] -= mym * v[t];
          ld_rot<T, K>(bc + (bi + C::IZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] -= myp * v[t];
          ld_rot<T, K>(bc + (bi - 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] -= mzm * v[t];
          ld_rot<T, K>(bc + (bi + 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ab[t] -= mzp * v[t];
          T dv[K];
#pragma unroll
          for (int t = 0; t < K; ++t) {
            const T xo = c0 * bv[t];          // k_mg_pre0
            const T rv = bv[t] - c0 * ab[t];
            dv[t] = cd * xo + cr * rv;        // k_mg_pre1
            if (own) {
              x1C[t] = xo;
              r1C[t] = rv;
              dC[t] = dv[t];
            }
          }
          st_rot<T, K>(up + (ry * C::RZ + rz) * K, dv, rot);
          if (own) {
            mC[0] = mxm; mC[1] = mxp; mC[2] = mym; mC[3] = myp; mC[4] = mzm; mC[5] = mzp;
          }
        };
        stage1(tz + 1, ty + 1, true);
        if (tid < C::NHALO) stage1(hz, hy, false);
      }
      ++uc;
      // d1 of plane q complete; input plane q-1 no longer read: its stage may refill
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      if (tid == 0 && j - 2 + C::NS < nin) issue(j - 2 + C::NS);
      // ---- stage 2: plane o = q - 1 = xa - 4 + j (d1 planes o-1, o, o+1)
      if (j >= 4 && inb) {
        const int x = xa - 4 + j;
        const long long n = ((long long)x * d.ny + y) * d.nz + z;
        const T* uo = reinterpret_cast<const T*>(base + C::O_U + ((uc - 2) % 3) * C::UPLP);
        const int ui = (ty + 1) * C::RZ + (tz + 1);
        T ad[K], v[K];
#pragma unroll
        for (int t = 0; t < K; ++t) {
          ad[t] = dB[t];
          ad[t] -= mB[0] * dA[t];
        }
#pragma unroll
        for (int t = 0; t < K; ++t) ad[t] -= mB[1] * dC[t];
        ld_rot<T, K>(uo + (ui - C::RZ) * K, v, rot);
#pragma unroll
        for (int t = 0; t < K; ++t) ad[t] -= mB[2] * v[t];
        ld_rot<T, K>(uo + (ui + C::RZ) * K, v, rot);
#pragma unroll
        for (int t = 0; t < K; ++t) ad[t] -= mB[3] * v[t];
        ld_rot<T, K>(uo + (ui - 1) * K, v, rot);
#pragma unroll
        for (int t = 0; t < K; ++t) ad[t] -= mB[4] * v[t];
        ld_rot<T, K>(uo + (ui + 1) * K, v, rot);
        T xo[K], ro[K];
#pragma unroll
        for (int t = 0; t < K; ++t) {
          ad[t] -= mB[5] * v[t];
          xo[t] = x1B[t] + dB[t];
          ro[t] = r1B[t] - ad[t];
        }
        st_rot<T, K>(x2 + n * K, xo, rot);
        st_rot<T, K>(r2 + n * K, ro, rot);
      }
      // shift the own-node pipeline by one plane
#pragma unroll
      for (int t = 0; t < K; ++t) {
        dA[t] = dB[t];
        dB[t] = dC[t];
        r1B[t] = r1C[t];
        x1B[t] = x1C[t];
      }
#pragma unroll
      for (int e = 0; e < 6; ++e) mB[e] = mC[e];
    }
    ticket += nin;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      *err = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
}

// ---- multigrid: degree-2 post-smoothing in one pass ------------------------------
// k_mg_residual then k_mg_post2 compute r0 = b - A~x (written, then read back at
// every node and its six neighbours) and xout = x + alpha r0 + beta A~r0.  Here
// one x-march does both, with the tiles of k_mg_pre_fused: x with a two-node
// halo and the three mass tiles by TMA, r0 on the tile plus a one-node halo into
// a three-plane ring (stage 1), A~r0 one plane behind at the interior (stage 2)
// from that ring and from the r0, x and masses of the thread's own node kept in
// registers.  b is only needed at the node itself: a plain load.  x and b are
// read once and only xout is written: 3 vectors + the masses per node instead of
// 6 + twice the masses.  The arithmetic, and its order, is that of the two
// kernels.
template <typename T, int K>
__global__ void __launch_bounds__(SmoothTile<T, K>::THREADS, 2)
    k_mg_post_fused(Dims d, const __grid_constant__ CUtensorMap tm_x,
                    const __grid_constant__ CUtensorMap tm_ex,
                    const __grid_constant__ CUtensorMap tm_ey,
                    const __grid_constant__ CUtensorMap tm_ez, const T* __restrict__ b,
                    T* __restrict__ xout, T alpha, T beta, const int* __restrict__ done,
                    int* __restrict__ err) {
  using C = SmoothTile<T, K>;
  if (*done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::O_BAR);
  const int tid = threadIdx.x;
  const int tz = tid % C::TZ, ty = tid / C::TZ;
  const int rot = chunk_rot<T, K>();
  int hz = 0, hy = 0;  // the halo-ring node of this thread (tid < NHALO)
  if (tid < 2 * C::RZ) {
    hz = tid % C::RZ;
    hy = tid < C::RZ ? 0 : C::RY - 1;
  } else if (tid < C::NHALO) {
    const int k2 = tid - 2 * C::RZ;
    hy = 1 + k2 / 2;
    hz = (k2 & 1) ? C::RZ - 1 : 0;
  }
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  int u = 0, u_end = 0;  // column-planes
  fs::march_range<int>(d, nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  int ticket = 0, uc = 0;
  bool failed = false, bad = false;
  while (u < u_end && !failed) {
    const int col = u / d.nx;
    const int xa = u - col * d.nx;
    const int xb = min(d.nx, xa + (u_end - u));
    const int by = col / nbz, bz = col - by * nbz;
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nin = (xb - xa) + 4;  // input planes xa-2 .. xb+1
    auto issue = [&](int j) {
      const int s = (ticket + j) % C::NS;
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 2 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      smooth_tile_load<T, K>(slot, &tm_x, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_M0, &tm_ex, &bar[s], z0 - C::ZP, y0 - 2, x);
      tma_load_3d(slot + C::O_M0 + C::MBOXP, &tm_ey, &bar[s], z0 - C::ZP, y0 - 2, x);
      tma_load_3d(slot + C::O_M0 + 2 * C::MBOXP, &tm_ez, &bar[s], z0 - C::ZP, y0 - 2, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nin; ++j) issue(j);
    // own interior node: r0 of planes q-2 (rA), q-1 (rB), q (rC); x and the six
    // masses of planes q-1 (B) and q (C)
    T rA[K], rB[K], rC[K], xB[K], xC[K];
    T mB[6], mC[6];
    for (int j = 0; j < nin; ++j) {
      const int tk = ticket + j;
      const int s = tk % C::NS;
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j < 2) continue;
      // ---- stage 1: r0 on plane q = xa - 3 + j (input planes q-1, q, q+1)
      const int q = xa - 3 + j;
      const unsigned char* sm = base + ((tk - 2) % C::NS) * C::SLOT;
      const unsigned char* sc = base + ((tk - 1) % C::NS) * C::SLOT;
      const unsigned char* sp = base + s * C::SLOT;
      T* up = reinterpret_cast<T*>(base + C::O_U + (uc % 3) * C::UPLP);
      if (!bad) {
        const T* vm = reinterpret_cast<const T*>(sm);
        const T* vc = reinterpret_cast<const T*>(sc);
        const T* vp = reinterpret_cast<const T*>(sp);
        const T* exm = reinterpret_cast<const T*>(sm + C::O_M0);
        const T* exc = reinterpret_cast<const T*>(sc + C::O_M0);
        const T* eyc = reinterpret_cast<const T*>(sc + C::O_M0 + C::MBOXP);
        const T* ezc = reinterpret_cast<const T*>(sc + C::O_M0 + 2 * C::MBOXP);
        auto stage1 = [&](int rz, int ry, bool own) {
          const int bi = (ry + 1) * C::IZ + (rz + 1);
          const int mi = (ry + 1) * C::WZ + (rz - 1 + C::ZP);
          const T mxm = exm[mi], mxp = exc[mi];
          const T mym = eyc[mi - C::WZ], myp = eyc[mi];
          const T mzm = ezc[mi - 1], mzp = ezc[mi];
          T xv[K], ax[K], v[K], bv[K];
          // b at the node itself (0 off the grid, where x and the masses are 0 too)
          const int gz = z0 - 1 + rz, gy = y0 - 1 + ry;
          if (gz >= 0 && gz < d.nz && gy >= 0 && gy < d.ny && q >= 0 && q < d.nx) {
            ld_rot<T, K>(b + (((long long)q * d.ny + gy) * d.nz + gz) * K, bv, rot);
          } else {
#pragma unroll
            for (int t = 0; t < K; ++t) bv[t] = (T)0;
          }
          ld_rot<T, K>(vc + bi * K, xv, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ax[t] = xv[t];
          ld_rot<T, K>(vm + bi * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ax[t] -= mxm * v[t];
          ld_rot<T, K>(vp + bi * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ax[t] -= mxp * v[t];
          ld_rot<T, K>(vc + (bi - C::IZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ax[t] -= mym * v[t];
          ld_rot<T, K>(vc + (bi + C::IZ) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ax[t] -= myp * v[t];
          ld_rot<T, K>(vc + (bi - 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) ax[t] -= mzm * v[t];
          ld_rot<T, K>(vc + (bi + 1) * K, v, rot);
#pragma unroll
          for (int t = 0; t < K; ++t) {
            ax[t] -= mzp * v[t];
            bv[t] -= ax[t];  // r0, k_mg_residual
          }
          st_rot<T, K>(up + (ry * C::RZ + rz) * K, bv, rot);
          if (own) {
#pragma unroll
            for (int t = 0; t < K; ++t) {
              rC[t] = bv[t];
              xC[t] = xv[t];
            }
            mC[0] = mxm; mC[1] = mxp; mC[2] = mym; mC[3] = myp; mC[4] = mzm; mC[5] = mzp;
          }
        };
        stage1(tz + 1, ty + 1, true);
        if (tid < C::NHALO) stage1(hz, hy, false);
      }
      ++uc;
      // r0 of plane q complete; input plane q-1 no longer read: its stage may refill
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      if (tid == 0 && j - 2 + C::NS < nin) issue(j - 2 + C::NS);
      // ---- stage 2: plane o = q - 1 (r0 planes o-1, o, o+1), k_mg_post2
      if (j >= 4 && inb) {
        const int x = q - 1;
        const long long n = ((long long)x * d.ny + y) * d.nz + z;
        const T* uo = reinterpret_cast<const T*>(base + C::O_U + ((uc - 2) % 3) * C::UPLP);
        const int ui = (ty + 1) * C::RZ + (tz + 1);
        T ar[K], v[K];
#pragma unroll
        for (int t = 0; t < K; ++t) {
          ar[t] = rB[t];
          ar[t] -= mB[0] * rA[t];
        }
#pragma unroll
        for (int t = 0; t < K; ++t) ar[t] -= mB[1] * rC[t];
        ld_rot<T, K>(uo + (ui - C::RZ) * K, v, rot);
#pragma unroll
        for (int t = 0; t < K; ++t) ar[t] -= mB[2] * v[t];
        ld_rot<T, K>(uo + (ui + C::RZ) * K, v, rot);
#pragma unroll
        for (int t = 0; t < K; ++t) ar[t] -= mB[3] * v[t];
        ld_rot<T, K>(uo + (ui - 1) * K, v, rot);
#pragma unroll
        for (int t = 0; t < K; ++t) ar[t] -= mB[4] * v[t];
        ld_rot<T, K>(uo + (ui + 1) * K, v, rot);
        T xo[K];
#pragma unroll
        for (int t = 0; t < K; ++t) {
          ar[t] -= mB[5] * v[t];
          xo[t] = xB[t];
          xo[t] += alpha * rB[t] + beta * ar[t];
        }
        st_rot<T, K>(xout + n * K, xo, rot);
      }
#pragma unroll
      for (int t = 0; t < K; ++t) {
        rA[t] = rB[t];
        rB[t] = rC[t];
        xB[t] = xC[t];
      }
#pragma unroll
      for (int e = 0; e < 6; ++e) mB[e] = mC[e];
    }
    ticket += nin;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      *err = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
}

// gamma = r~.z (tot, per RHS) into the CG state: beta = gamma / gamma_old.
// Called by every thread of the last block of the r.z reduction.
template <int K>
__device__ void rz_apply(const double (&tot)[K], RhsState* st, Control* ctl) {
  if (threadIdx.x < K) {
    RhsState& s = st[threadIdx.x];
    if (s.active) {
      const double g = tot[threadIdx.x];
      if (!(g > 0.0) || !isfinite(g)) {
        // M is SPD: r.Mr = 0 means r = 0; r.Mr < 0 means the FP32
        // preconditioner lost definiteness on a mode below its resolution
        // (reported as a stall, so "auto" continues in FP64); NaN/Inf is a
        // breakdown.
        s.active = 0;
        s.status = (g == 0.0) ? FS_OK : (isfinite(g) ? FS_STALLED : FS_NAN);
      } else if (s.fresh) {
        s.gamma = g;
        s.gamma_old = g;
        s.beta = 0.0;
        s.fresh = 0;
      } else {
        s.gamma_old = s.gamma;
        s.gamma = g;
        s.beta = g / s.gamma_old;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) refresh_done(st, ctl, K);
}

// ---- the fused smoothing passes with each node split over two threads ------------
// For 32-byte nodes (8 FP32 or 4 FP64 RHS) k_mg_pre_fused and k_mg_post_fused
// are latency-bound on the warps two 256-thread CTAs per SM give them.  Here
// the same tiles and shared-memory layout (SmoothTile) run 512 threads: thread
// 2v+h owns 16-byte chunk h of node v, so a quarter-warp reads 128 contiguous
// bytes (no bank conflicts, no rotation) and a warp stores whole sectors.  To
// stay within 64 registers, stage 2 reads the node's own b / x and masses
// from the input ring (the plane's stage is released after a second barrier,
// when stage 2 is done with it) instead of carrying them in registers.
template <typename T, int K>
struct SplitTile {
  using C = SmoothTile<T, K>;
  static constexpr int W = K >= 2 ? K / 2 : 1;    // values in one 16-byte chunk
  static constexpr int THREADS = 2 * C::TZ * C::TY;
  static constexpr bool OK = C::OK && C::B == 32;
};

template <typename T, int W>
__device__ __forceinline__ void ld16(const T* p, T (&v)[W]) {
  if constexpr (sizeof(T) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
  } else {
    const double2 t = *reinterpret_cast<const double2*>(p);
    v[0] = t.x; v[1] = t.y;
  }
}

template <typename T, int W>
__device__ __forceinline__ void st16(T* p, const T (&v)[W]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  }
}

// POST = false: k_mg_pre_fused's arithmetic (src = b; out1 = x2, out2 = r2).
// POST = true:  k_mg_post_fused's (src = x, b by loads; out1 = xout).  On the
// finest level b is the CG residual r~ and xout is z = M r~: with rz_partials
// set, the pass also forms gamma = r~.z (k_rz: per-block FP64 partials, the
// last block updates beta), so no separate pass re-reads r~ and z.
template <typename T, int K, bool POST>
__global__ void __launch_bounds__(SplitTile<T, K>::THREADS, 2)
    k_mg_smooth_split(Dims d, const __grid_constant__ CUtensorMap tm_s,
                      const __grid_constant__ CUtensorMap tm_ex,
                      const __grid_constant__ CUtensorMap tm_ey,
                      const __grid_constant__ CUtensorMap tm_ez, const T* __restrict__ b,
                      T* __restrict__ out1, T* __restrict__ out2, T c0, T cd, T cr,
                      const int* __restrict__ done, int* __restrict__ err,
                      double* __restrict__ rz_partials, RhsState* st, Control* ctl) {
  using C = SmoothTile<T, K>;
  constexpr int W = SplitTile<T, K>::W;
  if (*done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::O_BAR);
  const int tid = threadIdx.x;
  const int hf = tid & 1, v = tid >> 1;  // chunk, node of the tile
  const int tz = v % C::TZ, ty = v / C::TZ;
  int hz = 0, hy = 0;  // the halo-ring node of this thread pair (v < NHALO)
  if (v < 2 * C::RZ) {
    hz = v % C::RZ;
    hy = v < C::RZ ? 0 : C::RY - 1;
  } else if (v < C::NHALO) {
    const int k2 = v - 2 * C::RZ;
    hy = 1 + k2 / 2;
    hz = (k2 & 1) ? C::RZ - 1 : 0;
  }
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  int u = 0, u_end = 0;  // column-planes
  fs::march_range<int>(d, nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  int ticket = 0, uc = 0;
  bool failed = false, bad = false;
  double rzacc[W];
#pragma unroll
  for (int t = 0; t < W; ++t) rzacc[t] = 0.0;
  while (u < u_end && !failed) {
    const int col = u / d.nx;
    const int xa = u - col * d.nx;
    const int xb = min(d.nx, xa + (u_end - u));
    const int by = col / nbz, bz = col - by * nbz;
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nin = (xb - xa) + 4;  // input planes xa-2 .. xb+1
    auto issue = [&](int j) {
      const int s = (ticket + j) % C::NS;
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 2 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      smooth_tile_load<T, K>(slot, &tm_s, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_M0, &tm_ex, &bar[s], z0 - C::ZP, y0 - 2, x);
      tma_load_3d(slot + C::O_M0 + C::MBOXP, &tm_ey, &bar[s], z0 - C::ZP, y0 - 2, x);
      tma_load_3d(slot + C::O_M0 + 2 * C::MBOXP, &tm_ez, &bar[s], z0 - C::ZP, y0 - 2, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nin; ++j) issue(j);
    // own node, this thread's chunk: the stage-1 value (d1, or r0) of planes
    // q-2 (A), q-1 (B), q (C); r1 of planes q-1, q (pre); the -x mass of q-1, q
    T fA[W], fB[W], fC[W], r1B[W], r1C[W];
    T mxB = (T)0, mxC = (T)0;
    for (int j = 0; j < nin; ++j) {
      const int tk = ticket + j;
      const int s = tk % C::NS;
      const int q = xa - 3 + j;
      // post: b of this step's stage-1 nodes, loaded before the stage wait so
      // the two latencies overlap (0 off the grid)
      T bo[W], bh[W];
      if constexpr (POST) {
        auto load_b = [&](int rz, int ry, T(&f)[W]) {
          const int gz = z0 - 1 + rz, gy = y0 - 1 + ry;
          if (j >= 2 && gz >= 0 && gz < d.nz && gy >= 0 && gy < d.ny && q >= 0 && q < d.nx) {
            ld16<T, W>(b + (((long long)q * d.ny + gy) * d.nz + gz) * K + hf * W, f);
          } else {
#pragma unroll
            for (int t = 0; t < W; ++t) f[t] = (T)0;
          }
        };
        load_b(tz + 1, ty + 1, bo);
        if (v < C::NHALO) {
          load_b(hz, hy, bh);
        } else {
#pragma unroll
          for (int t = 0; t < W; ++t) bh[t] = (T)0;
        }
      }
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j < 2) continue;
      // ---- stage 1 on plane q (input planes q-1, q, q+1)
      const unsigned char* sm = base + ((tk - 2) % C::NS) * C::SLOT;
      const unsigned char* sc = base + ((tk - 1) % C::NS) * C::SLOT;
      const unsigned char* sp = base + s * C::SLOT;
      T* up = reinterpret_cast<T*>(base + C::O_U + (uc % 3) * C::UPLP);
      if (!bad) {
        const T* vm = reinterpret_cast<const T*>(sm) + hf * W;
        const T* vc = reinterpret_cast<const T*>(sc) + hf * W;
        const T* vp = reinterpret_cast<const T*>(sp) + hf * W;
        const T* exm = reinterpret_cast<const T*>(sm + C::O_M0);
        const T* exc = reinterpret_cast<const T*>(sc + C::O_M0);
        const T* eyc = reinterpret_cast<const T*>(sc + C::O_M0 + C::MBOXP);
        const T* ezc = reinterpret_cast<const T*>(sc + C::O_M0 + 2 * C::MBOXP);
        auto stage1 = [&](int rz, int ry, bool own, const T(&bb)[W]) {
          const int bi = (ry + 1) * C::IZ + (rz + 1);
          const int mi = (ry + 1) * C::WZ + (rz - 1 + C::ZP);
          const T mxm = exm[mi], mxp = exc[mi];
          const T mym = eyc[mi - C::WZ], myp = eyc[mi];
          const T mzm = ezc[mi - 1], mzp = ezc[mi];
          T cv[W], a[W], w[W];
          ld16<T, W>(vc + bi * K, cv);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] = cv[t];
          ld16<T, W>(vm + bi * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] -= mxm * w[t];
          ld16<T, W>(vp + bi * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] -= mxp * w[t];
          ld16<T, W>(vc + (bi - C::IZ) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] -= mym * w[t];
          ld16<T, W>(vc + (bi + C::IZ) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] -= myp * w[t];
          ld16<T, W>(vc + (bi - 1) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] -= mzm * w[t];
          ld16<T, W>(vc + (bi + 1) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) a[t] -= mzp * w[t];
          T f[W];
          if constexpr (POST) {
            // r0 = b - A~x (k_mg_residual)
#pragma unroll
            for (int t = 0; t < W; ++t) f[t] = bb[t] - a[t];
          } else {
#pragma unroll
            for (int t = 0; t < W; ++t) {
              const T xo = c0 * cv[t];          // k_mg_pre0
              const T rv = cv[t] - c0 * a[t];
              f[t] = cd * xo + cr * rv;         // k_mg_pre1: d1
              if (own) r1C[t] = rv;
            }
          }
          st16<T, W>(up + (ry * C::RZ + rz) * K + hf * W, f);
          if (own) {
#pragma unroll
            for (int t = 0; t < W; ++t) fC[t] = f[t];
            mxC = mxm;
          }
        };
        stage1(tz + 1, ty + 1, true, bo);
        if (v < C::NHALO) stage1(hz, hy, false, bh);
      }
      ++uc;
      // the plane-q values are complete
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      // ---- stage 2 on plane o = q - 1 (its input stage sm is still resident)
      if (j >= 4 && inb) {
        const int x = q - 1;
        const long long n = ((long long)x * d.ny + y) * d.nz + z;
        const T* uo = reinterpret_cast<const T*>(base + C::O_U + ((uc - 2) % 3) * C::UPLP) +
                      hf * W;
        const int ui = (ty + 1) * C::RZ + (tz + 1);
        const int bi = (ty + 2) * C::IZ + (tz + 2);
        const int mi = (ty + 2) * C::WZ + (tz + C::ZP);
        const T* exo = reinterpret_cast<const T*>(sm + C::O_M0);
        const T* eyo = reinterpret_cast<const T*>(sm + C::O_M0 + C::MBOXP);
        const T* ezo = reinterpret_cast<const T*>(sm + C::O_M0 + 2 * C::MBOXP);
        T a[K / 2], w[W], cv[W];
#pragma unroll
        for (int t = 0; t < W; ++t) {
          a[t] = fB[t];
          a[t] -= mxB * fA[t];
        }
        const T mxp = exo[mi];
#pragma unroll
        for (int t = 0; t < W; ++t) a[t] -= mxp * fC[t];
        ld16<T, W>(uo + (ui - C::RZ) * K, w);
        const T mym = eyo[mi - C::WZ];
#pragma unroll
        for (int t = 0; t < W; ++t) a[t] -= mym * w[t];
        ld16<T, W>(uo + (ui + C::RZ) * K, w);
        const T myp = eyo[mi];
#pragma unroll
        for (int t = 0; t < W; ++t) a[t] -= myp * w[t];
        ld16<T, W>(uo + (ui - 1) * K, w);
        const T mzm = ezo[mi - 1];
#pragma unroll
        for (int t = 0; t < W; ++t) a[t] -= mzm * w[t];
        ld16<T, W>(uo + (ui + 1) * K, w);
        const T mzp = ezo[mi];
        ld16<T, W>(reinterpret_cast<const T*>(sm) + bi * K + hf * W, cv);  // b or x at o
        T o1[W];
        if constexpr (POST) {
#pragma unroll
          for (int t = 0; t < W; ++t) {
            a[t] -= mzp * w[t];
            o1[t] = cv[t];
            o1[t] += c0 * fB[t] + cd * a[t];  // k_mg_post2: x + alpha r0 + beta A~r0
          }
          st16<T, W>(out1 + n * K + hf * W, o1);
          if (rz_partials) {  // r~.z: b was read one plane ago (an L2 hit; carrying
            T bo2[W];          // it in registers spilled and was slower)
            ld16<T, W>(b + n * K + hf * W, bo2);
#pragma unroll
            for (int t = 0; t < W; ++t) rzacc[t] += (double)bo2[t] * (double)o1[t];
          }
        } else {
          T o2[W];
#pragma unroll
          for (int t = 0; t < W; ++t) {
            a[t] -= mzp * w[t];
            o1[t] = c0 * cv[t];     // x1
            o1[t] += fB[t];         // x2 = x1 + d1
            o2[t] = r1B[t] - a[t];  // r2 = r1 - A~d1
          }
          st16<T, W>(out1 + n * K + hf * W, o1);
          st16<T, W>(out2 + n * K + hf * W, o2);
        }
      }
      // stage 2 done with plane q-1: its stage may refill
      __syncthreads();
      if (tid == 0 && j - 2 + C::NS < nin) issue(j - 2 + C::NS);
#pragma unroll
      for (int t = 0; t < W; ++t) {
        fA[t] = fB[t];
        fB[t] = fC[t];
        if constexpr (!POST) r1B[t] = r1C[t];
      }
      mxB = mxC;
    }
    ticket += nin;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      *err = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
  if constexpr (POST) {
    if (rz_partials) {
      // the d1 ring (written by threads only, never by TMA) is free now
      constexpr int NT = SplitTile<T, K>::THREADS;
      static_assert(NT * 8 <= 3 * C::UPLP, "reduction scratch exceeds the d1 ring");
      double* scr = reinterpret_cast<double*>(base + C::O_U);
      __syncthreads();
      double acc[K];
#pragma unroll
      for (int t = 0; t < K; ++t) acc[t] = (t / W == hf) ? rzacc[t % W] : 0.0;
      fs::block_partials_to<K, NT>(acc, rz_partials, scr);
      if (fs::last_block(&ctl->tickets[kTicketRz])) {
        double tot[K];
        fs::grid_total_to<K, NT>(rz_partials, gridDim.x, tot, scr);
        rz_apply<K>(tot, st, ctl);
      }
    }
  }
}

// ---- full-weighting restriction by x-march, fine planes staged by TMA ------------
//   b_c(I) = s_c(I) * sum_f P(f, I) sd_f(f) r(f)
// (k_mg_restrict's formula, trilinear weights per axis, the last fine node of
// an even-length axis weighted 1 towards the last coarse node).  A CTA owns a
// column of CZ x CY coarse nodes and marches its coarse planes I; the fine
// planes 2I-1, 2I, 2I+1 stream through a ring as TMA boxes (the residual with
// a one-node halo, 34 x 17 nodes, and sd from a 16-byte aligned start; out of
// range reads zero, which is a zero contribution).  Each thread (one 16-byte
// chunk of one coarse node) sums its 3 x 3 fine (y, z) neighbourhood per
// plane and carries two coarse planes in registers: a fine plane 2I adds to I,
// a plane 2I+1 adds to I and I+1, after which plane I is complete and stored.
// The residual is read once from DRAM (k_mg_restrict's gather read each fine
// node for up to 8 coarse threads from L1/L2); the sums run in another order,
// so results agree with k_mg_restrict to FP rounding.
template <typename T, int K>
struct RestrictTile {
  static constexpr int B = K * (int)sizeof(T);       // bytes per node
  static constexpr int NCH = B / 16;                 // 16-byte chunks per node
  static constexpr int W = 16 / (int)sizeof(T);      // values per chunk
  static constexpr int CZ = 16, CY = 8;              // coarse nodes of a column tile
  static constexpr int FZ = 2 * CZ + 2;              // residual box: z from 2*Z0 - 1
  static constexpr int FY = 2 * CY + 1;              //               y from 2*Y0 - 1
  static constexpr int ZP = 16 / (int)sizeof(T);     // sd box: z from 2*Z0 - ZP
  static constexpr int SZ = 2 * CZ + 2 * ZP;
  static constexpr int NS = 4;                       // fine planes in the ring
  static constexpr int VBOX = FZ * FY * B;
  static constexpr int SBOX = SZ * FY * (int)sizeof(T);
  static constexpr int O_S = (VBOX + 127) / 128 * 128;
  static constexpr int SLOT = O_S + (SBOX + 127) / 128 * 128;
  static constexpr int O_BAR = NS * SLOT;
  static constexpr size_t SMEM = (size_t)O_BAR + NS * 8 + 128;
  static constexpr int THREADS = CZ * CY * (NCH > 0 ? NCH : 1);
  static constexpr uint32_t TX = (uint32_t)(VBOX + SBOX);
  static constexpr bool OK = (B == 16 || B == 32);
};

template <typename T, int K>
__global__ void __launch_bounds__(RestrictTile<T, K>::THREADS, 2)
    k_mg_restrict_tma(Dims f, Dims c, const __grid_constant__ CUtensorMap tm_r,
                      const __grid_constant__ CUtensorMap tm_sd, const T* __restrict__ sc,
                      T* __restrict__ bc, const int* __restrict__ done,
                      int* __restrict__ err) {
  using R = RestrictTile<T, K>;
  constexpr int W = R::W;
  if (*done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + R::O_BAR);
  const int tid = threadIdx.x;
  const int h = tid % R::NCH, v = tid / R::NCH;
  const int cz = v % R::CZ, cy = v / R::CZ;
  const int ncz = (c.nz + R::CZ - 1) / R::CZ, ncy = (c.ny + R::CY - 1) / R::CY;
  int u = 0, u_end = 0;
  fs::march_range<int>(c, ncz * ncy, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < R::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  int ticket = 0;
  bool failed = false;
  while (u < u_end && !failed) {
    const int col = u / c.nx;
    const int Ia = u - col * c.nx;
    const int Ib = min(c.nx, Ia + (u_end - u));
    const int by = col / ncz, bz = col - by * ncz;
    const int Z0 = bz * R::CZ, Y0 = by * R::CY;
    const int Kc = Z0 + cz, J = Y0 + cy;
    const bool inb = Kc < c.nz && J < c.ny;
    const int nin = 2 * (Ib - Ia) + 1;  // fine planes 2Ia-1 .. 2Ib-1
    auto issue = [&](int j) {
      const int s = (ticket + j) % R::NS;
      unsigned char* slot = base + s * R::SLOT;
      const int x = 2 * Ia - 1 + j;
      fs::mbar_arrive_expect_tx(&bar[s], R::TX);
      fs::tma_load_4d(slot, &tm_r, &bar[s], 0, 2 * Z0 - 1, 2 * Y0 - 1, x);
      tma_load_3d(slot + R::O_S, &tm_sd, &bar[s], 2 * Z0 - R::ZP, 2 * Y0 - 1, x);
    };
    if (tid == 0)
      for (int j = 0; j < R::NS && j < nin; ++j) issue(j);
    // weight of the fine node 2I+1 towards I on each axis: 1/2, or 1 when I
    // is the last coarse node (no I+1 to share it with)
    const T wz1 = (Kc + 1 < c.nz) ? (T)0.5 : (T)1;
    const T wy1 = (J + 1 < c.ny) ? (T)0.5 : (T)1;
    T accI[W], accN[W];
#pragma unroll
    for (int t = 0; t < W; ++t) {
      accI[t] = (T)0;
      accN[t] = (T)0;
    }
    bool bad = false;
    for (int j = 0; j < nin; ++j) {
      const int tk = ticket + j;
      const int s = tk % R::NS;
      const int x = 2 * Ia - 1 + j;
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / R::NS) & 1), kWaitBudget);
      T part[W];
#pragma unroll
      for (int t = 0; t < W; ++t) part[t] = (T)0;
      if (inb && !bad) {
        const T* vb = reinterpret_cast<const T*>(base + s * R::SLOT) + h * W;
        const T* sdb = reinterpret_cast<const T*>(base + s * R::SLOT + R::O_S);
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
          const T wy = dy == 1 ? (T)1 : (dy == 0 ? (T)0.5 : wy1);
          const int yi = 2 * cy + dy;
#pragma unroll
          for (int dz = 0; dz < 3; ++dz) {
            const T wz = dz == 1 ? (T)1 : (dz == 0 ? (T)0.5 : wz1);
            const int zi = 2 * cz + dz;
            const T w = (wy * wz) * sdb[yi * R::SZ + zi + R::ZP - 1];
            if (w != (T)0) {
              T val[W];
              ld16<T, W>(vb + (yi * R::FZ + zi) * K, val);
#pragma unroll
              for (int t = 0; t < W; ++t) part[t] += w * val[t];
            }
          }
        }
      }
      if ((x & 1) == 0) {  // x = 2I: weight 1 towards I
#pragma unroll
        for (int t = 0; t < W; ++t) accI[t] += part[t];
      } else {  // x = 2I+1: towards I and I+1; plane I is then complete
        const int I = (x - 1) >> 1;
        const T wx1 = (I + 1 < c.nx) ? (T)0.5 : (T)1;
#pragma unroll
        for (int t = 0; t < W; ++t) {
          accI[t] += wx1 * part[t];
          accN[t] += (T)0.5 * part[t];
        }
        if (I >= Ia && inb && !bad) {
          const long long n = ((long long)I * c.ny + J) * c.nz + Kc;
          const T scale = sc[n];
          T o[W];
#pragma unroll
          for (int t = 0; t < W; ++t) o[t] = scale != (T)0 ? accI[t] * scale : (T)0;
          st16<T, W>(bc + n * K + h * W, o);
        }
#pragma unroll
        for (int t = 0; t < W; ++t) {
          accI[t] = accN[t];
          accN[t] = (T)0;
        }
      }
      // every thread is done with this plane's slot: it may refill
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      if (tid == 0 && j + R::NS < nin) issue(j + R::NS);
    }
    ticket += nin;
    u += (Ib - Ia);
  }
  if (failed) {
    if (tid == 0) {
      *err = 1;
      for (int s = 0; s < R::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
}

// ---- K1 with each node split over two threads (stencil kind 4) -------------------
// k_stencil_tma_m's tiles, ring and single barrier per plane, for 32-byte
// nodes: 512 threads, thread 2v+h owning 16-byte chunk h of node v (chunk reads
// of a quarter-warp are 128 contiguous bytes, q stores cover whole sectors).
// One of the candidates the stencil autotuner times.
template <typename T, int K>
struct TmaTileSplit {
  using M = TmaTileM<T, K>;
  static constexpr int W = K >= 2 ? K / 2 : 1;
  static constexpr int THREADS = 2 * M::TZ * M::TY;
  static constexpr bool OK = M::OK && M::B == 32;
};

template <typename T, int K>
__global__ void __launch_bounds__(TmaTileSplit<T, K>::THREADS, 2)
    k_stencil_split(Dims d, const __grid_constant__ CUtensorMap tm_p,
                    const __grid_constant__ CUtensorMap tm_ex,
                    const __grid_constant__ CUtensorMap tm_ey,
                    const __grid_constant__ CUtensorMap tm_ez, T* __restrict__ q,
                    double* __restrict__ partials, RhsState* st, Control* ctl) {
  using C = TmaTileM<T, K>;
  constexpr int W = TmaTileSplit<T, K>::W;
  if (ctl->all_done) return;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + C::NS * C::SLOT);
  const int tid = threadIdx.x;
  const int hf = tid & 1, v = tid >> 1;
  const int tz = v % C::TZ, ty = v / C::TZ;
  const int nbz = (d.nz + C::TZ - 1) / C::TZ, nby = (d.ny + C::TY - 1) / C::TY;
  int u = 0, u_end = 0;  // column-planes
  fs::march_range<int>(d, nbz * nby, u, u_end);
  if (tid == 0) {
    for (int s = 0; s < C::NS; ++s) fs::mbar_init(&bar[s], 1);
    fs::fence_mbar_init();
  }
  __syncthreads();
  double acc[W];
#pragma unroll
  for (int t = 0; t < W; ++t) acc[t] = 0.0;
  const int cpos = (ty + 1) * C::HZ + (tz + 1);
  int ticket = 0;
  bool failed = false, bad = false;
  while (u < u_end && !failed) {
    const int col = u / d.nx;
    const int xa = u - col * d.nx;
    const int xb = min(d.nx, xa + (u_end - u));
    const int by = col / nbz, bz = col - by * nbz;
    const int z0 = bz * C::TZ, y0 = by * C::TY;
    const int z = z0 + tz, y = y0 + ty;
    const bool inb = z < d.nz && y < d.ny;
    const int nplanes = (xb - xa) + 2;  // planes xa-1 .. xb
    auto issue = [&](int j) {
      const int s = (ticket + j) % C::NS;
      unsigned char* slot = base + s * C::SLOT;
      const int x = xa - 1 + j;
      fs::mbar_arrive_expect_tx(&bar[s], C::TX);
      fs::tma_load_4d(slot, &tm_p, &bar[s], 0, z0 - 1, y0 - 1, x);
      tma_load_3d(slot + C::O_EX, &tm_ex, &bar[s], z0, y0, x);
      tma_load_3d(slot + C::O_EY, &tm_ey, &bar[s], z0, y0 - 1, x);
      tma_load_3d(slot + C::O_EZ, &tm_ez, &bar[s], z0 - C::ZP, y0, x);
    };
    if (tid == 0)
      for (int j = 0; j < C::NS && j < nplanes; ++j) issue(j);
    for (int j = 0; j < nplanes; ++j) {
      const int tk = ticket + j;
      const int s = tk % C::NS;
      bad |= !fs::mbar_wait_bounded(&bar[s], (uint32_t)((tk / C::NS) & 1), kWaitBudget);
      if (j >= 2) {
        if (inb && !bad) {
          const int x = xa - 2 + j;
          const long long n = ((long long)x * d.ny + y) * d.nz + z;
          const unsigned char* sm = base + ((tk - 2) % C::NS) * C::SLOT;  // plane x-1
          const unsigned char* sc = base + ((tk - 1) % C::NS) * C::SLOT;  // plane x
          const unsigned char* sp = base + s * C::SLOT;                   // plane x+1
          const T* pm = reinterpret_cast<const T*>(sm) + hf * W;
          const T* pc = reinterpret_cast<const T*>(sc) + hf * W;
          const T* pp = reinterpret_cast<const T*>(sp) + hf * W;
          const T* exm = reinterpret_cast<const T*>(sm + C::O_EX);
          const T* exc = reinterpret_cast<const T*>(sc + C::O_EX);
          const T* eyc = reinterpret_cast<const T*>(sc + C::O_EY);
          const T* ezc = reinterpret_cast<const T*>(sc + C::O_EZ);
          const T mxm = exm[ty * C::TZ + tz], mxp = exc[ty * C::TZ + tz];
          const T mym = eyc[ty * C::TZ + tz], myp = eyc[(ty + 1) * C::TZ + tz];
          const T mzm = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP - 1];
          const T mzp = ezc[ty * (C::TZ + C::ZP) + tz + C::ZP];
          T c[W], w[W], qv[W];
          ld16<T, W>(pc + cpos * K, c);
#pragma unroll
          for (int t = 0; t < W; ++t) qv[t] = c[t];
          ld16<T, W>(pm + cpos * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) qv[t] -= mxm * w[t];
          ld16<T, W>(pp + cpos * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) qv[t] -= mxp * w[t];
          ld16<T, W>(pc + (cpos - C::HZ) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) qv[t] -= mym * w[t];
          ld16<T, W>(pc + (cpos + C::HZ) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) qv[t] -= myp * w[t];
          ld16<T, W>(pc + (cpos - 1) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) qv[t] -= mzm * w[t];
          ld16<T, W>(pc + (cpos + 1) * K, w);
#pragma unroll
          for (int t = 0; t < W; ++t) {
            qv[t] -= mzp * w[t];
            acc[t] += (double)c[t] * (double)qv[t];
          }
          st16<T, W>(q + n * K + hf * W, qv);
        }
        // plane j-2 no longer read: its stage may refill
        if (__syncthreads_or(bad)) {
          failed = true;
          break;
        }
        if (tid == 0 && j - 2 + C::NS < nplanes) issue(j - 2 + C::NS);
      }
    }
    ticket += nplanes;
    u += (xb - xa);
  }
  if (failed) {
    if (tid == 0) {
      ctl->error = 1;
      for (int s = 0; s < C::NS; ++s) (void)fs::mbar_wait_bounded(&bar[s], 0, kWaitBudget / 8);
    }
    __syncthreads();
  }
  double full[K];  // this thread's chunk in RHS order, 0 for the other half
#pragma unroll
  for (int t = 0; t < K; ++t) full[t] = (t / W == hf) ? acc[t % W] : 0.0;
  finish_pq<T, K, TmaTileSplit<T, K>::THREADS>(full, partials, st, ctl);
}

// ---- preconditioned CG: gamma = r~.z, beta = gamma / gamma_old ------------------
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_rz(Dims d, const T* __restrict__ r, const T* __restrict__ z,
         double* __restrict__ partials, RhsState* st, Control* ctl) {
  if (ctl->all_done) return;
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T rv[K], zv[K];
    fs::ldv_ro<T, K, true>(r, n, rv);
    fs::ldv_ro<T, K, true>(z, n, zv);
#pragma unroll
    for (int t = 0; t < K; ++t) acc[t] += (double)rv[t] * (double)zv[t];
  }
  fs::block_partials<K>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketRz])) {
    double tot[K];
    fs::grid_total<K>(partials, gridDim.x, tot);
    rz_apply<K>(tot, st, ctl);
  }
}

// ---- flexible CG (nonlinear preconditioner): gamma = r~.z and
// beta = -(z . A~p_old) / (p_old . A~p_old), the A~-orthogonalisation of the
// new direction against the previous one (FCG with one stored direction).
// q still holds A~p_old from this iteration's stencil, pq its p.q.
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_rz_flex(Dims d, const T* __restrict__ r, const T* __restrict__ z,
              const T* __restrict__ q, double* __restrict__ partials, RhsState* st,
              Control* ctl) {
  if (ctl->all_done) return;
  double acc[2 * K];
#pragma unroll
  for (int t = 0; t < 2 * K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T rv[K], zv[K], qv[K];
    fs::ldv_ro<T, K, true>(r, n, rv);
    fs::ldv_ro<T, K, true>(z, n, zv);
    fs::ldv_ro<T, K, true>(q, n, qv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      acc[t] += (double)rv[t] * (double)zv[t];
      acc[K + t] += (double)zv[t] * (double)qv[t];
    }
  }
  fs::block_partials<2 * K>(acc, partials);
  if (fs::last_block(&ctl->tickets[kTicketRz])) {
    double tot[2 * K];
    fs::grid_total<2 * K>(partials, gridDim.x, tot);
    if (threadIdx.x < K) {
      RhsState& s = st[threadIdx.x];
      if (s.active) {
        const double g = tot[threadIdx.x], zq = tot[K + threadIdx.x];
        if (!isfinite(g) || !isfinite(zq)) {
          s.active = 0;
          s.status = FS_NAN;
        } else if (s.fresh || !(s.pq > 0.0)) {
          s.gamma = g;
          s.gamma_old = g;
          s.beta = 0.0;
          s.fresh = 0;
        } else {
          s.gamma_old = s.gamma;
          s.gamma = g;
          s.beta = -zq / s.pq;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) refresh_done(st, ctl, K);
  }
}

// ---- fallback for rows narrower than 16 B (float k <= 2, double k = 1) -----
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_pnew(Dims d, const T* __restrict__ r, const T* __restrict__ pold,
           T* __restrict__ pnew, RhsState* st, Control* ctl) {
  if (ctl->all_done) return;
  __shared__ T beta[K];
  __shared__ int act[K];
  if (threadIdx.x < K) {
    beta[threadIdx.x] = (T)st[threadIdx.x].beta;
    act[threadIdx.x] = st[threadIdx.x].active;
  }
  __syncthreads();
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    T rv[K], pv[K];
    fs::ldv_ro<T, K, true>(r, n, rv);
    fs::ldv_ro<T, K, true>(pold, n, pv);
#pragma unroll
    for (int t = 0; t < K; ++t) pv[t] = act[t] ? rv[t] + beta[t] * pv[t] : pv[t];
    fs::stv<T, K, true>(pnew, n, pv);
  }
}

template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock, fs::mg_min_blocks<T, K>())
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
    if (d.per) {  // periodic plans (cached-load kernel only): wrap edges
      fs::edge6(d, ex, ey, ez, n, i, j, k, [&](bool ok, T m, long long nb) {
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
    fs::stv<T, K>(q, n, qv);
#pragma unroll
    for (int t = 0; t < K; ++t) acc[t] += (double)pc[t] * (double)qv[t];
  }
  finish_pq<T, K, fs::kBlock>(acc, partials, st, ctl);
}

// ---- K2: x~ += alpha p, r~ -= alpha q, r~.r~ --------------------------------------
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
    fs::ldv_ro<T, K, true>(p, n, pv);
    fs::ldv_ro<T, K, true>(q, n, qv);
    fs::ldv<T, K, true>(x, n, xv);
    fs::ldv<T, K, true>(r, n, rv);
#pragma unroll
    for (int t = 0; t < K; ++t) {
      xv[t] += alpha[t] * pv[t];
      rv[t] -= alpha[t] * qv[t];
      acc[t] += (double)rv[t] * (double)rv[t];
    }
    fs::stv<T, K, true>(x, n, xv);
    fs::stv<T, K, true>(r, n, rv);
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
          s.rr = g;
          if (!ctl->precond) {
            s.gamma_old = s.gamma;
            s.gamma = g;
            s.beta = g / s.gamma_old;
          }
          const double rn = sqrt(g);
          // Reliable update: to verify convergence, at the cap, and in mixed
          // mode after a 1/delta drop or every kRefreshEvery iterations (so
          // a stagnating low-precision recurrence is noticed).  In mixed mode
          // the convergence check may wait for the other RHS (ru = 3, see
          // refresh_done); FP64 solves check at once, as the reference does.
          if (s.iters >= ctl->maxiter ||
              (ctl->delta > 0.0 &&
               (rn < ctl->delta * s.rmax || s.iters % kRefreshEvery == 0))) {
            s.ru = 1;
          } else if (rn < ctl->tol * s.bnorm) {
            if (ctl->delta <= 0.0) {
              s.ru = 1;
            } else if (s.ru == 0) {
              s.ru = 3;
              s.cand = s.iters;
            }
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) refresh_done(st, ctl, K);
  }
}

// ---- K3a/K3b: reliable update ---------------------------------------------------
// K3a folds the correction accumulated since the last update into the FP64
// solution (phi += s x~, x~ = 0) for the flagged right-hand sides; K3b then
// recomputes their TRUE residual r = f - L phi with the FP64 masses, replaces
// the recurrence residual with it and decides convergence on it.  K3a (and
// k_finalize) stream the node's values one thread per FP64 chunk
// (fs::Chunks): 0.32 -> 0.26 ms per fold at 256x256x128 with 8 RHS.  K3b
// (and k_init) gather six neighbours and keep one thread per node: split
// into chunks they were slower (k_reliable 0.63 -> 0.80 ms, k_init 0.64 ->
// 0.96 ms; the masses, labels and index arithmetic repeat per chunk).  They
// move the FP64 solution with 256-bit accesses instead (two per 64-byte
// node): 0.4 ms less per extraction.
template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_fold(Dims d, const double* __restrict__ s64, double* __restrict__ phi,
           T* __restrict__ x, RhsState* st, Control* ctl) {
  if (!ctl->any_ru) return;
  using CH = fs::Chunks<K>;
  constexpr int W = CH::W, NCH = CH::NCH;
  const int h = threadIdx.x % NCH;
  __shared__ int ru[K];
  if (threadIdx.x < K) ru[threadIdx.x] = st[threadIdx.x].ru;
  __syncthreads();
  const long long total = d.N * NCH;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long n = g / NCH;
    const double s = s64[n];
    if (s == 0.0) continue;  // x~ is 0 off the free nodes
    const long long o = n * K + h * W;
    T xv[W];
    double ph[W];
    fs::ldw<T, W>(x + o, xv);
    fs::ldw<double, W>(phi + o, ph);
#pragma unroll
    for (int t = 0; t < W; ++t)
      if (ru[h * W + t]) {
        ph[t] += (double)xv[t] * s;
        xv[t] = (T)0;
      }
    fs::stw<double, W>(phi + o, ph);
    fs::stw<T, W>(x + o, xv);
  }
}

template <typename T, int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_reliable(Dims d, const double* __restrict__ mx,
               const double* __restrict__ my, const double* __restrict__ mz,
               const double* __restrict__ dgn,
               const double* __restrict__ s64, const double* __restrict__ phi,
               const double* __restrict__ f, T* __restrict__ r,
               double* __restrict__ partials, RhsState* st, Control* ctl) {
  if (!ctl->any_ru) return;
  __shared__ int ru[K];
  if (threadIdx.x < K) ru[threadIdx.x] = st[threadIdx.x].ru;
  __syncthreads();
  double acc[K];
#pragma unroll
  for (int t = 0; t < K; ++t) acc[t] = 0.0;
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    const double sc = s64[n];
    if (sc == 0.0) continue;  // only free nodes carry a residual
    int i, j, k;
    fs::node_ijk(d, n, i, j, k);
    double c[K], res[K];
    fs::ldv_ro<double, K, true>(phi, n, c);
    if (f) {
      fs::ldv_ro<double, K>(f, n, res);
    } else {
#pragma unroll
      for (int t = 0; t < K; ++t) res[t] = 0.0;
    }
    auto edge = [&](bool ok, double m, long long nb) {
      if (!ok || m == 0.0) return;
      double v[K];
      fs::ldv_ro<double, K, true>(phi, nb, v);
#pragma unroll
      for (int t = 0; t < K; ++t) res[t] -= m * (c[t] - v[t]);
    };
    edge6(d, mx, my, mz, n, i, j, k, edge);
    if (dgn) {
      const double dd = dgn[n];
#pragma unroll
      for (int t = 0; t < K; ++t) res[t] -= dd * c[t];
    }
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
        const bool own = s.ru == 1 || s.ru == 3;
        s.nru += 1;
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
          // Progress is judged on the updates this RHS asked for; one taken
          // along with another RHS neither counts as a stall nor moves the
          // reference point.
          if (own) {
            if (rn < 0.5 * s.best) {
              s.best = rn;
              s.nstall = 0;
            } else {
              s.nstall += 1;
            }
          }
          if (ctl->delta > 0.0 && s.nstall >= kStallUpdates) {
            // Low-precision iterations no longer reduce the FP64 residual
            // (a mode below FP32 resolution): stop and report it.
            s.active = 0;
            s.status = FS_STALLED;
          } else {
            s.rr = g;
            if (!ctl->precond) {
              s.gamma = g;
              s.beta = g / s.gamma_old;
            }
            s.rmax = rn;
            // flexible CG keeps one previous direction; after the residual
            // is replaced, restart from the preconditioned residual
            if (ctl->flexible) s.fresh = 1;
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) refresh_done(st, ctl, K);
  }
}

// ---- after the loop: fold what is pending, zero RHS with b == 0 ------------------
template <typename T, int K>
__global__ void k_finalize(Dims d, const uint8_t* __restrict__ label,
                           const double* __restrict__ s64,
                           double* __restrict__ phi, T* __restrict__ x,
                           RhsState* st, Control* ctl) {
  using CH = fs::Chunks<K>;
  constexpr int W = CH::W, NCH = CH::NCH;
  const int h = threadIdx.x % NCH;
  __shared__ int zero[K];
  if (threadIdx.x < K) zero[threadIdx.x] = st[threadIdx.x].zero;
  __syncthreads();
  const long long total = d.N * NCH;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long n = g / NCH;
    if (label[n] != FS_LABEL_FREE) continue;
    const double s = s64[n];
    const long long o = n * K + h * W;
    T xv[W];
    double ph[W];
    fs::ldw<T, W>(x + o, xv);
    fs::ldw<double, W>(phi + o, ph);
#pragma unroll
    for (int t = 0; t < W; ++t) {
      ph[t] += (double)xv[t] * s;  // correction since the last fold
      xv[t] = (T)0;
      if (zero[h * W + t]) ph[t] = 0.0;
    }
    fs::stw<double, W>(phi + o, ph);
    fs::stw<T, W>(x + o, xv);
  }
  if (fs::last_block(&ctl->tickets[kTicketFin])) {
    if (threadIdx.x < K) st[threadIdx.x].zero = 0;
  }
}

size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

// ---- multigrid hierarchy ---------------------------------------------------------
constexpr int kMaxLevels = 12;
// Multigrid and stencil options of one plan (fs_mg_params, copied at
// creation; nothing process-wide).  Defaults from sweeps on the
// 256x256x128 8-terminal extraction: degree-2 smoothing on [0.3, 2] and a
// degree-32 Chebyshev solve on [0.06, 2] on a coarsest level of at most 4096
// nodes (21 iterations, 39.4 ms; [0.03, 2]: 22 iterations, 41.0 ms; degree 16
// or 24, [0.1, 2], 512 or 32768 coarsest nodes, smoothing on [0.25, 2] or
// [0.35, 2]: no faster).
struct MgParams {
  int smooth_deg = 2;          // Chebyshev degree, pre and post
  double smooth_lo = 0.3;      // smoothing interval [lo, 2] of A~
  int coarse_deg = 32;         // coarsest-level Chebyshev degree
  double coarse_lo = 0.06;
  long long coarsest_nodes = 4096;
  int stencil_kind = -1;       // CG stencil 0..5; -1: FS_STENCIL, else autotuned
  // over-correction of the aggregation hierarchy's coarse corrections:
  // measured on the copper/oxide EQS step at 192x192x96, 119 iterations at 1,
  // 71 at 1.4, 67 at 1.7, 72 at 2.0 (early transient steps, FP64, 1e-10)
  double agg_alpha = 1.7;
};

// Options from the caller's struct (NULL: defaults); false if out of range.
bool mg_params_from(const fs_mg_params* o, MgParams* out) {
  MgParams m;
  if (o) {
    if (o->smooth_deg < 1 || o->smooth_deg > 16 || o->coarse_deg < 1 || o->coarse_deg > 64 ||
        !(o->smooth_lo > 0.0 && o->smooth_lo < 2.0) ||
        !(o->coarse_lo > 0.0 && o->coarse_lo < 2.0) || o->coarsest_nodes < 8 ||
        o->stencil_kind < -1 || o->stencil_kind > 7 ||
        !(o->agg_alpha > 0.0 && o->agg_alpha < 2.0))
      return false;
    m.smooth_deg = o->smooth_deg;
    m.smooth_lo = o->smooth_lo;
    m.coarse_deg = o->coarse_deg;
    m.coarse_lo = o->coarse_lo;
    m.coarsest_nodes = o->coarsest_nodes;
    m.stencil_kind = o->stencil_kind;
    m.agg_alpha = o->agg_alpha;
  }
  *out = m;
  return true;
}

struct MgLevel {
  Dims d;
  // level >= 1: original-scale FP64 masses, labels, scale (setup only)
  double *m64[3], *s64, *d64;
  uint8_t *label_in, *label;
  void *em[3];       // equilibrated masses (T); level 0 uses the plan's
  void *s, *sd;      // diag^-1/2, diag^1/2 (T), 0 on fixed nodes
  void *x[2], *b, *dv, *res;  // K-interleaved vectors (T); level 0 b = r~
  size_t off_d64, off_m64[3], off_s64, off_label_in, off_label, off_em[3], off_s, off_sd,
      off_x[2], off_b, off_dv, off_res;
};

// Level sizes: every axis of at least 5 nodes is halved (n -> (n + 1) / 2),
// shorter axes are kept (semi-coarsening, e.g. the two node planes of a 2-D
// cross-section), until the level holds at most `coarsest` nodes or no axis
// can be coarsened.
int mg_dims(const Dims& fine, long long coarsest, Dims* out) {
  int nl = 0;
  Dims d = fine;
  out[nl++] = d;
  auto half = [](int n) { return n >= 5 ? (n + 1) / 2 : n; };
  while (nl < kMaxLevels && d.N > coarsest) {
    const int nx = half(d.nx), ny = half(d.ny), nz = half(d.nz);
    if (nx == d.nx && ny == d.ny && nz == d.nz) break;
    d = fs::make_dims(nx, ny, nz, fine.per);  // a periodic axis stays periodic
    out[nl++] = d;
  }
  return nl;
}

// Chebyshev step coefficients (cd, cr) for degree `deg` on [lo, hi].
void cheb_coeffs(int deg, double lo, double hi, double* cd, double* cr) {
  const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo);
  const double sigma = theta / delta;
  double rho_old = 1.0 / sigma;
  cd[0] = 0.0;
  cr[0] = 1.0 / theta;
  for (int k = 1; k < deg; ++k) {
    const double rho = 1.0 / (2.0 * sigma - rho_old);
    cd[k] = rho * rho_old;
    cr[k] = 2.0 * rho / delta;
    rho_old = rho;
  }
}

struct Layout {
  size_t label, s64, ex, ey, ez, x, r, p0, p1, q, partials, st, ctl, total;
  int nlev;
  MgLevel lev[kMaxLevels];
};

constexpr int kMaxBlocks = 4096;

// Upper bound on the stencil grid over every tile shape (TY >= 2, XC = 32).
long long fused_blocks(const Dims& d) {
  return (long long)((d.nz + 31) / 32) * ((d.ny + 1) / 2) * ((d.nx + 31) / 32);
}

long long max_blocks(const Dims& d) {
  long long f = fused_blocks(d);
  return f > kMaxBlocks ? f : kMaxBlocks;
}

Layout make_layout(const Dims& d, int nrhs, int precision, int precond,
                   long long coarsest_nodes) {
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
  L.p0 = o; o = align_up(o + N * nrhs * tb);
  L.p1 = o; o = align_up(o + N * nrhs * tb);
  L.q = o; o = align_up(o + N * nrhs * tb);
  L.partials = o;
  o = align_up(o + (size_t)max_blocks(d) * 2 * fs::kMaxRhs * 8);
  L.st = o; o = align_up(o + sizeof(RhsState) * fs::kMaxRhs);
  L.ctl = o; o = align_up(o + sizeof(Control));
  L.nlev = 0;
  if (precond == FS_PRECOND_MG || precond == FS_PRECOND_MG_AGG) {
    Dims dl[kMaxLevels];
    L.nlev = mg_dims(d, coarsest_nodes, dl);
    for (int l = 0; l < L.nlev; ++l) {
      MgLevel& m = L.lev[l];
      m = MgLevel{};
      m.d = dl[l];
      const size_t n = (size_t)dl[l].N;
      if (l > 0) {
        for (int a = 0; a < 3; ++a) { m.off_m64[a] = o; o = align_up(o + n * 8); }
        m.off_d64 = o; o = align_up(o + n * 8);
        m.off_s64 = o; o = align_up(o + n * 8);
        m.off_label_in = o; o = align_up(o + n);
        m.off_label = o; o = align_up(o + n);
        for (int a = 0; a < 3; ++a) { m.off_em[a] = o; o = align_up(o + n * tb); }
        m.off_b = o; o = align_up(o + n * nrhs * tb);
      }
      m.off_s = o; o = align_up(o + n * tb);
      m.off_sd = o; o = align_up(o + n * tb);
      for (int a = 0; a < 2; ++a) { m.off_x[a] = o; o = align_up(o + n * nrhs * tb); }
      m.off_dv = o; o = align_up(o + n * nrhs * tb);
      m.off_res = o; o = align_up(o + n * nrhs * tb);
    }
  }
  L.total = o;
  return L;
}

bool valid_nrhs(int k) { return k == 1 || k == 2 || k == 4 || k == 8 || k == 16; }

}  // namespace

// Page-locked host slots for a plan's completion flag and per-RHS stats,
// pinned once per process and reused: creating and destroying a plan per
// extraction then makes no cudaMallocHost / cudaFreeHost call (the latter
// synchronises the whole device).  Slots are kept until the process exits.
struct HostSlot {
  int flag;
  int pad[3];
  RhsState st[fs::kMaxRhs];
};

namespace {
std::mutex g_slot_mu;
std::vector<HostSlot*> g_slot_free;

cudaError_t host_slot_get(HostSlot** out) {
  {
    std::lock_guard<std::mutex> lk(g_slot_mu);
    if (!g_slot_free.empty()) {
      *out = g_slot_free.back();
      g_slot_free.pop_back();
      return cudaSuccess;
    }
  }
  return cudaMallocHost((void**)out, sizeof(HostSlot));
}

void host_slot_put(HostSlot* slot) {
  std::lock_guard<std::mutex> lk(g_slot_mu);
  g_slot_free.push_back(slot);
}
}  // namespace

struct fs_pcg_plan {
  Dims d;
  Dims dm;                 // d with the x-marching assignment of the CG stencil
  int nrhs, precision, precond;
  int agg;                 // multigrid levels by aggregation (Galerkin coarse operators)
  int nlev;
  MgLevel lev[kMaxLevels];
  void* z;                 // preconditioned residual (level-0 V-cycle output)
  int g_rz;
  int rz_request;          // set while the CG preconditioner runs: the finest
                           // post-smoothing may form r~.z itself
  int rz_fused;            // the last V-cycle did (no k_rz launch needed)
  long long launches_per_iter;
  MgParams mg;
  const double *mx, *my, *mz;
  const double* dg;        // node diagonal term (NULL: pure Laplacian)
  double* phi;
  const double* f;
  uint8_t* label;
  double* s64;
  void *ex, *ey, *ez, *x, *r, *p[2], *q;
  double* partials;
  RhsState* st;
  Control* ctl;
  int g_init, g_apply, g_pnew, g_update, g_rel, g_fin, g_fold;
  int use_tma;
  CUtensorMap tm_p[2];
  CUtensorMap tm_m[3];     // ex, ey, ez tiles of the mass-staging stencil
  CUtensorMap tm_q;        // q tiles of the TMA-store stencil
  CUtensorMap tm_z;        // z (r without a preconditioner) tiles of the fused stencil
  int zmap_ok = 0;         // tm_z encoded (kind 5 available)
  int stencil_kind;        // 0: cached loads, 1: TMA p, 2: TMA p + masses,
                           // 3: as 2 with q written by TMA stores
  int autotune = 0;        // time kinds 2, 3, 0, 4, 5 at creation and keep the fastest
  float tune_ms[8] = {-1.f, -1.f, -1.f, -1.f, -1.f, -1.f, -1.f, -1.f};  // ms by kind (-1: untimed)
  int chunk;
  // A chunk of `chunk` CG iterations runs as the graph `exec` (the first
  // `head` iterations, the event samples in the first) followed by `reps`
  // launches of the graph `body` (`body_iters` iterations each), so only
  // head + body_iters iterations are captured and instantiated per plan.
  cudaGraphExec_t exec;
  cudaGraphExec_t body = nullptr;
  int head = 0, body_iters = 0, reps = 0;
  cudaStream_t cap;
  HostSlot* slot = nullptr;  // page-locked flag and stats (h_flag, h_st point in)
  int* h_flag = nullptr;
  RhsState* h_st = nullptr;
  long long launches;
  // Event samples around the kernels of the first iteration of every graph
  // launch: live per-kernel durations for the roofline figures.
  cudaEvent_t ev[8];
  // fs_pcg_plan_solve_begin / _poll: the stream, the event after the last
  // enqueued step, 0 idle / 1 a chunk in flight / 2 the finish in flight
  cudaEvent_t ev_async = nullptr;
  cudaStream_t async_s = nullptr;
  int async_stage = 0;
  int async_timed_out = 0;
  long long async_chunks = 0, async_max_chunks = 0;
  double kernel_ms[6];
  int trace;               // record ev[6..7] around fine-level post-smoothing
  long long kernel_samples;
  // Learned preconditioner: the V-cycle stops at level `learned` and the
  // U-Net maps that level's right-hand side to its correction; CG becomes
  // flexible.  -1: plain multigrid.
  int learned = -1;
  int learned_mode = 0;    // 0: network only, 1: network + V-cycle on its residual
  fs_unet* net = nullptr;
  void *net_u = nullptr, *net_r = nullptr;  // level vectors of mode 1
  int net_status = FS_OK;
  // fs_pcg_plan_precondition: the caller's level-0 right-hand side and the
  // level buffer that holds the V-cycle's output
  const void* ext_b = nullptr;
  void* ext_z = nullptr;
};

namespace {

// The TMA-staged stencil is the default; FS_STENCIL=plain selects the
// cached-load kernel (the same arithmetic) for comparison.
// Vectors larger than this march in lockstep (Dims::xc): their halo rows
// would not stay in the 126 MB L2 between neighbouring columns otherwise.
constexpr long long kMarchL2Bytes = 64LL << 20;

// Marching assignment of the CG stencils (lockstep unless FS_MARCH=contig)
// and of the fused smoothing passes (contiguous unless FS_MARCH=lockstep):
// measured at 256x256x128, 8 FP32 RHS, lockstep takes the fused stencil
// from 0.272 to 0.251 ms but the smoothing passes from 0.296 to 0.311 ms
// (two CTAs per SM leave 40 of 296 slots idle in lockstep).
bool march_lockstep() {
  const char* sel = getenv("FS_MARCH");
  return !(sel && strcmp(sel, "contig") == 0);
}
bool march_lockstep_smoothing() {
  const char* sel = getenv("FS_MARCH");
  return sel && strcmp(sel, "lockstep") == 0;
}

// The CG stencil asked for: the plan's option, else FS_STENCIL (plain, tma1,
// tma_m, tmas, tma_split, pz), else -1 (autotuned).
int stencil_request(int opt) {
  if (opt >= 0) return opt;
  const char* sel = getenv("FS_STENCIL");
  if (!sel) return -1;
  static const char* names[8] = {"plain", "tma1", "tma_m", "tmas", "tma_split", "pz",
                                 "pz4", "pz16"};
  for (int k = 0; k < 8; ++k)
    if (strcmp(sel, names[k]) == 0) return k;
  return -1;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    else
      (void)cudaGetLastError();
  }
  return fn;
}

// Process-wide cache of the fastest CG stencil kernel per shape class, filled
// by the first plan of each class (the stencil autotuner): RHS block,
// precision, node count to a power of two, and whether the z extent fills
// whole 32-node tiles.  Plans whose vectors are smaller than
// kTuneMinBytes are not tuned (the kernels differ by launch latency there)
// and run the mass-staging stencil.
constexpr long long kTuneMinBytes = 32LL << 20;

struct StencilKey {
  int k, es, log2n, zfull;
  bool operator<(const StencilKey& o) const {
    if (k != o.k) return k < o.k;
    if (es != o.es) return es < o.es;
    if (log2n != o.log2n) return log2n < o.log2n;
    return zfull < o.zfull;
  }
};
std::mutex g_stencil_mu;
std::map<StencilKey, int> g_stencil_choice;

StencilKey stencil_class(const Dims& d, int k, int es) {
  int l = 0;
  while ((1LL << (l + 1)) <= d.N) ++l;
  return StencilKey{k, es, l, d.nz % 32 == 0 ? 1 : 0};
}

int stencil_choice_get(const Dims& d, int k, int es) {
  if (d.N * k * es < kTuneMinBytes) return 2;
  std::lock_guard<std::mutex> lk(g_stencil_mu);
  auto it = g_stencil_choice.find(stencil_class(d, k, es));
  return it == g_stencil_choice.end() ? -1 : it->second;
}

void stencil_choice_put(const Dims& d, int k, int es, int kind) {
  std::lock_guard<std::mutex> lk(g_stencil_mu);
  g_stencil_choice[stencil_class(d, k, es)] = kind;
}

template <typename T, int K>
struct Impl {
  // Launch grid of the selected CG stencil kernel (persistent TMA kernels:
  // SMs x resident CTAs, capped by the number of (z, y) column tiles x planes).
  static void apply_grid(fs_pcg_plan* P) {
    const long long N = P->d.N;
    // persistent x-marching kernels: resident CTAs per SM x SMs, the lockstep
    // column assignment (Dims::xc) when the vectors do not fit in L2
    auto marching = [&](const void* kern, int threads, size_t smem, int tz, int ty) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      int per_sm = 0, dev = 0, sms = 148;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) !=
              cudaSuccess ||
          per_sm < 1)
        per_sm = 1;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const long long ncols = (long long)((P->d.nz + tz - 1) / tz) * ((P->d.ny + ty - 1) / ty);
      P->dm = P->d;
      P->g_apply = (int)fs::march_grid(&P->dm, ncols, (long long)sms * per_sm,
                                       march_lockstep() ? N * K * (long long)sizeof(T) : 0,
                                       kMarchL2Bytes);
    };
    P->dm = P->d;
    if (P->stencil_kind == 3) {
      using CS = TmaTileS<T, K>;
      marching((const void*)k_stencil_tma_s<T, K>, CS::THREADS, CS::SMEM, CS::TZ, CS::TY);
    } else if (P->stencil_kind == 5) {
      using CZ = TmaTilePZ<T, K>;
      marching((const void*)k_stencil_pz<T, K>, CZ::THREADS, CZ::SMEM, CZ::TZ, CZ::TY);
    } else if (P->stencil_kind == 6 || P->stencil_kind == 7) {
      if constexpr (TmaTileM<T, K>::B <= 32) {
        if (P->stencil_kind == 6) {
          using CZ = TmaTilePZ<T, K, 4>;
          marching((const void*)k_stencil_pz<T, K, 4>, CZ::THREADS, CZ::SMEM, CZ::TZ, CZ::TY);
        } else {
          using CZ = TmaTilePZ<T, K, 16>;
          marching((const void*)k_stencil_pz<T, K, 16>, CZ::THREADS, CZ::SMEM, CZ::TZ, CZ::TY);
        }
      }
    } else if (P->stencil_kind == 4) {
      if constexpr (TmaTileSplit<T, K>::OK) {
        using CM = TmaTileM<T, K>;
        marching((const void*)k_stencil_split<T, K>, TmaTileSplit<T, K>::THREADS, CM::SMEM,
                 CM::TZ, CM::TY);
      }
    } else if (P->stencil_kind == 2) {
      using CM = TmaTileM<T, K>;
      marching((const void*)k_stencil_tma_m<T, K>, CM::THREADS, CM::SMEM, CM::TZ, CM::TY);
    } else if (P->stencil_kind == 1) {
      using C = TmaTile<T, K>;
      marching((const void*)k_stencil_tma<T, K>, C::THREADS, C::SMEM, C::TZ, C::TY);
    } else {
      P->g_apply = fs_grid_blocks((const void*)k_apply_pq<T, K>, N);
    }
  }
  // Time the TMA-staged (2), TMA-store (3), cached-load (0) and split (4)
  // stencils on this plan's buffers (a warm-up, then 3 launches each timed
  // alone with CUDA events on the creation stream) and keep the fastest.
  // Every CG kernel returns at once when the control block says all
  // right-hand sides are done, which a stencil launch on this not yet
  // initialised state sets (no RHS is active), so the flag is cleared before
  // each launch, outside its event pair.  The launches write q, the partials
  // and the per-RHS state; the state and control block are saved and
  // restored around them.
  static int autotune(fs_pcg_plan* P, cudaStream_t s) {
    if constexpr (!TmaTile<T, K>::OK) {
      return FS_OK;
    } else {
      unsigned char* st0 = (unsigned char*)P->st;
      const size_t sbytes = (size_t)((unsigned char*)(P->ctl + 1) - st0);
      std::vector<unsigned char> saved(sbytes);
      FS_CHECK(cudaMemcpyAsync(saved.data(), st0, sbytes, cudaMemcpyDeviceToHost, s));
      FS_CHECK(cudaMemsetAsync(P->p[1], 0, (size_t)P->d.N * K * sizeof(T), s));
      // kind 4 (two threads per node) only for 32-byte nodes; kind 5 (the
      // direction update fused in) once its z tensor map exists.  Every
      // candidate is timed with the direction update it needs: k_pnew and
      // the stencil, or the fused kernel alone.
      // kinds 6 and 7: the fused stencil on 32x4 and 32x16 tiles (nodes of
      // at most 32 bytes), with their own tensor-map boxes
      const bool shapes = P->zmap_ok && TmaTileM<T, K>::B <= 32;
      const int cands[7] = {2, 3, 0, TmaTileSplit<T, K>::OK ? 4 : -1, P->zmap_ok ? 5 : -1,
                            shapes ? 6 : -1, shapes ? 7 : -1};
      float best = 3.4e38f;
      int bestk = 2;
      for (int c = 0; c < 8; ++c) P->tune_ms[c] = -1.f;
      int* done = &P->ctl->all_done;
      for (int c : cands) {
        if (c < 0) continue;
        if (set_kind(P, c) != FS_OK) continue;
        FS_CHECK(cudaMemsetAsync(done, 0, sizeof(int), s));
        kernel(P, 0, 0, s);
        FS_CHECK(cudaMemsetAsync(done, 0, sizeof(int), s));
        kernel(P, 1, 0, s);
        float ms = 0.f;
        for (int r = 0; r < 3; ++r) {
          FS_CHECK(cudaMemsetAsync(done, 0, sizeof(int), s));
          FS_CHECK(cudaEventRecord(P->ev[0], s));
          kernel(P, 0, 0, s);
          kernel(P, 1, 0, s);
          FS_CHECK(cudaEventRecord(P->ev[1], s));
          FS_CHECK(cudaGetLastError());
          FS_CHECK(cudaEventSynchronize(P->ev[1]));
          float one = 0.f;
          FS_CHECK(cudaEventElapsedTime(&one, P->ev[0], P->ev[1]));
          ms += one;
        }
        P->tune_ms[c] = ms / 3.f;
        if (ms < best) {
          best = ms;
          bestk = c;
        }
      }
      if (set_kind(P, bestk) != FS_OK) (void)set_kind(P, 2);
      FS_CHECK(cudaMemcpyAsync(st0, saved.data(), sbytes, cudaMemcpyHostToDevice, s));
      FS_CHECK(cudaStreamSynchronize(s));
      stencil_choice_put(P->d, K, (int)sizeof(T), bestk);
      return FS_OK;
    }
  }
  static void grids(fs_pcg_plan* P) {
    const long long N = P->d.N;
    P->g_init = fs_grid_blocks((const void*)k_init<T, K>, N);
    using C = TmaTile<T, K>;
    P->g_pnew = fs_grid_blocks((const void*)k_pnew<T, K>, N);
    {
      const int want = stencil_request(P->mg.stencil_kind);
      const bool mass_ok = ((long long)P->d.nz * (long long)sizeof(T)) % 16 == 0;
      // k_stencil_tma_m counts its column-planes in 32 bits
      using CM = TmaTileM<T, K>;
      const bool fits32 = (long long)((P->d.nz + CM::TZ - 1) / CM::TZ) *
                              ((P->d.ny + CM::TY - 1) / CM::TY) * P->d.nx <
                          (1LL << 30);
      P->autotune = 0;
      if (!C::OK || want == 0 || P->d.per) {  // only the cached-load kernel wraps
        P->stencil_kind = 0;
      } else if (!mass_ok || !fits32 || want == 1) {
        P->stencil_kind = 1;
      } else if (want == 3) {
        P->stencil_kind = 3;
      } else if (want == 2) {
        P->stencil_kind = 2;
      } else if (want == 5) {
        P->stencil_kind = 5;  // falls back to 2 if the z tensor map cannot be made
      } else if (want == 6 || want == 7) {
        P->stencil_kind = TmaTileM<T, K>::B <= 32 ? want : 5;
      } else if (want == 4) {
        P->stencil_kind = TmaTileSplit<T, K>::OK ? 4 : 2;
      } else {
        // chosen by timing the candidates on the first plan of this shape
        const int cached = stencil_choice_get(P->d, K, (int)sizeof(T));
        P->stencil_kind = cached >= 0 ? cached : 2;
        P->autotune = cached < 0;
      }
    }
    apply_grid(P);
    P->g_update = fs_grid_blocks((const void*)k_update<T, K>, N);
    P->g_rel = fs_grid_blocks((const void*)k_reliable<T, K>, N);
    P->g_fold = fs_grid_blocks((const void*)k_fold<T, K>, N * fs::Chunks<K>::NCH);
    P->g_fin = fs_grid_blocks((const void*)k_finalize<T, K>, N * fs::Chunks<K>::NCH);
    P->g_rz = fs_grid_blocks((const void*)k_rz<T, K>, N);
  }
  // The z (or r) tensor map of the fused direction-update stencil (kind 5),
  // once the multigrid output buffer is known; without it kind 5 is not
  // offered (a plan that asked for it runs kind 2).
  // Tile height of the TMA stencil kinds 2..7 (their tensor-map boxes).
  static int kind_ty(int kind) {
    return kind == 6 ? 4 : (kind == 7 ? 16 : TmaTileM<T, K>::TY);
  }
  // Switch the plan to stencil kind c: the tensor maps of its tile shape,
  // the z map of the fused kinds, its grid.  Not FS_OK if a map cannot be
  // made (the plan keeps a consistent earlier kind in that case).
  static int set_kind(fs_pcg_plan* P, int c) {
    if ((c == 6 || c == 7) && TmaTileM<T, K>::B > 32) return FS_BAD_ARG;
    const int prev = P->stencil_kind;
    P->stencil_kind = c;
    int st = maps(P);
    if (st == FS_OK && c >= 5) {
      zmap(P);
      if (P->stencil_kind != c) st = FS_BAD_ARG;  // z map refused: fell back to 2
    }
    if (st != FS_OK) {
      P->stencil_kind = prev;
      (void)maps(P);
      if (prev >= 5) zmap(P);
    }
    apply_grid(P);
    return st;
  }
  static int zmap(fs_pcg_plan* P) {
    P->zmap_ok = 0;
    if constexpr (!TmaTileM<T, K>::OK) {
      return FS_OK;
    } else {
      const void* zb = P->precond ? P->z : P->r;
      if (P->stencil_kind < 2 || !zb || P->d.per) {
        if (P->stencil_kind >= 5) {
          P->stencil_kind = 2;
          (void)maps(P);
          apply_grid(P);
        }
        return FS_OK;
      }
      auto encode = encode_fn();
      if (!encode) return FS_OK;
      const cuuint64_t B = TmaTileM<T, K>::B;
      cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)P->d.nz, (cuuint64_t)P->d.ny,
                            (cuuint64_t)P->d.nx};
      cuuint64_t strides[3] = {B, B * P->d.nz, B * P->d.nz * P->d.ny};
      // the z box has the p box's shape: the tile of the kind that runs
      const int zhy = P->stencil_kind >= 5 ? kind_ty(P->stencil_kind) + 2 : TmaTileM<T, K>::HY;
      cuuint32_t box[4] = {(cuuint32_t)K, (cuuint32_t)TmaTileM<T, K>::HZ, (cuuint32_t)zhy, 1};
      cuuint32_t es[4] = {1, 1, 1, 1};
      const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
      CUresult rc = encode(&P->tm_z, dt, 4, const_cast<void*>(zb), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (rc == CUDA_SUCCESS) {
        P->zmap_ok = 1;
      } else if (P->stencil_kind >= 5) {
        P->stencil_kind = 2;
        (void)maps(P);
      }
      apply_grid(P);
      return FS_OK;
    }
  }
  static int maps(fs_pcg_plan* P) {
    using C = TmaTile<T, K>;
    P->use_tma = P->stencil_kind != 0 ? 1 : 0;
    if constexpr (!C::OK) return FS_OK;
    if (!P->use_tma) return FS_OK;
    auto encode = encode_fn();
    if (!encode) {
      fs_set_error_msg("cuTensorMapEncodeTiled is unavailable from the driver");
      return FS_CUDA_ERROR;
    }
    const cuuint64_t B = C::B;
    cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)P->d.nz,
                          (cuuint64_t)P->d.ny, (cuuint64_t)P->d.nx};
    cuuint64_t strides[3] = {B, B * P->d.nz, B * P->d.nz * P->d.ny};
    // the p box of the kernel that will run: its tile has its own halo height
    const int hz = P->stencil_kind >= 2 ? TmaTileM<T, K>::HZ : C::HZ;
    const int hy = P->stencil_kind >= 2 ? kind_ty(P->stencil_kind) + 2 : C::HY;
    cuuint32_t box[4] = {(cuuint32_t)K, (cuuint32_t)hz, (cuuint32_t)hy, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    CUtensorMap* maps[2] = {&P->tm_p[0], &P->tm_p[1]};
    void* bases[2] = {P->p[0], P->p[1]};
    for (int m = 0; m < 2; ++m) {
      CUresult rc = encode(maps[m], dt, 4, bases[m], dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (rc != CUDA_SUCCESS) {
        fs_set_error_msg("cuTensorMapEncodeTiled rejected the stencil tensor map");
        return FS_CUDA_ERROR;
      }
    }
    if (P->stencil_kind == 2 || P->stencil_kind == 3) {  // 2 may be tuned into 3
      using CS = TmaTileS<T, K>;
      cuuint32_t qbox[4] = {(cuuint32_t)K, (cuuint32_t)CS::TZ, (cuuint32_t)CS::TY, 1};
      CUresult rc = encode(&P->tm_q, dt, 4, P->q, dims, strides, qbox, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (rc != CUDA_SUCCESS) {
        fs_set_error_msg("cuTensorMapEncodeTiled rejected the q tensor map");
        return FS_CUDA_ERROR;
      }
    }
    if (P->stencil_kind >= 2) {
      using CM = TmaTileM<T, K>;
      const cuuint64_t MB = sizeof(T);
      const int ty = kind_ty(P->stencil_kind);
      cuuint64_t mdims[3] = {(cuuint64_t)P->d.nz, (cuuint64_t)P->d.ny, (cuuint64_t)P->d.nx};
      cuuint64_t mstr[2] = {MB * P->d.nz, MB * P->d.nz * P->d.ny};
      cuuint32_t mes[3] = {1, 1, 1};
      cuuint32_t boxes[3][3] = {{(cuuint32_t)CM::TZ, (cuuint32_t)ty, 1},
                                {(cuuint32_t)CM::TZ, (cuuint32_t)(ty + 1), 1},
                                {(cuuint32_t)(CM::TZ + CM::ZP), (cuuint32_t)ty, 1}};
      void* mb[3] = {P->ex, P->ey, P->ez};
      for (int m = 0; m < 3; ++m) {
        CUresult rc = encode(&P->tm_m[m], dt, 3, mb[m], mdims, mstr, boxes[m], mes,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (rc != CUDA_SUCCESS) {
          fs_set_error_msg("cuTensorMapEncodeTiled rejected a mass tensor map");
          return FS_CUDA_ERROR;
        }
      }
    }
    return FS_OK;
  }
  static void setup_masses(fs_pcg_plan* P, cudaStream_t s) {
    int g = fs_grid_blocks((const void*)k_eq_masses<T>, P->d.N);
    k_eq_masses<T><<<g, fs::kBlock, 0, s>>>(P->d, P->mx, P->my, P->mz, P->s64,
                                            (T*)P->ex, (T*)P->ey, (T*)P->ez);
  }
  static void init(fs_pcg_plan* P, int warm, double tol, int maxiter,
                   double delta, cudaStream_t s) {
    k_init<T, K><<<P->g_init, fs::kBlock, 0, s>>>(
        P->d, P->mx, P->my, P->mz, P->dg, P->label, P->s64, P->phi, P->f, warm,
        (T*)P->x, (T*)P->r, (T*)P->p[0], P->partials, P->st, P->ctl, tol, maxiter,
        delta, P->precond ? (P->learned >= 0 ? 2 : 1) : 0);
  }
  // Iteration with parity `par` reads p[par] and writes p[1 - par].
  // Iteration with parity `par` reads p[par] and writes p[1 - par].
  static void iteration(fs_pcg_plan* P, int par, cudaStream_t s) {
    for (int w = 0; w < 4; ++w) kernel(P, w, par, s);
    if (P->precond) precondition(P, s);
  }
  static void kernel(fs_pcg_plan* P, int which, int par, cudaStream_t s) {
    switch (which) {
      case 0:
        if (P->stencil_kind >= 5) break;  // the fused stencils form p themselves
        k_pnew<T, K><<<P->g_pnew, fs::kBlock, 0, s>>>(
            P->d, (const T*)(P->precond ? P->z : P->r), (const T*)P->p[par],
            (T*)P->p[1 - par], P->st, P->ctl);
        break;
      case 1:
        if constexpr (TmaTile<T, K>::OK) {
          if (P->stencil_kind == 6 || P->stencil_kind == 7) {
            if constexpr (TmaTileM<T, K>::B <= 32) {
              if (P->stencil_kind == 6) {
                using CZ = TmaTilePZ<T, K, 4>;
                k_stencil_pz<T, K, 4><<<P->g_apply, CZ::THREADS, CZ::SMEM, s>>>(
                    P->dm, P->tm_z, P->tm_p[par], P->tm_m[0], P->tm_m[1], P->tm_m[2],
                    (T*)P->p[1 - par], (T*)P->q, P->partials, P->st, P->ctl);
              } else {
                using CZ = TmaTilePZ<T, K, 16>;
                k_stencil_pz<T, K, 16><<<P->g_apply, CZ::THREADS, CZ::SMEM, s>>>(
                    P->dm, P->tm_z, P->tm_p[par], P->tm_m[0], P->tm_m[1], P->tm_m[2],
                    (T*)P->p[1 - par], (T*)P->q, P->partials, P->st, P->ctl);
              }
            }
            break;
          }
          if (P->stencil_kind == 5) {
            using CZ = TmaTilePZ<T, K>;
            k_stencil_pz<T, K><<<P->g_apply, CZ::THREADS, CZ::SMEM, s>>>(
                P->dm, P->tm_z, P->tm_p[par], P->tm_m[0], P->tm_m[1], P->tm_m[2],
                (T*)P->p[1 - par], (T*)P->q, P->partials, P->st, P->ctl);
            break;
          }
          if (P->stencil_kind == 3) {
            using CS = TmaTileS<T, K>;
            k_stencil_tma_s<T, K><<<P->g_apply, CS::THREADS, CS::SMEM, s>>>(
                P->dm, P->tm_p[1 - par], P->tm_m[0], P->tm_m[1], P->tm_m[2], P->tm_q,
                P->partials, P->st, P->ctl);
            break;
          }
          if (P->stencil_kind == 2) {
            using CM = TmaTileM<T, K>;
            k_stencil_tma_m<T, K><<<P->g_apply, CM::THREADS, CM::SMEM, s>>>(
                P->dm, P->tm_p[1 - par], P->tm_m[0], P->tm_m[1], P->tm_m[2], (T*)P->q,
                P->partials, P->st, P->ctl);
            break;
          }
          if constexpr (TmaTileSplit<T, K>::OK) {
            if (P->stencil_kind == 4) {
              using CM = TmaTileM<T, K>;
              k_stencil_split<T, K><<<P->g_apply, TmaTileSplit<T, K>::THREADS, CM::SMEM, s>>>(
                  P->dm, P->tm_p[1 - par], P->tm_m[0], P->tm_m[1], P->tm_m[2], (T*)P->q,
                  P->partials, P->st, P->ctl);
              break;
            }
          }
          if (!P->use_tma) {
            k_apply_pq<T, K><<<P->g_apply, fs::kBlock, 0, s>>>(
                P->d, (const T*)P->ex, (const T*)P->ey, (const T*)P->ez,
                (const T*)P->p[1 - par], (T*)P->q, P->partials, P->st, P->ctl);
            break;
          }
          using C = TmaTile<T, K>;
          k_stencil_tma<T, K><<<P->g_apply, C::THREADS, C::SMEM, s>>>(
              P->dm, P->tm_p[1 - par], (const T*)P->ex, (const T*)P->ey,
              (const T*)P->ez, (const T*)P->p[1 - par], (T*)P->q, P->partials,
              P->st, P->ctl);
        } else {
          k_apply_pq<T, K><<<P->g_apply, fs::kBlock, 0, s>>>(
              P->d, (const T*)P->ex, (const T*)P->ey, (const T*)P->ez,
              (const T*)P->p[1 - par], (T*)P->q, P->partials, P->st, P->ctl);
        }
        break;
      case 2:
        k_update<T, K><<<P->g_update, fs::kBlock, 0, s>>>(
            P->d, (const T*)P->p[1 - par], (const T*)P->q, (T*)P->x, (T*)P->r,
            P->partials, P->st, P->ctl);
        break;
      default:
        k_fold<T, K><<<P->g_fold, fs::kBlock, 0, s>>>(P->d, P->s64, P->phi,
                                                      (T*)P->x, P->st, P->ctl);
        k_reliable<T, K><<<P->g_rel, fs::kBlock, 0, s>>>(
            P->d, P->mx, P->my, P->mz, P->dg, P->s64, P->phi, P->f, (T*)P->r,
            P->partials, P->st, P->ctl);
        break;
    }
  }
  // ---- multigrid ----------------------------------------------------------
  static void mg_setup(fs_pcg_plan* P, cudaStream_t s) {
    // the cap every coarsest level that fits k_mg_coarse stays under (the
    // attribute is process-wide: plans of other sizes share it)
    cudaFuncSetAttribute(fs::k_mg_coarse<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)fs::kCoarseSmemCap);
    pre_fused_setup();
    for (int l = 0; l + 1 < P->nlev && !P->agg; ++l) {  // kernel attributes before capture
      (void)restrict_tma_ok(P->lev[l], P->lev[l + 1]);
    }
    MgLevel& L0 = P->lev[0];
    L0.em[0] = P->ex;
    L0.em[1] = P->ey;
    L0.em[2] = P->ez;
    L0.b = P->r;
    int g = fs_grid_blocks((const void*)fs::k_mg_scales<T>, P->d.N);
    fs::k_mg_scales<T><<<g, fs::kBlock, 0, s>>>(P->d.N, P->s64, (T*)L0.s,
                                                (T*)L0.sd);
    for (int l = 1; l < P->nlev; ++l) {
      MgLevel& f = P->lev[l - 1];
      MgLevel& c = P->lev[l];
      const double* fm[3] = {l == 1 ? P->mx : f.m64[0], l == 1 ? P->my : f.m64[1],
                             l == 1 ? P->mz : f.m64[2]};
      const uint8_t* flab = l == 1 ? P->label : f.label;
      // the fine level's node term: the plan's (level 1) or the Galerkin
      // remainder of the level above (aggregation)
      const double* fdg = l == 1 ? P->dg : ((P->agg || P->dg) ? f.d64 : nullptr);
      if (P->agg) {
        g = fs_grid_blocks((const void*)fs::k_agg_coarsen, c.d.N);
        fs::k_agg_coarsen<<<g, fs::kBlock, 0, s>>>(f.d, c.d, fm[0], fm[1], fm[2], fdg, flab,
                                                   c.m64[0], c.m64[1], c.m64[2], c.d64,
                                                   c.label_in);
      } else {
        g = fs_grid_blocks((const void*)fs::k_mg_coarsen, c.d.N);
        fs::k_mg_coarsen<<<g, fs::kBlock, 0, s>>>(f.d, c.d, fm[0], fm[1], fm[2],
                                                  flab, c.m64[0], c.m64[1],
                                                  c.m64[2], c.label_in);
        if (P->dg) {
          g = fs_grid_blocks((const void*)fs::k_mg_coarsen_diag, c.d.N);
          fs::k_mg_coarsen_diag<<<g, fs::kBlock, 0, s>>>(f.d, c.d, fdg, c.d64);
        }
      }
      const bool cdiag = P->agg || P->dg;
      g = fs_grid_blocks((const void*)k_classify, c.d.N);
      k_classify<<<g, fs::kBlock, 0, s>>>(c.d, c.m64[0], c.m64[1], c.m64[2],
                                          cdiag ? c.d64 : nullptr, c.label_in, c.label,
                                          c.s64, nullptr);
      g = fs_grid_blocks((const void*)k_eq_masses<T>, c.d.N);
      k_eq_masses<T><<<g, fs::kBlock, 0, s>>>(c.d, c.m64[0], c.m64[1], c.m64[2],
                                              c.s64, (T*)c.em[0], (T*)c.em[1],
                                              (T*)c.em[2]);
      g = fs_grid_blocks((const void*)fs::k_mg_scales<T>, c.d.N);
      fs::k_mg_scales<T><<<g, fs::kBlock, 0, s>>>(c.d.N, c.s64, (T*)c.s,
                                                  (T*)c.sd);
    }
  }
  // Launch one V-cycle on level l for right-hand side b; returns the index
  // of the level's x buffer that holds the result, and counts launches.
  // One V-cycle on level l; at the learned level the network takes over:
  // mode 0 returns its output as the level's correction, mode 1 adds a
  // V-cycle on the residual of that output (network guess + multigrid
  // cleanup).  Returns the index of the level's x buffer holding the result.
  static int vcycle(fs_pcg_plan* P, int l, const T* b, cudaStream_t s,
                    long long* nl, bool dry = false) {
    if constexpr (std::is_same<T, float>::value) {
      if (l == P->learned && P->net) {
        MgLevel& L = P->lev[l];
        const int* done = &P->ctl->all_done;
        float* u = P->learned_mode ? (float*)P->net_u : (float*)L.x[0];
        if (!dry) {
          // rhs and output K-interleaved, geometry shared by the K samples
          const int st = unet_forward(P->net, b, K, 1, (const float*)L.em[0],
                                      (const float*)L.em[1], (const float*)L.em[2], 0,
                                      l ? L.label : P->label, 0, u, K, 1, false, s);
          if (st != FS_OK) P->net_status = st;
        }
        *nl += unet_forward_launches();
        if (!P->learned_mode) return 0;
        const int g = fs_grid_blocks((const void*)fs::k_mg_residual<T, K>, L.d.N);
        if (!dry)
          fs::k_mg_residual<T, K><<<g, fs::kBlock, 0, s>>>(
              L.d, (const T*)L.em[0], (const T*)L.em[1], (const T*)L.em[2], (const T*)u, b,
              (T*)P->net_r, done);
        ++*nl;
        const int cur = vcycle_plain(P, l, (const T*)P->net_r, s, nl, dry);
        if (!dry)
          fs::k_mg_add<T, K><<<g, fs::kBlock, 0, s>>>(L.d, (T*)L.x[cur], (const T*)u, done);
        ++*nl;
        return cur;
      }
    }
    return vcycle_plain(P, l, b, s, nl, dry);
  }
  // Whether a level's degree-2 pre-smoothing (post = false) or post-smoothing
  // (post = true) runs as a fused single pass (k_mg_pre_fused,
  // k_mg_post_fused); FS_MG_PRE=plain / FS_MG_POST=plain keep the two-kernel
  // forms.
  static bool smooth_fused_ok(const MgLevel& L, bool post) {
    if (L.d.per) return false;  // the TMA tiles do not wrap
    using CP = SmoothTile<T, K>;
    if constexpr (!CP::OK) {
      return false;
    } else {
      const char* sel = getenv(post ? "FS_MG_POST" : "FS_MG_PRE");
      if (sel && strcmp(sel, "plain") == 0) return false;
      if ((post ? post_per_sm() : pre_per_sm()) <= 0) return false;
      if (((long long)L.d.nz * (long long)sizeof(T)) % 16 != 0) return false;  // mass rows
      if (((long long)L.d.nz * CP::B) % 16 != 0) return false;  // merged vector rows
      const long long cols = (long long)((L.d.nz + CP::TZ - 1) / CP::TZ) *
                             ((L.d.ny + CP::TY - 1) / CP::TY) * L.d.nx;
      return cols < (1LL << 30);
    }
  }
  // The two-threads-per-node form of the fused passes (32-byte nodes);
  // FS_MG_SPLIT=0 keeps one thread per node.
  static bool split_ok(bool post) {
    if constexpr (!SplitTile<T, K>::OK) {
      return false;
    } else {
      const char* sel = getenv("FS_MG_SPLIT");
      if (sel && strcmp(sel, "0") == 0) return false;
      return split_per_sm(post) > 0;
    }
  }
  // Resident k_mg_pre_fused blocks per SM (set with the shared-memory limit
  // when a plan builds its hierarchy; 0 = the kernel cannot run), per device:
  // the shared-memory attribute is a per-device setting.
  static int& pre_per_sm() {
    static int v[fs::kMaxDevices] = {};
    return v[fs::current_device_slot()];
  }
  static int& post_per_sm() {
    static int v[fs::kMaxDevices] = {};
    return v[fs::current_device_slot()];
  }
  // k_mg_smooth_split (32-byte nodes): resident blocks per SM, pre and post
  static int& split_per_sm(bool post) {
    static int v[fs::kMaxDevices][2] = {};
    return v[fs::current_device_slot()][post ? 1 : 0];
  }
  template <bool POST>
  static void split_setup() {
    using CP = SmoothTile<T, K>;
    using CS = SplitTile<T, K>;
    if constexpr (CS::OK) {
      if (split_per_sm(POST) > 0) return;
      if (cudaFuncSetAttribute(k_mg_smooth_split<T, K, POST>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)CP::SMEM) != cudaSuccess)
        return;
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_smooth_split<T, K, POST>,
                                                        CS::THREADS, CP::SMEM) == cudaSuccess)
        split_per_sm(POST) = per_sm;
    }
  }
  static void pre_fused_setup() {
    using CP = SmoothTile<T, K>;
    split_setup<false>();
    split_setup<true>();
    if constexpr (CP::OK) {
      if (pre_per_sm() == 0 &&
          cudaFuncSetAttribute(k_mg_pre_fused<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)CP::SMEM) == cudaSuccess) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_pre_fused<T, K>,
                                                          CP::THREADS, CP::SMEM) == cudaSuccess)
          pre_per_sm() = per_sm;
      }
      if (post_per_sm() == 0 &&
          cudaFuncSetAttribute(k_mg_post_fused<T, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)CP::SMEM) == cudaSuccess) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_post_fused<T, K>,
                                                          CP::THREADS, CP::SMEM) == cudaSuccess)
          post_per_sm() = per_sm;
      }
    }
  }
  // The tensor maps of a fused smoothing pass on level L: the K-interleaved
  // vector `src` (two-node halo box) and the three equilibrated mass arrays.
  static bool smooth_maps(const MgLevel& L, const T* src, CUtensorMap* tv, CUtensorMap* tm) {
    using CP = SmoothTile<T, K>;
    auto encode = encode_fn();
    if (!encode) return false;
    const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t Bn = CP::B, MB = sizeof(T);
    cuuint32_t es[4] = {1, 1, 1, 1};
    if constexpr (CP::MERGED) {
      // rows of nz*K values; boxes of IZ*K values from (z0 - 2)*K
      cuuint64_t dims[3] = {(cuuint64_t)L.d.nz * K, (cuuint64_t)L.d.ny, (cuuint64_t)L.d.nx};
      cuuint64_t strides[2] = {Bn * L.d.nz, Bn * L.d.nz * L.d.ny};
      cuuint32_t box[3] = {(cuuint32_t)(CP::IZ * K), (cuuint32_t)CP::IY, 1};
      if (encode(tv, dt, 3, (void*)src, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    } else {
      cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)L.d.nz, (cuuint64_t)L.d.ny,
                            (cuuint64_t)L.d.nx};
      cuuint64_t strides[3] = {Bn, Bn * L.d.nz, Bn * L.d.nz * L.d.ny};
      cuuint32_t box[4] = {(cuuint32_t)K, (cuuint32_t)CP::IZ, (cuuint32_t)CP::IY, 1};
      if (encode(tv, dt, 4, (void*)src, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    }
    cuuint64_t mdims[3] = {(cuuint64_t)L.d.nz, (cuuint64_t)L.d.ny, (cuuint64_t)L.d.nx};
    cuuint64_t mstr[2] = {MB * L.d.nz, MB * L.d.nz * L.d.ny};
    cuuint32_t mbox[3] = {(cuuint32_t)CP::WZ, (cuuint32_t)CP::WY, 1};
    for (int m = 0; m < 3; ++m)
      if (encode(&tm[m], dt, 3, L.em[m], mdims, mstr, mbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    return true;
  }
  // Persistent grid of a fused smoothing pass on level L.
  // Grid of a fused smoothing pass on level L with per_sm resident CTAs per
  // SM; *dl receives the level's dims with the marching assignment.
  static int smooth_grid(const MgLevel& L, int per_sm, Dims* dl) {
    using CP = SmoothTile<T, K>;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long ncols = (long long)((L.d.nz + CP::TZ - 1) / CP::TZ) *
                            ((L.d.ny + CP::TY - 1) / CP::TY);
    *dl = L.d;
    return (int)fs::march_grid(dl, ncols, (long long)sms * per_sm,
                               march_lockstep_smoothing() ? L.d.N * K * (long long)sizeof(T) : 0,
                               kMarchL2Bytes);
  }
  // k_mg_pre_fused on level L (x2 into x[1], r2 into dv); false if a tensor
  // map cannot be made for these buffers.
  static bool launch_pre_fused(fs_pcg_plan* P, MgLevel& L, const T* b, T c0, T cd, T cr,
                               cudaStream_t s) {
    using CP = SmoothTile<T, K>;
    if constexpr (!CP::OK) {
      return false;
    } else {
      CUtensorMap tb, tm[3];
      if (!smooth_maps(L, b, &tb, tm)) return false;
      if constexpr (SplitTile<T, K>::OK) {
        if (split_ok(false)) {
          Dims dl;
          const int g = smooth_grid(L, split_per_sm(false), &dl);
          k_mg_smooth_split<T, K, false><<<g, SplitTile<T, K>::THREADS, CP::SMEM, s>>>(
              dl, tb, tm[0], tm[1], tm[2], b, (T*)L.x[1], (T*)L.dv, c0, cd, cr,
              &P->ctl->all_done, &P->ctl->error, nullptr, nullptr, nullptr);
          return true;
        }
      }
      Dims dl;
      const int g = smooth_grid(L, pre_per_sm(), &dl);
      k_mg_pre_fused<T, K><<<g, CP::THREADS, CP::SMEM, s>>>(
          dl, tb, tm[0], tm[1], tm[2], (T*)L.x[1], (T*)L.dv, c0, cd, cr, &P->ctl->all_done,
          &P->ctl->error);
      return true;
    }
  }
  // k_mg_restrict_tma: resident CTAs per SM (0 = cannot run), per device.
  static int& restrict_per_sm() {
    static int v[fs::kMaxDevices] = {};
    return v[fs::current_device_slot()];
  }
  // The TMA restriction from level L to C: 16- or 32-byte nodes, every axis
  // halved, no wrap, sd rows whose stride is a multiple of 16 bytes;
  // FS_MG_RESTRICT=plain keeps k_mg_restrict.
  static bool restrict_tma_ok(const MgLevel& L, const MgLevel& C) {
    using R = RestrictTile<T, K>;
    if constexpr (!R::OK) {
      return false;
    } else {
      const char* sel = getenv("FS_MG_RESTRICT");
      if (sel && strcmp(sel, "plain") == 0) return false;
      if (L.d.per || L.d.nx == C.d.nx || L.d.ny == C.d.ny || L.d.nz == C.d.nz) return false;
      if (((long long)L.d.nz * (long long)sizeof(T)) % 16 != 0) return false;
      if (restrict_per_sm() == 0) {
        if (cudaFuncSetAttribute(k_mg_restrict_tma<T, K>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)R::SMEM) != cudaSuccess)
          return false;
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_restrict_tma<T, K>,
                                                          R::THREADS, R::SMEM) != cudaSuccess)
          return false;
        restrict_per_sm() = per_sm;
      }
      return restrict_per_sm() > 0;
    }
  }
  // k_mg_restrict_tma from level L (residual `res`) into C.b; false if a
  // tensor map cannot be made for these buffers (nothing launched).
  static bool launch_restrict_tma(fs_pcg_plan* P, const MgLevel& L, MgLevel& C, const T* res,
                                  cudaStream_t s) {
    using R = RestrictTile<T, K>;
    if constexpr (!R::OK) {
      return false;
    } else {
      auto encode = encode_fn();
      if (!encode) return false;
      const CUtensorMapDataType dt = sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                    : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
      const cuuint64_t Bn = R::B, MB = sizeof(T);
      CUtensorMap tr, tsd;
      cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)L.d.nz, (cuuint64_t)L.d.ny,
                            (cuuint64_t)L.d.nx};
      cuuint64_t strides[3] = {Bn, Bn * L.d.nz, Bn * L.d.nz * L.d.ny};
      cuuint32_t box[4] = {(cuuint32_t)K, (cuuint32_t)R::FZ, (cuuint32_t)R::FY, 1};
      cuuint32_t es[4] = {1, 1, 1, 1};
      if (encode(&tr, dt, 4, (void*)res, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
      cuuint64_t sdims[3] = {(cuuint64_t)L.d.nz, (cuuint64_t)L.d.ny, (cuuint64_t)L.d.nx};
      cuuint64_t sstr[2] = {MB * L.d.nz, MB * L.d.nz * L.d.ny};
      cuuint32_t sbox[3] = {(cuuint32_t)R::SZ, (cuuint32_t)R::FY, 1};
      if (encode(&tsd, dt, 3, (void*)L.sd, sdims, sstr, sbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
      int dev = 0, sms = 148;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      const long long ncols = (long long)((C.d.nz + R::CZ - 1) / R::CZ) *
                              ((C.d.ny + R::CY - 1) / R::CY);
      Dims dc = C.d;
      const int g = (int)fs::march_grid(&dc, ncols, (long long)sms * restrict_per_sm(), 0, 0);
      k_mg_restrict_tma<T, K><<<g, R::THREADS, R::SMEM, s>>>(
          L.d, dc, tr, tsd, (const T*)C.s, (T*)C.b, &P->ctl->all_done, &P->ctl->error);
      return true;
    }
  }
  // Whether the finest post-smoothing runs as k_mg_smooth_split, which can
  // form r~.z in the same pass.
  static bool post_split(const MgLevel& L) {
    if constexpr (SplitTile<T, K>::OK) {
      return smooth_fused_ok(L, true) && split_ok(true);
    } else {
      return false;
    }
  }
  // k_mg_post_fused on level L (xout = x + alpha r0 + beta A~r0, r0 = b - A~x).
  // Returns 0 if a tensor map cannot be made for these buffers (nothing
  // launched), 1 when launched, 2 when launched with r~.z formed in the pass
  // (rz requested and the two-threads-per-node form runs).
  static int launch_post_fused(fs_pcg_plan* P, MgLevel& L, const T* x, const T* b, T* xout,
                               T alpha, T beta, bool rz, cudaStream_t s) {
    using CP = SmoothTile<T, K>;
    if constexpr (!CP::OK) {
      return 0;
    } else {
      CUtensorMap tx, tm[3];
      if (!smooth_maps(L, x, &tx, tm)) return 0;
      if constexpr (SplitTile<T, K>::OK) {
        if (split_ok(true)) {
          Dims dl;
          const int g = smooth_grid(L, split_per_sm(true), &dl);
          const bool with_rz = rz && g <= kMaxBlocks;  // partials hold kMaxBlocks rows
          k_mg_smooth_split<T, K, true><<<g, SplitTile<T, K>::THREADS, CP::SMEM, s>>>(
              dl, tx, tm[0], tm[1], tm[2], b, xout, nullptr, alpha, beta, (T)0,
              &P->ctl->all_done, &P->ctl->error, with_rz ? P->partials : nullptr, P->st,
              P->ctl);
          return with_rz ? 2 : 1;
        }
      }
      Dims dl;
      const int g = smooth_grid(L, post_per_sm(), &dl);
      k_mg_post_fused<T, K><<<g, CP::THREADS, CP::SMEM, s>>>(
          dl, tx, tm[0], tm[1], tm[2], b, xout, alpha, beta, &P->ctl->all_done,
          &P->ctl->error);
      return 1;
    }
  }
  static int vcycle_plain(fs_pcg_plan* P, int l, const T* b, cudaStream_t s,
                          long long* nl, bool dry = false) {
    MgLevel& L = P->lev[l];
    const int* done = &P->ctl->all_done;
    const bool last = l == P->nlev - 1;
    const int deg = last ? P->mg.coarse_deg : P->mg.smooth_deg;
    double cd[64], cr[64];
    cheb_coeffs(deg, last ? P->mg.coarse_lo : P->mg.smooth_lo, 2.0, cd, cr);
    const T *e0 = (const T*)L.em[0], *e1 = (const T*)L.em[1], *e2 = (const T*)L.em[2];
    const int g = fs_grid_blocks((const void*)fs::k_mg_cheb<T, K>, L.d.N);
    int cur = 0;
    // Degree-2 pre-smoothing carries its residual along (x in x[1], the
    // residual in dv); otherwise Chebyshev steps then a residual pass.
    const bool resform = !last && deg == 2;
    const T* rfine = (const T*)L.res;
    if (resform && smooth_fused_ok(L, false)) {
      // x2 -> x[1], r2 -> dv in one pass over b; the two-kernel form if the
      // tensor maps cannot be made for these buffers
      if (!dry && !launch_pre_fused(P, L, b, (T)cr[0], (T)cd[1], (T)cr[1], s)) {
        fs::k_mg_pre0<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, b, (T*)L.x[0], (T*)L.res, (T)cr[0], done);
        fs::k_mg_pre1<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, (const T*)L.x[0], (const T*)L.res, (T*)L.x[1],
            (T*)L.dv, (T)cd[1], (T)cr[1], done);
      }
      cur = 1;
      rfine = (const T*)L.dv;
      *nl += 1;
    } else if (resform) {
      if (!dry) {
        fs::k_mg_pre0<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, b, (T*)L.x[0], (T*)L.res, (T)cr[0], done);
        fs::k_mg_pre1<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, (const T*)L.x[0], (const T*)L.res, (T*)L.x[1],
            (T*)L.dv, (T)cd[1], (T)cr[1], done);
      }
      cur = 1;
      rfine = (const T*)L.dv;
      *nl += 2;
    } else if (last && !L.d.per && fs::coarse_fits<T>(L.d.N, deg)) {
      // the whole coarsest-level solve in one launch, one block per RHS
      fs::CoarseCoef<T> coef;
      for (int k = 0; k < deg; ++k) {
        coef.cd[k] = (T)cd[k];
        coef.cr[k] = (T)cr[k];
      }
      cur = (deg - 1) % 2;  // the buffer the step-by-step solve ends in
      if (!dry)
        fs::k_mg_coarse<T, K><<<K, fs::kCoarseThreads, fs::coarse_smem<T>(L.d.N), s>>>(
            L.d, e0, e1, e2, b, (T*)L.x[cur], coef, deg, done);
      ++*nl;
    } else {
      for (int k = 0; k < deg; ++k) {  // pre-smoothing (or coarse solve) from 0
        const int out = k == 0 ? 0 : 1 - cur;
        if (!dry)
          fs::k_mg_cheb<T, K><<<g, fs::kBlock, 0, s>>>(
              L.d, e0, e1, e2, (const T*)L.x[cur], (T*)L.x[out], (T*)L.dv, b,
              (T)cd[k], (T)cr[k], k == 0 ? 1 : 0, k < deg - 1 ? 1 : 0, done);
        cur = out;
        ++*nl;
      }
    }
    if (last) return cur;
    MgLevel& C = P->lev[l + 1];
    const int gc = fs_grid_blocks((const void*)fs::k_mg_restrict<T, K>, C.d.N);
    if (!dry) {
      if (!resform)
        fs::k_mg_residual<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, (const T*)L.x[cur], b, (T*)L.res, done);
      if (P->agg)
        fs::k_agg_restrict<T, K><<<gc, fs::kBlock, 0, s>>>(
            L.d, C.d, rfine, (const T*)L.sd, (const T*)C.s, (T*)C.b, done);
      else if (!(restrict_tma_ok(L, C) && launch_restrict_tma(P, L, C, rfine, s)))
        fs::k_mg_restrict<T, K><<<gc, fs::kBlock, 0, s>>>(
            L.d, C.d, rfine, (const T*)L.sd, (const T*)C.s, (T*)C.b, done);
    }
    *nl += resform ? 1 : 2;
    const int cc = vcycle(P, l + 1, (const T*)C.b, s, nl, dry);
    if (!dry) {
      if (P->agg) {
        const int gp = fs_grid_blocks((const void*)fs::k_agg_prolong<T, K>, L.d.N);
        fs::k_agg_prolong<T, K><<<gp, fs::kBlock, 0, s>>>(
            L.d, C.d, (const T*)C.x[cc], (const T*)C.s, (const T*)L.sd, (T*)L.x[cur],
            (T)P->mg.agg_alpha, done);
      } else {
        const int gp = fs_grid_blocks((const void*)fs::k_mg_prolong_cell<T, K>, C.d.N);
        fs::k_mg_prolong_cell<T, K><<<gp, fs::kBlock, 0, s>>>(
            L.d, C.d, (const T*)C.x[cc], (const T*)C.s, (const T*)L.sd,
            (T*)L.x[cur], done);
      }
    }
    ++*nl;
    const bool tr = !dry && l == 0 && P->trace;
    if (tr) cudaEventRecordWithFlags(P->ev[6], s, cudaEventRecordExternal);
    if (deg == 2) {  // post-smoothing as residual pass + polynomial pass
      const int out = 1 - cur;
      const double alpha = cr[0] * (1.0 + cd[1]) + cr[1], beta = -cr[1] * cr[0];
      const bool fused = smooth_fused_ok(L, true);
      const bool want_rz = l == 0 && P->rz_request;
      int how = 0;
      if (!dry && fused)
        how = launch_post_fused(P, L, (const T*)L.x[cur], b, (T*)L.x[out], (T)alpha,
                                (T)beta, want_rz, s);
      if (want_rz) P->rz_fused = dry ? (post_split(L) ? 1 : 0) : (how == 2 ? 1 : 0);
      if (!dry && how == 0) {
        fs::k_mg_residual<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, (const T*)L.x[cur], b, (T*)L.res, done);
        fs::k_mg_post2<T, K><<<g, fs::kBlock, 0, s>>>(
            L.d, e0, e1, e2, (const T*)L.x[cur], (const T*)L.res, (T*)L.x[out], (T)alpha,
            (T)beta, done);
      }
      cur = out;
      *nl += fused ? 1 : 2;
    } else {
      for (int k = 0; k < deg; ++k) {  // post-smoothing from the corrected x
        const int out = 1 - cur;
        if (!dry)
          fs::k_mg_cheb<T, K><<<g, fs::kBlock, 0, s>>>(
              L.d, e0, e1, e2, (const T*)L.x[cur], (T*)L.x[out], (T*)L.dv, b,
              (T)cd[k], (T)cr[k], 0, k < deg - 1 ? 1 : 0, done);
        cur = out;
        ++*nl;
      }
    }
    if (tr) cudaEventRecordWithFlags(P->ev[7], s, cudaEventRecordExternal);
    return cur;
  }
  // Fix the level-0 output buffer (z) without launching anything; the graph
  // captures kernels that read z before the first V-cycle of an iteration.
  static void locate_z(fs_pcg_plan* P) {
    long long nl = 0;
    P->rz_request = P->learned < 0 ? 1 : 0;
    P->rz_fused = 0;
    const int zi = vcycle(P, 0, (const T*)P->r, nullptr, &nl, true);
    P->rz_request = 0;
    P->z = P->lev[0].x[zi];
    P->launches_per_iter = nl + (P->rz_fused ? 0 : 1);
  }
  // z = M r~ and gamma = r~.z: in the finest post-smoothing pass when it can
  // form the product (plain multigrid), else by k_rz / k_rz_flex.  Returns
  // the number of launches.
  static long long precondition(fs_pcg_plan* P, cudaStream_t s) {
    long long nl = 0;
    P->rz_request = P->learned < 0 ? 1 : 0;
    P->rz_fused = 0;
    const int zi = vcycle(P, 0, (const T*)P->r, s, &nl);
    P->rz_request = 0;
    P->z = P->lev[0].x[zi];
    if (P->learned >= 0)
      k_rz_flex<T, K><<<P->g_rz, fs::kBlock, 0, s>>>(P->d, (const T*)P->r, (const T*)P->z,
                                                     (const T*)P->q, P->partials, P->st,
                                                     P->ctl);
    else if (!P->rz_fused)
      k_rz<T, K><<<P->g_rz, fs::kBlock, 0, s>>>(P->d, (const T*)P->r,
                                                (const T*)P->z, P->partials,
                                                P->st, P->ctl);
    return nl + (P->rz_fused ? 0 : 1);
  }
  // One V-cycle on a caller's equilibrated right-hand side (P->ext_b).
  static void vcycle_ext(fs_pcg_plan* P, cudaStream_t s) {
    long long nl = 0;
    const int zi = vcycle(P, 0, (const T*)P->ext_b, s, &nl);
    P->ext_z = P->lev[0].x[zi];
  }
  static void finalize(fs_pcg_plan* P, cudaStream_t s) {
    k_finalize<T, K><<<P->g_fin, fs::kBlock, 0, s>>>(P->d, P->label, P->s64,
                                                     P->phi, (T*)P->x, P->st,
                                                     P->ctl);
  }
};

template <typename T>
bool dispatch_k(int k, fs_pcg_plan* P, int op, cudaStream_t s, int warm = 0,
                double tol = 0, int maxiter = 0, double delta = 0,
                int par = 0) {
#define FS_OP(KK)                                                   \
  case KK:                                                          \
    if (op == 0) Impl<T, KK>::grids(P);                             \
    if (op == 1) Impl<T, KK>::setup_masses(P, s);                   \
    if (op == 2) Impl<T, KK>::init(P, warm, tol, maxiter, delta, s); \
    if (op == 3) Impl<T, KK>::iteration(P, par, s);                 \
    if (op == 4) Impl<T, KK>::finalize(P, s);                       \
    if (op >= 5 && op <= 8) Impl<T, KK>::kernel(P, op - 5, par, s); \
    if (op == 9) { Impl<T, KK>::mg_setup(P, s); Impl<T, KK>::locate_z(P); } \
    if (op == 10) P->launches_per_iter = Impl<T, KK>::precondition(P, s); \
    if (op == 11) Impl<T, KK>::locate_z(P);                        \
    if (op == 12) Impl<T, KK>::vcycle_ext(P, s);                   \
    if (op == 13) P->net_status = Impl<T, KK>::autotune(P, s);      \
    if (op == 14) P->net_status = Impl<T, KK>::zmap(P);             \
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

template <typename T>
int maps_k(int k, fs_pcg_plan* P) {
  switch (k) {
    case 1: return Impl<T, 1>::maps(P);
    case 2: return Impl<T, 2>::maps(P);
    case 4: return Impl<T, 4>::maps(P);
    case 8: return Impl<T, 8>::maps(P);
    case 16: return Impl<T, 16>::maps(P);
    default: return FS_BAD_ARG;
  }
}

int make_maps(fs_pcg_plan* P) {
  return P->precision == FS_PRECISION_MIXED ? maps_k<float>(P->nrhs, P)
                                            : maps_k<double>(P->nrhs, P);
}

bool dispatch(fs_pcg_plan* P, int op, cudaStream_t s, int warm = 0,
              double tol = 0, int maxiter = 0, double delta = 0, int par = 0) {
  if (P->precision == FS_PRECISION_MIXED)
    return dispatch_k<float>(P->nrhs, P, op, s, warm, tol, maxiter, delta, par);
  return dispatch_k<double>(P->nrhs, P, op, s, warm, tol, maxiter, delta, par);
}

// One CG iteration with event records between its kernels (captured into
// the graph as event nodes).
// A plain cudaEventRecord inside a capture only orders streams; the
// External flag makes it an event-record node that executes with the graph.
void dispatch_first(fs_pcg_plan* P, cudaStream_t s) {
  for (int w = 0; w < 4; ++w) {
    cudaEventRecordWithFlags(P->ev[w], s, cudaEventRecordExternal);
    dispatch(P, 5 + w, s);  // K0 p update, K1 stencil, K2 update, K3 (parity 0)
  }
  cudaEventRecordWithFlags(P->ev[4], s, cudaEventRecordExternal);
  P->trace = 1;
  if (P->precond) dispatch(P, 10, s);  // V-cycle and r.z
  P->trace = 0;
  cudaEventRecordWithFlags(P->ev[5], s, cudaEventRecordExternal);
}

void locate_z_all(fs_pcg_plan* P) { dispatch(P, 11, nullptr); }

// (Re)capture the graphs of a chunk on the plan's capture stream: the head
// (its first iteration with the event samples) and, when the chunk repeats
// one, the body.  head and body_iters are even, so every launch starts on
// parity 0 (p[0] = p_old).
int capture_graph(fs_pcg_plan* P) {
  cudaError_t e;
  if (P->exec) {
    cudaGraphExecDestroy(P->exec);
    P->exec = nullptr;
  }
  if (P->body) {
    cudaGraphExecDestroy(P->body);
    P->body = nullptr;
  }
  if (P->precond) locate_z_all(P);
  for (int part = 0; part < (P->body_iters > 0 ? 2 : 1); ++part) {
    cudaGraph_t graph = nullptr;
    if ((e = cudaStreamBeginCapture(P->cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
      return fs_cuda_status("cudaStreamBeginCapture", e);
    const int n = part == 0 ? P->head : P->body_iters;
    for (int it = 0; it < n; ++it) {
      if (part == 0 && it == 0) {
        dispatch_first(P, P->cap);
      } else {
        dispatch(P, 3, P->cap, 0, 0, 0, 0, it & 1);
      }
    }
    e = cudaStreamEndCapture(P->cap, &graph);
    if (e != cudaSuccess) return fs_cuda_status("cudaStreamEndCapture", e);
    if (P->net_status != FS_OK) {
      cudaGraphDestroy(graph);
      return P->net_status;
    }
    e = cudaGraphInstantiate(part == 0 ? &P->exec : &P->body, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fs_cuda_status("cudaGraphInstantiate", e);
  }
  return FS_OK;
}

}  // namespace

extern "C" {

void fs_mg_params_default(fs_mg_params* p) {
  if (!p) return;
  const MgParams m;
  p->smooth_deg = m.smooth_deg;
  p->smooth_lo = m.smooth_lo;
  p->coarse_deg = m.coarse_deg;
  p->coarse_lo = m.coarse_lo;
  p->coarsest_nodes = m.coarsest_nodes;
  p->stencil_kind = m.stencil_kind;
  p->agg_alpha = m.agg_alpha;
}

int fs_pcg_workspace_bytes_opt(int nx, int ny, int nz, int nrhs, int precision,
                               int precond, const fs_mg_params* opt, size_t* bytes) {
  if (nx < 2 || ny < 2 || nz < 2 || !valid_nrhs(nrhs) || !bytes) return FS_BAD_ARG;
  if (precision != FS_PRECISION_FP64 && precision != FS_PRECISION_MIXED)
    return FS_BAD_ARG;
  if (precond != FS_PRECOND_JACOBI && precond != FS_PRECOND_MG && precond != FS_PRECOND_MG_AGG)
    return FS_BAD_ARG;
  MgParams m;
  if (!mg_params_from(opt, &m)) return FS_BAD_ARG;
  *bytes = make_layout(fs::make_dims(nx, ny, nz), nrhs, precision, precond,
                       m.coarsest_nodes).total;
  return FS_OK;
}

int fs_pcg_workspace_bytes(int nx, int ny, int nz, int nrhs, int precision,
                           int precond, size_t* bytes) {
  return fs_pcg_workspace_bytes_opt(nx, ny, nz, nrhs, precision, precond, nullptr, bytes);
}

int fs_pcg_plan_create(int nx, int ny, int nz, int nrhs, int precision,
                       int precond, const double* mx, const double* my,
                       const double* mz, const uint8_t* label_in, double* phi,
                       const double* f, void* workspace, size_t workspace_bytes,
                       fs_pcg_plan** plan, void* stream) {
  return fs_pcg_plan_create_diag(nx, ny, nz, nrhs, precision, precond, mx, my, mz, nullptr,
                                 label_in, phi, f, workspace, workspace_bytes, plan, stream);
}

int fs_pcg_plan_create_diag(int nx, int ny, int nz, int nrhs, int precision,
                            int precond, const double* mx, const double* my,
                            const double* mz, const double* diag,
                            const uint8_t* label_in, double* phi,
                            const double* f, void* workspace, size_t workspace_bytes,
                            fs_pcg_plan** plan, void* stream) {
  return fs_pcg_plan_create_ex(nx, ny, nz, nrhs, precision, precond, mx, my, mz, diag, 0,
                               label_in, phi, f, workspace, workspace_bytes, plan, stream);
}

int fs_pcg_plan_create_ex(int nx, int ny, int nz, int nrhs, int precision, int precond,
                          const double* mx, const double* my, const double* mz,
                          const double* diag, int periodic, const uint8_t* label_in,
                          double* phi, const double* f, void* workspace,
                          size_t workspace_bytes, fs_pcg_plan** plan, void* stream) {
  return fs_pcg_plan_create_opt(nx, ny, nz, nrhs, precision, precond, mx, my, mz, diag,
                                periodic, nullptr, label_in, phi, f, workspace,
                                workspace_bytes, plan, stream);
}

int fs_pcg_plan_create_opt(int nx, int ny, int nz, int nrhs, int precision, int precond,
                           const double* mx, const double* my, const double* mz,
                           const double* diag, int periodic, const fs_mg_params* opt,
                           const uint8_t* label_in, double* phi, const double* f,
                           void* workspace, size_t workspace_bytes, fs_pcg_plan** plan,
                           void* stream) {
  if (!plan) return FS_BAD_ARG;
  *plan = nullptr;
  if (periodic < 0 || periodic > 7) return FS_BAD_ARG;
  MgParams mgp;
  if (!mg_params_from(opt, &mgp)) return FS_BAD_ARG;
  if (periodic && precond == FS_PRECOND_MG) {
    fs_set_error_msg("periodic axes: the rediscretised multigrid hierarchy does not wrap; "
                     "use FS_PRECOND_MG_AGG (aggregates wrap) or Jacobi PCG");
    return FS_BAD_ARG;
  }
  size_t need = 0;
  int st = fs_pcg_workspace_bytes_opt(nx, ny, nz, nrhs, precision, precond, opt, &need);
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
  P->d = fs::make_dims(nx, ny, nz, periodic);
  P->nrhs = nrhs;
  P->precision = precision;
  P->precond = (precond == FS_PRECOND_MG || precond == FS_PRECOND_MG_AGG) ? 1 : 0;
  P->agg = precond == FS_PRECOND_MG_AGG ? 1 : 0;
  P->mg = mgp;
  P->launches_per_iter = 0;
  P->rz_request = 0;
  P->rz_fused = 0;
  P->mx = mx;
  P->dg = diag;
  P->my = my;
  P->mz = mz;
  P->phi = phi;
  P->f = f;
  Layout L = make_layout(P->d, nrhs, precision, precond, mgp.coarsest_nodes);
  char* w = (char*)workspace;
  P->nlev = L.nlev;
  for (int l = 0; l < L.nlev; ++l) {
    MgLevel& m = P->lev[l];
    m = L.lev[l];
    if (l > 0) {
      for (int a = 0; a < 3; ++a) {
        m.m64[a] = (double*)(w + m.off_m64[a]);
        m.em[a] = w + m.off_em[a];
      }
      m.s64 = (double*)(w + m.off_s64);
      m.d64 = (double*)(w + m.off_d64);
      m.label_in = (uint8_t*)(w + m.off_label_in);
      m.label = (uint8_t*)(w + m.off_label);
      m.b = w + m.off_b;
    }
    m.s = w + m.off_s;
    m.sd = w + m.off_sd;
    m.x[0] = w + m.off_x[0];
    m.x[1] = w + m.off_x[1];
    m.dv = w + m.off_dv;
    m.res = w + m.off_res;
  }
  P->z = nullptr;
  P->label = (uint8_t*)(w + L.label);
  P->s64 = (double*)(w + L.s64);
  P->ex = w + L.ex;
  P->ey = w + L.ey;
  P->ez = w + L.ez;
  P->x = w + L.x;
  P->r = w + L.r;
  P->p[0] = w + L.p0;
  P->p[1] = w + L.p1;
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
  if (P->g_init > kMaxBlocks || P->g_apply > max_blocks(P->d) ||
      P->g_update > kMaxBlocks || P->g_rel > kMaxBlocks ||
      P->g_fin > kMaxBlocks) {
    delete P;
    return FS_BAD_ARG;
  }
  for (int t = 0; t < 8; ++t) P->ev[t] = nullptr;
  for (int t = 0; t < 6; ++t) P->kernel_ms[t] = 0.0;
  P->trace = 0;
  P->kernel_samples = 0;
  auto fail = [&](const char* where, cudaError_t e) {
    fs_pcg_plan_destroy(P);
    return fs_cuda_status(where, e);
  };
  cudaError_t e;
  if ((e = cudaMemsetAsync(w + L.st, 0, L.total - L.st, s)) != cudaSuccess)
    return fail("memset state", e);
  int g = fs_grid_blocks((const void*)k_classify, P->d.N);
  k_classify<<<g, fs::kBlock, 0, s>>>(P->d, mx, my, mz, P->dg, label_in, P->label,
                                      P->s64, P->ctl->label_counts);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail("k_classify", e);
  dispatch(P, 1, s);
  if ((e = cudaGetLastError()) != cudaSuccess) return fail("k_eq_masses", e);
  {
    int ms = make_maps(P);
    if (ms != FS_OK) {
      fs_pcg_plan_destroy(P);
      return ms;
    }
  }
  if (P->precond) {
    dispatch(P, 9, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail("multigrid setup", e);
  }
  dispatch(P, 14, s);  // the fused stencil's z map, now that z is known
  P->net_status = FS_OK;
  if ((e = host_slot_get(&P->slot)) != cudaSuccess) return fail("cudaMallocHost", e);
  P->h_flag = &P->slot->flag;
  P->h_st = P->slot->st;

  // Capture `chunk` CG iterations once; the graph is replayed until the
  // device reports that every RHS has finished.  Multigrid solves take ~20
  // iterations to 1e-10, so 12 per graph wastes at most a few launches that
  // return at once after convergence (16 wasted up to 10); Jacobi takes
  // thousands, where longer graphs save host round trips.
  P->chunk = P->precond ? 12 : 32;
  // multigrid: a 2-iteration head and a 2-iteration body launched 5 times
  // (capture and instantiation of 4 iterations instead of 12: 0.3 ms less
  // per plan); Jacobi's 5 launches per iteration are captured whole
  P->head = P->precond ? 2 : P->chunk;
  P->body_iters = P->precond ? 2 : 0;
  P->reps = P->body_iters > 0 ? (P->chunk - P->head) / P->body_iters : 0;
  if ((e = cudaStreamCreateWithFlags(&P->cap, cudaStreamNonBlocking)) !=
      cudaSuccess)
    return fail("cudaStreamCreate", e);
  for (int t = 0; t < 8; ++t)
    if ((e = cudaEventCreate(&P->ev[t])) != cudaSuccess)
      return fail("cudaEventCreate", e);
  if (P->autotune) {
    dispatch(P, 13, s);
    const int at = P->net_status;
    P->net_status = FS_OK;
    if (at != FS_OK) {
      fs_pcg_plan_destroy(P);
      return at;
    }
  }
  const int cst = capture_graph(P);
  if (cst != FS_OK) {
    fs_pcg_plan_destroy(P);
    return cst;
  }
  *plan = P;
  return FS_OK;
}

}  // extern "C"

namespace {

// Start a solve on stream s: k_init, then (preconditioned) z = M r and r.z.
int solve_begin(fs_pcg_plan* P, int warm_start, double tol, int maxiter,
                cudaStream_t s) {
  // Mixed precision: refresh the residual after a 10x drop under Jacobi CG
  // (hundreds of FP32 iterations per decade) and after a 1e4 drop under
  // multigrid (a decade every ~2 iterations, so little FP32 drift; measured
  // at 256x256x128: 22 iterations with 1e-3 and 1e-4, one reliable update
  // fewer and 0.96 ms less per extraction with 1e-4; 1e-5 and 1e-6 let the
  // FP32 recurrence drift until RHS stalled into FP64 continuations and
  // 64-geometry batches failed to converge).
  const double delta = P->precision != FS_PRECISION_MIXED ? 0.0
                       : (P->precond ? 1e-4 : 0.1);
  cudaError_t e;
  dispatch(P, 2, s, warm_start ? 1 : 0, tol, maxiter, delta);
  FS_CHECK_LAUNCH("k_init");
  P->launches = 1;
  if (P->precond) {
    dispatch(P, 10, s);  // z = M r and r.z for the first direction
    FS_CHECK_LAUNCH("multigrid V-cycle");
    P->launches += P->launches_per_iter;
  }
  for (int t = 0; t < 6; ++t) P->kernel_ms[t] = 0.0;
  P->kernel_samples = 0;
  return FS_OK;
}

// Enqueue one graph chunk and the copy of the all-done flag.
int solve_chunk(fs_pcg_plan* P, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaGraphLaunch(P->exec, s)) != cudaSuccess)
    return fs_cuda_status("cudaGraphLaunch", e);
  for (int r = 0; r < P->reps; ++r)
    if ((e = cudaGraphLaunch(P->body, s)) != cudaSuccess)
      return fs_cuda_status("cudaGraphLaunch", e);
  P->launches += (5LL + (P->precond ? P->launches_per_iter : 0)) * P->chunk;
  if ((e = cudaMemcpyAsync(P->h_flag, &P->ctl->all_done, sizeof(int),
                           cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fs_cuda_status("cudaMemcpyAsync", e);
  return FS_OK;
}

// After the chunk's stream has drained: accumulate the kernel timings of
// its first iteration; returns 1 when every RHS is done.
int solve_check(fs_pcg_plan* P) {
  float ms[6] = {0, 0, 0, 0, 0, 0};
  bool ok = true;
  for (int t = 0; t < 5 && ok; ++t)
    ok = cudaEventElapsedTime(&ms[t], P->ev[t], P->ev[t + 1]) == cudaSuccess;
  if (ok && P->precond)
    ok = cudaEventElapsedTime(&ms[5], P->ev[6], P->ev[7]) == cudaSuccess;
  if (ok) {
    // the fine-level post-smoothing: one pass at degree 2 (fused, or the
    // residual + polynomial pair), else one Chebyshev step per launch
    if (P->mg.smooth_deg != 2) ms[5] /= (float)P->mg.smooth_deg;
    for (int t = 0; t < 6; ++t) P->kernel_ms[t] += ms[t];
    P->kernel_samples += 1;
  } else {
    (void)cudaGetLastError();  // timing unavailable: not a solve failure
  }
  return *P->h_flag ? 1 : 0;
}

// k_finalize and the copy of the per-RHS state to the host, enqueued.
int solve_finish_enqueue(fs_pcg_plan* P, cudaStream_t s) {
  cudaError_t e;
  dispatch(P, 4, s);
  FS_CHECK_LAUNCH("k_finalize");
  P->launches += 1;
  if ((e = cudaMemcpyAsync(P->h_st, P->st, sizeof(RhsState) * P->nrhs,
                           cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return fs_cuda_status("cudaMemcpyAsync", e);
  return FS_OK;
}

// The per-RHS state (on the host after solve_finish_enqueue's copy) folded
// into stats and a status.
int solve_finish_read(fs_pcg_plan* P, int timed_out, fs_rhs_stats* stats);

// k_finalize, copy the per-RHS state back and fold it into a status.
int solve_finish(fs_pcg_plan* P, int timed_out, fs_rhs_stats* stats,
                 cudaStream_t s) {
  cudaError_t e;
  int st = solve_finish_enqueue(P, s);
  if (st != FS_OK) return st;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
    return fs_cuda_status("cudaStreamSynchronize", e);
  return solve_finish_read(P, timed_out, stats);
}

int solve_finish_read(fs_pcg_plan* P, int timed_out, fs_rhs_stats* stats) {
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
    else if (h.status == FS_STALLED && worst != FS_NAN) worst = FS_STALLED;
    else if (h.status == FS_NOT_CONVERGED && worst == FS_OK) worst = FS_NOT_CONVERGED;
    else if (h.status == FS_TIMEOUT && worst == FS_OK) worst = FS_TIMEOUT;
  }
  if (timed_out) return FS_TIMEOUT;
  return worst;
}

}  // namespace

extern "C" {

// Host bound on the iterations of a solve: maxiter, or for the device-side
// default (maxiter <= 0) its largest possible value, n_free <= N.
static long long host_maxiter(const fs_pcg_plan* P, int maxiter) {
  if (maxiter > 0) return maxiter;
  const long long d = (long long)(10.0 * sqrt((double)P->d.N));
  return d > 500 ? d : 500;
}

int fs_pcg_plan_solve(fs_pcg_plan* P, int warm_start, double tol, int maxiter,
                      fs_rhs_stats* stats, void* stream) {
  if (!P || !(tol > 0.0)) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int st = solve_begin(P, warm_start, tol, maxiter, s);
  if (st != FS_OK) return st;
  const long long max_chunks = host_maxiter(P, maxiter) / P->chunk + 4;
  int timed_out = 1;
  cudaError_t e;
  for (long long c = 0; c < max_chunks; ++c) {
    if ((st = solve_chunk(P, s)) != FS_OK) return st;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
      return fs_cuda_status("cudaStreamSynchronize", e);
    if (solve_check(P)) {
      timed_out = 0;
      break;
    }
  }
  return solve_finish(P, timed_out, stats, s);
}

int fs_pcg_plans_solve(fs_pcg_plan* const* plans, int nplans,
                       void* const* streams, int warm_start, double tol,
                       int maxiter, fs_rhs_stats* const* stats, int* status) {
  if (!plans || nplans < 1 || !streams || !status || !(tol > 0.0)) return FS_BAD_ARG;
  for (int i = 0; i < nplans; ++i)
    if (!plans[i]) return FS_BAD_ARG;
  std::vector<int> active(nplans, 1);
  std::vector<long long> chunks(nplans, 0);
  int st;
  cudaError_t e;
  for (int i = 0; i < nplans; ++i) {
    status[i] = FS_TIMEOUT;
    if ((st = solve_begin(plans[i], warm_start, tol, maxiter,
                          (cudaStream_t)streams[i])) != FS_OK)
      return st;
  }
  // Round robin: one chunk per unfinished plan on its own stream, so the
  // chunks of small systems overlap those of large ones, then a check of
  // each; a plan leaves the rotation when all its RHS are done.
  int left = nplans;
  while (left > 0) {
    for (int i = 0; i < nplans; ++i) {
      if (!active[i]) continue;
      if ((st = solve_chunk(plans[i], (cudaStream_t)streams[i])) != FS_OK) return st;
      ++chunks[i];
    }
    for (int i = 0; i < nplans; ++i) {
      if (!active[i]) continue;
      fs_pcg_plan* P = plans[i];
      if ((e = cudaStreamSynchronize((cudaStream_t)streams[i])) != cudaSuccess)
        return fs_cuda_status("cudaStreamSynchronize", e);
      const int done = solve_check(P);
      const bool out = chunks[i] >= host_maxiter(P, maxiter) / P->chunk + 4;
      if (done || out) {
        active[i] = 0;
        --left;
        status[i] = solve_finish(P, done ? 0 : 1, stats ? stats[i] : nullptr,
                                 (cudaStream_t)streams[i]);
      }
    }
  }
  int worst = FS_OK;
  for (int i = 0; i < nplans; ++i)
    if (status[i] != FS_OK && (worst == FS_OK || status[i] == FS_CUDA_ERROR)) worst = status[i];
  return worst;
}

int fs_pcg_plan_solve_begin(fs_pcg_plan* P, int warm_start, double tol, int maxiter,
                            void* stream) {
  if (!P || !(tol > 0.0) || P->async_stage != 0) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (!P->ev_async &&
      (e = cudaEventCreateWithFlags(&P->ev_async, cudaEventDisableTiming)) != cudaSuccess)
    return fs_cuda_status("cudaEventCreate", e);
  int st = solve_begin(P, warm_start, tol, maxiter, s);
  if (st != FS_OK) return st;
  if ((st = solve_chunk(P, s)) != FS_OK) return st;
  if ((e = cudaEventRecord(P->ev_async, s)) != cudaSuccess)
    return fs_cuda_status("cudaEventRecord", e);
  P->async_s = s;
  P->async_chunks = 1;
  P->async_max_chunks = host_maxiter(P, maxiter) / P->chunk + 4;
  P->async_timed_out = 1;
  P->async_stage = 1;
  return FS_OK;
}

int fs_pcg_plan_solve_poll(fs_pcg_plan* P, fs_rhs_stats* stats, int* done) {
  if (!P || !done || P->async_stage == 0) return FS_BAD_ARG;
  *done = 0;
  cudaError_t e = cudaEventQuery(P->ev_async);
  if (e == cudaErrorNotReady) return FS_OK;
  if (e != cudaSuccess) {
    P->async_stage = 0;
    return fs_cuda_status("cudaEventQuery", e);
  }
  int st;
  if (P->async_stage == 1) {  // a chunk has finished: next chunk, or finish
    if (solve_check(P)) {
      P->async_timed_out = 0;
    } else if (P->async_chunks < P->async_max_chunks) {
      if ((st = solve_chunk(P, P->async_s)) != FS_OK) {
        P->async_stage = 0;
        return st;
      }
      ++P->async_chunks;
      if ((e = cudaEventRecord(P->ev_async, P->async_s)) != cudaSuccess) {
        P->async_stage = 0;
        return fs_cuda_status("cudaEventRecord", e);
      }
      return FS_OK;
    }
    if ((st = solve_finish_enqueue(P, P->async_s)) != FS_OK ||
        (e = cudaEventRecord(P->ev_async, P->async_s)) != cudaSuccess) {
      P->async_stage = 0;
      return st != FS_OK ? st : fs_cuda_status("cudaEventRecord", e);
    }
    P->async_stage = 2;
    return FS_OK;
  }
  P->async_stage = 0;  // the finish has landed: the state is on the host
  *done = 1;
  return solve_finish_read(P, P->async_timed_out, stats);
}

}  // extern "C"

namespace {

// y = A~ x on free nodes (unit diagonal, equilibrated masses), 0 elsewhere.
template <int K>
__global__ void __launch_bounds__(fs::kBlock)
    k_eq_apply(Dims d, const float* __restrict__ ex, const float* __restrict__ ey,
               const float* __restrict__ ez, const uint8_t* __restrict__ label,
               const float* __restrict__ x, float* __restrict__ y) {
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < d.N;
       n += (long long)gridDim.x * blockDim.x) {
    float ax[K];
    fs::apply_eq<float, K>(d, ex, ey, ez, x, n, ax);
    if (label[n] != FS_LABEL_FREE)
#pragma unroll
      for (int t = 0; t < K; ++t) ax[t] = 0.0f;
    fs::stv<float, K>(y, n, ax);
  }
}

}  // namespace

extern "C" {

int fs_eq_apply(const float* x, float* y, const float* ex, const float* ey, const float* ez,
                const uint8_t* label, int nx, int ny, int nz, int nrhs, void* stream) {
  if (!x || !y || !ex || !ey || !ez || !label || nx < 1 || ny < 1 || nz < 1) return FS_BAD_ARG;
  const Dims d = fs::make_dims(nx, ny, nz);
  cudaStream_t s = (cudaStream_t)stream;
#define FS_EQ(KK)                                                                  \
  case KK: {                                                                       \
    const int g = fs_grid_blocks((const void*)k_eq_apply<KK>, d.N);                \
    k_eq_apply<KK><<<g, fs::kBlock, 0, s>>>(d, ex, ey, ez, label, x, y);           \
    break;                                                                         \
  }
  switch (nrhs) {
    FS_EQ(1)
    FS_EQ(2)
    FS_EQ(4)
    FS_EQ(8)
    FS_EQ(16)
    default:
      return FS_BAD_ARG;
  }
#undef FS_EQ
  FS_CHECK_LAUNCH("k_eq_apply");
  return FS_OK;
}

int fs_pcg_plan_stencil_kind(const fs_pcg_plan* P) { return P ? P->stencil_kind : -1; }

int fs_pcg_plan_stencil_times(const fs_pcg_plan* P, float* ms) {
  if (!P || !ms) return FS_BAD_ARG;
  for (int c = 0; c < 8; ++c) ms[c] = P->tune_ms[c];
  return FS_OK;
}

int fs_pcg_plan_label_counts(const fs_pcg_plan* P, long long* counts, void* stream) {
  if (!P || !counts) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned long long h[4];
  FS_CHECK(cudaMemcpyAsync(h, P->ctl->label_counts, sizeof(h), cudaMemcpyDeviceToHost, s));
  FS_CHECK(cudaStreamSynchronize(s));
  for (int t = 0; t < 4; ++t) counts[t] = (long long)h[t];
  return FS_OK;
}

int fs_pcg_plan_scale(const fs_pcg_plan* P, const double** s64, const uint8_t** label) {
  if (!P || !s64 || !label) return FS_BAD_ARG;
  *s64 = P->s64;
  *label = P->label;
  return FS_OK;
}

int fs_pcg_plan_precondition(fs_pcg_plan* P, const void* r, void* z, void* stream) {
  if (!P || !r || !z) return FS_BAD_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (size_t)P->d.N * P->nrhs *
                       (P->precision == FS_PRECISION_MIXED ? sizeof(float) : sizeof(double));
  if (!P->precond) {  // Jacobi: the identity on the equilibrated system
    FS_CHECK(cudaMemcpyAsync(z, r, bytes, cudaMemcpyDeviceToDevice, s));
    return FS_OK;
  }
  if (P->learned >= 0) {
    fs_set_error_msg("fs_pcg_plan_precondition: the plan carries a learned level");
    return FS_BAD_ARG;
  }
  // the V-cycle kernels skip their work once a solve of this plan finished
  FS_CHECK(cudaMemsetAsync(&P->ctl->all_done, 0, sizeof(int), s));
  P->ext_b = r;
  if (!dispatch(P, 12, s)) return FS_BAD_ARG;
  FS_CHECK(cudaGetLastError());
  FS_CHECK(cudaMemcpyAsync(z, P->ext_z, bytes, cudaMemcpyDeviceToDevice, s));
  return FS_OK;
}

int fs_pcg_plan_levels(const fs_pcg_plan* P, int* nlev, int* dims) {
  if (!P || !nlev) return FS_BAD_ARG;
  *nlev = P->precond ? P->nlev : 1;
  if (dims)
    for (int l = 0; l < *nlev; ++l) {
      const Dims& d = P->precond ? P->lev[l].d : P->d;
      dims[3 * l] = d.nx;
      dims[3 * l + 1] = d.ny;
      dims[3 * l + 2] = d.nz;
    }
  return FS_OK;
}

int fs_pcg_plan_level_data(const fs_pcg_plan* P, int level, const void** em, const uint8_t** label,
                           const void** scale) {
  if (!P || !P->precond || level < 0 || level >= P->nlev || !em || !label) return FS_BAD_ARG;
  const MgLevel& L = P->lev[level];
  em[0] = level ? L.em[0] : P->ex;
  em[1] = level ? L.em[1] : P->ey;
  em[2] = level ? L.em[2] : P->ez;
  *label = level ? L.label : P->label;
  if (scale) *scale = level ? (const void*)L.s : nullptr;
  return FS_OK;
}

int fs_pcg_plan_unet_workspace_bytes(const fs_pcg_plan* P, int level, size_t* bytes) {
  if (!P || !bytes || !P->precond || P->precision != FS_PRECISION_MIXED || level < 0 ||
      level >= P->nlev)
    return FS_BAD_ARG;
  const Dims& d = P->lev[level].d;
  size_t nb = 0;
  const int st = fs_unet_workspace_bytes(d.nx, d.ny, d.nz, P->nrhs, 0, &nb);
  if (st != FS_OK) return st;
  const size_t vec = ((size_t)d.N * P->nrhs * sizeof(float) + 255) & ~(size_t)255;
  *bytes = ((nb + 255) & ~(size_t)255) + 2 * vec;
  return FS_OK;
}

int fs_pcg_plan_set_unet(fs_pcg_plan* P, int level, int mode, float* theta, void* workspace,
                         size_t workspace_bytes, void* stream) {
  if (!P || !P->precond || P->precision != FS_PRECISION_MIXED || level < -1 ||
      level >= P->nlev || mode < 0 || mode > 1) {
    fs_set_error_msg("learned preconditioner: needs a mixed-precision multigrid plan, a valid level and mode");
    return FS_BAD_ARG;
  }
  if (P->net) {
    fs_unet_destroy(P->net);
    P->net = nullptr;
  }
  P->learned = -1;
  P->net_u = P->net_r = nullptr;
  P->net_status = FS_OK;
  if (level >= 0) {
    if (!theta || !workspace || ((uintptr_t)workspace & 255)) return FS_BAD_ARG;
    const Dims& d = P->lev[level].d;
    size_t need = 0, nb = 0;
    int st = fs_pcg_plan_unet_workspace_bytes(P, level, &need);
    if (st != FS_OK) return st;
    if (workspace_bytes < need) {
      fs_set_error_msg("learned preconditioner: workspace too small");
      return FS_BAD_ARG;
    }
    st = fs_unet_workspace_bytes(d.nx, d.ny, d.nz, P->nrhs, 0, &nb);
    if (st != FS_OK) return st;
    nb = (nb + 255) & ~(size_t)255;
    const size_t vec = ((size_t)d.N * P->nrhs * sizeof(float) + 255) & ~(size_t)255;
    fs_unet* net = nullptr;
    st = fs_unet_create(d.nx, d.ny, d.nz, P->nrhs, 0, theta, workspace, nb, &net, stream);
    if (st != FS_OK) return st;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return fs_cuda_status("cudaStreamSynchronize", e);
    P->net = net;
    P->net_u = (uint8_t*)workspace + nb;
    P->net_r = (uint8_t*)workspace + nb + vec;
    P->learned = level;
    P->learned_mode = mode;
  }
  return capture_graph(P);
}

int fs_pcg_plan_sync_unet(fs_pcg_plan* P, void* stream) {
  if (!P || !P->net) return FS_BAD_ARG;
  return fs_unet_sync(P->net, stream);
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
  for (int t = 0; t < 6; ++t) ms[t] = P->kernel_ms[t];
  *samples = P->kernel_samples;
  return FS_OK;
}

int fs_pcg_plan_destroy(fs_pcg_plan* P) {
  if (!P) return FS_OK;
  if (P->net) fs_unet_destroy(P->net);
  for (int t = 0; t < 8; ++t)
    if (P->ev[t]) cudaEventDestroy(P->ev[t]);
  if (P->ev_async) cudaEventDestroy(P->ev_async);
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->body) cudaGraphExecDestroy(P->body);
  if (P->cap) cudaStreamDestroy(P->cap);
  if (P->slot) host_slot_put(P->slot);
  delete P;
  return FS_OK;
}

}  // extern "C"
