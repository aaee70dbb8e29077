// Krylov solvers of the SIMPLEC iteration on B200: CSR SpMV, Jacobi-preconditioned BiCGSTAB
// (flowtrace/linalg/krylov.py:68-121) and AMG-preconditioned CG (krylov.py:25-65 with the
// V-cycle of flowtrace/linalg/amg.py:130-146).
//
// Both solvers are single cooperative (persistent) launches: the whole iteration, its
// reductions and its stopping tests stay on the device, with grid-wide barriers between the
// phases and no host synchronisation. Control flow around every grid.sync() is uniform:
// each decision is taken from totals that every block computes from the same partial sums
// in the same order, so all blocks take identical branches, and every loop is bounded by
// maxiter. Partial sums alternate between two buffers so that a block writing the next
// reduction never overtakes a block still reading the previous one.
#include <mutex>

#include "b2s_common.cuh"

namespace b2s {

__device__ __forceinline__ double spmv_row(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                           const double* __restrict__ val, int i, const double* __restrict__ x) {
  double s = 0.0;
  for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) s += val[j] * x[col[j]];
  return s;
}

__global__ void spmv_k(int n, int k, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int j0 = rowptr[i], j1 = rowptr[i + 1];
    for (int c = 0; c < k; ++c) {
      const double* xc = x + (int64_t)c * n;
      double s = 0.0;
      for (int j = j0; j < j1; ++j) s += val[j] * xc[col[j]];
      y[(int64_t)c * n + i] = s;
    }
  }
}

// ---------------------------------------------------------------------------------- reductions
// Block-level sum of NQ values into the current partial buffer, a grid barrier, then the
// fixed-order totals into tot[] (shared) for every block.
template <int NQ>
__device__ __forceinline__ void grid_reduce(cg::grid_group& grid, const double (&v)[NQ], double* red, double* part,
                                            double* tot) {
  block_partials<NQ>(v, red, part);
  grid.sync();
  grid_totals(part, gridDim.x, NQ, tot);
}

// Entries of a row issued as one straight-line block (predicated on the row's length) before
// the rest are walked in a loop: their loads are in flight together.
constexpr int kRowUnroll = 8;

// Rows [0, n) of a grid phase, one thread per row: emit(i, s) with s[k] the sum over row i's
// entries j of entry(j, k). A row's entries are issued kRowUnroll at a time as one straight-line
// block so that their loads are in flight together; the sums keep the entries' stored order.
template <int NR, class Entry, class Emit>
__device__ __forceinline__ void walk_rows_nr(int n, int gt, int gs, const int32_t* __restrict__ rowptr, Entry entry,
                                             Emit emit) {
  for (int i = gt; i < n; i += gs) {
    const int ja = rowptr[i], jae = rowptr[i + 1];
    double sa[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) sa[k] = 0.0;
    for (int j = ja; j < jae; j += kRowUnroll) {
#pragma unroll
      for (int k = 0; k < kRowUnroll; ++k)
        if (j + k < jae) entry(j + k, sa);
    }
    emit(i, sa);
  }
}

// ---------------------------------------------------------------------------------- BiCGSTAB
// T is the storage type of the matrix values and the vectors (double, or float for the
// mixed-precision path); scalars and every reduction are accumulated in double.
template <class T>
struct BicgArgsT {
  int n, nr;
  const int32_t* rowptr;
  const int32_t* col;
  const T* val;
  const T* b;
  const T* inv;
  T* x;
  double tol;
  int maxiter, rel;
  int zero_x0;           // start from x = 0 (x is not read)
  T* work;
  double* part0;
  double* part1;
  b2s_solve_info* info;
  double* out64;         // when set: out64 = base64 + x at the end (a correction added in double)
  const double* base64;
};
using BicgArgs = BicgArgsT<double>;

enum { ACTIVE = 0, CONVERGED = 1, STOPPED = 2 };

// Three grid phases per iteration (the reference's algorithm has five dependent steps). The
// Jacobi-preconditioned vectors a neighbour's row needs are kept as u = inv r, w = inv (p - omega v)
// and z = inv v, so that every matrix entry gathers two values:
//   1. p = r + beta (p - omega v), h = inv p = u + beta w, v = A h with the neighbours' h
//      formed from their u and w, z = inv v; r_hat.v;
//   2. s = r - alpha v, hs = inv s = u - alpha z, t = A hs formed the same way; s.s, t.t, t.s
//      (t is wasted only on the iteration where |s| converges);
//   3. r = s - omega t, u = inv r, w = inv (p - omega v); r.r, r_hat.r.
// x gets alpha h + omega hs one phase later (after the breakdown test), as the reference does.
// Every row reads and writes only its own p, v, h, hs, s and t; u, w and z are written in the
// phase before the one that gathers them. Storage is T; the arithmetic is double.
template <int NR, class T>
__global__ void __launch_bounds__(kCoopThreads) bicgstab_coop_k(BicgArgsT<T> a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[(kCoopThreads / 32 + 1) * 3 * NR];
  __shared__ double tot[3 * NR];
  const int n = a.n;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  double* part[2] = {a.part0, a.part1};
  int pb = 0;
  T *r[NR], *rh[NR], *p[NR], *v[NR], *h[NR], *s[NR], *hs[NR], *t[NR], *u[NR], *w[NR], *z[NR], *x[NR];
  const T* b[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    T* wk = a.work + (int64_t)kBicgVectors * k * n;
    r[k] = wk;
    rh[k] = wk + n;
    p[k] = wk + 2 * (int64_t)n;
    v[k] = wk + 3 * (int64_t)n;
    h[k] = wk + 4 * (int64_t)n;
    s[k] = wk + 5 * (int64_t)n;
    hs[k] = wk + 6 * (int64_t)n;
    t[k] = wk + 7 * (int64_t)n;
    u[k] = wk + 8 * (int64_t)n;
    w[k] = wk + 9 * (int64_t)n;
    z[k] = wk + 10 * (int64_t)n;
    x[k] = a.x + (int64_t)k * n;
    b[k] = a.b + (int64_t)k * n;
  }
  const T* inv = a.inv;
  // ---- r = b - A x, r_hat = r, u = inv r, p = v = w = 0
  {
    double acc[3 * NR];
#pragma unroll
    for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
    for (int i = gt; i < n; i += gs) {
      const int j0 = a.rowptr[i], j1 = a.rowptr[i + 1];
      const double iv = inv[i];
      double ax[NR];
#pragma unroll
      for (int k = 0; k < NR; ++k) ax[k] = 0.0;
      if (!a.zero_x0) {
        for (int j = j0; j < j1; ++j) {
          const double av = a.val[j];
          const int c = a.col[j];
#pragma unroll
          for (int k = 0; k < NR; ++k) ax[k] += av * x[k][c];
        }
      }
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        const double bi = b[k][i], ri = bi - ax[k];
        if (a.zero_x0) x[k][i] = 0.0;
        r[k][i] = ri;
        rh[k][i] = ri;
        u[k][i] = iv * ri;
        p[k][i] = 0.0;
        v[k][i] = 0.0;
        w[k][i] = 0.0;
        acc[k] += ri * ri;
        acc[NR + k] += bi * bi;
      }
    }
    grid_reduce<3 * NR>(grid, acc, red, part[pb], tot);
    pb ^= 1;
  }
  int st[NR], its[NR];
  bool pend[NR], pend_a[NR];
  double rho[NR], alpha[NR], omega[NR], bnorm[NR], babs[NR], rnorm[NR], res[NR], rho_new[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const double rr = tot[k], bb = tot[NR + k];
    rnorm[k] = sqrt(rr);
    babs[k] = sqrt(bb);
    bnorm[k] = a.rel ? rnorm[k] : babs[k];
    if (bnorm[k] == 0.0) bnorm[k] = 1.0;
    st[k] = ACTIVE;
    its[k] = 0;
    res[k] = rnorm[k] / bnorm[k];
    if (rnorm[k] / bnorm[k] < a.tol || rnorm[k] <= 1e-14 * babs[k]) st[k] = CONVERGED;
    rho[k] = alpha[k] = omega[k] = 1.0;
    rho_new[k] = rr;
    pend[k] = pend_a[k] = false;
  }
  __syncthreads();
  for (int it = 1; it <= a.maxiter; ++it) {
    bool any = false;
    double beta[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      beta[k] = 0.0;
      if (st[k] != ACTIVE) continue;
      if (rho_new[k] == 0.0) {
        st[k] = STOPPED;
        its[k] = it;
        res[k] = rnorm[k] / bnorm[k];
        continue;
      }
      beta[k] = (rho_new[k] / rho[k]) * (alpha[k] / omega[k]);
      rho[k] = rho_new[k];
      any = true;
    }
    // ---- phase 1: deferred x update; p, h, v = A h, z = inv v; r_hat.v
    {
      double acc[3 * NR];
#pragma unroll
      for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
      auto xupd = [&](int i) {
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (pend[k]) x[k][i] = (x[k][i] + alpha[k] * h[k][i]) + omega[k] * hs[k][i];
      };
      if (!any) {
        for (int i = gt; i < n; i += gs) xupd(i);
      } else {
        walk_rows_nr<NR>(
            n, gt, gs, a.rowptr,
            [&](int j, double (&sv)[NR]) {
              const double aij = a.val[j];
              const int c = a.col[j];
#pragma unroll
              for (int k = 0; k < NR; ++k)
                if (st[k] == ACTIVE) sv[k] += aij * ((double)u[k][c] + beta[k] * w[k][c]);
            },
            [&](int i, const double (&av_)[NR]) {
              xupd(i);
              const double iv = inv[i];
#pragma unroll
              for (int k = 0; k < NR; ++k)
                if (st[k] == ACTIVE) {
                  p[k][i] = r[k][i] + beta[k] * (p[k][i] - omega[k] * v[k][i]);
                  h[k][i] = (double)u[k][i] + beta[k] * w[k][i];
                  v[k][i] = av_[k];
                  z[k][i] = iv * av_[k];
                  acc[k] += rh[k][i] * av_[k];
                }
            });
      }
#pragma unroll
      for (int k = 0; k < NR; ++k) pend[k] = false;
      if (!any) break;
      grid_reduce<3 * NR>(grid, acc, red, part[pb], tot);
      pb ^= 1;
    }
    any = false;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (st[k] != ACTIVE) continue;
      const double denom = tot[k];
      if (denom == 0.0) {
        st[k] = STOPPED;
        its[k] = it;
        res[k] = rnorm[k] / bnorm[k];
        continue;
      }
      alpha[k] = rho[k] / denom;
      any = true;
    }
    __syncthreads();
    if (!any) break;
    // ---- phase 2: s = r - alpha v, hs = u - alpha z, t = A hs; s.s, t.t, t.s
    {
      double acc[3 * NR];
#pragma unroll
      for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
      walk_rows_nr<NR>(
          n, gt, gs, a.rowptr,
          [&](int j, double (&sv)[NR]) {
            const double aij = a.val[j];
            const int c = a.col[j];
#pragma unroll
            for (int k = 0; k < NR; ++k)
              if (st[k] == ACTIVE) sv[k] += aij * ((double)u[k][c] - alpha[k] * z[k][c]);
          },
          [&](int i, const double (&at)[NR]) {
#pragma unroll
            for (int k = 0; k < NR; ++k)
              if (st[k] == ACTIVE) {
                const double si = r[k][i] - alpha[k] * v[k][i];
                s[k][i] = si;
                hs[k][i] = (double)u[k][i] - alpha[k] * z[k][i];
                t[k][i] = at[k];
                acc[k] += si * si;
                acc[NR + k] += at[k] * at[k];
                acc[2 * NR + k] += at[k] * si;
              }
          });
      grid_reduce<3 * NR>(grid, acc, red, part[pb], tot);
      pb ^= 1;
    }
    any = false;
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (st[k] != ACTIVE) continue;
      const double sn = sqrt(tot[k]);
      if (sn / bnorm[k] < a.tol) {
        st[k] = CONVERGED;
        its[k] = it;
        res[k] = sn / bnorm[k];
        pend_a[k] = true;  // x += alpha h
        continue;
      }
      omega[k] = tot[NR + k] > 0.0 ? tot[2 * NR + k] / tot[NR + k] : 0.0;
      any = true;
    }
    __syncthreads();
    // ---- phase 3: r = s - omega t, u = inv r, w = inv (p - omega v); r.r, r_hat.r (systems
    // converged in phase 2 take x += alpha h)
    {
      double acc[3 * NR];
#pragma unroll
      for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
      for (int i = gt; i < n; i += gs) {
        const double iv = inv[i];
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          if (pend_a[k]) x[k][i] = x[k][i] + alpha[k] * h[k][i];
          if (st[k] == ACTIVE) {
            const double ri = s[k][i] - omega[k] * t[k][i];
            r[k][i] = ri;
            u[k][i] = iv * ri;
            w[k][i] = iv * (p[k][i] - omega[k] * v[k][i]);
            acc[k] += ri * ri;
            acc[NR + k] += rh[k][i] * ri;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < NR; ++k) pend_a[k] = false;
      if (!any) break;
      grid_reduce<3 * NR>(grid, acc, red, part[pb], tot);
      pb ^= 1;
    }
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (st[k] != ACTIVE) continue;
      const double rn = sqrt(tot[k]);
      if (!isfinite(rn)) {  // breakdown: keep the last finite iterate
        st[k] = STOPPED;
        its[k] = it;
        res[k] = nan("");
        continue;
      }
      rnorm[k] = rn;
      pend[k] = true;
      rho_new[k] = tot[NR + k];
      if (rn / bnorm[k] < a.tol || rn <= 1e-14 * babs[k]) {
        st[k] = CONVERGED;
        its[k] = it;
        res[k] = rn / bnorm[k];
      } else if (omega[k] == 0.0) {
        st[k] = STOPPED;
        its[k] = it;
        res[k] = rn / bnorm[k];
      }
    }
    __syncthreads();
  }
  // epilogue: pending updates; systems still active ran out of iterations
  for (int i = gt; i < n; i += gs) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (pend_a[k]) x[k][i] = x[k][i] + alpha[k] * h[k][i];
      if (pend[k]) x[k][i] = (x[k][i] + alpha[k] * h[k][i]) + omega[k] * hs[k][i];
      if (a.out64) a.out64[(int64_t)k * n + i] = a.base64[(int64_t)k * n + i] + (double)x[k][i];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (st[k] == ACTIVE) {
        its[k] = a.maxiter;
        res[k] = rnorm[k] / bnorm[k];
      }
      a.info[k].iterations = its[k];
      a.info[k].converged = st[k] == CONVERGED ? 1 : 0;
      a.info[k].residual = res[k];
    }
  }
}

// ---------------------------------------------------------------------------------- AMG-PCG
// T is the storage type of the level matrices and the V-cycle/CG vectors: double, or float on
// the mixed-precision path. Scalars, reductions and the coarse solve's arithmetic stay double.
template <class T>
struct VBufT {  // per-level V-cycle vectors
  T* b;
  T* x;
  T* y;
  T* r;
};

template <class T>
struct LvVals {  // per-level values in the storage type
  const T* val;
  const T* dinv;
  const T* p_val;
  const T* r_val;
};

template <class T>
struct PcgArgsT {
  b2s_amg h;
  LvVals<T> lvv[B2S_AMG_MAX_LEVELS];
  int n;                 // the operator A (the current matrix)
  const int32_t* rowptr;
  const int32_t* col;
  const T* val;
  const T* b;
  T* x;
  double tol;
  int maxiter, project;
  T* r;
  T* p;
  T* p2;
  T* q;
  T* cb;   // coarse right-hand side
  T* cx;   // coarse solution
  double* part0;
  double* part1;
  VBufT<T> lv[B2S_AMG_MAX_LEVELS];
  b2s_solve_info* info;
  int csize;    // blocks per thread-block cluster of the launch (0: no clusters)
  int sub_nnz;  // largest level (entries) run on the subset of the grid (first cluster or block 0)
};
using PcgArgs = PcgArgsT<double>;

// Rows of a V-cycle phase, walked by groups of g lanes (g a power of two, 1..32): a group takes
// a row, its lanes stride the row's entries, and an xor-shuffle tree over the group sums them.
// A phase is latency-bound when one group walks many rows one after another, so g is the
// largest size that still leaves at most one row per group (the phase's threads over the rows),
// capped by the mean row length (no more lanes than entries) and raised to keep at most 32
// entries per lane. Whole warps step through the rows together (a row index past the end
// contributes nothing) so every lane takes part in the shuffles. The phase's thread count and
// the warps' first thread indices are multiples of 32.
struct Rows {
  int first, stride, sub, lane, g;
  __device__ __forceinline__ Rows(int n, int64_t nnz, int t, int nthreads) {
    const int64_t avg = n > 0 ? (nnz + n - 1) / n : 1;
    int gg = 1;
    while (gg < 32 && (int64_t)n * (gg * 2) <= nthreads && avg > gg) gg <<= 1;
    while (gg < 32 && avg > 32 * (int64_t)gg) gg <<= 1;
    g = gg;
    const int gpw = 32 / gg;
    first = (t >> 5) * gpw;
    stride = (nthreads >> 5) * gpw;
    sub = (t & 31) / gg;
    lane = (t & 31) & (gg - 1);
  }
  __device__ __forceinline__ double total(double s) const {
    for (int o = g >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
  }
  __device__ __forceinline__ bool writer() const { return lane == 0; }
};

// The rows [0, n) of a phase: emit(i, sum over row i's entries j of entry(j)). With one lane per
// row and more rows than lanes, two rows are walked together, kRowUnroll entries of both at a
// time in one straight-line block, so that both rows' loads are in flight at once. Otherwise a
// lane takes kRowUnroll of its row's entries (every g-th) at a time the same way. Each row's
// sum keeps the entries' stored order per lane (then the group's xor tree), and every lane
// emits its rows in increasing order.
template <class Entry, class Emit>
__device__ __forceinline__ void walk_rows(const Rows& R, int n, const int32_t* __restrict__ rowptr, Entry entry,
                                          Emit emit) {
  if (R.g == 1 && n > R.stride) {
    for (int i0 = R.first; i0 < n; i0 += 2 * R.stride) {
      const int ia = i0 + R.sub, ib = ia + R.stride;
      int ja = 0, jae = 0, jb = 0, jbe = 0;
      if (ia < n) {
        ja = ldro(rowptr + ia);
        jae = ldro(rowptr + ia + 1);
      }
      if (ib < n) {
        jb = ldro(rowptr + ib);
        jbe = ldro(rowptr + ib + 1);
      }
      double sa = 0.0, sb = 0.0;
      while (ja < jae || jb < jbe) {
#pragma unroll
        for (int k = 0; k < kRowUnroll; ++k) {
          if (ja + k < jae) sa += entry(ja + k);
          if (jb + k < jbe) sb += entry(jb + k);
        }
        ja += kRowUnroll;
        jb += kRowUnroll;
      }
      if (ia < n) emit(ia, sa);
      if (ib < n) emit(ib, sb);
    }
  } else {
    for (int i0 = R.first; i0 < n; i0 += R.stride) {
      const int i = i0 + R.sub;
      const bool act = i < n;
      double s = 0.0;
      if (act) {
        const int je = ldro(rowptr + i + 1);
        for (int j = ldro(rowptr + i) + R.lane; j < je; j += kRowUnroll * R.g) {
#pragma unroll
          for (int k = 0; k < kRowUnroll; ++k)
            if (j + k * R.g < je) s += entry(j + k * R.g);
        }
      }
      s = R.total(s);
      if (act && R.writer()) emit(i, s);
    }
  }
}

// One damped-Jacobi step y = x + (w Dinv)(b - A x); x == NULL means x = w Dinv b (fused).
template <class T>
__device__ __forceinline__ void jacobi_step(const b2s_amg_level& L, const LvVals<T>& V, double w, const T* b,
                                            const T* x, T* y, int gt, int gs) {
  const Rows R(L.n, L.nnz, gt, gs);
  auto emit = [&](int i, double s) {
    const double wd = w * ldro(V.dinv + i);
    const double xi = x ? (double)x[i] : wd * b[i];
    y[i] = xi + wd * (b[i] - s);
  };
  if (x) {
    walk_rows(R, L.n, L.rowptr, [&](int j) { return (double)ldro(V.val + j) * x[ldro(L.col + j)]; }, emit);
  } else {
    walk_rows(R, L.n, L.rowptr, [&](int j) {
      const int c = ldro(L.col + j);
      return (double)ldro(V.val + j) * ((w * ldro(V.dinv + c)) * b[c]);
    }, emit);
  }
}

// Barrier of a V-cycle phase: the whole grid for the large levels, block 0 alone for the tail.
// kGrid: every block; kBlock: block 0 alone (block barriers); kCluster: the blocks of the
// launch's first thread-block cluster (cluster barriers, which also order the cluster's global
// memory accesses).
enum { kGrid = 0, kBlock = 1, kCluster = 2 };
struct Phase {
  cg::grid_group* grid;
  int kind;
  int t, n;  // this thread's index and the number of threads in the phase
  __device__ __forceinline__ void sync() const {
    if (kind == kBlock) __syncthreads();
    else if (kind == kCluster) cg::this_cluster().sync();
    else grid->sync();
  }
};

// The first sweep from x = 0, x1 = w D^-1 b (amg.py:135), of level l's row i, stored by the
// phase that produces row i of b (the PCG residual update for level 0, the restriction for the
// coarser levels) into the level's y buffer, so that the pre-smoothing phase gathers one value
// per matrix entry instead of two. Same arithmetic as evaluating it on the fly.
template <class T>
__device__ __forceinline__ void store_first_sweep(const PcgArgsT<T>& a, int l, int i, T bi) {
  a.lv[l].y[i] = (T)((a.h.omega * (double)ldro(a.lvv[l].dinv + i)) * (double)bi);
}

// Down-leg of level l (amg.py:135-139): pre-smoothing, residual, restriction to the next level.
// The first two sweeps are one phase: with pre, the first sweep x1 = w D^-1 b is already in the
// level's y buffer (store_first_sweep); otherwise it is evaluated on the fly for each neighbour.
// The restriction also stores the next level's first sweep.
template <class T>
__device__ __forceinline__ T* vdown(const PcgArgsT<T>& a, int l, const T* b, const Phase& ph, bool pre) {
  const b2s_amg& h = a.h;
  const b2s_amg_level& lv = h.levels[l];
  const LvVals<T>& V = a.lvv[l];
  const int L = h.nlevels;
  const double w = h.omega;
  T* X = a.lv[l].x;
  T* Y = a.lv[l].y;
  T* c = X;
  if (h.sweeps <= 1) {
    for (int i = ph.t; i < lv.n; i += ph.n) X[i] = (w * ldro(V.dinv + i)) * b[i];
  } else {
    jacobi_step(lv, V, w, b, pre ? (const T*)Y : (const T*)nullptr, X, ph.t, ph.n);
    T* o = Y;
    for (int sw = 2; sw < h.sweeps; ++sw) {
      ph.sync();
      jacobi_step(lv, V, w, b, (const T*)c, o, ph.t, ph.n);
      T* tmp = c;
      c = o;
      o = tmp;
    }
  }
  ph.sync();
  T* Rv = a.lv[l].r;
  walk_rows(Rows(lv.n, lv.nnz, ph.t, ph.n), lv.n, lv.rowptr,
            [&](int j) { return (double)ldro(V.val + j) * c[ldro(lv.col + j)]; },
            [&](int i, double s) { Rv[i] = b[i] - s; });
  ph.sync();
  T* bn = (l + 1 < L) ? a.lv[l + 1].b : a.cb;
  const bool pre_next = l + 1 < L && h.sweeps >= 2;
  walk_rows(Rows(lv.nc, lv.p_nnz, ph.t, ph.n), lv.nc, lv.r_rowptr,
            [&](int j) { return (double)ldro(V.r_val + j) * Rv[ldro(lv.r_col + j)]; },
            [&](int I, double s) {
              bn[I] = s;
              if (pre_next) store_first_sweep(a, l + 1, I, (T)s);
            });
  ph.sync();
  return c;
}

// Up-leg of level l (amg.py:139-142): x += P xc, then the post-smoothing sweeps. With stats
// (level 0 on the grid) the last sweep also accumulates sum z, sum r z and sum r for the PCG
// and ends with their grid-wide reduction into stats.
template <class T>
__device__ __forceinline__ T* vup(const PcgArgsT<T>& a, int l, const T* b, T* c, const T* xc, const Phase& ph,
                                  const T* rr, double* red, double* stats, int pb) {
  const b2s_amg& h = a.h;
  const b2s_amg_level& lv = h.levels[l];
  const LvVals<T>& V = a.lvv[l];
  const double w = h.omega;
  T* o = (c == a.lv[l].x) ? a.lv[l].y : a.lv[l].x;
  const bool want = stats != nullptr;
  double acc[3] = {0.0, 0.0, 0.0};
  walk_rows(Rows(lv.n, lv.p_nnz, ph.t, ph.n), lv.n, lv.p_rowptr,
            [&](int j) { return (double)ldro(V.p_val + j) * xc[ldro(lv.p_col + j)]; },
            [&](int i, double s) {
              const double zi = c[i] + s;
              c[i] = zi;
              if (want && h.sweeps == 0) {
                acc[0] += zi;
                acc[1] += rr[i] * zi;
                acc[2] += rr[i];
              }
            });
  const Rows R(lv.n, lv.nnz, ph.t, ph.n);
  for (int sw = 0; sw < h.sweeps; ++sw) {
    ph.sync();
    const bool last = sw + 1 == h.sweeps;
    walk_rows(R, lv.n, lv.rowptr, [&](int j) { return (double)ldro(V.val + j) * c[ldro(lv.col + j)]; },
              [&](int i, double s) {
                const double zi = c[i] + (w * ldro(V.dinv + i)) * (b[i] - s);
                o[i] = zi;
                if (want && last) {
                  acc[0] += zi;
                  acc[1] += rr[i] * zi;
                  acc[2] += rr[i];
                }
              });
    T* tmp = c;
    c = o;
    o = tmp;
  }
  if (want) {
    block_partials<3>(acc, red, pb ? a.part1 : a.part0);
    ph.grid->sync();
    grid_totals(pb ? a.part1 : a.part0, gridDim.x, 3, stats);
  } else {
    ph.sync();
  }
  return c;
}

// Coarse solve cx = inv(Ac) cb, one warp per row; the inverse and the arithmetic are double.
template <class T>
__device__ __forceinline__ void vcoarse(const PcgArgsT<T>& a, const T* cb, const Phase& ph) {
  const int nc = a.h.coarse_n, lane = threadIdx.x & 31;
  for (int I = ph.t >> 5; I < nc; I += ph.n >> 5) {
    const double* row = a.h.coarse_inv + (int64_t)I * nc;
    double s = 0.0;
    for (int J = lane; J < nc; J += 32 * kRowUnroll) {
#pragma unroll
      for (int k = 0; k < kRowUnroll; ++k)
        if (J + 32 * k < nc) s += ldro(row + J + 32 * k) * cb[J + 32 * k];
    }
    s = warp_sum(s);
    if (lane == 0) a.cx[I] = s;
  }
  ph.sync();
}

// Buffer holding level l's solution after its up-leg: the down-leg ends in x after sweeps-2
// ping-pong swaps (x alone for one sweep), the up-leg swaps once per sweep. Every block can thus
// name the buffer without having run the level.
template <class T>
__device__ __forceinline__ T* tail_result(const PcgArgsT<T>& a, int l) {
  const int sw = a.h.sweeps;
  const int down = sw <= 1 ? 0 : sw - 2;
  return ((down + sw) & 1) ? a.lv[l].y : a.lv[l].x;
}

// The small end of the hierarchy runs on a subset of the grid while the other blocks wait at
// the next grid barrier. A phase costs about a barrier (grid ~1.3 us, cluster ~0.35 us, block
// ~0.05 us on B200) plus its gathers, which an SM issues at roughly one scattered cache line per
// cycle: a level of E entries is worth moving from the 148 SMs to a subset of S SMs when
// E (1/S - 1/148) / 2 ns is below the barrier time saved. The subset is the launch's first
// thread-block cluster when the launch is made of clusters (PcgArgsT::csize > 0), else block 0;
// it takes every level (and the coarse solve) with at most PcgArgsT::sub_nnz entries (matrix,
// prolongation; coarse_n^2 for the coarse solve) and at most 4 rows per thread.
constexpr int kSubRowsPerThread = 4;

// z = M r: the V-cycle of flowtrace/linalg/amg.py:130-142. Returns the buffer holding z. pre0:
// the caller stored level 0's first sweep from rhs0 (store_first_sweep) when it wrote rhs0. With
// stats != nullptr, when level 0 runs on the whole grid, stats[0..2] receive sum z, sum r z and
// sum r (r = rhs0) and *have_stats is set; otherwise the caller reduces them itself.
template <class T>
__device__ T* vcycle(cg::grid_group& grid, const PcgArgsT<T>& a, const T* rhs0, bool pre0, int gt, int gs,
                     double* red = nullptr, double* stats = nullptr, int pb = 0, bool* have_stats = nullptr) {
  const b2s_amg& h = a.h;
  const int L = h.nlevels;
  T* cur[B2S_AMG_MAX_LEVELS];
  const T* cb = (L == 0) ? rhs0 : a.cb;
  const bool cl = a.csize > 0;
  const int64_t sub_rows = (int64_t)(cl ? a.csize : 1) * blockDim.x * kSubRowsPerThread;
  const int64_t sub_nnz = a.sub_nnz;
  int Lg = L;  // levels from Lg on (all small) run on the subset; the others on the whole grid
  while (Lg > 0 && h.levels[Lg - 1].n <= sub_rows && h.levels[Lg - 1].nnz <= sub_nnz &&
         h.levels[Lg - 1].p_nnz <= sub_nnz)
    --Lg;
  const bool sub_coarse = (int64_t)h.coarse_n * h.coarse_n <= sub_nnz;
  const Phase gph = {&grid, kGrid, gt, gs};
  const Phase sph = cl ? Phase{&grid, kCluster, (int)(blockIdx.x * blockDim.x + threadIdx.x), a.csize * (int)blockDim.x}
                       : Phase{&grid, kBlock, (int)threadIdx.x, (int)blockDim.x};
  const bool in_sub = cl ? (int)blockIdx.x < a.csize : blockIdx.x == 0;
  for (int l = 0; l < Lg; ++l) cur[l] = vdown(a, l, (l == 0) ? rhs0 : (const T*)a.lv[l].b, gph, l > 0 || pre0);
  if (Lg == L && !sub_coarse) {
    vcoarse(a, cb, gph);
  } else {
    if (in_sub) {
      for (int l = Lg; l < L; ++l) cur[l] = vdown(a, l, (l == 0) ? rhs0 : (const T*)a.lv[l].b, sph, l > 0 || pre0);
      vcoarse(a, cb, sph);
      for (int l = L - 1; l >= Lg; --l)
        cur[l] = vup(a, l, (l == 0) ? rhs0 : (const T*)a.lv[l].b, cur[l], (const T*)((l + 1 < L) ? cur[l + 1] : a.cx),
                     sph, (const T*)nullptr, nullptr, nullptr, 0);
    }
    grid.sync();
  }
  for (int l = Lg - 1; l >= 0; --l) {
    const T* xc;
    if (l + 1 < L) {
      // the next level's solution: every block tracks it on the grid levels; for the first level
      // run by the subset every block names it from the sweep parity
      if (l + 1 < Lg) xc = cur[l + 1];
      else xc = tail_result(a, l + 1);
    } else {
      xc = a.cx;
    }
    const bool st = (l == 0) && stats != nullptr;
    cur[l] = vup(a, l, (l == 0) ? rhs0 : (const T*)a.lv[l].b, cur[l], xc, gph, rhs0, st ? red : nullptr,
                 st ? stats : nullptr, pb);
    if (st && have_stats) *have_stats = true;
  }
  if (L == 0) return a.cx;
  if (Lg == 0) return tail_result(a, 0);
  return cur[0];
}

struct CgOutcome {
  int its, conv;
  double res;
};

// Preconditioned CG (flowtrace/linalg/krylov.py:25-65) of A x = b from x = 0, with a.r, a.p,
// a.p2, a.q as work vectors. Per iteration: one phase computes p = z' + beta p_old into a
// second buffer and q = A p with the neighbours' p evaluated on the fly (same arithmetic), one
// phase updates x and r, then the V-cycle, whose last sweep also reduces sum z, sum r z and
// sum r; z' = z - mean(z) (the projection) is applied lazily and r.z' = sum r z - mean(z) sum r.
// pb is the partial buffer to use next (updated).
template <class T>
__device__ CgOutcome pcg_core(cg::grid_group& grid, const PcgArgsT<T>& a, const T* bvec, T* x, double tol,
                              int maxiter, double* red, double* tot, double* stats, int& pb) {
  const int n = a.n;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  double* part[2] = {a.part0, a.part1};
  const bool pre0 = a.h.nlevels > 0 && a.h.sweeps >= 2;  // level 0's first sweep stored with r
  T* r = a.r;
  T* q = a.q;
  T* pbuf[2] = {a.p, a.p2};
  int pc = 0;
  const double nd = (double)n;
  double bb, rr;
  {
    double acc[2] = {0.0, 0.0};
    for (int i = gt; i < n; i += gs) {
      const double bi = bvec[i];
      x[i] = 0.0;
      r[i] = bi;
      if (pre0 && !a.project) store_first_sweep(a, 0, i, (T)bi);
      acc[0] += bi * bi;
      acc[1] += bi;
    }
    grid_reduce<2>(grid, acc, red, part[pb], tot);
    pb ^= 1;
    bb = tot[0];
    rr = bb;
    if (a.project) {
      const double mean = tot[1] / nd;
      double acc2[2] = {0.0, 0.0};
      for (int i = gt; i < n; i += gs) {
        const double ri = r[i] - mean;
        r[i] = ri;
        if (pre0) store_first_sweep(a, 0, i, (T)ri);
        acc2[0] += ri * ri;
      }
      __syncthreads();
      grid_reduce<2>(grid, acc2, red, part[pb], tot);
      pb ^= 1;
      rr = tot[0];
    }
  }
  double bnorm = sqrt(bb);
  if (bnorm == 0.0) bnorm = 1.0;
  double rnorm = sqrt(rr);
  int its = 0, conv = 0;
  double res = rnorm / bnorm;
  bool done = false;
  if (rnorm / bnorm < tol) {
    conv = 1;
    done = true;
  }
  // z = M r with the statistics of its projection
  double rz = 0.0, zm = 0.0;
  T* z = nullptr;
  auto precondition = [&]() {
    __syncthreads();
    bool have = false;
    z = vcycle(grid, a, (const T*)r, pre0, gt, gs, red, stats, pb, &have);
    double sz, srz, sr;
    if (have) {
      pb ^= 1;
      sz = stats[0];
      srz = stats[1];
      sr = stats[2];
    } else {
      double acc[3] = {0.0, 0.0, 0.0};
      for (int i = gt; i < n; i += gs) {
        const double zi = z[i], ri = r[i];
        acc[0] += zi;
        acc[1] += ri * zi;
        acc[2] += ri;
      }
      grid_reduce<3>(grid, acc, red, part[pb], tot);
      pb ^= 1;
      sz = tot[0];
      srz = tot[1];
      sr = tot[2];
    }
    zm = a.project ? sz / nd : 0.0;
    __syncthreads();
    return a.project ? srz - zm * sr : srz;
  };
  if (!done) rz = precondition();
  double beta = 0.0;
  bool first = true;
  for (int k = 1; k <= maxiter && !done; ++k) {
    // p = z' + beta p_old (z' on the first iteration); q = A p; p.q
    T* pn = pbuf[pc];
    const T* po = pbuf[pc ^ 1];
    {
      double acc[2] = {0.0, 0.0};
      walk_rows_nr<1>(
          n, gt, gs, a.rowptr,
          [&](int j, double (&sv)[1]) {
            const int c = ldro(a.col + j);
            const double pj = first ? z[c] - zm : (z[c] - zm) + beta * po[c];
            sv[0] += ldro(a.val + j) * pj;
          },
          [&](int i, const double (&sv)[1]) {
            const double pi = first ? z[i] - zm : (z[i] - zm) + beta * po[i];
            pn[i] = pi;
            q[i] = sv[0];
            acc[0] += pi * sv[0];
          });
      grid_reduce<2>(grid, acc, red, part[pb], tot);
      pb ^= 1;
    }
    first = false;
    pc ^= 1;
    const double pAp = tot[0];
    __syncthreads();
    if (pAp <= 0.0) {
      its = k;
      res = rnorm / bnorm;
      done = true;
      break;
    }
    const double alpha = rz / pAp;
    {
      double acc[2] = {0.0, 0.0};
      for (int i = gt; i < n; i += gs) {
        x[i] = x[i] + alpha * pn[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        if (pre0) store_first_sweep(a, 0, i, (T)ri);
        acc[0] += ri * ri;
      }
      grid_reduce<2>(grid, acc, red, part[pb], tot);
      pb ^= 1;
    }
    rnorm = sqrt(tot[0]);
    __syncthreads();
    if (rnorm / bnorm < tol) {
      its = k;
      res = rnorm / bnorm;
      conv = 1;
      done = true;
      break;
    }
    const double rz_new = precondition();
    if (rz == 0.0) {
      its = k;
      res = rnorm / bnorm;
      done = true;
      break;
    }
    beta = rz_new / rz;
    rz = rz_new;
    its = k;
    res = rnorm / bnorm;
  }
  return {its, conv, res};
}

__global__ void __launch_bounds__(kCoopThreads) pcg_amg_coop_k(PcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[(kCoopThreads / 32 + 1) * 3];
  __shared__ double tot[3];
  __shared__ double stats[3];
  int pb = 0;
  const CgOutcome o = pcg_core(grid, a, a.b, a.x, a.tol, a.maxiter, red, tot, stats, pb);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.info->iterations = o.its;
    a.info->converged = o.conv;
    a.info->residual = o.res;
  }
}

// ---------------------------------------------------------------------------------- mixed PCG
// Mixed-precision pressure-correction solve: the AMG-PCG above in float (level matrices, the
// operator and the vectors in float; reductions and the coarse solve in double) inside an
// iterative-refinement loop kept in double: x64 += the float correction, then the true residual
// r64 = b - A x64 is evaluated in double from the double face coefficients (A x)_c =
// sum_f cf_f (x_c - x_nb) + sum_b cb_b x_c, the operator the pressure assembly defines
// (diag = sum cf + sum cb, off-diagonals -cf). The stopping test is the reference's,
// |r| / |b| < tol with r projected when the system is singular, on r64.
struct PcgMixedArgs {
  PcgArgsT<float> a;     // the float solver; a.b is the float right-hand side of each pass
  b2s_mesh m;            // cell/face topology of the operator
  const double* cf;      // [nf] interior face coefficients
  const double* cbf;     // [nb] boundary face coefficients
  const double* b64;     // [n] right-hand side
  double* x64;           // [n] solution
  double* r64;           // [n] work: the double residual
  float* rb32;           // [n] work: the float right-hand side of a pass
  float* d32;            // [n] work: the float correction of a pass
  double tol;
  int maxiter, maxpass;
  double min_inner_tol;  // floor of a pass's relative tolerance (the float solver's reach)
};

__global__ void __launch_bounds__(kCoopThreads) pcg_mixed_coop_k(PcgMixedArgs M) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[(kCoopThreads / 32 + 1) * 3];
  __shared__ double tot[3];
  __shared__ double stats[3];
  const PcgArgsT<float>& a = M.a;
  const b2s_mesh& m = M.m;
  const int n = a.n;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  double* part[2] = {a.part0, a.part1};
  int pb = 0;
  const double nd = (double)n;
  double bb, sb;
  {
    double acc[2] = {0.0, 0.0};
    for (int i = gt; i < n; i += gs) {
      const double bi = M.b64[i];
      M.x64[i] = 0.0;
      acc[0] += bi * bi;
      acc[1] += bi;
    }
    grid_reduce<2>(grid, acc, red, part[pb], tot);
    pb ^= 1;
    bb = tot[0];
    sb = tot[1];
  }
  double bnorm = sqrt(bb);
  if (bnorm == 0.0) bnorm = 1.0;
  // pass 0 residual: r = b (projected)
  double mean = a.project ? sb / nd : 0.0;
  double rr;
  {
    double acc[2] = {0.0, 0.0};
    for (int i = gt; i < n; i += gs) {
      const double ri = M.b64[i] - mean;
      M.r64[i] = ri;
      M.rb32[i] = (float)ri;
      acc[0] += ri * ri;
    }
    __syncthreads();
    grid_reduce<2>(grid, acc, red, part[pb], tot);
    pb ^= 1;
    rr = tot[0];
  }
  double res = sqrt(rr) / bnorm;
  int its = 0, conv = res < M.tol ? 1 : 0;
  for (int pass = 0; pass < M.maxpass && !conv && its < M.maxiter; ++pass) {
    double tin = M.tol / res;
    if (tin < M.min_inner_tol) tin = M.min_inner_tol;
    __syncthreads();
    const CgOutcome o = pcg_core(grid, a, (const float*)M.rb32, M.d32, tin, M.maxiter - its, red, tot, stats, pb);
    its += o.its;
    // x64 += d; then r64 = b - A x64 in double, its sum and sum of squares
    for (int i = gt; i < n; i += gs) M.x64[i] = M.x64[i] + (double)M.d32[i];
    grid.sync();
    double acc[2] = {0.0, 0.0};
    for (int c = gt; c < n; c += gs) {
      const double xc = M.x64[c];
      double ax = 0.0;
      for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) ax += M.cf[f] * (xc - M.x64[m.fN[f]]);
      for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
        const int f = m.nei_face[k];
        ax += M.cf[f] * (xc - M.x64[m.fP[f]]);
      }
      for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) ax += M.cbf[f] * xc;
      const double ri = M.b64[c] - ax;
      M.r64[c] = ri;
      acc[0] += ri * ri;
      acc[1] += ri;
    }
    __syncthreads();
    grid_reduce<2>(grid, acc, red, part[pb], tot);
    pb ^= 1;
    mean = a.project ? tot[1] / nd : 0.0;
    rr = a.project ? tot[0] - tot[1] * mean : tot[0];
    if (rr < 0.0) rr = 0.0;
    res = sqrt(rr) / bnorm;
    __syncthreads();
    if (!(res == res)) break;
    if (res < M.tol) {
      conv = 1;
      break;
    }
    if (o.its == 0 && !o.conv) break;  // the float solver made no progress
    for (int i = gt; i < n; i += gs) M.rb32[i] = (float)(M.r64[i] - mean);
    grid.sync();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.info->iterations = its;
    a.info->converged = conv;
    a.info->residual = res;
  }
}

// ---------------------------------------------------------------------------------- launch helpers
template <class K>
static int coop_grid(K kernel, int* grid_out) {
  static int cached_dev = -1, cached_grid = 0;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return B2S_ERR_DEVICE;
  int sms = 0, per = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return B2S_ERR_DEVICE;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kCoopThreads, 0) != cudaSuccess) return B2S_ERR_DEVICE;
  if (per <= 0) return B2S_ERR_DEVICE;
  if (per > 1) per = 1;
  int g = sms * per;
  if (g > kMaxCoopBlocks) g = kMaxCoopBlocks;
  (void)cached_dev;
  (void)cached_grid;
  *grid_out = g;
  return B2S_OK;
}

// Cooperative launches of the AMG-PCG kernels as thread-block clusters of g_pcg_cluster blocks
// (the small end of each V-cycle then runs on the first cluster with cluster barriers). The
// grid is every cluster that co-resides on the device, which leaves a few SMs idle when the
// cluster size does not divide the SMs of a GPC; a launch is made with clusters only when that
// grid still covers three quarters of the SMs, and falls back to a plain cooperative launch
// (csize = 0) when the cluster launch is refused.
static int g_pcg_cluster = 0;
static int g_sub_nnz[2] = {4096, 32768};  // without / with clusters

static int coop_cluster_grid(const void* kernel, int C, int* grid_out) {
  struct Entry {
    const void* kernel;
    int dev, C, grid;
  };
  static Entry cache[32];
  static int ncache = 0;
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return B2S_ERR_DEVICE;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (int i = 0; i < ncache; ++i)
      if (cache[i].kernel == kernel && cache[i].dev == dev && cache[i].C == C) {
        *grid_out = cache[i].grid;
        return cache[i].grid > 0 ? B2S_OK : B2S_ERR_DEVICE;
      }
  }
  if (C > 8) cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeCooperative;
  attr[1].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)C, 1, 1);
  cfg.blockDim = dim3(kCoopThreads, 1, 1);
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  int ncl = 0, g = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, kernel, &cfg) == cudaSuccess && ncl > 0) {
    g = ncl * C;
    if (g > kMaxCoopBlocks) g = kMaxCoopBlocks - kMaxCoopBlocks % C;
  } else {
    cudaGetLastError();
  }
  std::lock_guard<std::mutex> lock(mu);
  if (ncache < 32) cache[ncache++] = {kernel, dev, C, g};
  *grid_out = g;
  return g > 0 ? B2S_OK : B2S_ERR_DEVICE;
}

// Launch an AMG-PCG kernel whose argument block is *args_block; its csize and sub_nnz fields
// (at *csize, *sub_nnz) are set to the launch shape used.
template <class K>
static int launch_pcg_kernel(K kernel, void* args_block, int* csize, int* sub_nnz, b2s_stream_t s) {
  void* args[] = {args_block};
  const int C = g_pcg_cluster;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return B2S_ERR_DEVICE;
  int g = 0;
  if (C > 1 && coop_cluster_grid((const void*)kernel, C, &g) == B2S_OK && 4 * g >= 3 * sms) {
    *csize = C;
    *sub_nnz = g_sub_nnz[1];
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeCooperative;
    attr[1].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)g, 1, 1);
    cfg.blockDim = dim3(kCoopThreads, 1, 1);
    cfg.stream = (cudaStream_t)s;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    if (cudaLaunchKernelExC(&cfg, (const void*)kernel, args) == cudaSuccess) {
      B2S_LAUNCH_CHECK();
      return B2S_OK;
    }
    cudaGetLastError();  // a refused launch configuration: launch without clusters
  }
  *csize = 0;
  *sub_nnz = g_sub_nnz[0];
  int rc;
  if ((rc = coop_grid(kernel, &g)) != B2S_OK) return rc;
  if (cudaLaunchCooperativeKernel((void*)kernel, g, kCoopThreads, args, 0, (cudaStream_t)s) != cudaSuccess)
    return B2S_ERR_LAUNCH;
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

template <class T>
static T* pcg_layout(const b2s_amg* h, T* w, PcgArgsT<T>& a) {
  const int64_t n = h->nlevels ? h->levels[0].n : h->coarse_n;
  a.r = w;
  a.p = w + n;
  a.p2 = w + 2 * n;
  a.q = w + 3 * n;
  T* c = w + 4 * n;
  a.cb = c;
  a.cx = c + h->coarse_n;
  c += 2 * (int64_t)h->coarse_n;
  for (int l = 0; l < h->nlevels; ++l) {
    const int64_t m = h->levels[l].n;
    a.lv[l].b = c;
    a.lv[l].x = c + m;
    a.lv[l].y = c + 2 * m;
    a.lv[l].r = c + 3 * m;
    c += 4 * m;
  }
  return c;
}

template <class T, int NR>
static int launch_bicgstab_nr(BicgArgsT<T>& a, b2s_stream_t s) {
  void* args[] = {&a};
  int g = 0, rc;
  if ((rc = coop_grid(bicgstab_coop_k<NR, T>, &g)) != B2S_OK) return rc;
  if (cudaLaunchCooperativeKernel((void*)bicgstab_coop_k<NR, T>, g, kCoopThreads, args, 0, (cudaStream_t)s) !=
      cudaSuccess)
    return B2S_ERR_LAUNCH;
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

template <class T>
static int launch_bicgstab(BicgArgsT<T>& a, int nrhs, b2s_stream_t s) {
  switch (nrhs) {
    case 1: return launch_bicgstab_nr<T, 1>(a, s);
    case 2: return launch_bicgstab_nr<T, 2>(a, s);
    default: return launch_bicgstab_nr<T, 3>(a, s);
  }
}

}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_pcg_set_launch(int cluster_blocks, int sub_entries) {
  if (cluster_blocks != 0 && cluster_blocks != 2 && cluster_blocks != 4 && cluster_blocks != 8 &&
      cluster_blocks != 16)
    return B2S_ERR_ARG;
  if (sub_entries < 0) return B2S_ERR_ARG;
  g_pcg_cluster = cluster_blocks;
  g_sub_nnz[cluster_blocks > 0 ? 1 : 0] = sub_entries;
  return B2S_OK;
}

int b2s_spmv_d(int32_t n, int k, const int32_t* rowptr, const int32_t* col, const double* val, const double* x,
               double* y, b2s_stream_t s) {
  if (n <= 0 || k < 1 || !rowptr || !col || !val || !x || !y) return B2S_ERR_ARG;
  spmv_k<<<grid_for(n), kThreads, 0, (cudaStream_t)s>>>(n, k, rowptr, col, val, x, y);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int64_t b2s_bicgstab_workspace_bytes(int32_t n, int nrhs) {
  if (n <= 0 || nrhs < 1 || nrhs > 3) return -1;
  return (int64_t)sizeof(double) * ((int64_t)kBicgVectors * nrhs * n + (int64_t)2 * kMaxCoopBlocks * 3 * nrhs);
}

int b2s_bicgstab_jacobi_d(int32_t n, int nrhs, const int32_t* rowptr, const int32_t* col, const double* val,
                          const double* b, const double* inv_diag, double* x, double tol, int maxiter,
                          int relative_to_initial, void* work, int64_t work_bytes, b2s_solve_info* info,
                          b2s_stream_t s) {
  if (n <= 0 || nrhs < 1 || nrhs > 3 || !rowptr || !col || !val || !b || !inv_diag || !x || !work || !info ||
      maxiter < 0)
    return B2S_ERR_ARG;
  if (work_bytes < b2s_bicgstab_workspace_bytes(n, nrhs)) return B2S_ERR_WORKSPACE;
  BicgArgs a;
  a.n = n;
  a.nr = nrhs;
  a.rowptr = rowptr;
  a.col = col;
  a.val = val;
  a.b = b;
  a.inv = inv_diag;
  a.x = x;
  a.tol = tol;
  a.maxiter = maxiter;
  a.rel = relative_to_initial ? 1 : 0;
  a.zero_x0 = 0;
  a.work = (double*)work;
  a.part0 = a.work + (int64_t)kBicgVectors * nrhs * n;
  a.part1 = a.part0 + (int64_t)kMaxCoopBlocks * 3 * nrhs;
  a.info = info;
  a.out64 = nullptr;
  a.base64 = nullptr;
  return launch_bicgstab(a, nrhs, s);
}

int64_t b2s_bicgstab_f32_workspace_bytes(int32_t n, int nrhs) {
  if (n <= 0 || nrhs < 1 || nrhs > 3) return -1;
  return (int64_t)sizeof(float) * ((int64_t)kBicgVectors * nrhs * n) + (int64_t)sizeof(double) * 2 * kMaxCoopBlocks * 3 * nrhs;
}

int b2s_bicgstab_jacobi_f32_d(int32_t n, int nrhs, const int32_t* rowptr, const int32_t* col, const float* val,
                              const float* b, const float* inv_diag, float* x, double tol, int maxiter,
                              int relative_to_initial, int zero_x0, double* out64, const double* base64, void* work,
                              int64_t work_bytes, b2s_solve_info* info, b2s_stream_t s) {
  if (n <= 0 || nrhs < 1 || nrhs > 3 || !rowptr || !col || !val || !b || !inv_diag || !x || !work || !info ||
      maxiter < 0 || ((out64 == nullptr) != (base64 == nullptr)))
    return B2S_ERR_ARG;
  if (work_bytes < b2s_bicgstab_f32_workspace_bytes(n, nrhs)) return B2S_ERR_WORKSPACE;
  BicgArgsT<float> a;
  a.n = n;
  a.nr = nrhs;
  a.rowptr = rowptr;
  a.col = col;
  a.val = val;
  a.b = b;
  a.inv = inv_diag;
  a.x = x;
  a.tol = tol;
  a.maxiter = maxiter;
  a.rel = relative_to_initial ? 1 : 0;
  a.zero_x0 = zero_x0 ? 1 : 0;
  a.work = (float*)work;
  a.part0 = (double*)((char*)work + sizeof(float) * (int64_t)kBicgVectors * nrhs * n);
  a.part1 = a.part0 + (int64_t)kMaxCoopBlocks * 3 * nrhs;
  a.info = info;
  a.out64 = out64;
  a.base64 = base64;
  return launch_bicgstab(a, nrhs, s);
}

static bool amg_ok(const b2s_amg* h) {
  if (!h || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS || h->coarse_n < 1 || !h->coarse_inv) return false;
  if (h->nlevels == 0 && (!h->coarse_rowptr || !h->coarse_col || !h->coarse_val)) return false;
  for (int l = 0; l < h->nlevels; ++l) {
    const b2s_amg_level& L = h->levels[l];
    if (L.n < 1 || !L.rowptr || !L.col || !L.val || !L.dinv || !L.p_rowptr || !L.r_rowptr) return false;
    const int next = (l + 1 < h->nlevels) ? h->levels[l + 1].n : h->coarse_n;
    if (L.nc != next) return false;
  }
  return true;
}

int64_t b2s_pcg_workspace_bytes(const b2s_amg* h) {
  if (!amg_ok(h)) return -1;
  int64_t n = h->nlevels ? h->levels[0].n : h->coarse_n, tot = 4 * n + 2 * (int64_t)h->coarse_n;
  for (int l = 0; l < h->nlevels; ++l) tot += 4 * (int64_t)h->levels[l].n;
  tot += 2 * (int64_t)kMaxCoopBlocks * 3;
  return tot * (int64_t)sizeof(double);
}

static void pcg_layout(const b2s_amg* h, double* w, PcgArgs& a) {
  double* c = pcg_layout<double>(h, w, a);
  a.part0 = c;
  a.part1 = c + (int64_t)kMaxCoopBlocks * 3;
  for (int l = 0; l < h->nlevels; ++l)
    a.lvv[l] = {h->levels[l].val, h->levels[l].dinv, h->levels[l].p_val, h->levels[l].r_val};
}

int b2s_pcg_amg_d(const b2s_amg* h, int32_t n, const int32_t* rowptr, const int32_t* col, const double* val,
                  const double* b, double* x, double tol, int maxiter, int project, void* work, int64_t work_bytes,
                  b2s_solve_info* info, b2s_stream_t s) {
  if (!amg_ok(h) || !rowptr || !col || !val || !b || !x || !work || !info || maxiter < 0) return B2S_ERR_ARG;
  if (n != (h->nlevels ? h->levels[0].n : h->coarse_n)) return B2S_ERR_ARG;
  if (work_bytes < b2s_pcg_workspace_bytes(h)) return B2S_ERR_WORKSPACE;
  PcgArgs a;
  a.h = *h;
  a.n = n;
  a.rowptr = rowptr;
  a.col = col;
  a.val = val;
  a.b = b;
  a.x = x;
  a.tol = tol;
  a.maxiter = maxiter;
  a.project = project ? 1 : 0;
  a.info = info;
  pcg_layout(h, (double*)work, a);
  return launch_pcg_kernel(pcg_amg_coop_k, &a, &a.csize, &a.sub_nnz, s);
}

static bool amg32_ok(const b2s_amg* h, const b2s_amg_f32* h32) {
  if (!h32) return false;
  for (int l = 0; l < h->nlevels; ++l)
    if (!h32->val[l] || !h32->dinv[l] || !h32->p_val[l] || !h32->r_val[l]) return false;
  return true;
}

int64_t b2s_pcg_mixed_workspace_bytes(const b2s_amg* h) {
  if (!amg_ok(h)) return -1;
  const int64_t n = h->nlevels ? h->levels[0].n : h->coarse_n;
  int64_t f = 4 * n + 2 * (int64_t)h->coarse_n + 2 * n;  // float vectors
  for (int l = 0; l < h->nlevels; ++l) f += 4 * (int64_t)h->levels[l].n;
  const int64_t d = n + 2 * (int64_t)kMaxCoopBlocks * 3;  // r64 and the partial sums
  return d * (int64_t)sizeof(double) + f * (int64_t)sizeof(float) + 16;
}

int b2s_pcg_amg_mixed_d(const b2s_amg* h, const b2s_amg_f32* h32, const b2s_mesh* m, const double* cf,
                        const double* cb, int32_t n, const int32_t* rowptr, const int32_t* col, const float* val,
                        const double* b, double* x, double tol, int maxiter, int project, int maxpass,
                        double min_inner_tol, void* work, int64_t work_bytes, b2s_solve_info* info, b2s_stream_t s) {
  if (!amg_ok(h) || !amg32_ok(h, h32) || !m || !cf || (!cb && m->nb) || !rowptr || !col || !val || !b || !x ||
      !work || !info || maxiter < 0 || maxpass < 1 || !(min_inner_tol > 0.0))
    return B2S_ERR_ARG;
  if (n != (h->nlevels ? h->levels[0].n : h->coarse_n) || n != m->nc) return B2S_ERR_ARG;
  if (!m->own_ptr || !m->nei_ptr || !m->nei_face || !m->fN || !m->fP || !m->bptr) return B2S_ERR_ARG;
  if (work_bytes < b2s_pcg_mixed_workspace_bytes(h)) return B2S_ERR_WORKSPACE;
  PcgMixedArgs M;
  PcgArgsT<float>& a = M.a;
  a.h = *h;
  for (int l = 0; l < h->nlevels; ++l) a.lvv[l] = {h32->val[l], h32->dinv[l], h32->p_val[l], h32->r_val[l]};
  a.n = n;
  a.rowptr = rowptr;
  a.col = col;
  a.val = val;
  a.x = nullptr;
  a.tol = tol;
  a.maxiter = maxiter;
  a.project = project ? 1 : 0;
  a.info = info;
  double* dw = (double*)work;
  M.r64 = dw;
  a.part0 = dw + n;
  a.part1 = a.part0 + (int64_t)kMaxCoopBlocks * 3;
  float* fw = (float*)(a.part1 + (int64_t)kMaxCoopBlocks * 3);
  float* rest = pcg_layout<float>(h, fw, a);
  M.rb32 = rest;
  M.d32 = rest + n;
  a.b = M.rb32;
  M.m = *m;
  M.cf = cf;
  M.cbf = cb;
  M.b64 = b;
  M.x64 = x;
  M.tol = tol;
  M.maxiter = maxiter;
  M.maxpass = maxpass;
  M.min_inner_tol = min_inner_tol;
  return launch_pcg_kernel(pcg_mixed_coop_k, &M, &M.a.csize, &M.a.sub_nnz, s);
}

}  // extern "C"

namespace b2s {
__global__ void __launch_bounds__(kCoopThreads) vcycle_coop_k(PcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const double* z = vcycle(grid, a, a.b, false, gt, gs);
  const int n = a.h.nlevels ? a.h.levels[0].n : a.h.coarse_n;
  for (int i = gt; i < n; i += gs) a.x[i] = z[i];
}
}  // namespace b2s

extern "C" int b2s_amg_vcycle_d(const b2s_amg* h, const double* b, double* x, void* work, int64_t work_bytes,
                                b2s_stream_t s) {
  if (!amg_ok(h) || !b || !x || !work) return B2S_ERR_ARG;
  if (work_bytes < b2s_pcg_workspace_bytes(h)) return B2S_ERR_WORKSPACE;
  PcgArgs a;
  a.h = *h;
  a.n = h->nlevels ? h->levels[0].n : h->coarse_n;
  a.rowptr = h->nlevels ? h->levels[0].rowptr : h->coarse_rowptr;
  a.col = h->nlevels ? h->levels[0].col : h->coarse_col;
  a.val = h->nlevels ? h->levels[0].val : h->coarse_val;
  a.b = b;
  a.x = x;
  a.tol = 0.0;
  a.maxiter = 0;
  a.project = 0;
  a.info = nullptr;
  pcg_layout(h, (double*)work, a);
  return launch_pcg_kernel(vcycle_coop_k, &a, &a.csize, &a.sub_nnz, s);
}
