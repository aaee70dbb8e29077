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

// ---------------------------------------------------------------------------------- BiCGSTAB
struct BicgArgs {
  int n, nr;
  const int32_t* rowptr;
  const int32_t* col;
  const double* val;
  const double* b;
  const double* inv;
  double* x;
  double tol;
  int maxiter, rel;
  double* work;
  double* part0;
  double* part1;
  b2s_solve_info* info;
};

enum { ACTIVE = 0, CONVERGED = 1, STOPPED = 2 };

// Three grid phases per iteration (the reference's algorithm has five dependent steps):
//   1. p = r + beta (p_old - omega v_old), h = inv p, v = A h with every neighbour's h evaluated
//      on the fly from p_old, v_old and r (same arithmetic as storing it), r_hat.v;
//   2. s = r - alpha v, hs = inv s, and t = A hs evaluated the same way, with s.s, t.t, t.s
//      (t is wasted only on the iteration where |s| converges);
//   3. r = s - omega t, r.r, r_hat.r.
// p and v alternate between two buffers so that neighbours read the previous iteration's values.
// x gets alpha h + omega hs one phase later (after the breakdown test), as the reference does.
template <int NR>
__global__ void __launch_bounds__(kCoopThreads) bicgstab_coop_k(BicgArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[(kCoopThreads / 32 + 1) * 3 * NR];
  __shared__ double tot[3 * NR];
  const int n = a.n;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  double* part[2] = {a.part0, a.part1};
  int pb = 0;
  double *r[NR], *rh[NR], *pp[2][NR], *vv[2][NR], *h[NR], *s[NR], *hs[NR], *t[NR], *x[NR];
  const double* b[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    double* w = a.work + (int64_t)10 * k * n;
    r[k] = w;
    rh[k] = w + n;
    pp[0][k] = w + 2 * (int64_t)n;
    vv[0][k] = w + 3 * (int64_t)n;
    h[k] = w + 4 * (int64_t)n;
    s[k] = w + 5 * (int64_t)n;
    hs[k] = w + 6 * (int64_t)n;
    t[k] = w + 7 * (int64_t)n;
    pp[1][k] = w + 8 * (int64_t)n;
    vv[1][k] = w + 9 * (int64_t)n;
    x[k] = a.x + (int64_t)k * n;
    b[k] = a.b + (int64_t)k * n;
  }
  const double* inv = a.inv;
  int cur = 0;  // p, v of the previous iteration are pp[cur], vv[cur]
  // ---- r = b - A x, r_hat = r, p = v = 0
  {
    double acc[3 * NR];
#pragma unroll
    for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
    for (int i = gt; i < n; i += gs) {
      const int j0 = a.rowptr[i], j1 = a.rowptr[i + 1];
      double ax[NR];
#pragma unroll
      for (int k = 0; k < NR; ++k) ax[k] = 0.0;
      for (int j = j0; j < j1; ++j) {
        const double av = a.val[j];
        const int c = a.col[j];
#pragma unroll
        for (int k = 0; k < NR; ++k) ax[k] += av * x[k][c];
      }
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        const double bi = b[k][i], ri = bi - ax[k];
        r[k][i] = ri;
        rh[k][i] = ri;
        pp[0][k][i] = 0.0;
        vv[0][k][i] = 0.0;
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
    // ---- phase 1: deferred x update; p, h, v = A h; r_hat.v
    {
      double acc[3 * NR];
#pragma unroll
      for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
      double* po[NR];
      double* vo[NR];
      double* pn[NR];
      double* vn[NR];
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        po[k] = pp[cur][k];
        vo[k] = vv[cur][k];
        pn[k] = pp[cur ^ 1][k];
        vn[k] = vv[cur ^ 1][k];
      }
      for (int i = gt; i < n; i += gs) {
        const double iv = inv[i];
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (pend[k]) x[k][i] = (x[k][i] + alpha[k] * h[k][i]) + omega[k] * hs[k][i];
        if (!any) continue;
        const int j0 = a.rowptr[i], j1 = a.rowptr[i + 1];
        double av_[NR];
#pragma unroll
        for (int k = 0; k < NR; ++k) av_[k] = 0.0;
        for (int j = j0; j < j1; ++j) {
          const double aij = a.val[j];
          const int c = a.col[j];
          const double ic = inv[c];
#pragma unroll
          for (int k = 0; k < NR; ++k)
            if (st[k] == ACTIVE) av_[k] += aij * (ic * (r[k][c] + beta[k] * (po[k][c] - omega[k] * vo[k][c])));
        }
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (st[k] == ACTIVE) {
            const double pi = r[k][i] + beta[k] * (po[k][i] - omega[k] * vo[k][i]);
            pn[k][i] = pi;
            h[k][i] = iv * pi;
            vn[k][i] = av_[k];
            acc[k] += rh[k][i] * av_[k];
          }
      }
#pragma unroll
      for (int k = 0; k < NR; ++k) pend[k] = false;
      if (!any) break;
      grid_reduce<3 * NR>(grid, acc, red, part[pb], tot);
      pb ^= 1;
      cur ^= 1;
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
    // ---- phase 2: s = r - alpha v, hs = inv s, t = A hs; s.s, t.t, t.s
    {
      double acc[3 * NR];
#pragma unroll
      for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
      double* v[NR];
#pragma unroll
      for (int k = 0; k < NR; ++k) v[k] = vv[cur][k];
      for (int i = gt; i < n; i += gs) {
        const double iv = inv[i];
        const int j0 = a.rowptr[i], j1 = a.rowptr[i + 1];
        double at[NR];
#pragma unroll
        for (int k = 0; k < NR; ++k) at[k] = 0.0;
        for (int j = j0; j < j1; ++j) {
          const double aij = a.val[j];
          const int c = a.col[j];
          const double ic = inv[c];
#pragma unroll
          for (int k = 0; k < NR; ++k)
            if (st[k] == ACTIVE) at[k] += aij * (ic * (r[k][c] - alpha[k] * v[k][c]));
        }
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (st[k] == ACTIVE) {
            const double si = r[k][i] - alpha[k] * v[k][i];
            s[k][i] = si;
            hs[k][i] = iv * si;
            t[k][i] = at[k];
            acc[k] += si * si;
            acc[NR + k] += at[k] * at[k];
            acc[2 * NR + k] += at[k] * si;
          }
      }
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
    // ---- phase 3: r = s - omega t; r.r, r_hat.r (systems converged in phase 2 take x += alpha h)
    {
      double acc[3 * NR];
#pragma unroll
      for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.0;
      for (int i = gt; i < n; i += gs) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
          if (pend_a[k]) x[k][i] = x[k][i] + alpha[k] * h[k][i];
          if (st[k] == ACTIVE) {
            const double ri = s[k][i] - omega[k] * t[k][i];
            r[k][i] = ri;
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
struct VBuf {  // per-level V-cycle vectors
  double* b;
  double* x;
  double* y;
  double* r;
};

struct PcgArgs {
  b2s_amg h;
  int n;                 // the operator A (the current matrix)
  const int32_t* rowptr;
  const int32_t* col;
  const double* val;
  const double* b;
  double* x;
  double tol;
  int maxiter, project;
  double* r;
  double* p;
  double* p2;
  double* q;
  double* cb;   // coarse right-hand side
  double* cx;   // coarse solution
  double* part0;
  double* part1;
  VBuf lv[B2S_AMG_MAX_LEVELS];
  b2s_solve_info* info;
};

// One damped-Jacobi step y = x + (w Dinv)(b - A x); x == NULL means x = w Dinv b (fused).
__device__ __forceinline__ void jacobi_step(const b2s_amg_level& L, double w, const double* b, const double* x,
                                            double* y, int gt, int gs) {
  for (int i = gt; i < L.n; i += gs) {
    double s = 0.0, xi;
    const double wd = w * L.dinv[i];
    if (x) {
      for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) s += L.val[j] * x[L.col[j]];
      xi = x[i];
    } else {
      for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
        const int c = L.col[j];
        s += L.val[j] * ((w * L.dinv[c]) * b[c]);
      }
      xi = wd * b[i];
    }
    y[i] = xi + wd * (b[i] - s);
  }
}

struct Mat0 {
  int n;
  const int32_t* rowptr;
  const int32_t* col;
  const double* val;
};

// Level-0 matrix: the finest smoothing level, or the coarse matrix itself when the hierarchy
// has no smoothing level (a matrix at or below max_coarse rows, amg.py:90 with no iteration).
__device__ __forceinline__ Mat0 level0(const b2s_amg& h) {
  if (h.nlevels > 0) return {h.levels[0].n, h.levels[0].rowptr, h.levels[0].col, h.levels[0].val};
  return {h.coarse_n, h.coarse_rowptr, h.coarse_col, h.coarse_val};
}

// Barrier of a V-cycle phase: the whole grid for the large levels, block 0 alone for the tail.
struct Phase {
  cg::grid_group* grid;
  bool tail;
  int t, n;  // this thread's index and the number of threads in the phase
  __device__ __forceinline__ void sync() const {
    if (tail) __syncthreads();
    else grid->sync();
  }
};

// Down-leg of level l (amg.py:135-139): pre-smoothing (the first two sweeps fused: the first
// sweep's x = w D^-1 b is evaluated on the fly), residual, restriction to the next level.
__device__ __forceinline__ double* vdown(const PcgArgs& a, int l, const double* b, const Phase& ph) {
  const b2s_amg& h = a.h;
  const b2s_amg_level& lv = h.levels[l];
  const int L = h.nlevels;
  const double w = h.omega;
  double* X = a.lv[l].x;
  double* Y = a.lv[l].y;
  double* c = X;
  if (h.sweeps <= 1) {
    for (int i = ph.t; i < lv.n; i += ph.n) X[i] = (w * lv.dinv[i]) * b[i];
  } else {
    jacobi_step(lv, w, b, nullptr, X, ph.t, ph.n);
    double* o = Y;
    for (int sw = 2; sw < h.sweeps; ++sw) {
      ph.sync();
      jacobi_step(lv, w, b, c, o, ph.t, ph.n);
      double* tmp = c;
      c = o;
      o = tmp;
    }
  }
  ph.sync();
  double* R = a.lv[l].r;
  for (int i = ph.t; i < lv.n; i += ph.n) {
    double s = 0.0;
    for (int j = lv.rowptr[i]; j < lv.rowptr[i + 1]; ++j) s += lv.val[j] * c[lv.col[j]];
    R[i] = b[i] - s;
  }
  ph.sync();
  double* bn = (l + 1 < L) ? a.lv[l + 1].b : a.cb;
  for (int I = ph.t; I < lv.nc; I += ph.n) {
    double s = 0.0;
    for (int j = lv.r_rowptr[I]; j < lv.r_rowptr[I + 1]; ++j) s += lv.r_val[j] * R[lv.r_col[j]];
    bn[I] = s;
  }
  ph.sync();
  return c;
}

// Up-leg of level l (amg.py:139-142): x += P xc, then the post-smoothing sweeps. With stats
// (level 0 on the grid) the last sweep also accumulates sum z, sum r z and sum r for the PCG
// and ends with their grid-wide reduction into stats.
__device__ __forceinline__ double* vup(const PcgArgs& a, int l, const double* b, double* c, const double* xc,
                                       const Phase& ph, const double* rr, double* red, double* stats, int pb) {
  const b2s_amg& h = a.h;
  const b2s_amg_level& lv = h.levels[l];
  const double w = h.omega;
  double* o = (c == a.lv[l].x) ? a.lv[l].y : a.lv[l].x;
  const bool want = stats != nullptr;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = ph.t; i < lv.n; i += ph.n) {
    double s = 0.0;
    for (int j = lv.p_rowptr[i]; j < lv.p_rowptr[i + 1]; ++j) s += lv.p_val[j] * xc[lv.p_col[j]];
    const double zi = c[i] + s;
    c[i] = zi;
    if (want && h.sweeps == 0) {
      acc[0] += zi;
      acc[1] += rr[i] * zi;
      acc[2] += rr[i];
    }
  }
  for (int sw = 0; sw < h.sweeps; ++sw) {
    ph.sync();
    const bool last = sw + 1 == h.sweeps;
    for (int i = ph.t; i < lv.n; i += ph.n) {
      double s = 0.0;
      for (int j = lv.rowptr[i]; j < lv.rowptr[i + 1]; ++j) s += lv.val[j] * c[lv.col[j]];
      const double zi = c[i] + (w * lv.dinv[i]) * (b[i] - s);
      o[i] = zi;
      if (want && last) {
        acc[0] += zi;
        acc[1] += rr[i] * zi;
        acc[2] += rr[i];
      }
    }
    double* tmp = c;
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

// Coarse solve cx = inv(Ac) cb, one warp per row.
__device__ __forceinline__ void vcoarse(const PcgArgs& a, const double* cb, const Phase& ph) {
  const int nc = a.h.coarse_n, lane = threadIdx.x & 31;
  for (int I = ph.t >> 5; I < nc; I += ph.n >> 5) {
    const double* row = a.h.coarse_inv + (int64_t)I * nc;
    double s = 0.0;
    for (int J = lane; J < nc; J += 32) s += row[J] * cb[J];
    s = warp_sum(s);
    if (lane == 0) a.cx[I] = s;
  }
  ph.sync();
}

// Buffer holding level l's solution after its up-leg: the down-leg ends in x after sweeps-2
// ping-pong swaps (x alone for one sweep), the up-leg swaps once per sweep. Every block can thus
// name the buffer without having run the level.
__device__ __forceinline__ double* tail_result(const PcgArgs& a, int l) {
  const int sw = a.h.sweeps;
  const int down = sw <= 1 ? 0 : sw - 2;
  return ((down + sw) & 1) ? a.lv[l].y : a.lv[l].x;
}

// Levels of at most kTailRows rows (no more rows than one block has threads), and the coarse
// solve, run in block 0 with block barriers while the other blocks wait at the next grid
// barrier: below that size a level is latency-bound and a grid barrier costs more than it saves.
constexpr int kTailRows = kCoopThreads;

// z = M r: the V-cycle of flowtrace/linalg/amg.py:130-142. Returns the buffer holding z. With
// stats != nullptr, when level 0 runs on the whole grid, stats[0..2] receive sum z, sum r z and
// sum r (r = rhs0) and *have_stats is set; otherwise the caller reduces them itself.
__device__ double* vcycle(cg::grid_group& grid, const PcgArgs& a, const double* rhs0, int gt, int gs,
                          double* red = nullptr, double* stats = nullptr, int pb = 0, bool* have_stats = nullptr) {
  const b2s_amg& h = a.h;
  const int L = h.nlevels;
  double* cur[B2S_AMG_MAX_LEVELS];
  const double* cb = (L == 0) ? rhs0 : a.cb;
  int Lg = 0;  // levels with more than kTailRows rows run on the whole grid
  while (Lg < L && h.levels[Lg].n > kTailRows) ++Lg;
  const Phase gph = {&grid, false, gt, gs};
  const Phase tph = {&grid, true, (int)threadIdx.x, (int)blockDim.x};
  for (int l = 0; l < Lg; ++l) cur[l] = vdown(a, l, (l == 0) ? rhs0 : a.lv[l].b, gph);
  if (Lg == L && h.coarse_n > kTailRows) {
    vcoarse(a, cb, gph);
  } else {
    if (blockIdx.x == 0) {
      for (int l = Lg; l < L; ++l) cur[l] = vdown(a, l, (l == 0) ? rhs0 : a.lv[l].b, tph);
      vcoarse(a, cb, tph);
      for (int l = L - 1; l >= Lg; --l)
        cur[l] = vup(a, l, (l == 0) ? rhs0 : a.lv[l].b, cur[l], (l + 1 < L) ? cur[l + 1] : a.cx, tph, nullptr,
                     nullptr, nullptr, 0);
    }
    grid.sync();
  }
  for (int l = Lg - 1; l >= 0; --l) {
    const double* xc;
    if (l + 1 < L) {
      // the next level's solution: every block tracks it on the grid levels; for the first tail
      // level (run by block 0 alone) every block names it from the sweep parity
      if (l + 1 < Lg) xc = cur[l + 1];
      else xc = tail_result(a, l + 1);
    } else {
      xc = a.cx;
    }
    const bool st = (l == 0) && stats != nullptr;
    cur[l] = vup(a, l, (l == 0) ? rhs0 : a.lv[l].b, cur[l], xc, gph, rhs0, st ? red : nullptr, st ? stats : nullptr,
                 pb);
    if (st && have_stats) *have_stats = true;
  }
  if (L == 0) return a.cx;
  if (Lg == 0) return tail_result(a, 0);
  return cur[0];
}

// Preconditioned CG (flowtrace/linalg/krylov.py:25-65). Per iteration: one phase computes
// p = z' + beta p_old into a second buffer and q = A p with the neighbours' p evaluated on the
// fly (same arithmetic), one phase updates x and r, then the V-cycle, whose last sweep also
// reduces sum z, sum r z and sum r; z' = z - mean(z) (the projection) is applied lazily and
// r.z' = sum r z - mean(z) sum r.
__global__ void __launch_bounds__(kCoopThreads) pcg_amg_coop_k(PcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[(kCoopThreads / 32 + 1) * 3];
  __shared__ double tot[3];
  __shared__ double stats[3];
  const Mat0 A = {a.n, a.rowptr, a.col, a.val};
  const int n = A.n;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  double* part[2] = {a.part0, a.part1};
  int pb = 0;
  double* r = a.r;
  double* q = a.q;
  double* x = a.x;
  double* pbuf[2] = {a.p, a.p2};
  int pc = 0;
  const double nd = (double)n;
  double bb, rr;
  {
    double acc[2] = {0.0, 0.0};
    for (int i = gt; i < n; i += gs) {
      const double bi = a.b[i];
      x[i] = 0.0;
      r[i] = bi;
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
  if (rnorm / bnorm < a.tol) {
    conv = 1;
    done = true;
  }
  // z = M r with the statistics of its projection
  double rz = 0.0, zm = 0.0;
  double* z = nullptr;
  auto precondition = [&]() {
    __syncthreads();
    bool have = false;
    z = vcycle(grid, a, r, gt, gs, red, stats, pb, &have);
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
  for (int k = 1; k <= a.maxiter && !done; ++k) {
    // p = z' + beta p_old (z' on the first iteration); q = A p; p.q
    double* pn = pbuf[pc];
    const double* po = pbuf[pc ^ 1];
    {
      double acc[2] = {0.0, 0.0};
      for (int i = gt; i < n; i += gs) {
        double s = 0.0;
        for (int j = A.rowptr[i]; j < A.rowptr[i + 1]; ++j) {
          const int c = A.col[j];
          const double pj = first ? z[c] - zm : (z[c] - zm) + beta * po[c];
          s += A.val[j] * pj;
        }
        const double pi = first ? z[i] - zm : (z[i] - zm) + beta * po[i];
        pn[i] = pi;
        q[i] = s;
        acc[0] += pi * s;
      }
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
        acc[0] += ri * ri;
      }
      grid_reduce<2>(grid, acc, red, part[pb], tot);
      pb ^= 1;
    }
    rnorm = sqrt(tot[0]);
    __syncthreads();
    if (rnorm / bnorm < a.tol) {
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

}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_spmv_d(int32_t n, int k, const int32_t* rowptr, const int32_t* col, const double* val, const double* x,
               double* y, b2s_stream_t s) {
  if (n <= 0 || k < 1 || !rowptr || !col || !val || !x || !y) return B2S_ERR_ARG;
  spmv_k<<<grid_for(n), kThreads, 0, (cudaStream_t)s>>>(n, k, rowptr, col, val, x, y);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int64_t b2s_bicgstab_workspace_bytes(int32_t n, int nrhs) {
  if (n <= 0 || nrhs < 1 || nrhs > 3) return -1;
  return (int64_t)sizeof(double) * ((int64_t)10 * nrhs * n + (int64_t)2 * kMaxCoopBlocks * 3 * nrhs);
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
  a.work = (double*)work;
  a.part0 = a.work + (int64_t)10 * nrhs * n;
  a.part1 = a.part0 + (int64_t)kMaxCoopBlocks * 3 * nrhs;
  a.info = info;
  void* args[] = {&a};
  int g = 0, rc;
  switch (nrhs) {
    case 1:
      if ((rc = coop_grid(bicgstab_coop_k<1>, &g)) != B2S_OK) return rc;
      if (cudaLaunchCooperativeKernel((void*)bicgstab_coop_k<1>, g, kCoopThreads, args, 0, (cudaStream_t)s) !=
          cudaSuccess)
        return B2S_ERR_LAUNCH;
      break;
    case 2:
      if ((rc = coop_grid(bicgstab_coop_k<2>, &g)) != B2S_OK) return rc;
      if (cudaLaunchCooperativeKernel((void*)bicgstab_coop_k<2>, g, kCoopThreads, args, 0, (cudaStream_t)s) !=
          cudaSuccess)
        return B2S_ERR_LAUNCH;
      break;
    default:
      if ((rc = coop_grid(bicgstab_coop_k<3>, &g)) != B2S_OK) return rc;
      if (cudaLaunchCooperativeKernel((void*)bicgstab_coop_k<3>, g, kCoopThreads, args, 0, (cudaStream_t)s) !=
          cudaSuccess)
        return B2S_ERR_LAUNCH;
      break;
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
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
  const int64_t n = h->nlevels ? h->levels[0].n : h->coarse_n;
  a.r = w;
  a.p = w + n;
  a.p2 = w + 2 * n;
  a.q = w + 3 * n;
  double* c = w + 4 * n;
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
  a.part0 = c;
  a.part1 = c + (int64_t)kMaxCoopBlocks * 3;
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
  void* args[] = {&a};
  int g = 0, rc;
  if ((rc = coop_grid(pcg_amg_coop_k, &g)) != B2S_OK) return rc;
  if (cudaLaunchCooperativeKernel((void*)pcg_amg_coop_k, g, kCoopThreads, args, 0, (cudaStream_t)s) != cudaSuccess)
    return B2S_ERR_LAUNCH;
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"

namespace b2s {
__global__ void __launch_bounds__(kCoopThreads) vcycle_coop_k(PcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  const double* z = vcycle(grid, a, a.b, gt, gs);
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
  void* args[] = {&a};
  int g = 0, rc;
  if ((rc = coop_grid(vcycle_coop_k, &g)) != B2S_OK) return rc;
  if (cudaLaunchCooperativeKernel((void*)vcycle_coop_k, g, kCoopThreads, args, 0, (cudaStream_t)s) != cudaSuccess)
    return B2S_ERR_LAUNCH;
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}
