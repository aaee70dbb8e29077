// Block-diagonal batches of independent SIMPLEC cases on B200.
//
// The cases of a batch share one device mesh (their disjoint union, each case's cells
// contiguous) and every finite-volume stage runs over all of them in one launch; the stages
// that reduce (residual and continuity sums, the pressure mean) are launched over a tiling of
// the cells in which no tile straddles two cases, so that their per-tile partial sums add up to
// per-case sums here. The Krylov solves are per case: each case keeps its own scalars (alpha,
// beta, omega, convergence), as if it were solved alone. They are persistent launches in which
// a team - the blocks of one thread-block cluster - takes whole cases from a fixed work list
// (largest first, dealt round-robin over the teams) and runs each one's solve with cluster
// barriers and distributed-shared-memory sums only: no grid barrier, no atomics, every
// reduction in a fixed order.
//
// The AMG hierarchy of a batch is block diagonal too (aggregates never cross cases, and are
// numbered case by case), so a case's V-cycle touches only its own rows on every level, and its
// coarsest level is solved with its own dense inverse.
#include "b2s_common.cuh"

namespace b2s {

constexpr int kBatchThreads = 1024;
constexpr int kBatchWarps = kBatchThreads / 32;

// ---------------------------------------------------------------------------------- sums per case
// out[g][q] = sum of part[q][t] over the tiles t of case g, one warp per (g, q).
__global__ void group_sums_k(const double* __restrict__ part, int nblk, int nq, int ngroups,
                             const int32_t* __restrict__ group_tiles, double* __restrict__ out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= ngroups * nq) return;
  const int g = w / nq, q = w - g * nq;
  double s = 0.0;
  for (int t = group_tiles[g] + lane; t < group_tiles[g + 1]; t += 32) s += part[(int64_t)q * nblk + t];
  s = warp_sum(s);
  if (lane == 0) out[(int64_t)g * nq + q] = s;
}

// x -= mean of x over each singular case; the case sums are part[q][tiles of the case]. One
// block per tile; warp 0 of every block of a case sums the same partials in the same order.
__global__ void remove_group_means_k(b2s_mesh m, double* __restrict__ x, const double* __restrict__ part, int nblk,
                                     int q, const int32_t* __restrict__ group_tiles,
                                     const int32_t* __restrict__ tile_group, const int32_t* __restrict__ group_cells,
                                     const int32_t* __restrict__ singular) {
  __shared__ double mean;
  const int t = blockIdx.x, g = tile_group[t];
  if (!singular[g]) return;
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int k = group_tiles[g] + (int)threadIdx.x; k < group_tiles[g + 1]; k += 32) s += part[(int64_t)q * nblk + k];
    s = warp_sum(s);
    if (threadIdx.x == 0) mean = s / (double)(group_cells[g + 1] - group_cells[g]);
  }
  __syncthreads();
  const int c = m.tiles[t] + (int)threadIdx.x;
  if (c < m.tiles[t + 1]) x[c] = x[c] - mean;
}

// ---------------------------------------------------------------------------------- case teams
// A case is solved by a team: the blocks of one thread-block cluster (b2s_team_config: 1-8
// blocks of up to 1024 threads, 4 x 1024 by default; the autotuner of the batch solver picks it). Rows are dealt over all the team's threads; a team barrier is the
// cluster barrier (which also orders the team's global-memory accesses), and a team sum adds
// the block sums of the team's blocks read from their shared memory (distributed shared
// memory), in rank order, so that every thread of the team gets the same bits.
constexpr int kClusterBlocks = 4;  // default team shape

struct Team {
  int t, n;      // this thread's index in the team and the team's size
  int rank, nb;  // this block's rank in the cluster and the cluster's blocks
  int pb;        // which of the two exchange buffers the next sum writes
  double* xbuf;  // [2][8] block sums exchanged between the cluster's blocks
  __device__ __forceinline__ void sync() const { cg::this_cluster().sync(); }
  template <int NQ>
  __device__ __forceinline__ void sum(double (&v)[NQ], double* red) {
    static_assert(NQ <= 8, "team sums of at most 8 values");
    double out[NQ];
    block_sum<NQ>(v, red, out);
    double* mine = xbuf + pb * 8;
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < NQ; ++q) mine[q] = out[q];
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    for (int r = 0; r < nb; ++r) {
      const double* other = cl.map_shared_rank(mine, r);
#pragma unroll
      for (int q = 0; q < NQ; ++q) v[q] += other[q];
    }
    pb ^= 1;  // the next sum writes the other buffer: a block still reading this one is safe
  }
};

__device__ __forceinline__ Team make_team(double* xbuf) {
  cg::cluster_group cl = cg::this_cluster();
  Team tm;
  tm.rank = (int)cl.block_rank();
  tm.nb = (int)cl.num_blocks();
  tm.t = tm.rank * (int)blockDim.x + (int)threadIdx.x;
  tm.n = tm.nb * (int)blockDim.x;
  tm.pb = 0;
  tm.xbuf = xbuf;
  return tm;
}

// Rows [lo, hi) of a team: one thread per row, or one warp per row for long rows.
struct BRows {
  int first, stride, lane, step;
  bool wide;
  __device__ __forceinline__ BRows(bool w, int lo, const Team& tm) {
    wide = w;
    first = lo + (w ? (tm.t >> 5) : tm.t);
    stride = w ? (tm.n >> 5) : tm.n;
    lane = w ? (tm.t & 31) : 0;
    step = w ? 32 : 1;
  }
  __device__ __forceinline__ double total(double s) const { return wide ? warp_sum(s) : s; }
  __device__ __forceinline__ bool writer() const { return lane == 0; }
};

constexpr int kBatchWideRow = 24;  // default: rows averaging this many entries go one warp per row

// Whether a range of rows is walked one warp per row (wide_row > 0 and rows averaging at least
// wide_row entries).
__device__ __forceinline__ bool wide_rows(int64_t nnz, int64_t rows, int wide_row) {
  return wide_row > 0 && nnz >= (int64_t)wide_row * rows;
}

// ---------------------------------------------------------------------------------- BiCGSTAB
template <class T>
struct BicgGroupArgs {
  int ngroups, nr, n;
  const int32_t* group_ptr;  // [ngroups+1] rows of each case
  const int32_t* order;      // [ngroups] processing order (largest first)
  const int32_t* rowptr;
  const int32_t* col;
  const T* val;
  const T* b;     // [nr][n]
  const T* inv;   // [n]
  T* x;           // [nr][n]
  double tol;
  int maxiter, rel, zero_x0;
  T* work;        // 7 [nr][n] vectors
  int wide_row;   // rows-per-warp switch (b2s_team_config)
  b2s_solve_info* info;  // [ngroups][nr]
  double* out64;  // when set: out64 = base64 + x
  const double* base64;
};

// Jacobi-BiCGSTAB of one case's rows (flowtrace/linalg/krylov.py:68-121 with
// relative_to_initial), NR systems sharing the matrix, each with its own scalars.
template <int NR, class T>
__device__ void bicgstab_group(const BicgGroupArgs<T>& a, int lo, int hi, double* red, b2s_solve_info* info,
                               Team& tm) {
  const int n = a.n;
  const int64_t nnz = a.rowptr[hi] - a.rowptr[lo];
  T *x[NR], *r[NR], *rh[NR], *p[NR], *v[NR], *h[NR], *s[NR], *t[NR];
  const T* b[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    T* w = a.work + (int64_t)7 * k * n;
    r[k] = w;
    rh[k] = w + n;
    p[k] = w + 2 * (int64_t)n;
    v[k] = w + 3 * (int64_t)n;
    h[k] = w + 4 * (int64_t)n;
    s[k] = w + 5 * (int64_t)n;
    t[k] = w + 6 * (int64_t)n;
    x[k] = a.x + (int64_t)k * n;
    b[k] = a.b + (int64_t)k * n;
  }
  const T* inv = a.inv;
  const bool wide = wide_rows(nnz, hi - lo, a.wide_row);
  // r = b - A x, r_hat = r, p = v = 0
  double acc[2 * NR];
#pragma unroll
  for (int q = 0; q < 2 * NR; ++q) acc[q] = 0.0;
  {
    const BRows R(wide, lo, tm);
    for (int i = R.first; i < hi; i += R.stride) {
#pragma unroll
      for (int k = 0; k < NR; ++k) {
        double sx = 0.0;
        if (!a.zero_x0)
          for (int j = a.rowptr[i] + R.lane; j < a.rowptr[i + 1]; j += R.step) sx += (double)a.val[j] * (double)x[k][a.col[j]];
        sx = R.total(sx);
        if (R.writer()) {
          const double bi = b[k][i], ri = bi - sx;
          if (a.zero_x0) x[k][i] = 0.0;
          r[k][i] = ri;
          rh[k][i] = ri;
          p[k][i] = 0.0;
          v[k][i] = 0.0;
          acc[k] += ri * ri;
          acc[NR + k] += bi * bi;
        }
      }
    }
  }
  tm.sum<2 * NR>(acc, red);
  bool act[NR];
  int its[NR], conv[NR];
  double rho[NR], alpha[NR], omega[NR], bnorm[NR], babs[NR], rnorm[NR], res[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    rnorm[k] = sqrt(acc[k]);
    babs[k] = sqrt(acc[NR + k]);
    bnorm[k] = a.rel ? rnorm[k] : babs[k];
    if (bnorm[k] == 0.0) bnorm[k] = 1.0;
    rho[k] = alpha[k] = omega[k] = 1.0;
    its[k] = 0;
    res[k] = rnorm[k] / bnorm[k];
    conv[k] = (rnorm[k] / bnorm[k] < a.tol || rnorm[k] <= 1e-14 * babs[k]) ? 1 : 0;
    act[k] = !conv[k];
  }
  for (int it = 1; it <= a.maxiter; ++it) {
    bool any = false;
#pragma unroll
    for (int k = 0; k < NR; ++k) any |= act[k];
    if (!any) break;
    // rho_new = r_hat . r
    double d1[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) d1[k] = 0.0;
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k)
        if (act[k]) d1[k] += (double)rh[k][i] * (double)r[k][i];
    tm.sum<NR>(d1, red);
    double beta[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      beta[k] = 0.0;
      if (!act[k]) continue;
      if (d1[k] == 0.0) {
        act[k] = false;
        its[k] = it;
        res[k] = rnorm[k] / bnorm[k];
        continue;
      }
      beta[k] = (d1[k] / rho[k]) * (alpha[k] / omega[k]);
      rho[k] = d1[k];
    }
    // p = r + beta (p - omega v), h = inv p
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k)
        if (act[k]) {
          const double pi = (double)r[k][i] + beta[k] * ((double)p[k][i] - omega[k] * (double)v[k][i]);
          p[k][i] = pi;
          h[k][i] = (double)inv[i] * pi;
        }
    tm.sync();
    // v = A h, r_hat . v
    double d2[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) d2[k] = 0.0;
    {
      const BRows R(wide, lo, tm);
      for (int i = R.first; i < hi; i += R.stride)
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (act[k]) {
            double sv = 0.0;
            for (int j = a.rowptr[i] + R.lane; j < a.rowptr[i + 1]; j += R.step)
              sv += (double)a.val[j] * (double)h[k][a.col[j]];
            sv = R.total(sv);
            if (R.writer()) {
              v[k][i] = sv;
              d2[k] += (double)rh[k][i] * sv;
            }
          }
    }
    tm.sum<NR>(d2, red);
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      if (!act[k]) continue;
      if (d2[k] == 0.0) {
        act[k] = false;
        its[k] = it;
        res[k] = rnorm[k] / bnorm[k];
        continue;
      }
      alpha[k] = rho[k] / d2[k];
    }
    // s = r - alpha v, |s|
    double d3[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) d3[k] = 0.0;
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k)
        if (act[k]) {
          const double si = (double)r[k][i] - alpha[k] * (double)v[k][i];
          s[k][i] = si;
          d3[k] += si * si;
        }
    tm.sum<NR>(d3, red);
    bool sdone[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      sdone[k] = false;
      if (!act[k]) continue;
      const double sn = sqrt(d3[k]);
      if (sn / bnorm[k] < a.tol) {
        sdone[k] = true;
        its[k] = it;
        res[k] = sn / bnorm[k];
        conv[k] = 1;
      }
    }
    // systems converged on |s|: x += alpha h (hs = inv s is evaluated on the fly below)
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k)
        if (sdone[k]) x[k][i] = (double)x[k][i] + alpha[k] * (double)h[k][i];
#pragma unroll
    for (int k = 0; k < NR; ++k)
      if (sdone[k]) act[k] = false;
    tm.sync();
    // t = A (inv s); t.t, t.s
    double d4[2 * NR];
#pragma unroll
    for (int q = 0; q < 2 * NR; ++q) d4[q] = 0.0;
    {
      const BRows R(wide, lo, tm);
      for (int i = R.first; i < hi; i += R.stride)
#pragma unroll
        for (int k = 0; k < NR; ++k)
          if (act[k]) {
            double st = 0.0;
            for (int j = a.rowptr[i] + R.lane; j < a.rowptr[i + 1]; j += R.step) {
              const int c = a.col[j];
              st += (double)a.val[j] * ((double)inv[c] * (double)s[k][c]);
            }
            st = R.total(st);
            if (R.writer()) {
              t[k][i] = st;
              d4[k] += st * st;
              d4[NR + k] += st * (double)s[k][i];
            }
          }
    }
    tm.sum<2 * NR>(d4, red);
#pragma unroll
    for (int k = 0; k < NR; ++k)
      if (act[k]) omega[k] = d4[k] > 0.0 ? d4[NR + k] / d4[k] : 0.0;
    // r = s - omega t; |r|, and the candidate x update
    double d5[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) d5[k] = 0.0;
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k)
        if (act[k]) {
          const double ri = (double)s[k][i] - omega[k] * (double)t[k][i];
          d5[k] += ri * ri;
        }
    tm.sum<NR>(d5, red);
    bool upd[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      upd[k] = false;
      if (!act[k]) continue;
      const double rn = sqrt(d5[k]);
      if (!isfinite(rn)) {  // breakdown: keep the last finite iterate
        act[k] = false;
        its[k] = it;
        res[k] = nan("");
        continue;
      }
      upd[k] = true;
      rnorm[k] = rn;
      if (rn / bnorm[k] < a.tol || rn <= 1e-14 * babs[k]) {
        act[k] = false;
        conv[k] = 1;
        its[k] = it;
        res[k] = rn / bnorm[k];
      } else if (omega[k] == 0.0) {
        act[k] = false;
        its[k] = it;
        res[k] = rn / bnorm[k];
      } else {
        its[k] = it;
        res[k] = rn / bnorm[k];
      }
    }
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k)
        if (upd[k]) {
          const double si = s[k][i];
          x[k][i] = ((double)x[k][i] + alpha[k] * (double)h[k][i]) + omega[k] * ((double)inv[i] * si);
          r[k][i] = si - omega[k] * (double)t[k][i];
        }
    tm.sync();
  }
  if (a.out64)
    for (int i = lo + tm.t; i < hi; i += tm.n)
#pragma unroll
      for (int k = 0; k < NR; ++k) a.out64[(int64_t)k * n + i] = a.base64[(int64_t)k * n + i] + (double)x[k][i];
  if (tm.t == 0)
#pragma unroll
    for (int k = 0; k < NR; ++k) {
      info[k].iterations = its[k] ? its[k] : (conv[k] ? 0 : a.maxiter);
      info[k].converged = conv[k];
      info[k].residual = res[k];
    }
  tm.sync();
}

// Cluster c of the launch takes cases order[c], order[c + nclusters], ...
template <int NR, class T>
__global__ void __launch_bounds__(kBatchThreads) bicgstab_groups_k(BicgGroupArgs<T> a) {
  __shared__ double red[(kBatchWarps + 1) * 2 * NR];
  __shared__ double xbuf[16];
  Team tm = make_team(xbuf);
  const int cid = (int)blockIdx.x / tm.nb, ncl = (int)gridDim.x / tm.nb;
  for (int k = cid; k < a.ngroups; k += ncl) {
    const int g = a.order[k];
    bicgstab_group<NR, T>(a, a.group_ptr[g], a.group_ptr[g + 1], red, a.info + (int64_t)g * NR, tm);
  }
  tm.sync();  // no block leaves while another may still read its shared memory
}

// ---------------------------------------------------------------------------------- AMG-PCG
template <class T>
struct PcgGroupArgs {
  b2s_amg h;
  const T* lval[B2S_AMG_MAX_LEVELS];
  const T* ldinv[B2S_AMG_MAX_LEVELS];
  const T* lpval[B2S_AMG_MAX_LEVELS];
  const T* lrval[B2S_AMG_MAX_LEVELS];
  T* lb[B2S_AMG_MAX_LEVELS];
  T* lx[B2S_AMG_MAX_LEVELS];
  T* ly[B2S_AMG_MAX_LEVELS];
  T* lr[B2S_AMG_MAX_LEVELS];
  int n;
  const int32_t* rowptr;  // the operator (current level-0 matrix)
  const int32_t* col;
  const T* val;
  T* r;
  T* p;
  T* q;
  T* cb;
  T* cx;
  // refinement in double
  b2s_mesh m;
  const double* cf;
  const double* cbf;
  const double* b64;
  double* x64;
  double* r64;
  T* rb;   // float right-hand side of a pass
  T* d;    // float correction of a pass
  const int32_t* order;
  const int32_t* project;  // [ngroups] singular cases
  int wide_row;            // rows-per-warp switch (b2s_team_config)
  double tol;
  int maxiter, maxpass;
  double min_inner_tol;
  b2s_solve_info* info;  // [ngroups]
};

// z = M r on case g (flowtrace/linalg/amg.py:130-142): pre-smoothing (first sweep fused),
// residual, restriction on every level, the case's dense coarse inverse, then prolongation and
// post-smoothing; returns the buffer holding z (rows of case g on level 0).
template <class T>
__device__ T* vcycle_group(const PcgGroupArgs<T>& a, int g, const T* rhs0, double* red, Team& tm) {
  const b2s_amg& h = a.h;
  const int L = h.nlevels;
  const double w = h.omega;
  T* cur[B2S_AMG_MAX_LEVELS];
  for (int l = 0; l < L; ++l) {
    const b2s_amg_level& lv = h.levels[l];
    const int lo = lv.group_ptr[g], hi = lv.group_ptr[g + 1];
    const T* b = (l == 0) ? rhs0 : (const T*)a.lb[l];
    const T* val = a.lval[l];
    const T* dinv = a.ldinv[l];
    const bool wide = wide_rows(lv.nnz, lv.n, a.wide_row);
    T* X = a.lx[l];
    T* Y = a.ly[l];
    T* c = X;
    // first sweep fused: x = w D^-1 b; then y = x + w D^-1 (b - A x) with x on the fly
    if (h.sweeps <= 1) {
      for (int i = lo + tm.t; i < hi; i += tm.n) X[i] = (w * (double)dinv[i]) * (double)b[i];
    } else {
      const BRows R(wide, lo, tm);
      for (int i = R.first; i < hi; i += R.stride) {
        double s = 0.0;
        for (int j = lv.rowptr[i] + R.lane; j < lv.rowptr[i + 1]; j += R.step) {
          const int cc = lv.col[j];
          s += (double)val[j] * ((w * (double)dinv[cc]) * (double)b[cc]);
        }
        s = R.total(s);
        const double wd = w * (double)dinv[i];
        if (R.writer()) X[i] = wd * (double)b[i] + wd * ((double)b[i] - s);
      }
      T* o = Y;
      for (int sw = 2; sw < h.sweeps; ++sw) {
        tm.sync();
        const BRows R2(wide, lo, tm);
        for (int i = R2.first; i < hi; i += R2.stride) {
          double s = 0.0;
          for (int j = lv.rowptr[i] + R2.lane; j < lv.rowptr[i + 1]; j += R2.step) s += (double)val[j] * (double)c[lv.col[j]];
          s = R2.total(s);
          if (R2.writer()) o[i] = (double)c[i] + (w * (double)dinv[i]) * ((double)b[i] - s);
        }
        T* tmp = c;
        c = o;
        o = tmp;
      }
    }
    tm.sync();
    T* Rv = a.lr[l];
    {
      const BRows R(wide, lo, tm);
      for (int i = R.first; i < hi; i += R.stride) {
        double s = 0.0;
        for (int j = lv.rowptr[i] + R.lane; j < lv.rowptr[i + 1]; j += R.step) s += (double)val[j] * (double)c[lv.col[j]];
        s = R.total(s);
        if (R.writer()) Rv[i] = (double)b[i] - s;
      }
    }
    tm.sync();
    const int clo = (l + 1 < L) ? h.levels[l + 1].group_ptr[g] : h.coarse_group_ptr[g];
    const int chi = (l + 1 < L) ? h.levels[l + 1].group_ptr[g + 1] : h.coarse_group_ptr[g + 1];
    T* bn = (l + 1 < L) ? a.lb[l + 1] : a.cb;
    {
      const BRows R(wide_rows(lv.p_nnz, lv.nc, a.wide_row), clo, tm);
      for (int I = R.first; I < chi; I += R.stride) {
        double s = 0.0;
        for (int j = lv.r_rowptr[I] + R.lane; j < lv.r_rowptr[I + 1]; j += R.step) s += (double)a.lrval[l][j] * (double)Rv[lv.r_col[j]];
        s = R.total(s);
        if (R.writer()) bn[I] = s;
      }
    }
    tm.sync();
    cur[l] = c;
  }
  // coarse: cx = inv_g cb (double inverse), one warp per row
  const T* cb = (L == 0) ? rhs0 : (const T*)a.cb;
  {
    const int clo = h.coarse_group_ptr[g], nn = h.coarse_group_ptr[g + 1] - clo;
    const double* inv = h.coarse_inv + h.coarse_inv_off[g];
    const int lane = tm.t & 31;
    for (int I = tm.t >> 5; I < nn; I += tm.n >> 5) {
      double s = 0.0;
      for (int J = lane; J < nn; J += 32) s += inv[(int64_t)I * nn + J] * (double)cb[clo + J];
      s = warp_sum(s);
      if (lane == 0) a.cx[clo + I] = s;
    }
  }
  tm.sync();
  for (int l = L - 1; l >= 0; --l) {
    const b2s_amg_level& lv = h.levels[l];
    const int lo = lv.group_ptr[g], hi = lv.group_ptr[g + 1];
    const T* b = (l == 0) ? rhs0 : (const T*)a.lb[l];
    const T* val = a.lval[l];
    const T* dinv = a.ldinv[l];
    const bool wide = wide_rows(lv.nnz, lv.n, a.wide_row);
    const T* xc = (l + 1 < L) ? (const T*)cur[l + 1] : (const T*)a.cx;
    T* c = cur[l];
    T* o = (c == a.lx[l]) ? a.ly[l] : a.lx[l];
    {
      const BRows R(wide_rows(lv.p_nnz, lv.n, a.wide_row), lo, tm);
      for (int i = R.first; i < hi; i += R.stride) {
        double s = 0.0;
        for (int j = lv.p_rowptr[i] + R.lane; j < lv.p_rowptr[i + 1]; j += R.step) s += (double)a.lpval[l][j] * (double)xc[lv.p_col[j]];
        s = R.total(s);
        if (R.writer()) c[i] = (double)c[i] + s;
      }
    }
    for (int sw = 0; sw < h.sweeps; ++sw) {
      tm.sync();
      const BRows R(wide, lo, tm);
      for (int i = R.first; i < hi; i += R.stride) {
        double s = 0.0;
        for (int j = lv.rowptr[i] + R.lane; j < lv.rowptr[i + 1]; j += R.step) s += (double)val[j] * (double)c[lv.col[j]];
        s = R.total(s);
        if (R.writer()) o[i] = (double)c[i] + (w * (double)dinv[i]) * ((double)b[i] - s);
      }
      T* tmp = c;
      c = o;
      o = tmp;
    }
    tm.sync();
    cur[l] = c;
  }
  (void)red;
  return L == 0 ? a.cx : cur[0];
}

struct GroupOutcome {
  int its, conv;
  double res;
};

// Preconditioned CG (flowtrace/linalg/krylov.py:25-65) of case g's rows, x = 0 at the start;
// with project the residual and the preconditioned residual are kept mean-free.
template <class T>
__device__ GroupOutcome pcg_group(const PcgGroupArgs<T>& a, int g, const T* bvec, T* x, double tol, int maxiter, Team& tm,
                                  bool project, double* red) {
  const int lo = a.h.nlevels ? a.h.levels[0].group_ptr[g] : a.h.coarse_group_ptr[g];
  const int hi = a.h.nlevels ? a.h.levels[0].group_ptr[g + 1] : a.h.coarse_group_ptr[g + 1];
  const double nd = (double)(hi - lo);
  T* r = a.r;
  T* p = a.p;
  T* q = a.q;
  double v2[2] = {0.0, 0.0};
  for (int i = lo + tm.t; i < hi; i += tm.n) {
    const double bi = bvec[i];
    x[i] = 0.0;
    v2[0] += bi * bi;
    v2[1] += bi;
  }
  tm.sum<2>(v2, red);
  const double bb = v2[0], mb = project ? v2[1] / nd : 0.0;
  double v1[1] = {0.0};
  for (int i = lo + tm.t; i < hi; i += tm.n) {
    const double ri = (double)bvec[i] - mb;
    r[i] = ri;
    v1[0] += ri * ri;
  }
  tm.sum<1>(v1, red);
  double bnorm = sqrt(bb);
  if (bnorm == 0.0) bnorm = 1.0;
  double rnorm = sqrt(v1[0]);
  GroupOutcome o = {0, 0, rnorm / bnorm};
  if (rnorm / bnorm < tol) {
    o.conv = 1;
    return o;
  }
  auto precondition = [&](double& rz) -> T* {
    T* z = vcycle_group(a, g, (const T*)r, red, tm);
    double s3[3] = {0.0, 0.0, 0.0};
    for (int i = lo + tm.t; i < hi; i += tm.n) {
      const double zi = z[i], ri = r[i];
      s3[0] += zi;
      s3[1] += ri * zi;
      s3[2] += ri;
    }
    tm.sum<3>(s3, red);
    const double zm = project ? s3[0] / nd : 0.0;
    if (project)
      for (int i = lo + tm.t; i < hi; i += tm.n) z[i] = (double)z[i] - zm;
    rz = project ? s3[1] - zm * s3[2] : s3[1];
    tm.sync();
    return z;
  };
  double rz;
  T* z = precondition(rz);
  for (int i = lo + tm.t; i < hi; i += tm.n) p[i] = z[i];
  tm.sync();
  for (int k = 1; k <= maxiter; ++k) {
    double pq[1] = {0.0};
    {
      const BRows R(false, lo, tm);
      for (int i = R.first; i < hi; i += R.stride) {
        double s = 0.0;
        for (int j = a.rowptr[i]; j < a.rowptr[i + 1]; ++j) s += (double)a.val[j] * (double)p[a.col[j]];
        q[i] = s;
        pq[0] += (double)p[i] * s;
      }
    }
    tm.sum<1>(pq, red);
    if (pq[0] <= 0.0) {
      o.its = k;
      o.res = rnorm / bnorm;
      return o;
    }
    const double alpha = rz / pq[0];
    double rr[1] = {0.0};
    for (int i = lo + tm.t; i < hi; i += tm.n) {
      x[i] = (double)x[i] + alpha * (double)p[i];
      const double ri = (double)r[i] - alpha * (double)q[i];
      r[i] = ri;
      rr[0] += ri * ri;
    }
    tm.sum<1>(rr, red);
    rnorm = sqrt(rr[0]);
    o.its = k;
    o.res = rnorm / bnorm;
    if (rnorm / bnorm < tol) {
      o.conv = 1;
      return o;
    }
    double rz_new;
    z = precondition(rz_new);
    if (rz == 0.0) return o;
    const double beta = rz_new / rz;
    rz = rz_new;
    for (int i = lo + tm.t; i < hi; i += tm.n) p[i] = (double)z[i] + beta * (double)p[i];
    tm.sync();
  }
  return o;
}

// Refined solve of case g: float PCG passes, double x += d and double residual from the face
// coefficients, the reference's stopping test on it (as b2s_pcg_amg_mixed_d, per case).
template <class T>
__device__ void pcg_refined_group(const PcgGroupArgs<T>& a, int g, double* red, Team& tm) {
  const b2s_mesh& m = a.m;
  const int lo = a.h.nlevels ? a.h.levels[0].group_ptr[g] : a.h.coarse_group_ptr[g];
  const int hi = a.h.nlevels ? a.h.levels[0].group_ptr[g + 1] : a.h.coarse_group_ptr[g + 1];
  const bool project = a.project[g] != 0;
  const double nd = (double)(hi - lo);
  double v2[2] = {0.0, 0.0};
  for (int i = lo + tm.t; i < hi; i += tm.n) {
    const double bi = a.b64[i];
    a.x64[i] = 0.0;
    v2[0] += bi * bi;
    v2[1] += bi;
  }
  tm.sum<2>(v2, red);
  double bnorm = sqrt(v2[0]);
  if (bnorm == 0.0) bnorm = 1.0;
  double mean = project ? v2[1] / nd : 0.0;
  double v1[1] = {0.0};
  for (int i = lo + tm.t; i < hi; i += tm.n) {
    const double ri = a.b64[i] - mean;
    a.r64[i] = ri;
    a.rb[i] = ri;
    v1[0] += ri * ri;
  }
  tm.sum<1>(v1, red);
  double res = sqrt(v1[0]) / bnorm;
  int its = 0, conv = res < a.tol ? 1 : 0;
  for (int pass = 0; pass < a.maxpass && !conv && its < a.maxiter; ++pass) {
    double tin = a.tol / res;
    if (tin < a.min_inner_tol) tin = a.min_inner_tol;
    const GroupOutcome o = pcg_group(a, g, (const T*)a.rb, a.d, tin, a.maxiter - its, tm, project, red);
    its += o.its;
    for (int i = lo + tm.t; i < hi; i += tm.n) a.x64[i] = a.x64[i] + (double)a.d[i];
    tm.sync();
    double s2[2] = {0.0, 0.0};
    for (int c = lo + tm.t; c < hi; c += tm.n) {
      const double xc = a.x64[c];
      double ax = 0.0;
      for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) ax += a.cf[f] * (xc - a.x64[m.fN[f]]);
      for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
        const int f = m.nei_face[k];
        ax += a.cf[f] * (xc - a.x64[m.fP[f]]);
      }
      for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) ax += a.cbf[f] * xc;
      const double ri = a.b64[c] - ax;
      a.r64[c] = ri;
      s2[0] += ri * ri;
      s2[1] += ri;
    }
    tm.sum<2>(s2, red);
    mean = project ? s2[1] / nd : 0.0;
    double rr = project ? s2[0] - s2[1] * mean : s2[0];
    if (rr < 0.0) rr = 0.0;
    res = sqrt(rr) / bnorm;
    if (!(res == res)) break;
    if (res < a.tol) {
      conv = 1;
      break;
    }
    if (o.its == 0 && !o.conv) break;
    for (int i = lo + tm.t; i < hi; i += tm.n) a.rb[i] = a.r64[i] - mean;
    tm.sync();
  }
  if (tm.t == 0) {
    a.info[g].iterations = its;
    a.info[g].converged = conv;
    a.info[g].residual = res;
  }
  tm.sync();
}

template <class T>
__global__ void __launch_bounds__(kBatchThreads) pcg_groups_k(PcgGroupArgs<T> a) {
  __shared__ double red[(kBatchWarps + 1) * 3];
  __shared__ double xbuf[16];
  Team tm = make_team(xbuf);
  const int cid = (int)blockIdx.x / tm.nb, ncl = (int)gridDim.x / tm.nb;
  for (int k = cid; k < a.h.ngroups; k += ncl) pcg_refined_group<T>(a, a.order[k], red, tm);
  tm.sync();  // no block leaves while another may still read its shared memory
}

}  // namespace b2s

using namespace b2s;

// The team shape of a call: the caller's configuration, or the default.
static int team_shape(const b2s_team_config* team, b2s_team_config* out) {
  b2s_team_config t = {kClusterBlocks, kBatchThreads, kBatchWideRow, 0};
  if (team) t = *team;
  if (t.cluster_blocks < 1 || t.cluster_blocks > 8 || t.block_threads < 64 || t.block_threads > kBatchThreads ||
      t.block_threads % 32 != 0 || t.wide_row < 0)
    return B2S_ERR_ARG;
  *out = t;
  return B2S_OK;
}

// Launch one team (a cluster of team.cluster_blocks blocks) per case up to the number of
// clusters that fit on the device at once; the teams then walk the case list.
static int launch_teams(const void* kernel, int ngroups, void** args, const b2s_team_config& team, b2s_stream_t s) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)team.cluster_blocks;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)team.cluster_blocks, 1, 1);
  cfg.blockDim = dim3((unsigned)team.block_threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = (cudaStream_t)s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int ncl = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, kernel, &cfg) != cudaSuccess || ncl < 1) return B2S_ERR_DEVICE;
  if (ncl > ngroups) ncl = ngroups;
  cfg.gridDim = dim3((unsigned)(ncl * team.cluster_blocks), 1, 1);
  if (cudaLaunchKernelExC(&cfg, kernel, args) != cudaSuccess) return B2S_ERR_LAUNCH;
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

template <class T>
static int launch_bicg_groups(BicgGroupArgs<T>& a, const b2s_team_config& team, b2s_stream_t s) {
  void* args[] = {&a};
  const void* k = a.nr == 1 ? (const void*)bicgstab_groups_k<1, T>
                  : a.nr == 2 ? (const void*)bicgstab_groups_k<2, T> : (const void*)bicgstab_groups_k<3, T>;
  return launch_teams(k, a.ngroups, args, team, s);
}

extern "C" {

int b2s_mesh_part_blocks(const b2s_mesh* m) {
  if (!m || m->nc <= 0) return -1;
  if (m->tiles) return m->ntiles;
  return b2s_part_blocks(m->nc);
}

int b2s_group_sums_d(const double* part, int nblk, int nq, int ngroups, const int32_t* group_tiles, double* out,
                     b2s_stream_t s) {
  if (!part || nblk <= 0 || nq <= 0 || ngroups <= 0 || !group_tiles || !out) return B2S_ERR_ARG;
  const int64_t warps = (int64_t)ngroups * nq;
  group_sums_k<<<grid_for(warps * 32), kThreads, 0, (cudaStream_t)s>>>(part, nblk, nq, ngroups, group_tiles, out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_remove_group_means_d(const b2s_mesh* m, double* x, const double* part, int nblk, int q,
                             const int32_t* group_tiles, const int32_t* tile_group, const int32_t* group_cells,
                             const int32_t* singular, b2s_stream_t s) {
  if (!m || !m->tiles || m->ntiles <= 0 || !x || !part || nblk != m->ntiles || q < 0 || !group_tiles ||
      !tile_group || !group_cells || !singular)
    return B2S_ERR_ARG;
  remove_group_means_k<<<(unsigned)m->ntiles, kThreads, 0, (cudaStream_t)s>>>(*m, x, part, nblk, q, group_tiles,
                                                                               tile_group, group_cells, singular);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int64_t b2s_bicgstab_groups_workspace_bytes(int32_t n, int nrhs, int single) {
  if (n <= 0 || nrhs < 1 || nrhs > 3) return -1;
  return (int64_t)(single ? sizeof(float) : sizeof(double)) * 7 * nrhs * (int64_t)n;
}

int b2s_bicgstab_groups_f32_d(int ngroups, const int32_t* group_ptr, const int32_t* order, int32_t n, int nrhs,
                              const int32_t* rowptr, const int32_t* col, const float* val, const float* b,
                              const float* inv_diag, float* x, double tol, int maxiter, int relative_to_initial,
                              int zero_x0, double* out64, const double* base64, void* work, int64_t work_bytes,
                              b2s_solve_info* info, const b2s_team_config* team, b2s_stream_t s) {
  if (ngroups <= 0 || !group_ptr || !order || n <= 0 || nrhs < 1 || nrhs > 3 || !rowptr || !col || !val || !b ||
      !inv_diag || !x || !work || !info || maxiter < 0 || ((out64 == nullptr) != (base64 == nullptr)))
    return B2S_ERR_ARG;
  b2s_team_config tc;
  if (team_shape(team, &tc) != B2S_OK) return B2S_ERR_ARG;
  if (work_bytes < b2s_bicgstab_groups_workspace_bytes(n, nrhs, 1)) return B2S_ERR_WORKSPACE;
  BicgGroupArgs<float> a;
  a.ngroups = ngroups;
  a.nr = nrhs;
  a.n = n;
  a.group_ptr = group_ptr;
  a.order = order;
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
  a.info = info;
  a.out64 = out64;
  a.base64 = base64;
  a.wide_row = tc.wide_row;
  return launch_bicg_groups(a, tc, s);
}

static bool amg_groups_ok(const b2s_amg* h, const b2s_amg_f32* h32) {
  if (!h || h->ngroups <= 0 || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS || !h->coarse_group_ptr ||
      !h->coarse_inv_off || !h->coarse_inv || !h32)
    return false;
  for (int l = 0; l < h->nlevels; ++l) {
    const b2s_amg_level& L = h->levels[l];
    if (!L.group_ptr || !L.rowptr || !L.p_rowptr || !L.r_rowptr || !h32->val[l] || !h32->dinv[l] || !h32->p_val[l] ||
        !h32->r_val[l])
      return false;
  }
  return true;
}

int64_t b2s_pcg_groups_workspace_bytes(const b2s_amg* h) {
  if (!h || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS) return -1;
  const int64_t n = h->nlevels ? h->levels[0].n : h->coarse_n;
  int64_t f = 3 * n + 2 * (int64_t)h->coarse_n + 2 * n;  // r, p, q, cb, cx, rb, d
  for (int l = 0; l < h->nlevels; ++l) f += 4 * (int64_t)h->levels[l].n;
  return n * (int64_t)sizeof(double) + f * (int64_t)sizeof(float) + 16;
}

int b2s_pcg_groups_mixed_d(const b2s_amg* h, const b2s_amg_f32* h32, const int32_t* order, const int32_t* project,
                           const b2s_mesh* m, const double* cf, const double* cb, int32_t n, const int32_t* rowptr,
                           const int32_t* col, const float* val, const double* b, double* x, double tol, int maxiter,
                           int maxpass, double min_inner_tol, void* work, int64_t work_bytes, b2s_solve_info* info,
                           const b2s_team_config* team, b2s_stream_t s) {
  if (!amg_groups_ok(h, h32) || !order || !project || !m || !cf || (!cb && m->nb) || !rowptr || !col || !val || !b ||
      !x || !work || !info || maxiter < 0 || maxpass < 1 || !(min_inner_tol > 0.0))
    return B2S_ERR_ARG;
  b2s_team_config tc;
  if (team_shape(team, &tc) != B2S_OK) return B2S_ERR_ARG;
  if (n != (h->nlevels ? h->levels[0].n : h->coarse_n) || n != m->nc) return B2S_ERR_ARG;
  if (work_bytes < b2s_pcg_groups_workspace_bytes(h)) return B2S_ERR_WORKSPACE;
  PcgGroupArgs<float> a;
  a.h = *h;
  double* dw = (double*)work;
  a.r64 = dw;
  float* fw = (float*)(dw + n);
  a.r = fw;
  a.p = fw + n;
  a.q = fw + 2 * (int64_t)n;
  a.cb = fw + 3 * (int64_t)n;
  a.cx = a.cb + h->coarse_n;
  float* c = a.cx + h->coarse_n;
  for (int l = 0; l < h->nlevels; ++l) {
    const int64_t ml = h->levels[l].n;
    a.lval[l] = h32->val[l];
    a.ldinv[l] = h32->dinv[l];
    a.lpval[l] = h32->p_val[l];
    a.lrval[l] = h32->r_val[l];
    a.lb[l] = c;
    a.lx[l] = c + ml;
    a.ly[l] = c + 2 * ml;
    a.lr[l] = c + 3 * ml;
    c += 4 * ml;
  }
  a.rb = c;
  a.d = c + n;
  a.n = n;
  a.rowptr = rowptr;
  a.col = col;
  a.val = val;
  a.m = *m;
  a.cf = cf;
  a.cbf = cb;
  a.b64 = b;
  a.x64 = x;
  a.order = order;
  a.project = project;
  a.tol = tol;
  a.maxiter = maxiter;
  a.maxpass = maxpass;
  a.min_inner_tol = min_inner_tol;
  a.info = info;
  a.wide_row = tc.wide_row;
  void* args[] = {&a};
  return launch_teams((const void*)pcg_groups_k<float>, h->ngroups, args, tc, s);
}

}  // extern "C"
