// Smoothed-aggregation AMG for the pressure-correction solve on B200.
//
// The reference builds its hierarchy on the host every 10 outer iterations
// (flowtrace/linalg/amg.py:80-117, flowtrace/unstructured/simple.py:624-628). Here the
// aggregates and the sparsity patterns of P, W = A P and A_c = P^T A P come from a set-up (the
// device set-up of b2s_amg_setup.cu, or the host one with b2s_host_aggregate below), and every
// numeric quantity is rebuilt on the device from the current matrix values:
//   D^-1, the spectral radius of D^-1 A (15 power iterations from a fixed start vector, as
//   amg.py:69-77), P = T - 4/(3 rho) D^-1 A T (amg.py:95-101), R = P^T, A_c = R (A P), and the
//   inverse of the coarsest matrix (shifted by 1e-10 mean|diag| when singular, amg.py:106-112).
// Products with a fixed output pattern are row-owned gathers: a thread accumulates one output
// row, locating each term's slot by binary search in the row's sorted columns; no atomics.
#include "b2s_common.cuh"

namespace b2s {

__device__ __forceinline__ int find_sorted(const int32_t* __restrict__ cols, int lo, int hi, int key) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (cols[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__global__ void dinv_k(b2s_amg_level L) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x)
    L.dinv[i] = 1.0 / L.val[L.diag_slot[i]];
}

// rho(D^-1 A) by 15 power iterations (amg.py:69-77): y = D^-1 A x, lam = |y|/max(|x|,1e-300),
// x = y/max(|y|,1e-300). The normalisation of x is folded into the next product (x_j = y_j/s
// read on the fly), so each iteration costs one grid barrier.
__global__ void __launch_bounds__(kCoopThreads) power_coop_k(b2s_amg_level L, double* ya, double* yb, double* part0,
                                                              double* part1) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double red[(kCoopThreads / 32 + 1) * 2];
  __shared__ double tot[2];
  const int n = L.n;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  double* part[2] = {part0, part1};
  double* ybuf[2] = {ya, yb};
  double lam = 1.0, sc = 1.0;
  for (int it = 0; it < 15; ++it) {
    const double* xin = it == 0 ? L.x0 : ybuf[(it - 1) & 1];
    double* yout = ybuf[it & 1];
    double acc[2] = {0.0, 0.0};
    for (int i = gt; i < n; i += gs) {
      const double di = L.dinv[i];
      double s = 0.0;
      for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
        const int c = L.col[j];
        const double xc = it == 0 ? xin[c] : xin[c] / sc;
        s += (di * L.val[j]) * xc;
      }
      yout[i] = s;
      acc[0] += s * s;
      const double xi = it == 0 ? xin[i] : xin[i] / sc;
      acc[1] += xi * xi;
    }
    block_partials<2>(acc, red, part[it & 1]);
    grid.sync();
    grid_totals(part[it & 1], gridDim.x, 2, tot);
    const double ny = sqrt(tot[0]), nx = sqrt(tot[1]);
    lam = ny / fmax(nx, 1e-300);
    sc = fmax(ny, 1e-300);
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *L.rho = lam;
}

// The same power iteration by one block (levels of at most kPowerBlockRows rows, where a grid
// barrier per iteration costs more than the work).
constexpr int kPowerBlockRows = 2048;

// Batches: the power iteration of power_block_k per case (one block per case on its rows). A
// case that this level does not coarsen (every row its own aggregate, next_ptr giving the same
// row count) gets rho = infinity, so that its prolongation is the plain injection P = T and its
// coarse block the same matrix.
__global__ void __launch_bounds__(kCoopThreads) power_groups_k(b2s_amg_level L, const int32_t* __restrict__ next_ptr,
                                                              double* ya, double* yb) {
  __shared__ double red[(kCoopThreads / 32 + 1) * 2];
  const int g = blockIdx.x, lo = L.group_ptr[g], hi = L.group_ptr[g + 1];
  if (next_ptr[g + 1] - next_ptr[g] == hi - lo) {
    if (threadIdx.x == 0) L.rho[g] = INFINITY;
    return;
  }
  double* ybuf[2] = {ya, yb};
  double lam = 1.0, sc = 1.0;
  for (int it = 0; it < 15; ++it) {
    const double* xin = it == 0 ? L.x0 : ybuf[(it - 1) & 1];
    double* yout = ybuf[it & 1];
    double acc[2] = {0.0, 0.0};
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      const double di = L.dinv[i];
      double s = 0.0;
      for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
        const int c = L.col[j];
        const double xc = it == 0 ? xin[c] : xin[c] / sc;
        s += (di * L.val[j]) * xc;
      }
      yout[i] = s;
      acc[0] += s * s;
      const double xi = it == 0 ? xin[i] : xin[i] / sc;
      acc[1] += xi * xi;
    }
    double tot[2];
    block_sum<2>(acc, red, tot);
    const double ny = sqrt(tot[0]), nx = sqrt(tot[1]);
    lam = ny / fmax(nx, 1e-300);
    sc = fmax(ny, 1e-300);
  }
  if (threadIdx.x == 0) L.rho[g] = lam;
}

__global__ void __launch_bounds__(kCoopThreads) power_block_k(b2s_amg_level L, double* ya, double* yb) {
  __shared__ double red[(kCoopThreads / 32 + 1) * 2];
  double* ybuf[2] = {ya, yb};
  double lam = 1.0, sc = 1.0;
  for (int it = 0; it < 15; ++it) {
    const double* xin = it == 0 ? L.x0 : ybuf[(it - 1) & 1];
    double* yout = ybuf[it & 1];
    double acc[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) {
      const double di = L.dinv[i];
      double s = 0.0;
      for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
        const int c = L.col[j];
        const double xc = it == 0 ? xin[c] : xin[c] / sc;
        s += (di * L.val[j]) * xc;
      }
      yout[i] = s;
      acc[0] += s * s;
      const double xi = it == 0 ? xin[i] : xin[i] / sc;
      acc[1] += xi * xi;
    }
    double tot[2];
    block_sum<2>(acc, red, tot);
    const double ny = sqrt(tot[0]), nx = sqrt(tot[1]);
    lam = ny / fmax(nx, 1e-300);
    sc = fmax(ny, 1e-300);
  }
  if (threadIdx.x == 0) *L.rho = lam;
}

// P[i,J] = T[i,J] - c sum_{k in row i, agg[k] = J} (Dinv_i A_ik) T[k,J], c = (4/3)/rho
// With ngroups > 0 (batches) the spectral radius is per case: rho[g] for the rows of case g.
__global__ void pvals_k(b2s_amg_level L, int ngroups) {
  const double c0 = ngroups > 0 ? 0.0 : (4.0 / 3.0) / *L.rho;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x) {
    double c = c0;
    if (ngroups > 0) {
      int lo = 0, hi = ngroups;  // the case g with group_ptr[g] <= i < group_ptr[g+1]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (L.group_ptr[mid] <= i) lo = mid;
        else hi = mid;
      }
      c = (4.0 / 3.0) / L.rho[lo];
    }
    const int p0 = L.p_rowptr[i], p1 = L.p_rowptr[i + 1];
    for (int s = p0; s < p1; ++s) L.p_val[s] = 0.0;
    const double di = L.dinv[i];
    for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
      const int J = L.agg[L.col[j]];
      const int s = find_sorted(L.p_col, p0, p1, J);
      L.p_val[s] += (di * L.val[j]) * L.tval[J];
    }
    const int ai = L.agg[i];
    for (int s = p0; s < p1; ++s) {
      const int J = L.p_col[s];
      const double t = (J == ai) ? L.tval[J] : 0.0;
      L.p_val[s] = t - c * L.p_val[s];
    }
  }
}

// The same P from the level's term lists: thread per row, each slot's terms in list order (the
// order pvals_k adds them), no search; batches take rho of the row's case, as pvals_k does.
__global__ void pvals_terms_k(b2s_amg_level L, int ngroups) {
  const double c0 = ngroups > 0 ? 0.0 : (4.0 / 3.0) / *L.rho;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x) {
    double c = c0;
    if (ngroups > 0) {
      int lo = 0, hi = ngroups;  // the case g with group_ptr[g] <= i < group_ptr[g+1]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (L.group_ptr[mid] <= i) lo = mid;
        else hi = mid;
      }
      c = (4.0 / 3.0) / L.rho[lo];
    }
    const double di = L.dinv[i];
    const int ai = L.agg[i];
    for (int s = L.p_rowptr[i]; s < L.p_rowptr[i + 1]; ++s) {
      const int J = L.p_col[s];
      const double tJ = L.tval[J];
      double acc = 0.0;
      for (int t = L.p_tptr[s]; t < L.p_tptr[s + 1]; ++t) acc += (di * L.val[L.p_tj[t]]) * tJ;
      L.p_val[s] = ((J == ai) ? tJ : 0.0) - c * acc;
    }
  }
}

// W = A P from the term lists: thread per W entry, terms in the order wvals_k adds them.
__global__ void wvals_terms_k(b2s_amg_level L) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.w_nnz; s += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int t = L.w_tptr[s]; t < L.w_tptr[s + 1]; ++t) acc += L.val[L.w_tj[t]] * L.p_val[L.w_te[t]];
    L.w_val[s] = acc;
  }
}

// A_c = R W from the term lists: thread per A_c entry, terms in R-entry order (as acvals_k).
__global__ void acvals_terms_k(b2s_amg_level L, double* __restrict__ cval) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.c_nnz; s += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int t = L.c_tptr[s]; t < L.c_tptr[s + 1]; ++t) acc += L.r_val[L.c_te[t]] * L.w_val[L.c_ts[t]];
    cval[s] = acc;
  }
}

__global__ void rvals_k(b2s_amg_level L) {
  const int nnz = L.p_nnz;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += gridDim.x * blockDim.x)
    L.r_val[e] = L.p_val[L.r_from_p[e]];
}

// W = A P, row-owned
__global__ void wvals_k(b2s_amg_level L) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x) {
    const int w0 = L.w_rowptr[i], w1 = L.w_rowptr[i + 1];
    for (int s = w0; s < w1; ++s) L.w_val[s] = 0.0;
    for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
      const double a = L.val[j];
      const int k = L.col[j];
      for (int e = L.p_rowptr[k]; e < L.p_rowptr[k + 1]; ++e) {
        const int s = find_sorted(L.w_col, w0, w1, L.p_col[e]);
        L.w_val[s] += a * L.p_val[e];
      }
    }
  }
}

// A_c = R W (the next level's matrix). One warp per coarse row I: the row's sorted columns and
// an accumulator are staged in shared memory; for each R entry (I, i) in order, the lanes split
// W row i, whose columns are distinct, so every accumulator slot receives its terms in the
// fixed order of the R entries (deterministic, no atomics). Rows longer than the staging
// capacity are processed in windows of kRowCap consecutive columns.
constexpr int kRowCap = 256;
constexpr int kGalWarps = 8;

__global__ void __launch_bounds__(kGalWarps * 32) acvals_k(b2s_amg_level L, const int32_t* __restrict__ crowptr,
                                                           const int32_t* __restrict__ ccol,
                                                           double* __restrict__ cval) {
  __shared__ int scol[kGalWarps][kRowCap];
  __shared__ double sacc[kGalWarps][kRowCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (int I = blockIdx.x * kGalWarps + wib; I < L.nc; I += gridDim.x * kGalWarps) {
    const int c0 = crowptr[I], c1 = crowptr[I + 1], m = c1 - c0;
    const int e0 = L.r_rowptr[I], e1 = L.r_rowptr[I + 1];
    if (m <= kRowCap) {
      for (int t = lane; t < m; t += 32) {
        scol[wib][t] = ccol[c0 + t];
        sacc[wib][t] = 0.0;
      }
      __syncwarp();
      for (int e = e0; e < e1; ++e) {
        const double rv = L.r_val[e];
        const int i = L.r_col[e];
        const int w1 = L.w_rowptr[i + 1];
        for (int s = L.w_rowptr[i] + lane; s < w1; s += 32) {
          const int t = find_sorted(scol[wib], 0, m, L.w_col[s]);
          sacc[wib][t] += rv * L.w_val[s];
        }
        __syncwarp();
      }
      for (int t = lane; t < m; t += 32) cval[c0 + t] = sacc[wib][t];
      __syncwarp();
    } else {
      // a long row: windows of kRowCap columns, each staged and accumulated as above; W entries
      // outside the window's column range are skipped (every slot still receives its terms in
      // the order of the R entries)
      for (int t0 = 0; t0 < m; t0 += kRowCap) {
        const int mw = (m - t0) < kRowCap ? (m - t0) : kRowCap;
        for (int t = lane; t < mw; t += 32) {
          scol[wib][t] = ccol[c0 + t0 + t];
          sacc[wib][t] = 0.0;
        }
        __syncwarp();
        const int lo = scol[wib][0], hi = scol[wib][mw - 1];
        for (int e = e0; e < e1; ++e) {
          const double rv = L.r_val[e];
          const int i = L.r_col[e];
          const int w1 = L.w_rowptr[i + 1];
          for (int s = L.w_rowptr[i] + lane; s < w1; s += 32) {
            const int c = L.w_col[s];
            if (c < lo || c > hi) continue;
            const int t = find_sorted(scol[wib], 0, mw, c);
            if (t < mw && scol[wib][t] == c) sacc[wib][t] += rv * L.w_val[s];
          }
          __syncwarp();
        }
        for (int t = lane; t < mw; t += 32) cval[c0 + t0 + t] = sacc[wib][t];
        __syncwarp();
      }
    }
  }
}

// Dense coarse matrix M (n x n, row-major) with the singular shift, then its inverse by
// Gauss-Jordan elimination in place, by one block.
constexpr int kGJThreads = 1024;
constexpr int kSmemCoarse = 160;  // n <= 160: the matrix lives in shared memory (<= 200 KB)

// Dense inverse of the n x n matrix whose CSR rows are rows r0 .. r0+n-1 (columns r0 ..
// r0+n-1) of (rowptr, col, val), by the calling block; M is the n x n work matrix.
__device__ __forceinline__ void gj_inverse(int n, int r0, const int32_t* __restrict__ rowptr,
                                           const int32_t* __restrict__ col, const double* __restrict__ val,
                                           int singular, double* M, double* __restrict__ inv, double* rowk,
                                           double* colk, double* shift_s) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < n * n; e += nt) M[e] = 0.0;
  __syncthreads();
  for (int r = tid; r < n; r += nt)
    for (int j = rowptr[r0 + r]; j < rowptr[r0 + r + 1]; ++j) M[(int64_t)r * n + (col[j] - r0)] = val[j];
  __syncthreads();
  if (singular) {
    if (tid < 32) {
      double s = 0.0;
      for (int r = tid; r < n; r += 32) s += fabs(M[(int64_t)r * n + r]);
      s = warp_sum(s);
      if (tid == 0) *shift_s = 1e-10 * (s / (double)n);
    }
    __syncthreads();
    for (int r = tid; r < n; r += nt) M[(int64_t)r * n + r] = M[(int64_t)r * n + r] + *shift_s;
    __syncthreads();
  }
  // In-place Gauss-Jordan inversion. The coarse matrix is symmetric positive definite (a
  // Galerkin product of the SPD pressure-correction matrix, shifted when singular), so no
  // pivoting is needed. Step k copies the pivot column and the pivot row scaled by 1/p (one
  // division per step), then updates every entry at once:
  //   M[k][k] = 1/p, M[k][c] = M[k][c]/p, M[r][k] = -M[r][k]/p, M[r][c] -= M[r][k] (M[k][c]/p).
  for (int k = 0; k < n; ++k) {
    const double rp = 1.0 / M[(int64_t)k * n + k];
    for (int i = tid; i < n; i += nt) {
      rowk[i] = M[(int64_t)k * n + i] * rp;
      colk[i] = M[(int64_t)i * n + k];
    }
    __syncthreads();
    for (int r = tid >> 5; r < n; r += nt >> 5) {  // rows over warps, columns over lanes
      double* Mr = M + (int64_t)r * n;
      const double cr = colk[r];
      for (int c = tid & 31; c < n; c += 32) {
        double v;
        if (r == k) v = (c == k) ? rp : rowk[c];
        else if (c == k) v = -cr * rp;
        else v = Mr[c] - cr * rowk[c];
        Mr[c] = v;
      }
    }
    __syncthreads();
  }
  for (int e = tid; e < n * n; e += nt) inv[e] = M[e];
  __syncthreads();
}

__global__ void __launch_bounds__(kGJThreads) coarse_inverse_k(int n, const int32_t* __restrict__ rowptr,
                                                              const int32_t* __restrict__ col,
                                                              const double* __restrict__ val, int singular,
                                                              double* __restrict__ Mg, double* __restrict__ inv) {
  extern __shared__ double smem[];
  __shared__ double shift_s;
  __shared__ double rowk[1024];
  __shared__ double colk[1024];
  double* M = n <= kSmemCoarse ? smem : Mg;
  gj_inverse(n, 0, rowptr, col, val, singular, M, inv, rowk, colk, &shift_s);
}

// Batches: the dense inverse of every case's coarse block, one block per case (n_g <= kSmemCoarse).
__global__ void __launch_bounds__(kGJThreads) coarse_inverse_groups_k(const int32_t* __restrict__ gptr,
                                                                     const int64_t* __restrict__ off,
                                                                     const int32_t* __restrict__ gsing,
                                                                     const int32_t* __restrict__ rowptr,
                                                                     const int32_t* __restrict__ col,
                                                                     const double* __restrict__ val,
                                                                     double* __restrict__ inv) {
  extern __shared__ double smem[];
  __shared__ double shift_s;
  __shared__ double rowk[kSmemCoarse];
  __shared__ double colk[kSmemCoarse];
  const int g = blockIdx.x, r0 = gptr[g], n = gptr[g + 1] - r0;
  gj_inverse(n, r0, rowptr, col, val, gsing[g], smem, inv + off[g], rowk, colk, &shift_s);
}

__global__ void strength_changes_k(b2s_amg_level L, double theta, int32_t* __restrict__ count) {
  int local = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.n; i += gridDim.x * blockDim.x) {
    const double di = fabs(L.val[L.diag_slot[i]]);
    for (int j = L.rowptr[i]; j < L.rowptr[i + 1]; ++j) {
      const int c = L.col[j];
      if (c == i) continue;
      const double dc = fabs(L.val[L.diag_slot[c]]);
      const int strong = fabs(L.val[j]) >= theta * sqrt(di * dc) ? 1 : 0;
      local += strong != (int)L.strong[j];
    }
  }
  if (local) atomicAdd(count, local);  // integer sum: order-independent
}

}  // namespace b2s

using namespace b2s;

static int power_grid(int* g) {
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return B2S_ERR_DEVICE;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return B2S_ERR_DEVICE;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, power_coop_k, kCoopThreads, 0) != cudaSuccess)
    return B2S_ERR_DEVICE;
  if (per <= 0) return B2S_ERR_DEVICE;
  if (per > 1) per = 1;
  *g = sms * per;
  if (*g > kMaxCoopBlocks) *g = kMaxCoopBlocks;
  return B2S_OK;
}

namespace b2s {
// ---------------------------------------------------------------------------------- float copies
struct F32Segs {
  int n;
  const double* src[4 * B2S_AMG_MAX_LEVELS];
  float* dst[4 * B2S_AMG_MAX_LEVELS];
  int64_t len[4 * B2S_AMG_MAX_LEVELS];
};

__global__ void to_f32_k(F32Segs s) {
  const int k = blockIdx.y;
  if (k >= s.n) return;
  const double* src = s.src[k];
  float* dst = s.dst[k];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < s.len[k]; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}
}  // namespace b2s

extern "C" {

int64_t b2s_amg_workspace_bytes(const b2s_amg* h) {
  if (!h || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS || h->coarse_n < 1) return -1;
  int64_t nmax = 0;
  for (int l = 0; l < h->nlevels; ++l) nmax = h->levels[l].n > nmax ? h->levels[l].n : nmax;
  int64_t dense = (h->ngroups == 0 && h->coarse_n > kSmemCoarse) ? (int64_t)h->coarse_n * h->coarse_n : 0;
  return (int64_t)sizeof(double) * (2 * nmax + 4 * (int64_t)kMaxCoopBlocks + dense);
}

}  // extern "C"

namespace {
// Numeric rebuild of one level from its matrix values: D^-1, rho, P, R, W = A P and the next
// level's values A_c = R W on the pattern (crow, ccol).
int rebuild_level(const b2s_amg_level& L, int ngroups, const int32_t* next_group_ptr, const int32_t* crow,
                  const int32_t* ccol, double* cval, double* xa, double* xb, double* part0, double* part1, int g,
                  cudaStream_t st) {
  if (!L.diag_slot || !L.agg || !L.tval || !L.x0 || !L.p_col || !L.p_val || !L.r_col || !L.r_from_p || !L.r_val ||
      !L.w_rowptr || !L.w_col || !L.w_val || !L.rho || !crow || !ccol || !cval)
    return B2S_ERR_ARG;
  dinv_k<<<grid_for(L.n), kThreads, 0, st>>>(L);
  B2S_LAUNCH_CHECK();
  if (ngroups > 0) {
    if (!L.group_ptr || !next_group_ptr) return B2S_ERR_ARG;
    power_groups_k<<<(unsigned)ngroups, kCoopThreads, 0, st>>>(L, next_group_ptr, xa, xb);
  } else if (L.n <= kPowerBlockRows) {
    power_block_k<<<1, kCoopThreads, 0, st>>>(L, xa, xb);
  } else {
    b2s_amg_level Lc = L;
    void* args[] = {&Lc, &xa, &xb, &part0, &part1};  // xa, xb: the two power-iteration buffers
    if (cudaLaunchCooperativeKernel((void*)power_coop_k, g, kCoopThreads, args, 0, st) != cudaSuccess)
      return B2S_ERR_LAUNCH;
  }
  const bool terms = L.p_tptr && L.p_tj && L.w_tptr && L.w_tj && L.w_te;
  if (terms) pvals_terms_k<<<grid_for(L.n), kThreads, 0, st>>>(L, ngroups);
  else pvals_k<<<grid_for(L.n), kThreads, 0, st>>>(L, ngroups);
  rvals_k<<<grid_for(L.p_nnz), kThreads, 0, st>>>(L);
  if (terms) wvals_terms_k<<<grid_for(L.w_nnz), kThreads, 0, st>>>(L);
  else wvals_k<<<grid_for(L.n), kThreads, 0, st>>>(L);
  B2S_LAUNCH_CHECK();
  if (terms && L.c_tptr && L.c_te && L.c_ts && L.c_nnz > 0)
    acvals_terms_k<<<grid_for(L.c_nnz), kThreads, 0, st>>>(L, cval);
  else
    acvals_k<<<(unsigned)cdiv(L.nc, kGalWarps), kGalWarps * 32, 0, st>>>(L, crow, ccol, cval);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int coarse_inverse(const b2s_amg* h, double* dense, cudaStream_t st) {
  if (h->ngroups > 0) {  // one dense block per case, each at most kSmemCoarse rows (checked at set-up)
    const size_t gsm = (size_t)kSmemCoarse * kSmemCoarse * sizeof(double);
    if (cudaFuncSetAttribute(coarse_inverse_groups_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsm) !=
        cudaSuccess)
      return B2S_ERR_LAUNCH;
    coarse_inverse_groups_k<<<(unsigned)h->ngroups, kGJThreads, gsm, st>>>(
        h->coarse_group_ptr, h->coarse_inv_off, h->group_singular, h->coarse_rowptr, h->coarse_col, h->coarse_val,
        h->coarse_inv);
    B2S_LAUNCH_CHECK();
    return B2S_OK;
  }
  const int n = h->coarse_n;
  const size_t smem = n <= kSmemCoarse ? (size_t)n * n * sizeof(double) : 0;
  // the dynamic share above 48 KB minus the kernel's static 16 KB needs the opt-in
  if (smem > 0 && cudaFuncSetAttribute(coarse_inverse_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                      cudaSuccess)
    return B2S_ERR_LAUNCH;
  coarse_inverse_k<<<1, kGJThreads, smem, st>>>(n, h->coarse_rowptr, h->coarse_col, h->coarse_val, h->singular,
                                                dense, h->coarse_inv);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

bool hierarchy_ok(const b2s_amg* h) {
  return h && h->nlevels >= 0 && h->nlevels <= B2S_AMG_MAX_LEVELS && h->coarse_n >= 1 &&
         !(h->ngroups == 0 && h->coarse_n > 1024) && h->coarse_inv && h->coarse_rowptr && h->coarse_col &&
         h->coarse_val && !(h->ngroups > 0 && (!h->coarse_group_ptr || !h->coarse_inv_off || !h->group_singular));
}
}  // namespace

extern "C" {

int b2s_amg_rebuild_d(const b2s_amg* h, void* work, int64_t work_bytes, b2s_stream_t s) {
  if (!hierarchy_ok(h) || !work) return B2S_ERR_ARG;
  if (work_bytes < b2s_amg_workspace_bytes(h)) return B2S_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)s;
  int64_t nmax = 0;
  for (int l = 0; l < h->nlevels; ++l) nmax = h->levels[l].n > nmax ? h->levels[l].n : nmax;
  double* xa = (double*)work;
  double* xb = xa + nmax;
  double* part0 = xb + nmax;
  double* part1 = part0 + 2 * (int64_t)kMaxCoopBlocks;
  double* dense = part1 + 2 * (int64_t)kMaxCoopBlocks;
  int g = 0, rc;
  if ((rc = power_grid(&g)) != B2S_OK) return rc;
  for (int l = 0; l < h->nlevels; ++l) {
    const bool last = l + 1 == h->nlevels;
    const int32_t* next_gp = last ? h->coarse_group_ptr : h->levels[l + 1].group_ptr;
    const int32_t* crow = last ? h->coarse_rowptr : h->levels[l + 1].rowptr;
    const int32_t* ccol = last ? h->coarse_col : h->levels[l + 1].col;
    double* cval = last ? h->coarse_val : h->levels[l + 1].val;
    if ((rc = rebuild_level(h->levels[l], h->ngroups, next_gp, crow, ccol, cval, xa, xb, part0, part1, g, st)) !=
        B2S_OK)
      return rc;
  }
  return coarse_inverse(h, dense, st);
}

int64_t b2s_amg_level_workspace_bytes(const b2s_amg_level* L) {
  if (!L || L->n < 1) return -1;
  return (int64_t)sizeof(double) * (2 * (int64_t)L->n + 4 * (int64_t)kMaxCoopBlocks);
}

int b2s_amg_level_rebuild_d(const b2s_amg_level* L, const int32_t* crow, const int32_t* ccol, double* cval,
                            void* work, int64_t work_bytes, b2s_stream_t s) {
  if (!L || L->n < 1 || !work) return B2S_ERR_ARG;
  if (work_bytes < b2s_amg_level_workspace_bytes(L)) return B2S_ERR_WORKSPACE;
  double* xa = (double*)work;
  double* xb = xa + L->n;
  double* part0 = xb + L->n;
  double* part1 = part0 + 2 * (int64_t)kMaxCoopBlocks;
  int g = 0, rc;
  if ((rc = power_grid(&g)) != B2S_OK) return rc;
  return rebuild_level(*L, 0, nullptr, crow, ccol, cval, xa, xb, part0, part1, g, (cudaStream_t)s);
}

int b2s_amg_coarse_inverse_d(const b2s_amg* h, void* work, int64_t work_bytes, b2s_stream_t s) {
  if (!hierarchy_ok(h) || !work) return B2S_ERR_ARG;
  if (work_bytes < b2s_amg_workspace_bytes(h)) return B2S_ERR_WORKSPACE;
  int64_t nmax = 0;
  for (int l = 0; l < h->nlevels; ++l) nmax = h->levels[l].n > nmax ? h->levels[l].n : nmax;
  double* dense = (double*)work + 2 * nmax + 4 * (int64_t)kMaxCoopBlocks;
  return coarse_inverse(h, dense, (cudaStream_t)s);
}

int b2s_amg_strength_changes_d(const b2s_amg* h, double theta, int32_t* count, b2s_stream_t s) {
  if (!h || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS || !count) return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (cudaMemsetAsync(count, 0, sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  for (int l = 0; l < h->nlevels; ++l) {
    const b2s_amg_level& L = h->levels[l];
    if (!L.strong || !L.diag_slot) return B2S_ERR_ARG;
    strength_changes_k<<<grid_for(L.n), kThreads, 0, st>>>(L, theta, count);
    B2S_LAUNCH_CHECK();
  }
  return B2S_OK;
}

int b2s_amg_level_strength_changes_d(const b2s_amg* h, double theta, int32_t* counts, b2s_stream_t s) {
  if (!h || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS || (h->nlevels > 0 && !counts)) return B2S_ERR_ARG;
  if (h->nlevels == 0) return B2S_OK;
  cudaStream_t st = (cudaStream_t)s;
  if (cudaMemsetAsync(counts, 0, sizeof(int32_t) * h->nlevels, st) != cudaSuccess) return B2S_ERR_LAUNCH;
  for (int l = 0; l < h->nlevels; ++l) {
    const b2s_amg_level& L = h->levels[l];
    if (!L.strong || !L.diag_slot) return B2S_ERR_ARG;
    strength_changes_k<<<grid_for(L.n), kThreads, 0, st>>>(L, theta, counts + l);
    B2S_LAUNCH_CHECK();
  }
  return B2S_OK;
}

/* Greedy three-pass aggregation of flowtrace/linalg/amg.py:25-57 on the strength graph
 * (host CSR); agg[n] receives the aggregate of every node, the return value their number. */
int64_t b2s_host_aggregate(int64_t n, const int64_t* indptr, const int64_t* indices, int64_t* agg) {
  if (n < 0 || !indptr || !indices || !agg) return -1;
  for (int64_t i = 0; i < n; ++i) agg[i] = -1;
  int64_t na = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool free_ = true;
    for (int64_t k = indptr[i]; k < indptr[i + 1]; ++k)
      if (agg[indices[k]] >= 0) {
        free_ = false;
        break;
      }
    if (free_) {
      agg[i] = na;
      for (int64_t k = indptr[i]; k < indptr[i + 1]; ++k) agg[indices[k]] = na;
      ++na;
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    for (int64_t k = indptr[i]; k < indptr[i + 1]; ++k) {
      const int64_t j = indices[k];
      if (agg[j] >= 0) {
        agg[i] = agg[j];
        break;
      }
    }
  }
  for (int64_t i = 0; i < n; ++i)
    if (agg[i] < 0) agg[i] = na++;
  return na;
}

int b2s_amg_to_f32_d(const b2s_amg* h, const b2s_amg_f32* h32, b2s_stream_t s) {
  if (!h || !h32 || h->nlevels < 0 || h->nlevels > B2S_AMG_MAX_LEVELS) return B2S_ERR_ARG;
  F32Segs g;
  g.n = 0;
  int64_t longest = 1;
  for (int l = 0; l < h->nlevels; ++l) {
    const b2s_amg_level& L = h->levels[l];
    const double* src[4] = {L.val, L.dinv, L.p_val, L.r_val};
    float* dst[4] = {h32->val[l], h32->dinv[l], h32->p_val[l], h32->r_val[l]};
    const int64_t len[4] = {L.nnz, L.n, L.p_nnz, L.p_nnz};
    for (int q = 0; q < 4; ++q) {
      if (!src[q] || !dst[q]) return B2S_ERR_ARG;
      g.src[g.n] = src[q];
      g.dst[g.n] = dst[q];
      g.len[g.n] = len[q];
      if (len[q] > longest) longest = len[q];
      ++g.n;
    }
  }
  if (g.n == 0) return B2S_OK;
  int64_t gx = cdiv(longest, kThreads);
  if (gx > 4 * kMaxCoopBlocks) gx = 4 * kMaxCoopBlocks;
  to_f32_k<<<dim3((unsigned)gx, (unsigned)g.n), kThreads, 0, (cudaStream_t)s>>>(g);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"
