// Device set-up of the SA-AMG hierarchy: strength of connection, transposed entry slots and the
// greedy three-pass aggregation of flowtrace/linalg/amg.py:25-57, reproduced exactly.
//
// The reference's aggregation visits the nodes one after another in index order (the "priority"
// here: the reference numbering on level 0, the aggregate numbering below):
//   pass 1: a node becomes a root when it and all its strong neighbours S(i) are still free; the
//           root takes S(i) into its aggregate;
//   pass 2: a node left free joins the aggregate of its first strong neighbour (column order)
//           that already has one;
//   pass 3: nodes still free become aggregates of their own.
// Pass 1 is a lexicographically-first independent set: at its turn a node i is free with a
// free neighbourhood exactly when no earlier root r is in conflict with it, where r conflicts
// with i when i is in S(r), r is in S(i), or S(i) and S(r) share a node. So i is a root iff
// every conflicting node of lower priority is decided "not a root". The kernel below decides
// every node as soon as that holds, by dataflow: thread t owns the nodes of priority t, t + T,
// ... (T threads, all resident through a cooperative launch), visits them in increasing
// priority, and polls the decisions of the node's lower-priority conflicts until it can
// decide. The undecided node of lowest priority can always decide, and its owner is working
// on it, so the kernel finishes in as many dependent steps as the longest chain of decisions;
// every poll loop is bounded and a run that exhausts it reports an error instead of waiting.
// Roots are numbered in priority order (a scan), exactly as the reference's counter; every
// other node finds its root (at most one root has it in its S), and pass 2's choice - the
// lowest-priority strong neighbour that is aggregated at that point, i.e. aggregated in pass 1
// or left over with a lower priority - is resolved by following those links down in priority.
#include "b2s_common.cuh"

namespace b2s {

constexpr int32_t kUndecided = 0, kRoot = 1, kNotRoot = 2;
constexpr int kScanTile = 1024;

__device__ __forceinline__ int32_t ld_relaxed(const int32_t* p) {
  int32_t v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_relaxed(int32_t* p, int32_t v) {
  asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// strong[e] = 1 where |a_e| >= theta sqrt(|a_ii a_jj|), j = col[e] != i (amg.py:60-66, the same
// operations in the same order).
__global__ void strength_k(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                           const double* __restrict__ val, const int32_t* __restrict__ diag_slot, double theta,
                           uint8_t* __restrict__ strong) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double di = fabs(val[diag_slot[i]]);
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      const int c = col[e];
      uint8_t s = 0;
      if (c != i) s = fabs(val[e]) >= theta * sqrt(di * fabs(val[diag_slot[c]])) ? 1 : 0;
      strong[e] = s;
    }
  }
}

// tslot[e] = the slot of (col[e], i) for every entry e = (i, col[e]) of a structurally symmetric
// pattern; a missing transpose is counted in *missing and its slot set to e itself.
__global__ void transpose_slots_k(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                  int sorted, int32_t* __restrict__ tslot, int32_t* __restrict__ missing) {
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      const int c = col[e];
      int lo = rowptr[c], hi = rowptr[c + 1], found = -1;
      if (c == i) {
        found = e;
      } else if (sorted) {
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (col[mid] < i) lo = mid + 1;
          else hi = mid;
        }
        if (lo < rowptr[c + 1] && col[lo] == i) found = lo;
      } else {
        for (int q = lo; q < hi; ++q)
          if (col[q] == i) {
            found = q;
            break;
          }
      }
      if (found < 0) {
        ++bad;
        found = e;
      }
      tslot[e] = found;
    }
  }
  if (bad) atomicAdd(missing, bad);
}

struct AggGraph {
  int n;
  const int32_t* rowptr;
  const int32_t* col;
  const uint8_t* strong;  // strong[e]: col[e] in S(row)
  const int32_t* tslot;   // strong[tslot[e]]: row in S(col[e])
  const int32_t* prio;    // [n] priority (visiting order) of every node
  const int32_t* rank_node;  // [n] node of every priority
};

// The lower-priority conflicts of node i, in a fixed order: j in row i with i in S(j) or j in
// S(i); then, for every j in S(i), the nodes r with j in S(r) (they would have taken j). A node
// may appear more than once. count only (out == nullptr) or write them to out.
__device__ int node_conflicts(const AggGraph& g, int i, int32_t* out) {
  const int p = g.prio[i];
  int c = 0;
  for (int e = g.rowptr[i]; e < g.rowptr[i + 1]; ++e) {
    const int j = g.col[e];
    if (j == i) continue;
    const bool sij = g.strong[e] != 0;
    if ((sij || g.strong[g.tslot[e]] != 0) && g.prio[j] < p) {
      if (out) out[c] = j;
      ++c;
    }
    if (!sij) continue;
    for (int e2 = g.rowptr[j]; e2 < g.rowptr[j + 1]; ++e2) {
      const int r = g.col[e2];
      if (r == i || r == j || g.strong[g.tslot[e2]] == 0 || g.prio[r] >= p) continue;
      if (out) out[c] = r;
      ++c;
    }
  }
  return c;
}

__global__ void conflict_counts_k(AggGraph g, int32_t* cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    cnt[i] = node_conflicts(g, i, nullptr);
}

// Writes the lists at their scanned offsets when they fit the capacity (else error 3).
__global__ void conflict_lists_k(AggGraph g, const int32_t* __restrict__ off, const int32_t* __restrict__ total,
                                 int64_t capacity, int32_t* lists, int32_t* err) {
  if ((int64_t)*total > capacity) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(err, 3);
    return;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    node_conflicts(g, i, lists + off[i]);
}

// Decides node i (pass 1) from its conflict list [k0, k1): kNotRoot as soon as one of them is a
// root, kRoot once all are decided "not a root"; -1 when the poll budget ran out or another
// thread reported an error. A poll reads the list from the first entry found undecided on (the
// ones before it are decided "not a root" and stay so); the list is read-only (cached), the
// decisions are relaxed loads at device scope, kPollBatch of them issued before any is tested
// (straight-line loads, the last entry repeated past the list's end), so a poll costs a few
// load latencies rather than one per entry.
constexpr int kPollBatch = 8;

__device__ int decide_node(const int32_t* __restrict__ lists, int k0, int k1, const int32_t* status, int64_t limit,
                           int64_t& polls, const int32_t* err) {
  for (;;) {
    int first = -1;
    for (int k = k0; k < k1; k += kPollBatch) {
      int32_t s[kPollBatch];
#pragma unroll
      for (int j = 0; j < kPollBatch; ++j) s[j] = ld_relaxed(status + __ldg(lists + min(k + j, k1 - 1)));
      bool root = false;
#pragma unroll
      for (int j = 0; j < kPollBatch; ++j) {
        root = root || s[j] == kRoot;
        if (first < 0 && k + j < k1 && s[j] == kUndecided) first = k + j;
      }
      if (root) return kNotRoot;
    }
    if (first < 0) return kRoot;
    if (++polls > limit) return -1;
    if ((polls & 63) == 0 && ld_relaxed(err) != 0) return -1;
    k0 = first;
    __nanosleep(64);
  }
}

__global__ void __launch_bounds__(kCoopThreads) aggregate_roots_k(AggGraph g, const int32_t* lists,
                                                                  const int32_t* off, int32_t* status, int64_t limit,
                                                                  int32_t* err) {
  if (ld_relaxed(err) != 0) return;
  const int T = gridDim.x * blockDim.x;
  int64_t polls = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += T) {
    const int i = g.rank_node[p];
    const int d = decide_node(lists, off[i], off[i + 1], status, limit, polls, err);
    if (d < 0) {
      atomicExch(err, 1);
      return;
    }
    st_relaxed(status + i, d);
  }
}

// ------------------------------------------------------------------ exclusive scan of int32 flags
// Three launches: tile sums, a one-block scan of the tile sums, the scan of every tile.
__device__ __forceinline__ int block_excl_scan(int v, int* sm, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < nw ? sm[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) sm[lane] = w;
  }
  __syncthreads();
  const int before = (warp > 0 ? sm[warp - 1] : 0) + x - v;
  if (total) *total = sm[nw - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kScanTile) tile_sums_k(int n, const int32_t* __restrict__ flag, int32_t* tsum) {
  __shared__ int sm[32];
  const int i = blockIdx.x * kScanTile + threadIdx.x;
  int tot = 0;
  block_excl_scan(i < n ? flag[i] : 0, sm, &tot);
  if (threadIdx.x == 0) tsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kScanTile) tile_offsets_k(int ntiles, int32_t* tsum, int32_t* total) {
  __shared__ int sm[32];
  int carry = 0;
  for (int b = 0; b < ntiles; b += kScanTile) {
    const int i = b + threadIdx.x;
    const int v = i < ntiles ? tsum[i] : 0;
    int tot = 0;
    const int ex = block_excl_scan(v, sm, &tot);
    if (i < ntiles) tsum[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kScanTile) tile_scan_k(int n, const int32_t* __restrict__ flag,
                                                         const int32_t* __restrict__ toff, int32_t* out) {
  __shared__ int sm[32];
  const int i = blockIdx.x * kScanTile + threadIdx.x;
  const int ex = block_excl_scan(i < n ? flag[i] : 0, sm, nullptr);
  if (i < n) out[i] = toff[blockIdx.x] + ex;
}

// ------------------------------------------------------------------ numbering and passes 2 and 3
// flag[p] = 1 where the node of priority p is a root
__global__ void root_flags_k(AggGraph g, const int32_t* __restrict__ status, int32_t* flag) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < g.n; p += gridDim.x * blockDim.x)
    flag[p] = status[g.rank_node[p]] == kRoot ? 1 : 0;
}

// Pass 1's aggregates: a root's number is its rank among the roots (rid, by priority); any other
// node takes the number of the root r with the node in S(r), if there is one; else -1.
__global__ void assign_pass1_k(AggGraph g, const int32_t* __restrict__ status, const int32_t* __restrict__ rid,
                               int32_t* agg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    int a = -1;
    if (status[i] == kRoot) {
      a = rid[g.prio[i]];
    } else {
      for (int e = g.rowptr[i]; e < g.rowptr[i + 1]; ++e) {
        const int r = g.col[e];
        if (r != i && g.strong[g.tslot[e]] && status[r] == kRoot) {
          a = rid[g.prio[r]];
          break;
        }
      }
    }
    agg[i] = a;
  }
}

// Pass 2 links: a node left over joins its lowest-priority strong neighbour that is aggregated
// when its turn comes - aggregated in pass 1, or left over with a lower priority (joined before
// it). link[i] = that neighbour, -1 when none (pass 3), i itself for nodes of pass 1.
__global__ void pass2_links_k(AggGraph g, const int32_t* __restrict__ agg1, int32_t* link) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    if (agg1[i] >= 0) {
      link[i] = i;
      continue;
    }
    const int pi = g.prio[i];
    int best = -1, bp = 0x7fffffff;
    for (int e = g.rowptr[i]; e < g.rowptr[i + 1]; ++e) {
      const int j = g.col[e];
      if (j == i || !g.strong[e]) continue;
      const int pj = g.prio[j];
      if ((agg1[j] >= 0 || pj < pi) && pj < bp) best = j, bp = pj;
    }
    link[i] = best;
  }
}

// Resolves the links (each step strictly lower in priority, so every chain ends at a node of
// pass 1 or at one without a link); flag[p] = 1 for the nodes of pass 3.
__global__ void pass2_resolve_k(AggGraph g, const int32_t* __restrict__ agg1, const int32_t* __restrict__ link,
                                int32_t* agg, int32_t* flag, int32_t* err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    int x = i, a = agg1[i];
    for (int step = 0; a < 0 && step <= g.n; ++step) {
      const int j = link[x];
      if (j < 0) break;
      x = j;
      a = agg1[x];
    }
    if (a < 0 && link[x] >= 0) atomicExch(err, 2);  // a chain longer than n: not possible
    agg[i] = a;
    flag[g.prio[i]] = a < 0 ? 1 : 0;
  }
}

// Pass 3: the nodes still without an aggregate, numbered after the others in priority order.
__global__ void pass3_k(AggGraph g, const int32_t* __restrict__ off, const int32_t* __restrict__ na1,
                        int32_t* agg) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
    if (agg[i] < 0) agg[i] = *na1 + off[g.prio[i]];
}

__global__ void aggregate_total_k(int32_t* info) { info[0] = info[2] + info[3]; }

__global__ void aggregate_sizes_k(int n, const int32_t* __restrict__ agg, int32_t* cnt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) atomicAdd(cnt + agg[i], 1);
}

// ------------------------------------------------------------------ P and W patterns, per row
// P = A T has, in row i, one entry per distinct aggregate among the columns of A's row i; W = A P
// one per distinct column among the P rows of those columns. One thread builds one row in
// local arrays (at most kMaxRowP distinct P columns and kMaxRowW distinct W columns a row, any
// number of A entries and W terms; a row with more raises *overflow and the caller builds the
// level with sorted keys instead). The term lists
// follow the order the row-owned rebuild kernels add terms in: P slot (i, J) lists the A
// entries of row i with aggregate J in stored order; W slot (i, c) lists the pairs (A entry e of
// row i, P entry f of row col[e]) with column c, e in stored order, then f.
constexpr int kMaxRowP = 64;
constexpr int kMaxRowW = 128;

// Inserts v into the ascending distinct list u[0..m); returns the new length (cap: no insert
// past it, *full set).
__device__ __forceinline__ int insert_distinct(int32_t* u, int m, int cap, int32_t v, bool& full) {
  int lo = 0, hi = m;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (u[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  if (lo < m && u[lo] == v) return m;
  if (m >= cap) {
    full = true;
    return m;
  }
  for (int k = m; k > lo; --k) u[k] = u[k - 1];
  u[lo] = v;
  return m + 1;
}

__device__ __forceinline__ int find_distinct(const int32_t* u, int m, int32_t v) {
  int lo = 0, hi = m;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (u[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// pass 0: pcnt[i] = distinct aggregates of row i. pass 1: p_idx, p_tptr (slot starts), p_tj.
__global__ void p_pattern_k(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ cl,
                            const int32_t* __restrict__ agg, int pass, int32_t* __restrict__ pcnt,
                            const int32_t* __restrict__ p_ptr, int64_t p_cap, int32_t* __restrict__ p_idx,
                            int32_t* __restrict__ p_tptr, int32_t* __restrict__ p_tj, int64_t nnz,
                            int32_t* __restrict__ overflow) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int e0 = rp[i], e1 = rp[i + 1];
    int32_t u[kMaxRowP];
    int m = 0;
    bool full = false;
    for (int e = e0; e < e1 && !full; ++e) m = insert_distinct(u, m, kMaxRowP, agg[cl[e]], full);
    if (full) {
      atomicExch(overflow, 1);
      if (pass == 0) pcnt[i] = 0;
      continue;
    }
    if (pass == 0) {
      pcnt[i] = m;
      continue;
    }
    const int64_t base = p_ptr[i];
    if (base + m > p_cap || p_ptr[i + 1] - base != m) {
      atomicExch(overflow, 2);
      continue;
    }
    int32_t cnt[kMaxRowP];
    for (int k = 0; k < m; ++k) cnt[k] = 0;
    for (int e = e0; e < e1; ++e) {
      const int r = find_distinct(u, m, agg[cl[e]]);
      if (r < m) ++cnt[r];
    }
    int acc = e0;
    for (int k = 0; k < m; ++k) {  // slot starts, then the running positions
      p_idx[base + k] = u[k];
      p_tptr[base + k] = acc;
      const int c = cnt[k];
      cnt[k] = acc;
      acc += c;
    }
    for (int e = e0; e < e1; ++e) {
      const int r = find_distinct(u, m, agg[cl[e]]);
      if (r >= m) continue;
      const int pos = cnt[r]++;
      if (pos >= 0 && pos < nnz) p_tj[pos] = e;
    }
    if (i == n - 1) p_tptr[base + m] = (int32_t)nnz;
  }
}

// pass 0: wcnt[i] = distinct W columns, tcnt[i] = W terms of row i. pass 1: w_idx, w_tptr,
// w_tj, w_te (row i's terms from t_ptr[i]).
__global__ void w_pattern_k(int n, const int32_t* __restrict__ rp, const int32_t* __restrict__ cl,
                            const int32_t* __restrict__ p_ptr, const int32_t* __restrict__ p_idx, int pass,
                            int32_t* __restrict__ wcnt, int32_t* __restrict__ tcnt, const int32_t* __restrict__ w_ptr,
                            const int32_t* __restrict__ t_ptr, int64_t w_cap, int64_t t_cap,
                            int32_t* __restrict__ w_idx, int32_t* __restrict__ w_tptr, int32_t* __restrict__ w_tj,
                            int32_t* __restrict__ w_te, int32_t* __restrict__ overflow) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int e0 = rp[i], e1 = rp[i + 1];
    int32_t u[kMaxRowW];
    int m = 0;
    int64_t terms = 0;
    bool full = false;
    for (int e = e0; e < e1 && !full; ++e) {
      const int j = cl[e];
      for (int f = p_ptr[j]; f < p_ptr[j + 1]; ++f) m = insert_distinct(u, m, kMaxRowW, p_idx[f], full);
      terms += p_ptr[j + 1] - p_ptr[j];
    }
    if (full || terms > INT32_MAX) {
      atomicExch(overflow, 1);
      if (pass == 0) wcnt[i] = tcnt[i] = 0;
      continue;
    }
    if (pass == 0) {
      wcnt[i] = m;
      tcnt[i] = (int32_t)terms;
      continue;
    }
    const int64_t base = w_ptr[i], tb = t_ptr[i];
    if (base + m > w_cap || w_ptr[i + 1] - base != m || tb + terms > t_cap || t_ptr[i + 1] - tb != terms) {
      atomicExch(overflow, 2);
      continue;
    }
    int32_t cnt[kMaxRowW];
    for (int k = 0; k < m; ++k) cnt[k] = 0;
    for (int e = e0; e < e1; ++e) {
      const int j = cl[e];
      for (int f = p_ptr[j]; f < p_ptr[j + 1]; ++f) {
        const int r = find_distinct(u, m, p_idx[f]);
        if (r < m) ++cnt[r];
      }
    }
    int64_t acc = tb;
    for (int k = 0; k < m; ++k) {
      w_idx[base + k] = u[k];
      w_tptr[base + k] = (int32_t)acc;
      const int c = cnt[k];
      cnt[k] = (int32_t)(acc - tb);
      acc += c;
    }
    for (int e = e0; e < e1; ++e) {
      const int j = cl[e];
      for (int f = p_ptr[j]; f < p_ptr[j + 1]; ++f) {
        const int r = find_distinct(u, m, p_idx[f]);
        if (r >= m) continue;
        const int64_t pos = tb + cnt[r]++;
        if (pos >= tb && pos < tb + terms) {
          w_tj[pos] = e;
          w_te[pos] = f;
        }
      }
    }
    if (i == n - 1) w_tptr[base + m] = (int32_t)(tb + terms);
  }
}

// ------------------------------------------------------------------ R = P^T and A_c = R W, per row
// R row I lists the fine rows i whose P row holds aggregate I, ascending, with the P entry of
// each (r_from_p). A_c row I has one entry per distinct column among the W rows of R row I's
// fine rows; its term list holds, per column, the pairs (R entry q, W entry s) in the order the
// row-owned Galerkin kernel adds them: q ascending, then s. Rows of at most kMaxRowR R entries
// and kMaxRowC distinct A_c columns; a longer row raises *overflow and the caller builds the
// level with sorted keys instead.
constexpr int kMaxRowR = 256;
constexpr int kMaxRowC = 128;

__global__ void r_count_k(int64_t p_nnz, const int32_t* __restrict__ p_idx, int na, int32_t* __restrict__ rcnt) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < p_nnz; f += (int64_t)gridDim.x * blockDim.x) {
    const int c = p_idx[f];
    if (c >= 0 && c < na) atomicAdd(rcnt + c, 1);
  }
}

// Places every fine row i at a free position of each R row its P row names (the order inside an
// R row is fixed afterwards by r_sort_k); cursor holds the R row starts on entry.
__global__ void r_fill_k(int n, const int32_t* __restrict__ p_ptr, const int32_t* __restrict__ p_idx, int na,
                         int32_t* __restrict__ cursor, int64_t p_nnz, int32_t* __restrict__ r_col) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int f = p_ptr[i]; f < p_ptr[i + 1]; ++f) {
      const int c = p_idx[f];
      if (c < 0 || c >= na) continue;
      const int pos = atomicAdd(cursor + c, 1);
      if (pos >= 0 && pos < p_nnz) r_col[pos] = i;
    }
  }
}

// Sorts each R row's fine rows ascending (distinct: a P row names an aggregate once) and finds
// the P entry of each by a binary search of the fine row's ascending P columns.
__global__ void r_sort_k(int na, const int32_t* __restrict__ r_rowptr, const int32_t* __restrict__ p_ptr,
                         const int32_t* __restrict__ p_idx, int32_t* __restrict__ r_col, int32_t* __restrict__ r_from_p,
                         int32_t* __restrict__ overflow) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
    const int q0 = r_rowptr[I], len = r_rowptr[I + 1] - q0;
    if (len > kMaxRowR) {
      atomicExch(overflow, 1);
      continue;
    }
    int32_t v[kMaxRowR];
    for (int k = 0; k < len; ++k) {
      const int32_t x = r_col[q0 + k];
      int j = k;
      while (j > 0 && v[j - 1] > x) {
        v[j] = v[j - 1];
        --j;
      }
      v[j] = x;
    }
    for (int k = 0; k < len; ++k) {
      const int i = v[k], f0 = p_ptr[i];
      r_col[q0 + k] = i;
      r_from_p[q0 + k] = f0 + find_distinct(p_idx + f0, p_ptr[i + 1] - f0, I);
    }
  }
}

// pass 0: ccnt[I] = distinct A_c columns, tcnt[I] = A_c terms of row I. pass 1: c_idx, c_diag
// (the slot of column I in row I, or where it would sit), c_tptr, c_te, c_ts (row I's terms from
// t_ptr[I]).
__global__ void c_pattern_k(int na, const int32_t* __restrict__ r_rowptr, const int32_t* __restrict__ r_col,
                            const int32_t* __restrict__ w_ptr, const int32_t* __restrict__ w_idx, int pass,
                            int32_t* __restrict__ ccnt, int32_t* __restrict__ tcnt, const int32_t* __restrict__ c_ptr,
                            const int32_t* __restrict__ t_ptr, int64_t c_cap, int64_t t_cap,
                            int32_t* __restrict__ c_idx, int32_t* __restrict__ c_diag, int32_t* __restrict__ c_tptr,
                            int32_t* __restrict__ c_te, int32_t* __restrict__ c_ts, int32_t* __restrict__ overflow) {
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < na; I += gridDim.x * blockDim.x) {
    const int q0 = r_rowptr[I], q1 = r_rowptr[I + 1];
    int32_t u[kMaxRowC];
    int m = 0;
    int64_t terms = 0;
    bool full = false;
    for (int q = q0; q < q1 && !full; ++q) {
      const int i = r_col[q];
      for (int s = w_ptr[i]; s < w_ptr[i + 1]; ++s) m = insert_distinct(u, m, kMaxRowC, w_idx[s], full);
      terms += w_ptr[i + 1] - w_ptr[i];
    }
    if (full || terms > INT32_MAX) {
      atomicExch(overflow, 1);
      if (pass == 0) ccnt[I] = tcnt[I] = 0;
      continue;
    }
    if (pass == 0) {
      ccnt[I] = m;
      tcnt[I] = (int32_t)terms;
      continue;
    }
    const int64_t base = c_ptr[I], tb = t_ptr[I];
    if (base + m > c_cap || c_ptr[I + 1] - base != m || tb + terms > t_cap || t_ptr[I + 1] - tb != terms) {
      atomicExch(overflow, 2);
      continue;
    }
    int32_t cnt[kMaxRowC];
    for (int k = 0; k < m; ++k) cnt[k] = 0;
    for (int q = q0; q < q1; ++q) {
      const int i = r_col[q];
      for (int s = w_ptr[i]; s < w_ptr[i + 1]; ++s) {
        const int r = find_distinct(u, m, w_idx[s]);
        if (r < m) ++cnt[r];
      }
    }
    int64_t acc = tb;
    for (int k = 0; k < m; ++k) {
      c_idx[base + k] = u[k];
      c_tptr[base + k] = (int32_t)acc;
      const int c = cnt[k];
      cnt[k] = (int32_t)(acc - tb);
      acc += c;
    }
    c_diag[I] = (int32_t)(base + find_distinct(u, m, I));
    for (int q = q0; q < q1; ++q) {
      const int i = r_col[q];
      for (int s = w_ptr[i]; s < w_ptr[i + 1]; ++s) {
        const int r = find_distinct(u, m, w_idx[s]);
        if (r >= m) continue;
        const int64_t pos = tb + cnt[r]++;
        if (pos >= tb && pos < tb + terms) {
          c_te[pos] = q;
          c_ts[pos] = s;
        }
      }
    }
    if (I == na - 1) c_tptr[base + m] = (int32_t)(tb + terms);
  }
}

// ------------------------------------------------------------------ the same patterns, one warp per row
// For levels of at most kWarpRowCols columns (the coarse levels, whose rows are dense and whose
// terms one thread would walk one after another): a warp builds one row with a counter per
// column in shared memory. The row's terms are a two-level walk - outer entries o of the row,
// then the inner range of each - each term landing on a column. The warp counts the terms per
// column (lanes take outer entries in turn), turns the counts into the sorted distinct columns
// and their slot starts by one sweep over the columns, then places the terms 32 at a time in
// the walk's order: a lane finds its outer entry by a binary search over the 32 outer entries'
// running term counts, lanes landing on the same column take consecutive positions in lane
// order (__match_any_sync), so every slot lists its terms in the walk's order - the order of
// the thread-per-row kernels above, bit for bit.
constexpr int kWarpRowCols = 2048;
constexpr int kPatternWarps = 4;
int g_warp_cols = kWarpRowCols;  // levels of at most this many columns are built one warp per row

struct PTerms {  // P = A T: the A entries e of row i, each one term on column agg[col[e]]
  const int32_t* rp;
  const int32_t* cl;
  const int32_t* agg;
  __device__ int o0(int r) const { return rp[r]; }
  __device__ int o1(int r) const { return rp[r + 1]; }
  __device__ int i0(int o) const { return o; }
  __device__ int i1(int o) const { return o + 1; }
  __device__ int col(int x) const { return agg[cl[x]]; }
};
struct WTerms {  // W = A P: A entry e of row i, then P entry f of row col[e], on column p_idx[f]
  const int32_t* rp;
  const int32_t* cl;
  const int32_t* p_ptr;
  const int32_t* p_idx;
  __device__ int o0(int r) const { return rp[r]; }
  __device__ int o1(int r) const { return rp[r + 1]; }
  __device__ int i0(int o) const { return p_ptr[cl[o]]; }
  __device__ int i1(int o) const { return p_ptr[cl[o] + 1]; }
  __device__ int col(int x) const { return p_idx[x]; }
};
struct CTerms {  // A_c = R W: R entry q of row I, then W entry s of row r_col[q], on column w_idx[s]
  const int32_t* r_rowptr;
  const int32_t* r_col;
  const int32_t* w_ptr;
  const int32_t* w_idx;
  __device__ int o0(int r) const { return r_rowptr[r]; }
  __device__ int o1(int r) const { return r_rowptr[r + 1]; }
  __device__ int i0(int o) const { return w_ptr[r_col[o]]; }
  __device__ int i1(int o) const { return w_ptr[r_col[o] + 1]; }
  __device__ int col(int x) const { return w_idx[x]; }
};

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// pass 0: cnt_out[r] = distinct columns, tcnt[r] (if not null) = terms of row r. pass 1: idx (the distinct
// columns, ascending, from c_ptr[r]), tptr (each slot's first term, from t_ptr[r]; tptr[c_nnz]
// written by the last row), pay_o/pay_i (each term's outer and inner entry; pay_i may be null),
// diag (if not null: the slot of column r, or where it would sit). Terms whose columns fall
// outside [0, ncols) are not counted and raise *overflow (1); offsets that disagree with the
// counts raise 2.
template <class T>
__global__ void __launch_bounds__(kPatternWarps * 32)
    warp_pattern_k(T t, int nrows, int ncols, int pass, int32_t* __restrict__ cnt_out, int32_t* __restrict__ tcnt,
                   const int32_t* __restrict__ c_ptr, const int32_t* __restrict__ t_ptr, int64_t c_cap, int64_t t_cap,
                   int32_t* __restrict__ idx, int32_t* __restrict__ tptr, int32_t* __restrict__ pay_o,
                   int32_t* __restrict__ pay_i, int32_t* __restrict__ diag, int32_t* __restrict__ overflow) {
  __shared__ int32_t cnt_all[kPatternWarps][kWarpRowCols];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
  int32_t* cnt = cnt_all[warp];
  for (int c = lane; c < ncols; c += 32) cnt[c] = 0;
  __syncwarp();
  for (int r = blockIdx.x * kPatternWarps + warp; r < nrows; r += gridDim.x * kPatternWarps) {
    const int o0 = t.o0(r), o1 = t.o1(r);
    int fresh = 0, bad = 0;
    int64_t my_terms = 0;
    for (int o = o0 + lane; o < o1; o += 32) {
      const int x1 = t.i1(o);
      for (int x = t.i0(o); x < x1; ++x) {
        const int c = t.col(x);
        if (c < 0 || c >= ncols) {
          bad = 1;
          continue;
        }
        if (atomicAdd(cnt + c, 1) == 0) ++fresh;
      }
      my_terms += x1 - t.i0(o);
    }
    int m = fresh;
    int64_t terms = my_terms;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
      m += __shfl_xor_sync(0xffffffffu, m, s);
      terms += __shfl_xor_sync(0xffffffffu, terms, s);
    }
    const bool fail = __any_sync(0xffffffffu, bad) || terms > INT32_MAX;
    __syncwarp();
    if (fail) {
      if (lane == 0) {
        atomicExch(overflow, 1);
        if (pass == 0) {
          cnt_out[r] = 0;
          if (tcnt != nullptr) tcnt[r] = 0;
        }
      }
    } else if (pass == 0) {
      if (lane == 0) {
        cnt_out[r] = m;
        if (tcnt != nullptr) tcnt[r] = (int32_t)terms;
      }
    } else {
      const int64_t base = c_ptr[r], tb = t_ptr[r];
      const bool ok = base + m <= c_cap && c_ptr[r + 1] - base == m && tb + terms <= t_cap &&
                      t_ptr[r + 1] - tb == terms;
      if (!ok) {
        if (lane == 0) atomicExch(overflow, 2);
      } else {
        // distinct columns and slot starts; each counter becomes its slot's next position
        int run_m = 0;
        int64_t run_t = tb;
        for (int c0 = 0; c0 < ncols; c0 += 32) {
          const int c = c0 + lane;
          const int v = c < ncols ? cnt[c] : 0;
          const unsigned hit = __ballot_sync(0xffffffffu, v > 0);
          const int incl = warp_incl_scan(v, lane);
          if (v > 0) {
            const int rank = run_m + __popc(hit & below);
            idx[base + rank] = c;
            tptr[base + rank] = (int32_t)(run_t + incl - v);
            cnt[c] = (int32_t)(run_t + incl - v);
          }
          if (diag != nullptr && lane == 0 && r >= c0 && r < c0 + 32)
            diag[r] = (int32_t)(base + run_m + __popc(hit & ((1u << (r - c0)) - 1u)));
          run_m += __popc(hit);
          run_t += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (diag != nullptr && lane == 0 && r >= ncols) diag[r] = (int32_t)(base + m);
        if (r == nrows - 1 && lane == 0) tptr[base + m] = (int32_t)(tb + terms);
        __syncwarp();
        // the terms in the walk's order, 32 at a time
        for (int ob = o0; ob < o1; ob += 32) {
          const int o = ob + lane;
          const int x0 = o < o1 ? t.i0(o) : 0;
          const int len = o < o1 ? t.i1(o) - x0 : 0;
          const int incl = warp_incl_scan(len, lane);
          const int total = __shfl_sync(0xffffffffu, incl, 31);
          for (int tt0 = 0; tt0 < total; tt0 += 32) {
            const int tt = tt0 + lane;
            int lo = 0, hi = 31;  // the first outer entry whose running count exceeds tt
#pragma unroll
            for (int step = 0; step < 5; ++step) {
              const int mid = (lo + hi) >> 1;
              if (__shfl_sync(0xffffffffu, incl, mid) > tt) hi = mid;
              else lo = mid + 1;
            }
            const int start = __shfl_sync(0xffffffffu, incl - len, lo);
            const int xk = __shfl_sync(0xffffffffu, x0, lo);
            const bool act = tt < total;
            const int x = xk + (tt - start);
            const int c = act ? t.col(x) : -1 - lane;
            const unsigned peers = __match_any_sync(0xffffffffu, c);
            const int rank = __popc(peers & below);
            const int pos = act ? cnt[c] + rank : 0;
            __syncwarp();
            if (act && rank == 0) cnt[c] += __popc(peers);
            __syncwarp();
            if (act && pos >= tb && pos < tb + terms) {
              pay_o[pos] = ob + lo;
              if (pay_i != nullptr) pay_i[pos] = x;
            }
          }
        }
      }
    }
    __syncwarp();
    for (int c = lane; c < ncols; c += 32) cnt[c] = 0;
    __syncwarp();
  }
}

}  // namespace b2s

using namespace b2s;

namespace {
int coop_grid(const void* kernel, int threads, int* grid) {
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return B2S_ERR_DEVICE;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return B2S_ERR_DEVICE;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0) != cudaSuccess || per <= 0)
    return B2S_ERR_DEVICE;
  *grid = sms * per;
  return B2S_OK;
}

int scan_flags(int n, const int32_t* flag, int32_t* out, int32_t* tsum, int32_t* total, cudaStream_t st) {
  const int tiles = (int)cdiv(n, kScanTile);
  tile_sums_k<<<tiles, kScanTile, 0, st>>>(n, flag, tsum);
  tile_offsets_k<<<1, kScanTile, 0, st>>>(tiles, tsum, total);
  tile_scan_k<<<tiles, kScanTile, 0, st>>>(n, flag, tsum, out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}
}  // namespace

extern "C" {

int b2s_amg_strength_d(int32_t n, const int32_t* rowptr, const int32_t* col, const double* val,
                       const int32_t* diag_slot, double theta, uint8_t* strong, b2s_stream_t s) {
  if (n < 0 || (n > 0 && (!rowptr || !col || !val || !diag_slot || !strong))) return B2S_ERR_ARG;
  if (n == 0) return B2S_OK;
  strength_k<<<grid_for(n), kThreads, 0, (cudaStream_t)s>>>(n, rowptr, col, val, diag_slot, theta, strong);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_csr_transpose_slots_d(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t sorted, int32_t* tslot,
                              int32_t* missing, b2s_stream_t s) {
  if (n < 0 || !missing || (n > 0 && (!rowptr || !col || !tslot))) return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (cudaMemsetAsync(missing, 0, sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  if (n == 0) return B2S_OK;
  transpose_slots_k<<<grid_for(n), kThreads, 0, st>>>(n, rowptr, col, sorted != 0, tslot, missing);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int64_t b2s_amg_aggregate_workspace_bytes(int32_t n, int64_t capacity) {
  if (n < 0 || capacity < 0) return -1;
  const int64_t tiles = cdiv(n > 0 ? n : 1, kScanTile);
  return (int64_t)sizeof(int32_t) * (5 * (int64_t)n + tiles + 9 + capacity);
}

int b2s_amg_aggregate_d(int32_t n, const int32_t* rowptr, const int32_t* col, const uint8_t* strong,
                        const int32_t* tslot, const int32_t* prio, const int32_t* rank_node, int32_t* agg,
                        int32_t* counts, int32_t* info, void* work, int64_t work_bytes, b2s_stream_t s) {
  if (n < 1 || !rowptr || !col || !strong || !tslot || !prio || !rank_node || !agg || !counts || !info || !work)
    return B2S_ERR_ARG;
  const int64_t tiles = cdiv(n, kScanTile);
  const int64_t fixed = (int64_t)sizeof(int32_t) * (5 * (int64_t)n + tiles + 9);
  if (work_bytes < fixed) return B2S_ERR_WORKSPACE;
  int64_t capacity = (work_bytes - fixed) / (int64_t)sizeof(int32_t);
  cudaStream_t st = (cudaStream_t)s;
  int32_t* status = (int32_t*)work;
  int32_t* flag = status + n;
  int32_t* ids = flag + n;
  int32_t* link = ids + n;
  int32_t* off = link + n;  // [n + 1] offsets of the conflict lists
  int32_t* tsum = off + n + 1;
  int32_t* lists = tsum + tiles + 8;
  // info: [0] aggregates, [1] error (1: poll budget exhausted, 2: broken link chain, 3: conflict
  //       lists above the work space's capacity), [2] aggregates of passes 1-2, [3] nodes of pass 3
  if (cudaMemsetAsync(info, 0, 4 * sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  if (cudaMemsetAsync(status, 0, (size_t)n * sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  AggGraph g{n, rowptr, col, strong, tslot, prio, rank_node};
  int32_t* err = info + 1;
  int rc;
  const unsigned gn = grid_for(n);
  conflict_counts_k<<<gn, kThreads, 0, st>>>(g, flag);
  B2S_LAUNCH_CHECK();
  if ((rc = scan_flags(n, flag, off, tsum, off + n, st)) != B2S_OK) return rc;
  conflict_lists_k<<<gn, kThreads, 0, st>>>(g, off, off + n, capacity, lists, err);
  B2S_LAUNCH_CHECK();
  int grid = 0;
  if ((rc = coop_grid((const void*)aggregate_roots_k, kCoopThreads, &grid)) != B2S_OK) return rc;
  int64_t limit = 1 << 22;  // polls of one thread, ~0.3 s of waiting: far above any chain
  const int32_t* lists_c = lists;
  const int32_t* off_c = off;
  void* args[] = {&g, &lists_c, &off_c, &status, &limit, &err};
  if (cudaLaunchCooperativeKernel((const void*)aggregate_roots_k, grid, kCoopThreads, args, 0, st) != cudaSuccess)
    return B2S_ERR_LAUNCH;
  root_flags_k<<<gn, kThreads, 0, st>>>(g, status, flag);
  B2S_LAUNCH_CHECK();
  if ((rc = scan_flags(n, flag, ids, tsum, info + 2, st)) != B2S_OK) return rc;
  assign_pass1_k<<<gn, kThreads, 0, st>>>(g, status, ids, agg);
  pass2_links_k<<<gn, kThreads, 0, st>>>(g, agg, link);
  // agg holds pass 1's numbers; resolve into status (free now), then number pass 3 into agg
  pass2_resolve_k<<<gn, kThreads, 0, st>>>(g, agg, link, status, flag, err);
  B2S_LAUNCH_CHECK();
  if ((rc = scan_flags(n, flag, ids, tsum, info + 3, st)) != B2S_OK) return rc;
  if (cudaMemcpyAsync(agg, status, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return B2S_ERR_LAUNCH;
  pass3_k<<<gn, kThreads, 0, st>>>(g, ids, info + 2, agg);
  aggregate_total_k<<<1, 1, 0, st>>>(info);
  B2S_LAUNCH_CHECK();
  if (cudaMemsetAsync(counts, 0, (size_t)n * sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  aggregate_sizes_k<<<gn, kThreads, 0, st>>>(n, agg, counts);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

/* P and W patterns with their term lists (the order of the row-owned rebuild kernels; see
 * p_pattern_k / w_pattern_k): one warp per row where P and W have at most g_warp_cols columns
 * (ncols: the level's aggregates), else one thread per row. Each builder has two passes: pass 0
 * writes per-row counts (pcnt; wcnt and tcnt), the caller scans them into p_ptr (w_ptr, t_ptr)
 * and allocates; pass 1 fills. *overflow (device int, not cleared here): 1 where a row exceeds
 * the per-thread capacity (64 distinct P columns, 128 distinct W columns), 2 where the offsets
 * disagree with the counts. */
int b2s_amg_p_pattern_d(int32_t n, int32_t ncols, const int32_t* rp, const int32_t* cl, const int32_t* agg,
                        int32_t pass, int32_t* pcnt, const int32_t* p_ptr, int64_t p_cap, int32_t* p_idx,
                        int32_t* p_tptr, int32_t* p_tj, int64_t nnz, int32_t* overflow, b2s_stream_t s) {
  if (n < 1 || ncols < 1 || !rp || !cl || !agg || !overflow || (pass == 0 && !pcnt) ||
      (pass == 1 && (!p_ptr || !p_idx || !p_tptr || !p_tj)) || (pass != 0 && pass != 1))
    return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (ncols <= g_warp_cols) {
    warp_pattern_k<PTerms><<<grid_for((int64_t)n * 32, kPatternWarps * 32), kPatternWarps * 32, 0, st>>>(
        PTerms{rp, cl, agg}, n, ncols, pass, pcnt, nullptr, p_ptr, rp, p_cap, nnz, p_idx, p_tptr, p_tj, nullptr,
        nullptr, overflow);
  } else {
    p_pattern_k<<<grid_for(n, 128), 128, 0, st>>>(n, rp, cl, agg, pass, pcnt, p_ptr, p_cap, p_idx, p_tptr, p_tj, nnz,
                                                  overflow);
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_amg_w_pattern_d(int32_t n, int32_t ncols, const int32_t* rp, const int32_t* cl, const int32_t* p_ptr,
                        const int32_t* p_idx, int32_t pass, int32_t* wcnt, int32_t* tcnt, const int32_t* w_ptr,
                        const int32_t* t_ptr, int64_t w_cap, int64_t t_cap, int32_t* w_idx, int32_t* w_tptr,
                        int32_t* w_tj, int32_t* w_te, int32_t* overflow, b2s_stream_t s) {
  if (n < 1 || ncols < 1 || !rp || !cl || !p_ptr || !p_idx || !overflow || (pass == 0 && (!wcnt || !tcnt)) ||
      (pass == 1 && (!w_ptr || !t_ptr || !w_idx || !w_tptr || !w_tj || !w_te)) || (pass != 0 && pass != 1))
    return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (ncols <= g_warp_cols) {
    warp_pattern_k<WTerms><<<grid_for((int64_t)n * 32, kPatternWarps * 32), kPatternWarps * 32, 0, st>>>(
        WTerms{rp, cl, p_ptr, p_idx}, n, ncols, pass, wcnt, tcnt, w_ptr, t_ptr, w_cap, t_cap, w_idx, w_tptr, w_tj,
        w_te, nullptr, overflow);
  } else {
    w_pattern_k<<<grid_for(n, 128), 128, 0, st>>>(n, rp, cl, p_ptr, p_idx, pass, wcnt, tcnt, w_ptr, t_ptr, w_cap,
                                                  t_cap, w_idx, w_tptr, w_tj, w_te, overflow);
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

/* R = P^T of a level with n fine rows and na aggregates, from P's pattern (p_ptr [n + 1], p_idx
 * [p_nnz], each row's columns ascending): r_rowptr [na + 1], r_col [p_nnz] (fine rows,
 * ascending in each R row) and r_from_p [p_nnz] (the P entry of each R entry). Needs no host
 * synchronisation (R has p_nnz entries). *overflow (device int, not cleared here): 1 where an R
 * row holds more than 256 entries (that row is left unsorted). */
int64_t b2s_amg_r_workspace_bytes(int32_t na) {
  if (na < 0) return -1;
  const int64_t m = na > 0 ? na : 1;
  return (int64_t)sizeof(int32_t) * (m + cdiv(m, kScanTile) + 8);
}

int b2s_amg_r_pattern_d(int32_t n, int32_t na, const int32_t* p_ptr, const int32_t* p_idx, int64_t p_nnz,
                        int32_t* r_rowptr, int32_t* r_col, int32_t* r_from_p, void* work, int64_t work_bytes,
                        int32_t* overflow, b2s_stream_t s) {
  if (n < 1 || na < 1 || p_nnz < 0 || p_nnz > INT32_MAX || !p_ptr || !p_idx || !r_rowptr || !r_col || !r_from_p ||
      !work || !overflow)
    return B2S_ERR_ARG;
  if (work_bytes < b2s_amg_r_workspace_bytes(na)) return B2S_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)s;
  int32_t* cnt = (int32_t*)work;  // counts, then the running positions
  int32_t* tsum = cnt + na;
  if (cudaMemsetAsync(cnt, 0, (size_t)na * sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  if (p_nnz > 0) r_count_k<<<grid_for(p_nnz), kThreads, 0, st>>>(p_nnz, p_idx, na, cnt);
  B2S_LAUNCH_CHECK();
  int rc;
  if ((rc = scan_flags(na, cnt, r_rowptr, tsum, r_rowptr + na, st)) != B2S_OK) return rc;
  if (cudaMemcpyAsync(cnt, r_rowptr, (size_t)na * sizeof(int32_t), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return B2S_ERR_LAUNCH;
  r_fill_k<<<grid_for(n), kThreads, 0, st>>>(n, p_ptr, p_idx, na, cnt, p_nnz, r_col);
  r_sort_k<<<grid_for(na, 128), 128, 0, st>>>(na, r_rowptr, p_ptr, p_idx, r_col, r_from_p, overflow);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

/* Pattern and term lists of A_c = R W (the order of the row-owned Galerkin kernel; see
 * c_pattern_k), one warp per coarse row where na <= g_warp_cols, else one thread per row, in
 * two passes like the P and W builders: pass 0 writes ccnt and tcnt, the caller scans them into
 * c_ptr and t_ptr and allocates; pass 1 writes c_idx, c_diag [na], c_tptr [c_nnz + 1], c_te and
 * c_ts. *overflow: 1 where a row has more than 128 distinct columns (one thread per row), 2 where
 * the offsets disagree with the counts. */
int b2s_amg_c_pattern_d(int32_t na, const int32_t* r_rowptr, const int32_t* r_col, const int32_t* w_ptr,
                        const int32_t* w_idx, int32_t pass, int32_t* ccnt, int32_t* tcnt, const int32_t* c_ptr,
                        const int32_t* t_ptr, int64_t c_cap, int64_t t_cap, int32_t* c_idx, int32_t* c_diag,
                        int32_t* c_tptr, int32_t* c_te, int32_t* c_ts, int32_t* overflow, b2s_stream_t s) {
  if (na < 1 || !r_rowptr || !r_col || !w_ptr || !w_idx || !overflow || (pass == 0 && (!ccnt || !tcnt)) ||
      (pass == 1 && (!c_ptr || !t_ptr || !c_idx || !c_diag || !c_tptr || !c_te || !c_ts)) ||
      (pass != 0 && pass != 1))
    return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (na <= g_warp_cols) {
    warp_pattern_k<CTerms><<<grid_for((int64_t)na * 32, kPatternWarps * 32), kPatternWarps * 32, 0, st>>>(
        CTerms{r_rowptr, r_col, w_ptr, w_idx}, na, na, pass, ccnt, tcnt, c_ptr, t_ptr, c_cap, t_cap, c_idx, c_tptr,
        c_te, c_ts, c_diag, overflow);
  } else {
    c_pattern_k<<<grid_for(na, 128), 128, 0, st>>>(na, r_rowptr, r_col, w_ptr, w_idx, pass, ccnt, tcnt, c_ptr, t_ptr,
                                                   c_cap, t_cap, c_idx, c_diag, c_tptr, c_te, c_ts, overflow);
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

/* The largest column count whose pattern builders run one warp per row (default and maximum
 * kWarpRowCols; 0: one thread per row always); ncols < 0 only queries. Returns the previous
 * value. Process-wide and not synchronised: set it before the builders run. */
int b2s_amg_pattern_warp_cols(int32_t ncols) {
  const int prev = g_warp_cols;
  if (ncols >= 0) g_warp_cols = ncols < kWarpRowCols ? ncols : kWarpRowCols;
  return prev;
}

/* Exclusive scan of n int32 counts into out[0..n] (out[n] the total), for the pattern builders. */
int64_t b2s_scan_workspace_bytes(int32_t n) {
  if (n < 0) return -1;
  return (int64_t)sizeof(int32_t) * (cdiv(n > 0 ? n : 1, kScanTile) + 8);
}

int b2s_scan_counts_d(int32_t n, const int32_t* counts, int32_t* out, void* work, int64_t work_bytes, b2s_stream_t s) {
  if (n < 1 || !counts || !out || !work) return B2S_ERR_ARG;
  if (work_bytes < b2s_scan_workspace_bytes(n)) return B2S_ERR_WORKSPACE;
  return scan_flags(n, counts, out, (int32_t*)work, out + n, (cudaStream_t)s);
}

}  // extern "C"
