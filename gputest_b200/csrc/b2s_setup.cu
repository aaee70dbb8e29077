// Device set-up of the finite-volume data of an unstructured mesh: face centres and area
// vectors, cell volumes and centroids (flowtrace/mesh/unstructured.py:171-261), the face and
// cell quantities of flowtrace/unstructured/fvmesh.py:61-230 (d, w, alpha, T, least-squares
// matrices and their inverses, boundary normals), all in the reference's numbering and with
// the reference's operation order, so that the results equal the host set-up's bit for bit
// (the least-squares inverses excepted: LU with partial pivoting here, LAPACK on the host).
//
// The reference accumulates per-cell sums with np.bincount, which adds a cell's terms in
// increasing face order, one family of faces after another (owned faces, then neighbour
// faces, then boundary faces, each summed on its own before the families are added). The
// cell-centric kernels below walk a cell's face lists in that order: own[] holds the faces a
// cell owns (interior and boundary, increasing index), nei[] the interior faces whose
// neighbour it is. Arrays of points and vectors are row-major [n][dim], as in NumPy.
#include <vector>

#include "b2s_common.cuh"

namespace b2s {

#define B2S_HD __host__ __device__ __forceinline__

// The per-row dot product of np.einsum("fd,fd->f", a, b) as NumPy evaluates it: a0 b0 + a1 b1
// in 2-D, (a0 b0 + a2 b2) + a1 b1 in 3-D (its two-lane accumulation; checked against NumPy).
template <int D>
B2S_HD double edot(const double* a, const double* b) {
  if (D == 2) return a[0] * b[0] + a[1] * b[1];
  return (a[0] * b[0] + a[2] * b[2]) + a[1] * b[1];
}

// NumPy's sum of a short contiguous row (pairwise summation: sequential below 9 terms, eight
// interleaved partial sums above).
B2S_HD double numpy_row_sum(const double* a, int n) {
  if (n < 8) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i];
    return s;
  }
  double r[8];
  for (int j = 0; j < 8; ++j) r[j] = a[j];
  int i = 8;
  for (; i + 8 <= n; i += 8)
    for (int j = 0; j < 8; ++j) r[j] += a[i + j];
  double s = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
  for (; i < n; ++i) s += a[i];
  return s;
}

constexpr int kMaxFaceNodes = 32;

// The geometry of one face, one cell, ... as functions of the item index, shared by the device
// kernels (one thread per item) and the host loop of b2s_host_geometry.

// Face centre and area vector of face f (unstructured.py:171-212). 2-D: the segment midpoint
// and S = (e_y, -e_x). 3-D: the k-node face fanned into triangles about the node mean, the
// centre the triangle centroids weighted by their areas projected on S. False when the face's
// node count is not allowed (2-D: 2; 3-D: 3..32).
template <int D>
B2S_HD bool face_geometry(int64_t f, const double* X, const int32_t* fptr, const int32_t* fnodes, double* fc,
                          double* S) {
  const int p0 = fptr[f], k = fptr[f + 1] - p0;
  if (D == 2) {
    if (k != 2) return false;
    const double* a = X + 2 * (int64_t)fnodes[p0];
    const double* b = X + 2 * (int64_t)fnodes[p0 + 1];
    fc[2 * f] = 0.5 * (a[0] + b[0]);
    fc[2 * f + 1] = 0.5 * (a[1] + b[1]);
    const double ex = b[0] - a[0], ey = b[1] - a[1];
    S[2 * f] = ey;
    S[2 * f + 1] = -ex;
    return true;
  }
  if (k < 3 || k > kMaxFaceNodes) return false;
  double mean[3];
  for (int j = 0; j < k; ++j) {
    const double* p = X + 3 * (int64_t)fnodes[p0 + j];
    for (int c = 0; c < 3; ++c) mean[c] = j ? mean[c] + p[c] : p[c];
  }
  for (int c = 0; c < 3; ++c) mean[c] /= (double)k;
  double tri[kMaxFaceNodes][3], Sk[3];
  for (int j = 0; j < k; ++j) {
    const double* p = X + 3 * (int64_t)fnodes[p0 + j];
    const double* q = X + 3 * (int64_t)fnodes[p0 + (j + 1) % k];
    const double a0 = p[0] - mean[0], a1 = p[1] - mean[1], a2 = p[2] - mean[2];
    const double b0 = q[0] - mean[0], b1 = q[1] - mean[1], b2 = q[2] - mean[2];
    tri[j][0] = 0.5 * (a1 * b2 - a2 * b1);
    tri[j][1] = 0.5 * (a2 * b0 - a0 * b2);
    tri[j][2] = 0.5 * (a0 * b1 - a1 * b0);
    for (int c = 0; c < 3; ++c) Sk[c] = j ? Sk[c] + tri[j][c] : tri[j][c];
  }
  const double den = fmax(sqrt((Sk[0] * Sk[0] + Sk[1] * Sk[1]) + Sk[2] * Sk[2]), 1e-300);
  const double u[3] = {Sk[0] / den, Sk[1] / den, Sk[2] / den};
  double wt[kMaxFaceNodes], acc[3];
  for (int j = 0; j < k; ++j) {
    const double* p = X + 3 * (int64_t)fnodes[p0 + j];
    const double* q = X + 3 * (int64_t)fnodes[p0 + (j + 1) % k];
    wt[j] = edot<3>(tri[j], u);
    for (int c = 0; c < 3; ++c) {
      const double t = wt[j] * (((mean[c] + p[c]) + q[c]) / 3.0);
      acc[c] = j ? acc[c] + t : t;
    }
  }
  double wsum = numpy_row_sum(wt, k);
  if (!(fabs(wsum) > 0.0)) wsum = 1.0;
  for (int c = 0; c < 3; ++c) {
    fc[3 * f + c] = acc[c] / wsum;
    S[3 * f + c] = Sk[c];
  }
  return true;
}

// Approximate centre of cell c: the mean of its face centres (owned faces, then neighbour faces).
template <int D>
B2S_HD void centre_estimate(int64_t c, const int32_t* own_ptr, const int32_t* own, const int32_t* nei_ptr,
                            const int32_t* nei, const double* fc, double* ca) {
  double so[D], sn[D];
  for (int a = 0; a < D; ++a) so[a] = sn[a] = 0.0;
  for (int q = own_ptr[c]; q < own_ptr[c + 1]; ++q)
    for (int a = 0; a < D; ++a) so[a] += fc[D * (int64_t)own[q] + a];
  for (int q = nei_ptr[c]; q < nei_ptr[c + 1]; ++q)
    for (int a = 0; a < D; ++a) sn[a] += fc[D * (int64_t)nei[q] + a];
  const int cnt = (own_ptr[c + 1] - own_ptr[c]) + (nei_ptr[c + 1] - nei_ptr[c]);
  const double den = (double)(cnt > 1 ? cnt : 1);
  for (int a = 0; a < D; ++a) ca[D * c + a] = (so[a] + sn[a]) / den;
}

// Orientation repair of face f: S must point from the owner towards the neighbour (towards the
// face, on the boundary). True when S was turned.
template <int D>
B2S_HD bool orient(int64_t f, const int32_t* owner, const int32_t* neighbour, const double* fc, const double* ca,
                   double* S) {
  const int o = owner[f], n = neighbour[f];
  double ref[D];
  for (int a = 0; a < D; ++a)
    ref[a] = n >= 0 ? ca[D * (int64_t)n + a] - ca[D * (int64_t)o + a] : fc[D * f + a] - ca[D * (int64_t)o + a];
  if (!(edot<D>(S + D * f, ref) < 0.0)) return false;
  for (int a = 0; a < D; ++a) S[D * f + a] *= -1.0;
  return true;
}

// The pyramid of a face over the cell's approximate centre: volume v and v times its centroid.
template <int D>
B2S_HD void pyramid(const double* fcf, const double* Sf, double sign, const double* cac, double& v, double* vc) {
  double h[D], ss[D];
  for (int a = 0; a < D; ++a) {
    h[a] = fcf[a] - cac[a];
    ss[a] = Sf[a] * sign;
  }
  v = edot<D>(ss, h) / (double)D;
  const double frac = D == 2 ? 2.0 / 3.0 : 0.75;
  for (int a = 0; a < D; ++a) vc[a] = v * (cac[a] + frac * h[a]);
}

// Volume and centroid of cell c from its pyramids: owned faces, then neighbour faces. False
// when the volume is not positive.
template <int D>
B2S_HD bool cell_volume(int64_t c, const int32_t* own_ptr, const int32_t* own, const int32_t* nei_ptr,
                        const int32_t* nei, const double* fc, const double* S, const double* ca, double* vol,
                        double* xc) {
  const double* cac = ca + D * c;
  double vo = 0.0, vn = 0.0, mo[D], mn[D], v, vc[D];
  for (int a = 0; a < D; ++a) mo[a] = mn[a] = 0.0;
  for (int q = own_ptr[c]; q < own_ptr[c + 1]; ++q) {
    const int64_t f = own[q];
    pyramid<D>(fc + D * f, S + D * f, 1.0, cac, v, vc);
    vo += v;
    for (int a = 0; a < D; ++a) mo[a] += vc[a];
  }
  for (int q = nei_ptr[c]; q < nei_ptr[c + 1]; ++q) {
    const int64_t f = nei[q];
    pyramid<D>(fc + D * f, S + D * f, -1.0, cac, v, vc);
    vn += v;
    for (int a = 0; a < D; ++a) mn[a] += vc[a];
  }
  const double V = vo + vn;
  vol[c] = V;
  for (int a = 0; a < D; ++a) xc[D * c + a] = (mo[a] + mn[a]) / V;
  return V > 0.0;
}

template <int D>
__global__ void face_geometry_k(int nf, const double* __restrict__ X, const int32_t* __restrict__ fptr,
                                const int32_t* __restrict__ fnodes, double* __restrict__ fc, double* __restrict__ S,
                                int32_t* __restrict__ bad) {
  int local = 0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x)
    local += face_geometry<D>(f, X, fptr, fnodes, fc, S) ? 0 : 1;
  if (local) atomicAdd(bad, local);
}

template <int D>
__global__ void centre_estimate_k(int nc, const int32_t* __restrict__ own_ptr, const int32_t* __restrict__ own,
                                  const int32_t* __restrict__ nei_ptr, const int32_t* __restrict__ nei,
                                  const double* __restrict__ fc, double* __restrict__ ca) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    centre_estimate<D>(c, own_ptr, own, nei_ptr, nei, fc, ca);
}

template <int D>
__global__ void orient_k(int nf, const int32_t* __restrict__ owner, const int32_t* __restrict__ neighbour,
                         const double* __restrict__ fc, const double* __restrict__ ca, double* __restrict__ S,
                         int32_t* __restrict__ flipped) {
  int local = 0;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x)
    local += orient<D>(f, owner, neighbour, fc, ca, S) ? 1 : 0;
  if (local) atomicAdd(flipped, local);
}

template <int D>
__global__ void cell_volumes_k(int nc, const int32_t* __restrict__ own_ptr, const int32_t* __restrict__ own,
                               const int32_t* __restrict__ nei_ptr, const int32_t* __restrict__ nei,
                               const double* __restrict__ fc, const double* __restrict__ S,
                               const double* __restrict__ ca, double* __restrict__ vol, double* __restrict__ xc,
                               int32_t* __restrict__ nonpos) {
  int local = 0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
    local += cell_volume<D>(c, own_ptr, own, nei_ptr, nei, fc, S, ca, vol, xc) ? 0 : 1;
  if (local) atomicAdd(nonpos, local);
}

// Interior-face quantities (fvmesh.py:61-230), in interior-face order; cmin[0] receives the
// smallest cosine between S and d (its arccos is the mesh's non-orthogonality).
struct InteriorOut {
  double *d, *w, *alpha, *wl, *Tv, *dPf, *dNf, *dxm;
};

__device__ __forceinline__ double atomic_min_double(double* addr, double v) {
  unsigned long long* a = (unsigned long long*)addr;
  unsigned long long old = *a, assumed;
  do {
    assumed = old;
    if (__longlong_as_double((long long)assumed) <= v) break;
    old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(v));
  } while (assumed != old);
  return __longlong_as_double((long long)old);
}

template <int D>
__global__ void interior_faces_k(int n_if, const int32_t* __restrict__ fidx, const int32_t* __restrict__ P,
                                 const int32_t* __restrict__ N, const double* __restrict__ xc,
                                 const double* __restrict__ fc, const double* __restrict__ S, InteriorOut o,
                                 double* __restrict__ cmin) {
  double lmin = 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_if; i += gridDim.x * blockDim.x) {
    const int f = fidx[i];
    const double* xP = xc + D * (int64_t)P[i];
    const double* xN = xc + D * (int64_t)N[i];
    const double* xf = fc + D * (int64_t)f;
    const double* Sf = S + D * (int64_t)f;
    double d[D], t[D];
#pragma unroll
    for (int a = 0; a < D; ++a) d[a] = xN[a] - xP[a];
    const double dd = edot<D>(d, d);
#pragma unroll
    for (int a = 0; a < D; ++a) t[a] = xN[a] - xf[a];
    const double w = fmin(fmax(edot<D>(t, d) / dd, 0.0), 1.0);
    const double Sd = edot<D>(Sf, d), SS = edot<D>(Sf, Sf);
    const double alpha = SS / Sd;
    const double cs = fmin(fmax(Sd / sqrt(SS * dd), -1.0), 1.0);
    lmin = fmin(lmin, cs);
    o.w[i] = w;
    o.alpha[i] = alpha;
    o.wl[i] = 1.0 / dd;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const int64_t k = D * (int64_t)i + a;
      o.d[k] = d[a];
      o.Tv[k] = Sf[a] - alpha * d[a];
      o.dPf[k] = xf[a] - xP[a];
      o.dNf[k] = xf[a] - xN[a];
      o.dxm[k] = xf[a] - (w * xP[a] + (1.0 - w) * xN[a]);
    }
  }
  if (lmin < 1.0) atomic_min_double(cmin, lmin);
}

__global__ void fill_k(double* p, double v) { *p = v; }

struct BoundaryOut {
  double *db, *alpha_b, *wlb, *Sb_mag, *nb, *db_t, *yb;
};

template <int D>
__global__ void boundary_faces_k(int n_bf, const int32_t* __restrict__ fidx, const int32_t* __restrict__ Pb,
                                 const double* __restrict__ xc, const double* __restrict__ fc,
                                 const double* __restrict__ S, BoundaryOut o) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_bf; i += gridDim.x * blockDim.x) {
    const int f = fidx[i];
    const double* xP = xc + D * (int64_t)Pb[i];
    const double* xf = fc + D * (int64_t)f;
    const double* Sb = S + D * (int64_t)f;
    double db[D], nb[D];
#pragma unroll
    for (int a = 0; a < D; ++a) db[a] = xf[a] - xP[a];
    const double Sdb = edot<D>(Sb, db), SSb = edot<D>(Sb, Sb);
    const double mag = sqrt(SSb);
#pragma unroll
    for (int a = 0; a < D; ++a) nb[a] = Sb[a] / mag;
    const double dn = edot<D>(db, nb);
    o.alpha_b[i] = SSb / Sdb;
    o.wlb[i] = 1.0 / edot<D>(db, db);
    o.Sb_mag[i] = mag;
    o.yb[i] = fabs(edot<D>(db, Sb)) / mag;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const int64_t k = D * (int64_t)i + a;
      o.db[k] = db[a];
      o.nb[k] = nb[a];
      o.db_t[k] = db[a] - dn * nb[a];
    }
  }
}

// Least-squares matrices (three per-cell sums: faces as owner, as neighbour, boundary faces;
// then added) and their inverses by LU with partial pivoting. flag[c] = 1 where |det| <= 1e-300
// or the inverse is not finite (the caller substitutes the pseudo-inverse there).
template <int D>
__global__ void ls_matrices_k(int nc, const int32_t* __restrict__ pi_ptr, const int32_t* __restrict__ pi,
                              const int32_t* __restrict__ ni_ptr, const int32_t* __restrict__ ni,
                              const int32_t* __restrict__ pb_ptr, const int32_t* __restrict__ pb,
                              const double* __restrict__ d, const double* __restrict__ wl,
                              const double* __restrict__ db, const double* __restrict__ wlb, double* __restrict__ G,
                              double* __restrict__ Ginv, int32_t* __restrict__ flag) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    double g[D][D];
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = a; b < D; ++b) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int q = pi_ptr[c]; q < pi_ptr[c + 1]; ++q) {
          const int64_t i = pi[q];
          s1 += (wl[i] * d[D * i + a]) * d[D * i + b];
        }
        for (int q = ni_ptr[c]; q < ni_ptr[c + 1]; ++q) {
          const int64_t i = ni[q];
          s2 += (wl[i] * d[D * i + a]) * d[D * i + b];
        }
        for (int q = pb_ptr[c]; q < pb_ptr[c + 1]; ++q) {
          const int64_t i = pb[q];
          s3 += (wlb[i] * db[D * i + a]) * db[D * i + b];
        }
        g[a][b] = g[b][a] = (s1 + s2) + s3;
      }
    double* Gc = G + (int64_t)c * D * D;
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = 0; b < D; ++b) Gc[a * D + b] = g[a][b];
    // LU with partial pivoting, then the inverse column by column
    double A[D][D];
    int perm[D];
#pragma unroll
    for (int a = 0; a < D; ++a) {
      perm[a] = a;
#pragma unroll
      for (int b = 0; b < D; ++b) A[a][b] = g[a][b];
    }
    double det = 1.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      int p = k;
#pragma unroll
      for (int i = k + 1; i < D; ++i)
        if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
      if (p != k) {
#pragma unroll
        for (int b = 0; b < D; ++b) {
          const double t = A[k][b];
          A[k][b] = A[p][b];
          A[p][b] = t;
        }
        const int t = perm[k];
        perm[k] = perm[p];
        perm[p] = t;
        det = -det;
      }
      det *= A[k][k];
      const double r = 1.0 / A[k][k];
#pragma unroll
      for (int i = k + 1; i < D; ++i) {
        const double l = A[i][k] * r;
        A[i][k] = l;
#pragma unroll
        for (int b = k + 1; b < D; ++b) A[i][b] -= l * A[k][b];
      }
    }
    double* Ic = Ginv + (int64_t)c * D * D;
    bool ok = fabs(det) > 1e-300;
#pragma unroll
    for (int col = 0; col < D; ++col) {
      double y[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        double s = perm[i] == col ? 1.0 : 0.0;
#pragma unroll
        for (int j = 0; j < i; ++j) s -= A[i][j] * y[j];
        y[i] = s;
      }
#pragma unroll
      for (int i = D - 1; i >= 0; --i) {
        double s = y[i];
#pragma unroll
        for (int j = i + 1; j < D; ++j) s -= A[i][j] * y[j];
        y[i] = s / A[i][i];
      }
#pragma unroll
      for (int i = 0; i < D; ++i) {
        Ic[i * D + col] = y[i];
        ok = ok && isfinite(y[i]);
      }
    }
    flag[c] = ok ? 0 : 1;
  }
}

}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_face_geometry_d(int32_t dim, int32_t nf, const double* nodes, const int32_t* face_ptr,
                        const int32_t* face_nodes, double* fc, double* S, int32_t* bad, b2s_stream_t s) {
  if ((dim != 2 && dim != 3) || nf < 0 || !bad || (nf > 0 && (!nodes || !face_ptr || !face_nodes || !fc || !S)))
    return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (cudaMemsetAsync(bad, 0, sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  if (nf == 0) return B2S_OK;
  if (dim == 2) face_geometry_k<2><<<grid_for(nf), kThreads, 0, st>>>(nf, nodes, face_ptr, face_nodes, fc, S, bad);
  else face_geometry_k<3><<<grid_for(nf, 128), 128, 0, st>>>(nf, nodes, face_ptr, face_nodes, fc, S, bad);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_cell_geometry_d(int32_t dim, int32_t nc, int32_t nf, const int32_t* owner, const int32_t* neighbour,
                        const int32_t* own_ptr, const int32_t* own, const int32_t* nei_ptr, const int32_t* nei,
                        const double* fc, double* S, double* ca, double* vol, double* xc, int32_t* counts,
                        b2s_stream_t s) {
  if ((dim != 2 && dim != 3) || nc < 0 || nf < 0 || !counts ||
      (nc > 0 && (!owner || !neighbour || !own_ptr || !own || !nei_ptr || !nei || !fc || !S || !ca || !vol || !xc)))
    return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  // counts: [0] faces flipped by the orientation repair, [1] cells of non-positive volume
  if (cudaMemsetAsync(counts, 0, 2 * sizeof(int32_t), st) != cudaSuccess) return B2S_ERR_LAUNCH;
  if (nc == 0) return B2S_OK;
  if (dim == 2) {
    centre_estimate_k<2><<<grid_for(nc), kThreads, 0, st>>>(nc, own_ptr, own, nei_ptr, nei, fc, ca);
    orient_k<2><<<grid_for(nf), kThreads, 0, st>>>(nf, owner, neighbour, fc, ca, S, counts);
    cell_volumes_k<2><<<grid_for(nc), kThreads, 0, st>>>(nc, own_ptr, own, nei_ptr, nei, fc, S, ca, vol, xc,
                                                         counts + 1);
  } else {
    centre_estimate_k<3><<<grid_for(nc), kThreads, 0, st>>>(nc, own_ptr, own, nei_ptr, nei, fc, ca);
    orient_k<3><<<grid_for(nf), kThreads, 0, st>>>(nf, owner, neighbour, fc, ca, S, counts);
    cell_volumes_k<3><<<grid_for(nc), kThreads, 0, st>>>(nc, own_ptr, own, nei_ptr, nei, fc, S, ca, vol, xc,
                                                         counts + 1);
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_fv_faces_d(int32_t dim, int32_t n_if, const int32_t* if_idx, const int32_t* P, const int32_t* N,
                   int32_t n_bf, const int32_t* bf_idx, const int32_t* Pb, const double* xc, const double* fc,
                   const double* S, double* d, double* w, double* alpha, double* wl, double* Tv, double* dPf,
                   double* dNf, double* dxm, double* db, double* alpha_b, double* wlb, double* Sb_mag, double* nb,
                   double* db_t, double* yb, double* cos_min, b2s_stream_t s) {
  if ((dim != 2 && dim != 3) || n_if < 0 || n_bf < 0 || !cos_min || !xc || !fc || !S) return B2S_ERR_ARG;
  if (n_if > 0 && (!if_idx || !P || !N || !d || !w || !alpha || !wl || !Tv || !dPf || !dNf || !dxm))
    return B2S_ERR_ARG;
  if (n_bf > 0 && (!bf_idx || !Pb || !db || !alpha_b || !wlb || !Sb_mag || !nb || !db_t || !yb)) return B2S_ERR_ARG;
  cudaStream_t st = (cudaStream_t)s;
  fill_k<<<1, 1, 0, st>>>(cos_min, 1.0);
  InteriorOut io{d, w, alpha, wl, Tv, dPf, dNf, dxm};
  BoundaryOut bo{db, alpha_b, wlb, Sb_mag, nb, db_t, yb};
  if (n_if > 0) {
    if (dim == 2) interior_faces_k<2><<<grid_for(n_if), kThreads, 0, st>>>(n_if, if_idx, P, N, xc, fc, S, io, cos_min);
    else interior_faces_k<3><<<grid_for(n_if), kThreads, 0, st>>>(n_if, if_idx, P, N, xc, fc, S, io, cos_min);
  }
  if (n_bf > 0) {
    if (dim == 2) boundary_faces_k<2><<<grid_for(n_bf), kThreads, 0, st>>>(n_bf, bf_idx, Pb, xc, fc, S, bo);
    else boundary_faces_k<3><<<grid_for(n_bf), kThreads, 0, st>>>(n_bf, bf_idx, Pb, xc, fc, S, bo);
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_ls_matrices_d(int32_t dim, int32_t nc, const int32_t* pi_ptr, const int32_t* pi, const int32_t* ni_ptr,
                      const int32_t* ni, const int32_t* pb_ptr, const int32_t* pb, const double* d, const double* wl,
                      const double* db, const double* wlb, double* G, double* Ginv, int32_t* flag, b2s_stream_t s) {
  if ((dim != 2 && dim != 3) || nc < 0 ||
      (nc > 0 && (!pi_ptr || !pi || !ni_ptr || !ni || !pb_ptr || !pb || !d || !wl || !db || !wlb || !G || !Ginv ||
                  !flag)))
    return B2S_ERR_ARG;
  if (nc == 0) return B2S_OK;
  cudaStream_t st = (cudaStream_t)s;
  if (dim == 2)
    ls_matrices_k<2><<<grid_for(nc), kThreads, 0, st>>>(nc, pi_ptr, pi, ni_ptr, ni, pb_ptr, pb, d, wl, db, wlb, G, Ginv,
                                                        flag);
  else
    ls_matrices_k<3><<<grid_for(nc), kThreads, 0, st>>>(nc, pi_ptr, pi, ni_ptr, ni, pb_ptr, pb, d, wl, db, wlb, G, Ginv,
                                                        flag);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

/* Host counterpart of b2s_face_geometry_d (host pointers): the number of faces whose node count
 * the dimension does not allow, or B2S_ERR_ARG. */
int b2s_host_face_geometry(int32_t dim, int32_t nf, const double* nodes, const int32_t* face_ptr,
                           const int32_t* face_nodes, double* fc, double* S) {
  if ((dim != 2 && dim != 3) || nf < 0 || (nf > 0 && (!nodes || !face_ptr || !face_nodes || !fc || !S)))
    return B2S_ERR_ARG;
  int bad = 0;
  for (int64_t f = 0; f < nf; ++f) {
    const bool ok = dim == 2 ? face_geometry<2>(f, nodes, face_ptr, face_nodes, fc, S)
                             : face_geometry<3>(f, nodes, face_ptr, face_nodes, fc, S);
    if (!ok) ++bad;
  }
  return bad;
}

/* Host counterpart of b2s_face_geometry_d + b2s_cell_geometry_d (the same per-face and per-cell
 * code, run in loops): the geometry of flowtrace/mesh/unstructured.py:171-261 for host callers
 * (tests without a device, reports). repair != 0 turns the area vectors away from their owners;
 * counts[3]: faces with a node count the dimension does not allow, faces turned, cells of
 * non-positive volume. Returns B2S_OK or B2S_ERR_ARG. */
int b2s_host_geometry(int32_t dim, int32_t nc, int32_t nf, const double* nodes, const int32_t* face_ptr,
                      const int32_t* face_nodes, const int32_t* owner, const int32_t* neighbour, int32_t repair,
                      double* fc, double* S, double* xc, double* vol, int32_t* counts) {
  if ((dim != 2 && dim != 3) || nc < 0 || nf < 0 || !counts ||
      (nf > 0 && (!nodes || !face_ptr || !face_nodes || !owner || !neighbour || !fc || !S)) ||
      (nc > 0 && (!xc || !vol)))
    return B2S_ERR_ARG;
  counts[0] = counts[1] = counts[2] = 0;
  for (int64_t f = 0; f < nf; ++f)
    if (owner[f] < 0 || owner[f] >= nc || neighbour[f] >= nc) return B2S_ERR_ARG;
  // per-cell face lists in increasing face index (counting sort)
  std::vector<int32_t> own_ptr(nc + 1, 0), nei_ptr(nc + 1, 0);
  for (int64_t f = 0; f < nf; ++f) {
    ++own_ptr[owner[f] + 1];
    if (neighbour[f] >= 0) ++nei_ptr[neighbour[f] + 1];
  }
  for (int64_t c = 0; c < nc; ++c) {
    own_ptr[c + 1] += own_ptr[c];
    nei_ptr[c + 1] += nei_ptr[c];
  }
  std::vector<int32_t> own(own_ptr[nc]), nei(nei_ptr[nc]), po(own_ptr.begin(), own_ptr.end() - 1),
      pn(nei_ptr.begin(), nei_ptr.end() - 1);
  for (int64_t f = 0; f < nf; ++f) {
    own[po[owner[f]]++] = (int32_t)f;
    if (neighbour[f] >= 0) nei[pn[neighbour[f]]++] = (int32_t)f;
  }
  std::vector<double> ca((size_t)nc * dim);
  const int32_t* op = own_ptr.data();
  const int32_t* np_ = nei_ptr.data();
  for (int64_t f = 0; f < nf; ++f) {
    const bool ok = dim == 2 ? face_geometry<2>(f, nodes, face_ptr, face_nodes, fc, S)
                             : face_geometry<3>(f, nodes, face_ptr, face_nodes, fc, S);
    if (!ok) ++counts[0];
  }
  if (counts[0]) return B2S_OK;
  for (int64_t c = 0; c < nc; ++c) {
    if (dim == 2) centre_estimate<2>(c, op, own.data(), np_, nei.data(), fc, ca.data());
    else centre_estimate<3>(c, op, own.data(), np_, nei.data(), fc, ca.data());
  }
  if (repair)
    for (int64_t f = 0; f < nf; ++f) {
      const bool t = dim == 2 ? orient<2>(f, owner, neighbour, fc, ca.data(), S)
                              : orient<3>(f, owner, neighbour, fc, ca.data(), S);
      if (t) ++counts[1];
    }
  for (int64_t c = 0; c < nc; ++c) {
    const bool ok = dim == 2 ? cell_volume<2>(c, op, own.data(), np_, nei.data(), fc, S, ca.data(), vol, xc)
                             : cell_volume<3>(c, op, own.data(), np_, nei.data(), fc, S, ca.data(), vol, xc);
    if (!ok) ++counts[2];
  }
  return B2S_OK;
}

}  // extern "C"
