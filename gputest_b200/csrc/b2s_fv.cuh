// Row-level helpers shared by the finite-volume stages (b2s_fv.cu) and the k-omega SST stages
// (b2s_sst.cu): NumPy-compatible min/max, the merged walk over a cell's Cdiff row, the cell
// range of a partial-sum stage, and one row of a convection-diffusion system.
#pragma once

#include "b2s_common.cuh"

namespace b2s {

// numpy.maximum(x, 0.0): NaN propagates, -0.0 stays -0.0.
__device__ __forceinline__ double npmax0(double x) { return (x < 0.0) ? 0.0 : x; }
__device__ __forceinline__ double npmin(double a, double b) { return (a <= b || a != a) ? a : b; }
__device__ __forceinline__ double npmax(double a, double b) { return (a >= b || a != a) ? a : b; }

// Visit the rows of Cdiff: the owned and neighbour faces of cell c merged by reference face
// index; fn(face, +1/-1).
template <class Fn>
__device__ __forceinline__ void for_cdiff(const b2s_mesh& m, int c, Fn fn) {
  int j = m.own_ptr[c], je = m.own_ptr[c + 1];
  int k = m.nei_ptr[c], ke = m.nei_ptr[c + 1];
  int kf = k < ke ? m.nei_face[k] : 0;
  while (j < je || k < ke) {
    bool own = (k >= ke) || (j < je && m.forig[j] < m.forig[kf]);
    if (own) {
      fn(j, true);
      ++j;
    } else {
      fn(kf, false);
      ++k;
      if (k < ke) kf = m.nei_face[k];
    }
  }
}

// Cells of this block in a stage that writes one partial sum per block: a grid-stride range
// of cells, or, on a tiled mesh (block-diagonal batches), exactly the cells of tile blockIdx.x.
struct CellRange {
  int c, end, step;
};
__device__ __forceinline__ CellRange cell_range(const b2s_mesh& m) {
  if (m.tiles) return {m.tiles[blockIdx.x] + (int)threadIdx.x, m.tiles[blockIdx.x + 1], (int)blockDim.x};
  return {(int)(blockIdx.x * blockDim.x + threadIdx.x), m.nc, (int)(gridDim.x * blockDim.x)};
}


// ------------------------------------------------------------------------------ transport rows
// One row of a convection-diffusion system (simple.py:340-374): coefficients, the CSR row,
// and the right-hand side of NQ scalar fields that share the matrix.
//   diag = (Cown(D + max(F,0)) + Cnei(D + max(-F,0))) + Cb(Db + max(Fb,0)),  D = gamma alpha
//   aPN = -(D + max(-F,0)), aNP = -(D + max(F,0)),  Db = gamma alpha_b dirichlet
//   rhs = Cb((Db + max(-Fb,0)) phib) + Cdiff(gamma gf.T) [- Cdiff(F (ho - up))] + extra
template <int DIM, int NQ>
struct RowOut {
  double diag;     // a_P (before relaxation and extra diagonal terms)
  double sumnb;    // scatter(-aPN, -aNP)
  double rhs[NQ];  // without the extra source
};

// Diffusivity of a row: one value on every face (laminar), or per-face values (interior faces
// in device order, boundary faces) as the turbulence model supplies them (simple.py:333-338).
struct ScalarGamma {
  double g;
  __device__ __forceinline__ double in(int) const { return g; }
  __device__ __forceinline__ double bd(int) const { return g; }
};
struct FaceGamma {
  const double* gf;  // [nf]
  const double* gb;  // [nb]
  __device__ __forceinline__ double in(int f) const { return gf[f]; }
  __device__ __forceinline__ double bd(int f) const { return gb[f]; }
};

template <int DIM, int NQ, class VT, class GT>
__device__ __forceinline__ RowOut<DIM, NQ> transport_row_g(const b2s_mesh& m, int c, const GT& gam,
                                                         const double* dirichlet, const double* F, const double* Fb,
                                                         const double* phi, int64_t phi_stride,
                                                         const double* grad, int64_t grad_stride,
                                                         const double* phib, int64_t phib_stride, bool second,
                                                         VT* val, bool write_offdiag) {
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  RowOut<DIM, NQ> o;
  double s_own = 0.0, s_nei = 0.0, s_b = 0.0, nb_own = 0.0, nb_nei = 0.0;
  for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
    const double D = gam.in(f) * m.alpha[f], Ff = F[f];
    s_own += D + npmax0(Ff);
    const double aPN = -(D + npmax0(-Ff));
    nb_own += -aPN;
    if (write_offdiag) val[m.slot_PN[f]] = aPN;
  }
  for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
    const int f = m.nei_face[k];
    const double D = gam.in(f) * m.alpha[f], Ff = F[f];
    s_nei += D + npmax0(-Ff);
    const double aNP = -(D + npmax0(Ff));
    nb_nei += -aNP;
    if (write_offdiag) val[m.slot_NP[f]] = aNP;
  }
  double rb[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) rb[q] = 0.0;
  for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
    const double Db = gam.bd(f) * m.alpha_b[f] * dirichlet[f];
    const double Fbf = Fb[f];
    s_b += Db + npmax0(Fbf);
    const double coef = Db + npmax0(-Fbf);
#pragma unroll
    for (int q = 0; q < NQ; ++q) rb[q] += coef * phib[q * phib_stride + f];
  }
  o.diag = (s_own + s_nei) + s_b;
  o.sumnb = nb_own + nb_nei;
  // explicit non-orthogonal diffusion and deferred second-order correction over Cdiff rows
  double rn[NQ], rh[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) rn[q] = rh[q] = 0.0;
  for_cdiff(m, c, [&](int f, bool own) {
    const int P = m.fP[f], N = m.fN[f];
    const double w = m.w[f], w1 = 1.0 - w, Ff = F[f];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const double* g = grad + q * grad_stride;
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        const double gf = w * g[(int64_t)a * nc + P] + w1 * g[(int64_t)a * nc + N];
        const double t = gf * m.Tv[(int64_t)a * nf + f];
        s = (a == 0) ? t : s + t;
      }
      const double v = gam.in(f) * s;
      rn[q] += own ? v : -v;
      if (second) {
        const double* ph = phi + q * phi_stride;
        const double phP = ph[P], phN = ph[N];
        double hoP = 0.0, hoN = 0.0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const double tP = g[(int64_t)a * nc + P] * m.dPf[(int64_t)a * nf + f];
          const double tN = g[(int64_t)a * nc + N] * m.dNf[(int64_t)a * nf + f];
          hoP = (a == 0) ? tP : hoP + tP;
          hoN = (a == 0) ? tN : hoN + tN;
        }
        hoP = phP + hoP;
        hoN = phN + hoN;
        const bool up = Ff >= 0.0;
        const double lo = npmin(phP, phN), hi = npmax(phP, phN);
        const double ho = npmin(npmax(up ? hoP : hoN, lo), hi);
        const double dc = Ff * (ho - (up ? phP : phN));
        rh[q] += own ? dc : -dc;
      }
    }
  });
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double r = rb[q] + rn[q];
    if (second) r = r - rh[q];
    o.rhs[q] = r;
  }
  return o;
}

template <int DIM, int NQ, class VT>
__device__ __forceinline__ RowOut<DIM, NQ> transport_row(const b2s_mesh& m, int c, double gamma,
                                                         const double* dirichlet, const double* F, const double* Fb,
                                                         const double* phi, int64_t phi_stride,
                                                         const double* grad, int64_t grad_stride,
                                                         const double* phib, int64_t phib_stride, bool second,
                                                         VT* val, bool write_offdiag) {
  return transport_row_g<DIM, NQ>(m, c, ScalarGamma{gamma}, dirichlet, F, Fb, phi, phi_stride, grad, grad_stride,
                                   phib, phib_stride, second, val, write_offdiag);
}

// (A x)_c over the CSR row in stored order with a_cc = dval (scipy's csr_matvec order).
__device__ __forceinline__ double row_apply(const b2s_mesh& m, const double* val, int c, double dval,
                                            const double* x) {
  const int sd = m.slot_diag[c];
  double s = 0.0;
  for (int j = m.rowptr[c]; j < m.rowptr[c + 1]; ++j) s += (j == sd ? dval : val[j]) * x[m.col[j]];
  return s;
}

}  // namespace b2s
