// k-omega SST turbulence model on B200 (Menter, Kuntz & Langtry 2003 form, as
// flowtrace/unstructured/turbulence.py:116-438 uses it inside the SIMPLEC iteration).
//
// Per outer iteration the model adds two groups of stages:
//   1. before the momentum assembly, momentum_terms_k: the face viscosities of the momentum
//      equations (mu + interpolated mu_t inside; on walls the viscosity that Spalding's law of
//      the wall gives, solved by Newton's method per wall face), the turbulent heat diffusivity
//      k/cp + mu_t/Pr_t and the explicit transpose-stress source div(mu_t (grad U)^T);
//   2. after the energy equation: boundary values of k and omega (bvals_k), their least-
//      squares gradients (the shared gradient kernel), the blending function, production and
//      cross-diffusion per cell (sources_k), for k and then omega an assembly
//      (transport_assemble_k) and a finishing pass (transport_finish_k: the near-wall omega
//      pin, whose 1e10 x max(diag) penalty needs the grid-wide maximum of the assembled
//      diagonal, the residual and the relaxation), the Jacobi-BiCGSTAB solves, and the floors,
//      F2 and mu_t (update_k).
//
// Layout and determinism follow b2s_fv.cu: one thread per cell, rows summed in the reference's
// sparse-product order, no atomics; reductions are per-block partials in fixed order.
// Transcendentals (exp, log, tanh, pow, sqrt) are CUDA's own, so the model agrees with the
// reference to a few units in the last place rather than to the bit.
#include "b2s_fv.cuh"

namespace b2s {
namespace sst {

// turbulence.py:51-57, 356-359
constexpr double kKappa = 0.41, kEWall = 9.793;
constexpr double kSk1 = 0.85, kSw1 = 0.5, kB1 = 0.075;
constexpr double kSk2 = 1.0, kSw2 = 0.856, kB2 = 0.0828;
constexpr double kBstar = 0.09, kA1 = 0.31;
constexpr double kPrT = 0.85;

// u+ of Spalding's law for the wall Reynolds number Re_y = U_t y / nu (turbulence.py:65-87):
// Newton's method on Re_y / u+ - y+(u+), started at sqrt(Re_y) (Re_y < 120) or at the log law,
// each step at most halving u+, stopped when the step is below 1e-10 u+ (per face; the
// reference stops when every face has met that test, which changes converged faces by less
// than an ulp). At most 30 steps.
__device__ __forceinline__ double spalding_uplus(double re_y, double eb) {
  const double ry = npmax0(re_y);
  double up = ry < 120.0 ? sqrt(npmax(ry, 1e-300)) : log(npmax(kEWall * sqrt(npmax(ry, 1.0)), 1.0)) / kKappa + 1.0;
  for (int it = 0; it < 30; ++it) {
    const double x = npmin(kKappa * up, 60.0);
    const double ex = exp(x);
    const double g = up + eb * (ex - 1 - x - (x * x) / 2 - pow(x, 3.0) / 6);
    const double dg = 1 + eb * kKappa * (ex - 1 - x - (x * x) / 2);
    const double uc = npmax(up, 1e-300);
    const double f = ry / uc - g;
    const double df = -ry / (uc * uc) - dg;
    const double du = f / df;
    up = npmax(up - du, 0.5 * up);
    if (fabs(du) <= 1e-10 * npmax(up, 1e-12)) break;
  }
  return ry > 0.0 ? up : 0.0;
}

// mu_t interpolated to interior face f.
__device__ __forceinline__ double mut_face(const b2s_mesh& m, const double* mut, int f) {
  const double w = m.w[f];
  return w * mut[m.fP[f]] + (1.0 - w) * mut[m.fN[f]];
}

// Diffusivity of a transport row from a cell field: interpolated inside, the owner's value on
// boundary faces (turbulence.py:284-286).
struct CellGamma {
  const double* g;
  const int32_t* fP;
  const int32_t* fN;
  const int32_t* bP;
  const double* w;
  __device__ __forceinline__ double in(int f) const { return w[f] * g[fP[f]] + (1.0 - w[f]) * g[fN[f]]; }
  __device__ __forceinline__ double bd(int f) const { return g[bP[f]]; }
};

// ------------------------------------------------------------------------------ momentum terms
// turbulence.py:235-261 and 399-417. Every cell writes the faces it owns (mu_f, kT_f), its
// boundary faces (mu_b, yplus, kT_b) and its transpose-stress source.
template <int DIM>
__global__ void momentum_terms_k(b2s_mesh m, b2s_bc bc, b2s_sst t, const double* __restrict__ Up,
                                 const double* __restrict__ gUp, const double* __restrict__ mut,
                                 double* __restrict__ mu_f, double* __restrict__ mu_b, double* __restrict__ yplus,
                                 double* __restrict__ tsrc, double* __restrict__ kT_f, double* __restrict__ kT_b) {
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  const double* gU = gUp + (int64_t)DIM * nc;  // gU[(i*DIM + a)*nc + c] = d u_i / d x_a
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
      const double mf = mut_face(m, mut, f);
      mu_f[f] = t.mu + mf;
      if (kT_f) kT_f[f] = t.k_over_cp + mf / kPrT;
    }
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      double mb = t.mu + mut[c], yp = 0.0;
      if (bc.m_wall[f] != 0.0) {
        // wall-parallel speed of the owner relative to the wall
        double rel[DIM], un = 0.0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          rel[a] = Up[(int64_t)(1 + a) * nc + c] - bc.ub_fixed[(int64_t)a * nb + f];
          const double p = rel[a] * m.nbv[(int64_t)a * nb + f];
          un = (a == 0) ? p : un + p;
        }
        double ss = 0.0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const double ta = rel[a] - un * m.nbv[(int64_t)a * nb + f];
          ss = (a == 0) ? ta * ta : ss + ta * ta;
        }
        const double re_y = sqrt(ss) * t.yb[f] / t.nu;
        const double up = spalding_uplus(re_y, t.eb);
        mb = t.mu;
        if (re_y > 1e-12 && up > 0.0) {
          mb = t.mu * re_y / (up * up);
          yp = re_y / up;
        }
      }
      mu_b[f] = mb;
      if (yplus) yplus[f] = yp;
      if (kT_b) kT_b[f] = t.k_over_cp + (bc.m_wall[f] != 0.0 ? 0.0 : mut[c] / kPrT);
    }
    // div(mu_t (grad U)^T): component k, face value mu_t,f sum_j (d u_j / d x_k)_f S_j
    double acc[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) acc[k] = 0.0;
    for_cdiff(m, c, [&](int f, bool own) {
      const int P = m.fP[f], N = m.fN[f];
      const double w = m.w[f], w1 = 1.0 - w;
      const double mf = w * mut[P] + w1 * mut[N];
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
          const double* g = gU + (int64_t)(j * DIM + k) * nc;
          const double v = (w * g[P] + w1 * g[N]) * m.S[(int64_t)j * nf + f];
          s = (j == 0) ? v : s + v;
        }
        const double v = mf * s;
        acc[k] += own ? v : -v;
      }
    });
#pragma unroll
    for (int k = 0; k < DIM; ++k) tsrc[(int64_t)k * nc + c] = acc[k];
  }
}

// ------------------------------------------------------------------------------ boundary values
// Fixed (inflow values) at inlets and at open faces with inflow, zero-gradient elsewhere
// (turbulence.py:263-269); also the mask of fixed faces, the Dirichlet mask of the transport rows.
__global__ void bvals_k(b2s_mesh m, b2s_bc bc, b2s_sst t, const double* __restrict__ KW,
                        const double* __restrict__ Fb, double* __restrict__ KWb, double* __restrict__ fixed) {
  const int nc = m.nc, nb = m.nb;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nb; f += gridDim.x * blockDim.x) {
    const int P = m.bP[f];
    const bool fx = bc.m_inlet[f] != 0.0 || (bc.m_pres[f] != 0.0 && Fb[f] < 0.0);
    KWb[f] = fx ? t.kb_in[f] : KW[P];
    KWb[nb + f] = fx ? t.wb_in[f] : KW[nc + P];
    fixed[f] = fx ? 1.0 : 0.0;
  }
}

// ------------------------------------------------------------------------------ sources
// coef rows: 0 mu + sigma_k mu_t, 1 mu + sigma_w mu_t, 2 Sc_k, 3 Sp_k, 4 Sc_w, 5 Sp_w, 6 |S|,
// 7 near-wall omega (turbulence.py:99-113, 367-380, 390-397, 419-436).
template <int DIM>
__global__ void sources_k(b2s_mesh m, b2s_sst t, const double* __restrict__ gU, const double* __restrict__ KW,
                          const double* __restrict__ gKW, const double* __restrict__ mut, double* __restrict__ coef) {
  const int nc = m.nc;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
#pragma unroll
      for (int j = 0; j < DIM; ++j) {
        const double e = 0.5 * (gU[(int64_t)(i * DIM + j) * nc + c] + gU[(int64_t)(j * DIM + i) * nc + c]);
        acc = acc + e * e;
      }
    }
    const double S = sqrt(2.0 * acc);
    const double S2 = S * S;
    const double k = KW[c], w = KW[nc + c], y = t.y[c], mt = mut[c], rho = t.rho;
    double kw = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const double p = gKW[(int64_t)a * nc + c] * gKW[(int64_t)(DIM + a) * nc + c];
      kw = (a == 0) ? p : kw + p;
    }
    const double cd = npmax(2.0 * rho * kSw2 * kw / w, 1e-10);
    const double sk = sqrt(k);
    const double visc = 500.0 * t.nu / (y * y * w);
    const double arg1 = npmin(npmax(sk / (kBstar * w * y), visc), 4.0 * rho * kSw2 * k / (cd * y * y));
    const double F1 = tanh(pow(arg1, 4.0));
    const double G1 = 1.0 - F1;
    const double Pk = npmin(mt * S2, 10.0 * kBstar * rho * k * w);
    const double cross = G1 * 2.0 * rho * kSw2 * kw / w;
    coef[c] = t.mu + (F1 * kSk1 + G1 * kSk2) * mt;
    coef[(int64_t)1 * nc + c] = t.mu + (F1 * kSw1 + G1 * kSw2) * mt;
    coef[(int64_t)2 * nc + c] = Pk;
    coef[(int64_t)3 * nc + c] = kBstar * rho * w;
    coef[(int64_t)4 * nc + c] = (F1 * t.g1 + G1 * t.g2) * rho * S2 + npmax0(cross);
    coef[(int64_t)5 * nc + c] = (F1 * kB1 + G1 * kB2) * rho * w + npmax0(-cross) / w;
    coef[(int64_t)6 * nc + c] = S;
    const double yc = t.y_wall[c];
    double wfix = 0.0;
    if (isfinite(yc)) {
      const double w_vis = 6.0 * t.nu / (kB1 * (yc * yc));
      const double w_log = sqrt(npmax0(k)) / (t.cmu25 * kKappa * yc);
      wfix = sqrt(w_vis * w_vis + w_log * w_log);
    }
    coef[(int64_t)7 * nc + c] = wfix;
  }
}

// ------------------------------------------------------------------------------ transport
// Field q (0: k, 1: omega): div(F phi) - div(gamma grad phi) = Sc - Sp phi, assembled as the
// reference's _coefficients/_rhs with the cell diffusivity coef[q] (turbulence.py:271-290);
// the unrelaxed diagonal and right-hand side are kept for the finishing pass and each block
// writes the maximum of its diagonals.
template <int DIM>
__global__ void transport_assemble_k(b2s_mesh m, b2s_sst t, int q, const double* __restrict__ KW,
                                     const double* __restrict__ KWb, const double* __restrict__ fixed,
                                     const double* __restrict__ gKW, const double* __restrict__ F,
                                     const double* __restrict__ Fb, const double* __restrict__ coef,
                                     double* __restrict__ val, double* __restrict__ diag_out,
                                     double* __restrict__ b_out, double* __restrict__ part_max) {
  __shared__ double red[kThreads / 32];
  const int nc = m.nc, nb = m.nb;
  const CellGamma gam{coef + (int64_t)q * nc, m.fP, m.fN, m.bP, m.w};
  const double* Sc = coef + (int64_t)(2 + 2 * q) * nc;
  const double* Sp = coef + (int64_t)(3 + 2 * q) * nc;
  double mx = -INFINITY;
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    RowOut<DIM, 1> o = transport_row_g<DIM, 1>(m, c, gam, fixed, F, Fb, KW + (int64_t)q * nc, nc,
                                               gKW + (int64_t)q * DIM * nc, (int64_t)DIM * nc, KWb + (int64_t)q * nb,
                                               nb, t.second_order != 0, val, true);
    const double V = m.vol[c];
    const double diag = o.diag + Sp[c] * V;
    diag_out[c] = diag;
    b_out[c] = o.rhs[0] + Sc[c] * V;
    mx = fmax(mx, diag);
  }
  mx = warp_max(mx);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) red[warp] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = red[0];
    for (int i = 1; i < nw; ++i) v = fmax(v, red[i]);
    part_max[blockIdx.x] = v;
  }
}

// The near-wall pin of omega (wall cells to coef[7] by a 1e10 max(diag) penalty), the residual
// sum |b - A phi| / sum |diag phi| over the cells above the floor and not pinned, and the
// relaxed system (diagonal diag / relax, b + (1 - relax)/relax diag phi) (turbulence.py:291-304).
template <int DIM>
__global__ void transport_finish_k(b2s_mesh m, b2s_sst t, int q, const double* __restrict__ KW,
                                   const double* __restrict__ coef, const double* __restrict__ part_max, int nblk,
                                   double* __restrict__ val, double* __restrict__ diag_io, double* __restrict__ b_io,
                                   double* __restrict__ inv_out, double* __restrict__ br_out,
                                   double* __restrict__ part_res) {
  __shared__ double red[(kThreads / 32 + 1) * 2];
  __shared__ double s_big;
  const int nc = m.nc;
  const bool pin = q == 1;
  if (pin) {
    double v = -INFINITY;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) v = fmax(v, part_max[i]);
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mx = red[0];
      for (int i = 1; i < (int)(blockDim.x >> 5); ++i) mx = fmax(mx, red[i]);
      s_big = 1e10 * mx;
    }
    __syncthreads();
  }
  const double big = pin ? s_big : 0.0;
  const double* phi = KW + (int64_t)q * nc;
  const double floor = q == 0 ? t.k_min : t.w_min;
  const double relax = q == 0 ? t.relax_k : t.relax_w;
  const double cr = (1.0 - relax) / relax;
  double acc[2] = {0.0, 0.0};
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    double d = diag_io[c], r = b_io[c];
    const bool pinned = pin && isfinite(t.y_wall[c]);
    if (pinned) {
      d = d + big;
      r = r + big * coef[(int64_t)7 * nc + c];
      diag_io[c] = d;
      b_io[c] = r;
    }
    const double ph = phi[c];
    const double Ax = row_apply(m, val, c, d, phi);
    if (ph > floor * (1.0 + 1e-9) && !pinned) {
      acc[0] += fabs(r - Ax);
      acc[1] += fabs(d * ph);
    }
    const double dr = d / relax;
    val[m.slot_diag[c]] = dr;
    inv_out[c] = 1.0 / dr;
    br_out[c] = r + (cr * d) * ph;
  }
  block_partials<2>(acc, red, part_res);
}

// Floors, then mu_t = rho a1 k / max(a1 omega, |S| F2) (turbulence.py:382-388, 434-437).
__global__ void update_k(b2s_mesh m, b2s_sst t, const double* __restrict__ KWn, const double* __restrict__ coef,
                         double* __restrict__ KW, double* __restrict__ mut) {
  const int nc = m.nc;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const double k = npmax(KWn[c], t.k_min), w = npmax(KWn[nc + c], t.w_min);
    KW[c] = k;
    KW[nc + c] = w;
    const double y = t.y[c];
    const double arg2 = npmax(2.0 * sqrt(k) / (kBstar * w * y), 500.0 * t.nu / (y * y * w));
    const double F2 = tanh(arg2 * arg2);
    mut[c] = t.rho * kA1 * k / npmax(kA1 * w, coef[(int64_t)6 * nc + c] * F2);
  }
}

}  // namespace sst
}  // namespace b2s

using namespace b2s;

static bool sst_ok(const b2s_mesh* m, const b2s_sst* t) {
  return m && m->nc > 0 && m->nf >= 0 && m->nb >= 0 && (m->dim == 2 || m->dim == 3) && m->own_ptr && m->fP &&
         m->fN && m->bptr && t && t->y && t->y_wall && (m->nb == 0 || (t->yb && t->kb_in && t->wb_in)) &&
         t->nu > 0.0 && t->relax_k > 0.0 && t->relax_w > 0.0;
}

static unsigned sst_part_grid(const b2s_mesh& m) {
  if (m.tiles) return (unsigned)m.ntiles;
  int64_t g = cdiv(m.nc, kThreads);
  return (unsigned)(g < kMaxCoopBlocks ? g : kMaxCoopBlocks);
}

extern "C" {

int b2s_sst_part_blocks(const b2s_mesh* m) { return m ? (int)sst_part_grid(*m) : 0; }

int b2s_sst_momentum_terms_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_sst* t, const double* Up,
                             const double* gUp, const double* mut, double* mu_f, double* mu_b, double* yplus,
                             double* tsrc, double* kT_f, double* kT_b, b2s_stream_t s) {
  if (!sst_ok(m, t) || !bc || !Up || !gUp || !mut || (!mu_f && m->nf) || (!mu_b && m->nb) || !tsrc ||
      (!kT_f != !kT_b))
    return B2S_ERR_ARG;
  unsigned g = grid_for(m->nc);
  if (m->dim == 2)
    sst::momentum_terms_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *t, Up, gUp, mut, mu_f, mu_b, yplus, tsrc,
                                                                   kT_f, kT_b);
  else
    sst::momentum_terms_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *t, Up, gUp, mut, mu_f, mu_b, yplus, tsrc,
                                                                   kT_f, kT_b);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_sst_bvals_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_sst* t, const double* KW, const double* Fb,
                    double* KWb, double* fixed, b2s_stream_t s) {
  if (!sst_ok(m, t) || !bc || !KW || !Fb || !KWb || !fixed) return B2S_ERR_ARG;
  if (m->nb == 0) return B2S_OK;
  sst::bvals_k<<<grid_for(m->nb), kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *t, KW, Fb, KWb, fixed);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_sst_sources_d(const b2s_mesh* m, const b2s_sst* t, const double* gU, const double* KW, const double* gKW,
                      const double* mut, double* coef, b2s_stream_t s) {
  if (!sst_ok(m, t) || !gU || !KW || !gKW || !mut || !coef) return B2S_ERR_ARG;
  unsigned g = grid_for(m->nc);
  if (m->dim == 2) sst::sources_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *t, gU, KW, gKW, mut, coef);
  else sst::sources_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *t, gU, KW, gKW, mut, coef);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_sst_transport_assemble_d(const b2s_mesh* m, const b2s_sst* t, int q, const double* KW, const double* KWb,
                                 const double* fixed, const double* gKW, const double* F, const double* Fb,
                                 const double* coef, double* val, double* diag, double* b, double* part_max,
                                 b2s_stream_t s) {
  if (!sst_ok(m, t) || (q != 0 && q != 1) || !KW || (m->nb && (!KWb || !fixed || !Fb)) || !gKW || (!F && m->nf) ||
      !coef || !val || !diag || !b || !part_max)
    return B2S_ERR_ARG;
  unsigned g = sst_part_grid(*m);
  if (m->dim == 2)
    sst::transport_assemble_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *t, q, KW, KWb, fixed, gKW, F, Fb, coef,
                                                                       val, diag, b, part_max);
  else
    sst::transport_assemble_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *t, q, KW, KWb, fixed, gKW, F, Fb, coef,
                                                                       val, diag, b, part_max);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_sst_transport_finish_d(const b2s_mesh* m, const b2s_sst* t, int q, const double* KW, const double* coef,
                               const double* part_max, double* val, double* diag, double* b, double* inv, double* br,
                               double* part_res, b2s_stream_t s) {
  if (!sst_ok(m, t) || (q != 0 && q != 1) || !KW || !coef || !part_max || !val || !diag || !b || !inv || !br ||
      !part_res)
    return B2S_ERR_ARG;
  unsigned g = sst_part_grid(*m);
  if (m->dim == 2)
    sst::transport_finish_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *t, q, KW, coef, part_max, (int)g, val, diag,
                                                                     b, inv, br, part_res);
  else
    sst::transport_finish_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *t, q, KW, coef, part_max, (int)g, val, diag,
                                                                     b, inv, br, part_res);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_sst_update_d(const b2s_mesh* m, const b2s_sst* t, const double* KWn, const double* coef, double* KW,
                     double* mut, b2s_stream_t s) {
  if (!sst_ok(m, t) || !KWn || !coef || !KW || !mut) return B2S_ERR_ARG;
  sst::update_k<<<grid_for(m->nc), kThreads, 0, (cudaStream_t)s>>>(*m, *t, KWn, coef, KW, mut);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"
