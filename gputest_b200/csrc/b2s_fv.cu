// Finite-volume stages of the SIMPLEC outer iteration on B200: face interpolation, least-
// squares and Green-Gauss gradients, CSR assembly, and the fused momentum, Rhie-Chow /
// pressure-correction, correction and energy stages.
//
// Every kernel is cell-centric: one thread per cell walks the faces it owns (a contiguous
// range, faces being sorted by owner), the faces it neighbours (a short index list) and its
// boundary faces (a contiguous range). A cell writes only its own rows and its owned faces,
// so there are no atomics and the results are deterministic. Per cell the terms are summed in
// the order of the reference's sparse products (flowtrace/unstructured/fvmesh.py:254-309):
// owned faces, then neighbour faces, then boundary faces, each in reference face order, and
// the rows of Cdiff (owned and neighbour faces merged by reference face index); compiled
// without FMA contraction, the results then match the reference's NumPy path to the bit
// wherever the reference's own reductions are not involved.
//
// Bandwidth: each interior face is read by its two cells; with RCM-ordered cells the second
// read falls inside a window that L2 (126 MB) holds, so DRAM sees each face once.
#include "b2s_fv.cuh"

namespace b2s {

// ------------------------------------------------------------------------------ face interp
__global__ void face_interp_k(b2s_mesh m, int k, const double* __restrict__ phi, double* __restrict__ out) {
  const int64_t nf = m.nf, nc = m.nc;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nf * k; t += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = t / nf, f = t - c * nf;
    double wf = m.w[f];
    out[t] = wf * phi[c * nc + m.fP[f]] + (1.0 - wf) * phi[c * nc + m.fN[f]];
  }
}

// ------------------------------------------------------------------------------ LS gradient
// r = Cown(wl dphi d) + Cnei(wl dphi d) + Cb(wlb dphib db); grad = Ginv r
// (flowtrace/unstructured/fvmesh.py:268-286).
template <int DIM, int NF>
__global__ void ls_gradient_k(b2s_mesh m, const double* __restrict__ phi, const double* __restrict__ phib,
                              double* __restrict__ grad) {
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    double ro[NF][DIM], rn[NF][DIM], rb[NF][DIM];
#pragma unroll
    for (int q = 0; q < NF; ++q)
#pragma unroll
      for (int a = 0; a < DIM; ++a) ro[q][a] = rn[q][a] = rb[q][a] = 0.0;
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
      const int P = m.fP[f], N = m.fN[f];
      const double wl = m.wl[f];
#pragma unroll
      for (int q = 0; q < NF; ++q) {
        const double coef = wl * (phi[(int64_t)q * nc + N] - phi[(int64_t)q * nc + P]);
#pragma unroll
        for (int a = 0; a < DIM; ++a) ro[q][a] += coef * m.d[(int64_t)a * nf + f];
      }
    }
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
      const int f = m.nei_face[k];
      const int P = m.fP[f], N = m.fN[f];
      const double wl = m.wl[f];
#pragma unroll
      for (int q = 0; q < NF; ++q) {
        const double coef = wl * (phi[(int64_t)q * nc + N] - phi[(int64_t)q * nc + P]);
#pragma unroll
        for (int a = 0; a < DIM; ++a) rn[q][a] += coef * m.d[(int64_t)a * nf + f];
      }
    }
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      const double wlb = m.wlb[f];
#pragma unroll
      for (int q = 0; q < NF; ++q) {
        const double coef = wlb * (phib[(int64_t)q * nb + f] - phi[(int64_t)q * nc + c]);
#pragma unroll
        for (int a = 0; a < DIM; ++a) rb[q][a] += coef * m.db[(int64_t)a * nb + f];
      }
    }
#pragma unroll
    for (int q = 0; q < NF; ++q) {
      double r[DIM];
#pragma unroll
      for (int a = 0; a < DIM; ++a) r[a] = (ro[q][a] + rn[q][a]) + rb[q][a];
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < DIM; ++b) s += m.Ginv[(int64_t)(a * DIM + b) * nc + c] * r[b];
        grad[((int64_t)q * DIM + a) * nc + c] = s;
      }
    }
  }
}

// ------------------------------------------------------------------------------ GG gradient
// (1/V)(Cdiff(pf S) + Cb(phib Sb)), pf = face_interp(phi) + face_interp(grad).dxm
// (flowtrace/unstructured/fvmesh.py:288-309).
template <int DIM>
__device__ __forceinline__ double gg_face_value(const b2s_mesh& m, int f, const double* phi, const double* grad) {
  const int nc = m.nc, nf = m.nf, P = m.fP[f], N = m.fN[f];
  const double w = m.w[f];
  double pf = w * phi[P] + (1.0 - w) * phi[N];
  if (grad) {
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const double gf = w * grad[(int64_t)a * nc + P] + (1.0 - w) * grad[(int64_t)a * nc + N];
      s = (a == 0) ? gf * m.dxm[(int64_t)a * nf + f] : s + gf * m.dxm[(int64_t)a * nf + f];
    }
    pf = pf + s;
  }
  return pf;
}

template <int DIM>
__global__ void gg_gradient_k(b2s_mesh m, const double* __restrict__ phi, const double* __restrict__ phib,
                              const double* __restrict__ grad, double* __restrict__ out) {
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    double si[DIM], sb[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) si[a] = sb[a] = 0.0;
    for_cdiff(m, c, [&](int f, bool own) {
      const double pf = gg_face_value<DIM>(m, f, phi, grad);
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        const double v = pf * m.S[(int64_t)a * nf + f];
        si[a] += own ? v : -v;
      }
    });
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
#pragma unroll
      for (int a = 0; a < DIM; ++a) sb[a] += phib[f] * m.Sb[(int64_t)a * nb + f];
    }
    const double v = m.vol[c];
#pragma unroll
    for (int a = 0; a < DIM; ++a) out[(int64_t)a * nc + c] = (si[a] + sb[a]) / v;
  }
}

// ------------------------------------------------------------------------------ assembly
// data[slot_diag] = diag; data[slot_PN] += aPN; data[slot_NP] += aNP
// (flowtrace/unstructured/fvmesh.py:332-348); row-owned, no atomics.
__global__ void assemble_k(b2s_mesh m, const double* __restrict__ diag, const double* __restrict__ aPN,
                           const double* __restrict__ aNP, double* __restrict__ val) {
  const int nc = m.nc;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    for (int s = m.rowptr[c]; s < m.rowptr[c + 1]; ++s) val[s] = 0.0;
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) val[m.slot_PN[f]] += aPN[f];
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
      const int f = m.nei_face[k];
      val[m.slot_NP[f]] += aNP[f];
    }
    val[m.slot_diag[c]] = diag[c];
  }
}

// ------------------------------------------------------------------------------ boundary values
// ub = (m_wall + m_inlet) ub_fixed + m_sym (UP - (UP.n) n) + m_pres UP, UP = U_P (+ gU_P . dbt);
// pb = m_pres pb_fixed + (1 - m_pres)(p_P (+ gp_P . db))   (simple.py:305-325)
template <int DIM>
__global__ void flow_bvals_k(b2s_mesh m, b2s_bc bc, const double* __restrict__ Up, const double* __restrict__ gUp,
                             const double* __restrict__ gpf, double* __restrict__ bUp) {
  const int nc = m.nc, nb = m.nb;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nb; f += gridDim.x * blockDim.x) {
    const int P = m.bP[f];
    double UP[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      UP[k] = Up[(int64_t)(1 + k) * nc + P];
      if (gUp) {
        double s = 0.0;
#pragma unroll
        for (int a = 0; a < DIM; ++a) {
          const double t = gUp[((int64_t)(1 + k) * DIM + a) * nc + P] * m.dbt[(int64_t)a * nb + f];
          s = (a == 0) ? t : s + t;
        }
        UP[k] = UP[k] + s;
      }
    }
    double un = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      const double t = UP[k] * m.nbv[(int64_t)k * nb + f];
      un = (k == 0) ? t : un + t;
    }
    const double fixed = bc.m_wall[f] + bc.m_inlet[f], msym = bc.m_sym[f], mp = bc.m_pres[f];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      const double sym = UP[k] - un * m.nbv[(int64_t)k * nb + f];
      bUp[(int64_t)(1 + k) * nb + f] = (fixed * bc.ub_fixed[(int64_t)k * nb + f] + msym * sym) + mp * UP[k];
    }
    double pP = Up[P];
    if (gpf) {
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        const double t = gpf[(int64_t)a * nc + P] * m.db[(int64_t)a * nb + f];
        s = (a == 0) ? t : s + t;
      }
      pP = pP + s;
    }
    bUp[f] = mp * bc.pb_fixed[f] + (1.0 - mp) * pP;
  }
}


// ------------------------------------------------------------------------------ momentum
// 2-D: at most 64 registers, so four 256-thread blocks fit per SM and a 131k-cell mesh runs in
// one wave (80 registers gave 1.16 waves; measured 0.045 -> 0.033 ms); 3-D at most 80 registers,
// three blocks per SM (measured against 128 registers and two blocks: 2.12 -> 1.90 ms on a
// 4.2M-cell duct, 0.262 -> 0.227 ms on the 524k duct, despite 180 bytes of spills; 64 registers
// and four blocks spilled twice as much and gained nothing).
// TURB: per-face viscosities mu_f [nf] / mu_b [nb] and a per-cell source tsrc [DIM][nc] from the
// turbulence model (mu + mu_t, the wall-function viscosity on walls, the transpose stress;
// simple.py:545-548); the laminar instantiation is the scalar-viscosity kernel unchanged.
template <int DIM, bool TURB>
__global__ void __launch_bounds__(kThreads, DIM == 2 ? 4 : 3) momentum_assemble_k(b2s_mesh m, b2s_bc bc, b2s_flow_params prm, const double* __restrict__ Up,
                                    const double* __restrict__ gUp, const double* __restrict__ gp,
                                    const double* __restrict__ bUp, const double* __restrict__ F,
                                    const double* __restrict__ Fb, const double* __restrict__ por,
                                    const double* __restrict__ msrc, double* __restrict__ val,
                                    double* __restrict__ diag_out, double* __restrict__ inv_out,
                                    double* __restrict__ dP_out, double* __restrict__ b_out,
                                    double* __restrict__ br_out, double* __restrict__ part,
                                    const double* __restrict__ mu_f, const double* __restrict__ mu_b,
                                    const double* __restrict__ tsrc) {
  __shared__ double red[(kThreads / 32 + 1) * 2 * DIM];
  const int nc = m.nc, nb = m.nb;
  double acc[2 * DIM];
#pragma unroll
  for (int q = 0; q < 2 * DIM; ++q) acc[q] = 0.0;
  const bool drive = prm.body[0] != 0.0 || prm.body[1] != 0.0 || (DIM == 3 && prm.body[2] != 0.0);
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    const double au = prm.relax_u_cell ? prm.relax_u_cell[c] : prm.relax_u;
    const bool simplec = prm.simplec_cell ? prm.simplec_cell[c] != 0 : prm.simplec != 0;
    RowOut<DIM, DIM> o;
    if constexpr (TURB)
      o = transport_row_g<DIM, DIM>(m, c, FaceGamma{mu_f, mu_b}, bc.m_dirvel, F, Fb, Up + nc, nc,
                                    gUp + (int64_t)DIM * nc, (int64_t)DIM * nc, bUp + nb, nb, prm.second_order != 0,
                                    val, true);
    else
      o = transport_row<DIM, DIM>(m, c, prm.mu, bc.m_dirvel, F, Fb, Up + nc, nc, gUp + (int64_t)DIM * nc,
                                  (int64_t)DIM * nc, bUp + nb, nb, prm.second_order != 0, val, true);
    double diag = o.diag;
    const double V = m.vol[c];
    if (por) diag = diag + por[c] * V;
    const double diag_r = diag / au;
    val[m.slot_diag[c]] = diag_r;
    inv_out[c] = 1.0 / diag_r;
    diag_out[c] = diag;
    double denom = diag_r;
    if (simplec) {
      denom = diag_r - o.sumnb;
      denom = (denom > 1e-12 * diag_r) ? denom : diag_r;
    }
    dP_out[c] = V / denom;
    const double cr = (1.0 - au) / au;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      double src = -gp[(int64_t)k * nc + c] * V;
      if (drive) src = src + V * prm.body[k];
      if (msrc) src = src + msrc[(int64_t)k * nc + c];
      if constexpr (TURB) src = src + tsrc[(int64_t)k * nc + c];
      const double rhs = o.rhs[k] + src;
      const double* u = Up + (int64_t)(1 + k) * nc;
      const double Au = row_apply(m, val, c, diag, u);
      acc[k] += fabs(rhs - Au);
      acc[DIM + k] += fabs(diag * u[c]);
      b_out[(int64_t)k * nc + c] = rhs;
      br_out[(int64_t)k * nc + c] = rhs + (cr * diag) * u[c];
    }
  }
  block_partials<2 * DIM>(acc, red, part);
}

// ------------------------------------------------------------------------------ pressure correction
// Rhie-Chow predictor fluxes and the p' system (simple.py:583-623). Face values are computed
// identically from both sides of a face, so owner and neighbour see the same bits.
template <int DIM>
__device__ __forceinline__ void rc_face(const b2s_mesh& m, const b2s_flow_params& prm, int f, const double* Ustar,
                                        const double* p, const double* gp, const double* dP, double& Fst,
                                        double& cf) {
  const int nc = m.nc, nf = m.nf, P = m.fP[f], N = m.fN[f];
  const double w = m.w[f], w1 = 1.0 - w;
  const double dF = w * dP[P] + w1 * dP[N];
  double us = 0.0, gd = 0.0;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const double uf = w * Ustar[(int64_t)a * nc + P] + w1 * Ustar[(int64_t)a * nc + N];
    const double gf = w * gp[(int64_t)a * nc + P] + w1 * gp[(int64_t)a * nc + N];
    const double t1 = uf * m.S[(int64_t)a * nf + f], t2 = gf * m.d[(int64_t)a * nf + f];
    us = (a == 0) ? t1 : us + t1;
    gd = (a == 0) ? t2 : gd + t2;
  }
  const double al = m.alpha[f];
  Fst = prm.rho * (us - dF * al * (p[N] - p[P] - gd));
  cf = prm.rho * dF * al;
}

template <int DIM>
__device__ __forceinline__ void rc_bface(const b2s_mesh& m, const b2s_bc& bc, const b2s_flow_params& prm, int f,
                                         int P, const double* Ustar, const double* p, const double* gp,
                                         const double* dP, double& Fbst, double& cb) {
  const int nc = m.nc, nb = m.nb;
  double ui = 0.0, us = 0.0, gd = 0.0;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
    const double sb = m.Sb[(int64_t)a * nb + f];
    const double t0 = bc.ub_fixed[(int64_t)a * nb + f] * sb;
    const double t1 = Ustar[(int64_t)a * nc + P] * sb;
    const double t2 = gp[(int64_t)a * nc + P] * m.db[(int64_t)a * nb + f];
    ui = (a == 0) ? t0 : ui + t0;
    us = (a == 0) ? t1 : us + t1;
    gd = (a == 0) ? t2 : gd + t2;
  }
  const double mp = bc.m_pres[f];
  const double fb_in = prm.rho * ui * bc.m_inlet[f];
  const double fb_pr = prm.rho * (us - dP[P] * m.alpha_b[f] * (bc.pb_fixed[f] - p[P] - gd));
  Fbst = fb_in + fb_pr * mp;
  cb = prm.rho * dP[P] * m.alpha_b[f] * mp;
}

template <int DIM, class VT>
__global__ void pressure_assemble_k(b2s_mesh m, b2s_bc bc, b2s_flow_params prm, const double* __restrict__ Ustar,
                                    const double* __restrict__ p, const double* __restrict__ gp,
                                    const double* __restrict__ dP, double* __restrict__ Fst_out,
                                    double* __restrict__ cf_out, double* __restrict__ Fbst_out,
                                    double* __restrict__ cb_out, VT* __restrict__ val, double* __restrict__ rhs,
                                    double* __restrict__ part) {
  __shared__ double red[(kThreads / 32 + 1) * 1];
  double acc[1] = {0.0};
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    double d_own = 0.0, d_nei = 0.0, d_b = 0.0, m_int = 0.0, m_b = 0.0;
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
      double Fst, cf;
      rc_face<DIM>(m, prm, f, Ustar, p, gp, dP, Fst, cf);
      Fst_out[f] = Fst;
      cf_out[f] = cf;
      d_own += cf;
      val[m.slot_PN[f]] = -cf;
    }
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
      const int f = m.nei_face[k];
      double Fst, cf;
      rc_face<DIM>(m, prm, f, Ustar, p, gp, dP, Fst, cf);
      d_nei += cf;
      val[m.slot_NP[f]] = -cf;
    }
    for_cdiff(m, c, [&](int f, bool own) {
      double Fst, cf;
      rc_face<DIM>(m, prm, f, Ustar, p, gp, dP, Fst, cf);
      m_int += own ? Fst : -Fst;
    });
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      double Fbst, cb;
      rc_bface<DIM>(m, bc, prm, f, c, Ustar, p, gp, dP, Fbst, cb);
      Fbst_out[f] = Fbst;
      cb_out[f] = cb;
      d_b += cb;
      m_b += Fbst;
    }
    val[m.slot_diag[c]] = (d_own + d_nei) + d_b;
    const double mass = m_int + m_b;
    rhs[c] = -mass;
    acc[0] += fabs(mass);
  }
  block_partials<1>(acc, red, part);
}

// ------------------------------------------------------------------------------ corrections
template <int DIM>
__global__ void correct_k(b2s_mesh m, b2s_bc bc, b2s_flow_params prm, const double* __restrict__ Fst,
                          const double* __restrict__ cf, const double* __restrict__ Fbst,
                          const double* __restrict__ cb, const double* __restrict__ pp, const double* __restrict__ p,
                          const double* __restrict__ Ustar, const double* __restrict__ dP, double* __restrict__ F,
                          double* __restrict__ Fb, double* __restrict__ Up_new, double* __restrict__ part) {
  __shared__ double red[(kThreads / 32 + 1) * 3];
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  double acc[3] = {0.0, 0.0, 0.0};
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    double ro[DIM], rn[DIM], rb[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) ro[a] = rn[a] = rb[a] = 0.0;
    const double ppc = pp[c];
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
      const int N = m.fN[f];
      const double ppN = pp[N];
      const double Fn = Fst[f] + cf[f] * (ppc - ppN);
      F[f] = Fn;
      acc[1] += fabs(Fn);
      const double coef = m.wl[f] * (ppN - ppc);
#pragma unroll
      for (int a = 0; a < DIM; ++a) ro[a] += coef * m.d[(int64_t)a * nf + f];
    }
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
      const int f = m.nei_face[k];
      const double coef = m.wl[f] * (ppc - pp[m.fP[f]]);
#pragma unroll
      for (int a = 0; a < DIM; ++a) rn[a] += coef * m.d[(int64_t)a * nf + f];
    }
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      const double fbn = Fbst[f] + cb[f] * ppc;
      Fb[f] = fbn;
      acc[2] += fabs(fbn);
      const double ppb = (1.0 - bc.m_pres[f]) * ppc;
      const double coef = m.wlb[f] * (ppb - ppc);
#pragma unroll
      for (int a = 0; a < DIM; ++a) rb[a] += coef * m.db[(int64_t)a * nb + f];
    }
    const double pn = p[c] + (prm.relax_p_cell ? prm.relax_p_cell[c] : prm.relax_p) * ppc;
    Up_new[c] = pn;
    acc[0] += pn;
    double r[DIM];
#pragma unroll
    for (int a = 0; a < DIM; ++a) r[a] = (ro[a] + rn[a]) + rb[a];
    const double dp = dP[c];
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < DIM; ++b) s += m.Ginv[(int64_t)(a * DIM + b) * nc + c] * r[b];
      Up_new[(int64_t)(1 + a) * nc + c] = Ustar[(int64_t)a * nc + c] - dp * s;
    }
  }
  block_partials<3>(acc, red, part);
}

__global__ void remove_mean_k(int n, double* __restrict__ x, const double* __restrict__ part, int nblk, int nq,
                              int q) {
  __shared__ double tot[1];
  grid_totals(part + (int64_t)q * nblk, nblk, 1, tot);
  const double mean = tot[0] / (double)n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = x[i] - mean;
}

__global__ void sum_partials_k(const double* __restrict__ part, int nblk, int nq, int npairs,
                               const int32_t* __restrict__ q_of, double* __restrict__ out) {
  for (int j = blockIdx.x; j < npairs; j += gridDim.x) {
    const double t = warp_total(part, nblk, nq, q_of[j]);
    if (threadIdx.x == 0) out[j] = t;
  }
}

// ------------------------------------------------------------------------------ energy
// Tb = fixed ? tval : T_P (+ gT_P . dbt); outlet backflow (Fb < 0) takes tval (simple.py:783-791)
template <int DIM>
__global__ void energy_bvals_k(b2s_mesh m, b2s_bc bc, const double* __restrict__ T, const double* __restrict__ gT,
                               const double* __restrict__ Fb, double* __restrict__ Tb) {
  const int nc = m.nc, nb = m.nb;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nb; f += gridDim.x * blockDim.x) {
    const int P = m.bP[f];
    double TP = T[P];
    if (gT) {
      double s = 0.0;
#pragma unroll
      for (int a = 0; a < DIM; ++a) {
        const double t = gT[(int64_t)a * nc + P] * m.dbt[(int64_t)a * nb + f];
        s = (a == 0) ? t : s + t;
      }
      TP = TP + s;
    }
    double v = bc.m_tfix[f] != 0.0 ? bc.tval[f] : TP;
    if (bc.m_out[f] != 0.0 && Fb[f] < 0.0) v = bc.tval[f];
    Tb[f] = v;
  }
}

// GT: ScalarGamma (k/cp) or FaceGamma (k/cp + mu_t/Pr_t per face from the turbulence model,
// simple.py:781-782).
template <int DIM, class GT>
__global__ void energy_assemble_k(b2s_mesh m, b2s_bc bc, GT gamma, double cp, double aT, int second,
                                  const double* __restrict__ T, const double* __restrict__ gT,
                                  const double* __restrict__ Tb, const double* __restrict__ F,
                                  const double* __restrict__ Fb, const double* __restrict__ esrc,
                                  double* __restrict__ val, double* __restrict__ diag_out, double* __restrict__ inv_out,
                                  double* __restrict__ b_out, double* __restrict__ br_out, double* __restrict__ part) {
  __shared__ double red[(kThreads / 32 + 1) * 2];
  const int nc = m.nc, nb = m.nb;
  double acc[2] = {0.0, 0.0};
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    RowOut<DIM, 1> o = transport_row_g<DIM, 1>(m, c, gamma, bc.m_tfix, F, Fb, T, nc, gT, (int64_t)DIM * nc, Tb, nb,
                                             second != 0, val, true);
    // q_in = Cb(flux tval |Sb| / cp) (+ source)
    double q = 0.0;
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) q += bc.m_tflux[f] * bc.tval[f] * m.Sb_mag[f] / cp;
    if (esrc) q = q + esrc[c];
    const double rhs = o.rhs[0] + q;
    const double diag = o.diag;
    const double Au = row_apply(m, val, c, diag, T);
    acc[0] += fabs(rhs - Au);
    acc[1] += fabs(diag * T[c]);
    const double dr = diag / aT;
    val[m.slot_diag[c]] = dr;
    inv_out[c] = 1.0 / dr;
    diag_out[c] = diag;
    b_out[c] = rhs;
    br_out[c] = rhs + (((1.0 - aT) / aT) * diag) * T[c];
  }
  block_partials<2>(acc, red, part);
}

// ------------------------------------------------------------------------------ mixed precision
// The mixed-precision iteration solves every linear system in correction form: the residual
// r = b - A phi of the unrelaxed system is evaluated in double from the coefficients in
// registers (the nonlinear residual, whose zero is the converged solution), and the relaxed
// system A_r dphi = r (A_r: diagonal a_P / alpha; the same iterates as A_r phi = b_r from
// x0 = phi) is stored in float for the Krylov solve; phi + dphi is formed in double.

// sum_nb a_nb phi_nb of row c for NQ fields: upwind + diffusion off-diagonals recomputed from
// the face data the row assembly has just read (simple.py:340-353).
template <int NQ, class GT>
__device__ __forceinline__ void offdiag_apply_g(const b2s_mesh& m, int c, const GT& gam, const double* F,
                                                const double* phi, int64_t phi_stride, double (&out)[NQ]) {
#pragma unroll
  for (int q = 0; q < NQ; ++q) out[q] = 0.0;
  for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
    const double aPN = -(gam.in(f) * m.alpha[f] + npmax0(-F[f]));
    const int N = m.fN[f];
#pragma unroll
    for (int q = 0; q < NQ; ++q) out[q] += aPN * phi[q * phi_stride + N];
  }
  for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
    const int f = m.nei_face[k];
    const double aNP = -(gam.in(f) * m.alpha[f] + npmax0(F[f]));
    const int P = m.fP[f];
#pragma unroll
    for (int q = 0; q < NQ; ++q) out[q] += aNP * phi[q * phi_stride + P];
  }
}

template <int NQ>
__device__ __forceinline__ void offdiag_apply(const b2s_mesh& m, int c, double gamma, const double* F,
                                              const double* phi, int64_t phi_stride, double (&out)[NQ]) {
  offdiag_apply_g<NQ>(m, c, ScalarGamma{gamma}, F, phi, phi_stride, out);
}

// 2-D: at most 64 registers, so four 256-thread blocks fit per SM and a 131k-cell mesh runs in
// one wave (80 registers gave 1.16 waves; measured 0.045 -> 0.033 ms); 3-D at most 80 registers,
// three blocks per SM (measured against 128 registers and two blocks: 2.12 -> 1.90 ms on a
// 4.2M-cell duct, 0.262 -> 0.227 ms on the 524k duct, despite 180 bytes of spills; 64 registers
// and four blocks spilled twice as much and gained nothing).
// TURB: per-face viscosities and the transpose-stress source, as momentum_assemble_k<DIM, true>.
template <int DIM, bool TURB>
__global__ void __launch_bounds__(kThreads, DIM == 2 ? 4 : 2) momentum_assemble_mixed_k(b2s_mesh m, b2s_bc bc, b2s_flow_params prm, const double* __restrict__ Up,
                                          const double* __restrict__ gUp, const double* __restrict__ gp,
                                          const double* __restrict__ bUp, const double* __restrict__ F,
                                          const double* __restrict__ Fb, const double* __restrict__ por,
                                          const double* __restrict__ msrc, float* __restrict__ val,
                                          float* __restrict__ inv_out, double* __restrict__ dP_out,
                                          float* __restrict__ r_out, double* __restrict__ part,
                                          const double* __restrict__ mu_f, const double* __restrict__ mu_b,
                                          const double* __restrict__ tsrc) {
  __shared__ double red[(kThreads / 32 + 1) * 2 * DIM];
  const int nc = m.nc, nb = m.nb;
  double acc[2 * DIM];
#pragma unroll
  for (int q = 0; q < 2 * DIM; ++q) acc[q] = 0.0;
  const bool drive = prm.body[0] != 0.0 || prm.body[1] != 0.0 || (DIM == 3 && prm.body[2] != 0.0);
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    const double au = prm.relax_u_cell ? prm.relax_u_cell[c] : prm.relax_u;
    const bool simplec = prm.simplec_cell ? prm.simplec_cell[c] != 0 : prm.simplec != 0;
    RowOut<DIM, DIM> o;
    if constexpr (TURB)
      o = transport_row_g<DIM, DIM>(m, c, FaceGamma{mu_f, mu_b}, bc.m_dirvel, F, Fb, Up + nc, nc,
                                    gUp + (int64_t)DIM * nc, (int64_t)DIM * nc, bUp + nb, nb, prm.second_order != 0,
                                    val, true);
    else
      o = transport_row<DIM, DIM>(m, c, prm.mu, bc.m_dirvel, F, Fb, Up + nc, nc, gUp + (int64_t)DIM * nc,
                                  (int64_t)DIM * nc, bUp + nb, nb, prm.second_order != 0, val, true);
    double diag = o.diag;
    const double V = m.vol[c];
    if (por) diag = diag + por[c] * V;
    const double diag_r = diag / au;
    val[m.slot_diag[c]] = (float)diag_r;
    inv_out[c] = (float)(1.0 / diag_r);
    double denom = diag_r;
    if (simplec) {
      denom = diag_r - o.sumnb;
      denom = (denom > 1e-12 * diag_r) ? denom : diag_r;
    }
    dP_out[c] = V / denom;
    double anb[DIM];
    if constexpr (TURB) offdiag_apply_g<DIM>(m, c, FaceGamma{mu_f, mu_b}, F, Up + nc, nc, anb);
    else offdiag_apply<DIM>(m, c, prm.mu, F, Up + nc, nc, anb);
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      double src = -gp[(int64_t)k * nc + c] * V;
      if (drive) src = src + V * prm.body[k];
      if (msrc) src = src + msrc[(int64_t)k * nc + c];
      if constexpr (TURB) src = src + tsrc[(int64_t)k * nc + c];
      const double rhs = o.rhs[k] + src;
      const double uc = Up[(int64_t)(1 + k) * nc + c];
      const double r = rhs - (diag * uc + anb[k]);
      acc[k] += fabs(r);
      acc[DIM + k] += fabs(diag * uc);
      r_out[(int64_t)k * nc + c] = (float)r;
    }
  }
  block_partials<2 * DIM>(acc, red, part);
}

template <int DIM, class GT>
__global__ void energy_assemble_mixed_k(b2s_mesh m, b2s_bc bc, GT gamma, double cp, double aT, int second,
                                        const double* __restrict__ T, const double* __restrict__ gT,
                                        const double* __restrict__ Tb, const double* __restrict__ F,
                                        const double* __restrict__ Fb, const double* __restrict__ esrc,
                                        float* __restrict__ val, float* __restrict__ inv_out, float* __restrict__ r_out,
                                        double* __restrict__ part) {
  __shared__ double red[(kThreads / 32 + 1) * 2];
  const int nc = m.nc, nb = m.nb;
  double acc[2] = {0.0, 0.0};
  for (CellRange r_ = cell_range(m); r_.c < r_.end; r_.c += r_.step) {
    const int c = r_.c;
    RowOut<DIM, 1> o = transport_row_g<DIM, 1>(m, c, gamma, bc.m_tfix, F, Fb, T, nc, gT, (int64_t)DIM * nc, Tb, nb,
                                             second != 0, val, true);
    double q = 0.0;
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) q += bc.m_tflux[f] * bc.tval[f] * m.Sb_mag[f] / cp;
    if (esrc) q = q + esrc[c];
    const double rhs = o.rhs[0] + q;
    const double diag = o.diag;
    double anb[1];
    offdiag_apply_g<1>(m, c, gamma, F, T, nc, anb);
    const double Tc = T[c];
    const double r = rhs - (diag * Tc + anb[0]);
    acc[0] += fabs(r);
    acc[1] += fabs(diag * Tc);
    const double dr = diag / aT;
    val[m.slot_diag[c]] = (float)dr;
    inv_out[c] = (float)(1.0 / dr);
    r_out[c] = (float)r;
  }
  block_partials<2>(acc, red, part);
}

// ------------------------------------------------------------------------------ diagnostics
// r = b - A x, s = |b| + |A| |x| per row over the CSR in stored order; dval (when given)
// replaces the diagonal values (the unrelaxed a_P of a system stored relaxed)
// (flowtrace/unstructured/diagnostics.py:146-151).
__global__ void row_residuals_k(int n, const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                                const double* __restrict__ val, const int32_t* __restrict__ slot_diag,
                                const double* __restrict__ dval, const double* __restrict__ b,
                                const double* __restrict__ x, double* __restrict__ r, double* __restrict__ sc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int sd = dval ? slot_diag[i] : -1;
    double ax = 0.0, as = 0.0;
    for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) {
      const double a = (j == sd) ? dval[i] : val[j];
      const double xj = x[col[j]];
      ax += a * xj;
      as += fabs(a) * fabs(xj);
    }
    r[i] = b[i] - ax;
    sc[i] = fabs(b[i]) + as;
  }
}

// Cell mass imbalance m = Cdiff F + Cb Fb and throughflow t = Cown|F| + Cnei|F| + Cb|Fb|
// (diagnostics.py:253-257).
__global__ void flux_balance_k(b2s_mesh m, const double* __restrict__ F, const double* __restrict__ Fb,
                               double* __restrict__ mout, double* __restrict__ tout) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m.nc; c += gridDim.x * blockDim.x) {
    double mi = 0.0, mb = 0.0, to = 0.0, tn = 0.0, tb = 0.0;
    for_cdiff(m, c, [&](int f, bool own) { mi += own ? F[f] : -F[f]; });
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) to += fabs(F[f]);
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) tn += fabs(F[m.nei_face[k]]);
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      mb += Fb[f];
      tb += fabs(Fb[f]);
    }
    mout[c] = mi + mb;
    tout[c] = (to + tn) + tb;
  }
}

// Properties of a cell-cell matrix on the mesh pattern that decide whether CG applies
// (flowtrace/unstructured/diagnostics.py:384-412, restated from the definitions): per row the
// diagonal and the sum of |off-diagonal| in stored order, per owned face the pair
// (a_PN, a_NP), which is the whole off-diagonal pattern (every off-diagonal entry belongs to
// one face, no pair repeats). Per block: max |a|, max |a_PN - a_NP|, max off-diagonal entry,
// min (a_ii - sum_j |a_ij|) / max(|a_ii|, 1e-300), min a_ii; NaN propagates through every max
// and min. Max and min are exact, so the result does not depend on the order.
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? NAN : fmax(a, b); }
__device__ __forceinline__ double nan_min(double a, double b) { return (a != a || b != b) ? NAN : fmin(a, b); }

constexpr int kPropQ = 5;
constexpr int kPropBlocks = 1024;

__global__ void matrix_properties_k(b2s_mesh m, const double* __restrict__ val, double* __restrict__ part) {
  __shared__ double red[kPropQ][kThreads / 32];
  double q[kPropQ] = {0.0, 0.0, -INFINITY, INFINITY, INFINITY};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m.nc; c += gridDim.x * blockDim.x) {
    double dg = 0.0, off = 0.0;
    for (int j = m.rowptr[c]; j < m.rowptr[c + 1]; ++j) {
      const double a = val[j];
      q[0] = nan_max(q[0], fabs(a));
      if (m.col[j] == c) {
        dg = a;
      } else {
        off += fabs(a);
        q[2] = nan_max(q[2], a);
      }
    }
    q[3] = nan_min(q[3], (dg - off) / fmax(fabs(dg), 1e-300));
    q[4] = nan_min(q[4], dg);
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) q[1] = nan_max(q[1], fabs(val[m.slot_PN[f]] - val[m.slot_NP[f]]));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kPropQ; ++k) {
    double v = q[k];
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_xor_sync(0xffffffffu, v, o);
      v = (k >= 3) ? nan_min(v, u) : nan_max(v, u);
    }
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < kPropQ) {
    const int k = threadIdx.x;
    double v = red[k][0];
    for (int w = 1; w < kThreads / 32; ++w) v = (k >= 3) ? nan_min(v, red[k][w]) : nan_max(v, red[k][w]);
    part[k * kPropBlocks + blockIdx.x] = v;
  }
}

__global__ void matrix_properties_finish_k(int nblk, const double* __restrict__ part, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= kPropQ) return;
  double v = part[k * kPropBlocks];
  for (int b = 1; b < nblk; ++b) v = (k >= 3) ? nan_min(v, part[k * kPropBlocks + b]) : nan_max(v, part[k * kPropBlocks + b]);
  out[k] = v;
}

}  // namespace b2s

using namespace b2s;

static unsigned part_grid(int64_t n);
static unsigned part_grid_m(const b2s_mesh& m) { return m.tiles ? (unsigned)m.ntiles : part_grid(m.nc); }
static unsigned part_grid(int64_t n) {
  int64_t g = cdiv(n > 0 ? n : 1, kThreads);
  return (unsigned)(g < kMaxCoopBlocks ? g : kMaxCoopBlocks);
}

template <int DIM>
static void launch_ls(const b2s_mesh* m, int nfield, const double* phi, const double* phib, double* grad,
                      cudaStream_t st) {
  unsigned g = grid_for(m->nc);
  switch (nfield) {
    case 1: ls_gradient_k<DIM, 1><<<g, kThreads, 0, st>>>(*m, phi, phib, grad); break;
    case 2: ls_gradient_k<DIM, 2><<<g, kThreads, 0, st>>>(*m, phi, phib, grad); break;
    case 3: ls_gradient_k<DIM, 3><<<g, kThreads, 0, st>>>(*m, phi, phib, grad); break;
    default: ls_gradient_k<DIM, 4><<<g, kThreads, 0, st>>>(*m, phi, phib, grad); break;
  }
}

extern "C" {

int b2s_abi_version(void) { return B2S_ABI_VERSION; }

int b2s_device_sm_count(void) {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return n;
}

int b2s_part_blocks(int32_t n) { return (int)part_grid(n); }

static bool mesh_ok(const b2s_mesh* m) {
  return m && m->nc > 0 && m->nf >= 0 && m->nb >= 0 && (m->dim == 2 || m->dim == 3) && m->own_ptr && m->fP &&
         m->fN && m->bptr;
}

int b2s_face_interp_d(const b2s_mesh* m, int k, const double* phi, double* out, b2s_stream_t s) {
  if (!mesh_ok(m) || k < 1 || !phi || !out) return B2S_ERR_ARG;
  if (m->nf == 0) return B2S_OK;
  face_interp_k<<<grid_for((int64_t)m->nf * k), kThreads, 0, (cudaStream_t)s>>>(*m, k, phi, out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_ls_gradient_d(const b2s_mesh* m, int nfield, const double* phi, const double* phib, double* grad,
                      b2s_stream_t s) {
  if (!mesh_ok(m) || nfield < 1 || nfield > 4 || !phi || (!phib && m->nb) || !grad) return B2S_ERR_ARG;
  if (m->dim == 2) launch_ls<2>(m, nfield, phi, phib, grad, (cudaStream_t)s);
  else launch_ls<3>(m, nfield, phi, phib, grad, (cudaStream_t)s);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_gg_gradient_d(const b2s_mesh* m, const double* phi, const double* phib, const double* grad, double* out,
                      b2s_stream_t s) {
  if (!mesh_ok(m) || !phi || (!phib && m->nb) || !out) return B2S_ERR_ARG;
  unsigned g = grid_for(m->nc);
  if (m->dim == 2) gg_gradient_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, phi, phib, grad, out);
  else gg_gradient_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, phi, phib, grad, out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_assemble_d(const b2s_mesh* m, const double* diag, const double* aPN, const double* aNP, double* val,
                   b2s_stream_t s) {
  if (!mesh_ok(m) || !diag || (!aPN && m->nf) || (!aNP && m->nf) || !val || !m->rowptr) return B2S_ERR_ARG;
  assemble_k<<<grid_for(m->nc), kThreads, 0, (cudaStream_t)s>>>(*m, diag, aPN, aNP, val);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_flow_bvals_d(const b2s_mesh* m, const b2s_bc* bc, const double* Up, const double* gUp, const double* gpf,
                     double* bUp, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !Up || !bUp) return B2S_ERR_ARG;
  if (m->nb == 0) return B2S_OK;
  unsigned g = grid_for(m->nb);
  if (m->dim == 2) flow_bvals_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, Up, gUp, gpf, bUp);
  else flow_bvals_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, Up, gUp, gpf, bUp);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"

template <bool TURB>
static int momentum_assemble(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Up,
                             const double* gUp, const double* gp, const double* bUp, const double* F,
                             const double* Fb, const double* porosity, const double* msrc, double* val,
                             double* diag, double* inv, double* dP, double* b, double* br, double* part,
                             const double* mu_f, const double* mu_b, const double* tsrc, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !prm || !Up || !gUp || !gp || !bUp || !F || !Fb || !val || !diag || !inv || !dP || !b ||
      !br || !part || !(prm->relax_u > 0.0))
    return B2S_ERR_ARG;
  if (TURB && (!mu_f || (!mu_b && m->nb) || !tsrc)) return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    momentum_assemble_k<2, TURB><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Up, gUp, gp, bUp, F, Fb,
                                                                       porosity, msrc, val, diag, inv, dP, b, br,
                                                                       part, mu_f, mu_b, tsrc);
  else
    momentum_assemble_k<3, TURB><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Up, gUp, gp, bUp, F, Fb,
                                                                       porosity, msrc, val, diag, inv, dP, b, br,
                                                                       part, mu_f, mu_b, tsrc);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

extern "C" {

int b2s_momentum_assemble_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Up,
                            const double* gUp, const double* gp, const double* bUp, const double* F,
                            const double* Fb, const double* porosity, const double* msrc, double* val,
                            double* diag, double* inv, double* dP, double* b, double* br, double* part,
                            b2s_stream_t s) {
  return momentum_assemble<false>(m, bc, prm, Up, gUp, gp, bUp, F, Fb, porosity, msrc, val, diag, inv, dP, b, br,
                                  part, nullptr, nullptr, nullptr, s);
}

int b2s_momentum_assemble_turb_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Up,
                                 const double* gUp, const double* gp, const double* bUp, const double* F,
                                 const double* Fb, const double* porosity, const double* msrc, const double* mu_f,
                                 const double* mu_b, const double* tsrc, double* val, double* diag, double* inv,
                                 double* dP, double* b, double* br, double* part, b2s_stream_t s) {
  return momentum_assemble<true>(m, bc, prm, Up, gUp, gp, bUp, F, Fb, porosity, msrc, val, diag, inv, dP, b, br,
                                 part, mu_f, mu_b, tsrc, s);
}

int b2s_pressure_assemble_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Ustar,
                            const double* p, const double* gp, const double* dP, double* Fst, double* cf,
                            double* Fbst, double* cb, double* val, double* rhs, double* part, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !prm || !Ustar || !p || !gp || !dP || !Fst || !cf || !Fbst || !cb || !val || !rhs ||
      !part)
    return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    pressure_assemble_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Ustar, p, gp, dP, Fst, cf, Fbst, cb,
                                                                 val, rhs, part);
  else
    pressure_assemble_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Ustar, p, gp, dP, Fst, cf, Fbst, cb,
                                                                 val, rhs, part);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_correct_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm, const double* Fst,
                  const double* cf, const double* Fbst, const double* cb, const double* pp, const double* p,
                  const double* Ustar, const double* dP, double* F, double* Fb, double* Up_new, double* part,
                  b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !prm || !Fst || !cf || !Fbst || !cb || !pp || !p || !Ustar || !dP || !F || !Fb ||
      !Up_new || !part)
    return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    correct_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Fst, cf, Fbst, cb, pp, p, Ustar, dP, F, Fb,
                                                       Up_new, part);
  else
    correct_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Fst, cf, Fbst, cb, pp, p, Ustar, dP, F, Fb,
                                                       Up_new, part);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_remove_mean_d(int32_t n, double* x, const double* part, int nblk, int nq, int q, b2s_stream_t s) {
  if (n <= 0 || !x || !part || nblk <= 0 || nq <= 0 || q < 0 || q >= nq) return B2S_ERR_ARG;
  remove_mean_k<<<part_grid(n), kThreads, 0, (cudaStream_t)s>>>(n, x, part, nblk, nq, q);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_sum_partials_d(const double* part, int nblk, int nq, int npairs, const int32_t* q_of, double* out,
                       b2s_stream_t s) {
  if (!part || nblk <= 0 || nq <= 0 || npairs <= 0 || !q_of || !out) return B2S_ERR_ARG;
  sum_partials_k<<<(unsigned)npairs, 32, 0, (cudaStream_t)s>>>(part, nblk, nq, npairs, q_of, out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_energy_bvals_d(const b2s_mesh* m, const b2s_bc* bc, const double* T, const double* gT, const double* Fb,
                       double* Tb, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !T || !Fb || !Tb) return B2S_ERR_ARG;
  if (m->nb == 0) return B2S_OK;
  unsigned g = grid_for(m->nb);
  if (m->dim == 2) energy_bvals_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, T, gT, Fb, Tb);
  else energy_bvals_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, T, gT, Fb, Tb);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"

template <class GT>
static int energy_assemble(const b2s_mesh* m, const b2s_bc* bc, GT gamma, double cp, double relax_T,
                           int second_order, const double* T, const double* gT, const double* Tb, const double* F,
                           const double* Fb, const double* esrc, double* val, double* diag, double* inv, double* b,
                           double* br, double* part, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !T || !gT || (!Tb && m->nb) || !F || !Fb || !val || !diag || !inv || !b || !br ||
      !part || !(relax_T > 0.0) || !(cp != 0.0))
    return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    energy_assemble_k<2, GT><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, gamma, cp, relax_T, second_order, T, gT,
                                                                   Tb, F, Fb, esrc, val, diag, inv, b, br, part);
  else
    energy_assemble_k<3, GT><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, gamma, cp, relax_T, second_order, T, gT,
                                                                   Tb, F, Fb, esrc, val, diag, inv, b, br, part);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

extern "C" {

int b2s_energy_assemble_d(const b2s_mesh* m, const b2s_bc* bc, double gamma, double cp, double relax_T,
                          int second_order, const double* T, const double* gT, const double* Tb, const double* F,
                          const double* Fb, const double* esrc, double* val, double* diag, double* inv, double* b,
                          double* br, double* part, b2s_stream_t s) {
  return energy_assemble(m, bc, ScalarGamma{gamma}, cp, relax_T, second_order, T, gT, Tb, F, Fb, esrc, val, diag,
                         inv, b, br, part, s);
}

int b2s_energy_assemble_turb_d(const b2s_mesh* m, const b2s_bc* bc, const double* gamma_f, const double* gamma_b,
                               double cp, double relax_T, int second_order, const double* T, const double* gT,
                               const double* Tb, const double* F, const double* Fb, const double* esrc, double* val,
                               double* diag, double* inv, double* b, double* br, double* part, b2s_stream_t s) {
  if (!gamma_f || (!gamma_b && m && m->nb)) return B2S_ERR_ARG;
  return energy_assemble(m, bc, FaceGamma{gamma_f, gamma_b}, cp, relax_T, second_order, T, gT, Tb, F, Fb, esrc, val,
                         diag, inv, b, br, part, s);
}

}  // extern "C"

template <bool TURB>
static int momentum_assemble_mixed(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                   const double* Up, const double* gUp, const double* gp, const double* bUp,
                                   const double* F, const double* Fb, const double* porosity, const double* msrc,
                                   float* val, float* inv, double* dP, float* r, double* part, const double* mu_f,
                                   const double* mu_b, const double* tsrc, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !prm || !Up || !gUp || !gp || !bUp || !F || !Fb || !val || !inv || !dP || !r || !part ||
      !(prm->relax_u > 0.0))
    return B2S_ERR_ARG;
  if (TURB && (!mu_f || (!mu_b && m->nb) || !tsrc)) return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    momentum_assemble_mixed_k<2, TURB><<<g, kThreads, 0, (cudaStream_t)s>>>(
        *m, *bc, *prm, Up, gUp, gp, bUp, F, Fb, porosity, msrc, val, inv, dP, r, part, mu_f, mu_b, tsrc);
  else
    momentum_assemble_mixed_k<3, TURB><<<g, kThreads, 0, (cudaStream_t)s>>>(
        *m, *bc, *prm, Up, gUp, gp, bUp, F, Fb, porosity, msrc, val, inv, dP, r, part, mu_f, mu_b, tsrc);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

extern "C" {

int b2s_momentum_assemble_mixed_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                  const double* Up, const double* gUp, const double* gp, const double* bUp,
                                  const double* F, const double* Fb, const double* porosity, const double* msrc,
                                  float* val, float* inv, double* dP, float* r, double* part, b2s_stream_t s) {
  return momentum_assemble_mixed<false>(m, bc, prm, Up, gUp, gp, bUp, F, Fb, porosity, msrc, val, inv, dP, r, part,
                                        nullptr, nullptr, nullptr, s);
}

int b2s_momentum_assemble_mixed_turb_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                       const double* Up, const double* gUp, const double* gp, const double* bUp,
                                       const double* F, const double* Fb, const double* porosity,
                                       const double* msrc, const double* mu_f, const double* mu_b,
                                       const double* tsrc, float* val, float* inv, double* dP, float* r,
                                       double* part, b2s_stream_t s) {
  return momentum_assemble_mixed<true>(m, bc, prm, Up, gUp, gp, bUp, F, Fb, porosity, msrc, val, inv, dP, r, part,
                                       mu_f, mu_b, tsrc, s);
}

int b2s_pressure_assemble_mixed_d(const b2s_mesh* m, const b2s_bc* bc, const b2s_flow_params* prm,
                                  const double* Ustar, const double* p, const double* gp, const double* dP,
                                  double* Fst, double* cf, double* Fbst, double* cb, float* val, double* rhs,
                                  double* part, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !prm || !Ustar || !p || !gp || !dP || !Fst || !cf || !Fbst || !cb || !val || !rhs ||
      !part)
    return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    pressure_assemble_k<2><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Ustar, p, gp, dP, Fst, cf, Fbst, cb,
                                                                 val, rhs, part);
  else
    pressure_assemble_k<3><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, *prm, Ustar, p, gp, dP, Fst, cf, Fbst, cb,
                                                                 val, rhs, part);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"

template <class GT>
static int energy_assemble_mixed(const b2s_mesh* m, const b2s_bc* bc, GT gamma, double cp, double relax_T,
                                 int second_order, const double* T, const double* gT, const double* Tb,
                                 const double* F, const double* Fb, const double* esrc, float* val, float* inv,
                                 float* r, double* part, b2s_stream_t s) {
  if (!mesh_ok(m) || !bc || !T || !gT || (!Tb && m->nb) || !F || !Fb || !val || !inv || !r || !part ||
      !(relax_T > 0.0) || !(cp != 0.0))
    return B2S_ERR_ARG;
  unsigned g = part_grid_m(*m);
  if (m->dim == 2)
    energy_assemble_mixed_k<2, GT><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, gamma, cp, relax_T, second_order,
                                                                         T, gT, Tb, F, Fb, esrc, val, inv, r, part);
  else
    energy_assemble_mixed_k<3, GT><<<g, kThreads, 0, (cudaStream_t)s>>>(*m, *bc, gamma, cp, relax_T, second_order,
                                                                         T, gT, Tb, F, Fb, esrc, val, inv, r, part);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

extern "C" {

int b2s_energy_assemble_mixed_d(const b2s_mesh* m, const b2s_bc* bc, double gamma, double cp, double relax_T,
                                int second_order, const double* T, const double* gT, const double* Tb,
                                const double* F, const double* Fb, const double* esrc, float* val, float* inv,
                                float* r, double* part, b2s_stream_t s) {
  return energy_assemble_mixed(m, bc, ScalarGamma{gamma}, cp, relax_T, second_order, T, gT, Tb, F, Fb, esrc, val, inv,
                               r, part, s);
}

int b2s_energy_assemble_mixed_turb_d(const b2s_mesh* m, const b2s_bc* bc, const double* gamma_f,
                                     const double* gamma_b, double cp, double relax_T, int second_order,
                                     const double* T, const double* gT, const double* Tb, const double* F,
                                     const double* Fb, const double* esrc, float* val, float* inv, float* r,
                                     double* part, b2s_stream_t s) {
  if (!gamma_f || (!gamma_b && m && m->nb)) return B2S_ERR_ARG;
  return energy_assemble_mixed(m, bc, FaceGamma{gamma_f, gamma_b}, cp, relax_T, second_order, T, gT, Tb, F, Fb, esrc,
                               val, inv, r, part, s);
}

int b2s_row_residuals_d(int32_t n, const int32_t* rowptr, const int32_t* col, const double* val,
                        const int32_t* slot_diag, const double* dval, const double* b, const double* x, double* r,
                        double* s_out, b2s_stream_t s) {
  if (n <= 0 || !rowptr || !col || !val || !b || !x || !r || !s_out || (dval && !slot_diag)) return B2S_ERR_ARG;
  row_residuals_k<<<grid_for(n), kThreads, 0, (cudaStream_t)s>>>(n, rowptr, col, val, slot_diag, dval, b, x, r, s_out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int b2s_flux_balance_d(const b2s_mesh* m, const double* F, const double* Fb, double* mass, double* through,
                       b2s_stream_t s) {
  if (!mesh_ok(m) || !F || !Fb || !mass || !through) return B2S_ERR_ARG;
  flux_balance_k<<<grid_for(m->nc), kThreads, 0, (cudaStream_t)s>>>(*m, F, Fb, mass, through);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

int64_t b2s_matrix_properties_workspace_bytes(void) { return (int64_t)kPropQ * kPropBlocks * (int64_t)sizeof(double); }

int b2s_matrix_properties_d(const b2s_mesh* m, const double* val, double* work, int64_t work_bytes, double* out,
                            b2s_stream_t s) {
  if (!mesh_ok(m) || m->nc <= 0 || !val || !work || !out) return B2S_ERR_ARG;
  if (work_bytes < b2s_matrix_properties_workspace_bytes()) return B2S_ERR_WORKSPACE;
  const unsigned g = grid_for(m->nc) < (unsigned)kPropBlocks ? grid_for(m->nc) : (unsigned)kPropBlocks;
  matrix_properties_k<<<g, kThreads, 0, (cudaStream_t)s>>>(*m, val, work);
  B2S_LAUNCH_CHECK();
  matrix_properties_finish_k<<<1, 32, 0, (cudaStream_t)s>>>((int)g, work, out);
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"
