// Vector-Jacobian product of the steady SIMPLEC residual on B200 (the discrete adjoint's
// operator). The residual, with the lagged and derived quantities of the iteration as unknowns:
//
//   x = (U [dim][nc], p [nc], g [dim][nc], F [nf], Fb [nb]),  theta = (alpha [nc], ub [dim][nb])
//   R_m  = b - A U         momentum: upwind + diffusion, Brinkman drag alpha V, force -g V
//   R_c  = Cdiff F + Cb Fb continuity
//   R_g  = g - GG(p, p_b)  Green-Gauss pressure gradient, p_b = p_P + g_P . d_b off pressure faces
//   R_F  = F - rho (u_f . S - dP_f alpha (p_N - p_P - g_f . d))          Rhie-Chow
//   R_Fb = Fb - rho ub . Sb [inlet] - rho (U_P . Sb - dP_P alpha_b (pb - p_P - g_P . d_b)) [pressure]
//   dP   = V / (a_P / alpha_u - sum a_nb)  (SIMPLEC; SIMPLE: V / (a_P / alpha_u))
//
// (flowtrace/unstructured/simple.py:340-374, 583-623 with upwind convection on a mesh without
// non-orthogonal terms). Given lambda in the residual's blocks, the kernels return
// (dR/dx)^T lambda in x's blocks and (dR/dtheta)^T lambda. Two cell-centric passes, no atomics:
// the first forms per cell the momentum coefficients, dP and the adjoint sensitivities of dP,
// a_P and sum a_nb; the second gathers every output of a cell (and of the faces it owns, and of
// its boundary faces) from its faces - the transposed face loop.
#include "b2s_common.cuh"

namespace b2s {

__device__ __forceinline__ double relu(double x) { return x > 0.0 ? x : 0.0; }
__device__ __forceinline__ double drelu(double x) { return x > 0.0 ? 1.0 : 0.0; }

struct VjpArgs {
  b2s_mesh m;
  b2s_bc bc;
  double rho, mu, relax_u;
  int simplec;
  const double* U;   // [dim][nc]
  const double* p;   // [nc]
  const double* g;   // [dim][nc]
  const double* F;   // [nf]
  const double* Fb;  // [nb]
  const double* por; // [nc] or NULL
  const double* lm;  // lambda: [dim][nc]
  const double* lc;  // [nc]
  const double* lg;  // [dim][nc]
  const double* lF;  // [nf]
  const double* lFb; // [nb]
  double* work;      // [4][nc]: dP, a_diag, a_sumnb, diag
  double* oU;        // (dR/dx)^T lambda: [dim][nc]
  double* op;        // [nc]
  double* og;        // [dim][nc]
  double* oF;        // [nf]
  double* oFb;       // [nb]
  double* opor;      // (dR/dalpha)^T lambda [nc], or NULL
  double* oub;       // (dR/dub)^T lambda [dim][nb], or NULL
};

template <int DIM>
__global__ void vjp_pass1_k(VjpArgs a) {
  const b2s_mesh& m = a.m;
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    double diag = 0.0, snb = 0.0;
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
      const double D = a.mu * m.alpha[f], Ff = a.F[f];
      diag += D + relu(Ff);
      snb += D + relu(-Ff);
    }
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
      const int f = m.nei_face[k];
      const double D = a.mu * m.alpha[f], Ff = a.F[f];
      diag += D + relu(-Ff);
      snb += D + relu(Ff);
    }
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) diag += a.mu * m.alpha_b[f] * a.bc.m_dirvel[f] + relu(a.Fb[f]);
    const double V = m.vol[c];
    if (a.por) diag += a.por[c] * V;
    const double denom = a.simplec ? diag / a.relax_u - snb : diag / a.relax_u;
    a.work[c] = V / denom;
    a.work[3 * (int64_t)nc + c] = diag;
  }
  // dP of every cell is needed by the neighbours' faces below: a second sweep after a grid-wide
  // dependency is done by the caller's second launch; here only per-cell quantities.
  (void)nf;
  (void)nb;
}

// Sensitivities of the residual to dP_c, then to a_P and sum a_nb of cell c.
template <int DIM>
__global__ void vjp_pass2_k(VjpArgs a) {
  const b2s_mesh& m = a.m;
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  const double* dP = a.work;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    double adP = 0.0;
    auto face_x = [&](int f) {
      const int P = m.fP[f], N = m.fN[f];
      const double w = m.w[f];
      double gd = 0.0;
#pragma unroll
      for (int q = 0; q < DIM; ++q)
        gd += (w * a.g[(int64_t)q * nc + P] + (1.0 - w) * a.g[(int64_t)q * nc + N]) * m.d[(int64_t)q * nf + f];
      return a.p[N] - a.p[P] - gd;
    };
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) adP += a.lF[f] * a.rho * m.w[f] * m.alpha[f] * face_x(f);
    for (int k = m.nei_ptr[c]; k < m.nei_ptr[c + 1]; ++k) {
      const int f = m.nei_face[k];
      adP += a.lF[f] * a.rho * (1.0 - m.w[f]) * m.alpha[f] * face_x(f);
    }
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      double gd = 0.0;
#pragma unroll
      for (int q = 0; q < DIM; ++q) gd += a.g[(int64_t)q * nc + c] * m.db[(int64_t)q * nb + f];
      adP += a.lFb[f] * a.bc.m_pres[f] * a.rho * m.alpha_b[f] * (a.bc.pb_fixed[f] - a.p[c] - gd);
    }
    const double V = m.vol[c], dPc = dP[c];
    const double denom = V / dPc;
    const double aden = -adP * V / (denom * denom);
    double adiag = aden / a.relax_u;
#pragma unroll
    for (int k = 0; k < DIM; ++k) adiag -= a.lm[(int64_t)k * nc + c] * a.U[(int64_t)k * nc + c];
    a.work[(int64_t)nc + c] = adiag;
    a.work[2 * (int64_t)nc + c] = a.simplec ? -aden : 0.0;
  }
}

// Every output of cell c, of the faces it owns and of its boundary faces.
template <int DIM>
__global__ void vjp_pass3_k(VjpArgs a) {
  const b2s_mesh& m = a.m;
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  const double* dP = a.work;
  const double* adiag = a.work + nc;
  const double* asnb = a.work + 2 * (int64_t)nc;
  const double* diag = a.work + 3 * (int64_t)nc;
  const double rho = a.rho;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    const double V = m.vol[c];
    double gU[DIM], gg[DIM], gp = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      gU[k] = -diag[c] * a.lm[(int64_t)k * nc + c];
      gg[k] = a.lg[(int64_t)k * nc + c] - V * a.lm[(int64_t)k * nc + c];
    }
    // owned faces: c = P
    for (int f = m.own_ptr[c]; f < m.own_ptr[c + 1]; ++f) {
      const int N = m.fN[f];
      const double w = m.w[f], D = a.mu * m.alpha[f], Ff = a.F[f], lF = a.lF[f];
      const double aNP = -(D + relu(Ff));
      const double dF = w * dP[c] + (1.0 - w) * dP[N];
      const double cf = rho * dF * m.alpha[f];
      double sUN = 0.0, sUP = 0.0, Sl = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        const double Sk = m.S[(int64_t)k * nf + f];
        gU[k] += -aNP * a.lm[(int64_t)k * nc + N] - rho * w * Sk * lF;
        gg[k] += -cf * w * m.d[(int64_t)k * nf + f] * lF;
        sUN += a.lm[(int64_t)k * nc + c] * a.U[(int64_t)k * nc + N];
        sUP += a.lm[(int64_t)k * nc + N] * a.U[(int64_t)k * nc + c];
        Sl += Sk * (-a.lg[(int64_t)k * nc + c] / V + a.lg[(int64_t)k * nc + N] / m.vol[N]);
      }
      gp += w * Sl - cf * lF;
      // the face's own output
      double oF = lF;
      oF += adiag[c] * drelu(Ff) - adiag[N] * drelu(-Ff);
      oF += -asnb[c] * drelu(-Ff) + asnb[N] * drelu(Ff);
      oF += -drelu(-Ff) * sUN + drelu(Ff) * sUP;
      oF += a.lc[c] - a.lc[N];
      a.oF[f] = oF;
    }
    // neighbour faces: c = N
    for (int k2 = m.nei_ptr[c]; k2 < m.nei_ptr[c + 1]; ++k2) {
      const int f = m.nei_face[k2];
      const int P = m.fP[f];
      const double w = m.w[f], D = a.mu * m.alpha[f], Ff = a.F[f], lF = a.lF[f];
      const double aPN = -(D + relu(-Ff));
      const double dF = w * dP[P] + (1.0 - w) * dP[c];
      const double cf = rho * dF * m.alpha[f];
      double Sl = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        const double Sk = m.S[(int64_t)k * nf + f];
        gU[k] += -aPN * a.lm[(int64_t)k * nc + P] - rho * (1.0 - w) * Sk * lF;
        gg[k] += -cf * (1.0 - w) * m.d[(int64_t)k * nf + f] * lF;
        Sl += Sk * (-a.lg[(int64_t)k * nc + P] / m.vol[P] + a.lg[(int64_t)k * nc + c] / V);
      }
      gp += (1.0 - w) * Sl + cf * lF;
    }
    // boundary faces
    for (int f = m.bptr[c]; f < m.bptr[c + 1]; ++f) {
      const double mp = a.bc.m_pres[f], mfix = a.bc.m_wall[f] + a.bc.m_inlet[f];
      const double Db = a.mu * m.alpha_b[f] * a.bc.m_dirvel[f], Fbf = a.Fb[f], lFb = a.lFb[f];
      const double cb = rho * dP[c] * m.alpha_b[f] * mp;
      const double coef = Db + relu(-Fbf);
      double Sl = 0.0, su = 0.0;
#pragma unroll
      for (int k = 0; k < DIM; ++k) {
        const double Sbk = m.Sb[(int64_t)k * nb + f];
        const double lmk = a.lm[(int64_t)k * nc + c];
        gU[k] += mp * coef * lmk - mp * rho * Sbk * lFb;
        gg[k] += -cb * m.db[(int64_t)k * nb + f] * lFb;
        Sl += Sbk * a.lg[(int64_t)k * nc + c];
        const double ubk = mfix * a.bc.ub_fixed[(int64_t)k * nb + f] + mp * a.U[(int64_t)k * nc + c];
        su += lmk * ubk;
        if (a.oub) a.oub[(int64_t)k * nb + f] = mfix * coef * lmk - a.bc.m_inlet[f] * rho * Sbk * lFb;
      }
      // p_b = p_P + g_P . d_b off pressure faces
      gp += -(1.0 - mp) * Sl / V - cb * lFb;
#pragma unroll
      for (int k = 0; k < DIM; ++k) gg[k] += -(1.0 - mp) * m.db[(int64_t)k * nb + f] * Sl / V;
      a.oFb[f] = lFb + adiag[c] * drelu(Fbf) - drelu(-Fbf) * su + a.lc[c];
    }
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
      a.oU[(int64_t)k * nc + c] = gU[k];
      a.og[(int64_t)k * nc + c] = gg[k];
    }
    a.op[c] = gp;
    if (a.opor) a.opor[c] = adiag[c] * V;
  }
}

}  // namespace b2s

using namespace b2s;

extern "C" {

int b2s_residual_vjp_d(const b2s_mesh* m, const b2s_bc* bc, double rho, double mu, double relax_u, int simplec,
                       const double* U, const double* p, const double* g, const double* F, const double* Fb,
                       const double* porosity, const double* lm, const double* lc, const double* lg,
                       const double* lF, const double* lFb, double* work, double* oU, double* op, double* og,
                       double* oF, double* oFb, double* opor, double* oub, b2s_stream_t s) {
  if (!m || !bc || m->nc <= 0 || (m->dim != 2 && m->dim != 3) || !U || !p || !g || (!F && m->nf) ||
      (!Fb && m->nb) || !lm || !lc || !lg || (!lF && m->nf) || (!lFb && m->nb) || !work || !oU || !op || !og ||
      (!oF && m->nf) || (!oFb && m->nb) || !(relax_u > 0.0))
    return B2S_ERR_ARG;
  VjpArgs a;
  a.m = *m;
  a.bc = *bc;
  a.rho = rho;
  a.mu = mu;
  a.relax_u = relax_u;
  a.simplec = simplec ? 1 : 0;
  a.U = U;
  a.p = p;
  a.g = g;
  a.F = F;
  a.Fb = Fb;
  a.por = porosity;
  a.lm = lm;
  a.lc = lc;
  a.lg = lg;
  a.lF = lF;
  a.lFb = lFb;
  a.work = work;
  a.oU = oU;
  a.op = op;
  a.og = og;
  a.oF = oF;
  a.oFb = oFb;
  a.opor = opor;
  a.oub = oub;
  const unsigned grid = grid_for(m->nc);
  cudaStream_t st = (cudaStream_t)s;
  if (m->dim == 2) {
    vjp_pass1_k<2><<<grid, kThreads, 0, st>>>(a);
    vjp_pass2_k<2><<<grid, kThreads, 0, st>>>(a);
    vjp_pass3_k<2><<<grid, kThreads, 0, st>>>(a);
  } else {
    vjp_pass1_k<3><<<grid, kThreads, 0, st>>>(a);
    vjp_pass2_k<3><<<grid, kThreads, 0, st>>>(a);
    vjp_pass3_k<3><<<grid, kThreads, 0, st>>>(a);
  }
  B2S_LAUNCH_CHECK();
  return B2S_OK;
}

}  // extern "C"
