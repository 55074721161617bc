// viscous.cu -- the laminar Navier-Stokes Galerkin term on tets
// (SpaceOperator::computeResidual adds it before the finite-volume term,
// SpaceOperator.C:570-573): ElemTet::computeGalerkinTerm (ElemTet.C:24-127)
// with FemEquationTermNS::computeVolumeTerm (FemEquationTermDesc.C:98-160),
// NavierStokesTerm (NavierStokesTerm.h:205-724), ViscoFcn (constant or
// Sutherland, ViscoFcn.h:46-103), constant-Prandtl conductivity
// (ThermalCondFcn.h:52-75).
//
// One thread per node walks the node's tets in ascending tet order (the
// order in which the reference's element loop adds into the node) and, per
// tet, recomputes the P1 shape-function gradients from the coordinates
// (ElemTet::computeGradientP1Function, ElemTetCore.C:1961-2010), the
// velocity and temperature gradients, the transport coefficients at the
// tet's mean temperature, the stress tensor and heat flux, and the node's
// share vol (r_0 dN_x + r_1 dN_y + r_2 dN_z); the sum, divided by the
// control volume, is added to R.  Deterministic (a gather, no atomics) and
// allocation-free; each tet is evaluated by its four nodes.
#include "common.cuh"
#include "physics.cuh"

namespace aerof {

struct ViscDev {
  int model;
  double ooreynolds, ooprandtl, bulk, alpha, Ts;
};

__device__ __forceinline__ double p1_grad(const double* __restrict__ X, const int* nd, double g[4][3]) {
  double x[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int a = 0; a < 3; ++a) x[k][a] = X[3 * (size_t)nd[k] + a];
  double jac[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    jac[a][0] = x[1][a] - x[0][a];
    jac[a][1] = x[2][a] - x[0][a];
    jac[a][2] = x[3][a] - x[0][a];
  }
  const double dOmega = jac[0][0] * (jac[1][1] * jac[2][2] - jac[1][2] * jac[2][1]) +
                        jac[1][0] * (jac[0][2] * jac[2][1] - jac[0][1] * jac[2][2]) +
                        jac[2][0] * (jac[0][1] * jac[1][2] - jac[0][2] * jac[1][1]);
  const double t17 = -1.0 / dOmega;
  g[1][0] = (-jac[1][1] * jac[2][2] + jac[1][2] * jac[2][1]) * t17;
  g[1][1] = (jac[0][1] * jac[2][2] - jac[0][2] * jac[2][1]) * t17;
  g[1][2] = -(jac[0][1] * jac[1][2] - jac[0][2] * jac[1][1]) * t17;
  g[2][0] = -(-jac[1][0] * jac[2][2] + jac[1][2] * jac[2][0]) * t17;
  g[2][1] = -(jac[0][0] * jac[2][2] - jac[0][2] * jac[2][0]) * t17;
  g[2][2] = (jac[0][0] * jac[1][2] - jac[0][2] * jac[1][0]) * t17;
  g[3][0] = -(jac[1][0] * jac[2][1] - jac[1][1] * jac[2][0]) * t17;
  g[3][1] = (jac[0][0] * jac[2][1] - jac[0][1] * jac[2][0]) * t17;
  g[3][2] = -(jac[0][0] * jac[1][1] - jac[0][1] * jac[1][0]) * t17;
#pragma unroll
  for (int a = 0; a < 3; ++a) g[0][a] = -(g[1][a] + g[2][a] + g[3][a]);
  return (1.0 / 6.0) * dOmega;
}

// R[i] += (sum over the node's tets of its Galerkin share) / vol[i];
// P: node records (V, X) in caller numbering
__global__ void k_galerkin_nodes(int N, Gas gs, ViscDev vp, const double* __restrict__ X,
                                 const int* __restrict__ tets, const int* __restrict__ nt_ptr,
                                 const int* __restrict__ nt_tet, const double* __restrict__ P,
                                 const double* __restrict__ vol, double* __restrict__ R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double invgam1 = gs.invgam1, cp = gs.gam * gs.invgam1;
  const double twothird = 2.0 / 3.0;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int q = nt_ptr[i]; q < nt_ptr[i + 1]; ++q) {
    const int tl = nt_tet[q];
    const int t = tl >> 2, kj = tl & 3;
    int nd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) nd[k] = tets[4 * (size_t)t + k];
    double g[4][3];
    const double tv = p1_grad(X, nd, g);
    double u[4][3], T[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double* v = P + 8 * (size_t)nd[k];
      u[k][0] = v[1]; u[k][1] = v[2]; u[k][2] = v[3];
      T[k] = invgam1 * v[4] / v[0];
    }
    double ucg[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ucg[a] = 0.25 * (u[0][a] + u[1][a] + u[2][a] + u[3][a]);
    const double Tcg = 0.25 * (T[0] + T[1] + T[2] + T[3]);
    double du[3][3], dT[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int j = 0; j < 3; ++j) du[a][j] = g[0][j] * u[0][a] + g[1][j] * u[1][a] + g[2][j] * u[2][a] + g[3][j] * u[3][a];
#pragma unroll
    for (int j = 0; j < 3; ++j) dT[j] = g[0][j] * T[0] + g[1][j] * T[1] + g[2][j] * T[2] + g[3][j] * T[3];
    double mu, lambda;
    if (vp.model == 2) {
      const double Ta = vp.alpha * Tcg;
      mu = Ta * sqrt(Ta) * (1.0 + vp.Ts) / (Ta + vp.Ts);
      lambda = -twothird * mu;
    } else {
      mu = 1.0;
      lambda = vp.bulk - twothird * mu;
    }
    double kappa = vp.ooprandtl * cp * mu;
    mu *= vp.ooreynolds;
    lambda *= vp.ooreynolds;
    kappa *= vp.ooreynolds;
    const double div = du[0][0] + du[1][1] + du[2][2];
    double tij[3][3];
    tij[0][0] = lambda * div + 2.0 * mu * du[0][0];
    tij[1][1] = lambda * div + 2.0 * mu * du[1][1];
    tij[2][2] = lambda * div + 2.0 * mu * du[2][2];
    tij[0][1] = mu * (du[1][0] + du[0][1]);
    tij[0][2] = mu * (du[2][0] + du[0][2]);
    tij[1][2] = mu * (du[2][1] + du[1][2]);
    tij[1][0] = tij[0][1];
    tij[2][0] = tij[0][2];
    tij[2][1] = tij[1][2];
    double r[3][5];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r[j][0] = 0.0;
      r[j][1] = tij[0][j];
      r[j][2] = tij[1][j];
      r[j][3] = tij[2][j];
      r[j][4] = ucg[0] * tij[0][j] + ucg[1] * tij[1][j] + ucg[2] * tij[2][j] - (-kappa * dT[j]);
    }
    double gk[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) gk[a] = kj == 0 ? g[0][a] : kj == 1 ? g[1][a] : kj == 2 ? g[2][a] : g[3][a];
#pragma unroll
    for (int k = 0; k < 5; ++k) acc[k] += tv * (r[0][k] * gk[0] + r[1][k] * gk[1] + r[2][k] * gk[2]);
  }
  const double iv = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) R[5 * (size_t)i + k] += acc[k] * iv;
}

// k_prim is defined in residual.cu; a local copy keeps the node records of
// caller numbering current for the viscous term
__global__ void k_prim_visc(int N, Gas g, const double* __restrict__ U, double* __restrict__ P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)i + k];
  cons2prim(g, u, v);
#pragma unroll
  for (int k = 0; k < 5; ++k) P[8 * (size_t)i + k] = v[k];
}

// R += G(U) / vol (R already holds the finite-volume residual divided by
// the control volumes); no allocation
void galerkin_add(aerof_gpu_ctx* c, const double* dU, double* dR) {
  if (c->visc.model == 0) return;
  DeviceMesh& m = c->mesh;
  const Gas g = make_gas(c->cfg.gamma);
  ViscDev vp{c->visc.model, 1.0 / c->visc.reynolds_mu, 1.0 / c->visc.prandtl, c->visc.bulk_viscosity,
             c->visc.sutherland_alpha, c->visc.sutherland_Ts};
  k_prim_visc<<<grid_for(m.N, 256), 256, 0, c->stream>>>(m.N, g, dU, m.P.p);
  AEROF_LAUNCH_CHECK();
  k_galerkin_nodes<<<grid_for(m.N, 128), 128, 0, c->stream>>>(m.N, g, vp, m.X.p, m.tets.p, m.nt_ptr.p, m.nt_tet.p,
                                                             m.P.p, m.vol.p, dR);
  AEROF_LAUNCH_CHECK();
}

}  // namespace aerof

using namespace aerof;

extern "C" int aerof_gpu_set_viscosity(aerof_gpu_ctx* c, const aerof_viscous_params* p) {
  return guard(c, [&]() -> int {
    if (!p || p->model < 0 || p->model > 2) return AEROF_EINVAL;
    if (p->model != 0 && !(p->reynolds_mu > 0.0 && p->prandtl > 0.0)) return AEROF_EINVAL;
    if (p->model == 2 && !(p->sutherland_alpha > 0.0 && p->sutherland_Ts >= 0.0)) return AEROF_EINVAL;
    c->visc = *p;
    c->imp.precision = 0;
    c->h2.ready = false;
    return AEROF_OK;
  });
}
