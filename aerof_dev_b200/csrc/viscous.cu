// viscous.cu -- the laminar Navier-Stokes Galerkin term on tets
// (SpaceOperator::computeResidual adds it before the finite-volume term,
// SpaceOperator.C:570-573): ElemTet::computeGalerkinTerm (ElemTet.C:24-127)
// with FemEquationTermNS::computeVolumeTerm (FemEquationTermDesc.C:98-160),
// NavierStokesTerm (NavierStokesTerm.h:205-724), ViscoFcn (constant or
// Sutherland, ViscoFcn.h:46-103), constant-Prandtl conductivity
// (ThermalCondFcn.h:52-75).
//
// One thread per tet computes the P1 shape-function gradients from the
// coordinates (ElemTet::computeGradientP1Function, ElemTetCore.C:1961-2010),
// the velocity and temperature gradients, the transport coefficients at the
// tet's mean temperature, the stress tensor and heat flux, and each of its
// four nodes' shares vol (r_0 dN_x + r_1 dN_y + r_2 dN_z), stored per
// (tet, vertex).  A gather then sums each node's shares in ascending tet
// order (the order in which the reference's element loop adds into the
// node) and adds the sum divided by the control volume to R.  Deterministic
// (no atomics); the per-tet buffer is reserved at set-up, so a residual
// call allocates nothing.
#include "common.cuh"
#include "physics.cuh"

namespace aerof {

struct ViscDev {
  int model;
  double ooreynolds, ooprandtl, bulk, alpha, Ts;
};

__device__ __forceinline__ double p1_grad(const double x[4][3], double g[4][3]) {
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

// One thread per tet: node k's share of the tet's Galerkin term,
// vol (r_1..4 . dN_k) (component 0 of r is zero), written as the record
// C[4 (4t + k) .. +3].  The block's records are staged in shared memory
// (row stride 17 doubles: conflict-free) and stored contiguously with
// evict-first stores (each record is read once, by k_tet_gather).
// Q: per-node records (u, v, w, T, x, y, z, 0) of k_visc_records
template <int TB>
__global__ void __launch_bounds__(TB) k_galerkin_tets(int T, Gas gs, ViscDev vp, const int* __restrict__ tets,
                                                      const double* __restrict__ Q, double* __restrict__ C) {
  constexpr int REC = 16, RS = REC + 1;
  __shared__ double st[TB * RS];
  const int t0 = blockIdx.x * TB, t = t0 + threadIdx.x;
  if (t < T) {
    const double cp = gs.gam * gs.invgam1;
    const double twothird = 2.0 / 3.0;
    const int4 q4 = *reinterpret_cast<const int4*>(tets + 4 * (size_t)t);
    const int nd[4] = {q4.x, q4.y, q4.z, q4.w};
    double u[4][3], Tn[4], x[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2* q = reinterpret_cast<const double2*>(Q + 8 * (size_t)nd[k]);
      const double2 a = q[0], b = q[1], c = q[2], d = q[3];
      u[k][0] = a.x; u[k][1] = a.y; u[k][2] = b.x; Tn[k] = b.y;
      x[k][0] = c.x; x[k][1] = c.y; x[k][2] = d.x;
    }
    double g[4][3];
    const double tv = p1_grad(x, g);
    double ucg[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ucg[a] = 0.25 * (u[0][a] + u[1][a] + u[2][a] + u[3][a]);
    const double Tcg = 0.25 * (Tn[0] + Tn[1] + Tn[2] + Tn[3]);
    double du[3][3], dT[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int j = 0; j < 3; ++j) du[a][j] = g[0][j] * u[0][a] + g[1][j] * u[1][a] + g[2][j] * u[2][a] + g[3][j] * u[3][a];
#pragma unroll
    for (int j = 0; j < 3; ++j) dT[j] = g[0][j] * Tn[0] + g[1][j] * Tn[1] + g[2][j] * Tn[2] + g[3][j] * Tn[3];
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
    double r[3][4];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      r[j][0] = tij[0][j];
      r[j][1] = tij[1][j];
      r[j][2] = tij[2][j];
      r[j][3] = ucg[0] * tij[0][j] + ucg[1] * tij[1][j] + ucg[2] * tij[2][j] - (-kappa * dT[j]);
    }
    double* row = st + threadIdx.x * RS;
#pragma unroll
    for (int kj = 0; kj < 4; ++kj)
#pragma unroll
      for (int k = 0; k < 4; ++k) row[4 * kj + k] = tv * (r[0][k] * g[kj][0] + r[1][k] * g[kj][1] + r[2][k] * g[kj][2]);
  }
  __syncthreads();
  const int cnt = min(TB, T - t0) * REC;
  double* out = C + (size_t)t0 * REC;
  for (int f = threadIdx.x; f < cnt; f += TB) __stcs(out + f, st[(f / REC) * RS + (f % REC)]);
}

// Per-node records of the Galerkin term: (u, v, w, T, x, y, z, 0) with
// T = p / ((gamma - 1) rho) from VarFcnSGEuler::conservativeToPrimitive,
// formed once per node instead of once per (tet, vertex)
__global__ void k_visc_records(int N, Gas g, const double* __restrict__ U, const double* __restrict__ X,
                               double* __restrict__ Q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)i + k];
  cons2prim(g, u, v);
  double2* q = reinterpret_cast<double2*>(Q + 8 * (size_t)i);
  q[0] = make_double2(v[1], v[2]);
  q[1] = make_double2(v[3], g.invgam1 * v[4] / v[0]);
  q[2] = make_double2(X[3 * (size_t)i], X[3 * (size_t)i + 1]);
  q[3] = make_double2(X[3 * (size_t)i + 2], 0.0);
}

// the per-tet buffer of the Galerkin term, sized at set-up so that the
// residual calls allocate nothing
void galerkin_reserve(aerof_gpu_ctx* c, int model) {
  if (model == 0 || !c->has_mesh) return;
  c->s.tetc.ensure(16 * (size_t)std::max(c->mesh.T, 1));
  c->s.viscq.ensure(8 * (size_t)c->mesh.N);
}

// R += G(U) / vol (R already holds the finite-volume residual divided by
// the control volumes): each tet evaluated once (k_galerkin_tets), then
// each node sums its tets' shares in ascending tet order (k_tet_gather)
void galerkin_add(aerof_gpu_ctx* c, const double* dU, double* dR) {
  if (c->visc.model == 0) return;
  DeviceMesh& m = c->mesh;
  if (c->s.tetc.n < 16 * (size_t)m.T || c->s.viscq.n < 8 * (size_t)m.N)
    throw ApiError{AEROF_ESTATE, "viscous term: per-tet buffer not reserved"};
  const Gas g = make_gas(c->cfg.gamma);
  ViscDev vp{c->visc.model, 1.0 / c->visc.reynolds_mu, 1.0 / c->visc.prandtl, c->visc.bulk_viscosity,
             c->visc.sutherland_alpha, c->visc.sutherland_Ts};
  k_visc_records<<<grid_for(m.N, 256), 256, 0, c->stream>>>(m.N, g, dU, m.X.p, c->s.viscq.p);
  AEROF_LAUNCH_CHECK();
  if (m.T) {
    k_galerkin_tets<128><<<grid_for(m.T, 128), 128, 0, c->stream>>>(m.T, g, vp, m.tets.p, c->s.viscq.p, c->s.tetc.p);
    AEROF_LAUNCH_CHECK();
  }
  k_tet_gather<4, 5, 1><<<grid_for(4 * (size_t)m.N, 256), 256, 0, c->stream>>>(m.N, m.nt_ptr.p, m.nt_tet.p,
                                                                                c->s.tetc.p, m.vol.p, dR);
  AEROF_LAUNCH_CHECK();
}

}  // namespace aerof

using namespace aerof;

extern "C" int aerof_gpu_set_viscosity(aerof_gpu_ctx* c, const aerof_viscous_params* p) {
  return guard(c, [&]() -> int {
    if (!p || p->model < 0 || p->model > 2) return AEROF_EINVAL;
    if (p->model != 0 && !(p->reynolds_mu > 0.0 && p->prandtl > 0.0)) return AEROF_EINVAL;
    if (p->model == 2 && !(p->sutherland_alpha > 0.0 && p->sutherland_Ts >= 0.0)) return AEROF_EINVAL;
    // the buffers first: a failed reservation leaves the previous model set
    galerkin_reserve(c, p->model);
    c->visc = *p;
    c->imp.precision = 0;
    c->h2.ready = false;
    return AEROF_OK;
  });
}
