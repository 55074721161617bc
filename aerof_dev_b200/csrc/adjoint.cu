// adjoint.cu -- exact linearisation of the second-order residual.
//
// Forward mode (aerof_gpu_jvp, aerof_gpu_dRdX): the residual pipeline run in
// dual numbers, so the derivative follows the primal arithmetic branch for
// branch (van Albada's a*b sign tests, the Roe upwind side, the
// Steger-Warming eigenvalue clipping), like the reference's hand-derived
// routines (Edge.C:1493-1573, RecFcn.h:451-476, g_roeflux*.f,
// g_boundflux5.f) do.  Geometry (normals, volumes, least-squares factors)
// is recomputed in dual numbers from X + eps Xdot.
//
// Reverse mode (aerof_gpu_vjp, aerof_gpu_dRdX_T): hand-written adjoints of
// the same kernels, recomputing the primal state per edge instead of
// storing it, accumulated per node by gathers in a fixed order.
#include <vector>

#include "common.cuh"
#include "physics.cuh"

namespace aerof {

constexpr int kAB = 256;


__global__ void k_d_seed(int N, Gas g, const double* __restrict__ U, const double* __restrict__ v,
                         const double* __restrict__ X, const double* __restrict__ Xdot, Dual* __restrict__ XD,
                         Dual* __restrict__ PD) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  Dual u[5], V[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = Dual(U[5 * (size_t)i + k], v ? v[5 * (size_t)i + k] : 0.0);
  cons2prim(g, u, V);
#pragma unroll
  for (int k = 0; k < 5; ++k) PD[8 * (size_t)i + k] = V[k];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Dual x(X[3 * (size_t)i + k], Xdot ? Xdot[3 * (size_t)i + k] : 0.0);
    XD[3 * (size_t)i + k] = x;
    PD[8 * (size_t)i + 5 + k] = x;
  }
}

// per-node least-squares constants (SubDomain.C:137-159), dual
__global__ void k_d_lsqW(int N, const Dual* __restrict__ R, Dual* __restrict__ W) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  Dual r[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) r[k] = R[(size_t)k * N + i];
  Dual or11 = 1.0 / r[0], or22 = 1.0 / r[3], or33 = 1.0 / r[5];
  W[i] = or11;
  W[(size_t)N + i] = or22;
  W[2 * (size_t)N + i] = or33;
  W[3 * (size_t)N + i] = r[1] * or11;
  W[4 * (size_t)N + i] = r[4] * or22;
  W[5 * (size_t)N + i] = (r[1] * r[4] - r[2] * r[3]) * or11 * or22;
}

__global__ void k_d_grad(int N, const Dual* __restrict__ P, const Dual* __restrict__ lsqW,
                         const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_node, Dual* __restrict__ G) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  Dual w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = lsqW[(size_t)k * N + i];
  const Dual* pi = P + 8 * (size_t)i;
  Dual gx[5], gy[5], gz[5];
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const Dual* pj = P + 8 * (size_t)nbr_node[p];
    Dual W0, W1, W2;
    lsq_weights(w, pj[5] - pi[5], pj[6] - pi[6], pj[7] - pi[7], W0, W1, W2);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      Dual dv = pj[k] - pi[k];
      gx[k] += W0 * dv;
      gy[k] += W1 * dv;
      gz[k] += W2 * dv;
    }
  }
  Dual* gi = G + 15 * (size_t)i;
#pragma unroll
  for (int k = 0; k < 5; ++k) { gi[k] = gx[k]; gi[5 + k] = gy[k]; gi[10 + k] = gz[k]; }
}

__global__ void k_d_edge_flux(int E, Gas g, int rec, double beta, const int2* __restrict__ edges,
                              const Dual* __restrict__ en, const Dual* __restrict__ P, const Dual* __restrict__ G,
                              Dual* __restrict__ flux, int* __restrict__ counters) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
  const int2 ij = edges[l];
  const Dual* pi = P + 8 * (size_t)ij.x;
  const Dual* pj = P + 8 * (size_t)ij.y;
  Dual Vi[5], Vj[5];
  if (rec == AEROF_REC_CONSTANT) {
#pragma unroll
    for (int k = 0; k < 5; ++k) { Vi[k] = pi[k]; Vj[k] = pj[k]; }
  } else {
    Dual dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
    const Dual* gi = G + 15 * (size_t)ij.x;
    const Dual* gj = G + 15 * (size_t)ij.y;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      Dual ddVij = dx0 * gi[k] + dx1 * gi[5 + k] + dx2 * gi[10 + k];
      Dual ddVji = dx0 * gj[k] + dx1 * gj[5 + k] + dx2 * gj[10 + k];
      if (rec == AEROF_REC_VANALBADA) vanalbada(beta, pi[k], ddVij, pj[k], ddVji, Vi[k], Vj[k]);
      else linear_rec(beta, pi[k], ddVij, pj[k], ddVji, Vi[k], Vj[k]);
    }
  }
  Dual f[5];
  const bool bad = Vi[0].v <= 0.0 || Vi[4].v <= 0.0 || Vj[0].v <= 0.0 || Vj[4].v <= 0.0;
  if (bad) {
    atomicAdd(&counters[0], 1);
  } else {
    Dual n0 = en[l], n1 = en[(size_t)E + l], n2 = en[2 * (size_t)E + l];
    if (sqrt(n0.v * n0.v + n1.v * n1.v + n2.v * n2.v) >= 1e-18) roe_flux(g, n0, n1, n2, Vi, Vj, f);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) flux[(size_t)k * E + l] = f[k];
}

__global__ void k_d_node_residual(int N, int E, int F, Gas g, const double* __restrict__ Ub0,
                                  const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                                  const Dual* __restrict__ flux, const int* __restrict__ nf_ptr,
                                  const int* __restrict__ nf_face, const int* __restrict__ fcode,
                                  const Dual* __restrict__ fn, const Dual* __restrict__ P,
                                  const Dual* __restrict__ vol, double* __restrict__ dR, double* __restrict__ R) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  Dual acc[5];
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const int e = nbr_edge[p];
    const size_t l = (size_t)(e & 0x7fffffff);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      if (e < 0) acc[k] -= flux[k * (size_t)E + l];
      else acc[k] += flux[k * (size_t)E + l];
    }
  }
  if (nf_ptr[i] < nf_ptr[i + 1]) {
    Dual V[5];
    double Ub[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { V[k] = P[8 * (size_t)i + k]; Ub[k] = Ub0[k]; }
    const double third = 1.0 / 3.0;
    for (int q = nf_ptr[i]; q < nf_ptr[i + 1]; ++q) {
      const int f = nf_face[q];
      Dual ff[5];
      face_flux(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, ff);
#pragma unroll
      for (int k = 0; k < 5; ++k) acc[k] += ff[k];
    }
  }
  Dual invcv = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    Dual r = acc[k] * invcv;
    dR[5 * (size_t)i + k] = r.d;
    if (R) R[5 * (size_t)i + k] = r.v;
  }
}

// Forward-mode residual: tangent of R at (U + eps v, X + eps Xdot) into dR.
int residual_forward(aerof_gpu_ctx* c, const double* dU, const double* dv, const double* dXdot, double* ddR) {
  DeviceMesh& m = c->mesh;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  DualWork& w = c->dual;
  w.XD.ensure(3 * (size_t)m.N); w.PD.ensure(8 * (size_t)m.N); w.GD.ensure(15 * (size_t)m.N);
  w.WD.ensure(6 * (size_t)m.N); w.RD.ensure(6 * (size_t)m.N); w.volD.ensure(m.N);
  w.enD.ensure(3 * (size_t)m.E); w.fnD.ensure(3 * (size_t)std::max(m.F, 1)); w.fluxD.ensure(5 * (size_t)m.E);
  const int gn = grid_for(m.N, kAB), ge = grid_for(m.E, kAB);
  k_d_seed<<<gn, kAB, 0, s>>>(m.N, g, dU, dv, m.X.p, dXdot, w.XD.p, w.PD.p);
  AEROF_LAUNCH_CHECK();
  geometry_dual(c, w.XD.p, w.volD.p, w.enD.p, w.fnD.p, w.RD.p);
  const int rec = c->cfg.reconstruction;
  if (rec != AEROF_REC_CONSTANT) {
    k_d_lsqW<<<gn, kAB, 0, s>>>(m.N, w.RD.p, w.WD.p);
    AEROF_LAUNCH_CHECK();
    k_d_grad<<<gn, kAB, 0, s>>>(m.N, w.PD.p, w.WD.p, m.nbr_ptr.p, m.nbr_node.p, w.GD.p);
    AEROF_LAUNCH_CHECK();
  }
  c->s.counters.ensure(8);
  int* cnt = c->s.counters.p + 6;
  AEROF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
  k_d_edge_flux<<<ge, kAB, 0, s>>>(m.E, g, rec, c->cfg.beta, m.edges.p, w.enD.p, w.PD.p, w.GD.p, w.fluxD.p, cnt);
  AEROF_LAUNCH_CHECK();
  k_d_node_residual<<<gn, kAB, 0, s>>>(m.N, m.E, m.F, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_edge.p, w.fluxD.p, m.nf_ptr.p,
                                       m.nf_face.p, m.fcode.p, w.fnD.p, w.PD.p, w.volD.p, ddR, nullptr);
  AEROF_LAUNCH_CHECK();
  int bad = 0;
  AEROF_CUDA(cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
  AEROF_CUDA(cudaStreamSynchronize(s));
  return bad;
}

}  // namespace aerof
