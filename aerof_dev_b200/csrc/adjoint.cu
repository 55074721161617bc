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
#include "geometry.cuh"

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
int residual_forward(aerof_gpu_ctx* c, const double* dU, const double* dv, const double* dXdot, double* ddR,
                     bool sync) {
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
  const int rec = c->cfg.reconstruction;
  // state-only tangents: the geometry (zero tangents) is reused between calls
  if (dXdot || !w.geom_static) {
    geometry_dual(c, w.XD.p, w.volD.p, w.enD.p, w.fnD.p, w.RD.p);
    k_d_lsqW<<<gn, kAB, 0, s>>>(m.N, w.RD.p, w.WD.p);
    AEROF_LAUNCH_CHECK();
    w.geom_static = (dXdot == nullptr);
  }
  if (rec != AEROF_REC_CONSTANT) {
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
  if (sync) {
    AEROF_CUDA(cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
  }
  return bad;
}

}  // namespace aerof

// ======================================================================
// Reverse mode.  Per-edge cotangents are written to a scratch record and
// gathered per node in the residual's neighbour order.
namespace aerof {


// lam[i] = w[i] / vol[i]: cotangent of the unscaled flux sum S_i (R = S/vol)
__global__ void k_a_lam(int N, const double* __restrict__ w, const double* __restrict__ vol, double* __restrict__ lam) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double iv = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) lam[5 * (size_t)i + k] = w[5 * (size_t)i + k] * iv;
}

// Edge adjoint: gF = lam_i - lam_j through the Roe flux and the
// reconstruction.  rec[l] (32 doubles): [0,5) gVi, [5,10) gVj, [10,15)
// gdd_ij, [15,20) gdd_ji, [20,23) g_normal, [23,26) g_dx.
__global__ void k_a_edges(int E, Gas g, int rec, double beta, const int2* __restrict__ edges,
                          const double* __restrict__ en, const double* __restrict__ P,
                          const double* __restrict__ G, const double* __restrict__ lam, double* __restrict__ out) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
  const int2 ij = edges[l];
  const double* pi = P + 8 * (size_t)ij.x;
  const double* pj = P + 8 * (size_t)ij.y;
  const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
  const double* gi = G + 16 * (size_t)ij.x;
  const double* gj = G + 16 * (size_t)ij.y;
  double Vi[5], Vj[5], ddij[5], ddji[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    if (rec == AEROF_REC_CONSTANT) {
      ddij[k] = ddji[k] = 0.0;
      Vi[k] = pi[k]; Vj[k] = pj[k];
    } else {
      ddij[k] = dx0 * gi[k] + dx1 * gi[5 + k] + dx2 * gi[10 + k];
      ddji[k] = dx0 * gj[k] + dx1 * gj[5 + k] + dx2 * gj[10 + k];
      if (rec == AEROF_REC_VANALBADA) vanalbada(beta, pi[k], ddij[k], pj[k], ddji[k], Vi[k], Vj[k]);
      else linear_rec(beta, pi[k], ddij[k], pj[k], ddji[k], Vi[k], Vj[k]);
    }
  }
  double gF[5], gL[5] = {0, 0, 0, 0, 0}, gR[5] = {0, 0, 0, 0, 0}, gn[3] = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < 5; ++k) gF[k] = lam[5 * (size_t)ij.x + k] - lam[5 * (size_t)ij.y + k];
  const double n0 = en[l], n1 = en[(size_t)E + l], n2 = en[2 * (size_t)E + l];
  if (sqrt(n0 * n0 + n1 * n1 + n2 * n2) >= 1e-18) roe_flux_adj(g, n0, n1, n2, Vi, Vj, gF, gL, gR, gn);
  double* o = out + 32 * (size_t)l;
  double gdx0 = 0.0, gdx1 = 0.0, gdx2 = 0.0;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double gvi = 0.0, gvj = 0.0, gdi, gdj;
    reconstruct_adj(rec, beta, pi[k], ddij[k], pj[k], ddji[k], gL[k], gR[k], gvi, gvj, gdi, gdj);
    o[k] = gvi;
    o[5 + k] = gvj;
    o[10 + k] = gdi;
    o[15 + k] = gdj;
    if (rec != AEROF_REC_CONSTANT) {
      gdx0 += gi[k] * gdi + gj[k] * gdj;
      gdx1 += gi[5 + k] * gdi + gj[5 + k] * gdj;
      gdx2 += gi[10 + k] * gdi + gj[10 + k] * gdj;
    }
  }
  o[20] = gn[0]; o[21] = gn[1]; o[22] = gn[2];
  o[23] = gdx0; o[24] = gdx1; o[25] = gdx2;
}

// Face flux cotangents by forward mode (5 state directions), g_V += J^T lam
__device__ void face_vjp_V(const Gas& g, int code, double nx, double ny, double nz, const double* V, const double* Ub,
                           const double* lam, double* gV) {
  for (int d = 0; d < 5; ++d) {
    Dual Vd[5], f[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Vd[k] = Dual(V[k], k == d ? 1.0 : 0.0);
    face_flux(g, code, Dual(nx), Dual(ny), Dual(nz), Vd, Ub, f);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += f[k].d * lam[k];
    gV[d] += s;
  }
}

// Per node: direct state cotangents (edges in neighbour order, faces),
// gradient cotangents g_grad_i = sum dx (x) gdd.
__global__ void k_a_node(int N, int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ nbr_ptr,
                         const int* __restrict__ nbr_node, const int* __restrict__ nbr_edge,
                         const double* __restrict__ erec, const int* __restrict__ nf_ptr,
                         const int* __restrict__ nf_face, const int* __restrict__ fcode, const double* __restrict__ fn,
                         const double* __restrict__ P, const double* __restrict__ lam, double* __restrict__ gV,
                         double* __restrict__ gG) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double gv[5] = {0, 0, 0, 0, 0}, gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
  const double* pi = P + 8 * (size_t)i;
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const int e = nbr_edge[p];
    const double* o = erec + 32 * (size_t)(e & 0x7fffffff);
    const double* pj = P + 8 * (size_t)nbr_node[p];
    // edge dx = X_second - X_first
    const double s = e < 0 ? -1.0 : 1.0;
    const double dx0 = s * (pj[5] - pi[5]), dx1 = s * (pj[6] - pi[6]), dx2 = s * (pj[7] - pi[7]);
    const double* gvs = e < 0 ? o + 5 : o;
    const double* gds = e < 0 ? o + 15 : o + 10;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      gv[k] += gvs[k];
      gx[k] += dx0 * gds[k];
      gy[k] += dx1 * gds[k];
      gz[k] += dx2 * gds[k];
    }
  }
  if (nf_ptr[i] < nf_ptr[i + 1]) {
    double V[5], Ub[5], lm[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { V[k] = pi[k]; Ub[k] = Ub0[k]; lm[k] = lam[5 * (size_t)i + k]; }
    const double third = 1.0 / 3.0;
    for (int q = nf_ptr[i]; q < nf_ptr[i + 1]; ++q) {
      const int f = nf_face[q];
      face_vjp_V(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, lm, gv);
    }
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    gV[5 * (size_t)i + k] = gv[k];
    gG[16 * (size_t)i + k] = gx[k];
    gG[16 * (size_t)i + 5 + k] = gy[k];
    gG[16 * (size_t)i + 10 + k] = gz[k];
  }
}

// Per node q: transpose of the least-squares gradient,
// g_V_q += sum_{i in nbr(q)} W_i(x_q - x_i) . g_grad_i - sum_{p} W_q(x_p - x_q) . g_grad_q,
// then (dV/dU)^T.
__global__ void k_a_lsq_prim(int N, Gas g, int rec, const double* __restrict__ U, const double* __restrict__ P,
                             const double* __restrict__ lsqW, const int* __restrict__ nbr_ptr,
                             const int* __restrict__ nbr_node, const double* __restrict__ gV,
                             const double* __restrict__ gG, double* __restrict__ out) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  double gv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) gv[k] = gV[5 * (size_t)q + k];
  if (rec != AEROF_REC_CONSTANT) {
    const double* pq = P + 8 * (size_t)q;
    double wq[6], Wsum0 = 0.0, Wsum1 = 0.0, Wsum2 = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) wq[k] = lsqW[(size_t)k * N + q];
    for (int p = nbr_ptr[q]; p < nbr_ptr[q + 1]; ++p) {
      const int i = nbr_node[p];
      const double* pi = P + 8 * (size_t)i;
      double wi[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) wi[k] = lsqW[(size_t)k * N + i];
      double W0, W1, W2;
      lsq_weights(wi, pq[5] - pi[5], pq[6] - pi[6], pq[7] - pi[7], W0, W1, W2);
      const double* gg = gG + 16 * (size_t)i;
#pragma unroll
      for (int k = 0; k < 5; ++k) gv[k] += W0 * gg[k] + W1 * gg[5 + k] + W2 * gg[10 + k];
      double V0, V1, V2;
      lsq_weights(wq, pi[5] - pq[5], pi[6] - pq[6], pi[7] - pq[7], V0, V1, V2);
      Wsum0 += V0; Wsum1 += V1; Wsum2 += V2;
    }
    const double* gq = gG + 16 * (size_t)q;
#pragma unroll
    for (int k = 0; k < 5; ++k) gv[k] -= Wsum0 * gq[k] + Wsum1 * gq[5 + k] + Wsum2 * gq[10 + k];
  }
  double u[5], gu[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)q + k];
  prim_adj(g, u, gv, gu);
#pragma unroll
  for (int k = 0; k < 5; ++k) out[5 * (size_t)q + k] = gu[k];
}

// J^T w for device state dU and cotangent dw, into dout ([N][5]).
void vjp_dev(aerof_gpu_ctx* c, const double* dU, const double* dw, double* dout) {
  DeviceMesh& m = c->mesh;
  AdjWork& a = c->adj;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const int rec = c->cfg.reconstruction;
  const int gn = grid_for(m.N, kAB), ge = grid_for(m.E, kAB);
  prim_dev(c, dU);
  c->s.G.ensure(16 * (size_t)m.N);
  if (rec != AEROF_REC_CONSTANT) gradients_dev(c);
  a.lam.ensure(5 * (size_t)m.N);
  a.edge.ensure(32 * (size_t)m.E);
  a.gV.ensure(5 * (size_t)m.N);
  a.gG.ensure(16 * (size_t)m.N);
  k_a_lam<<<gn, kAB, 0, s>>>(m.N, dw, m.vol.p, a.lam.p);
  AEROF_LAUNCH_CHECK();
  k_a_edges<<<ge, kAB, 0, s>>>(m.E, g, rec, c->cfg.beta, m.edges.p, m.en.p, m.P.p, c->s.G.p, a.lam.p, a.edge.p);
  AEROF_LAUNCH_CHECK();
  k_a_node<<<gn, kAB, 0, s>>>(m.N, m.F, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_node.p, m.nbr_edge.p, a.edge.p, m.nf_ptr.p,
                              m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, a.lam.p, a.gV.p, a.gG.p);
  AEROF_LAUNCH_CHECK();
  k_a_lsq_prim<<<gn, kAB, 0, s>>>(m.N, g, rec, dU, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p, a.gV.p, a.gG.p, dout);
  AEROF_LAUNCH_CHECK();
}

}  // namespace aerof

// ======================================================================
// (dR/dX)^T lambda.
namespace aerof {

// Face normal cotangent: g_fn_f = third * sum_l (d f/d n3)^T lam_{node l}
// (forward mode in the 3 normal directions).
__global__ void k_a_face_normal(int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ faces,
                                const int* __restrict__ fcode, const double* __restrict__ fn,
                                const double* __restrict__ P, const double* __restrict__ lam, double* __restrict__ gfn) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const double third = 1.0 / 3.0;
  double Ub[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) Ub[k] = Ub0[k];
  const double n3[3] = {third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f]};
  double acc[3] = {0, 0, 0};
  for (int l = 0; l < 3; ++l) {
    const int nd = faces[3 * (size_t)f + l];
    Dual V[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) V[k] = Dual(P[8 * (size_t)nd + k]);
    for (int d = 0; d < 3; ++d) {
      Dual nn[3] = {Dual(n3[0], d == 0), Dual(n3[1], d == 1), Dual(n3[2], d == 2)};
      Dual fl[5];
      face_flux(g, fcode[f], nn[0], nn[1], nn[2], V, Ub, fl);
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k) s += fl[k].d * lam[5 * (size_t)nd + k];
      acc[d] += third * s;
    }
  }
  gfn[3 * (size_t)f] = acc[0];
  gfn[3 * (size_t)f + 1] = acc[1];
  gfn[3 * (size_t)f + 2] = acc[2];
}

// Least-squares chain per node i: cotangents of the per-neighbour offsets
// d = x_p - x_i through W(w_i, d), through w_i = f(R_i) and through the
// Cholesky factor R_i of sum d d^T (SubDomainCore.C:1334-1381, 1755-1777;
// SubDomain.C:137-159).  gd[p] (3 doubles per neighbour entry).
__global__ void k_a_lsq_x(int N, const double* __restrict__ P, const double* __restrict__ lsqR,
                          const double* __restrict__ lsqW, const int* __restrict__ nbr_ptr,
                          const int* __restrict__ nbr_node, const double* __restrict__ gG, double* __restrict__ gd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double* pi = P + 8 * (size_t)i;
  const double* gg = gG + 16 * (size_t)i;
  double w[6], r[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) { w[k] = lsqW[(size_t)k * N + i]; r[k] = lsqR[(size_t)k * N + i]; }
  double gw[6] = {0, 0, 0, 0, 0, 0};
  // pass 1: through W(w, d)
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const double* pj = P + 8 * (size_t)nbr_node[p];
    const double d0 = pj[5] - pi[5], d1 = pj[6] - pi[6], d2 = pj[7] - pi[7];
    double gW0 = 0.0, gW1 = 0.0, gW2 = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      const double dv = pj[k] - pi[k];
      gW0 += gg[k] * dv; gW1 += gg[5 + k] * dv; gW2 += gg[10 + k] * dv;
    }
    const double alpha2 = (d1 - w[3] * d0) * w[1] * w[1];
    const double e3 = d2 - w[4] * d1 + w[5] * d0;
    const double alpha3 = e3 * w[2] * w[2];
    const double ga1 = gW0;
    const double ga2 = -w[3] * gW0 + gW1;
    const double ga3 = w[5] * gW0 - w[4] * gW1 + gW2;
    gw[3] += -alpha2 * gW0;
    gw[5] += alpha3 * gW0;
    gw[4] += -alpha3 * gW1;
    double gd0 = w[0] * w[0] * ga1, gd1 = 0.0, gd2 = 0.0;
    gw[0] += 2.0 * d0 * w[0] * ga1;
    const double e2 = d1 - w[3] * d0;
    const double ge2 = w[1] * w[1] * ga2;
    gw[1] += 2.0 * e2 * w[1] * ga2;
    gd1 += ge2; gw[3] += -d0 * ge2; gd0 += -w[3] * ge2;
    const double ge3 = w[2] * w[2] * ga3;
    gw[2] += 2.0 * e3 * w[2] * ga3;
    gd2 += ge3; gw[4] += -d1 * ge3; gd1 += -w[4] * ge3; gw[5] += d0 * ge3; gd0 += w[5] * ge3;
    gd[3 * (size_t)p] = gd0; gd[3 * (size_t)p + 1] = gd1; gd[3 * (size_t)p + 2] = gd2;
  }
  // w = f(R): w0=1/r11 w1=1/r22 w2=1/r33 w3=r12 w0 w4=r23 w1 w5=(r12 r23 - r13 r22) w0 w1
  const double r11 = r[0], r12 = r[1], r13 = r[2], r22 = r[3], r23 = r[4], r33 = r[5];
  const double psi0 = r12 * r23 - r13 * r22;
  double gr[6] = {0, 0, 0, 0, 0, 0};
  double gw0 = gw[0] + r12 * gw[3] + psi0 * w[1] * gw[5];
  double gw1 = gw[1] + r23 * gw[4] + psi0 * w[0] * gw[5];
  gr[1] += w[0] * gw[3] + r23 * w[0] * w[1] * gw[5];
  gr[4] += w[1] * gw[4] + r12 * w[0] * w[1] * gw[5];
  gr[2] += -r22 * w[0] * w[1] * gw[5];
  gr[3] += -r13 * w[0] * w[1] * gw[5];
  gr[0] += -w[0] * w[0] * gw0;
  gr[3] += -w[1] * w[1] * gw1;
  gr[5] += -w[2] * w[2] * gw[2];
  // Cholesky reverse (r33, r23, r22, r13, r12, r11)
  double gS[6] = {0, 0, 0, 0, 0, 0};
  gS[5] = 0.5 / r33 * gr[5];
  gr[2] += -r13 / r33 * gr[5];
  gr[4] += -r23 / r33 * gr[5];
  gS[4] = gr[4] / r22;
  gr[1] += -r13 / r22 * gr[4];
  gr[2] += -r12 / r22 * gr[4];
  gr[3] += -r23 / r22 * gr[4];
  gS[3] = 0.5 / r22 * gr[3];
  gr[1] += -r12 / r22 * gr[3];
  gS[2] = gr[2] / r11;
  gr[0] += -r13 / r11 * gr[2];
  gS[1] = gr[1] / r11;
  gr[0] += -r12 / r11 * gr[1];
  gS[0] = 0.5 / r11 * gr[0];
  // pass 2: S = sum d d^T
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const double* pj = P + 8 * (size_t)nbr_node[p];
    const double d0 = pj[5] - pi[5], d1 = pj[6] - pi[6], d2 = pj[7] - pi[7];
    gd[3 * (size_t)p] += 2.0 * d0 * gS[0] + d1 * gS[1] + d2 * gS[2];
    gd[3 * (size_t)p + 1] += d0 * gS[1] + 2.0 * d1 * gS[3] + d2 * gS[4];
    gd[3 * (size_t)p + 2] += d0 * gS[2] + d1 * gS[4] + 2.0 * d2 * gS[5];
  }
}

// g_vol_i = -(w_i . R_i) / vol_i   (R = S / vol)
__global__ void k_a_gvol(int N, const double* __restrict__ w, const double* __restrict__ R,
                         const double* __restrict__ vol, double* __restrict__ gvol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 5; ++k) s += w[5 * (size_t)i + k] * R[5 * (size_t)i + k];
  gvol[i] = -s / vol[i];
}

// Per node q: gather every coordinate cotangent.
//   neighbour offsets:  -sum_p gd[p] + sum_p gd[tpos[p]]
//   edge dx in the reconstruction:  +-g_dx of incident edges
//   tets: volume and dual-cell edge normals, forward mode in x_q's 3 directions
//   boundary faces: face normals, forward mode in x_q's 3 directions
__global__ void k_a_gather_x(int N, int rec, const double* __restrict__ X, const int* __restrict__ tets,
                             const int* __restrict__ tet_edge, const int* __restrict__ faces,
                             const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                             const int* __restrict__ nbr_tpos, const double* __restrict__ gd,
                             const double* __restrict__ erec, const int* __restrict__ nt_ptr,
                             const int* __restrict__ nt_tet, const int* __restrict__ nf_ptr,
                             const int* __restrict__ nf_face, const double* __restrict__ gvol,
                             const double* __restrict__ gfn, double* __restrict__ gX);

}  // namespace aerof

namespace aerof {

__global__ void k_a_gather_x(int N, int rec, const double* __restrict__ X, const int* __restrict__ tets,
                             const int* __restrict__ tet_edge, const int* __restrict__ faces,
                             const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                             const int* __restrict__ nbr_tpos, const double* __restrict__ gd,
                             const double* __restrict__ erec, const int* __restrict__ nt_ptr,
                             const int* __restrict__ nt_tet, const int* __restrict__ nf_ptr,
                             const int* __restrict__ nf_face, const double* __restrict__ gvol,
                             const double* __restrict__ gfn, double* __restrict__ gX) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= N) return;
  double gx[3] = {0, 0, 0};
  for (int p = nbr_ptr[q]; p < nbr_ptr[q + 1]; ++p) {
    const int e = nbr_edge[p];
    const double* o = erec + 32 * (size_t)(e & 0x7fffffff);
    const double s = e < 0 ? 1.0 : -1.0;  // dx = X_second - X_first
#pragma unroll
    for (int c = 0; c < 3; ++c) gx[c] += s * o[23 + c];
    if (rec != AEROF_REC_CONSTANT) {
      const size_t tp = (size_t)nbr_tpos[p];
#pragma unroll
      for (int c = 0; c < 3; ++c) gx[c] += gd[3 * tp + c] - gd[3 * (size_t)p + c];
    }
  }
  // tets: control volumes and dual-cell normals
  for (int p = nt_ptr[q]; p < nt_ptr[q + 1]; ++p) {
    const int t = nt_tet[p] >> 2, a = nt_tet[p] & 3;
    const int* nd = tets + 4 * (size_t)t;
    const double gvt = 0.25 * (gvol[nd[0]] + gvol[nd[1]] + gvol[nd[2]] + gvol[nd[3]]);
    int ed[6];
#pragma unroll
    for (int l = 0; l < 6; ++l) ed[l] = tet_edge[6 * (size_t)t + l];
    for (int c = 0; c < 3; ++c) {
      Dual xs[12];
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) xs[3 * v + k] = Dual(X[3 * (size_t)nd[v] + k], (v == a && k == c) ? 1.0 : 0.0);
      const int loc[4] = {0, 1, 2, 3};
      double acc = tet_volume(xs, loc).d * gvt;
      for (int l = 0; l < 6; ++l) {
        // orientation by global node ids, as in the set-up
        Vec3<Dual> n = tet_edge_normal_local(xs, nd, l);
        const double* gn = erec + 32 * (size_t)ed[l] + 20;
        acc += n.x.d * gn[0] + n.y.d * gn[1] + n.z.d * gn[2];
      }
      gx[c] += acc;
    }
  }
  // boundary faces: face normals
  for (int p = nf_ptr[q]; p < nf_ptr[q + 1]; ++p) {
    const int f = nf_face[p];
    const int* nd = faces + 3 * (size_t)f;
    const int a = nd[0] == q ? 0 : (nd[1] == q ? 1 : 2);
    for (int c = 0; c < 3; ++c) {
      Dual xs[9];
#pragma unroll
      for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int k = 0; k < 3; ++k) xs[3 * v + k] = Dual(X[3 * (size_t)nd[v] + k], (v == a && k == c) ? 1.0 : 0.0);
      const int loc[3] = {0, 1, 2};
      Vec3<Dual> n = face_normal(xs, loc);
      gx[c] += n.x.d * gfn[3 * (size_t)f] + n.y.d * gfn[3 * (size_t)f + 1] + n.z.d * gfn[3 * (size_t)f + 2];
    }
  }
  gX[3 * (size_t)q] = gx[0];
  gX[3 * (size_t)q + 1] = gx[1];
  gX[3 * (size_t)q + 2] = gx[2];
}

// (dR/dX)^T lambda for device state dU, cotangent dlam, into dgX [N][3];
// with dJT also J^T lambda into dJT [N][5] from the same reverse sweep.
void dRdX_T_dev(aerof_gpu_ctx* c, const double* dU, const double* dlam, double* dgX, double* dJT = nullptr) {
  DeviceMesh& m = c->mesh;
  AdjWork& a = c->adj;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const int rec = c->cfg.reconstruction;
  const int gn = grid_for(m.N, kAB), ge = grid_for(m.E, kAB);
  const size_t n5 = 5 * (size_t)m.N;
  c->s.k2.ensure(n5);
  double* R = c->s.k2.p;
  residual_dev(c, dU, R);
  // the node records P and gradients G in the caller's numbering (the
  // blocked residual keeps its own copies)
  prim_dev(c, dU);
  c->s.G.ensure(16 * (size_t)m.N);
  if (rec != AEROF_REC_CONSTANT) gradients_dev(c);
  a.lam.ensure(n5);
  a.edge.ensure(32 * (size_t)m.E);
  a.gV.ensure(n5);
  a.gG.ensure(16 * (size_t)m.N);
  a.gd.ensure(3 * 2 * (size_t)m.E);
  a.gvol.ensure(m.N);
  a.gfn.ensure(3 * (size_t)std::max(m.F, 1));
  k_a_lam<<<gn, kAB, 0, s>>>(m.N, dlam, m.vol.p, a.lam.p);
  AEROF_LAUNCH_CHECK();
  k_a_gvol<<<gn, kAB, 0, s>>>(m.N, dlam, R, m.vol.p, a.gvol.p);
  AEROF_LAUNCH_CHECK();
  k_a_edges<<<ge, kAB, 0, s>>>(m.E, g, rec, c->cfg.beta, m.edges.p, m.en.p, m.P.p, c->s.G.p, a.lam.p, a.edge.p);
  AEROF_LAUNCH_CHECK();
  if (m.F) {
    k_a_face_normal<<<grid_for(m.F, kAB), kAB, 0, s>>>(m.F, g, m.Ubd.p, m.faces.p, m.fcode.p, m.fnrm.p, m.P.p,
                                                         a.lam.p, a.gfn.p);
    AEROF_LAUNCH_CHECK();
  }
  if (rec != AEROF_REC_CONSTANT || dJT) {
    k_a_node<<<gn, kAB, 0, s>>>(m.N, m.F, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_node.p, m.nbr_edge.p, a.edge.p, m.nf_ptr.p,
                                m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, a.lam.p, a.gV.p, a.gG.p);
    AEROF_LAUNCH_CHECK();
  }
  if (rec != AEROF_REC_CONSTANT) {
    k_a_lsq_x<<<gn, kAB, 0, s>>>(m.N, m.P.p, m.lsqR.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p, a.gG.p, a.gd.p);
    AEROF_LAUNCH_CHECK();
  }
  if (dJT) {
    k_a_lsq_prim<<<gn, kAB, 0, s>>>(m.N, g, rec, dU, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p, a.gV.p, a.gG.p,
                                    dJT);
    AEROF_LAUNCH_CHECK();
  }
  k_a_gather_x<<<gn, kAB, 0, s>>>(m.N, rec, m.X.p, m.tets.p, m.tet_edge.p, m.faces.p, m.nbr_ptr.p, m.nbr_edge.p,
                                  m.nbr_tpos.p, a.gd.p, a.edge.p, m.nt_ptr.p, m.nt_tet.p, m.nf_ptr.p, m.nf_face.p,
                                  a.gvol.p, a.gfn.p, dgX);
  AEROF_LAUNCH_CHECK();
}

}  // namespace aerof

// ====================================================================== C ABI
using namespace aerof;

static int need(aerof_gpu_ctx* c) {
  if (!c->has_mesh) {
    c->last_error = "no mesh: call aerof_gpu_set_mesh first";
    return AEROF_ESTATE;
  }
  return AEROF_OK;
}

extern "C" int aerof_gpu_jvp(aerof_gpu_ctx* c, const double* U, const double* v, double* Jv) {
  return guard(c, [&]() -> int {
    if (int e = need(c)) return e;
    if (!U || !v || !Jv) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    const double* dU = in_dev(c, U, n, c->s.Ustage);
    const double* dv = in_dev(c, v, n, c->s.Vstage);
    double* dJ = out_dev(c, Jv, n, c->s.Rstage);
    int bad = residual_forward(c, dU, dv, nullptr, dJ);
    out_finish(c, Jv, dJ, n);
    return bad;
  });
}

extern "C" int aerof_gpu_dRdX(aerof_gpu_ctx* c, const double* U, const double* Xdot, double* dR) {
  return guard(c, [&]() -> int {
    if (int e = need(c)) return e;
    if (!U || !Xdot || !dR) return AEROF_EINVAL;
    const size_t N = c->mesh.N;
    const double* dU = in_dev(c, U, 5 * N, c->s.Ustage);
    const double* dX = in_dev(c, Xdot, 3 * N, c->s.Xstage);
    double* dd = out_dev(c, dR, 5 * N, c->s.Rstage);
    int bad = residual_forward(c, dU, nullptr, dX, dd);
    out_finish(c, dR, dd, 5 * N);
    return bad;
  });
}

extern "C" int aerof_gpu_vjp(aerof_gpu_ctx* c, const double* U, const double* w, double* JTw) {
  return guard(c, [&]() -> int {
    if (int e = need(c)) return e;
    if (!U || !w || !JTw) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    const double* dU = in_dev(c, U, n, c->s.Ustage);
    const double* dw = in_dev(c, w, n, c->s.Vstage);
    double* dout = out_dev(c, JTw, n, c->s.Rstage);
    vjp_dev(c, dU, dw, dout);
    out_finish(c, JTw, dout, n);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_adjoint_products(aerof_gpu_ctx* c, const double* U, const double* lambda, double* JTl,
                                          double* gX) {
  return guard(c, [&]() -> int {
    if (int e = need(c)) return e;
    if (!U || !lambda || !JTl || !gX) return AEROF_EINVAL;
    const size_t N = c->mesh.N;
    const double* dU = in_dev(c, U, 5 * N, c->s.Ustage);
    const double* dl = in_dev(c, lambda, 5 * N, c->s.Vstage);
    double* dJ = out_dev(c, JTl, 5 * N, c->s.Rstage);
    double* dg = out_dev(c, gX, 3 * N, c->s.Xstage);
    dRdX_T_dev(c, dU, dl, dg, dJ);
    out_finish(c, JTl, dJ, 5 * N);
    out_finish(c, gX, dg, 3 * N);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_dRdX_T(aerof_gpu_ctx* c, const double* U, const double* lambda, double* gX) {
  return guard(c, [&]() -> int {
    if (int e = need(c)) return e;
    if (!U || !lambda || !gX) return AEROF_EINVAL;
    const size_t N = c->mesh.N;
    const double* dU = in_dev(c, U, 5 * N, c->s.Ustage);
    const double* dl = in_dev(c, lambda, 5 * N, c->s.Vstage);
    double* dg = out_dev(c, gX, 3 * N, c->s.Xstage);
    dRdX_T_dev(c, dU, dl, dg);
    out_finish(c, gX, dg, 3 * N);
    return AEROF_OK;
  });
}
