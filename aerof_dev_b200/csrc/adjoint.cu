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
// doubles per spill slot of the blocked reverse sweeps: g_Vj (5), g_ddji
// (5), dx (3), padding to a 128-byte record read with 16-byte loads
constexpr int kSP = 16;


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

// Dual number with five tangents (the five state directions of a face
// flux in one evaluation).  Division through one reciprocal of the divisor.
struct Dual5 {
  double v, d[5];
  __device__ Dual5() : v(0.0), d{0.0, 0.0, 0.0, 0.0, 0.0} {}
  __device__ Dual5(double a) : v(a), d{0.0, 0.0, 0.0, 0.0, 0.0} {}
};
__device__ __forceinline__ Dual5 operator+(const Dual5& a, const Dual5& b) {
  Dual5 r(a.v + b.v);
#pragma unroll
  for (int k = 0; k < 5; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
__device__ __forceinline__ Dual5 operator-(const Dual5& a, const Dual5& b) {
  Dual5 r(a.v - b.v);
#pragma unroll
  for (int k = 0; k < 5; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
__device__ __forceinline__ Dual5 operator-(const Dual5& a) {
  Dual5 r(-a.v);
#pragma unroll
  for (int k = 0; k < 5; ++k) r.d[k] = -a.d[k];
  return r;
}
__device__ __forceinline__ Dual5 operator*(const Dual5& a, const Dual5& b) {
  Dual5 r(a.v * b.v);
#pragma unroll
  for (int k = 0; k < 5; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
__device__ __forceinline__ Dual5 operator/(const Dual5& a, const Dual5& b) {
  const double ib = 1.0 / b.v;
  Dual5 r(a.v * ib);
#pragma unroll
  for (int k = 0; k < 5; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
__device__ __forceinline__ Dual5 dsqrt(const Dual5& a) {
  Dual5 r(sqrt(a.v));
  const double h = 0.5 / r.v;
#pragma unroll
  for (int k = 0; k < 5; ++k) r.d[k] = a.d[k] * h;
  return r;
}
__device__ __forceinline__ double vof(const Dual5& a) { return a.v; }

// Face flux cotangents, g_V += (d flux / d V)^T lam, the five state
// directions in one forward-mode evaluation
__device__ void face_vjp_V(const Gas& g, int code, double nx, double ny, double nz, const double* V, const double* Ub,
                           const double* lam, double* gV) {
  Dual5 Vd[5], f[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    Vd[k] = Dual5(V[k]);
    Vd[k].d[k] = 1.0;
  }
  face_flux(g, code, Dual5(nx), Dual5(ny), Dual5(nz), Vd, Ub, f);
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += f[k].d[d] * lam[k];
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
__global__ void __launch_bounds__(256) k_a_lsq_prim(int N, Gas g, int rec, const double* __restrict__ U,
                                                    const double* __restrict__ P, const double* __restrict__ lsqW,
                                                    const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_node,
                                                    const double* __restrict__ gV, const double* __restrict__ gG,
                                                    double* __restrict__ out) {
  // four lanes per node share its neighbours (r, r+4, ...); fixed xor tree
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = t >> 2, r = t & 3;
  const bool act = q < N;
  double gv[5] = {0, 0, 0, 0, 0};
  double Wsum0 = 0.0, Wsum1 = 0.0, Wsum2 = 0.0;
  if (act && rec != AEROF_REC_CONSTANT) {
    const double* pq = P + 8 * (size_t)q;
    double wq[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) wq[k] = lsqW[(size_t)k * N + q];
    for (int p = nbr_ptr[q] + r; p < nbr_ptr[q + 1]; p += 4) {
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
  }
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 5; ++k) gv[k] += __shfl_xor_sync(0xffffffffu, gv[k], o);
    Wsum0 += __shfl_xor_sync(0xffffffffu, Wsum0, o);
    Wsum1 += __shfl_xor_sync(0xffffffffu, Wsum1, o);
    Wsum2 += __shfl_xor_sync(0xffffffffu, Wsum2, o);
  }
  if (!act || r != 0) return;
#pragma unroll
  for (int k = 0; k < 5; ++k) gv[k] += gV[5 * (size_t)q + k];
  if (rec != AEROF_REC_CONSTANT) {
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

// ---------------------------------------------------------------------
// BLOCKED reverse sweep (Morton blocks of the residual's blocked
// organisation).  lam2[n] = w[n2o[n]] / vol: the cotangent of the unscaled
// flux sum, as 48-byte records.
__global__ void k_a_lam2(int N, const int* __restrict__ n2o, const double* __restrict__ w,
                         const double* __restrict__ vol2, double* __restrict__ lam2) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int o = n2o[n];
  const double iv = 1.0 / vol2[n];
#pragma unroll
  for (int k = 0; k < 5; ++k) lam2[6 * (size_t)n + k] = w[5 * (size_t)o + k] * iv;
  lam2[6 * (size_t)n + 5] = 0.0;
}

// One CTA per block.  Phase 0: node records, gradients and lam of the
// block's nodes and forward halo are staged in shared memory (cp.async).
// Phase 1, thread per edge: the reconstruction is recomputed, the Roe flux
// reversed (gF = lam_i - lam_j), and the cotangents (gL, gR) of the two
// reconstructed states kept in shared memory; for a block-crossing edge the
// second endpoint's part (g_Vj, g_ddji, dx) goes to spill; with GEO the
// cotangents of the oriented edge normal and of dx go to geo in the
// original edge numbering and orientation.  Phase 2, L lanes per node: the
// node's edges in edge order, each reversed through the reconstruction for
// the node's side: g_V += g_Vside, g_grad += dx (x) g_ddside; xor-tree lane
// sum; written to gVp / gGp.
template <bool GEO>
__global__ void __launch_bounds__(256, 1) k_a_fv_blocked(int N, int E, int NB, Gas g, int rec, double beta,
                                                         const ushort2* __restrict__ bl, const double* __restrict__ bn,
                                                         const int* __restrict__ beptr, const int* __restrict__ hfptr,
                                                         const int* __restrict__ hfpad, int maxHf,
                                                         const double* __restrict__ P, const double* __restrict__ G,
                                                         const double* __restrict__ lam2, const int* __restrict__ lptr,
                                                         const int* __restrict__ lidx, const int* __restrict__ xslot,
                                                         const int* __restrict__ bsrc, double* __restrict__ gVp,
                                                         double* __restrict__ gGp, double* __restrict__ spill,
                                                         double* __restrict__ geo) {
  extern __shared__ double sm[];
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int nh = hfptr[blk + 1] - hfptr[blk];
  const int ns = nn + nh;
  const int e0 = beptr[blk], e1 = beptr[blk + 1];
  int L = 1;
  while (2 * L * NB <= (int)blockDim.x) L *= 2;
  const int t2 = threadIdx.x / L, r2 = threadIdx.x % L;
  const bool act2 = t2 < nn && (int)threadIdx.x < L * NB;
  const int lb = act2 ? lptr[n0 + t2] : 0, le = act2 ? lptr[n0 + t2 + 1] : 0;
  double* Pn = sm;                           // [ns][kPS]
  double* Gn = sm + kPS * ns;                // [ns][kGS]
  double* Ln = sm + (kPS + kGS) * ns;        // [ns][6]
  double* Es = sm + (kPS + kGS + 6) * ns;    // [e1 - e0][10]: gL, gR
  const bool grad = rec != AEROF_REC_CONSTANT;
  {
    const int* hf = hfpad + (size_t)blk * maxHf;
    double2* pd = reinterpret_cast<double2*>(Pn);
    double2* gd = reinterpret_cast<double2*>(Gn);
    double2* ld = reinterpret_cast<double2*>(Ln);
    const double2* ps = reinterpret_cast<const double2*>(P + 8 * (size_t)n0);
    const double2* gs = reinterpret_cast<const double2*>(G + 16 * (size_t)n0);
    const double2* ls = reinterpret_cast<const double2*>(lam2 + 6 * (size_t)n0);
    for (int k = threadIdx.x; k < 4 * nn; k += blockDim.x) cp_async16(pd + (kPS / 2) * (k >> 2) + (k & 3), ps + k);
    for (int k = threadIdx.x; k < 3 * nn; k += blockDim.x) cp_async16(ld + k, ls + k);
    if (grad)
      for (int k = threadIdx.x; k < 8 * nn; k += blockDim.x) cp_async16(gd + (kGS / 2) * (k >> 3) + (k & 7), gs + k);
    for (int k = threadIdx.x; k < 4 * nh; k += blockDim.x) {
      const int j = hf[k >> 2];
      cp_async16(pd + (kPS / 2) * (nn + (k >> 2)) + (k & 3),
                 reinterpret_cast<const double2*>(P + 8 * (size_t)j) + (k & 3));
    }
    for (int k = threadIdx.x; k < 3 * nh; k += blockDim.x) {
      const int j = hf[k / 3];
      cp_async16(ld + 3 * nn + k, reinterpret_cast<const double2*>(lam2 + 6 * (size_t)j) + k % 3);
    }
    if (grad)
      for (int k = threadIdx.x; k < 8 * nh; k += blockDim.x) {
        const int j = hf[k >> 3];
        cp_async16(gd + (kGS / 2) * (nn + (k >> 3)) + (k & 7),
                   reinterpret_cast<const double2*>(G + 16 * (size_t)j) + (k & 7));
      }
  }
  cp_async_wait_all();
  __syncthreads();
  for (int q = e0 + threadIdx.x; q < e1; q += blockDim.x) {
    const ushort2 lq = bl[q];
    const double n0_ = bn[q], n1_ = bn[(size_t)E + q], n2_ = bn[2 * (size_t)E + q];
    const double* pi = Pn + kPS * lq.x;
    const double* pj = Pn + kPS * lq.y;
    const double* gi = Gn + kGS * lq.x;
    const double* gj = Gn + kGS * lq.y;
    const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
    double Vi[5], Vj[5], ddij[5], ddji[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      if (!grad) {
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
    for (int k = 0; k < 5; ++k) gF[k] = Ln[6 * lq.x + k] - Ln[6 * lq.y + k];
    if (sqrt(n0_ * n0_ + n1_ * n1_ + n2_ * n2_) >= 1e-18) roe_flux_adj(g, n0_, n1_, n2_, Vi, Vj, gF, gL, gR, gn);
    double* es = Es + 10 * (q - e0);
#pragma unroll
    for (int k = 0; k < 5; ++k) { es[k] = gL[k]; es[5 + k] = gR[k]; }
    const int xs = xslot[q];
    if (GEO || xs >= 0) {
      double gdx0 = 0.0, gdx1 = 0.0, gdx2 = 0.0;
      double* sp = xs >= 0 ? spill + kSP * (size_t)xs : nullptr;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double gvi = 0.0, gvj = 0.0, gdi, gdj;
        reconstruct_adj(rec, beta, pi[k], ddij[k], pj[k], ddji[k], gL[k], gR[k], gvi, gvj, gdi, gdj);
        if (grad) {
          gdx0 += gi[k] * gdi + gj[k] * gdj;
          gdx1 += gi[5 + k] * gdi + gj[5 + k] * gdj;
          gdx2 += gi[10 + k] * gdi + gj[10 + k] * gdj;
        }
        if (sp) { sp[k] = gvj; sp[5 + k] = gdj; }
      }
      if (sp) { sp[10] = dx0; sp[11] = dx1; sp[12] = dx2; }
      if (GEO) {
        const int src = bsrc[q];
        const size_t l = (size_t)(src & 0x7fffffff);
        const double sg = src < 0 ? -1.0 : 1.0;
        double2* ge = reinterpret_cast<double2*>(geo + 6 * l);
        ge[0] = make_double2(sg * gn[0], sg * gn[1]);
        ge[1] = make_double2(sg * gn[2], sg * gdx0);
        ge[2] = make_double2(sg * gdx1, sg * gdx2);
      }
    }
  }
  __syncthreads();
  double av[5] = {0, 0, 0, 0, 0}, ag[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) ag[k] = 0.0;
  for (int k = lb + r2; k < le; k += L) {
    const int e = lidx[k];
    const int slot = e & 0x7fffffff;
    const bool second = e < 0;
    const ushort2 lq = bl[e0 + slot];
    const double* pi = Pn + kPS * lq.x;
    const double* pj = Pn + kPS * lq.y;
    const double* gi = Gn + kGS * lq.x;
    const double* gj = Gn + kGS * lq.y;
    const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
    const double* es = Es + 10 * slot;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double ddij = 0.0, ddji = 0.0;
      if (grad) {
        ddij = dx0 * gi[c] + dx1 * gi[5 + c] + dx2 * gi[10 + c];
        ddji = dx0 * gj[c] + dx1 * gj[5 + c] + dx2 * gj[10 + c];
      }
      double gvi = 0.0, gvj = 0.0, gdi, gdj;
      reconstruct_adj(rec, beta, pi[c], ddij, pj[c], ddji, es[c], es[5 + c], gvi, gvj, gdi, gdj);
      const double gd = second ? gdj : gdi;
      av[c] += second ? gvj : gvi;
      ag[c] += dx0 * gd;
      ag[5 + c] += dx1 * gd;
      ag[10 + c] += dx2 * gd;
    }
  }
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 5; ++c) av[c] += __shfl_xor_sync(0xffffffffu, av[c], o);
#pragma unroll
    for (int c = 0; c < 15; ++c) ag[c] += __shfl_xor_sync(0xffffffffu, ag[c], o);
  }
  if (act2 && r2 == 0) {
    const size_t n = (size_t)(n0 + t2);
#pragma unroll
    for (int c = 0; c < 5; ++c) gVp[5 * n + c] = av[c];
#pragma unroll
    for (int c = 0; c < 15; ++c) gGp[16 * n + c] = ag[c];
    gGp[16 * n + 15] = 0.0;
  }
}

// Per node (blocked numbering): in-block sums + the spilled parts of the
// incoming block-crossing edges (contiguous slots), written to the caller's
// numbering.
__global__ void k_a_fv_nodes(int N, const int* __restrict__ n2o, const double* __restrict__ gVp,
                             const double* __restrict__ gGp, const int* __restrict__ xin_ptr,
                             const double* __restrict__ spill, double* __restrict__ gV, double* __restrict__ gG) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double av[5], ag[16];
#pragma unroll
  for (int c = 0; c < 5; ++c) av[c] = gVp[5 * (size_t)n + c];
  {
    const double2* g2 = reinterpret_cast<const double2*>(gGp + 16 * (size_t)n);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double2 v = g2[c];
      ag[2 * c] = v.x;
      ag[2 * c + 1] = v.y;
    }
  }
  for (int k = xin_ptr[n]; k < xin_ptr[n + 1]; ++k) {
    double sp[14];
    const double2* s2 = reinterpret_cast<const double2*>(spill + kSP * (size_t)k);
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      const double2 v = s2[c];
      sp[2 * c] = v.x;
      sp[2 * c + 1] = v.y;
    }
    const double dx0 = sp[10], dx1 = sp[11], dx2 = sp[12];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      av[c] += sp[c];
      ag[c] += dx0 * sp[5 + c];
      ag[5 + c] += dx1 * sp[5 + c];
      ag[10 + c] += dx2 * sp[5 + c];
    }
  }
  const size_t o = (size_t)n2o[n];
#pragma unroll
  for (int c = 0; c < 5; ++c) gV[5 * o + c] = av[c];
#pragma unroll
  for (int c = 0; c < 15; ++c) gG[16 * o + c] = ag[c];
  gG[16 * o + 15] = 0.0;
}

// Boundary faces of node i (face order), added to g_V[i]: the face flux
// Jacobian transposed applied to lam_i = w_i / vol_i (forward mode in the
// 5 state directions).
__global__ void k_a_faces(int N, int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ nf_ptr,
                          const int* __restrict__ nf_face, const int* __restrict__ fcode,
                          const double* __restrict__ fn, const double* __restrict__ P, const double* __restrict__ w,
                          const double* __restrict__ vol, double* __restrict__ gV) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || nf_ptr[i] == nf_ptr[i + 1]) return;
  double V[5], Ub[5], lm[5], gv[5];
  const double iv = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    V[k] = P[8 * (size_t)i + k];
    Ub[k] = Ub0[k];
    lm[k] = w[5 * (size_t)i + k] * iv;
    gv[k] = gV[5 * (size_t)i + k];
  }
  const double third = 1.0 / 3.0;
  for (int q = nf_ptr[i]; q < nf_ptr[i + 1]; ++q) {
    const int f = nf_face[q];
    face_vjp_V(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, lm, gv);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) gV[5 * (size_t)i + k] = gv[k];
}

// Per node in the blocked numbering: in-block sums + the spilled parts of
// the incoming block-crossing edges (+ the boundary faces from the stored
// face Jacobians fj when given: g_V += (d F / d V)^T w / vol), kept in the
// blocked numbering for k_a_lsq_blocked.
__global__ void k_a_nodes_b(int N, const int* __restrict__ n2o, const double* __restrict__ gVp,
                            const double* __restrict__ gGp, const int* __restrict__ xin_ptr,
                            const double* __restrict__ spill, const int* __restrict__ brow, int nbrow,
                            const double* __restrict__ fj, const double* __restrict__ w,
                            const double* __restrict__ vol, double* __restrict__ gV2, double* __restrict__ gG2) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double av[5], ag[16];
#pragma unroll
  for (int c = 0; c < 5; ++c) av[c] = gVp[5 * (size_t)n + c];
  {
    const double2* g2 = reinterpret_cast<const double2*>(gGp + 16 * (size_t)n);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double2 v = g2[c];
      ag[2 * c] = v.x;
      ag[2 * c + 1] = v.y;
    }
  }
  for (int k = xin_ptr[n]; k < xin_ptr[n + 1]; ++k) {
    double sp[14];
    const double2* s2 = reinterpret_cast<const double2*>(spill + kSP * (size_t)k);
#pragma unroll
    for (int c = 0; c < 7; ++c) {
      const double2 v = s2[c];
      sp[2 * c] = v.x;
      sp[2 * c + 1] = v.y;
    }
    const double dx0 = sp[10], dx1 = sp[11], dx2 = sp[12];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      av[c] += sp[c];
      ag[c] += dx0 * sp[5 + c];
      ag[5 + c] += dx1 * sp[5 + c];
      ag[10 + c] += dx2 * sp[5 + c];
    }
  }
  const size_t o = (size_t)n2o[n];
  if (fj) {
    const int b = brow[o];
    if (b >= 0) {
      const double iv = 1.0 / vol[o];
      double lm[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) lm[k] = w[5 * o + k] * iv;
#pragma unroll
      for (int d = 0; d < 5; ++d) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) s += fj[(size_t)(5 * k + d) * nbrow + b] * lm[k];
        av[d] += s;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) gV2[5 * (size_t)n + c] = av[c];
  double2* gg = reinterpret_cast<double2*>(gG2 + 16 * (size_t)n);
#pragma unroll
  for (int c = 0; c < 7; ++c) gg[c] = make_double2(ag[2 * c], ag[2 * c + 1]);
  gg[7] = make_double2(ag[14], 0.0);
}

// Boundary rows (blocked numbering of gV2): g_V += (d F / d V)^T w / vol
// by forward mode per face, in face order (as k_a_faces).
__global__ void k_a_faces_b(int nbrow, int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ blist,
                            const int* __restrict__ o2n, const int* __restrict__ nf_ptr,
                            const int* __restrict__ nf_face, const int* __restrict__ fcode,
                            const double* __restrict__ fn, const double* __restrict__ P,
                            const double* __restrict__ w, const double* __restrict__ vol, double* __restrict__ gV2) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbrow) return;
  const size_t i = (size_t)blist[b];
  const size_t n = (size_t)o2n[i];
  double V[5], Ub[5], lm[5], gv[5];
  const double iv = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    V[k] = P[8 * i + k];
    Ub[k] = Ub0[k];
    lm[k] = w[5 * i + k] * iv;
    gv[k] = gV2[5 * n + k];
  }
  const double third = 1.0 / 3.0;
  for (int q = nf_ptr[i]; q < nf_ptr[i + 1]; ++q) {
    const int f = nf_face[q];
    face_vjp_V(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, lm, gv);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) gV2[5 * n + k] = gv[k];
}

// Transpose of the least-squares gradients and of V(U) in the blocked
// numbering (same sums as k_a_lsq_prim): CTA per Morton block; the node
// coordinates, LSQ constants and gradient cotangents of the block's nodes
// and of its halo (all neighbours outside the block) are staged in shared
// memory (26-double records: V4 x y z | 6 constants | 16 cotangents), then
// L lanes per node take its neighbours r, r + L, ...:
// g_V_q += sum_i W_i(x_q - x_i) . g_grad_i - (sum_i W_q(x_i - x_q)) . g_grad_q,
// fixed xor-tree lane sum, (dV/dU)^T, written in the caller's numbering.
constexpr int kLR = 26;
constexpr int kLsqThreads = 512;
template <int L>
__global__ void __launch_bounds__(kLsqThreads, 2) k_a_lsq_blocked(int N, int NB, Gas g, int rec, const int* __restrict__ n2o,
                                                          const double* __restrict__ U, const double* __restrict__ P2,
                                                          const double* __restrict__ W2,
                                                          const int* __restrict__ nb2_ptr,
                                                          const unsigned short* __restrict__ lnb,
                                                          const int* __restrict__ hptr, const int* __restrict__ hnode,
                                                          const double* __restrict__ gV2,
                                                          const double* __restrict__ gG2, double* __restrict__ out) {
  extern __shared__ double sm[];
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int h0 = hptr[blk], nh = hptr[blk + 1] - h0;
  const int ns = nn + nh;
  const int c0 = nb2_ptr[n0], nc = nb2_ptr[n0 + nn] - c0;
  const bool grad = rec != AEROF_REC_CONSTANT;
  double* rs = sm;                                                                       // [ns][kLR]
  unsigned short* ls = reinterpret_cast<unsigned short*>(rs + kLR * (size_t)ns);         // [nc]
  const int t = threadIdx.x / L, r = threadIdx.x % L;
  const bool act = t < nn;
  if (grad) {
    // thread per staged node, all its copies together; the first two node
    // ids of each thread are loaded before any copy is issued
    double2* rd = reinterpret_cast<double2*>(rs);
    auto stage = [&](int q, int j) {
      const double2* px = reinterpret_cast<const double2*>(P2 + 8 * (size_t)j) + 2;
      const double2* pg = reinterpret_cast<const double2*>(gG2 + 16 * (size_t)j);
      cp_async16(rd + (kLR / 2) * q, px);
      cp_async16(rd + (kLR / 2) * q + 1, px + 1);
#pragma unroll
      for (int c = 0; c < 8; ++c) cp_async16(rd + (kLR / 2) * q + 5 + c, pg + c);
#pragma unroll
      for (int a = 0; a < 6; ++a) cp_async8(rs + kLR * q + 4 + a, W2 + (size_t)a * N + j);
    };
    auto node_id = [&](int q) { return q < nn ? n0 + q : hnode[h0 + q - nn]; };
    const int q0 = threadIdx.x, q1 = threadIdx.x + blockDim.x;
    const int j0 = q0 < ns ? node_id(q0) : -1;
    const int j1 = q1 < ns ? node_id(q1) : -1;
    if (j0 >= 0) stage(q0, j0);
    if (j1 >= 0) stage(q1, j1);
    for (int q = threadIdx.x + 2 * blockDim.x; q < ns; q += blockDim.x) stage(q, node_id(q));
    for (int k = threadIdx.x; k < nc; k += blockDim.x) ls[k] = lnb[c0 + k];
    cp_async_wait_all();
  }
  __syncthreads();
  double gv[5] = {0, 0, 0, 0, 0};
  double ws0 = 0.0, ws1 = 0.0, ws2 = 0.0;
  if (act && grad) {
    const double* pq = rs + kLR * t;
    const int pb = nb2_ptr[n0 + t] - c0, pe = nb2_ptr[n0 + t + 1] - c0;
#pragma unroll 1
    for (int p = pb + r; p < pe; p += L) {
      const double* pi = rs + kLR * (int)ls[p];
      double W0, W1, W2_;
      lsq_weights(pi + 4, pq[1] - pi[1], pq[2] - pi[2], pq[3] - pi[3], W0, W1, W2_);
      const double* gi = pi + 10;
#pragma unroll
      for (int k = 0; k < 5; ++k) gv[k] += W0 * gi[k] + W1 * gi[5 + k] + W2_ * gi[10 + k];
      double V0, V1, V2;
      lsq_weights(pq + 4, pi[1] - pq[1], pi[2] - pq[2], pi[3] - pq[3], V0, V1, V2);
      ws0 += V0; ws1 += V1; ws2 += V2;
    }
  }
#pragma unroll
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 5; ++k) gv[k] += __shfl_xor_sync(0xffffffffu, gv[k], o);
    ws0 += __shfl_xor_sync(0xffffffffu, ws0, o);
    ws1 += __shfl_xor_sync(0xffffffffu, ws1, o);
    ws2 += __shfl_xor_sync(0xffffffffu, ws2, o);
  }
  if (!act || r != 0) return;
  const size_t n = (size_t)(n0 + t);
#pragma unroll
  for (int k = 0; k < 5; ++k) gv[k] += gV2[5 * n + k];
  if (grad) {
    const double* gq = rs + kLR * t + 10;
#pragma unroll
    for (int k = 0; k < 5; ++k) gv[k] -= ws0 * gq[k] + ws1 * gq[5 + k] + ws2 * gq[10 + k];
  }
  const size_t o = (size_t)n2o[n];
  double u[5], gu[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * o + k];
  prim_adj(g, u, gv, gu);
#pragma unroll
  for (int k = 0; k < 5; ++k) out[5 * o + k] = gu[k];
}

static size_t lsq_blocked_smem(const DeviceMesh& m) {
  return ((size_t)8 * kLR * (m.NB + m.maxH) + (size_t)2 * m.maxL + 15) / 16 * 16;
}

// After a blocked edge sweep (gVp, gGp, spill current): node assembly with
// the faces, the LSQ transpose and (dV/dU)^T at dU into dout, all in the
// blocked organisation.  fj: stored face Jacobians, or null for forward mode
// per face (needs P at dU).  False (nothing launched) when the staging does
// not fit in shared memory.
static bool lsq_blocked_fits(const DeviceMesh& m) {
  const int L = kLsqThreads / m.NB;
  return lsq_blocked_smem(m) <= 200 * 1024 && L >= 2 && L <= 8 && L * m.NB == kLsqThreads;
}

// node assembly of a blocked reverse sweep into gV2 / gG2 (blocked
// numbering), with the faces
static void assemble_blocked(aerof_gpu_ctx* c, const double* dw, const double* fj) {
  DeviceMesh& m = c->mesh;
  AdjWork& a = c->adj;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  a.gV2.ensure(5 * (size_t)m.N);
  a.gG2.ensure(16 * (size_t)m.N);
  k_a_nodes_b<<<grid_for(m.N, kAB), kAB, 0, s>>>(m.N, m.n2o.p, a.gVp.p, a.gGp.p, m.xin_ptr.p, a.spill.p, m.brow.p,
                                                 m.nbrow, fj, dw, m.vol.p, a.gV2.p, a.gG2.p);
  AEROF_LAUNCH_CHECK();
  if (!fj && m.nbrow) {
    k_a_faces_b<<<grid_for(m.nbrow, kAB), kAB, 0, s>>>(m.nbrow, m.F, g, m.Ubd.p, m.blist.p, m.o2n.p, m.nf_ptr.p,
                                                       m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, dw, m.vol.p, a.gV2.p);
    AEROF_LAUNCH_CHECK();
  }
}

// LSQ transpose and (dV/dU)^T at dU of gV2 / gG2 into dout
static void lsq_transpose_blocked(aerof_gpu_ctx* c, const double* dU, int rec, double* dout) {
  DeviceMesh& m = c->mesh;
  AdjWork& a = c->adj;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const size_t smem = lsq_blocked_smem(m);
  const int L = kLsqThreads / m.NB;
  auto go = [&](auto kern) {
    AEROF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<m.nblk, kLsqThreads, smem, s>>>(m.N, m.NB, g, rec, m.n2o.p, dU, m.P2.p, m.W2.p, m.nb2_ptr.p, m.lnb.p,
                                           m.hptr.p, m.hnode.p, a.gV2.p, a.gG2.p, dout);
    AEROF_LAUNCH_CHECK();
  };
  if (L == 8) go(k_a_lsq_blocked<8>);
  else if (L == 4) go(k_a_lsq_blocked<4>);
  else go(k_a_lsq_blocked<2>);
}

// After a blocked edge sweep (gVp, gGp, spill current): node assembly with
// the faces, the LSQ transpose and (dV/dU)^T at dU into dout, all in the
// blocked organisation.  fj: stored face Jacobians, or null for forward mode
// per face (needs P at dU).  False (nothing launched) when the staging does
// not fit in shared memory.
static bool assemble_lsq_blocked(aerof_gpu_ctx* c, const double* dU, const double* dw, const double* fj, int rec,
                                 double* dout) {
  if (!lsq_blocked_fits(c->mesh)) return false;
  assemble_blocked(c, dw, fj);
  lsq_transpose_blocked(c, dU, rec, dout);
  return true;
}

// Blocked reverse sweep over the edges and faces: a.gV, a.gG (caller
// numbering) from the cotangent dw; with geo, also the cotangents of the
// edge normals and dx.  Needs P (caller numbering) and P2/G2 current.
static void reverse_sweep_blocked(aerof_gpu_ctx* c, const double* dw, bool geo, bool assemble = true) {
  DeviceMesh& m = c->mesh;
  AdjWork& a = c->adj;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const int rec = c->cfg.reconstruction;
  const int gn = grid_for(m.N, kAB);
  a.lam2.ensure(6 * (size_t)m.N);
  a.gVp.ensure(5 * (size_t)m.N);
  a.gGp.ensure(16 * (size_t)m.N);
  a.spill.ensure(kSP * (size_t)std::max(m.nX, 1));
  a.gV.ensure(5 * (size_t)m.N);
  a.gG.ensure(16 * (size_t)m.N);
  if (geo) a.geo.ensure(6 * (size_t)std::max(m.E, 1));
  k_a_lam2<<<gn, kAB, 0, s>>>(m.N, m.n2o.p, dw, m.vol2.p, a.lam2.p);
  AEROF_LAUNCH_CHECK();
  const size_t smem = ((size_t)(kPS + kGS + 6) * (m.NB + m.maxHf) + (size_t)10 * m.maxE) * sizeof(double);
  auto go = [&](auto kern) {
    AEROF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<m.nblk, 256, smem, s>>>(m.N, m.E, m.NB, g, rec, c->cfg.beta, m.bl.p, m.bnorm.p, m.beptr.p, m.hfptr.p,
                                   m.hfpad.p, m.maxHf, m.P2.p, c->s.G2.p, a.lam2.p, m.lptr.p, m.lidx.p, m.xslot.p,
                                   m.bsrc.p, a.gVp.p, a.gGp.p, a.spill.p, geo ? a.geo.p : nullptr);
    AEROF_LAUNCH_CHECK();
  };
  if (geo) go(k_a_fv_blocked<true>);
  else go(k_a_fv_blocked<false>);
  if (!assemble) return;
  k_a_fv_nodes<<<gn, kAB, 0, s>>>(m.N, m.n2o.p, a.gVp.p, a.gGp.p, m.xin_ptr.p, a.spill.p, a.gV.p, a.gG.p);
  AEROF_LAUNCH_CHECK();
  if (m.F) {
    k_a_faces<<<gn, kAB, 0, s>>>(m.N, m.F, g, m.Ubd.p, m.nf_ptr.p, m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, dw,
                                 m.vol.p, a.gV.p);
    AEROF_LAUNCH_CHECK();
  }
}

// whether the blocked reverse sweep's shared memory fits
static bool reverse_blocked_fits(const DeviceMesh& m) {
  return m.nblk > 0 &&
         ((size_t)(kPS + kGS + 6) * (m.NB + m.maxHf) + (size_t)10 * m.maxE) * sizeof(double) <= 200 * 1024;
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
  a.gV.ensure(5 * (size_t)m.N);
  a.gG.ensure(16 * (size_t)m.N);
  if (reverse_blocked_fits(m)) {
    prim_grad_blocked_dev(c, dU, nullptr);
    if (lsq_blocked_fits(m)) {
      // edges, then assembly, faces, LSQ transpose and (dV/dU)^T in the
      // blocked organisation
      reverse_sweep_blocked(c, dw, false, false);
      if (assemble_lsq_blocked(c, dU, dw, nullptr, rec, dout)) return;
      k_a_fv_nodes<<<gn, kAB, 0, s>>>(m.N, m.n2o.p, a.gVp.p, a.gGp.p, m.xin_ptr.p, a.spill.p, a.gV.p, a.gG.p);
      AEROF_LAUNCH_CHECK();
      if (m.F) {
        k_a_faces<<<gn, kAB, 0, s>>>(m.N, m.F, g, m.Ubd.p, m.nf_ptr.p, m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, dw,
                                     m.vol.p, a.gV.p);
        AEROF_LAUNCH_CHECK();
      }
    } else {
      reverse_sweep_blocked(c, dw, false);
    }
  } else {
    c->s.G.ensure(16 * (size_t)m.N);
    if (rec != AEROF_REC_CONSTANT) gradients_dev(c);
    a.lam.ensure(5 * (size_t)m.N);
    a.edge.ensure(32 * (size_t)m.E);
    k_a_lam<<<gn, kAB, 0, s>>>(m.N, dw, m.vol.p, a.lam.p);
    AEROF_LAUNCH_CHECK();
    k_a_edges<<<ge, kAB, 0, s>>>(m.E, g, rec, c->cfg.beta, m.edges.p, m.en.p, m.P.p, c->s.G.p, a.lam.p, a.edge.p);
    AEROF_LAUNCH_CHECK();
    k_a_node<<<gn, kAB, 0, s>>>(m.N, m.F, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_node.p, m.nbr_edge.p, a.edge.p, m.nf_ptr.p,
                                m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, a.lam.p, a.gV.p, a.gG.p);
    AEROF_LAUNCH_CHECK();
  }
  k_a_lsq_prim<<<grid_for(4 * (size_t)m.N, kAB), kAB, 0, s>>>(m.N, g, rec, dU, m.P.p, m.lsqW.p, m.nbr_ptr.p,
                                                              m.nbr_node.p, a.gV.p, a.gG.p, dout);
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
                                const double* __restrict__ P, const double* __restrict__ lam,
                                double* __restrict__ gfn) {
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
__global__ void __launch_bounds__(256) k_a_lsq_x(int N, const double* __restrict__ P, const double* __restrict__ lsqR,
                                                 const double* __restrict__ lsqW, const int* __restrict__ nbr_ptr,
                                                 const int* __restrict__ nbr_node, const double* __restrict__ gG,
                                                 const int* __restrict__ o2n, double* __restrict__ gd) {
  // four lanes per node share its neighbours (lane, lane+4, ...) in both passes;
  // the cotangent of the node's constants is summed in a fixed xor tree.
  // gG is in the caller's numbering, or in the blocked one when o2n is given
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = min(t >> 2, N - 1), lane = t & 3;
  const bool act = (t >> 2) < N;
  const double* pi = P + 8 * (size_t)i;
  const double* gg = gG + 16 * (size_t)(o2n ? o2n[i] : i);
  double w[6], r[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) { w[k] = lsqW[(size_t)k * N + i]; r[k] = lsqR[(size_t)k * N + i]; }
  double gw[6] = {0, 0, 0, 0, 0, 0};
  // the lane's first KM entries keep their pass-1 cotangents in shared
  // memory for pass 2 (one store of gd each); further entries (nodes with
  // more than 4 KM neighbours) store gd in pass 1 and add to it in pass 2
  constexpr int KM = 4;
  __shared__ double kg[KM * 3][256];
  const int pb = nbr_ptr[i], pe = nbr_ptr[i + 1];
  // pass 1: through W(w, d)
  for (int p = pb + lane, m = 0; act && p < pe; p += 4, ++m) {
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
    if (m < KM) {
      kg[3 * m][threadIdx.x] = gd0; kg[3 * m + 1][threadIdx.x] = gd1; kg[3 * m + 2][threadIdx.x] = gd2;
    } else {
      gd[3 * (size_t)p] = gd0; gd[3 * (size_t)p + 1] = gd1; gd[3 * (size_t)p + 2] = gd2;
    }
  }
#pragma unroll
  for (int o = 1; o < 4; o <<= 1)
#pragma unroll
    for (int k = 0; k < 6; ++k) gw[k] += __shfl_xor_sync(0xffffffffu, gw[k], o);
  if (!act) return;
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
  for (int k = 0; k < KM; ++k) {
    const int p = pb + lane + 4 * k;
    if (p >= pe) break;
    const double* pj = P + 8 * (size_t)nbr_node[p];
    const double d0 = pj[5] - pi[5], d1 = pj[6] - pi[6], d2 = pj[7] - pi[7];
    gd[3 * (size_t)p] = kg[3 * k][threadIdx.x] + (2.0 * d0 * gS[0] + d1 * gS[1] + d2 * gS[2]);
    gd[3 * (size_t)p + 1] = kg[3 * k + 1][threadIdx.x] + (d0 * gS[1] + 2.0 * d1 * gS[3] + d2 * gS[4]);
    gd[3 * (size_t)p + 2] = kg[3 * k + 2][threadIdx.x] + (d0 * gS[2] + d1 * gS[4] + 2.0 * d2 * gS[5]);
  }
  for (int p = pb + lane + 4 * KM; p < pe; p += 4) {
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
__global__ void k_a_gather_x(int N, int rec, const double* __restrict__ X, const int* __restrict__ faces,
                             const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                             const int* __restrict__ nbr_tpos, const double* __restrict__ gd,
                             const double* __restrict__ geo, const int* __restrict__ nt_ptr,
                             const int* __restrict__ nt_tet, const int* __restrict__ nf_ptr,
                             const int* __restrict__ nf_face, const double* __restrict__ tg,
                             const double* __restrict__ gfn, double* __restrict__ gX);

}  // namespace aerof

namespace aerof {

// Per tet: cotangents of its four vertices' coordinates through the
// control volumes and the dual-cell edge normals, reverse mode in closed
// form.  Volume V = (e3 . (e1 x e2)) / 6, e_i = x_i - x_0; edge normal
// n = 1.5 s (xg1 x xg0) with xg = face centroid - tet centroid
// (ElemTetCore.C:281-330), so g_xg1 = xg0 x g_c, g_xg0 = g_c x xg1 with
// g_c = 1.5 s g_n, then a third to each vertex of the face and minus a
// quarter to every vertex for the centroid.  tg[t][3 a + c].
template <int TB>
__global__ void __launch_bounds__(TB) k_a_tet_x(int T, const double* __restrict__ X, const int* __restrict__ tets,
                                                const int* __restrict__ tet_edge, const double* __restrict__ geo,
                                                const double* __restrict__ gvol, double* __restrict__ tg) {
  // the block's 12-double rows are staged in shared memory (row stride 13:
  // conflict-free) and stored contiguously
  __shared__ double st[TB * 13];
  const int t0 = blockIdx.x * TB, t = t0 + threadIdx.x;
  if (t < T) {
    const int4 q4 = *reinterpret_cast<const int4*>(tets + 4 * (size_t)t);
    const int nd[4] = {q4.x, q4.y, q4.z, q4.w};
    const double gvt = 0.25 * (gvol[nd[0]] + gvol[nd[1]] + gvol[nd[2]] + gvol[nd[3]]);
    Vec3<double> x[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) x[v] = node_x(X, nd[v]);
    const Vec3<double> e1 = x[1] - x[0], e2 = x[2] - x[0], e3 = x[3] - x[0];
    const double sv = gvt / 6.0;
    Vec3<double> g[4];
    g[1] = scale(sv, cross(e2, e3));
    g[2] = scale(sv, cross(e3, e1));
    g[3] = scale(sv, cross(e1, e2));
    g[0] = v3(0.0, 0.0, 0.0) - (g[1] + g[2] + g[3]);
    const double third = 1.0 / 3.0;
    Vec3<double> f[4];
    f[0] = scale(third, x[0] + x[1] + x[2]);
    f[1] = scale(third, x[0] + x[1] + x[3]);
    f[2] = scale(third, x[0] + x[2] + x[3]);
    f[3] = scale(third, x[1] + x[2] + x[3]);
    const Vec3<double> gc0 = scale(0.25, x[0] + x[1] + x[2] + x[3]);
    Vec3<double> gf[4] = {v3(0.0, 0.0, 0.0), v3(0.0, 0.0, 0.0), v3(0.0, 0.0, 0.0), v3(0.0, 0.0, 0.0)};
    Vec3<double> gcen = v3(0.0, 0.0, 0.0);
#pragma unroll
    for (int l = 0; l < 6; ++l) {
      const int F0 = tet_edge_face(l, 0), F1 = tet_edge_face(l, 1);
      const Vec3<double> xg0 = f[F0] - gc0, xg1 = f[F1] - gc0;
      const size_t el = (size_t)tet_edge[6 * (size_t)t + l];
      const double sl = nd[tet_edge_end(l, 0)] < nd[tet_edge_end(l, 1)] ? 1.5 : -1.5;
      const double2 g01 = *reinterpret_cast<const double2*>(geo + 6 * el);
      const Vec3<double> gcv = v3(sl * g01.x, sl * g01.y, sl * geo[6 * el + 2]);
      const Vec3<double> g1 = cross(xg0, gcv), g0 = cross(gcv, xg1);
      gf[F0] = gf[F0] + g0;
      gf[F1] = gf[F1] + g1;
      gcen = gcen + g0 + g1;
    }
    // face k holds every vertex but 3 - k
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      Vec3<double> s = v3(0.0, 0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (a != 3 - k) s = s + gf[k];
      const Vec3<double> d = g[a] + scale(third, s) - scale(0.25, gcen);
      st[13 * threadIdx.x + 3 * a] = d.x;
      st[13 * threadIdx.x + 3 * a + 1] = d.y;
      st[13 * threadIdx.x + 3 * a + 2] = d.z;
    }
  }
  __syncthreads();
  const int cnt = 12 * min(TB, T - t0);
  double* out = tg + 12 * (size_t)t0;
  for (int f = threadIdx.x; f < cnt; f += TB) out[f] = st[13 * (f / 12) + f % 12];
}

__global__ void k_a_gather_x(int N, int rec, const double* __restrict__ X, const int* __restrict__ faces,
                             const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                             const int* __restrict__ nbr_tpos, const double* __restrict__ gd,
                             const double* __restrict__ geo, const int* __restrict__ nt_ptr,
                             const int* __restrict__ nt_tet, const int* __restrict__ nf_ptr,
                             const int* __restrict__ nf_face, const double* __restrict__ tg,
                             const double* __restrict__ gfn, double* __restrict__ gX) {
  // three lanes per node, lane c summing component c (each in the order of
  // the one-thread form: edges, tets, faces)
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * (long long)N) return;
  const int q = (int)(j / 3), c = (int)(j - 3 * (long long)q);
  double gx = 0.0;
  for (int p = nbr_ptr[q]; p < nbr_ptr[q + 1]; ++p) {
    const int e = nbr_edge[p];
    const size_t el = (size_t)(e & 0x7fffffff);
    const double s = e < 0 ? 1.0 : -1.0;  // dx = X_second - X_first
    gx += s * geo[6 * el + 3 + c];
    if (rec != AEROF_REC_CONSTANT) {
      const size_t tp = (size_t)nbr_tpos[p];
      gx += gd[3 * tp + c] - gd[3 * (size_t)p + c];
    }
  }
  // tets: the per-tet vertex cotangents of k_a_tet_x
  for (int p = nt_ptr[q]; p < nt_ptr[q + 1]; ++p) {
    const size_t t = (size_t)(nt_tet[p] >> 2);
    const int a = nt_tet[p] & 3;
    gx += tg[12 * t + 3 * a + c];
  }
  // boundary faces: n = (3 x02 x x01 + 3 x02 x x01) / 12 (FaceTriaCore.C:
  // 65-82) = x02 x x01 / 2, so g_x02 = x01 x g_n / 2, g_x01 = g_n x x02 / 2
  for (int p = nf_ptr[q]; p < nf_ptr[q + 1]; ++p) {
    const int f = nf_face[p];
    const int* nd = faces + 3 * (size_t)f;
    const int a = nd[0] == q ? 0 : (nd[1] == q ? 1 : 2);
    const Vec3<double> x0 = node_x(X, nd[0]);
    const Vec3<double> x01 = node_x(X, nd[1]) - x0, x02 = node_x(X, nd[2]) - x0;
    const Vec3<double> gn = v3(gfn[3 * (size_t)f], gfn[3 * (size_t)f + 1], gfn[3 * (size_t)f + 2]);
    const Vec3<double> g02 = scale(0.5, cross(x01, gn)), g01 = scale(0.5, cross(gn, x02));
    const Vec3<double> d = a == 2 ? g02 : (a == 1 ? g01 : v3(0.0, 0.0, 0.0) - (g02 + g01));
    gx += c == 0 ? d.x : (c == 1 ? d.y : d.z);
  }
  gX[3 * (size_t)q + c] = gx;
}

// cotangents of the edge normals and dx out of the per-edge records of the
// edge-parallel reverse sweep, in the layout of the blocked one
__global__ void k_a_geo_from_rec(int E, const double* __restrict__ erec, double* __restrict__ geo) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
#pragma unroll
  for (int k = 0; k < 6; ++k) geo[6 * (size_t)l + k] = erec[32 * (size_t)l + 20 + k];
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
  // node records P in the caller's numbering for the node and face passes
  prim_dev(c, dU);
  a.lam.ensure(n5);
  a.gV.ensure(n5);
  a.gG.ensure(16 * (size_t)m.N);
  a.gd.ensure(3 * 2 * (size_t)m.E);
  a.gvol.ensure(m.N);
  a.gfn.ensure(3 * (size_t)std::max(m.F, 1));
  a.geo.ensure(6 * (size_t)std::max(m.E, 1));
  k_a_lam<<<gn, kAB, 0, s>>>(m.N, dlam, m.vol.p, a.lam.p);
  AEROF_LAUNCH_CHECK();
  k_a_gvol<<<gn, kAB, 0, s>>>(m.N, dlam, R, m.vol.p, a.gvol.p);
  AEROF_LAUNCH_CHECK();
  // blocked organisation: node assembly and LSQ transposes read the
  // blocked-numbered cotangents
  const bool blk = reverse_blocked_fits(m) && lsq_blocked_fits(m);
  if (reverse_blocked_fits(m)) {
    // the residual above leaves P2 / G2 of dU when it ran blocked and
    // untagged
    if (!c->s.p2g2_valid) prim_grad_blocked_dev(c, dU, nullptr);
    reverse_sweep_blocked(c, dlam, true, !blk);
    if (blk) assemble_blocked(c, dlam, nullptr);
  } else {
    c->s.G.ensure(16 * (size_t)m.N);
    if (rec != AEROF_REC_CONSTANT) gradients_dev(c);
    a.edge.ensure(32 * (size_t)m.E);
    k_a_edges<<<ge, kAB, 0, s>>>(m.E, g, rec, c->cfg.beta, m.edges.p, m.en.p, m.P.p, c->s.G.p, a.lam.p, a.edge.p);
    AEROF_LAUNCH_CHECK();
    k_a_node<<<gn, kAB, 0, s>>>(m.N, m.F, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_node.p, m.nbr_edge.p, a.edge.p, m.nf_ptr.p,
                                m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, a.lam.p, a.gV.p, a.gG.p);
    AEROF_LAUNCH_CHECK();
    k_a_geo_from_rec<<<ge, kAB, 0, s>>>(m.E, a.edge.p, a.geo.p);
    AEROF_LAUNCH_CHECK();
  }
  if (m.F) {
    k_a_face_normal<<<grid_for(m.F, kAB), kAB, 0, s>>>(m.F, g, m.Ubd.p, m.faces.p, m.fcode.p, m.fnrm.p, m.P.p,
                                                         a.lam.p, a.gfn.p);
    AEROF_LAUNCH_CHECK();
  }
  if (rec != AEROF_REC_CONSTANT) {
    k_a_lsq_x<<<grid_for(4 * (size_t)m.N, kAB), kAB, 0, s>>>(m.N, m.P.p, m.lsqR.p, m.lsqW.p, m.nbr_ptr.p,
                                                             m.nbr_node.p, blk ? a.gG2.p : a.gG.p,
                                                             blk ? m.o2n.p : nullptr, a.gd.p);
    AEROF_LAUNCH_CHECK();
  }
  if (dJT && blk) {
    lsq_transpose_blocked(c, dU, rec, dJT);
  } else if (dJT) {
    k_a_lsq_prim<<<grid_for(4 * (size_t)m.N, kAB), kAB, 0, s>>>(m.N, g, rec, dU, m.P.p, m.lsqW.p, m.nbr_ptr.p,
                                                                m.nbr_node.p, a.gV.p, a.gG.p, dJT);
    AEROF_LAUNCH_CHECK();
  }
  a.tg.ensure(12 * (size_t)std::max(m.T, 1));
  if (m.T) {
    k_a_tet_x<128><<<grid_for(m.T, 128), 128, 0, s>>>(m.T, m.X.p, m.tets.p, m.tet_edge.p, a.geo.p, a.gvol.p, a.tg.p);
    AEROF_LAUNCH_CHECK();
  }
  k_a_gather_x<<<grid_for(3 * (size_t)m.N, kAB), kAB, 0, s>>>(m.N, rec, m.X.p, m.faces.p, m.nbr_ptr.p, m.nbr_edge.p,
                                                             m.nbr_tpos.p, a.gd.p, a.geo.p, m.nt_ptr.p, m.nt_tet.p,
                                                             m.nf_ptr.p, m.nf_face.p, a.tg.p, a.gfn.p, dgX);
  AEROF_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------
// STORED EXACT LINEARISATION (MatVecProdH2, MatVecProd.C:1462-1704).  The
// reference's evaluate keeps per edge the reconstruction coefficients
// (SubDomain::precomputeRec, SubDomain.C:3836-3865) and the two flux
// Jacobians (A at numNodes + 2l, + 1, computeH2); apply and applyTranspose
// (SubDomain::computeMatVecProdH2, SubDomain.C:4076-4190) form the
// direction's gradients, reconstruct it linearly, apply the blocks and
// assemble.  Here, per blocked edge, the 50 block entries and the 20
// reconstruction partials are stored as 35 16-byte pairs, SoA by pair
// ([35][E] double2, one coalesced 16-byte load per pair):
//   pair 5 r + c (r, c < 5): (d phi_r / d Vij_c, d phi_r / d Vji_c)
//   pair 25 + c:             (p1_c, p2_c)
//   pair 30 + c:             (q1_c, q2_c)
// and per boundary row the summed face-flux Jacobian; a product is one
// pass over that data in the blocked organisation plus the gradient
// (forward) or its transpose (reverse).

// Thread per blocked edge, CTA per block: the reconstruction at the
// linearisation state, d phi / d Vij and d phi / d Vji by five reverse
// evaluations of the Roe flux (row r from the unit cotangent e_r), and the
// partials of the reconstruction of each component.
__global__ void __launch_bounds__(128) k_h2_edges(int N, int E, int NB, Gas g, int rec, double beta,
                                                  const ushort2* __restrict__ bl, const double* __restrict__ bn,
                                                  const int* __restrict__ beptr, const int* __restrict__ hfpad,
                                                  int maxHf, const double* __restrict__ P2,
                                                  const double* __restrict__ G2, double2* __restrict__ h2) {
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int e0 = beptr[blk], e1 = beptr[blk + 1];
  const int* hf = hfpad + (size_t)blk * maxHf;
  const bool grad = rec != AEROF_REC_CONSTANT;
  const size_t sE = (size_t)E;
  for (int q = e0 + threadIdx.x; q < e1; q += blockDim.x) {
    const ushort2 lq = bl[q];
    // the first endpoint lies in the block, the second in it or in its
    // forward halo
    const size_t ni = (size_t)(n0 + lq.x);
    const size_t nj = (size_t)(lq.y < nn ? n0 + lq.y : hf[lq.y - nn]);
    const double* pi = P2 + 8 * ni;
    const double* pj = P2 + 8 * nj;
    const double* gi = G2 + 16 * ni;
    const double* gj = G2 + 16 * nj;
    const double n0_ = bn[q], n1_ = bn[sE + q], n2_ = bn[2 * sE + q];
    const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
    double Vi[5], Vj[5], cp1[5], cp2[5], cq1[5], cq2[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      if (!grad) {
        Vi[k] = pi[k]; Vj[k] = pj[k];
        cp1[k] = cp2[k] = cq1[k] = cq2[k] = 0.0;
        continue;
      }
      const double ddij = dx0 * gi[k] + dx1 * gi[5 + k] + dx2 * gi[10 + k];
      const double ddji = dx0 * gj[k] + dx1 * gj[5 + k] + dx2 * gj[10 + k];
      if (rec == AEROF_REC_VANALBADA) {
        vanalbada(beta, pi[k], ddij, pj[k], ddji, Vi[k], Vj[k]);
        // Vij = Vi + 0.5 f(dVi, dVji), Vji = Vj - 0.5 f(dVj, dVji),
        // dVji = Vj - Vi, dVi = b2 dVji + 2 beta ddij (RecFcn.h:432-446)
        const double b2 = 1.0 - 2.0 * beta;
        const double dVji = pj[k] - pi[k];
        const double dV = b2 * dVji;
        double A1, B1, A2, B2;
        vanalbada_fcn_partials(dV + 2.0 * beta * ddij, dVji, A1, B1);
        vanalbada_fcn_partials(dV + 2.0 * beta * ddji, dVji, A2, B2);
        cp1[k] = 0.5 * (B1 + b2 * A1);
        cp2[k] = 0.5 * (B2 + b2 * A2);
        cq1[k] = beta * A1;
        cq2[k] = beta * A2;
      } else {
        linear_rec(beta, pi[k], ddij, pj[k], ddji, Vi[k], Vj[k]);
        cp1[k] = cp2[k] = 0.5 - beta;
        cq1[k] = cq2[k] = beta;
      }
    }
    const bool live = sqrt(n0_ * n0_ + n1_ * n1_ + n2_ * n2_) >= 1e-18;
#pragma unroll 1
    for (int r = 0; r < 5; ++r) {
      double gF[5], gL[5] = {0, 0, 0, 0, 0}, gR[5] = {0, 0, 0, 0, 0};
#pragma unroll
      for (int k = 0; k < 5; ++k) gF[k] = k == r ? 1.0 : 0.0;
      if (live) roe_flux_adj(g, n0_, n1_, n2_, Vi, Vj, gF, gL, gR, nullptr);
#pragma unroll
      for (int k = 0; k < 5; ++k) h2[(size_t)(5 * r + k) * sE + q] = make_double2(gL[k], gR[k]);
    }
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      h2[(size_t)(25 + k) * sE + q] = make_double2(cp1[k], cp2[k]);
      h2[(size_t)(30 + k) * sE + q] = make_double2(cq1[k], cq2[k]);
    }
  }
}

// Per boundary row: the Jacobian d F / d V summed over the row's faces
// (subface normal n_f / 3), five tangents in one forward evaluation per
// face; SoA [25][nbrow], element (k, d) = d F_k / d V_d.
__global__ void k_h2_faces(int nbrow, int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ blist,
                           const int* __restrict__ nf_ptr, const int* __restrict__ nf_face,
                           const int* __restrict__ fcode, const double* __restrict__ fn,
                           const double* __restrict__ P, double* __restrict__ fj) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbrow) return;
  const int i = blist[b];
  double J[25], Ub[5];
  Dual5 Vd[5];
#pragma unroll
  for (int k = 0; k < 25; ++k) J[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    Ub[k] = Ub0[k];
    Vd[k] = Dual5(P[8 * (size_t)i + k]);
    Vd[k].d[k] = 1.0;
  }
  const double third = 1.0 / 3.0;
  for (int q = nf_ptr[i]; q < nf_ptr[i + 1]; ++q) {
    const int f = nf_face[q];
    Dual5 ff[5];
    face_flux(g, fcode[f], Dual5(third * fn[f]), Dual5(third * fn[(size_t)F + f]), Dual5(third * fn[2 * (size_t)F + f]),
              Vd, Ub, ff);
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
      for (int d = 0; d < 5; ++d) J[5 * k + d] += ff[k].d[d];
  }
#pragma unroll
  for (int k = 0; k < 25; ++k) fj[(size_t)k * nbrow + b] = J[k];
}

// (gL, gR) = ((d phi / d Vij)^T gF, (d phi / d Vji)^T gF) of edge q
__device__ __forceinline__ void h2_transpose_blocks(const double2* __restrict__ h2, size_t sE, int q,
                                                    const double* gF, double* gL, double* gR) {
#pragma unroll
  for (int c = 0; c < 5; ++c) { gL[c] = 0.0; gR[c] = 0.0; }
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double2 a = h2[(size_t)(5 * r + c) * sE + q];
      gL[c] += a.x * gF[r];
      gR[c] += a.y * gF[r];
    }
}

// J^T of the stored operator, edge part.  CTA per block.  Phase 0: the
// coordinates and lam2 of the block's nodes and forward halo are staged
// (cp.async; 32 B of each node record: V4, x, y, z).  Phase 1, thread per
// edge: gF = lam_i - lam_j, gL = (d phi / d Vij)^T gF, gR = (d phi /
// d Vji)^T gF kept in shared memory; a block-crossing edge sends the second
// endpoint's part (g_Vj, g_ddji, dx) to spill.  Phase 2, L lanes per node:
// the node's edges in edge order through the stored reconstruction
// partials, g_V += g_Vside, g_grad += dx (x) g_ddside; written to gVp /
// gGp as k_a_fv_blocked does.
__global__ void __launch_bounds__(256, 2) k_h2t_blocked(int N, int E, int NB, const ushort2* __restrict__ bl,
                                                        const int* __restrict__ beptr, const int* __restrict__ hfptr,
                                                        const int* __restrict__ hfpad, int maxHf,
                                                        const double* __restrict__ P2, const double* __restrict__ lam2,
                                                        const int* __restrict__ lptr, const int* __restrict__ lidx,
                                                        const int* __restrict__ xslot, const double2* __restrict__ h2,
                                                        double* __restrict__ gVp, double* __restrict__ gGp,
                                                        double* __restrict__ spill) {
  extern __shared__ double sm[];
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int nh = hfptr[blk + 1] - hfptr[blk];
  const int ns = nn + nh;
  const int e0 = beptr[blk], e1 = beptr[blk + 1];
  const size_t sE = (size_t)E;
  int L = 1;
  while (2 * L * NB <= (int)blockDim.x) L *= 2;
  const int t2 = threadIdx.x / L, r2 = threadIdx.x % L;
  const bool act2 = t2 < nn && (int)threadIdx.x < L * NB;
  const int lb = act2 ? lptr[n0 + t2] : 0, le = act2 ? lptr[n0 + t2 + 1] : 0;
  double* Xn = sm;             // [ns][4]: V4, x, y, z
  double* Ln = sm + 4 * ns;    // [ns][6]
  double* Es = sm + 10 * ns;   // [e1 - e0][10]: gL, gR
  {
    const int* hf = hfpad + (size_t)blk * maxHf;
    double2* xd = reinterpret_cast<double2*>(Xn);
    double2* ld = reinterpret_cast<double2*>(Ln);
    const double2* ps = reinterpret_cast<const double2*>(P2 + 8 * (size_t)n0);
    const double2* ls = reinterpret_cast<const double2*>(lam2 + 6 * (size_t)n0);
    for (int k = threadIdx.x; k < 2 * nn; k += blockDim.x) cp_async16(xd + k, ps + 4 * (k >> 1) + 2 + (k & 1));
    for (int k = threadIdx.x; k < 3 * nn; k += blockDim.x) cp_async16(ld + k, ls + k);
    for (int k = threadIdx.x; k < 2 * nh; k += blockDim.x) {
      const int j = hf[k >> 1];
      cp_async16(xd + 2 * nn + k, reinterpret_cast<const double2*>(P2 + 8 * (size_t)j) + 2 + (k & 1));
    }
    for (int k = threadIdx.x; k < 3 * nh; k += blockDim.x) {
      const int j = hf[k / 3];
      cp_async16(ld + 3 * nn + k, reinterpret_cast<const double2*>(lam2 + 6 * (size_t)j) + k % 3);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  for (int q = e0 + threadIdx.x; q < e1; q += blockDim.x) {
    const ushort2 lq = bl[q];
    double gF[5], gL[5], gR[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) gF[k] = Ln[6 * lq.x + k] - Ln[6 * lq.y + k];
    h2_transpose_blocks(h2, sE, q, gF, gL, gR);
    double* es = Es + 10 * (q - e0);
#pragma unroll
    for (int k = 0; k < 5; ++k) { es[k] = gL[k]; es[5 + k] = gR[k]; }
    const int xs = xslot[q];
    if (xs >= 0) {
      double* sp = spill + kSP * (size_t)xs;
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const double2 pp = h2[(size_t)(25 + c) * sE + q];
        const double q2 = h2[(size_t)(30 + c) * sE + q].y;
        sp[c] = pp.x * gL[c] + (1.0 - pp.y) * gR[c];
        sp[5 + c] = -q2 * gR[c];
      }
      const double* xi = Xn + 4 * lq.x;
      const double* xj = Xn + 4 * lq.y;
      sp[10] = xj[1] - xi[1]; sp[11] = xj[2] - xi[2]; sp[12] = xj[3] - xi[3];
    }
  }
  __syncthreads();
  double av[5] = {0, 0, 0, 0, 0}, ag[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) ag[k] = 0.0;
  for (int k = lb + r2; k < le; k += L) {
    const int e = lidx[k];
    const int slot = e & 0x7fffffff;
    const bool second = e < 0;
    const size_t qq = (size_t)(e0 + slot);
    const ushort2 lq = bl[qq];
    const double* xi = Xn + 4 * lq.x;
    const double* xj = Xn + 4 * lq.y;
    const double dx0 = xj[1] - xi[1], dx1 = xj[2] - xi[2], dx2 = xj[3] - xi[3];
    const double* es = Es + 10 * slot;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double2 pp = h2[(25 + c) * sE + qq], qv = h2[(30 + c) * sE + qq];
      const double gl = es[c], gr = es[5 + c];
      const double gv = second ? pp.x * gl + (1.0 - pp.y) * gr : (1.0 - pp.x) * gl + pp.y * gr;
      const double gd = second ? -qv.y * gr : qv.x * gl;
      av[c] += gv;
      ag[c] += dx0 * gd;
      ag[5 + c] += dx1 * gd;
      ag[10 + c] += dx2 * gd;
    }
  }
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 5; ++c) av[c] += __shfl_xor_sync(0xffffffffu, av[c], o);
#pragma unroll
    for (int c = 0; c < 15; ++c) ag[c] += __shfl_xor_sync(0xffffffffu, ag[c], o);
  }
  if (act2 && r2 == 0) {
    const size_t n = (size_t)(n0 + t2);
#pragma unroll
    for (int c = 0; c < 5; ++c) gVp[5 * n + c] = av[c];
#pragma unroll
    for (int c = 0; c < 15; ++c) gGp[16 * n + c] = ag[c];
    gGp[16 * n + 15] = 0.0;
  }
}

// J^T of the stored operator, edge part, wide form: one CTA of 1024
// threads per block, used when both endpoints' results of every edge fit in
// shared memory.  Phase 0 as k_h2t_blocked.  Phase 1 reads each edge's 35
// pairs once (coalesced) and leaves (g_Vi, g_ddij, g_Vj, g_ddji) in shared
// memory at a 21-double stride (conflict-free consecutive writes); phase 2
// gathers from shared memory only.  Same arithmetic as k_h2t_blocked.  The
// streamed pairs are in flight through L1, so the kernel is faster the less
// shared memory it holds: a second staging buffer (for a persistent,
// prefetching form) costs more than its latency hiding gains.
constexpr int kEW = 21;
constexpr int kWideThreads = 1024;
__global__ void __launch_bounds__(kWideThreads, 1) k_h2t_wide(int N, int E, int NB, const ushort2* __restrict__ bl,
                                                      const int* __restrict__ beptr, const int* __restrict__ hfptr,
                                                      const int* __restrict__ hfpad, int maxHf,
                                                      const double* __restrict__ P2, const double* __restrict__ lam2,
                                                      const int* __restrict__ lptr, const int* __restrict__ lidx,
                                                      const int* __restrict__ xslot, const double2* __restrict__ h2,
                                                      double* __restrict__ gVp, double* __restrict__ gGp,
                                                      double* __restrict__ spill) {
  extern __shared__ double sm[];
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int nh = hfptr[blk + 1] - hfptr[blk];
  const int ns = nn + nh;
  const int e0 = beptr[blk], e1 = beptr[blk + 1];
  const size_t sE = (size_t)E;
  int L = 1;
  while (2 * L * NB <= (int)blockDim.x) L *= 2;
  const int t2 = threadIdx.x / L, r2 = threadIdx.x % L;
  const bool act2 = t2 < nn && (int)threadIdx.x < L * NB;
  const int lb = act2 ? lptr[n0 + t2] : 0, le = act2 ? lptr[n0 + t2 + 1] : 0;
  double* Xn = sm;             // [ns][4]: V4, x, y, z
  double* Ln = sm + 4 * ns;    // [ns][6]
  double* Es = sm + 10 * ns;   // [e1 - e0][kEW]
  {
    const int* hf = hfpad + (size_t)blk * maxHf;
    double2* xd = reinterpret_cast<double2*>(Xn);
    double2* ld = reinterpret_cast<double2*>(Ln);
    const double2* ps = reinterpret_cast<const double2*>(P2 + 8 * (size_t)n0);
    const double2* ls = reinterpret_cast<const double2*>(lam2 + 6 * (size_t)n0);
    for (int k = threadIdx.x; k < 2 * nn; k += blockDim.x) cp_async16(xd + k, ps + 4 * (k >> 1) + 2 + (k & 1));
    for (int k = threadIdx.x; k < 3 * nn; k += blockDim.x) cp_async16(ld + k, ls + k);
    for (int k = threadIdx.x; k < 2 * nh; k += blockDim.x) {
      const int j = hf[k >> 1];
      cp_async16(xd + 2 * nn + k, reinterpret_cast<const double2*>(P2 + 8 * (size_t)j) + 2 + (k & 1));
    }
    for (int k = threadIdx.x; k < 3 * nh; k += blockDim.x) {
      const int j = hf[k / 3];
      cp_async16(ld + 3 * nn + k, reinterpret_cast<const double2*>(lam2 + 6 * (size_t)j) + k % 3);
    }
  }
  cp_async_wait_all();
  __syncthreads();
  for (int q = e0 + threadIdx.x; q < e1; q += blockDim.x) {
    const ushort2 lq = bl[q];
    double gF[5], gL[5], gR[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) gF[k] = Ln[6 * lq.x + k] - Ln[6 * lq.y + k];
    h2_transpose_blocks(h2, sE, q, gF, gL, gR);
    double* es = Es + kEW * (q - e0);
    const int xs = xslot[q];
    double* sp = xs >= 0 ? spill + kSP * (size_t)xs : nullptr;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double2 pp = h2[(size_t)(25 + c) * sE + q], qv = h2[(size_t)(30 + c) * sE + q];
      const double gvj = pp.x * gL[c] + (1.0 - pp.y) * gR[c];
      const double gdj = -qv.y * gR[c];
      es[c] = (1.0 - pp.x) * gL[c] + pp.y * gR[c];
      es[5 + c] = qv.x * gL[c];
      es[10 + c] = gvj;
      es[15 + c] = gdj;
      if (sp) { sp[c] = gvj; sp[5 + c] = gdj; }
    }
    if (sp) {
      const double* xi = Xn + 4 * lq.x;
      const double* xj = Xn + 4 * lq.y;
      sp[10] = xj[1] - xi[1]; sp[11] = xj[2] - xi[2]; sp[12] = xj[3] - xi[3];
    }
  }
  __syncthreads();
  double av[5] = {0, 0, 0, 0, 0}, ag[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) ag[k] = 0.0;
  for (int k = lb + r2; k < le; k += L) {
    const int e = lidx[k];
    const int slot = e & 0x7fffffff;
    const ushort2 lq = bl[e0 + slot];
    const double* xi = Xn + 4 * lq.x;
    const double* xj = Xn + 4 * lq.y;
    const double dx0 = xj[1] - xi[1], dx1 = xj[2] - xi[2], dx2 = xj[3] - xi[3];
    const double* es = Es + kEW * slot + (e < 0 ? 10 : 0);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double gd = es[5 + c];
      av[c] += es[c];
      ag[c] += dx0 * gd;
      ag[5 + c] += dx1 * gd;
      ag[10 + c] += dx2 * gd;
    }
  }
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 5; ++c) av[c] += __shfl_xor_sync(0xffffffffu, av[c], o);
#pragma unroll
    for (int c = 0; c < 15; ++c) ag[c] += __shfl_xor_sync(0xffffffffu, ag[c], o);
  }
  if (act2 && r2 == 0) {
    const size_t n = (size_t)(n0 + t2);
#pragma unroll
    for (int c = 0; c < 5; ++c) gVp[5 * n + c] = av[c];
#pragma unroll
    for (int c = 0; c < 15; ++c) gGp[16 * n + c] = ag[c];
    gGp[16 * n + 15] = 0.0;
  }
}

// J^T of the stored operator, boundary rows: g_V[i] += (d F / d V)^T
// (w_i / vol_i).
__global__ void k_h2t_faces(int nbrow, const int* __restrict__ blist, const double* __restrict__ fj,
                            const double* __restrict__ w, const double* __restrict__ vol, double* __restrict__ gV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbrow) return;
  const size_t i = (size_t)blist[b];
  const double iv = 1.0 / vol[i];
  double lm[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) lm[k] = w[5 * i + k] * iv;
#pragma unroll
  for (int d = 0; d < 5; ++d) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += fj[(size_t)(5 * k + d) * nbrow + b] * lm[k];
    gV[5 * i + d] += s;
  }
}

// Tangent records of the forward product: dP2[n] = (dV, X) with dV =
// (dV/dU) dp at the linearisation state (VarFcnSGEuler.h:307-327), in the
// blocked numbering.
__global__ void k_h2_seed(int N, Gas g, const int* __restrict__ n2o, const double* __restrict__ U,
                          const double* __restrict__ dp, const double* __restrict__ P2, double* __restrict__ dP2) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const size_t o = (size_t)n2o[n];
  double u[5], du[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) { u[k] = U[5 * o + k]; du[k] = dp[5 * o + k]; }
  const double ir = 1.0 / u[0];
  const double a = u[1] * ir, b = u[2] * ir, cc = u[3] * ir;
  double* d = dP2 + 8 * (size_t)n;
  d[0] = du[0];
  d[1] = (du[1] - a * du[0]) * ir;
  d[2] = (du[2] - b * du[0]) * ir;
  d[3] = (du[3] - cc * du[0]) * ir;
  d[4] = g.gam1 * (0.5 * (a * a + b * b + cc * cc) * du[0] - a * du[1] - b * du[2] - cc * du[3] + du[4]);
  const double* x = P2 + 8 * (size_t)n;
  d[5] = x[5]; d[6] = x[6]; d[7] = x[7];
}

// J of the stored operator, edge part: k_fv_blocked's organisation with the
// flux replaced by its stored linearisation.  Phase 0 stages the tangent
// records and tangent gradients of the block's nodes and forward halo;
// phase 1, thread per edge: dVij, dVji through the stored reconstruction
// partials, dphi = (d phi / d Vij) dVij + (d phi / d Vji) dVji into shared
// memory (and spill for block-crossing edges); phase 2 sums each node's
// edges in edge order (+ first endpoint, - second) into part.
template <int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) k_h2_blocked(int N, int E, int NB, int rec, const ushort2* __restrict__ bl,
                                                       const int* __restrict__ beptr, const int* __restrict__ hfptr,
                                                       const int* __restrict__ hfpad, int maxHf,
                                                       const double* __restrict__ dP2, const double* __restrict__ dG2,
                                                       const int* __restrict__ lptr, const int* __restrict__ lidx,
                                                       const int* __restrict__ xslot, const double2* __restrict__ h2,
                                                       double* __restrict__ part, double* __restrict__ spill,
                                                       int pf) {
  extern __shared__ double sm[];
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int nh = hfptr[blk + 1] - hfptr[blk];
  const int ns = nn + nh;
  const int e0 = beptr[blk], e1 = beptr[blk + 1];
  const size_t sE = (size_t)E;
  const bool grad = rec != AEROF_REC_CONSTANT;
  // the block's stored pairs start streaming into L2 before the staging
  if (pf) prefetch_pairs_l2(h2, sE, e0, e1, grad ? 35 : 30);
  int L = 1;
  while (2 * L * NB <= (int)blockDim.x) L *= 2;
  const int t2 = threadIdx.x / L, r2 = threadIdx.x % L;
  const bool act2 = t2 < nn && (int)threadIdx.x < L * NB;
  const int lb = act2 ? lptr[n0 + t2] : 0, le = act2 ? lptr[n0 + t2 + 1] : 0;
  double* Pn = sm;                      // [ns][kPS]
  double* Gn = sm + kPS * ns;           // [ns][kGS]
  double* Fs = sm + (kPS + kGS) * ns;   // [e1 - e0][5]
  {
    const int* hf = hfpad + (size_t)blk * maxHf;
    const double2* ps = reinterpret_cast<const double2*>(dP2 + 8 * (size_t)n0);
    const double2* gs = reinterpret_cast<const double2*>(dG2 + 16 * (size_t)n0);
    double2* pd = reinterpret_cast<double2*>(Pn);
    double2* gd = reinterpret_cast<double2*>(Gn);
    for (int k = threadIdx.x; k < 4 * nn; k += blockDim.x) cp_async16(pd + (kPS / 2) * (k >> 2) + (k & 3), ps + k);
    if (grad)
      for (int k = threadIdx.x; k < 8 * nn; k += blockDim.x) cp_async16(gd + (kGS / 2) * (k >> 3) + (k & 7), gs + k);
    for (int k = threadIdx.x; k < 4 * nh; k += blockDim.x) {
      const int j = hf[k >> 2];
      cp_async16(pd + (kPS / 2) * (nn + (k >> 2)) + (k & 3),
                 reinterpret_cast<const double2*>(dP2 + 8 * (size_t)j) + (k & 3));
    }
    if (grad)
      for (int k = threadIdx.x; k < 8 * nh; k += blockDim.x) {
        const int j = hf[k >> 3];
        cp_async16(gd + (kGS / 2) * (nn + (k >> 3)) + (k & 7),
                   reinterpret_cast<const double2*>(dG2 + 16 * (size_t)j) + (k & 7));
      }
  }
  cp_async_wait_all();
  __syncthreads();
  for (int q = e0 + threadIdx.x; q < e1; q += blockDim.x) {
    const ushort2 lq = bl[q];
    const double* pi = Pn + kPS * lq.x;
    const double* pj = Pn + kPS * lq.y;
    const double* gi = Gn + kGS * lq.x;
    const double* gj = Gn + kGS * lq.y;
    const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
    double vl[5], vr[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double2 pp = h2[(size_t)(25 + c) * sE + q];
      double a = (1.0 - pp.x) * pi[c] + pp.x * pj[c];
      double b = pp.y * pi[c] + (1.0 - pp.y) * pj[c];
      if (grad) {
        const double2 qv = h2[(size_t)(30 + c) * sE + q];
        const double ddij = dx0 * gi[c] + dx1 * gi[5 + c] + dx2 * gi[10 + c];
        const double ddji = dx0 * gj[c] + dx1 * gj[5 + c] + dx2 * gj[10 + c];
        a += qv.x * ddij;
        b -= qv.y * ddji;
      }
      vl[c] = a;
      vr[c] = b;
    }
    double* fs = Fs + 5 * (q - e0);
    const int xs = xslot[q];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double f = 0.0;
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        const double2 a = h2[(size_t)(5 * r + c) * sE + q];
        f += a.x * vl[c] + a.y * vr[c];
      }
      fs[r] = f;
      if (xs >= 0) spill[5 * (size_t)xs + r] = f;
    }
  }
  __syncthreads();
  double acc[5] = {0, 0, 0, 0, 0};
  for (int k = lb + r2; k < le; k += L) {
    const int e = lidx[k];
    const double* fs = Fs + 5 * (e & 0x7fffffff);
    if (e < 0) {
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[c] -= fs[c];
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[c] += fs[c];
    }
  }
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  }
  if (act2 && r2 == 0) {
#pragma unroll
    for (int c = 0; c < 5; ++c) part[5 * (size_t)(n0 + t2) + c] = acc[c];
  }
}

// J of the stored operator, per row (caller numbering): block sum minus the
// spilled tangent fluxes of incoming block-crossing edges, plus the face
// Jacobian times dV of a boundary row, times 1/ctrlVol.
__global__ void k_h2_nodes(int N, const int* __restrict__ o2n, const double* __restrict__ part,
                           const int* __restrict__ xin_ptr, const double* __restrict__ spill,
                           const int* __restrict__ brow, int nbrow, const double* __restrict__ fj,
                           const double* __restrict__ dP2, const double* __restrict__ vol, double* __restrict__ y) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= N) return;
  const int n = o2n[o];
  double acc[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] = part[5 * (size_t)n + c];
  for (int k = xin_ptr[n]; k < xin_ptr[n + 1]; ++k) {
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] -= spill[5 * (size_t)k + c];
  }
  const int b = brow[o];
  if (b >= 0) {
    double dv[5];
#pragma unroll
    for (int d = 0; d < 5; ++d) dv[d] = dP2[8 * (size_t)n + d];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double s = 0.0;
#pragma unroll
      for (int d = 0; d < 5; ++d) s += fj[(size_t)(5 * k + d) * nbrow + b] * dv[d];
      acc[k] += s;
    }
  }
  const double iv = 1.0 / vol[o];
#pragma unroll
  for (int c = 0; c < 5; ++c) y[5 * (size_t)o + c] = acc[c] * iv;
}

static size_t h2t_smem(const DeviceMesh& m) {
  return ((size_t)10 * (m.NB + m.maxHf) + (size_t)10 * m.maxE) * sizeof(double);
}
static size_t h2t_wide_smem(const DeviceMesh& m) {
  return ((size_t)10 * (m.NB + m.maxHf) + (size_t)kEW * m.maxE) * sizeof(double);
}
static size_t h2f_smem(const DeviceMesh& m) {
  return ((size_t)(kPS + kGS) * (m.NB + m.maxHf) + (size_t)5 * m.maxE) * sizeof(double);
}

// whether the stored operator's blocked kernels fit in shared memory
static bool h2_fits(const DeviceMesh& m) {
  return m.nblk > 0 && std::max(h2t_smem(m), h2f_smem(m)) <= 200 * 1024;
}

static double2* h2pairs(H2Op& h) { return reinterpret_cast<double2*>(h.a.p); }

void h2_evaluate_dev(aerof_gpu_ctx* c, const double* dU) {
  DeviceMesh& m = c->mesh;
  H2Op& h = c->h2;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  if (!h2_fits(m))
    throw ApiError{AEROF_ESTATE, "the stored operator needs the blocked organisation within 200 KB of shared memory"};
  h.ready = false;
  h.a.ensure((size_t)kH2Rec * std::max(m.E, 1));
  h.fj.ensure((size_t)25 * std::max(m.nbrow, 1));
  h.U.ensure(5 * (size_t)m.N);
  AEROF_CUDA(cudaMemcpyAsync(h.U.p, dU, 5 * (size_t)m.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  prim_dev(c, dU);
  prim_grad_blocked_dev(c, dU, nullptr);
  k_h2_edges<<<m.nblk, 128, 0, s>>>(m.N, m.E, m.NB, g, c->cfg.reconstruction, c->cfg.beta, m.bl.p, m.bnorm.p,
                                     m.beptr.p, m.hfpad.p, m.maxHf, m.P2.p, c->s.G2.p, h2pairs(h));
  AEROF_LAUNCH_CHECK();
  if (m.nbrow) {
    k_h2_faces<<<grid_for(m.nbrow, kAB), kAB, 0, s>>>(m.nbrow, m.F, g, m.Ubd.p, m.blist.p, m.nf_ptr.p, m.nf_face.p,
                                                      m.fcode.p, m.fnrm.p, m.P.p, h.fj.p);
    AEROF_LAUNCH_CHECK();
  }
  h.rec = c->cfg.reconstruction;
  h.ready = true;
}

// Bulk L2 prefetch of each block's stored pairs at the start of the
// forward product's edge kernel (1.22 against 1.25 ms per product at 101^3;
// in the transpose kernel it measured slower, 2.03 against 1.78 ms, and is
// not used there).  Tuning knob AEROF_H2_PREFETCH = 0 turns it off.
static int h2_prefetch() {
  static const int v = [] {
    const char* e = std::getenv("AEROF_H2_PREFETCH");
    return e ? std::atoi(e) : 1;
  }();
  return v;
}

// y = J^T w with the stored operator (MatVecProdH2::applyTranspose)
static void h2_vjp_dev(aerof_gpu_ctx* c, const double* dw, double* dout) {
  DeviceMesh& m = c->mesh;
  AdjWork& a = c->adj;
  H2Op& h = c->h2;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const int gn = grid_for(m.N, kAB);
  a.lam2.ensure(6 * (size_t)m.N);
  a.gVp.ensure(5 * (size_t)m.N);
  a.gGp.ensure(16 * (size_t)m.N);
  a.spill.ensure(kSP * (size_t)std::max(m.nX, 1));
  a.gV.ensure(5 * (size_t)m.N);
  a.gG.ensure(16 * (size_t)m.N);
  k_a_lam2<<<gn, kAB, 0, s>>>(m.N, m.n2o.p, dw, m.vol2.p, a.lam2.p);
  AEROF_LAUNCH_CHECK();
  // wide form when both endpoints' results fit in shared memory (tuning
  // knob AEROF_H2T_WIDE=0 selects the compact form)
  const char* wide_var = std::getenv("AEROF_H2T_WIDE");
  const bool wide = (!wide_var || std::atoi(wide_var) != 0) && h2t_wide_smem(m) <= 220 * 1024;
  if (wide) {
    const size_t smem = h2t_wide_smem(m);
    AEROF_CUDA(cudaFuncSetAttribute(k_h2t_wide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_h2t_wide<<<m.nblk, kWideThreads, smem, s>>>(m.N, m.E, m.NB, m.bl.p, m.beptr.p, m.hfptr.p, m.hfpad.p, m.maxHf,
                                                  m.P2.p, a.lam2.p, m.lptr.p, m.lidx.p, m.xslot.p, h2pairs(h),
                                                  a.gVp.p, a.gGp.p, a.spill.p);
  } else {
    const size_t smem = h2t_smem(m);
    AEROF_CUDA(cudaFuncSetAttribute(k_h2t_blocked, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_h2t_blocked<<<m.nblk, 256, smem, s>>>(m.N, m.E, m.NB, m.bl.p, m.beptr.p, m.hfptr.p, m.hfpad.p, m.maxHf,
                                            m.P2.p, a.lam2.p, m.lptr.p, m.lidx.p, m.xslot.p, h2pairs(h), a.gVp.p,
                                            a.gGp.p, a.spill.p);
  }
  AEROF_LAUNCH_CHECK();
  if (assemble_lsq_blocked(c, h.U.p, dw, h.fj.p, h.rec, dout)) return;
  k_a_fv_nodes<<<gn, kAB, 0, s>>>(m.N, m.n2o.p, a.gVp.p, a.gGp.p, m.xin_ptr.p, a.spill.p, a.gV.p, a.gG.p);
  AEROF_LAUNCH_CHECK();
  if (m.nbrow) {
    k_h2t_faces<<<grid_for(m.nbrow, kAB), kAB, 0, s>>>(m.nbrow, m.blist.p, h.fj.p, dw, m.vol.p, a.gV.p);
    AEROF_LAUNCH_CHECK();
  }
  k_a_lsq_prim<<<grid_for(4 * (size_t)m.N, kAB), kAB, 0, s>>>(m.N, g, h.rec, h.U.p, m.P.p, m.lsqW.p, m.nbr_ptr.p,
                                                              m.nbr_node.p, a.gV.p, a.gG.p, dout);
  AEROF_LAUNCH_CHECK();
}

// y = J p with the stored operator (MatVecProdH2::apply)
static void h2_jvp_dev(aerof_gpu_ctx* c, const double* dp, double* dout) {
  DeviceMesh& m = c->mesh;
  H2Op& h = c->h2;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const int gn = grid_for(m.N, kAB);
  h.dP2.ensure(8 * (size_t)m.N);
  h.dG2.ensure(16 * (size_t)m.N);
  h.part.ensure(5 * (size_t)m.N);
  h.spill.ensure(5 * (size_t)std::max(m.nX, 1));
  k_h2_seed<<<gn, kAB, 0, s>>>(m.N, g, m.n2o.p, h.U.p, dp, m.P2.p, h.dP2.p);
  AEROF_LAUNCH_CHECK();
  if (h.rec != AEROF_REC_CONSTANT) grad_records_blocked_dev(c, h.dP2.p, h.dG2.p);
  const size_t smem = h2f_smem(m);
  // one CTA of 1024 threads per SM by default: the streamed pairs are in
  // flight through L1, which two CTAs' shared memory would leave small
  // (tuning knob AEROF_H2F_THREADS = 512 or 256: two CTAs per SM)
  const char* fvar = std::getenv("AEROF_H2F_THREADS");
  const int fthreads = fvar && std::atoi(fvar) == 512 ? 512 : fvar && std::atoi(fvar) == 256 ? 256 : 1024;
  auto kf = fthreads == 512 ? k_h2_blocked<512, 2> : fthreads == 256 ? k_h2_blocked<256, 2> : k_h2_blocked<1024, 1>;
  AEROF_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kf<<<m.nblk, fthreads, smem, s>>>(m.N, m.E, m.NB, h.rec, m.bl.p, m.beptr.p, m.hfptr.p, m.hfpad.p, m.maxHf,
                                         h.dP2.p, h.dG2.p, m.lptr.p, m.lidx.p, m.xslot.p, h2pairs(h), h.part.p,
                                         h.spill.p, h2_prefetch());
  AEROF_LAUNCH_CHECK();
  k_h2_nodes<<<gn, kAB, 0, s>>>(m.N, m.o2n.p, h.part.p, m.xin_ptr.p, h.spill.p, m.brow.p, m.nbrow, h.fj.p, h.dP2.p,
                                m.vol.p, dout);
  AEROF_LAUNCH_CHECK();
}

static void h2_apply_dev(aerof_gpu_ctx* c, const double* p, double* y, bool trans) {
  if (trans) h2_vjp_dev(c, p, y);
  else h2_jvp_dev(c, p, y);
}

void exact_product(aerof_gpu_ctx* c, const double* dU, const double* p, double* y, bool trans) {
  if (c->h2.use && c->h2.ready) {
    h2_apply_dev(c, p, y, trans);
    return;
  }
  if (trans) vjp_dev(c, dU, p, y);
  else residual_forward(c, dU, p, nullptr, y, false);
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
    need_inviscid(c);
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
    need_inviscid(c);
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
    need_inviscid(c);
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
    need_inviscid(c);
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
    need_inviscid(c);
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

// MatVecProdH2::evaluate (MatVecProd.C:1498-1520): the exact linearisation
// at U stored in device memory.
extern "C" int aerof_gpu_h2_evaluate(aerof_gpu_ctx* c, const double* U) {
  return guard(c, [&]() -> int {
    need_inviscid(c);
    if (int e = need(c)) return e;
    if (!U) return AEROF_EINVAL;
    const double* dU = in_dev(c, U, 5 * (size_t)c->mesh.N, c->s.Ustage);
    h2_evaluate_dev(c, dU);
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    return AEROF_OK;
  });
}

// MatVecProdH2::apply / applyTranspose (MatVecProd.C:1622-1704) with the
// stored operator.
extern "C" int aerof_gpu_h2_apply(aerof_gpu_ctx* c, const double* p, double* y, int transpose) {
  return guard(c, [&]() -> int {
    need_inviscid(c);
    if (int e = need(c)) return e;
    if (!p || !y) return AEROF_EINVAL;
    if (!c->h2.ready) {
      c->last_error = "no stored operator: call aerof_gpu_h2_evaluate first";
      return AEROF_ESTATE;
    }
    const size_t n = 5 * (size_t)c->mesh.N;
    const double* dp = in_dev(c, p, n, c->s.Vstage);
    double* dy = out_dev(c, y, n, c->s.Rstage);
    h2_apply_dev(c, dp, dy, transpose != 0);
    out_finish(c, y, dy, n);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_h2_release(aerof_gpu_ctx* c) {
  return guard(c, [&]() -> int {
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    H2Op& h = c->h2;
    h.ready = false;
    h.use = false;
    h.a.release();
    h.fj.release();
    h.U.release();
    h.dP2.release();
    h.dG2.release();
    h.part.release();
    h.spill.release();
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_set_exact_operator(aerof_gpu_ctx* c, int stored) {
  return guard(c, [&]() -> int {
    if (stored != 0 && stored != 1) return AEROF_EINVAL;
    c->h2.in_solves = stored == 1;
    return AEROF_OK;
  });
}
