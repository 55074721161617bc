// residual.cu -- FP64 residual of the edge-based finite-volume scheme on the
// GPU: primitive conversion, least-squares gradients, Roe edge fluxes with
// MUSCL/van Albada reconstruction, boundary fluxes, 1/ctrlVol scaling; plus
// the local time step and the explicit RK2 driver built on them.
//
// Accumulation is deterministic and follows the reference's order per node:
// every node sums its incident edges in ascending-neighbour order (which is
// the order the reference's lexicographic edge loop visits them,
// Edge.C:391-435, SubDomain.C:341-370), then its boundary faces in face
// order (Face.C:1185-1215).  No floating-point atomics are used.
#include "common.cuh"
#include "physics.cuh"

namespace aerof {

constexpr int kBlock = 256;
constexpr int kRedBlocks = 1184;  // 8 x 148 SMs

// ------------------------------------------------------------------ kernels
// U[N][5] (conservative, caller layout) -> node record P[i] = (V[5], X[3]).
__global__ void k_prim(int N, Gas g, const double* __restrict__ U, double* __restrict__ P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)i + k];
  cons2prim(g, u, v);
#pragma unroll
  for (int k = 0; k < 5; ++k) P[8 * (size_t)i + k] = v[k];
}

// V[N][5] primitive (caller layout) copied into the node records.
__global__ void k_setV(int N, const double* __restrict__ V, double* __restrict__ P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
#pragma unroll
  for (int k = 0; k < 5; ++k) P[8 * (size_t)i + k] = V[5 * (size_t)i + k];
}

// Least-squares gradients, one thread per node gathering its neighbours in
// ascending order: ddV_i = sum_j W_i(X_j - X_i) (V_j - V_i).
__global__ void k_grad(int N, const double* __restrict__ P, const double* __restrict__ lsqW,
                       const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_node,
                       const int* __restrict__ tag, double* __restrict__ G) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) w[k] = lsqW[(size_t)k * N + i];
  const double* pi = P + 8 * (size_t)i;
  double vi[5], xi[3];
#pragma unroll
  for (int k = 0; k < 5; ++k) vi[k] = pi[k];
  xi[0] = pi[5]; xi[1] = pi[6]; xi[2] = pi[7];
  double gx[5] = {0, 0, 0, 0, 0}, gy[5] = {0, 0, 0, 0, 0}, gz[5] = {0, 0, 0, 0, 0};
  const int p1 = nbr_ptr[i + 1];
  for (int p = nbr_ptr[i]; p < p1; ++p) {
    const double* pj = P + 8 * (size_t)nbr_node[p];
    double W0, W1, W2;
    lsq_weights(w, pj[5] - xi[0], pj[6] - xi[1], pj[7] - xi[2], W0, W1, W2);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double dv = pj[k] - vi[k];
      gx[k] += W0 * dv;
      gy[k] += W1 * dv;
      gz[k] += W2 * dv;
    }
  }
  const bool zero = tag && tag[i];
  double* gi = G + 16 * (size_t)i;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    gi[k] = zero ? 0.0 : gx[k];
    gi[5 + k] = zero ? 0.0 : gy[k];
    gi[10 + k] = zero ? 0.0 : gz[k];
  }
}

// Roe flux of every edge into flux[5][E].  Non-positive reconstructed
// density/pressure (VarFcnSGEuler::checkReconstructedValues,
// VarFcnSGEuler.h:90-110) skips the edge, counts into counters[0] and, with
// failsafe, tags the offending node (EdgeCore.C:137-168).
__global__ void k_edge_flux(int E, Gas g, int rec, double beta, int failsafe, const int2* __restrict__ edges,
                            const double* __restrict__ en, const double* __restrict__ P,
                            const double* __restrict__ G, double* __restrict__ flux, int* __restrict__ tag,
                            int* __restrict__ counters) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
  const int2 ij = edges[l];
  const double* pi = P + 8 * (size_t)ij.x;
  const double* pj = P + 8 * (size_t)ij.y;
  double Vi[5], Vj[5];
  if (rec == AEROF_REC_CONSTANT) {
#pragma unroll
    for (int k = 0; k < 5; ++k) { Vi[k] = pi[k]; Vj[k] = pj[k]; }
  } else {
    const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
    const double* gi = G + 16 * (size_t)ij.x;
    const double* gj = G + 16 * (size_t)ij.y;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double ddVij = dx0 * gi[k] + dx1 * gi[5 + k] + dx2 * gi[10 + k];
      double ddVji = dx0 * gj[k] + dx1 * gj[5 + k] + dx2 * gj[10 + k];
      if (rec == AEROF_REC_VANALBADA) vanalbada(beta, pi[k], ddVij, pj[k], ddVji, Vi[k], Vj[k]);
      else linear_rec(beta, pi[k], ddVij, pj[k], ddVji, Vi[k], Vj[k]);
    }
  }
  const bool bi = Vi[0] <= 0.0 || Vi[4] <= 0.0;
  const bool bj = Vj[0] <= 0.0 || Vj[4] <= 0.0;
  double f[5] = {0, 0, 0, 0, 0};
  if (bi || bj) {
    atomicAdd(&counters[0], (int)bi + (int)bj);
    if (failsafe) {
      if (bi) tag[ij.x] = 1;
      if (bj) tag[ij.y] = 1;
    }
  } else {
    const double n0 = en[l], n1 = en[(size_t)E + l], n2 = en[2 * (size_t)E + l];
    if (sqrt(n0 * n0 + n1 * n1 + n2 * n2) >= 1e-18) roe_flux(g, n0, n1, n2, Vi, Vj, f);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) flux[(size_t)k * E + l] = f[k];
}

// Per-node assembly: edges in ascending-neighbour order (+flux when the node
// is the edge's first endpoint, -flux otherwise), then boundary faces with
// subface normals n_f/3 (FaceTriaCore.C:288-308), then R *= 1/ctrlVol
// (SpaceOperator.C:614-620).  R is written in the caller's [N][5] layout.
__global__ void k_node_residual(int N, int E, Gas g, const double* __restrict__ Ub0,
                                const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                                const double* __restrict__ flux, const int* __restrict__ nf_ptr,
                                const int* __restrict__ nf_face, const int* __restrict__ fcode,
                                const double* __restrict__ fn, int F, const double* __restrict__ P,
                                const double* __restrict__ vol, double* __restrict__ R) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double acc[5] = {0, 0, 0, 0, 0};
  const int p1 = nbr_ptr[i + 1];
  for (int p = nbr_ptr[i]; p < p1; ++p) {
    const int e = nbr_edge[p];
    const size_t l = (size_t)(e & 0x7fffffff);
    if (e < 0) {
#pragma unroll
      for (int k = 0; k < 5; ++k) acc[k] -= flux[k * (size_t)E + l];
    } else {
#pragma unroll
      for (int k = 0; k < 5; ++k) acc[k] += flux[k * (size_t)E + l];
    }
  }
  const int q1 = nf_ptr[i + 1];
  if (nf_ptr[i] < q1) {
    double V[5], Ub[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { V[k] = P[8 * (size_t)i + k]; Ub[k] = Ub0[k]; }
    const double third = 1.0 / 3.0;
    for (int q = nf_ptr[i]; q < q1; ++q) {
      const int f = nf_face[q];
      double ff[5];
      face_flux(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, ff);
#pragma unroll
      for (int k = 0; k < 5; ++k) acc[k] += ff[k];
    }
  }
  const double invcv = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) R[5 * (size_t)i + k] = acc[k] * invcv;
}

// Local time step (Edge.C:87-143, Face.C:242-289, Domain.C:70-96) with beta
// = 1: each node sums min(+-un - a, 0)*S over its edges (Vmid = mean of the
// two end states) and min(un - a, 0)*S/3 over its faces; dt = cfl*vol/(-sum).
__global__ void k_timestep(int N, int E, int F, Gas g, double cfl, const int2* __restrict__ edges,
                           const double* __restrict__ en, const int* __restrict__ nbr_ptr,
                           const int* __restrict__ nbr_edge, const int* __restrict__ nf_ptr,
                           const int* __restrict__ nf_face, const double* __restrict__ fn,
                           const double* __restrict__ P, const double* __restrict__ vol,
                           double* __restrict__ dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double idti = 0.0;
  const int p1 = nbr_ptr[i + 1];
  for (int p = nbr_ptr[i]; p < p1; ++p) {
    const int e = nbr_edge[p];
    const int l = e & 0x7fffffff;
    const int2 ij = edges[l];
    const double* pa = P + 8 * (size_t)ij.x;
    const double* pb = P + 8 * (size_t)ij.y;
    const double n0 = en[l], n1 = en[(size_t)E + l], n2 = en[2 * (size_t)E + l];
    double S = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    double invS = 1.0 / S;
    double vm0 = 0.5 * (pa[0] + pb[0]);
    double vm1 = 0.5 * (pa[1] + pb[1]);
    double vm2 = 0.5 * (pa[2] + pb[2]);
    double vm3 = 0.5 * (pa[3] + pb[3]);
    double vm4 = 0.5 * (pa[4] + pb[4]);
    double a = sqrt(g.gam * vm4 / vm0);
    double un = vm1 * (invS * n0) + vm2 * (invS * n1) + vm3 * (invS * n2);
    double coeff1 = 2.0 * un;
    double coeff2 = sqrt(2.0 * a * (2.0 * a));
    double c = (e < 0) ? 0.5 * (-coeff1 - coeff2) : 0.5 * (coeff1 - coeff2);
    idti += fmin(c, 0.0) * S;
  }
  const int q1 = nf_ptr[i + 1];
  if (nf_ptr[i] < q1) {
    const double* pi = P + 8 * (size_t)i;
    double a = sqrt(g.gam * pi[4] / pi[0]);
    for (int q = nf_ptr[i]; q < q1; ++q) {
      const int f = nf_face[q];
      const double n0 = fn[f], n1 = fn[(size_t)F + f], n2 = fn[2 * (size_t)F + f];
      double S = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
      double invS = 1.0 / S;
      double un = pi[1] * (invS * n0) + pi[2] * (invS * n1) + pi[3] * (invS * n2);
      double coeff1 = 2.0 * un;
      double coeff2 = sqrt(2.0 * a * (2.0 * a));
      idti += fmin(0.5 * (coeff1 - coeff2), 0.0) * S / 3;
    }
  }
  dt[i] = cfl * vol[i] / (-1.0 * idti);
}

// RK2 stage helpers (ExplicitTsDesc.C:98-117): k = dt*R; U0 = U - k1;
// U = U - 1/2 (k1 + k2).
__global__ void k_rk_stage1(int N, const double* __restrict__ dt, const double* __restrict__ U,
                            double* __restrict__ k1, double* __restrict__ U0) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 5 * (size_t)N) return;
  double k = k1[q] * dt[q / 5];
  k1[q] = k;
  U0[q] = U[q] - k;
}
__global__ void k_rk_stage2(int N, const double* __restrict__ dt, const double* __restrict__ k1,
                            const double* __restrict__ k2, double* __restrict__ U) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 5 * (size_t)N) return;
  double kk = k2[q] * dt[q / 5];
  U[q] = U[q] - 1.0 / 2.0 * (k1[q] + kk);
}

// Deterministic dot product: fixed grid, fixed per-block tree, then one block
// sums the partials in order.
__global__ void k_dot_partial(size_t n, const double* __restrict__ x, const double* __restrict__ y,
                              double* __restrict__ part) {
  __shared__ double sh[kBlock];
  double s = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    s += x[q] * y[q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_dot_final(int nb, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[kBlock];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

// ------------------------------------------------------------------ host side
void prim_dev(aerof_gpu_ctx* c, const double* dU) {
  DeviceMesh& m = c->mesh;
  k_prim<<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(m.N, make_gas(c->cfg.gamma), dU, m.P.p);
  AEROF_LAUNCH_CHECK();
}

void gradients_dev(aerof_gpu_ctx* c) {
  DeviceMesh& m = c->mesh;
  c->s.G.ensure(16 * (size_t)m.N);
  k_grad<<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(m.N, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
                                                          nullptr, c->s.G.p);
  AEROF_LAUNCH_CHECK();
}

static int* counters(aerof_gpu_ctx* c) {
  c->s.counters.ensure(8);
  return c->s.counters.p;
}

// Residual of device state dU into device dR (both [N][5]).  Returns the
// number of non-positive reconstructed states of the first pass (sync), or
// 0 with the count accumulated in counters[2] (no sync, failsafe off).
int residual_dev(aerof_gpu_ctx* c, const double* dU, double* dR, bool sync) {
  DeviceMesh& m = c->mesh;
  const Gas g = make_gas(c->cfg.gamma);
  const int rec = c->cfg.reconstruction;
  int* cnt = counters(c);
  if (sync) AEROF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * 2, c->stream));
  int* ecnt = sync ? cnt : cnt + 2;
  c->s.flux.ensure(5 * (size_t)m.E);
  c->s.G.ensure(16 * (size_t)m.N);
  if (c->cfg.failsafe) {
    c->s.tag.ensure(m.N);
    c->s.tag.zero(c->stream);
  }
  {
    TimerScope t(c, AEROF_T_NODAL_GRAD);
    prim_dev(c, dU);
    if (rec != AEROF_REC_CONSTANT) gradients_dev(c);
  }
  {
    TimerScope t(c, AEROF_T_FV_TERM);
    k_edge_flux<<<grid_for(m.E, kBlock), kBlock, 0, c->stream>>>(
        m.E, g, rec, c->cfg.beta, c->cfg.failsafe, m.edges.p, m.en.p, m.P.p, c->s.G.p, c->s.flux.p,
        c->s.tag.p, ecnt);
    AEROF_LAUNCH_CHECK();
  }
  int bad = 0;
  if (sync) {
    AEROF_CUDA(cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
  }
  if (bad && c->cfg.failsafe && rec != AEROF_REC_CONSTANT) {
    // Domain.C:886-918: zero the gradients of tagged nodes and recompute.
    TimerScope t(c, AEROF_T_FV_TERM);
    k_grad<<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(m.N, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
                                                            c->s.tag.p, c->s.G.p);
    AEROF_LAUNCH_CHECK();
    k_edge_flux<<<grid_for(m.E, kBlock), kBlock, 0, c->stream>>>(
        m.E, g, rec, c->cfg.beta, 0, m.edges.p, m.en.p, m.P.p, c->s.G.p, c->s.flux.p, c->s.tag.p, cnt + 1);
    AEROF_LAUNCH_CHECK();
  }
  {
    TimerScope t(c, AEROF_T_FV_TERM);
    k_node_residual<<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(
        m.N, m.E, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_edge.p,
        c->s.flux.p, m.nf_ptr.p, m.nf_face.p, m.fcode.p, m.fnrm.p, m.F, m.P.p, m.vol.p, dR);
    AEROF_LAUNCH_CHECK();
  }
  return bad;
}

void timestep_dev(aerof_gpu_ctx* c, const double* dU, double cfl, double* ddt) {
  DeviceMesh& m = c->mesh;
  TimerScope t(c, AEROF_T_TIME_STEP);
  prim_dev(c, dU);
  k_timestep<<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(
      m.N, m.E, m.F, make_gas(c->cfg.gamma), cfl, m.edges.p, m.en.p, m.nbr_ptr.p, m.nbr_edge.p, m.nf_ptr.p,
      m.nf_face.p, m.fnrm.p, m.P.p, m.vol.p, ddt);
  AEROF_LAUNCH_CHECK();
}

double dot_dev(aerof_gpu_ctx* c, const double* x, const double* y, size_t n) {
  c->s.red.ensure(kRedBlocks);
  c->s.redout.ensure(8);
  k_dot_partial<<<kRedBlocks, kBlock, 0, c->stream>>>(n, x, y, c->s.red.p);
  AEROF_LAUNCH_CHECK();
  k_dot_final<<<1, kBlock, 0, c->stream>>>(kRedBlocks, c->s.red.p, c->s.redout.p);
  AEROF_LAUNCH_CHECK();
  double r = 0.0;
  AEROF_CUDA(cudaMemcpyAsync(&r, c->s.redout.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  AEROF_CUDA(cudaStreamSynchronize(c->stream));
  return r;
}

double norm2_dev(aerof_gpu_ctx* c, const double* x, size_t n) { return sqrt(dot_dev(c, x, x, n)); }

}  // namespace aerof

using namespace aerof;

static int need_mesh(aerof_gpu_ctx* c) {
  if (!c->has_mesh) {
    c->last_error = "no mesh: call aerof_gpu_set_mesh first";
    return AEROF_ESTATE;
  }
  return AEROF_OK;
}

extern "C" int aerof_gpu_residual(aerof_gpu_ctx* c, const double* U, double* R) {
  return guard(c, [&]() -> int {
    if (int e = need_mesh(c)) return e;
    if (!U || !R) return AEROF_EINVAL;
    const size_t n5 = 5 * (size_t)c->mesh.N;
    const double* dU = in_dev(c, U, n5, c->s.Ustage);
    double* dR = out_dev(c, R, n5, c->s.Rstage);
    int bad = residual_dev(c, dU, dR);
    out_finish(c, R, dR, n5);
    return bad;
  });
}

extern "C" int aerof_gpu_residual_async(aerof_gpu_ctx* c, const double* U, double* R) {
  return guard(c, [&]() -> int {
    if (int e = need_mesh(c)) return e;
    if (!U || !R || c->cfg.failsafe) return AEROF_EINVAL;
    if (!is_device_ptr(U) || !is_device_ptr(R)) {
      c->last_error = "aerof_gpu_residual_async needs device pointers";
      return AEROF_EINVAL;
    }
    if (c->s.counters.n == 0) {
      counters(c);
      AEROF_CUDA(cudaMemsetAsync(c->s.counters.p, 0, sizeof(int) * 8, c->stream));
    }
    residual_dev(c, U, R, false);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_status(aerof_gpu_ctx* c) {
  return guard(c, [&]() -> int {
    int bad = 0;
    if (c->s.counters.n) {
      AEROF_CUDA(cudaMemcpyAsync(&bad, c->s.counters.p + 2, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaMemsetAsync(c->s.counters.p + 2, 0, sizeof(int), c->stream));
    }
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    return bad;
  });
}

extern "C" int aerof_gpu_gradients(aerof_gpu_ctx* c, const double* V, double* ddx, double* ddy, double* ddz) {
  return guard(c, [&]() -> int {
    if (int e = need_mesh(c)) return e;
    if (!V || !ddx || !ddy || !ddz) return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    const size_t n5 = 5 * (size_t)m.N;
    const double* dV = in_dev(c, V, n5, c->s.Vstage);
    k_setV<<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(m.N, dV, m.P.p);
    AEROF_LAUNCH_CHECK();
    gradients_dev(c);
    std::vector<double> G(16 * (size_t)m.N);
    AEROF_CUDA(cudaMemcpyAsync(G.data(), c->s.G.p, G.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    std::vector<double> hx(n5), hy(n5), hz(n5);
    for (int i = 0; i < m.N; ++i)
      for (int k = 0; k < 5; ++k) {
        hx[5 * (size_t)i + k] = G[16 * (size_t)i + k];
        hy[5 * (size_t)i + k] = G[16 * (size_t)i + 5 + k];
        hz[5 * (size_t)i + k] = G[16 * (size_t)i + 10 + k];
      }
    double* outs[3] = {ddx, ddy, ddz};
    std::vector<double>* src[3] = {&hx, &hy, &hz};
    for (int a = 0; a < 3; ++a) {
      if (is_device_ptr(outs[a]))
        AEROF_CUDA(cudaMemcpyAsync(outs[a], src[a]->data(), n5 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      else
        std::copy(src[a]->begin(), src[a]->end(), outs[a]);
    }
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_timestep(aerof_gpu_ctx* c, const double* U, double cfl, double* dt) {
  return guard(c, [&]() -> int {
    if (int e = need_mesh(c)) return e;
    if (!U || !dt || !(cfl > 0.0)) return AEROF_EINVAL;
    const size_t N = c->mesh.N;
    const double* dU = in_dev(c, U, 5 * N, c->s.Ustage);
    double* ddt = out_dev(c, dt, N, c->s.Rstage);
    timestep_dev(c, dU, cfl, ddt);
    out_finish(c, dt, ddt, N);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_rk2(aerof_gpu_ctx* c, double* U, double cfl, int nsteps) {
  return guard(c, [&]() -> int {
    if (int e = need_mesh(c)) return e;
    if (!U || nsteps < 0 || !(cfl > 0.0)) return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    const size_t n5 = 5 * (size_t)m.N;
    // U is read and written: stage in/out through Ustage when on the host
    double* dU;
    if (is_device_ptr(U)) dU = U;
    else {
      c->s.Ustage.ensure(n5);
      AEROF_CUDA(cudaMemcpyAsync(c->s.Ustage.p, U, n5 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      dU = c->s.Ustage.p;
    }
    c->s.dt.ensure(m.N); c->s.k1.ensure(n5); c->s.k2.ensure(n5); c->s.U0.ensure(n5);
    int bad = 0;
    const int gb = grid_for(n5, kBlock);
    for (int s = 0; s < nsteps; ++s) {
      timestep_dev(c, dU, cfl, c->s.dt.p);
      bad += residual_dev(c, dU, c->s.k1.p);
      k_rk_stage1<<<gb, kBlock, 0, c->stream>>>(m.N, c->s.dt.p, dU, c->s.k1.p, c->s.U0.p);
      AEROF_LAUNCH_CHECK();
      bad += residual_dev(c, c->s.U0.p, c->s.k2.p);
      k_rk_stage2<<<gb, kBlock, 0, c->stream>>>(m.N, c->s.dt.p, c->s.k1.p, c->s.k2.p, dU);
      AEROF_LAUNCH_CHECK();
    }
    if (dU != U)
      AEROF_CUDA(cudaMemcpyAsync(U, dU, n5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    return bad;
  });
}
