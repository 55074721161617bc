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
#include <cstdlib>
#include <cstring>

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

// Least-squares gradients, ddV_i = sum_j W_i(X_j - X_i) (V_j - V_i), with
// four lanes per node: lane r of a node's group takes the neighbours at
// positions r, r+4, ... of the node's ascending neighbour list, then the
// four partial sums are added in a fixed tree (lanes 0+1, 2+3, then both).
__device__ __forceinline__ void load_rec(const double* __restrict__ P, int j, double* r) {
  const double2* q = reinterpret_cast<const double2*>(P + 8 * (size_t)j);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double2 v = __ldg(q + k);
    r[2 * k] = v.x;
    r[2 * k + 1] = v.y;
  }
}
__device__ __forceinline__ void grad_acc(const double* w, const double* vi, const double* xi, const double* pj,
                                         double* gx, double* gy, double* gz) {
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
__global__ void __launch_bounds__(256) k_grad(int N, const double* __restrict__ P, const double* __restrict__ lsqW,
                                              const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_node,
                                              const int* __restrict__ tag, double* __restrict__ G) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t >> 2, r = t & 3;
  const bool act = i < N;
  double g[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) g[k] = 0.0;
  if (act) {
    double w[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = lsqW[(size_t)k * N + i];
    double pi[8];
    load_rec(P, i, pi);
    const int p1 = nbr_ptr[i + 1];
    for (int p = nbr_ptr[i] + r; p < p1; p += 4) {
      double pj[8];
      load_rec(P, nbr_node[p], pj);
      grad_acc(w, pi, pi + 5, pj, g, g + 5, g + 10);
    }
  }
  // fixed-order combination of the four partial sums
#pragma unroll
  for (int k = 0; k < 15; ++k) {
    g[k] += __shfl_xor_sync(0xffffffffu, g[k], 1);
    g[k] += __shfl_xor_sync(0xffffffffu, g[k], 2);
  }
  if (!act) return;
  const bool zero = tag && tag[i];
  // lane r stores doubles 4r..4r+3 of the node's 128-byte record (the
  // selection uses constant indices only, so g stays in registers)
  double o[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double v = 0.0;
#pragma unroll
    for (int rr = 0; rr < 4; ++rr)
      if (4 * rr + q < 15 && r == rr) v = g[4 * rr + q < 15 ? 4 * rr + q : 0];
    o[q] = zero ? 0.0 : v;
  }
  double2* gi = reinterpret_cast<double2*>(G + 16 * (size_t)i);
  gi[2 * r] = make_double2(o[0], o[1]);
  gi[2 * r + 1] = make_double2(o[2], o[3]);
}


// BLOCKED organisation: least-squares gradients of one Morton block of NB
// nodes per CTA.  The CTA stages the node records (V, X) of its own nodes
// and of its halo (every neighbour outside the block) in shared memory,
// then forms the gradients of its own nodes from shared memory only.
// FUSED: the records are built from U (caller numbering) by the primitive
// conversion, and V of the own nodes is written to P2 for the flux kernels;
// otherwise P2 already holds V and the records are copied with cp.async.
// L = blockDim / NB lanes share a node and take the neighbours at positions
// r, r+L, ...; their partial sums are added in a fixed shuffle tree.
// Staging is one pass of independent loads, so the gather latency is paid
// once per block instead of once per neighbour.
// P2 is read (X, never written here) and written (V of own nodes only).
__device__ __forceinline__ void stage_record(Gas g, const int* __restrict__ n2o, const double* __restrict__ U,
                                             double* P2, int j, double* rec, bool own) {
  const int o = n2o[j];
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = __ldg(U + 5 * (size_t)o + k);
  const double x0 = P2[8 * (size_t)j + 5], x1 = P2[8 * (size_t)j + 6], x2 = P2[8 * (size_t)j + 7];
  cons2prim(g, u, v);
  double2* r2 = reinterpret_cast<double2*>(rec);
  r2[0] = make_double2(v[0], v[1]);
  r2[1] = make_double2(v[2], v[3]);
  r2[2] = make_double2(v[4], x0);
  r2[3] = make_double2(x1, x2);
  if (own) {
#pragma unroll
    for (int k = 0; k < 5; ++k) P2[8 * (size_t)j + k] = v[k];
  }
}

template <int L, bool FUSED>
__global__ void __launch_bounds__(256, 3) k_grad_staged(int N, int NB, Gas g, const int* __restrict__ n2o,
                                                     const double* __restrict__ U, double* P2,
                                                     const double* __restrict__ W2, const int* __restrict__ nb2_ptr,
                                                     const unsigned short* __restrict__ lnb,
                                                     const int* __restrict__ hptr, const int* __restrict__ hnode,
                                                     const int* __restrict__ tag, double* __restrict__ G2) {
  extern __shared__ double sm[];
  const int blk = blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int h0 = hptr[blk], nh = hptr[blk + 1] - h0;
  const int c0 = nb2_ptr[n0], nc = nb2_ptr[n0 + nn] - c0;
  double* rec = sm;                                                        // [nn + nh][kPS]
  unsigned short* ls = reinterpret_cast<unsigned short*>(rec + kPS * (size_t)(nn + nh));  // [nc]
  const int t = threadIdx.x / L, r = threadIdx.x % L;
  const bool act = t < nn;
  // the thread's own node data is requested before the staging completes
  double w[6];
  int pb = 0, pe = 0;
  if (act) {
    const int i = n0 + t;
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = W2[(size_t)k * N + i];
    pb = nb2_ptr[i] - c0;
    pe = nb2_ptr[i + 1] - c0;
  }
  for (int k = threadIdx.x; k < nc; k += blockDim.x) ls[k] = lnb[c0 + k];
  if (FUSED) {
    for (int t = threadIdx.x; t < nn + nh; t += blockDim.x) {
      const bool own = t < nn;
      stage_record(g, n2o, U, P2, own ? n0 + t : hnode[h0 + t - nn], rec + kPS * t, own);
    }
  } else {
    const double2* ps = reinterpret_cast<const double2*>(P2 + 8 * (size_t)n0);
    double2* pd = reinterpret_cast<double2*>(rec);
    for (int k = threadIdx.x; k < 4 * nn; k += blockDim.x) cp_async16(pd + (kPS / 2) * (k >> 2) + (k & 3), ps + k);
    for (int k = threadIdx.x; k < 4 * nh; k += blockDim.x) {
      const int j = hnode[h0 + (k >> 2)];
      cp_async16(pd + (kPS / 2) * (nn + (k >> 2)) + (k & 3),
                 reinterpret_cast<const double2*>(P2 + 8 * (size_t)j) + (k & 3));
    }
    cp_async_wait_all();
  }
  __syncthreads();
  double gs[15];
#pragma unroll
  for (int k = 0; k < 15; ++k) gs[k] = 0.0;
  if (act) {
    double pi[8];
    const double2* qi = reinterpret_cast<const double2*>(rec + kPS * t);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2 v = qi[k];
      pi[2 * k] = v.x;
      pi[2 * k + 1] = v.y;
    }
#pragma unroll 1
    for (int p = pb + r; p < pe; p += L) {
      double pj[8];
      const double2* qj = reinterpret_cast<const double2*>(rec + kPS * (int)ls[p]);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double2 v = qj[k];
        pj[2 * k] = v.x;
        pj[2 * k + 1] = v.y;
      }
      grad_acc(w, pi, pi + 5, pj, gs, gs + 5, gs + 10);
    }
  }
#pragma unroll
  for (int k = 0; k < 15; ++k) {
    if (L > 1) gs[k] += __shfl_xor_sync(0xffffffffu, gs[k], 1);
    if (L > 2) gs[k] += __shfl_xor_sync(0xffffffffu, gs[k], 2);
  }
  if (!act) return;
  const int i = n0 + t;
  const bool zero = tag && tag[i];
  // lane r stores doubles (16/L) r .. (16/L)(r+1)-1 of the 128-byte record
  constexpr int S = 16 / L;
  double o[S];
#pragma unroll
  for (int q = 0; q < S; ++q) {
    double v = 0.0;
#pragma unroll
    for (int rr = 0; rr < L; ++rr)
      if (S * rr + q < 15 && r == rr) v = gs[S * rr + q < 15 ? S * rr + q : 0];
    o[q] = zero ? 0.0 : v;
  }
  double2* gi = reinterpret_cast<double2*>(G2 + 16 * (size_t)i + S * r);
#pragma unroll
  for (int q = 0; q < S / 2; ++q) gi[q] = make_double2(o[2 * q], o[2 * q + 1]);
}


// Shared-memory stage of the pipelined gradient kernel (offsets in doubles,
// all even so that every part is 16-byte aligned).
struct GradStage {
  int rec, w, ptr, ls, size;
};

// Persistent, software-pipelined form of the staged gradient kernel: each
// CTA walks the blocks blockIdx.x, + gridDim.x, ... and, while it forms the
// gradients of one block from shared memory, the asynchronous copies of the
// next block's node records (own and halo), LSQ constants, neighbour
// pointers and local neighbour slots are in flight into the other stage.
// The halo ids of the block after that are loaded into registers one
// iteration ahead, so no copy waits on a dependent load.  Halo of at most
// 512 nodes (two records per thread).
template <int L>
__global__ void __launch_bounds__(256, 2) k_grad_pipe(int N, int NB, int nblk, int maxH, int maxLp, GradStage st,
                                                      const double* __restrict__ P2, const double* __restrict__ W2,
                                                      const int* __restrict__ nb2_ptr,
                                                      const unsigned short* __restrict__ lpad,
                                                      const int* __restrict__ hpad, const int* __restrict__ tag,
                                                      double* __restrict__ G2, const int* __restrict__ blist) {
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  auto load_ids = [&](int b, int& a0, int& a1) {
    a0 = tid < maxH ? hpad[(size_t)b * maxH + tid] : -1;
    a1 = tid + 256 < maxH ? hpad[(size_t)b * maxH + tid + 256] : -1;
  };
  auto issue = [&](int b, double* S, int a0, int a1) {
    const int n0 = b * NB, nn = min(NB, N - n0);
    double2* rec = reinterpret_cast<double2*>(S + st.rec);
    const double2* ps = reinterpret_cast<const double2*>(P2 + 8 * (size_t)n0);
    for (int k = tid; k < 4 * nn; k += blockDim.x) cp_async16(rec + (kPS / 2) * (k >> 2) + (k & 3), ps + k);
    if (a0 >= 0) {
      const double2* src = reinterpret_cast<const double2*>(P2 + 8 * (size_t)a0);
#pragma unroll
      for (int c = 0; c < 4; ++c) cp_async16(rec + (kPS / 2) * (nn + tid) + c, src + c);
    }
    if (a1 >= 0) {
      const double2* src = reinterpret_cast<const double2*>(P2 + 8 * (size_t)a1);
#pragma unroll
      for (int c = 0; c < 4; ++c) cp_async16(rec + (kPS / 2) * (nn + tid + 256) + c, src + c);
    }
    // every copy below loops over the block's extent: a segment may be
    // longer than one copy per thread (the local slots of a 256-node block
    // are ~3600 entries, 16-byte copies carry 8)
    for (int k = tid; k < nn; k += blockDim.x) {
#pragma unroll
      for (int a = 0; a < 6; ++a) cp_async8(S + st.w + a * NB + k, W2 + (size_t)a * N + n0 + k);
    }
    for (int k = tid; 4 * k < nn + 1; k += blockDim.x) cp_async16(S + st.ptr + 2 * k, nb2_ptr + n0 + 4 * k);
    for (int k = tid; 8 * k < maxLp; k += blockDim.x) cp_async16(S + st.ls + 2 * k, lpad + (size_t)b * maxLp + 8 * k);
  };
  // blocks blist[0, nblk) (all blocks in order when blist is null)
  auto bid = [&](int i) { return blist ? blist[i] : i; };
  int i = blockIdx.x;
  if (i >= nblk) return;
  int a0, a1;
  load_ids(bid(i), a0, a1);
  issue(bid(i), sm, a0, a1);
  cp_async_commit();
  if (i + (int)gridDim.x < nblk) load_ids(bid(i + gridDim.x), a0, a1);
  for (int k = 0; i < nblk; ++k, i += gridDim.x) {
    const int b = bid(i);
    const int in = i + gridDim.x;
    if (in < nblk) issue(bid(in), sm + ((k + 1) & 1) * st.size, a0, a1);
    cp_async_commit();
    if (in + (int)gridDim.x < nblk) load_ids(bid(in + gridDim.x), a0, a1);
    cp_async_wait_prev();
    __syncthreads();
    const double* S = sm + (k & 1) * st.size;
    const double* rec = S + st.rec;
    const int* ptr = reinterpret_cast<const int*>(S + st.ptr);
    const unsigned short* ls = reinterpret_cast<const unsigned short*>(S + st.ls);
    const int n0 = b * NB, nn = min(NB, N - n0);
    const int t = tid / L, r = tid % L;
    const bool act = t < nn;
    double gs[15];
#pragma unroll
    for (int q = 0; q < 15; ++q) gs[q] = 0.0;
    if (act) {
      double w[6], pi[8];
#pragma unroll
      for (int a = 0; a < 6; ++a) w[a] = S[st.w + a * NB + t];
      const double2* qi = reinterpret_cast<const double2*>(rec + kPS * t);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 v = qi[q];
        pi[2 * q] = v.x;
        pi[2 * q + 1] = v.y;
      }
      const int c0 = ptr[0], pe = ptr[t + 1] - c0;
#pragma unroll 1
      for (int p = ptr[t] - c0 + r; p < pe; p += L) {
        double pj[8];
        const double2* qj = reinterpret_cast<const double2*>(rec + kPS * (int)ls[p]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double2 v = qj[q];
          pj[2 * q] = v.x;
          pj[2 * q + 1] = v.y;
        }
        grad_acc(w, pi, pi + 5, pj, gs, gs + 5, gs + 10);
      }
    }
#pragma unroll
    for (int q = 0; q < 15; ++q) {
      if (L > 1) gs[q] += __shfl_xor_sync(0xffffffffu, gs[q], 1);
      if (L > 2) gs[q] += __shfl_xor_sync(0xffffffffu, gs[q], 2);
    }
    if (act) {
      const int i = n0 + t;
      const bool zero = tag && tag[i];
      constexpr int SL = 16 / L;
      double o[SL];
#pragma unroll
      for (int q = 0; q < SL; ++q) {
        double v = 0.0;
#pragma unroll
        for (int rr = 0; rr < L; ++rr)
          if (SL * rr + q < 15 && r == rr) v = gs[SL * rr + q < 15 ? SL * rr + q : 0];
        o[q] = zero ? 0.0 : v;
      }
      double2* gi = reinterpret_cast<double2*>(G2 + 16 * (size_t)i + SL * r);
#pragma unroll
      for (int q = 0; q < SL / 2; ++q) gi[q] = make_double2(o[2 * q], o[2 * q + 1]);
    }
    __syncthreads();
  }
}

// Flux of one edge (i = first, j = second endpoint): reconstruction from the
// node records and gradients, positivity check (VarFcnSGEuler::
// checkReconstructedValues, VarFcnSGEuler.h:90-110; on failure the edge is
// skipped as in Edge.C:414-421, counted, and with failsafe the offending
// node tagged, EdgeCore.C:137-168), then the Roe flux.
__device__ __forceinline__ void edge_flux_rec(const Gas& g, int rec, double beta, int failsafe, int i, int j,
                                              double n0, double n1, double n2, const double* pi, const double* gi,
                                              const double* pj, const double* gj, int* __restrict__ tag,
                                              int* __restrict__ counter, double* f) {
  double Vi[5], Vj[5];
  if (rec == AEROF_REC_CONSTANT) {
#pragma unroll
    for (int k = 0; k < 5; ++k) { Vi[k] = pi[k]; Vj[k] = pj[k]; }
  } else {
    const double dx0 = pj[5] - pi[5], dx1 = pj[6] - pi[6], dx2 = pj[7] - pi[7];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double ddVij = dx0 * gi[k] + dx1 * gi[5 + k] + dx2 * gi[10 + k];
      double ddVji = dx0 * gj[k] + dx1 * gj[5 + k] + dx2 * gj[10 + k];
      if (rec == AEROF_REC_VANALBADA) vanalbada(beta, pi[k], ddVij, pj[k], ddVji, Vi[k], Vj[k]);
      else linear_rec(beta, pi[k], ddVij, pj[k], ddVji, Vi[k], Vj[k]);
    }
  }
  // written as !(x > 0) so that a non-finite state counts as unphysical too
  const bool bi = !(Vi[0] > 0.0) || !(Vi[4] > 0.0);
  const bool bj = !(Vj[0] > 0.0) || !(Vj[4] > 0.0);
#pragma unroll
  for (int k = 0; k < 5; ++k) f[k] = 0.0;
  if (bi || bj) {
    atomicAdd(counter, (int)bi + (int)bj);
    if (failsafe) {
      if (bi) tag[i] = 1;
      if (bj) tag[j] = 1;
    }
  } else if (n0 * n0 + n1 * n1 + n2 * n2 >= 1e-36) {
    roe_flux(g, n0, n1, n2, Vi, Vj, f);
  }
}
__device__ __forceinline__ void edge_flux_eval(const Gas& g, int rec, double beta, int failsafe, int i, int j,
                                               double n0, double n1, double n2, const double* __restrict__ P,
                                               const double* __restrict__ G, int* __restrict__ tag,
                                               int* __restrict__ counter, double* f) {
  edge_flux_rec(g, rec, beta, failsafe, i, j, n0, n1, n2, P + 8 * (size_t)i, G + 16 * (size_t)i, P + 8 * (size_t)j,
                G + 16 * (size_t)j, tag, counter, f);
}

// Roe flux of every edge into flux[5][E] (EDGE organisation).
__global__ void k_edge_flux(int E, Gas g, int rec, double beta, int failsafe, const int2* __restrict__ edges,
                            const double* __restrict__ en, const double* __restrict__ P,
                            const double* __restrict__ G, double* __restrict__ flux, int* __restrict__ tag,
                            int* __restrict__ counters) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
  const int2 ij = edges[l];
  double f[5];
  edge_flux_eval(g, rec, beta, failsafe, ij.x, ij.y, en[l], en[(size_t)E + l], en[2 * (size_t)E + l], P, G, tag,
                 counters, f);
#pragma unroll
  for (int k = 0; k < 5; ++k) flux[(size_t)k * E + l] = f[k];
}

// BLOCKED organisation: one thread block per NB consecutive (Morton
// ordered) nodes.  Phase 0: the node records (V, X) and gradients of the
// block's nodes and of its forward halo (second endpoints of the block's
// edges that lie in later blocks) are copied to shared memory with
// asynchronous 16-byte copies.  Phase 1: the block's threads evaluate the
// fluxes of the edges whose first endpoint is in the block, every operand
// from shared memory (bl[q] = the two endpoints as staged slots), into
// shared memory; fluxes of edges whose second endpoint lies in a later
// block also go to spill[].  Phase 2: thread t sums, for node blk*NB+t, its
// edges held in shared memory in ascending edge order (+ as first endpoint,
// - as second) into part[].
template <int THREADS, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    k_fv_blocked(int N, int E, int NB, Gas g, int rec, double beta, int failsafe,
                                                    const ushort2* __restrict__ bl, const double* __restrict__ bn,
                                                    const int* __restrict__ beptr, const int* __restrict__ hfptr,
                                                    const int* __restrict__ hfpad, int maxHf,
                                                    const double* __restrict__ P,
                                                    const double* __restrict__ G, const int* __restrict__ lptr,
                                                    const int* __restrict__ lidx, const int* __restrict__ xslot,
                                                    double* __restrict__ part, double* __restrict__ spill,
                                                    int* __restrict__ tag, int* __restrict__ counters,
                                                    const int* __restrict__ blist) {
  extern __shared__ double sm[];
  const int blk = blist ? blist[blockIdx.x] : blockIdx.x;
  const int n0 = blk * NB;
  const int nn = min(NB, N - n0);
  const int h0 = hfptr[blk], nh = hfptr[blk + 1] - h0;
  const int ns = nn + nh;
  const int e0 = beptr[blk], e1 = beptr[blk + 1];
  // phase 2: L lanes per node (the largest power of two with NB L <= the
  // block's threads); the node's list bounds are requested now
  int L = 1;
  while (2 * L * NB <= (int)blockDim.x) L *= 2;
  const int t2 = threadIdx.x / L, r2 = threadIdx.x % L;
  const bool act2 = t2 < nn && (int)threadIdx.x < L * NB;
  const int lb = act2 ? lptr[n0 + t2] : 0, le = act2 ? lptr[n0 + t2 + 1] : 0;
  double* Pn = sm;                      // [ns][kPS]
  double* Gn = sm + kPS * ns;           // [ns][kGS]
  double* Fs = sm + (kPS + kGS) * ns;   // [e1 - e0][5]
  int* hs = reinterpret_cast<int*>(Fs + 5 * (e1 - e0));  // [nh] halo node ids
  const int* hf = hfpad + (size_t)blk * maxHf;            // addresses from the block index alone
  for (int k = threadIdx.x; k < nh; k += blockDim.x) hs[k] = hf[k];
  {
    const bool grad = rec != AEROF_REC_CONSTANT;
    // own nodes: contiguous records
    const double2* ps = reinterpret_cast<const double2*>(P + 8 * (size_t)n0);
    const double2* gs = reinterpret_cast<const double2*>(G + 16 * (size_t)n0);
    double2* pd = reinterpret_cast<double2*>(Pn);
    double2* gd = reinterpret_cast<double2*>(Gn);
    for (int k = threadIdx.x; k < 4 * nn; k += blockDim.x) cp_async16(pd + (kPS / 2) * (k >> 2) + (k & 3), ps + k);
    if (grad)
      for (int k = threadIdx.x; k < 8 * nn; k += blockDim.x)
        cp_async16(gd + (kGS / 2) * (k >> 3) + (k & 7), gs + k);
    // forward halo: one 64 B and one 128 B record per node
    for (int k = threadIdx.x; k < 4 * nh; k += blockDim.x) {
      const int j = hf[k >> 2];
      cp_async16(pd + (kPS / 2) * (nn + (k >> 2)) + (k & 3),
                 reinterpret_cast<const double2*>(P + 8 * (size_t)j) + (k & 3));
    }
    if (grad)
      for (int k = threadIdx.x; k < 8 * nh; k += blockDim.x) {
        const int j = hf[k >> 3];
        cp_async16(gd + (kGS / 2) * (nn + (k >> 3)) + (k & 7),
                   reinterpret_cast<const double2*>(G + 16 * (size_t)j) + (k & 7));
      }
  }
  // the edge data of each iteration is requested one iteration ahead (the
  // first before the staging completes)
  int q = e0 + threadIdx.x;
  ushort2 lq = make_ushort2(0, 0);
  double nx = 0.0, ny = 0.0, nz = 0.0;
  int xs = -1;
  if (q < e1) {
    lq = bl[q];
    nx = bn[q]; ny = bn[(size_t)E + q]; nz = bn[2 * (size_t)E + q];
    xs = xslot[q];
  }
  cp_async_wait_all();
  __syncthreads();
  for (; q < e1; q += blockDim.x) {
    const int qn = q + blockDim.x;
    ushort2 lqn = make_ushort2(0, 0);
    double nxn = 0.0, nyn = 0.0, nzn = 0.0;
    int xsn = -1;
    if (qn < e1) {
      lqn = bl[qn];
      nxn = bn[qn]; nyn = bn[(size_t)E + qn]; nzn = bn[2 * (size_t)E + qn];
      xsn = xslot[qn];
    }
    const int li = lq.x, lj = lq.y;
    double f[5];
    // global node ids are needed only to tag unphysical states
    const int gi = n0 + li, gj = lj < nn ? n0 + lj : hs[lj - nn];
    edge_flux_rec(g, rec, beta, failsafe, gi, gj, nx, ny, nz, Pn + kPS * li, Gn + kGS * li, Pn + kPS * lj,
                  Gn + kGS * lj, tag, counters, f);
    double* fs = Fs + 5 * (q - e0);
#pragma unroll
    for (int k = 0; k < 5; ++k) fs[k] = f[k];
    if (xs >= 0) {
#pragma unroll
      for (int k = 0; k < 5; ++k) spill[5 * (size_t)xs + k] = f[k];
    }
    lq = lqn; nx = nxn; ny = nyn; nz = nzn; xs = xsn;
  }
  // the first kLI entries of this lane's part of the node's list are
  // requested before the barrier, the rest (long lists only) after it
  constexpr int kLI = 8;
  int li_pre[kLI];
#pragma unroll
  for (int m = 0; m < kLI; ++m) {
    const int k = lb + r2 + m * L;
    li_pre[m] = k < le ? lidx[k] : 0;
  }
  __syncthreads();
  // L lanes per node take entries r, r+L, ... of its list; the partial sums
  // are combined in a fixed xor tree
  const int n = n0 + t2;
  double acc[5] = {0, 0, 0, 0, 0};
  auto add = [&](int e) {
    const double* fs = Fs + 5 * (e & 0x7fffffff);
    if (e < 0) {
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[c] -= fs[c];
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[c] += fs[c];
    }
  };
#pragma unroll
  for (int m = 0; m < kLI; ++m)
    if (lb + r2 + m * L < le) add(li_pre[m]);
  for (int k = lb + r2 + kLI * L; k < le; k += L) add(lidx[k]);
  for (int o = 1; o < L; o <<= 1) {
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  }
  if (act2 && r2 == 0) {
#pragma unroll
    for (int c = 0; c < 5; ++c) part[5 * (size_t)n + c] = acc[c];
  }
}

// BLOCKED organisation, per node in the blocked numbering: block-local sum,
// minus the spilled fluxes of incoming block-crossing edges, plus the
// node's boundary subface fluxes (face order), times 1/ctrlVol; written to
// R in the caller's numbering through n2o.  Partial sums, spills and
// subface fluxes are read in node order (coalesced); the caller-order
// variant that gathers them through o2n measured slower.  FACES: the
// subface fluxes are evaluated here from the node's own state (the
// operations of k_face_flux: normal n_f / 3, face_flux), instead of being
// read from fbuf.
template <bool FACES>
__global__ void k_fv_nodes_b(int N, Gas g, const int* __restrict__ n2o, const double* __restrict__ part,
                             const int* __restrict__ xin_ptr, const double* __restrict__ spill,
                             const int* __restrict__ bnf_ptr, const int* __restrict__ bnf_ent,
                             const double* __restrict__ fbuf, int F, const double* __restrict__ Ub0,
                             const int* __restrict__ fcode, const double* __restrict__ fn,
                             const double* __restrict__ P2, const double* __restrict__ vol2, double* __restrict__ R,
                             const int* __restrict__ blist, int nlist, int NB) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (blist) {
    // the nodes of blocks blist[0, nlist)
    const int i = n / NB;
    if (i >= nlist) return;
    n = blist[i] * NB + n % NB;
  }
  if (n >= N) return;
  double acc[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] = part[5 * (size_t)n + c];
  for (int k = xin_ptr[n]; k < xin_ptr[n + 1]; ++k) {
    const double* sp = spill + 5 * (size_t)k;
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] -= sp[c];
  }
  const int q0 = bnf_ptr[n], q1 = bnf_ptr[n + 1];
  if (FACES) {
    if (q0 < q1) {
      const double third = 1.0 / 3.0;
      double V[5], Ub[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) { V[k] = P2[8 * (size_t)n + k]; Ub[k] = Ub0[k]; }
      for (int q = q0; q < q1; ++q) {
        const int f = bnf_ent[q] / 3;
        double ff[5];
        face_flux(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, ff);
#pragma unroll
        for (int c = 0; c < 5; ++c) acc[c] += ff[c];
      }
    }
  } else {
    for (int q = q0; q < q1; ++q) {
      const double* ff = fbuf + 5 * (size_t)bnf_ent[q];
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[c] += ff[c];
    }
  }
  const double invcv = 1.0 / vol2[n];
  const size_t o = (size_t)n2o[n];
#pragma unroll
  for (int c = 0; c < 5; ++c) R[5 * o + c] = acc[c] * invcv;
}

// U[N][5] (caller numbering) -> blocked node records P2[n].V
__global__ void k_prim_blocked(int N, Gas g, const int* __restrict__ n2o, const double* __restrict__ U,
                               double* __restrict__ P2) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int o = n2o[n];
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)o + k];
  cons2prim(g, u, v);
#pragma unroll
  for (int k = 0; k < 5; ++k) P2[8 * (size_t)n + k] = v[k];
}

// k_prim_blocked for the blocked nodes nlist[0, count) only.
__global__ void k_prim_nodes(const int* __restrict__ nlist, int count, Gas g, const int* __restrict__ n2o,
                             const double* __restrict__ U, double* __restrict__ P2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  const int n = nlist[t];
  const int o = n2o[n];
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)o + k];
  cons2prim(g, u, v);
#pragma unroll
  for (int k = 0; k < 5; ++k) P2[8 * (size_t)n + k] = v[k];
}

// The gradients of k_grad_pipe<L> for the blocked nodes nlist[0, count)
// only, from the records in global memory: the same L lanes per node with
// the same neighbour partition (r, r + L, ... of the ascending list) and
// the same xor tree, so the same sums bit for bit.
template <int L>
__global__ void __launch_bounds__(256) k_grad_nodes(const int* __restrict__ nlist, int count, int N,
                                                    const double* __restrict__ P2, const double* __restrict__ W2,
                                                    const int* __restrict__ nb2_ptr,
                                                    const int* __restrict__ nb2_node, double* __restrict__ G2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / L, r = t % L;
  const bool act = i < count;
  const int n = act ? nlist[i] : 0;
  double gs[15];
#pragma unroll
  for (int q = 0; q < 15; ++q) gs[q] = 0.0;
  if (act) {
    double w[6], pi[8];
#pragma unroll
    for (int a = 0; a < 6; ++a) w[a] = W2[(size_t)a * N + n];
    load_rec(P2, n, pi);
#pragma unroll 1
    for (int p = nb2_ptr[n] + r; p < nb2_ptr[n + 1]; p += L) {
      double pj[8];
      load_rec(P2, nb2_node[p], pj);
      grad_acc(w, pi, pi + 5, pj, gs, gs + 5, gs + 10);
    }
  }
#pragma unroll
  for (int q = 0; q < 15; ++q) {
    if (L > 1) gs[q] += __shfl_xor_sync(0xffffffffu, gs[q], 1);
    if (L > 2) gs[q] += __shfl_xor_sync(0xffffffffu, gs[q], 2);
  }
  if (!act) return;
  constexpr int SL = 16 / L;
  double o[SL];
#pragma unroll
  for (int q = 0; q < SL; ++q) {
    double v = 0.0;
#pragma unroll
    for (int rr = 0; rr < L; ++rr)
      if (SL * rr + q < 15 && r == rr) v = gs[SL * rr + q < 15 ? SL * rr + q : 0];
    o[q] = v;
  }
  double2* gi = reinterpret_cast<double2*>(G2 + 16 * (size_t)n + SL * r);
#pragma unroll
  for (int q = 0; q < SL / 2; ++q) gi[q] = make_double2(o[2 * q], o[2 * q + 1]);
}

// R rows rows[0, count) (caller numbering) copied into Rh, the device
// address of a page-locked host array of the same layout
__global__ void k_put_rows(const int* __restrict__ rows, int count, const double* __restrict__ R,
                           double* __restrict__ Rh) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 5 * count) return;
  const size_t q = 5 * (size_t)rows[t / 5] + t % 5;
  Rh[q] = R[q];
}

// Boundary fluxes, one thread per face, the three subface fluxes with
// normal n_f/3 (FaceTriaCore.C:288-308) into fbuf[3F][5].
__global__ void k_face_flux(int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ faces,
                            const int* __restrict__ fcode, const double* __restrict__ fn,
                            const double* __restrict__ P, const int* __restrict__ o2n, double* __restrict__ fbuf) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const double third = 1.0 / 3.0;
  double Ub[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) Ub[k] = Ub0[k];
  const double nx = third * fn[f], ny = third * fn[(size_t)F + f], nz = third * fn[2 * (size_t)F + f];
  const int code = fcode[f];
  for (int l = 0; l < 3; ++l) {
    const int nd0 = faces[3 * (size_t)f + l];
    const int nd = o2n ? o2n[nd0] : nd0;
    double V[5], ff[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) V[k] = P[8 * (size_t)nd + k];
    face_flux(g, code, nx, ny, nz, V, Ub, ff);
#pragma unroll
    for (int k = 0; k < 5; ++k) fbuf[5 * (3 * (size_t)f + l) + k] = ff[k];
  }
}

// Per-node assembly: edges in ascending-neighbour order (+flux when the node
// is the edge's first endpoint, -flux otherwise), then boundary faces in
// face order (Face.C:1185-1215), then R *= 1/ctrlVol (SpaceOperator.C:
// 614-620).  R is written in the caller's [N][5] layout.  FACEBUF: the face
// fluxes come precomputed from k_face_flux; otherwise they are evaluated
// here.
template <bool FACEBUF>
__global__ void k_node_residual_t(int N, int E, Gas g, const double* __restrict__ Ub0,
                                  const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                                  const double* __restrict__ flux, const int* __restrict__ nf_ptr,
                                  const int* __restrict__ nf_face, const int* __restrict__ fcode,
                                  const double* __restrict__ fn, int F, const int* __restrict__ faces,
                                  const double* __restrict__ fbuf, const double* __restrict__ P,
                                  const double* __restrict__ vol, double* __restrict__ R) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double acc[5] = {0, 0, 0, 0, 0};
  const int p1 = nbr_ptr[i + 1];
  for (int p = nbr_ptr[i]; p < p1; ++p) {
    const int e = nbr_edge[p];
    const size_t l = (size_t)(e & 0x7fffffff);
    const double sg = e < 0 ? -1.0 : 1.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) acc[k] += sg * flux[k * (size_t)E + l];
  }
  const int q1 = nf_ptr[i + 1];
  if (FACEBUF) {
    for (int q = nf_ptr[i]; q < q1; ++q) {
      const int f = nf_face[q];
      const int* fd = faces + 3 * (size_t)f;
      const int l = fd[0] == i ? 0 : (fd[1] == i ? 1 : 2);
      const double* ff = fbuf + 5 * (3 * (size_t)f + l);
#pragma unroll
      for (int k = 0; k < 5; ++k) acc[k] += ff[k];
    }
  } else if (nf_ptr[i] < q1) {
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
  k_grad<<<grid_for(4 * (size_t)m.N, kBlock), kBlock, 0, c->stream>>>(m.N, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
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
constexpr size_t kMaxStagedSmem = 160 * 1024;

static int grad_kernel_choice() {
  static const int v = [] {
    const char* e = std::getenv("AEROF_GRAD_KERNEL");
    const int k = e ? std::atoi(e) : 3;
    return k >= 0 && k <= 3 ? k : 3;
  }();
  return v;
}

// dynamic shared memory of k_fv_blocked: staged records of the block's
// nodes and forward halo, the fluxes of its edges, the halo node ids
static size_t fv_blocked_smem(const DeviceMesh& m) {
  return ((size_t)(kPS + kGS) * (m.NB + m.maxHf) + (size_t)5 * m.maxE) * sizeof(double) + (size_t)4 * m.maxHf;
}

static GradStage grad_stage(const DeviceMesh& m) {
  GradStage st;
  st.rec = 0;
  st.w = kPS * (m.NB + m.maxH);
  st.w += st.w & 1;
  st.ptr = st.w + 6 * m.NB;
  st.ls = st.ptr + (m.NB + 8) / 2;
  st.ls += st.ls & 1;
  st.size = st.ls + std::max(m.maxLp, 8) / 4;
  st.size += st.size & 1;
  return st;
}

// U -> the V part of the blocked records P2 (thread per blocked row,
// gathering U through n2o: measured faster than scattering the records
// through o2n)
static void prim_to_P2(const DeviceMesh& m, const Gas& g, const double* dU, cudaStream_t s) {
  k_prim_blocked<<<grid_for(m.N, kBlock), kBlock, 0, s>>>(m.N, g, m.n2o.p, dU, m.P2.p);
  AEROF_LAUNCH_CHECK();
}

// persistent pipelined gradients of the records P2src (with dU,
// k_prim_blocked writes the mesh's P2 first and P2src is that)
static void launch_grad_pipe(aerof_gpu_ctx* c, const Gas& g, const double* dU, const int* tag, double* G2,
                             cudaStream_t s, const double* P2src = nullptr) {
  const DeviceMesh& m = c->mesh;
  if (dU) {
    prim_to_P2(m, g, dU, s);
  }
  if (!P2src) P2src = m.P2.p;
  const GradStage st = grad_stage(m);
  const size_t smem = (size_t)2 * st.size * sizeof(double);
  const int L = kBlock / m.NB;
  auto go = [&](auto kern) {
    AEROF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    AEROF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem));
    int sms = 0;
    AEROF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->cfg.device));
    const int grid = std::max(1, std::min(m.nblk, std::max(per_sm, 1) * sms));
    kern<<<grid, kBlock, smem, s>>>(m.N, m.NB, m.nblk, m.maxH, m.maxLp, st, P2src, m.W2.p, m.nb2_ptr.p, m.lpad.p,
                                    m.hpad.p, tag, G2, nullptr);
    AEROF_LAUNCH_CHECK();
  };
  if (L == 4) go(k_grad_pipe<4>);
  else if (L == 2) go(k_grad_pipe<2>);
  else go(k_grad_pipe<1>);
}

// fused: prim conversion inside the gradient kernel; otherwise
// k_prim_blocked writes P2 first
static void launch_grad_staged(const DeviceMesh& m, const Gas& g, const double* dU, const int* tag, double* G2,
                               size_t smem, bool fused, cudaStream_t s) {
  const int L = kBlock / m.NB;
  if (!fused) {
    prim_to_P2(m, g, dU, s);
  }
  auto go = [&](auto kern) {
    AEROF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<m.nblk, kBlock, smem, s>>>(m.N, m.NB, g, m.n2o.p, dU, m.P2.p, m.W2.p, m.nb2_ptr.p, m.lnb.p, m.hptr.p,
                                      m.hnode.p, tag, G2);
    AEROF_LAUNCH_CHECK();
  };
  if (fused) {
    if (L == 4) go(k_grad_staged<4, true>);
    else if (L == 2) go(k_grad_staged<2, true>);
    else go(k_grad_staged<1, true>);
  } else {
    if (L == 4) go(k_grad_staged<4, false>);
    else if (L == 2) go(k_grad_staged<2, false>);
    else go(k_grad_staged<1, false>);
  }
}

// P2 = prim(U) in the blocked numbering and, unless the reconstruction is
// constant, the gradients G2 (zero at tagged nodes when tag is given).
void prim_grad_blocked_dev(aerof_gpu_ctx* c, const double* dU, const int* tag) {
  DeviceMesh& m = c->mesh;
  const Gas g = make_gas(c->cfg.gamma);
  cudaStream_t s = c->stream;
  c->s.G2.ensure(16 * (size_t)m.N);
  if (c->cfg.reconstruction == AEROF_REC_CONSTANT) {
    prim_to_P2(m, g, dU, s);
    return;
  }
  const size_t gsmem = ((size_t)8 * kPS * (m.NB + m.maxH) + (size_t)2 * m.maxL + 15) / 16 * 16;
  // gradient organisation (tuning knob AEROF_GRAD_KERNEL): 0 staged from
  // P2, 1 staged with the primitive conversion fused, 2 node-parallel,
  // 3 (default) staged, persistent and software pipelined
  const int gk = grad_kernel_choice();
  const bool staged = gsmem <= kMaxStagedSmem && gk != 2;
  const bool piped = gk == 3 && m.maxH <= 512 && 2 * grad_stage(m).size * sizeof(double) <= kMaxStagedSmem;
  if (piped) {
    launch_grad_pipe(c, g, dU, tag, c->s.G2.p, s);
  } else if (staged) {
    launch_grad_staged(m, g, dU, tag, c->s.G2.p, gsmem, gk == 1, s);
  } else {
    prim_to_P2(m, g, dU, s);
    k_grad<<<grid_for(4 * (size_t)m.N, kBlock), kBlock, 0, s>>>(m.N, m.P2.p, m.W2.p, m.nb2_ptr.p, m.nb2_node.p, tag,
                                                                c->s.G2.p);
    AEROF_LAUNCH_CHECK();
  }
}

// Least-squares gradients G2dst of the records P2src ([N][8] = (V, X),
// blocked numbering): the linear map the residual applies to V, here for
// tangent records.
void grad_records_blocked_dev(aerof_gpu_ctx* c, const double* P2src, double* G2dst) {
  const DeviceMesh& m = c->mesh;
  const Gas g = make_gas(c->cfg.gamma);
  cudaStream_t s = c->stream;
  const bool piped = grad_kernel_choice() == 3 && m.maxH <= 512 && 2 * grad_stage(m).size * sizeof(double) <= kMaxStagedSmem;
  if (piped) {
    launch_grad_pipe(c, g, nullptr, nullptr, G2dst, s, P2src);
  } else {
    k_grad<<<grid_for(4 * (size_t)m.N, kBlock), kBlock, 0, s>>>(m.N, P2src, m.W2.p, m.nb2_ptr.p, m.nb2_node.p, nullptr,
                                                                G2dst);
    AEROF_LAUNCH_CHECK();
  }
}

// BLOCKED organisation of residual_dev (see k_fv_blocked).
static int residual_blocked_dev(aerof_gpu_ctx* c, const double* dU, double* dR, bool sync) {
  DeviceMesh& m = c->mesh;
  const Gas g = make_gas(c->cfg.gamma);
  const int rec = c->cfg.reconstruction;
  cudaStream_t s = c->stream;
  int* cnt = counters(c);
  if (sync) AEROF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * 2, s));
  int* ecnt = sync ? cnt : cnt + 2;
  c->s.G2.ensure(16 * (size_t)m.N);
  c->s.part.ensure(5 * (size_t)m.N);
  c->s.spill.ensure(5 * (size_t)std::max(m.nX, 1));
  c->s.fbuf.ensure(15 * (size_t)std::max(m.F, 1));
  if (c->cfg.failsafe) {
    c->s.tag.ensure(m.N);
    c->s.tag.zero(s);
  }
  const size_t smem = fv_blocked_smem(m);
  // register budget from the CTAs per SM that shared memory allows
  // (228 KB per SM, 1 KB reserved per CTA)
  const int by_smem = (int)std::min<size_t>(4, (228 * 1024) / (smem + 1024));
  // 256 threads with the register budget of the CTAs that fit (384
  // threads at two CTAs per SM measured slower)
  // tuning knob AEROF_FV_THREADS = 512: two CTAs of 512 threads per SM at
  // 64 registers (more warps, some spilling) when shared memory allows two
  static const int fv_env = [] {
    const char* e = std::getenv("AEROF_FV_THREADS");
    return e ? std::atoi(e) : 256;
  }();
  const bool wide = fv_env == 512 && by_smem >= 2;
  const int fv_threads = wide ? 512 : 256;
  auto fvk = wide ? k_fv_blocked<512, 2>
                  : by_smem >= 4 ? k_fv_blocked<256, 4> : by_smem == 3 ? k_fv_blocked<256, 3> : k_fv_blocked<256, 2>;
  AEROF_CUDA(cudaFuncSetAttribute(fvk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  {
    TimerScope t(c, AEROF_T_NODAL_GRAD);
    prim_grad_blocked_dev(c, dU, nullptr);
  }
  auto fv = [&](int fs, int* counter) {
    fvk<<<m.nblk, fv_threads, smem, s>>>(m.N, m.E, m.NB, g, rec, c->cfg.beta, fs, m.bl.p, m.bnorm.p, m.beptr.p,
                                         m.hfptr.p, m.hfpad.p, m.maxHf, m.P2.p, c->s.G2.p, m.lptr.p, m.lidx.p,
                                         m.xslot.p, c->s.part.p, c->s.spill.p, c->s.tag.p, counter, nullptr);
    AEROF_LAUNCH_CHECK();
  };
  {
    TimerScope t(c, AEROF_T_FV_EDGES);
    fv(c->cfg.failsafe, ecnt);
  }
  int bad = 0;
  if (sync) {
    AEROF_CUDA(cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
  }
  c->s.p2g2_valid = true;
  if (bad && c->cfg.failsafe && rec != AEROF_REC_CONSTANT) {
    TimerScope t(c, AEROF_T_FV_TERM);
    prim_grad_blocked_dev(c, dU, c->s.tag.p);
    c->s.p2g2_valid = false;
    fv(0, cnt + 1);
  }
  {
    TimerScope t(c, AEROF_T_FV_TERM);
    // boundary fluxes in their own kernel (thread per face) or inside the
    // node assembly (tuning knob AEROF_FACES_IN_NODES=1)
    static const bool faces_in_nodes = [] {
      const char* e = std::getenv("AEROF_FACES_IN_NODES");
      return e && std::atoi(e) == 1;
    }();
    if (faces_in_nodes) {
      k_fv_nodes_b<true><<<grid_for(m.N, kBlock), kBlock, 0, s>>>(
          m.N, g, m.n2o.p, c->s.part.p, m.xin_ptr.p, c->s.spill.p, m.bnf_ptr.p, m.bnf_ent.p, nullptr, m.F, m.Ubd.p,
          m.fcode.p, m.fnrm.p, m.P2.p, m.vol2.p, dR, nullptr, 0, m.NB);
    } else {
      if (m.F) {
        k_face_flux<<<grid_for(m.F, kBlock), kBlock, 0, s>>>(m.F, g, m.Ubd.p, m.faces.p, m.fcode.p, m.fnrm.p,
                                                             m.P2.p, m.o2n.p, c->s.fbuf.p);
        AEROF_LAUNCH_CHECK();
      }
      k_fv_nodes_b<false><<<grid_for(m.N, kBlock), kBlock, 0, s>>>(
          m.N, g, m.n2o.p, c->s.part.p, m.xin_ptr.p, c->s.spill.p, m.bnf_ptr.p, m.bnf_ent.p, c->s.fbuf.p, m.F,
          m.Ubd.p, m.fcode.p, m.fnrm.p, m.P2.p, m.vol2.p, dR, nullptr, 0, m.NB);
    }
    AEROF_LAUNCH_CHECK();
    galerkin_add(c, dU, dR);
  }
  return bad;
}

int residual_dev(aerof_gpu_ctx* c, const double* dU, double* dR, bool sync) {
  DeviceMesh& m = c->mesh;
  c->s.p2g2_valid = false;
  if (c->cfg.residual_kernel == AEROF_KERNEL_BLOCKED && fv_blocked_smem(m) <= 200 * 1024)
    return residual_blocked_dev(c, dU, dR, sync);
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
    k_grad<<<grid_for(4 * (size_t)m.N, kBlock), kBlock, 0, c->stream>>>(m.N, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
                                                            c->s.tag.p, c->s.G.p);
    AEROF_LAUNCH_CHECK();
    k_edge_flux<<<grid_for(m.E, kBlock), kBlock, 0, c->stream>>>(
        m.E, g, rec, c->cfg.beta, 0, m.edges.p, m.en.p, m.P.p, c->s.G.p, c->s.flux.p, c->s.tag.p, cnt + 1);
    AEROF_LAUNCH_CHECK();
  }
  {
    TimerScope t(c, AEROF_T_FV_TERM);
    c->s.fbuf.ensure(15 * (size_t)std::max(m.F, 1));
    if (m.F) {
      k_face_flux<<<grid_for(m.F, kBlock), kBlock, 0, c->stream>>>(m.F, g, m.Ubd.p, m.faces.p, m.fcode.p, m.fnrm.p,
                                                                   m.P.p, nullptr, c->s.fbuf.p);
      AEROF_LAUNCH_CHECK();
    }
    k_node_residual_t<true><<<grid_for(m.N, kBlock), kBlock, 0, c->stream>>>(
        m.N, m.E, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_edge.p, c->s.flux.p, m.nf_ptr.p, m.nf_face.p, m.fcode.p, m.fnrm.p,
        m.F, m.faces.p, c->s.fbuf.p, m.P.p, m.vol.p, dR);
    AEROF_LAUNCH_CHECK();
    galerkin_add(c, dU, dR);
  }
  return bad;
}

// ------------------------------------------------------------------
// Residual of HOST arrays with the copies overlapped with the computation.
// U arrives in K chunks of caller rows on a copy stream.  For every chunk s
// that has arrived, the compute stream runs the work whose inputs are then
// complete (DeviceMesh::h_st_*): the primitive conversion of the nodes of
// chunk s, the gradients of the nodes whose neighbourhoods are complete
// (whole blocks by the persistent block kernel, the rest by a node
// kernel), the edge fluxes of the blocks whose nodes and forward halo have
// gradients, the node assembly with the boundary fluxes of the blocks
// whose own and incoming fluxes are done.
// A second copy stream (the copy engines run both directions at once)
// takes chunk c of R out after stage c + 1; its rows whose assembly runs in
// a later stage (their block depends on rows further on) are written again
// after the last stage, once that chunk's copy has landed, by a kernel
// storing into R through its device address.  The conversion runs per
// node (k_prim_nodes), the gradients per block (k_grad_pipe) or per node
// (k_grad_nodes, with the block kernel's lanes and order), the fluxes and
// assembly per block (k_fv_blocked, k_fv_nodes_b with the boundary fluxes
// of k_face_flux inside): the same arithmetic as residual_blocked_dev, so
// the same residual bit for bit.  Each stage's kernels are replayed as one
// CUDA graph.  Used for page-locked host U and R with the blocked kernel,
// failsafe off, no viscous term and timers off, on meshes of at least
// kPipeMinNodes nodes; otherwise aerof_gpu_residual stages the arrays
// around one residual_dev.
constexpr int kPipeMinNodes = 1 << 17;

// page-locked host memory (with its device address when dev is given)
static bool pinned_host(const void* p, void** dev = nullptr) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type != cudaMemoryTypeHost) return false;
  if (dev) {
    *dev = a.devicePointer;
    if (!*dev) return false;
  }
  return true;
}


// the edge-flux kernel of residual_blocked_dev for this mesh
static decltype(&k_fv_blocked<256, 2>) pipe_fv_kernel(const DeviceMesh& m) {
  const int by_smem = (int)std::min<size_t>(4, (228 * 1024) / (fv_blocked_smem(m) + 1024));
  return by_smem >= 4 ? k_fv_blocked<256, 4> : by_smem == 3 ? k_fv_blocked<256, 3> : k_fv_blocked<256, 2>;
}

static ResidualPipe& pipe_for(aerof_gpu_ctx* c) {
  if (c->pipe) return *c->pipe;
  const DeviceMesh& m = c->mesh;
  auto p = std::make_unique<ResidualPipe>();
  const int K = m.pipeK;
  p->K = K;
  {
    AEROF_CUDA(cudaFuncSetAttribute(pipe_fv_kernel(m), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)fv_blocked_smem(m)));
    const int L = kBlock / m.NB;
    auto gp = L == 4 ? k_grad_pipe<4> : L == 2 ? k_grad_pipe<2> : k_grad_pipe<1>;
    const size_t gsmem = (size_t)2 * grad_stage(m).size * sizeof(double);
    AEROF_CUDA(cudaFuncSetAttribute(gp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gsmem));
    int per_sm = 0, sms = 0;
    AEROF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gp, kBlock, gsmem));
    AEROF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->cfg.device));
    p->ggrid = std::max(per_sm, 1) * sms;
  }
  AEROF_CUDA(cudaStreamCreateWithFlags(&p->sin, cudaStreamNonBlocking));
  AEROF_CUDA(cudaStreamCreateWithFlags(&p->sout, cudaStreamNonBlocking));
  p->ev_in.assign(K, nullptr);
  p->ev_stage.assign(K, nullptr);
  for (auto& e : p->ev_in) AEROF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (auto& e : p->ev_stage) AEROF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  AEROF_CUDA(cudaEventCreateWithFlags(&p->ev_go, cudaEventDisableTiming));
  AEROF_CUDA(cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming));
  // kinds, by stage: 0 nodes converted; 1 blocks whose nodes all get their
  // gradients in the stage (the persistent block kernel); 2 blocks' edge
  // fluxes; 3 blocks' assembly (with their boundary fluxes); 4 the other
  // nodes getting their gradients (node kernel)
  const int NB = m.NB;
  std::vector<unsigned char> gmin(m.nblk, 255), gmax(m.nblk, 0);
  for (int n = 0; n < m.N; ++n) {
    gmin[n / NB] = std::min(gmin[n / NB], m.h_st_grad[n]);
    gmax[n / NB] = std::max(gmax[n / NB], m.h_st_grad[n]);
  }
  std::vector<int> lists;
  p->off.assign(5 * (K + 1), 0);
  for (int kind = 0; kind < 5; ++kind) {
    for (int s = 0; s < K; ++s) {
      p->off[kind * (K + 1) + s] = (int)lists.size();
      if (kind == 0) {
        for (int n = 0; n < m.N; ++n)
          if (m.h_st_prim[n] == s) lists.push_back(n);
      } else if (kind == 1) {
        for (int b = 0; b < m.nblk; ++b)
          if (gmin[b] == gmax[b] && gmax[b] == s) lists.push_back(b);
      } else if (kind == 2 || kind == 3) {
        const std::vector<unsigned char>& v = kind == 2 ? m.h_st_flux : m.h_st_node;
        for (int b = 0; b < m.nblk; ++b)
          if (v[b] == s) lists.push_back(b);
      } else {
        for (int n = 0; n < m.N; ++n)
          if (gmin[n / NB] != gmax[n / NB] && m.h_st_grad[n] == s) lists.push_back(n);
      }
    }
    p->off[kind * (K + 1) + K] = (int)lists.size();
  }
  if (lists.empty()) lists.push_back(0);
  // chunk c of R goes out after stage c + lag (lag 1; tuning knob
  // AEROF_PIPE_OUT_LAG, 0-2); its rows assembled later are the late rows
  int lag = 1;
  if (const char* env = std::getenv("AEROF_PIPE_OUT_LAG")) lag = std::min(std::max(std::atoi(env), 0), 2);
  p->out_stage.assign(K, 0);
  for (int k = 0; k < K; ++k) p->out_stage[k] = std::min(k + lag, K - 1);
  for (int k = 0; k < K; ++k) {
    const size_t r0 = m.pipe_rows[k], r1 = m.pipe_rows[k + 1];
    for (size_t o = r0; o < r1; ++o)
      if (m.h_st_node[m.h_o2n[o] / m.NB] > p->out_stage[k]) p->h_late.push_back((int)o);
  }
  p->lists.upload(lists.data(), lists.size(), c->stream);
  AEROF_CUDA(cudaHostAlloc((void**)&p->h_bad, sizeof(int), cudaHostAllocDefault));
  AEROF_CUDA(cudaEventCreateWithFlags(&p->ev_pre, cudaEventDisableTiming));
  if (!p->h_late.empty()) p->late.upload(p->h_late.data(), p->h_late.size(), c->stream);
  AEROF_CUDA(cudaStreamSynchronize(c->stream));
  c->pipe = std::move(p);
  return *c->pipe;
}

// The kernels of stage st of the overlapped residual, on stream s: the
// nodes converted in the stage, their gradients (per block where a whole
// block's gradients fall in the stage, else per node), the edge fluxes and
// the assembly (boundary fluxes inside) of the blocks the stage completes.
static void stage_kernels(aerof_gpu_ctx* c, ResidualPipe& p, int st, cudaStream_t s) {
  DeviceMesh& m = c->mesh;
  const int rec = c->cfg.reconstruction;
  const bool grad = rec != AEROF_REC_CONSTANT;
  const int K = p.K;
  const Gas g = make_gas(c->cfg.gamma);
  int* cnt = counters(c);
  double* dU = c->s.Ustage.p;
  double* dR = c->s.Rstage.p;
  // the kernels and launch shapes of residual_blocked_dev (attributes set
  // by pipe_for, outside any capture)
  const size_t fsmem = fv_blocked_smem(m);
  auto fvk = pipe_fv_kernel(m);
  const int L = kBlock / m.NB;
  auto gk = L == 4 ? k_grad_nodes<4> : L == 2 ? k_grad_nodes<2> : k_grad_nodes<1>;
  auto gp = L == 4 ? k_grad_pipe<4> : L == 2 ? k_grad_pipe<2> : k_grad_pipe<1>;
  const GradStage gst = grad_stage(m);
  const size_t gsmem = (size_t)2 * gst.size * sizeof(double);
  const int* lists = p.lists.p;
  auto seg = [&](int kind, int& count) {
    const int a = p.off[kind * (K + 1) + st];
    count = p.off[kind * (K + 1) + st + 1] - a;
    return lists + a;
  };
  int nl = 0;
  const int* lp = seg(0, nl);
  if (nl) {
    k_prim_nodes<<<grid_for(nl, kBlock), kBlock, 0, s>>>(lp, nl, g, m.n2o.p, dU, m.P2.p);
    AEROF_LAUNCH_CHECK();
  }
  lp = seg(1, nl);
  if (nl && grad) {
    gp<<<std::min(nl, p.ggrid), kBlock, gsmem, s>>>(m.N, m.NB, nl, m.maxH, m.maxLp, gst, m.P2.p, m.W2.p,
                                                    m.nb2_ptr.p, m.lpad.p, m.hpad.p, nullptr, c->s.G2.p, lp);
    AEROF_LAUNCH_CHECK();
  }
  lp = seg(4, nl);
  if (nl && grad) {
    gk<<<grid_for((size_t)nl * L, kBlock), kBlock, 0, s>>>(lp, nl, m.N, m.P2.p, m.W2.p, m.nb2_ptr.p, m.nb2_node.p,
                                                            c->s.G2.p);
    AEROF_LAUNCH_CHECK();
  }
  lp = seg(2, nl);
  if (nl) {
    fvk<<<nl, 256, fsmem, s>>>(m.N, m.E, m.NB, g, rec, c->cfg.beta, 0, m.bl.p, m.bnorm.p, m.beptr.p, m.hfptr.p,
                               m.hfpad.p, m.maxHf, m.P2.p, c->s.G2.p, m.lptr.p, m.lidx.p, m.xslot.p, c->s.part.p,
                               c->s.spill.p, c->s.tag.p, cnt, lp);
    AEROF_LAUNCH_CHECK();
  }
  lp = seg(3, nl);
  if (nl) {
    // the boundary fluxes inside the assembly (one launch instead of a
    // small face kernel per stage)
    k_fv_nodes_b<true><<<grid_for((size_t)nl * m.NB, kBlock), kBlock, 0, s>>>(
        m.N, g, m.n2o.p, c->s.part.p, m.xin_ptr.p, c->s.spill.p, m.bnf_ptr.p, m.bnf_ent.p, nullptr, m.F, m.Ubd.p,
        m.fcode.p, m.fnrm.p, m.P2.p, m.vol2.p, dR, lp, nl, m.NB);
    AEROF_LAUNCH_CHECK();
  }
}

// The stages' kernels captured once as graphs (they touch device buffers
// only, so one capture serves every U and R).  False when s cannot be
// captured (the legacy default stream, or a capture already running).
static bool pipe_graphs(aerof_gpu_ctx* c, ResidualPipe& p, cudaStream_t s) {
  // the device buffers the recorded kernels name: a buffer reallocated
  // since the capture invalidates the graphs
  const std::vector<const void*> key = {c->s.Ustage.p, c->s.Rstage.p, c->s.G2.p,  c->s.part.p,
                                        c->s.spill.p,  c->s.tag.p,    c->s.counters.p, c->mesh.P2.p};
  if (!p.stage_exec.empty() && key == p.graph_key) return true;
  for (auto e : p.stage_exec) cudaGraphExecDestroy(e);
  p.stage_exec.clear();
  p.stage_launches.clear();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  AEROF_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone || s == cudaStreamLegacy || s == nullptr) return false;
  std::vector<cudaGraphExec_t> ex(p.K, nullptr);
  std::vector<long long> nk(p.K, 0);
  auto drop = [&]() {
    for (auto e : ex)
      if (e) cudaGraphExecDestroy(e);
  };
  for (int st = 0; st < p.K; ++st) {
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      drop();
      return false;
    }
    cudaGraph_t gph = nullptr;
    const long long l0 = g_launch_count.load();
    try {
      stage_kernels(c, p, st, s);
    } catch (...) {
      cudaStreamEndCapture(s, &gph);
      if (gph) cudaGraphDestroy(gph);
      cudaGetLastError();
      drop();
      throw;
    }
    // launches are counted when the graph runs
    nk[st] = g_launch_count.load() - l0;
    g_launch_count.fetch_sub(nk[st]);
    const bool ok = cudaStreamEndCapture(s, &gph) == cudaSuccess && gph &&
                    cudaGraphInstantiate(&ex[st], gph, 0) == cudaSuccess;
    if (gph) cudaGraphDestroy(gph);
    if (!ok) {
      cudaGetLastError();
      drop();
      return false;
    }
  }
  p.stage_exec = ex;
  p.stage_launches = nk;
  p.graph_key = key;
  return true;
}

// The overlapped residual of U into R, queued on c->stream and the pipe's
// copy streams (joined back into c->stream at the end): the copies of U's
// chunks back to back on one stream, each stage's kernels (one graph, or
// launch by launch) on c->stream once its chunk has landed, the copies of
// R's chunks on the other stream as their stages complete, then the late
// rows.  Rdev is R's device address (for the late rows); the unphysical
// count goes to p.h_bad.
static void pipelined_enqueue(aerof_gpu_ctx* c, ResidualPipe& p, const double* U, double* R, double* Rdev,
                              bool graphs) {
  DeviceMesh& m = c->mesh;
  const int K = p.K;
  cudaStream_t s = c->stream;
  int* cnt = counters(c);
  double* dU = c->s.Ustage.p;
  double* dR = c->s.Rstage.p;
  AEROF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * 2, s));
  // the copy streams start after the work already queued on s (which may
  // still read Ustage or write Rstage)
  AEROF_CUDA(cudaEventRecord(p.ev_go, s));
  AEROF_CUDA(cudaStreamWaitEvent(p.sin, p.ev_go, 0));
  AEROF_CUDA(cudaStreamWaitEvent(p.sout, p.ev_go, 0));
  for (int k = 0; k < K; ++k) {
    const size_t r0 = m.pipe_rows[k], r1 = m.pipe_rows[k + 1];
    if (r1 > r0)
      AEROF_CUDA(cudaMemcpyAsync(dU + 5 * r0, U + 5 * r0, 5 * (r1 - r0) * sizeof(double), cudaMemcpyHostToDevice,
                                 p.sin));
    AEROF_CUDA(cudaEventRecord(p.ev_in[k], p.sin));
  }
  for (int st = 0; st < K; ++st) {
    AEROF_CUDA(cudaStreamWaitEvent(s, p.ev_in[st], 0));
    if (graphs) {
      AEROF_CUDA(cudaGraphLaunch(p.stage_exec[st], s));
      g_launch_count.fetch_add(p.stage_launches[st]);
    } else {
      stage_kernels(c, p, st, s);
    }
    AEROF_CUDA(cudaEventRecord(p.ev_stage[st], s));
  }
  // the copies of R's chunks as their stages complete
  for (int st = 0; st < K; ++st) {
    // every copy queued so far (the chunks that can hold late rows)
    if (st == K - 1) AEROF_CUDA(cudaEventRecord(p.ev_pre, p.sout));
    for (int k = 0; k < K; ++k) {
      if (p.out_stage[k] != st) continue;
      const size_t r0 = m.pipe_rows[k], r1 = m.pipe_rows[k + 1];
      AEROF_CUDA(cudaStreamWaitEvent(p.sout, p.ev_stage[st], 0));
      if (r1 > r0)
        AEROF_CUDA(cudaMemcpyAsync(R + 5 * r0, dR + 5 * r0, 5 * (r1 - r0) * sizeof(double), cudaMemcpyDeviceToHost,
                                   p.sout));
    }
  }
  const int nlate = (int)p.h_late.size();
  if (nlate) {
    // the late rows, final now, over their chunks' earlier copies (which
    // must have landed first)
    AEROF_CUDA(cudaStreamWaitEvent(s, p.ev_pre, 0));
    k_put_rows<<<grid_for(5 * (size_t)nlate, kBlock), kBlock, 0, s>>>(p.late.p, nlate, dR, Rdev);
    AEROF_LAUNCH_CHECK();
  }
  AEROF_CUDA(cudaMemcpyAsync(p.h_bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
  AEROF_CUDA(cudaEventRecord(p.ev_out, p.sout));
  AEROF_CUDA(cudaStreamWaitEvent(s, p.ev_out, 0));
}

// false: not applicable (the caller takes the staged path)
static bool residual_host_pipelined(aerof_gpu_ctx* c, const double* U, double* R, int& bad) {
  DeviceMesh& m = c->mesh;
  const int rec = c->cfg.reconstruction;
  const bool grad = rec != AEROF_REC_CONSTANT;
  if (m.N < kPipeMinNodes || c->cfg.failsafe || c->visc.model != 0 || c->timers.on) return false;
  if (c->cfg.residual_kernel != AEROF_KERNEL_BLOCKED || fv_blocked_smem(m) > 200 * 1024) return false;
  if (grad && grad_kernel_choice() != 3) return false;
  if (grad && !(m.maxH <= 512 && 2 * grad_stage(m).size * sizeof(double) <= kMaxStagedSmem)) return false;
  void* Rdev = nullptr;
  if (!pinned_host(U) || !pinned_host(R, &Rdev)) return false;
  ResidualPipe& p = pipe_for(c);
  cudaStream_t s = c->stream;
  const size_t n5 = 5 * (size_t)m.N;
  c->s.Ustage.ensure(n5);
  c->s.Rstage.ensure(n5);
  c->s.G2.ensure(16 * (size_t)m.N);
  c->s.part.ensure(5 * (size_t)m.N);
  c->s.spill.ensure(5 * (size_t)std::max(m.nX, 1));
  counters(c);
  // Each stage's ~5 kernels are one graph: launched one by one while the
  // copies saturate the host link, dependent kernels wait 5-9 us for their
  // launch commands.  The copies stay outside the graphs, in their own
  // streams, so that nothing holds them back.
  const bool graphs = pipe_graphs(c, p, s);
  pipelined_enqueue(c, p, U, R, static_cast<double*>(Rdev), graphs);
  AEROF_CUDA(cudaStreamSynchronize(s));
  bad = *p.h_bad;
  c->s.p2g2_valid = true;
  return true;
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
    int bad = 0;
    if (residual_host_pipelined(c, U, R, bad)) return bad;
    const double* dU = in_dev(c, U, n5, c->s.Ustage);
    double* dR = out_dev(c, R, n5, c->s.Rstage);
    bad = residual_dev(c, dU, dR);
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

// ====================================================================
// Residual without any allocation.
//
// Who needs it: callers that may not allocate device memory once they are
// running -- an application that has reserved all of the GPU's memory for
// its own pool before it calls us, or a host thread that must not take the
// device allocator's locks.  aerof_gpu_residual grows its scratch buffers
// (per-edge fluxes, gradients, counters) on first use; this variant keeps
// that scratch in one fixed array of device memory that is part of the
// library image instead, so the call itself allocates nothing.  The first
// call on a device looks up the array's device address (once per device,
// with that device current); make that first call before any stream
// capture.  All calls share the one array: two calls that overlap on the
// GPU (other streams, other contexts on the same device) race on it.
//
// Limit: the scratch holds the per-edge fluxes (5E doubles), the gradients
// (16N doubles, 16-byte vector stores) and 8 counters plus N failsafe tags
// (ints), each part starting on a 256-byte boundary:
//   noalloc_need(N, E) = a(a(5E) + 16N) + ceil((N + 8)/2) doubles, a(x) = x
//   rounded up to a multiple of 32,
// at most kNoAllocScratchDoubles = 2,097,152 doubles (16 MiB), i.e. meshes
// up to roughly 40,000 nodes (a 34^3 lattice).
//
// Residency: with lazy module loading (the CUDA 12 default) the array would
// only be reserved when this file's module first loads, which for a caller
// that hands the rest of the device to its own pool could be too late.  So
// aerof_gpu_create looks up its device address (noalloc_attach, with the
// context's device current), which loads the module and reserves the 16 MiB
// at context creation; the address is kept in the context, so a context
// created after a device reset looks it up afresh.  Every GPU on which a
// context is created holds these 16 MiB until the process exits.
namespace aerof {

constexpr size_t kNoAllocScratchDoubles = 2u * 1024u * 1024u;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

static size_t align32(size_t n) { return (n + 31) / 32 * 32; }

struct NoAllocLayout {
  size_t G, cnt, need;  // offsets of the gradients and the counters, total doubles
};
static NoAllocLayout noalloc_layout(size_t N, size_t E) {
  NoAllocLayout l;
  l.G = align32(5 * E);
  l.cnt = align32(l.G + 16 * N);
  l.need = l.cnt + (N + 8 + 1) / 2;
  return l;
}

// Called by aerof_gpu_create with the context's device current: host code
// cannot hand g_noalloc_scratch itself to a kernel (in host code the name is
// a host-side stand-in), so the device address is looked up here.
void noalloc_attach(aerof_gpu_ctx* c) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    c->noalloc_scratch = nullptr;
    c->noalloc_error = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
    return;
  }
  // with lazy loading a kernel's code is also placed in device memory on its
  // first launch; the kernels of the allocation-free path are loaded here
  const void* kernels[] = {(const void*)k_prim, (const void*)k_grad, (const void*)k_edge_flux,
                           (const void*)k_node_residual_t<false>};
  for (const void* k : kernels) {
    cudaFuncAttributes a;
    e = cudaFuncGetAttributes(&a, k);
    if (e != cudaSuccess) {
      cudaGetLastError();
      c->noalloc_scratch = nullptr;
      c->noalloc_error = std::string("cudaFuncGetAttributes: ") + cudaGetErrorString(e);
      return;
    }
  }
  c->noalloc_scratch = static_cast<double*>(p);
}

}  // namespace aerof

extern "C" int aerof_gpu_residual_noalloc(aerof_gpu_ctx* c, const double* U, double* R) {
  return guard(c, [&]() -> int {
    if (int e = need_mesh(c)) return e;
    if (!U || !R) return AEROF_EINVAL;
    if (!is_device_ptr(U) || !is_device_ptr(R)) {
      c->last_error = "aerof_gpu_residual_noalloc needs device pointers for U and R";
      return AEROF_EINVAL;
    }
    DeviceMesh& m = c->mesh;
    const NoAllocLayout lay = noalloc_layout(m.N, m.E);
    if (lay.need > kNoAllocScratchDoubles) {
      c->last_error = "mesh too large for aerof_gpu_residual_noalloc: needs " + std::to_string(lay.need) +
                      " doubles of scratch (5E + 16N + (N + 8)/2, parts on 256-byte boundaries), the fixed "
                      "array holds " + std::to_string(kNoAllocScratchDoubles);
      return AEROF_EINVAL;
    }
    double* base = c->noalloc_scratch;
    if (!base) {
      c->last_error = "allocation-free scratch unavailable on this device: " + c->noalloc_error;
      return AEROF_ECUDA;
    }
    double* flux = base;
    double* G = base + lay.G;
    int* cnt = reinterpret_cast<int*>(base + lay.cnt);
    int* tag = cnt + 8;
    // every part must start on a 256-byte boundary (G takes 16-byte vector
    // stores); a wrong offset fails here, never on the GPU
    if (reinterpret_cast<uintptr_t>(base) % 256 || reinterpret_cast<uintptr_t>(G) % 256 ||
        reinterpret_cast<uintptr_t>(cnt) % 256) {
      c->last_error = "allocation-free scratch misaligned";
      return AEROF_EINVAL;
    }
    cudaStream_t s = c->stream;
    const Gas g = make_gas(c->cfg.gamma);
    const int rec = c->cfg.reconstruction;
    // the array keeps the previous call's contents: clear the counters and tags
    AEROF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (8 + (size_t)m.N), s));
    k_prim<<<grid_for(m.N, kBlock), kBlock, 0, s>>>(m.N, g, U, m.P.p);
    AEROF_LAUNCH_CHECK();
    if (rec != AEROF_REC_CONSTANT) {
      k_grad<<<grid_for(4 * (size_t)m.N, kBlock), kBlock, 0, s>>>(m.N, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
                                                                  nullptr, G);
      AEROF_LAUNCH_CHECK();
    }
    k_edge_flux<<<grid_for(m.E, kBlock), kBlock, 0, s>>>(m.E, g, rec, c->cfg.beta, c->cfg.failsafe, m.edges.p,
                                                         m.en.p, m.P.p, G, flux, tag, cnt);
    AEROF_LAUNCH_CHECK();
    int bad = 0;
    AEROF_CUDA(cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
    if (bad && c->cfg.failsafe && rec != AEROF_REC_CONSTANT) {
      k_grad<<<grid_for(4 * (size_t)m.N, kBlock), kBlock, 0, s>>>(m.N, m.P.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
                                                                  tag, G);
      AEROF_LAUNCH_CHECK();
      k_edge_flux<<<grid_for(m.E, kBlock), kBlock, 0, s>>>(m.E, g, rec, c->cfg.beta, 0, m.edges.p, m.en.p, m.P.p, G,
                                                           flux, tag, cnt + 1);
      AEROF_LAUNCH_CHECK();
    }
    k_node_residual_t<false><<<grid_for(m.N, kBlock), kBlock, 0, s>>>(
        m.N, m.E, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_edge.p, flux, m.nf_ptr.p, m.nf_face.p, m.fcode.p, m.fnrm.p, m.F,
        m.faces.p, nullptr, m.P.p, m.vol.p, R);
    AEROF_LAUNCH_CHECK();
    galerkin_add(c, U, R);
    AEROF_CUDA(cudaStreamSynchronize(s));
    return bad;
  });
}
