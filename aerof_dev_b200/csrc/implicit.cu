// implicit.cu -- the Newton-Krylov inner loop on the GPU: first-order H1
// Jacobian assembly (FP32 or FP64 block storage), BSR matrix-vector product
// and its transpose, block-Jacobi preconditioner, right-preconditioned
// GMRES with FP64 modified Gram-Schmidt, and the pseudo-transient Newton
// driver.
//
// Storage: the H1 operator (MvpMat, MvpMatrix.h:10-80, keeps a[N + 2E][25]
// indexed by node and by edge) is held by rows instead: diag[N][25] and the
// off-diagonal blocks of row i at the positions of its neighbour list
// (ascending neighbour, the CSR used by the residual), so a row's blocks
// are contiguous and every product is a deterministic per-row gather in the
// reference's accumulation order (SubDomain.C:3916-3995).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "physics.cuh"

namespace aerof {

constexpr int kIB = 256;
constexpr int kGB = 1184;  // reduction grid: 8 x 148 SMs

// Sliced block layout (SELL-32): rows in slices of 32 (row r = 32 s + l);
// block k of the rows of slice s occupies 800 consecutive elements at
// (sptr[s] + k) * 800 (the diagonal blocks and their inverses at s * 800).
// Inside, elements 0..23 of lane l are stored as W-wide vectors (W = 4 for
// FP32, 2 for FP64: 16 bytes) at ((e / W) * 32 + l) * W + e % W and element
// 24 at 768 + l, so a warp reads a block as 16-byte loads of consecutive
// lanes, one coalesced 512-byte line per vector, with no padding.
template <class S> struct SlW { static constexpr int W = 16 / (int)sizeof(S); };
template <class S>
__host__ __device__ __forceinline__ size_t sl_el(int e, int l) {
  constexpr int W = SlW<S>::W;
  return e < 24 ? ((size_t)(e / W) * 32 + l) * W + e % W : (size_t)768 + l;
}
__device__ __forceinline__ size_t sl_blk(const int* __restrict__ sptr, int r, int k) {
  return ((size_t)sptr[r >> 5] + k) * 800;
}
__device__ __forceinline__ size_t sl_dblk(int r) { return (size_t)(r >> 5) * 800; }

// the 25 elements of lane l's block at base b, as doubles
template <class S>
__device__ __forceinline__ void load_block(const S* __restrict__ a, size_t b, int l, double* v);
template <>
__device__ __forceinline__ void load_block<float>(const float* __restrict__ a, size_t b, int l, double* v) {
  const float4* q = reinterpret_cast<const float4*>(a + b) + l;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const float4 t = q[32 * i];
    v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
  }
  v[24] = a[b + 768 + l];
}
template <>
__device__ __forceinline__ void load_block<double>(const double* __restrict__ a, size_t b, int l, double* v) {
  const double2* q = reinterpret_cast<const double2*>(a + b) + l;
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    const double2 t = q[32 * i];
    v[2 * i] = t.x; v[2 * i + 1] = t.y;
  }
  v[24] = a[b + 768 + l];
}

// the 25 values of lane l's block at base b written as 16-byte vectors
// (elements 0..23) and one scalar (element 24): one coalesced line per
// vector for the 32 rows of a warp
template <class S>
__device__ __forceinline__ void store_block_vec(S* __restrict__ a, size_t b, int l, const S* v);
template <>
__device__ __forceinline__ void store_block_vec<float>(float* __restrict__ a, size_t b, int l, const float* v) {
  float4* q = reinterpret_cast<float4*>(a + b) + l;
#pragma unroll
  for (int i = 0; i < 6; ++i) q[32 * i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  a[b + 768 + l] = v[24];
}
template <>
__device__ __forceinline__ void store_block_vec<double>(double* __restrict__ a, size_t b, int l, const double* v) {
  double2* q = reinterpret_cast<double2*>(a + b) + l;
#pragma unroll
  for (int i = 0; i < 12; ++i) q[32 * i] = make_double2(v[2 * i], v[2 * i + 1]);
  a[b + 768 + l] = v[24];
}

// v * scale rounded to S, written as block k of row r (TR: the transposed
// block), and the same for a diagonal block
template <class S, bool TR>
__device__ __forceinline__ void store_off(S* __restrict__ off, const int* __restrict__ sptr, int r, int k,
                                          const double* v, double scale) {
  const size_t b = sl_blk(sptr, r, k);
#pragma unroll
  for (int e = 0; e < 25; ++e) off[b + sl_el<S>(e, r & 31)] = (S)(v[TR ? 5 * (e % 5) + e / 5 : e] * scale);
}
template <class S, bool TR>
__device__ __forceinline__ void store_diag(S* __restrict__ diag, int r, const double* v) {
  S t[25];
#pragma unroll
  for (int e = 0; e < 25; ++e) t[e] = (S)v[TR ? 5 * (e % 5) + e / 5 : e];
  store_block_vec<S>(diag, sl_dblk(r), r & 31, t);
}

// One thread per row r; a warp is one slice of the sliced layout, so for
// each neighbour position k the 32 rows write every block element as one
// coalesced line.  For the edge e = (r, s) (r first endpoint, sg = +1) or
// (s, r) (r second, sg = -1) the approximate Roe Jacobians at the
// un-reconstructed states (roejacappr3Dgas, FluxFcnDescSG.C:155-262;
// roejac(n, Va, Vb, +1) = dF/dU of the first endpoint a, (.., -1) of the
// second) give the off-diagonal block A_rs = sg dF/dU_s / vol_r and the
// contribution sg dF/dU_r to the diagonal block (Edge.C:4503-4523).  Both
// Jacobians share the Roe dissipation matrix D, formed one column at a
// time with the convective parts H(V_s), H(V_r), so no 25-element block is
// held in registers besides the diagonal sum.  Then the row's boundary
// faces (Face.C:814-847), times 1/vol (SubDomain.C:1760-1765), + I/dt
// (TimeState.C:731-756).  Every edge's Jacobians are evaluated once by each
// of its two rows.  TR: the transpose H1^T is stored instead (block k of
// row r = A_sr^T with A_sr = -sg dF/dU_r / vol_s, the Jacobian formed for
// the diagonal), for products with the transpose that read coalesced.
// Boundary-face blocks of the boundary rows (Face.C:814-847: FD flux
// Jacobians for far field, the analytic wall block, in face order), summed
// per row into fsum; k_jac_rows adds them to the diagonal.  Kept apart so
// that the FD arithmetic does not set the register budget of the edge pass.
__global__ void k_jac_faces(int nbrow, int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ blist,
                            const int* __restrict__ nf_ptr, const int* __restrict__ nf_face,
                            const int* __restrict__ fcode, const double* __restrict__ fn,
                            const double* __restrict__ P, double* __restrict__ fsum) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbrow) return;
  const int r = blist[t];
  double V[5], Ub[5], a[25];
#pragma unroll
  for (int k = 0; k < 5; ++k) { V[k] = P[8 * (size_t)r + k]; Ub[k] = Ub0[k]; }
#pragma unroll
  for (int k = 0; k < 25; ++k) a[k] = 0.0;
  const double third = 1.0 / 3.0;
  for (int q = nf_ptr[r]; q < nf_ptr[r + 1]; ++q) {
    const int f = nf_face[q];
    double jac[25];
    face_jac(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, jac);
#pragma unroll
    for (int k = 0; k < 25; ++k) a[k] += jac[k];
  }
#pragma unroll
  for (int k = 0; k < 25; ++k) fsum[25 * (size_t)t + k] = a[k];
}

// block size of k_jac_rows: its shared scratch (two [25][threads] arrays)
// stays under the 48 KB static limit
// and, for FP32, the register budget of 4 CTAs per SM
template <class S> struct JacThreads {
  static constexpr int T = sizeof(S) == 4 ? 128 : 64;
  static constexpr int B = sizeof(S) == 4 ? 4 : 1;
};

template <class S, bool TR>
__global__ void __launch_bounds__(JacThreads<S>::T, JacThreads<S>::B)
    k_jac_rows(int N, int E, int F, Gas g, const double* __restrict__ Ub0,
                                                  const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_node,
                                                  const int* __restrict__ nbr_edge, const double* __restrict__ en,
                                                  const double* __restrict__ P, const double* __restrict__ vol,
                                                  const int* __restrict__ brow, const double* __restrict__ fsum,
                                                  const double* __restrict__ dt, const int* __restrict__ sptr,
                                                  S* __restrict__ off, S* __restrict__ diag) {
  // the diagonal sum lives in shared memory (element k of this thread at
  // a[T k], conflict-free), which keeps the register count low enough for
  // several CTAs per SM
  constexpr int T = JacThreads<S>::T;
  __shared__ double sdiag[25 * T];
  __shared__ S soff[25 * T];  // the block being formed, written out as vectors
  double* a = sdiag + threadIdx.x;
  S* so = soff + threadIdx.x;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
#pragma unroll
  for (int k = 0; k < 25; ++k) a[T * k] = 0.0;
  double Vr[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) Vr[k] = P[8 * (size_t)r + k];
  const double volr = 1.0 / vol[r];
  const int p0 = nbr_ptr[r], p1 = nbr_ptr[r + 1];
  for (int p = p0; p < p1; ++p) {
    const int s = nbr_node[p];
    const int er = nbr_edge[p];
    const size_t e = (size_t)(er & 0x7fffffff);
    const double sg = er < 0 ? -1.0 : 1.0;
    const double n0 = en[e], n1 = en[(size_t)E + e], n2 = en[2 * (size_t)E + e];
    double Vs[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Vs[k] = P[8 * (size_t)s + k];
    const double rnorm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
    const size_t b = sl_blk(sptr, r, p - p0);
    const int lane = r & 31;
    auto flush = [&]() {
      S t[25];
#pragma unroll
      for (int k = 0; k < 25; ++k) t[k] = so[T * k];
      store_block_vec<S>(off, b, lane, t);
    };
    if (rnorm < 1e-18) {
#pragma unroll
      for (int k = 0; k < 25; ++k) so[T * k] = (S)0.0;
      flush();
      continue;
    }
    // the Jacobians are formed in the storage precision S (FP32 for the
    // mixed-precision solver) and summed into the diagonal in FP64
    const double invnorm = 1.0 / rnorm;
    const S un[3] = {(S)(n0 * invnorm), (S)(n1 * invnorm), (S)(n2 * invnorm)};
    const S half_rn = (S)(0.5 * rnorm);
    const S sco = (S)(TR ? -sg * (1.0 / vol[s]) : sg * volr);
    const S sgS = (S)sg;
    S VrS[5], VsS[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) { VrS[k] = (S)Vr[k]; VsS[k] = (S)Vs[k]; }
    const auto A = roe_avg<S>(g, un, VrS, VsS);
    const auto hr = h_state<S>(g, un, VrS);
    const auto hs = h_state<S>(g, un, VsS);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      S d[5];
      D_col<S>(g, A, un, j, d);
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const int el = 5 * m + j;
        // diagonal contribution: roejac(n, Vr, Vs, sg)
        const S jd = (H_elem<S>(g, hr, un, el) + sgS * d[m]) * half_rn;
        a[T * el] += sg * (double)jd;
        if (TR) {
          so[T * (5 * j + m)] = jd * sco;
        } else {
          // off-diagonal block: roejac(n, Vs, Vr, -sg)
          const S jo = (H_elem<S>(g, hs, un, el) + (-sgS) * d[m]) * half_rn;
          so[T * el] = jo * sco;
        }
      }
    }
    flush();
  }
  const int br = brow[r];
  if (br >= 0) {
#pragma unroll
    for (int k = 0; k < 25; ++k) a[T * k] += fsum[25 * (size_t)br + k];
  }
  double v[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) v[k] = a[T * k] * volr;
  if (dt) {
    const double c = 1.0 / dt[r];
#pragma unroll
    for (int k = 0; k < 5; ++k) v[6 * k] += c;
  }
  store_diag<S, TR>(diag, r, v);
}

// y += A x (or A^T x) for the block of lane l at base b of the sliced
// layout; FP64 accumulation in the order of a row-major gemv
template <class S, class TX>
__device__ __forceinline__ void gemv_sl(const S* __restrict__ a, size_t b, int l, const TX* __restrict__ x, double* y,
                                        bool trans) {
  double av[25];
  load_block<S>(a, b, l, av);
  double xv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) xv[k] = (double)x[k];
  if (!trans) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double s = av[5 * r] * xv[0];
#pragma unroll
      for (int c = 1; c < 5; ++c) s += av[5 * r + c] * xv[c];
      y[r] += s;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double s = av[r] * xv[0];
#pragma unroll
      for (int c = 1; c < 5; ++c) s += av[5 * c + r] * xv[c];
      y[r] += s;
    }
  }
}

// y = A p (or A^T p): per row, diagonal block first, then the row's
// neighbours in ascending order (SubDomain::computeMatVecProdH1 and
// H1transpose, SubDomain.C:3916-3995).  Blocks in S (float or double),
// vectors and accumulation in double.  One thread per row; a warp is one
// slice, so every block element is read as one coalesced line.  TRANS
// (stored blocks not transposed): block A_sr is read from row s's slice.
template <class S, bool TRANS, class TI, class TO>
__global__ void __launch_bounds__(256) k_spmv(int N, const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_tpos,
                                              const int* __restrict__ sptr, const int* __restrict__ scol,
                                              const S* __restrict__ diag, const S* __restrict__ off,
                                              const TI* __restrict__ p, TO* __restrict__ y,
                                              const int* __restrict__ skip) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N || (skip && *skip)) return;
  double acc[5] = {0, 0, 0, 0, 0};
  gemv_sl(diag, sl_dblk(r), r & 31, p + 5 * (size_t)r, acc, TRANS);
  const int p0 = nbr_ptr[r], cnt = nbr_ptr[r + 1] - p0;
  const size_t cb = (size_t)sptr[r >> 5] * 32 + (r & 31);
  int k0 = 0;
  if constexpr (std::is_same<S, float>::value && !TRANS) {
    // FP32 blocks: two neighbours per trip with all their loads issued
    // before the arithmetic (more bytes in flight per thread); the blocks
    // stay in FP32 registers until used; same accumulation order
    const int l = r & 31;
    for (; k0 + 1 < cnt; k0 += 2) {
      const int s0 = scol[cb + (size_t)32 * k0], s1 = scol[cb + (size_t)32 * (k0 + 1)];
      float a0[25], a1[25];
      const float4* q0 = reinterpret_cast<const float4*>(off + sl_blk(sptr, r, k0)) + l;
      const float4* q1 = reinterpret_cast<const float4*>(off + sl_blk(sptr, r, k0 + 1)) + l;
#pragma unroll
      for (int i = 0; i < 6; ++i) {
        const float4 t0 = q0[32 * i], t1 = q1[32 * i];
        a0[4 * i] = t0.x; a0[4 * i + 1] = t0.y; a0[4 * i + 2] = t0.z; a0[4 * i + 3] = t0.w;
        a1[4 * i] = t1.x; a1[4 * i + 1] = t1.y; a1[4 * i + 2] = t1.z; a1[4 * i + 3] = t1.w;
      }
      a0[24] = off[sl_blk(sptr, r, k0) + 768 + l];
      a1[24] = off[sl_blk(sptr, r, k0 + 1) + 768 + l];
      double x0[5], x1[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) {
        x0[c] = (double)p[5 * (size_t)s0 + c];
        x1[c] = (double)p[5 * (size_t)s1 + c];
      }
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
        double t = (double)a0[5 * rr] * x0[0];
#pragma unroll
        for (int c = 1; c < 5; ++c) t += (double)a0[5 * rr + c] * x0[c];
        acc[rr] += t;
      }
#pragma unroll
      for (int rr = 0; rr < 5; ++rr) {
        double t = (double)a1[5 * rr] * x1[0];
#pragma unroll
        for (int c = 1; c < 5; ++c) t += (double)a1[5 * rr + c] * x1[c];
        acc[rr] += t;
      }
    }
  }
  for (int k = k0; k < cnt; ++k) {
    const int s = scol[cb + (size_t)32 * k];
    if (!TRANS) {
      gemv_sl(off, sl_blk(sptr, r, k), r & 31, p + 5 * (size_t)s, acc, false);
    } else {
      const int kt = nbr_tpos[p0 + k] - nbr_ptr[s];
      gemv_sl(off, sl_blk(sptr, s, kt), s & 31, p + 5 * (size_t)s, acc, true);
    }
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) y[5 * (size_t)r + k] = (TO)acc[k];
}

// y_q = A p_q (or A^T p_q) for the R vectors of a batch (pointer arrays):
// every block is read once per group of RB vectors and applied to each in
// k_spmv's per-row order (diagonal block, then the neighbours ascending).
template <class S, bool TRANS, class TV, int RB>
__global__ void __launch_bounds__(256) k_spmv_batch(int N, int R, const int* __restrict__ nbr_ptr,
                                                    const int* __restrict__ nbr_tpos, const int* __restrict__ sptr,
                                                    const int* __restrict__ scol, const S* __restrict__ diag,
                                                    const S* __restrict__ off, const TV* const* __restrict__ P,
                                                    TV* const* __restrict__ Y) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int p0 = nbr_ptr[r], cnt = nbr_ptr[r + 1] - p0;
  const size_t cb = (size_t)sptr[r >> 5] * 32 + (r & 31);
  for (int q0 = 0; q0 < R; q0 += RB) {
    double acc[RB][5];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
      for (int k = 0; k < 5; ++k) acc[q][k] = 0.0;
    auto apply = [&](const double* av, int col, bool tr) {
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        if (q0 + q >= R) break;
        const TV* x = P[q0 + q] + 5 * (size_t)col;
        double xv[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) xv[k] = (double)x[k];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) {
          double t = (tr ? av[rr] : av[5 * rr]) * xv[0];
#pragma unroll
          for (int k = 1; k < 5; ++k) t += (tr ? av[5 * k + rr] : av[5 * rr + k]) * xv[k];
          acc[q][rr] += t;
        }
      }
    };
    double av[25];
    load_block<S>(diag, sl_dblk(r), r & 31, av);
    apply(av, r, TRANS);
    for (int k = 0; k < cnt; ++k) {
      const int sn = scol[cb + (size_t)32 * k];
      if (!TRANS) {
        load_block<S>(off, sl_blk(sptr, r, k), r & 31, av);
        apply(av, sn, false);
      } else {
        const int kt = nbr_tpos[p0 + k] - nbr_ptr[sn];
        load_block<S>(off, sl_blk(sptr, sn, kt), sn & 31, av);
        apply(av, sn, true);
      }
    }
#pragma unroll
    for (int q = 0; q < RB; ++q) {
      if (q0 + q >= R) break;
      TV* y = Y[q0 + q] + 5 * (size_t)r;
#pragma unroll
      for (int k = 0; k < 5; ++k) y[k] = (TV)acc[q][k];
    }
  }
}

// Block-Jacobi set-up (JacobiPrec::setup -> DiagMat::invert, DiagMatrix.C:
// 44-80): blocks with a zero diagonal entry are left as they are (as the
// reference does); a zero pivot counts into bad[0].
template <class S>
__global__ void k_bj_invert(int N, int n_owned, const S* __restrict__ diag, S* __restrict__ dinv,
                            int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const size_t b = sl_dblk(i);
  S a[25];
  if (i >= n_owned) {
    // ghost row of a subdomain mesh: identity (its partial block is not used)
#pragma unroll
    for (int k = 0; k < 25; ++k) a[k] = (k % 6 == 0) ? S(1) : S(0);
    store_block_vec<S>(dinv, b, i & 31, a);
    return;
  }
  {
    double t[25];
    load_block<S>(diag, b, i & 31, t);
#pragma unroll
    for (int k = 0; k < 25; ++k) a[k] = (S)t[k];
  }
  bool inv = true;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    if (a[6 * k] == S(0)) inv = false;
  if (inv && invert5<S>(a)) atomicAdd(bad, 1);
  store_block_vec<S>(dinv, b, i & 31, a);
}

// z = D^-1 x (or D^-T x): JacobiPrec::apply/applyT (KspPrec.C:86-111)
template <class S, class TI, class TO>
__global__ void k_bj_apply(int N, const S* __restrict__ dinv, const TI* __restrict__ x, TO* __restrict__ z,
                           int trans, const int* __restrict__ skip) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N || (skip && *skip)) return;
  double acc[5] = {0, 0, 0, 0, 0};
  gemv_sl(dinv, sl_dblk(i), i & 31, x + 5 * (size_t)i, acc, trans != 0);
#pragma unroll
  for (int k = 0; k < 5; ++k) z[5 * (size_t)i + k] = (TO)acc[k];
}

// ------------------------------------------------------------ vector ops
__global__ void k_axpby(size_t n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        double* __restrict__ z) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) z[q] = a * x[q] + b * y[q];
}
template <class TI, class TO>
__global__ void k_scale(size_t n, double a, const TI* __restrict__ x, TO* __restrict__ z) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) z[q] = (TO)(a * (double)x[q]);
}
// z = b - w
template <class TW, class TO>
__global__ void k_sub(size_t n, const double* __restrict__ b, const TW* __restrict__ w, TO* __restrict__ z) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) z[q] = (TO)(b[q] - (double)w[q]);
}
// Deterministic grid reduction finished by the last block: every block
// writes its partial sum (warp xor trees, then the warps in order), takes a
// ticket, and the block that takes the last ticket adds the partials in
// block order, writes *out and re-arms the ticket.
__device__ __forceinline__ double block_sum(double v, double* ws) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += ws[k];
  return t;
}
__device__ __forceinline__ void grid_sum_last_block(double v, double* __restrict__ part,
                                                    unsigned* __restrict__ ticket, double* __restrict__ out) {
  __shared__ double ws[32];
  __shared__ bool last;
  const double b = block_sum(v, ws);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) t += __ldcg(part + k);
  t = block_sum(t, ws);
  if (threadIdx.x == 0) {
    *out = t;
    *ticket = 0u;
  }
}

template <class TV> struct Vec16;
template <> struct Vec16<float> { using T = float4; static constexpr int W = 4; };
template <> struct Vec16<double> { using T = double2; static constexpr int W = 2; };

// Modified Gram-Schmidt step with the projection of the previous step fused
// in, 16-byte loads, and the reduction finished in the same launch:
//   w -= hprev * Vprev    (skipped when hprev is null)
//   *out = w . Vcur       (NORM: *out = w . w)
// w is rounded to TV after the projection, before the product, as the
// stored vector is.  All vectors 16-byte aligned.
template <class TV, bool NORM>
__global__ void __launch_bounds__(kIB) k_mgs(size_t n, const double* __restrict__ hprev, const TV* __restrict__ Vprev,
                                             const TV* __restrict__ Vcur, TV* __restrict__ w,
                                             double* __restrict__ part, unsigned* __restrict__ ticket,
                                             double* __restrict__ out) {
  using VT = typename Vec16<TV>::T;
  constexpr int W = Vec16<TV>::W;
  const double h = hprev ? *hprev : 0.0;
  const size_t nv = n / W;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  double s = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < nv; q += stride) {
    VT wv = reinterpret_cast<const VT*>(w)[q];
    TV* wp = reinterpret_cast<TV*>(&wv);
    if (hprev) {
      const VT pv = reinterpret_cast<const VT*>(Vprev)[q];
      const TV* pp = reinterpret_cast<const TV*>(&pv);
#pragma unroll
      for (int k = 0; k < W; ++k) wp[k] = (TV)((double)wp[k] - h * (double)pp[k]);
      reinterpret_cast<VT*>(w)[q] = wv;
    }
    if (NORM) {
#pragma unroll
      for (int k = 0; k < W; ++k) s += (double)wp[k] * (double)wp[k];
    } else {
      const VT cv = reinterpret_cast<const VT*>(Vcur)[q];
      const TV* cp = reinterpret_cast<const TV*>(&cv);
#pragma unroll
      for (int k = 0; k < W; ++k) s += (double)wp[k] * (double)cp[k];
    }
  }
  for (size_t q = nv * W + (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) {
    double wq = (double)w[q];
    if (hprev) {
      w[q] = (TV)(wq - h * (double)Vprev[q]);
      wq = (double)w[q];
    }
    s += wq * (NORM ? wq : (double)Vcur[q]);
  }
  grid_sum_last_block(s, part, ticket, out);
}
// x += sum_m y_m V_m   (y on the device, k terms)
template <class TV>
__global__ void k_combine(size_t n, int k, const double* __restrict__ y, const TV* __restrict__ V, size_t ld,
                          TV* __restrict__ out) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  double s = 0.0;
  for (int m = 0; m < k; ++m) s += y[m] * (double)V[(size_t)m * ld + q];
  out[q] = (TV)s;
}
// ---------------------------------------------------------------------
// Device-driven GMRES iteration (GmresSolver::solve, KspSolver.C:396-449,
// with applyPreviousRotations / applyNewRotation / backwardSolve,
// KspSolver.C:917-982): the modified Gram-Schmidt steps of one iteration,
// the Givens update of the Hessenberg column and the next basis vector in
// one cooperative launch.  Every CTA owns a fixed slice of the vectors; the
// projections run in the reference's MGS order, one grid-wide sum per step
// (partials in CTA order, identical in every CTA); the grid barriers are
// bounded spins that record a timeout in ist[3] and never hang.  The
// rotation arithmetic is written with explicitly rounded operations (no
// contraction), so it is the host loop's arithmetic.  Once ist[1] (done)
// is set, the rest of the cycle's kernels return at once, so the host
// waits for the GPU only once per restart cycle.
constexpr int kMaxKrylov = 64;
constexpr int kCoopThreads = 256;
struct GmresState {
  double* H;        // [(m+1) * m], h(i, j) = H[i m + j]
  double* cs;       // [2 m] rotations
  double* g;        // [m + 1] right-hand side of the least-squares problem
  double* y;        // [m] its solution
  double* scal;     // [0] estimated residual norm, [1] target
  int* ist;         // [0] iterations, [1] done, [2] last column, [3] barrier timeout, [4] maxits, [5] breakdown
  double* part;     // [2][grid] per-CTA partial sums
  unsigned* bar;    // grid barrier arrivals (zeroed per cycle)
};

// bounded grid barrier: every CTA adds one arrival and waits until the
// count reaches target (co-residency is guaranteed by the cooperative
// launch); after about a second a timeout is recorded and the CTA goes on
__device__ __forceinline__ void grid_barrier(unsigned* bar, unsigned target, int* timeout) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    unsigned spins = 0;
    while (*(volatile unsigned*)bar < target) {
      if (++spins > (1u << 23)) {
        atomicExch(timeout, 1);
        break;
      }
      __nanosleep(128);
    }
    __threadfence();
  }
  __syncthreads();
}

template <class TV>
__global__ void __launch_bounds__(kCoopThreads, 4) k_gmres_iter(size_t n, int j, int m, TV* __restrict__ V,
                                                               size_t ld, TV* __restrict__ w, GmresState st,
                                                               unsigned base) {
  if (*(volatile int*)(st.ist + 1)) return;
  __shared__ double ws[32];
  __shared__ double hsh[kMaxKrylov + 2];
  __shared__ double css[2 * kMaxKrylov];
  __shared__ double sprev[3];  // g[j], estimated residual, target
  __shared__ int iprev[2];     // iterations, maxits
  __shared__ double sinv;
  __shared__ int sdone;
  // the previous state is read before the first barrier: CTA 0 overwrites
  // it only after the last one
  for (int k = threadIdx.x; k < 2 * j; k += blockDim.x) css[k] = st.cs[k];
  if (threadIdx.x == 0) {
    sprev[0] = st.g[j];
    sprev[1] = st.scal[0];
    sprev[2] = st.scal[1];
    iprev[0] = st.ist[0];
    iprev[1] = st.ist[4];
  }
  using VT = typename Vec16<TV>::T;
  constexpr int W = Vec16<TV>::W;
  const size_t nv = n / W;
  const size_t per = (nv + gridDim.x - 1) / gridDim.x;
  const size_t lo = min(nv, (size_t)blockIdx.x * per), hi = min(nv, lo + per);
  const bool tail = blockIdx.x == gridDim.x - 1;
  unsigned target = base;
  for (int i = 0; i <= j + 1; ++i) {
    const bool norm = i == j + 1;
    const bool proj = i > 0;
    const double h = proj ? hsh[i - 1] : 0.0;
    const TV* Vp = proj ? V + (size_t)(i - 1) * ld : nullptr;
    const TV* Vc = norm ? nullptr : V + (size_t)i * ld;
    double s = 0.0;
    // two vectors of each array per thread and trip, loads issued first
    constexpr int U = 2;
    for (size_t q0 = lo + threadIdx.x; q0 < hi; q0 += (size_t)U * blockDim.x) {
      VT wv[U], pv[U], cv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const size_t q = q0 + (size_t)u * blockDim.x;
        if (q < hi) {
          wv[u] = reinterpret_cast<const VT*>(w)[q];
          if (proj) pv[u] = reinterpret_cast<const VT*>(Vp)[q];
          if (!norm) cv[u] = reinterpret_cast<const VT*>(Vc)[q];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const size_t q = q0 + (size_t)u * blockDim.x;
        if (q >= hi) break;
        TV* wp = reinterpret_cast<TV*>(&wv[u]);
        if (proj) {
          const TV* pp = reinterpret_cast<const TV*>(&pv[u]);
#pragma unroll
          for (int k = 0; k < W; ++k) wp[k] = (TV)((double)wp[k] - h * (double)pp[k]);
          reinterpret_cast<VT*>(w)[q] = wv[u];
        }
        if (norm) {
#pragma unroll
          for (int k = 0; k < W; ++k) s += (double)wp[k] * (double)wp[k];
        } else {
          const TV* cp = reinterpret_cast<const TV*>(&cv[u]);
#pragma unroll
          for (int k = 0; k < W; ++k) s += (double)wp[k] * (double)cp[k];
        }
      }
    }
    if (tail)
      for (size_t q = nv * W + threadIdx.x; q < n; q += blockDim.x) {
        double wq = (double)w[q];
        if (proj) {
          w[q] = (TV)(wq - h * (double)Vp[q]);
          wq = (double)w[q];
        }
        s += wq * (norm ? wq : (double)Vc[q]);
      }
    const double b = block_sum(s, ws);
    double* part = st.part + (size_t)(i & 1) * gridDim.x;
    if (threadIdx.x == 0) part[blockIdx.x] = b;
    target += gridDim.x;
    grid_barrier(st.bar, target, st.ist + 3);
    double t = 0.0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) t += __ldcg(part + k);
    t = block_sum(t, ws);
    if (threadIdx.x == 0) hsh[i] = t;
    __syncthreads();
  }
  // Givens update of column j (every CTA computes it; CTA 0 stores it)
  if (threadIdx.x == 0) {
    double hc[kMaxKrylov + 1];
    for (int i = 0; i <= j; ++i) hc[i] = hsh[i];
    const double hj1 = __dsqrt_rn(hsh[j + 1]);
    const bool breakdown = hj1 == 0.0;
    for (int i = 0; i < j; ++i) {
      const double c0 = css[2 * i], c1 = css[2 * i + 1];
      const double a = hc[i], bb = hc[i + 1];
      hc[i] = __dadd_rn(__dmul_rn(c1, a), __dmul_rn(c0, bb));
      hc[i + 1] = __dadd_rn(__dmul_rn(-c0, a), __dmul_rn(c1, bb));
    }
    double c0, c1;
    const double hjj = hc[j];
    if (__dmul_rn(hjj, hjj) == 0.0) {
      c1 = 0.0;
      c0 = 1.0;
    } else {
      const double coef = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(__dmul_rn(hjj, hjj), __dmul_rn(hj1, hj1))));
      c1 = __dmul_rn(__dsqrt_rn(__dmul_rn(hjj, hjj)), coef);
      c0 = __ddiv_rn(__dmul_rn(c1, hj1), hjj);
    }
    hc[j] = __dadd_rn(__dmul_rn(c1, hjj), __dmul_rn(c0, hj1));
    const double gj = sprev[0];
    const double gj1 = __dmul_rn(-c0, gj);
    const int iter = iprev[0] + 1;
    double l2res = sprev[1];
    bool done = breakdown;
    if (!breakdown) {
      l2res = fabs(gj1);
      done = l2res <= sprev[2] || iter >= iprev[1];
    }
    sdone = done;
    sinv = breakdown ? 0.0 : 1. / hj1;
    if (blockIdx.x == 0) {
      for (int i = 0; i <= j; ++i) st.H[(size_t)i * m + j] = hc[i];
      st.H[(size_t)(j + 1) * m + j] = 0.0;
      st.cs[2 * j] = c0;
      st.cs[2 * j + 1] = c1;
      st.g[j + 1] = gj1;
      st.g[j] = __dmul_rn(c1, gj);
      st.scal[0] = l2res;
      st.ist[0] = iter;
      st.ist[2] = j;
      st.ist[5] = breakdown;
    }
  }
  __syncthreads();
  // every CTA has read what it needs of the previous state; CTA 0's done
  // flag is written after the grid's last barrier, so no CTA of this launch
  // reads it again
  if (sdone) {
    if (blockIdx.x == 0 && threadIdx.x == 0) st.ist[1] = 1;
    return;
  }
  const double a = sinv;
  TV* Vn = V + (size_t)(j + 1) * ld;
  for (size_t q = lo * W + threadIdx.x; q < hi * W; q += blockDim.x) Vn[q] = (TV)(a * (double)w[q]);
  if (tail)
    for (size_t q = nv * W + threadIdx.x; q < n; q += blockDim.x) Vn[q] = (TV)(a * (double)w[q]);
}

// back substitution (KspSolver.C:966-982) of the last cycle, one thread:
// y[0..jl] from the rotated Hessenberg matrix and g
__global__ void k_gmres_backsolve(int m, GmresState st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int j = st.ist[2];
  for (int i = j; i >= 0; --i) {
    double yi = st.g[i];
    for (int k = j; k >= i + 1; --k) yi = __dsub_rn(yi, __dmul_rn(st.H[(size_t)i * m + k], st.y[k]));
    st.y[i] = __ddiv_rn(yi, st.H[(size_t)i * m + i]);
  }
}
// out = sum_{m <= last column} y_m V_m
template <class TV>
__global__ void k_combine_dev(size_t n, const int* __restrict__ jl, const double* __restrict__ y,
                              const TV* __restrict__ V, size_t ld, TV* __restrict__ out) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int k = *jl + 1;
  double s = 0.0;
  for (int mm = 0; mm < k; ++mm) s += y[mm] * (double)V[(size_t)mm * ld + q];
  out[q] = (TV)s;
}

template <class TA>
__global__ void k_add(size_t n, const TA* __restrict__ a, double* __restrict__ x) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) x[q] += (double)a[q];
}

// SubDomain::checkSolution (SubDomain.C:6746-6806): per node, one count for
// a non-positive density and one for a non-positive pressure of the
// conservative state (NaN counts too: such a state is not physical either).
__global__ void k_check_solution(int N, Gas g, const double* __restrict__ U, int* __restrict__ nbad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) u[k] = U[5 * (size_t)i + k];
  cons2prim(g, u, v);
  const int b = (int)!(v[0] > 0.0) + (int)!(v[4] > 0.0);
  if (b) atomicAdd(nbad, b);
}

}  // namespace aerof

// ====================================================================== host
namespace aerof {

static void need_mesh_or_throw(aerof_gpu_ctx* c) {
  if (!c->has_mesh) throw ApiError{AEROF_ESTATE, "no mesh: call aerof_gpu_set_mesh first"};
}
static void need_jac(aerof_gpu_ctx* c) {
  need_mesh_or_throw(c);
  if (!c->imp.precision) throw ApiError{AEROF_ESTATE, "no Jacobian: call aerof_gpu_jacobian first"};
}

// Assemble the H1 operator at device state dU with device time steps ddt
// (may be null).
// sizes of the sliced arrays (elements)
static size_t sl_diag_size(const DeviceMesh& m) { return (size_t)m.nsl * 800; }
static size_t sl_off_size(const DeviceMesh& m) { return std::max<size_t>((size_t)m.h_sptr.back() * 800, 1); }

void jacobian_dev(aerof_gpu_ctx* c, const double* dU, const double* ddt, int precision, bool transposed) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const Gas g = make_gas(c->cfg.gamma);
  TimerScope tj(c, AEROF_T_FV_JAC);
  prim_dev(c, dU);
  J.fsum.ensure(25 * (size_t)std::max(m.nbrow, 1));
  if (m.nbrow) {
    k_jac_faces<<<grid_for((size_t)m.nbrow, 128), 128, 0, c->stream>>>(m.nbrow, m.F, g, m.Ubd.p, m.blist.p, m.nf_ptr.p,
                                                                      m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p,
                                                                      J.fsum.p);
    AEROF_LAUNCH_CHECK();
  }
  auto rows = [&](auto* off, auto* diag, auto kern) {
    constexpr int T = JacThreads<std::remove_pointer_t<decltype(off)>>::T;
    kern<<<grid_for((size_t)m.N, T), T, 0, c->stream>>>(m.N, m.E, m.F, g, m.Ubd.p, m.nbr_ptr.p, m.nbr_node.p,
                                                        m.nbr_edge.p, m.en.p, m.P.p, m.vol.p, m.brow.p, J.fsum.p, ddt,
                                                        m.sptr.p, off, diag);
    AEROF_LAUNCH_CHECK();
  };
  if (precision == AEROF_PREC_FP32) {
    J.diag64.release(); J.off64.release(); J.dinv64.release();
    J.diag32.alloc(sl_diag_size(m));
    J.off32.alloc(sl_off_size(m));
    if (transposed) rows(J.off32.p, J.diag32.p, k_jac_rows<float, true>);
    else rows(J.off32.p, J.diag32.p, k_jac_rows<float, false>);
  } else {
    J.diag32.release(); J.off32.release(); J.dinv32.release();
    J.diag64.alloc(sl_diag_size(m));
    J.off64.alloc(sl_off_size(m));
    if (transposed) rows(J.off64.p, J.diag64.p, k_jac_rows<double, true>);
    else rows(J.off64.p, J.diag64.p, k_jac_rows<double, false>);
  }
  J.precision = precision;
  J.transposed = transposed;
  J.prec_ready = false;
  J.ilu_ready = false;
}

// products with H1 (trans = 0) or H1^T (trans = 1); the stored blocks may
// hold either, so the kernel reads them plainly or transposed
// skip (device flag, may be null): when set, the kernel returns at once
// (the device-driven GMRES leaves the rest of a converged cycle idle)
template <class TI, class TO>
void matvec_t(aerof_gpu_ctx* c, const TI* p, TO* y, int trans, const int* skip = nullptr) {
  DeviceMesh& m = c->mesh;
  TimerScope tm(c, AEROF_T_KSP_MATVEC);
  Implicit& J = c->imp;
  const int gn = grid_for(m.N, kIB);
  const bool tr = (trans != 0) != J.transposed;
  auto go = [&](auto kern, auto* diag, auto* off) {
    kern<<<gn, kIB, 0, c->stream>>>(m.N, m.nbr_ptr.p, m.nbr_tpos.p, m.sptr.p, m.scol.p, diag, off, p, y, skip);
    AEROF_LAUNCH_CHECK();
  };
  if (J.precision == AEROF_PREC_FP32) {
    if (tr) go(k_spmv<float, true, TI, TO>, J.diag32.p, J.off32.p);
    else go(k_spmv<float, false, TI, TO>, J.diag32.p, J.off32.p);
  } else {
    if (tr) go(k_spmv<double, true, TI, TO>, J.diag64.p, J.off64.p);
    else go(k_spmv<double, false, TI, TO>, J.diag64.p, J.off64.p);
  }
}
void matvec_dev(aerof_gpu_ctx* c, const double* p, double* y, int trans) { matvec_t<double, double>(c, p, y, trans); }

// ---------------------------------------------------------------------
// Block ILU(0) (IluPrec, KspPrec.C:138-330; SparseMat::numericILU and
// lusol, SparseMatrix.C:353-450) in the multicolour ordering: the
// reference's algorithm (IKJ elimination, multiplier A_ik U_kk^-1, updates
// of the row's own pattern only, inverted diagonal; forward solve with the
// unit lower part, backward solve with the upper part and the inverted
// diagonal) on rows sorted by colour instead of the reference's RCM order,
// so the rows of one colour, which are never neighbours, factor and solve
// in parallel: one launch per colour.  The factors live in H1's sliced
// layout (slices of 32 rows of one colour, entry k of a slice as one
// lane-interleaved block), so a warp reads entry k of its 32 rows as
// coalesced 16-byte vectors.

// the operator's blocks (tr: transposed) copied into the sliced ILU
// pattern, thread per colour-order row
template <class S>
__global__ void k_ilu_gather(int N, int tr, const int* __restrict__ cperm, const int* __restrict__ rlen,
                             const int* __restrict__ rsl, const int* __restrict__ sr0, const int* __restrict__ isp,
                             const int* __restrict__ jsrc, const int* __restrict__ nbr_ptr,
                             const int* __restrict__ nbr_node, const int* __restrict__ nbr_tpos,
                             const int* __restrict__ sptr, const S* __restrict__ diag, const S* __restrict__ off,
                             S* __restrict__ lu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int r = cperm[i];
  const int ws = rsl[i], wl = i - sr0[ws];
  for (int k = 0; k < rlen[i]; ++k) {
    const size_t e = (size_t)isp[ws] + k;
    const int src = jsrc[e * 32 + wl];
    double v[25];
    if (src < 0) {
      load_block<S>(diag, sl_dblk(r), r & 31, v);
    } else if (!tr) {
      load_block<S>(off, sl_blk(sptr, r, src), r & 31, v);
    } else {
      const int p = nbr_ptr[r] + src;
      const int sn = nbr_node[p];
      load_block<S>(off, sl_blk(sptr, sn, nbr_tpos[p] - nbr_ptr[sn]), sn & 31, v);
    }
    S o[25];
#pragma unroll
    for (int q = 0; q < 25; ++q) o[q] = (S)(tr ? v[5 * (q % 5) + q / 5] : v[q]);
    store_block_vec<S>(lu, e * 800, wl, o);
  }
}

// numericILU for the rows of one colour (all their lower neighbours belong
// to earlier colours, already factored), thread per row, following the
// precomputed schedule: per lower entry the multiplier A_ik U_kk^-1, then
// the updates A_ij -= mult U_kj of the row's own pattern; finally the
// diagonal inverted.  Entry e is lane e % 32 of block e / 32.
template <class S>
__device__ __forceinline__ void ilu_ld(const S* __restrict__ lu, int e, double* v) {
  load_block<S>(lu, (size_t)(e >> 5) * 800, e & 31, v);
}
template <class S>
__device__ __forceinline__ void ilu_st(S* __restrict__ lu, int e, const double* v) {
  S o[25];
#pragma unroll
  for (int q = 0; q < 25; ++q) o[q] = (S)v[q];
  store_block_vec<S>(lu, (size_t)(e >> 5) * 800, e & 31, o);
}
template <class S>
__global__ void k_ilu_factor(int i0, int cnt, int s0, const int* __restrict__ rju, const int* __restrict__ isp,
                             const int* __restrict__ lo_ptr, const int2* __restrict__ lo,
                             const int* __restrict__ up_ptr, const int2* __restrict__ up, S* __restrict__ lu,
                             int* __restrict__ bad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cnt) return;
  const int i = i0 + t;
  for (int q = lo_ptr[i]; q < lo_ptr[i + 1]; ++q) {
    const int2 au = lo[q];
    double a[25], u[25], mult[25];
    ilu_ld<S>(lu, au.x, a);
    ilu_ld<S>(lu, au.y, u);
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int cc = 0; cc < 5; ++cc) {
        double x = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) x += a[5 * r + k] * u[5 * k + cc];
        mult[5 * r + cc] = x;
      }
    ilu_st<S>(lu, au.x, mult);
    for (int p = up_ptr[q]; p < up_ptr[q + 1]; ++p) {
      const int2 bm = up[p];
      double bb[25], am[25];
      ilu_ld<S>(lu, bm.x, bb);
      ilu_ld<S>(lu, bm.y, am);
#pragma unroll
      for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int cc = 0; cc < 5; ++cc) {
          double x = am[5 * r + cc];
#pragma unroll
          for (int k = 0; k < 5; ++k) x -= mult[5 * r + k] * bb[5 * k + cc];
          am[5 * r + cc] = x;
        }
      ilu_st<S>(lu, bm.y, am);
    }
  }
  const int ed = (isp[s0 + (t >> 5)] + rju[i]) * 32 + (t & 31);
  double dg[25];
  ilu_ld<S>(lu, ed, dg);
  if (invert5<double>(dg)) atomicAdd(bad, 1);
  ilu_st<S>(lu, ed, dg);
}

// lusol sweeps for one colour, L lanes per row (entries r, r + L, ... of
// the row, fixed xor-tree lane sum): row t of the colour is in slice
// s0 + t / 32 at lane t % 32.
// Forward: w_i = x_(perm i) - sum_{k<i} L_ik w_k.
template <int L, class S, class TI>
__global__ void k_ilu_fwd(int i0, int cnt, int s0, const int* __restrict__ cperm, const int* __restrict__ rju,
                          const int* __restrict__ isp, const int* __restrict__ jc, const S* __restrict__ lu,
                          const TI* __restrict__ x, double* __restrict__ w, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = g / L, sub = g % L;
  const bool act = t < cnt;
  double acc[5] = {0, 0, 0, 0, 0};
  if (act) {
    const int lane = t & 31;
    const size_t base = (size_t)isp[s0 + (t >> 5)];
    const int d = rju[i0 + t];
    for (int k = sub; k < d; k += L) {
      double a[25];
      load_block<S>(lu, (base + k) * 800, lane, a);
      const double* wk = w + 5 * (size_t)jc[(base + k) * 32 + lane];
      double v[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) v[c] = wk[c];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < 5; ++c) acc[rr] -= a[5 * rr + c] * v[c];
    }
  }
#pragma unroll
  for (int o = 1; o < L; o <<= 1)
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  if (!act || sub != 0) return;
  const int i = i0 + t;
  const size_t r = (size_t)cperm[i];
#pragma unroll
  for (int c = 0; c < 5; ++c) w[5 * (size_t)i + c] = (double)x[5 * r + c] + acc[c];
}

// Backward: w_i = U_ii^-1 (w_i - sum_{j>i} U_ij w_j), also written to z in
// the caller's numbering.
template <int L, class S, class TO>
__global__ void k_ilu_bwd(int i0, int cnt, int s0, const int* __restrict__ cperm, const int* __restrict__ rlen,
                          const int* __restrict__ rju, const int* __restrict__ isp, const int* __restrict__ jc,
                          const S* __restrict__ lu, double* __restrict__ w, TO* __restrict__ z,
                          const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = g / L, sub = g % L;
  const bool act = t < cnt;
  double acc[5] = {0, 0, 0, 0, 0};
  int lane = 0, d = 0;
  size_t base = 0;
  if (act) {
    lane = t & 31;
    base = (size_t)isp[s0 + (t >> 5)];
    d = rju[i0 + t];
    const int len = rlen[i0 + t];
    for (int k = d + 1 + sub; k < len; k += L) {
      double a[25];
      load_block<S>(lu, (base + k) * 800, lane, a);
      const double* wk = w + 5 * (size_t)jc[(base + k) * 32 + lane];
      double v[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) v[c] = wk[c];
#pragma unroll
      for (int rr = 0; rr < 5; ++rr)
#pragma unroll
        for (int c = 0; c < 5; ++c) acc[rr] -= a[5 * rr + c] * v[c];
    }
  }
#pragma unroll
  for (int o = 1; o < L; o <<= 1)
#pragma unroll
    for (int c = 0; c < 5; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
  if (!act || sub != 0) return;
  const int i = i0 + t;
#pragma unroll
  for (int c = 0; c < 5; ++c) acc[c] += w[5 * (size_t)i + c];
  double dg[25], res[5];
  load_block<S>(lu, (base + d) * 800, lane, dg);
#pragma unroll
  for (int rr = 0; rr < 5; ++rr) {
    double x = 0.0;
#pragma unroll
    for (int c = 0; c < 5; ++c) x += dg[5 * rr + c] * acc[c];
    res[rr] = x;
  }
  const size_t r = (size_t)cperm[i];
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    w[5 * (size_t)i + c] = res[c];
    z[5 * r + c] = (TO)res[c];
  }
}

// The same sweeps for R vectors at once (pointer arrays X, Z; work vectors
// W + q * ldw): every factor block is read once per group of RB vectors.
template <int L, int RB, class S, class TI>
__global__ void k_ilu_fwd_b(int i0, int cnt, int s0, int R, const int* __restrict__ cperm,
                            const int* __restrict__ rju, const int* __restrict__ isp, const int* __restrict__ jc,
                            const S* __restrict__ lu, const TI* const* __restrict__ X, double* __restrict__ W,
                            size_t ldw) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = g / L, sub = g % L;
  const bool act = t < cnt;
  const int lane = t & 31;
  const size_t base = act ? (size_t)isp[s0 + (t >> 5)] : 0;
  const int d = act ? rju[i0 + t] : 0;
  for (int q0 = 0; q0 < R; q0 += RB) {
    double acc[RB][5];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[q][c] = 0.0;
    for (int k = sub; k < d; k += L) {
      double a[25];
      load_block<S>(lu, (base + k) * 800, lane, a);
      const size_t col = 5 * (size_t)jc[(base + k) * 32 + lane];
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        if (q0 + q >= R) break;
        const double* wk = W + (size_t)(q0 + q) * ldw + col;
        double v[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) v[c] = wk[c];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
          for (int c = 0; c < 5; ++c) acc[q][rr] -= a[5 * rr + c] * v[c];
      }
    }
#pragma unroll
    for (int o = 1; o < L; o <<= 1)
#pragma unroll
      for (int q = 0; q < RB; ++q)
#pragma unroll
        for (int c = 0; c < 5; ++c) acc[q][c] += __shfl_xor_sync(0xffffffffu, acc[q][c], o);
    if (act && sub == 0) {
      const int i = i0 + t;
      const size_t r = (size_t)cperm[i];
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        if (q0 + q >= R) break;
        double* wi = W + (size_t)(q0 + q) * ldw + 5 * (size_t)i;
#pragma unroll
        for (int c = 0; c < 5; ++c) wi[c] = (double)X[q0 + q][5 * r + c] + acc[q][c];
      }
    }
  }
}
template <int L, int RB, class S, class TO>
__global__ void k_ilu_bwd_b(int i0, int cnt, int s0, int R, const int* __restrict__ cperm,
                            const int* __restrict__ rlen, const int* __restrict__ rju, const int* __restrict__ isp,
                            const int* __restrict__ jc, const S* __restrict__ lu, double* __restrict__ W, size_t ldw,
                            TO* const* __restrict__ Z) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = g / L, sub = g % L;
  const bool act = t < cnt;
  const int lane = t & 31;
  const size_t base = act ? (size_t)isp[s0 + (t >> 5)] : 0;
  const int d = act ? rju[i0 + t] : 0, len = act ? rlen[i0 + t] : 0;
  for (int q0 = 0; q0 < R; q0 += RB) {
    double acc[RB][5];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[q][c] = 0.0;
    for (int k = d + 1 + sub; k < len; k += L) {
      double a[25];
      load_block<S>(lu, (base + k) * 800, lane, a);
      const size_t col = 5 * (size_t)jc[(base + k) * 32 + lane];
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        if (q0 + q >= R) break;
        const double* wk = W + (size_t)(q0 + q) * ldw + col;
        double v[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) v[c] = wk[c];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
          for (int c = 0; c < 5; ++c) acc[q][rr] -= a[5 * rr + c] * v[c];
      }
    }
#pragma unroll
    for (int o = 1; o < L; o <<= 1)
#pragma unroll
      for (int q = 0; q < RB; ++q)
#pragma unroll
        for (int c = 0; c < 5; ++c) acc[q][c] += __shfl_xor_sync(0xffffffffu, acc[q][c], o);
    if (act && sub == 0) {
      const int i = i0 + t;
      const size_t r = (size_t)cperm[i];
      double dg[25];
      load_block<S>(lu, (base + d) * 800, lane, dg);
#pragma unroll
      for (int q = 0; q < RB; ++q) {
        if (q0 + q >= R) break;
        double* wi = W + (size_t)(q0 + q) * ldw + 5 * (size_t)i;
        double v[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) v[c] = acc[q][c] + wi[c];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr) {
          double x = 0.0;
#pragma unroll
          for (int c = 0; c < 5; ++c) x += dg[5 * rr + c] * v[c];
          wi[rr] = x;
          Z[q0 + q][5 * r + rr] = (TO)x;
        }
      }
    }
  }
}

// gather + factorisation of the operator read with orientation tr;
// returns the number of singular diagonal blocks (waits for the stream)
static int ilu_setup(aerof_gpu_ctx* c, int tr) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  cudaStream_t s = c->stream;
  c->s.counters.ensure(8);
  int* bad = c->s.counters.p + 5;
  AEROF_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
  const int gn = grid_for(m.N, kIB);
  auto run = [&](auto* lu, auto* diag, auto* off) {
    using S = std::remove_pointer_t<decltype(lu)>;
    k_ilu_gather<S><<<gn, kIB, 0, s>>>(m.N, tr, m.cperm.p, m.rlen.p, m.rsl.p, m.sr0.p, m.isp.p, m.jsrc.p,
                                       m.nbr_ptr.p, m.nbr_node.p, m.nbr_tpos.p, m.sptr.p, diag, off, lu);
    AEROF_LAUNCH_CHECK();
    for (int col = 0; col < m.ncolor; ++col) {
      const int i0 = m.h_cptr[col], cnt = m.h_cptr[col + 1] - i0;
      // 64-thread CTAs: one colour's rows spread over every SM and several
      // CTAs of this register-heavy kernel fit on each
      constexpr int kFT = 64;
      k_ilu_factor<S><<<grid_for(cnt, kFT), kFT, 0, s>>>(i0, cnt, m.h_cslice[col], m.rju.p, m.isp.p, m.lo_ptr.p,
                                                         m.lo.p, m.up_ptr.p, m.up.p, lu, bad);
      AEROF_LAUNCH_CHECK();
    }
  };
  if (J.precision == AEROF_PREC_FP32) {
    J.ilu32.ensure(800 * m.ilu_blocks);
    run(J.ilu32.p, J.diag32.p, J.off32.p);
  } else {
    J.ilu64.ensure(800 * m.ilu_blocks);
    run(J.ilu64.p, J.diag64.p, J.off64.p);
  }
  int h = 0;
  AEROF_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  AEROF_CUDA(cudaStreamSynchronize(s));
  J.ilu_ready = true;
  J.ilu_tr = tr;
  return h;
}

template <class TI, class TO>
static void ilu_apply(aerof_gpu_ctx* c, const TI* x, TO* z, const int* skip = nullptr) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  cudaStream_t s = c->stream;
  J.iluw.ensure(5 * (size_t)m.N);
  double* w = J.iluw.p;
  auto run = [&](const auto* lu) {
    using S = std::remove_const_t<std::remove_pointer_t<decltype(lu)>>;
    constexpr int L = 4;  // lanes per row
    for (int col = 0; col < m.ncolor; ++col) {
      const int i0 = m.h_cptr[col], cnt = m.h_cptr[col + 1] - i0;
      k_ilu_fwd<L, S, TI><<<grid_for((size_t)L * cnt, kIB), kIB, 0, s>>>(i0, cnt, m.h_cslice[col], m.cperm.p,
                                                                         m.rju.p, m.isp.p, m.jc.p, lu, x, w, skip);
      AEROF_LAUNCH_CHECK();
    }
    for (int col = m.ncolor - 1; col >= 0; --col) {
      const int i0 = m.h_cptr[col], cnt = m.h_cptr[col + 1] - i0;
      k_ilu_bwd<L, S, TO><<<grid_for((size_t)L * cnt, kIB), kIB, 0, s>>>(i0, cnt, m.h_cslice[col], m.cperm.p,
                                                                         m.rlen.p, m.rju.p, m.isp.p, m.jc.p, lu, w,
                                                                         z, skip);
      AEROF_LAUNCH_CHECK();
    }
  };
  if (J.precision == AEROF_PREC_FP32) run((const float*)J.ilu32.p);
  else run((const double*)J.ilu64.p);
}

// z_q = (LU)^-1 x_q for R vectors (device pointer arrays on the host)
template <class TI, class TO>
static void ilu_apply_batch(aerof_gpu_ctx* c, int R, const TI* const* x, TO* const* z) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  cudaStream_t s = c->stream;
  const size_t ldw = 5 * (size_t)m.N;
  J.iluw.ensure((size_t)R * ldw);
  J.iptr.ensure(2 * (size_t)R);
  std::vector<unsigned long long> p(2 * (size_t)R);
  for (int q = 0; q < R; ++q) {
    p[q] = (unsigned long long)x[q];
    p[R + q] = (unsigned long long)z[q];
  }
  AEROF_CUDA(cudaMemcpyAsync(J.iptr.p, p.data(), sizeof(unsigned long long) * 2 * (size_t)R, cudaMemcpyHostToDevice,
                             s));
  const TI* const* X = reinterpret_cast<const TI* const*>(J.iptr.p);
  TO* const* Z = reinterpret_cast<TO* const*>(J.iptr.p + R);
  double* w = J.iluw.p;
  auto run = [&](const auto* lu) {
    using S = std::remove_const_t<std::remove_pointer_t<decltype(lu)>>;
    constexpr int L = 4, RB = 4;
    for (int col = 0; col < m.ncolor; ++col) {
      const int i0 = m.h_cptr[col], cnt = m.h_cptr[col + 1] - i0;
      k_ilu_fwd_b<L, RB, S, TI><<<grid_for((size_t)L * cnt, kIB), kIB, 0, s>>>(
          i0, cnt, m.h_cslice[col], R, m.cperm.p, m.rju.p, m.isp.p, m.jc.p, lu, X, w, ldw);
      AEROF_LAUNCH_CHECK();
    }
    for (int col = m.ncolor - 1; col >= 0; --col) {
      const int i0 = m.h_cptr[col], cnt = m.h_cptr[col + 1] - i0;
      k_ilu_bwd_b<L, RB, S, TO><<<grid_for((size_t)L * cnt, kIB), kIB, 0, s>>>(
          i0, cnt, m.h_cslice[col], R, m.cperm.p, m.rlen.p, m.rju.p, m.isp.p, m.jc.p, lu, w, ldw, Z);
      AEROF_LAUNCH_CHECK();
    }
  };
  if (J.precision == AEROF_PREC_FP32) run((const float*)J.ilu32.p);
  else run((const double*)J.ilu64.p);
}

int prec_setup_dev(aerof_gpu_ctx* c, int trans = 0) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  TimerScope tp(c, AEROF_T_PREC_SETUP);
  if (J.pc == AEROF_PC_ILU0) {
    const int h = ilu_setup(c, ((trans != 0) != J.transposed) ? 1 : 0);
    J.prec_ready = true;
    return h;
  }
  c->s.counters.ensure(8);
  int* bad = c->s.counters.p + 4;
  AEROF_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  const int gn = grid_for(m.N, kIB);
  if (J.precision == AEROF_PREC_FP32) {
    J.dinv32.alloc(sl_diag_size(m));
    k_bj_invert<float><<<gn, kIB, 0, c->stream>>>(m.N, c->n_owned, J.diag32.p, J.dinv32.p, bad);
  } else {
    J.dinv64.alloc(sl_diag_size(m));
    k_bj_invert<double><<<gn, kIB, 0, c->stream>>>(m.N, c->n_owned, J.diag64.p, J.dinv64.p, bad);
  }
  AEROF_LAUNCH_CHECK();
  int h = 0;
  AEROF_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AEROF_CUDA(cudaStreamSynchronize(c->stream));
  J.prec_ready = true;
  return h;
}

// z = D^-1 x or D^-T x; with transposed storage the inverted blocks are
// those of D^T, so the roles swap
template <class TI, class TO>
void prec_apply_t(aerof_gpu_ctx* c, const TI* x, TO* z, int trans, const int* skip = nullptr) {
  DeviceMesh& m = c->mesh;
  TimerScope tp(c, AEROF_T_KSP_OTHER);
  Implicit& J = c->imp;
  const int gn = grid_for(m.N, kIB);
  const int tr = ((trans != 0) != J.transposed) ? 1 : 0;
  if (J.pc == AEROF_PC_ILU0) {
    // factored for the other orientation (or not yet): factor this one
    if (!J.ilu_ready || J.ilu_tr != tr) {
      if (int nb = ilu_setup(c, tr))
        throw ApiError{AEROF_ESINGULAR, std::to_string(nb) + " singular diagonal block(s) in the ILU(0) factors"};
    }
    ilu_apply(c, x, z, skip);
    return;
  }
  if (J.precision == AEROF_PREC_FP32)
    k_bj_apply<float, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, J.dinv32.p, x, z, tr, skip);
  else
    k_bj_apply<double, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, J.dinv64.p, x, z, tr, skip);
  AEROF_LAUNCH_CHECK();
}
void prec_apply_dev(aerof_gpu_ctx* c, const double* x, double* z, int trans) {
  prec_apply_t<double, double>(c, x, z, trans);
}

// Device-driven form of gmres_t for the assembled operator (block-Jacobi or
// block ILU(0)): per iteration the preconditioner, the product and
// k_gmres_iter, no host synchronisation inside a restart cycle;
// the host reads the cycle's status once at its end (AEROF_GMRES_DEVICE=0
// selects the host-driven loop).
static bool gmres_device_loop_enabled() {
  static const int v = [] {
    const char* e = std::getenv("AEROF_GMRES_DEVICE");
    return e ? std::atoi(e) : 1;
  }();
  return v != 0;
}

template <class TV>
static int gmres_devloop(aerof_gpu_ctx* c, const double* b, double* x, int numVec, int maxits, double eps, int trans,
                         double* final_res) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const size_t n = 5 * (size_t)m.N;
  const int gv = grid_for(n, kIB);
  cudaStream_t s = c->stream;
  const size_t ld = (n + 63) / 64 * 64;
  J.basis.ensure(((size_t)(numVec + 1) * ld * sizeof(TV) + 7) / 8);
  J.w.ensure((n * sizeof(TV) + 7) / 8);
  J.r.ensure((n * sizeof(TV) + 7) / 8);
  J.ticket.ensure(1);
  AEROF_CUDA(cudaMemsetAsync(J.ticket.p, 0, sizeof(unsigned), s));
  c->s.red.ensure(kGB);
  J.hcol.ensure(1);
  TV* Vb = reinterpret_cast<TV*>(J.basis.p);
  TV* w = reinterpret_cast<TV*>(J.w.p);
  TV* r = reinterpret_cast<TV*>(J.r.p);
  // cooperative grid: every CTA resident at once
  static int coop_grid = 0;
  if (!coop_grid) {
    int per_sm = 0, sms = 0;
    AEROF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gmres_iter<TV>, kCoopThreads, 0));
    AEROF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->cfg.device));
    coop_grid = std::max(1, std::min(per_sm, 4)) * sms;
  }
  const int grid = coop_grid;
  // device state: H, cs, g, y, scal | ist, part, bar
  const size_t nH = (size_t)(numVec + 1) * numVec;
  J.gst.ensure(nH + 2 * (size_t)numVec + (numVec + 1) + numVec + 2 + 2 * (size_t)grid);
  J.gsti.ensure(8 + 1);
  GmresState st;
  st.H = J.gst.p;
  st.cs = st.H + nH;
  st.g = st.cs + 2 * numVec;
  st.y = st.g + numVec + 1;
  st.scal = st.y + numVec;
  st.part = st.scal + 2;
  st.ist = J.gsti.p;
  st.bar = reinterpret_cast<unsigned*>(J.gsti.p + 8);
  double* part = c->s.red.p;
  unsigned* ticket = J.ticket.p;
  double* hd = J.hcol.p;
  auto norm2 = [&](TV* v) -> double {
    k_mgs<TV, true><<<kGB, kIB, 0, s>>>(n, nullptr, nullptr, nullptr, v, part, ticket, hd);
    AEROF_LAUNCH_CHECK();
    double h = 0.0;
    AEROF_CUDA(cudaMemcpyAsync(&h, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(h);
  };
  AEROF_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  int iter = 0;
  double target = 0.0, l2res = 0.0;
  const double bnorm = norm2_dev(c, b, n);
  std::vector<double> ginit(numVec + 1 + numVec + 2);
  for (;;) {
    if (iter == 0) {
      k_scale<double, TV><<<gv, kIB, 0, s>>>(n, 1.0, b, r);
      AEROF_LAUNCH_CHECK();
    } else {
      k_scale<double, TV><<<gv, kIB, 0, s>>>(n, 1.0, x, r);
      AEROF_LAUNCH_CHECK();
      matvec_t<TV, TV>(c, r, w, trans);
      k_sub<TV, TV><<<gv, kIB, 0, s>>>(n, b, w, r);
      AEROF_LAUNCH_CHECK();
    }
    const double beta = norm2(r);
    if (iter == 0) target = eps * bnorm;
    if (beta == 0.0) {
      if (final_res) *final_res = 0.0;
      return iter;
    }
    k_scale<TV, TV><<<gv, kIB, 0, s>>>(n, 1.0 / beta, r, Vb);
    AEROF_LAUNCH_CHECK();
    // this cycle's state: g = (beta, 0, ...), the estimate, the target,
    // the counters, zero barrier arrivals
    std::fill(ginit.begin(), ginit.end(), 0.0);
    ginit[0] = beta;
    ginit[2 * (size_t)numVec + 1] = l2res;
    ginit[2 * (size_t)numVec + 2] = target;
    AEROF_CUDA(cudaMemcpyAsync(st.g, ginit.data(), ginit.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    const int iinit[9] = {iter, 0, -1, 0, maxits, 0, 0, 0, 0};
    AEROF_CUDA(cudaMemcpyAsync(st.ist, iinit, sizeof(iinit), cudaMemcpyHostToDevice, s));
    unsigned base = 0;
    const int* done = st.ist + 1;
    // every four iterations the done flag is copied to pinned memory behind
    // an event; the host looks at the previous copy without waiting and
    // stops issuing the cycle once it shows convergence (the kernels issued
    // after convergence return at once anyway)
    if (!J.poll.done) {
      AEROF_CUDA(cudaMallocHost((void**)&J.poll.done, sizeof(int)));
      AEROF_CUDA(cudaEventCreateWithFlags(&J.poll.ev, cudaEventDisableTiming));
    }
    bool polled = false;
    for (int j = 0; j < numVec; ++j) {
      if (polled) {
        const cudaError_t q = cudaEventQuery(J.poll.ev);
        if (q == cudaSuccess) {
          polled = false;
          if (*J.poll.done) break;
        } else if (q != cudaErrorNotReady) {
          AEROF_CUDA(q);
        } else if (cudaPeekAtLastError() == cudaErrorNotReady) {
          cudaGetLastError();  // "not ready" is a state, not an error for the next launch check
        }
      }
      prec_apply_t<TV, TV>(c, Vb + (size_t)j * ld, r, trans, done);
      matvec_t<TV, TV>(c, r, w, trans, done);
      {
        TimerScope t(c, AEROF_T_KSP_OTHER);
        void* args[] = {(void*)&n, (void*)&j, (void*)&numVec, (void*)&Vb, (void*)&ld, (void*)&w, (void*)&st,
                        (void*)&base};
        AEROF_CUDA(cudaLaunchCooperativeKernel((const void*)k_gmres_iter<TV>, grid, kCoopThreads, args, 0, s));
        AEROF_LAUNCH_CHECK();
        base += (unsigned)(j + 2) * (unsigned)grid;
      }
      if ((j & 3) == 3 && !polled && j + 1 < numVec) {
        AEROF_CUDA(cudaMemcpyAsync(J.poll.done, done, sizeof(int), cudaMemcpyDeviceToHost, s));
        AEROF_CUDA(cudaEventRecord(J.poll.ev, s));
        polled = true;
      }
    }
    if (polled) AEROF_CUDA(cudaEventSynchronize(J.poll.ev));
    k_gmres_backsolve<<<1, 32, 0, s>>>(numVec, st);
    AEROF_LAUNCH_CHECK();
    k_combine_dev<TV><<<gv, kIB, 0, s>>>(n, st.ist + 2, st.y, Vb, ld, w);
    AEROF_LAUNCH_CHECK();
    prec_apply_t<TV, TV>(c, w, r, trans);
    k_add<TV><<<gv, kIB, 0, s>>>(n, r, x);
    AEROF_LAUNCH_CHECK();
    int ist[6];
    AEROF_CUDA(cudaMemcpyAsync(ist, st.ist, sizeof(ist), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaMemcpyAsync(&l2res, st.scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
    if (ist[3]) throw ApiError{AEROF_ETIMEDOUT, "GMRES grid barrier timed out"};
    iter = ist[0];
    if (ist[1]) break;  // converged, saturated or broke down
  }
  if (final_res) *final_res = l2res;
  return iter;
}

// GmresSolver::solve (KspSolver.C:351-492), typePrec = 2 (right
// preconditioning), MGS, Givens rotations and back substitution on the host
// (KspSolver.C:917-982).  x = 0 on entry.  Returns iterations.
// TV is the storage type of the Krylov vectors: double, or float for the
// mixed-precision solver (dots, norms and the Hessenberg system stay FP64;
// b and x stay FP64).  exactU != null selects the exact operator (TV =
// double only).
template <class TV>
static int gmres_t(aerof_gpu_ctx* c, const double* b, double* x, int numVec, int maxits, double eps, int trans,
                   double* final_res, const double* exactU) {
  if (!exactU && numVec <= kMaxKrylov && gmres_device_loop_enabled())
    return gmres_devloop<TV>(c, b, x, numVec, maxits, eps, trans, final_res);
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const size_t n = 5 * (size_t)m.N;
  const int gv = grid_for(n, kIB);
  cudaStream_t s = c->stream;
  const size_t ld = (n + 63) / 64 * 64;  // basis leading dimension: 256-byte aligned vectors
  const size_t vbytes = (size_t)(numVec + 1) * ld * sizeof(TV);
  J.basis.ensure((vbytes + 7) / 8);
  J.ticket.ensure(1);
  AEROF_CUDA(cudaMemsetAsync(J.ticket.p, 0, sizeof(unsigned), s));
  unsigned* ticket = J.ticket.p;
  J.w.ensure((n * sizeof(TV) + 7) / 8);
  J.r.ensure((n * sizeof(TV) + 7) / 8);
  J.hcol.ensure((size_t)numVec + 2 + (size_t)numVec + 1);
  c->s.red.ensure(kGB);
  TV* Vb = reinterpret_cast<TV*>(J.basis.p);
  TV* w = reinterpret_cast<TV*>(J.w.p);
  TV* r = reinterpret_cast<TV*>(J.r.p);
  double* hd = J.hcol.p;              // [numVec + 2] Hessenberg column
  double* yd = J.hcol.p + numVec + 2;  // [numVec + 1] solution coefficients
  double* part = c->s.red.p;
  auto op = [&](const TV* p, TV* y) {
    if (!exactU) { matvec_t<TV, TV>(c, p, y, trans); return; }
    TimerScope t(c, AEROF_T_KSP_MATVEC);
    exact_product(c, exactU, reinterpret_cast<const double*>(p), reinterpret_cast<double*>(y), trans);
  };
  auto norm2 = [&](TV* v) -> double {
    k_mgs<TV, true><<<kGB, kIB, 0, s>>>(n, nullptr, nullptr, nullptr, v, part, ticket, hd);
    AEROF_LAUNCH_CHECK();
    double h = 0.0;
    AEROF_CUDA(cudaMemcpyAsync(&h, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(h);
  };
  AEROF_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  std::vector<double> H((size_t)(numVec + 1) * numVec, 0.0), cs(2 * (size_t)numVec), g(numVec + 1), y(numVec),
      hcol(numVec + 2);
  auto h = [&](int i, int j) -> double& { return H[(size_t)i * numVec + j]; };
  auto dot_to = [&](const double* hp, const TV* vprev, const TV* vcur, double* out) {
    k_mgs<TV, false><<<kGB, kIB, 0, s>>>(n, hp, vprev, vcur, w, part, ticket, out);
    AEROF_LAUNCH_CHECK();
  };
  int iter = 0, exitLoop = 0;
  double target = 0.0, l2res = 0.0;
  const double bnorm = norm2_dev(c, b, n);
  do {
    // r = b - A x  (x == 0 on the first cycle)
    if (iter == 0) {
      k_scale<double, TV><<<gv, kIB, 0, s>>>(n, 1.0, b, r);
      AEROF_LAUNCH_CHECK();
    } else {
      k_scale<double, TV><<<gv, kIB, 0, s>>>(n, 1.0, x, r);
      AEROF_LAUNCH_CHECK();
      op(r, w);
      k_sub<TV, TV><<<gv, kIB, 0, s>>>(n, b, w, r);
      AEROF_LAUNCH_CHECK();
    }
    const double beta = norm2(r);
    if (iter == 0) target = eps * bnorm;
    if (beta == 0.0) { if (final_res) *final_res = 0.0; return iter; }
    k_scale<TV, TV><<<gv, kIB, 0, s>>>(n, 1.0 / beta, r, Vb);
    AEROF_LAUNCH_CHECK();
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j;
    for (j = 0; j < numVec; ++j) {
      {
        TimerScope t(c, AEROF_T_KSP_OTHER);
        prec_apply_t<TV, TV>(c, Vb + (size_t)j * ld, r, trans);
      }
      op(r, w);
      // h_ij = w . V_i ; w -= h_ij V_i   (i = 0..j), then ||w||
      TimerScope t(c, AEROF_T_KSP_OTHER);
      for (int i = 0; i <= j; ++i)
        dot_to(i ? hd + (i - 1) : nullptr, i ? Vb + (size_t)(i - 1) * ld : nullptr, Vb + (size_t)i * ld, hd + i);
      k_mgs<TV, true><<<kGB, kIB, 0, s>>>(n, hd + j, Vb + (size_t)j * ld, nullptr, w, part, ticket, hd + j + 1);
      AEROF_LAUNCH_CHECK();
      AEROF_CUDA(cudaMemcpyAsync(hcol.data(), hd, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, s));
      AEROF_CUDA(cudaStreamSynchronize(s));
      for (int i = 0; i <= j; ++i) h(i, j) = hcol[i];
      h(j + 1, j) = std::sqrt(hcol[j + 1]);
      const bool breakdown = (h(j + 1, j) == 0.0);
      if (!breakdown) {
        k_scale<TV, TV><<<gv, kIB, 0, s>>>(n, 1. / h(j + 1, j), w, Vb + (size_t)(j + 1) * ld);
        AEROF_LAUNCH_CHECK();
      }
      for (int i = 0; i < j; ++i) {
        double hj = cs[2 * i + 1] * h(i, j) + cs[2 * i] * h(i + 1, j);
        double hjp1 = -cs[2 * i] * h(i, j) + cs[2 * i + 1] * h(i + 1, j);
        h(i, j) = hj; h(i + 1, j) = hjp1;
      }
      if (h(j, j) * h(j, j) == 0.0) { cs[2 * j + 1] = 0.0; cs[2 * j] = 1.0; }
      else {
        double coef = 1.0 / std::sqrt(h(j, j) * h(j, j) + h(j + 1, j) * h(j + 1, j));
        cs[2 * j + 1] = std::sqrt(h(j, j) * h(j, j)) * coef;
        cs[2 * j] = cs[2 * j + 1] * h(j + 1, j) / h(j, j);
      }
      h(j, j) = cs[2 * j + 1] * h(j, j) + cs[2 * j] * h(j + 1, j);
      h(j + 1, j) = 0.0;
      g[j + 1] = -cs[2 * j] * g[j];
      g[j] = cs[2 * j + 1] * g[j];
      ++iter;
      if (breakdown) { exitLoop = 1; break; }
      l2res = std::fabs(g[j + 1]);
      if (l2res <= target || iter >= maxits) { exitLoop = 1; break; }
    }
    if (j == numVec) --j;
    for (int i = j; i >= 0; --i) {
      y[i] = g[i];
      for (int k = j; k >= i + 1; --k) y[i] -= h(i, k) * y[k];
      y[i] /= h(i, i);
    }
    AEROF_CUDA(cudaMemcpyAsync(yd, y.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice, s));
    k_combine<TV><<<gv, kIB, 0, s>>>(n, j + 1, yd, Vb, ld, w);
    AEROF_LAUNCH_CHECK();
    prec_apply_t<TV, TV>(c, w, r, trans);
    k_add<TV><<<gv, kIB, 0, s>>>(n, r, x);
    AEROF_LAUNCH_CHECK();
  } while (exitLoop == 0);
  AEROF_CUDA(cudaStreamSynchronize(s));
  if (final_res) *final_res = l2res;
  return iter;
}

// Flexible GMRES(m) on the exact linearisation at exactU (J or J^T by
// forward or reverse mode, FP64 vectors) whose preconditioner is itself a
// solve: z_j = (approximately) H1^{-1} v_j by inner_its iterations of the
// mixed-precision GMRES on the assembled first-order operator (FP32 blocks
// and Krylov vectors, block-Jacobi).  The corrections are kept (Z) and
// x = Z y, so the changing inner solve does not spoil the minimisation.
// x = 0 on entry.  Returns outer iterations.
static int fgmres_exact(aerof_gpu_ctx* c, const double* b, double* x, int numVec, int maxits, double eps, int trans,
                        double* final_res, const double* exactU, int inner_m, int inner_its, double inner_eps) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const size_t n = 5 * (size_t)m.N;
  const size_t ld = (n + 63) / 64 * 64;
  const int gv = grid_for(n, kIB);
  cudaStream_t s = c->stream;
  J.fV.ensure((size_t)(numVec + 1) * ld);
  J.fZ.ensure((size_t)numVec * ld);
  J.fw.ensure(ld);
  J.fr.ensure(ld);
  J.fh.ensure((size_t)numVec + 2 + (size_t)numVec + 1);
  J.ticket.ensure(1);
  c->s.red.ensure(kGB);
  double* V = J.fV.p;
  double* Z = J.fZ.p;
  double* w = J.fw.p;
  double* r = J.fr.p;
  double* hd = J.fh.p;
  double* yd = J.fh.p + numVec + 2;
  double* part = c->s.red.p;
  unsigned* ticket = J.ticket.p;
  AEROF_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  auto op = [&](const double* p, double* y) {
    TimerScope t(c, AEROF_T_KSP_MATVEC);
    exact_product(c, exactU, p, y, trans);
  };
  auto norm2 = [&](double* v) -> double {
    k_mgs<double, true><<<kGB, kIB, 0, s>>>(n, nullptr, nullptr, nullptr, v, part, ticket, hd);
    AEROF_LAUNCH_CHECK();
    double h = 0.0;
    AEROF_CUDA(cudaMemcpyAsync(&h, hd, sizeof(double), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
    return std::sqrt(h);
  };
  AEROF_CUDA(cudaMemsetAsync(x, 0, n * sizeof(double), s));
  std::vector<double> H((size_t)(numVec + 1) * numVec, 0.0), cs(2 * (size_t)numVec), g(numVec + 1), y(numVec),
      hcol(numVec + 2);
  auto h = [&](int i, int j) -> double& { return H[(size_t)i * numVec + j]; };
  int iter = 0, exitLoop = 0;
  double target = 0.0, l2res = 0.0;
  const double bnorm = norm2_dev(c, b, n);
  do {
    if (iter == 0) {
      AEROF_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else {
      op(x, w);
      k_sub<double, double><<<gv, kIB, 0, s>>>(n, b, w, r);
      AEROF_LAUNCH_CHECK();
    }
    const double beta = norm2(r);
    if (iter == 0) target = eps * bnorm;
    if (beta == 0.0) { if (final_res) *final_res = 0.0; return iter; }
    k_scale<double, double><<<gv, kIB, 0, s>>>(n, 1.0 / beta, r, V);
    AEROF_LAUNCH_CHECK();
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j;
    for (j = 0; j < numVec; ++j) {
      double* zj = Z + (size_t)j * ld;
      gmres_t<float>(c, V + (size_t)j * ld, zj, inner_m, inner_its, inner_eps, trans, nullptr, nullptr);
      op(zj, w);
      TimerScope t(c, AEROF_T_KSP_OTHER);
      for (int i = 0; i <= j; ++i) {
        k_mgs<double, false><<<kGB, kIB, 0, s>>>(n, i ? hd + (i - 1) : nullptr, i ? V + (size_t)(i - 1) * ld : nullptr,
                                                 V + (size_t)i * ld, w, part, ticket, hd + i);
        AEROF_LAUNCH_CHECK();
      }
      k_mgs<double, true><<<kGB, kIB, 0, s>>>(n, hd + j, V + (size_t)j * ld, nullptr, w, part, ticket, hd + j + 1);
      AEROF_LAUNCH_CHECK();
      AEROF_CUDA(cudaMemcpyAsync(hcol.data(), hd, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, s));
      AEROF_CUDA(cudaStreamSynchronize(s));
      for (int i = 0; i <= j; ++i) h(i, j) = hcol[i];
      h(j + 1, j) = std::sqrt(hcol[j + 1]);
      const bool breakdown = (h(j + 1, j) == 0.0);
      if (!breakdown) {
        k_scale<double, double><<<gv, kIB, 0, s>>>(n, 1. / h(j + 1, j), w, V + (size_t)(j + 1) * ld);
        AEROF_LAUNCH_CHECK();
      }
      for (int i = 0; i < j; ++i) {
        double hj = cs[2 * i + 1] * h(i, j) + cs[2 * i] * h(i + 1, j);
        double hjp1 = -cs[2 * i] * h(i, j) + cs[2 * i + 1] * h(i + 1, j);
        h(i, j) = hj; h(i + 1, j) = hjp1;
      }
      if (h(j, j) * h(j, j) == 0.0) { cs[2 * j + 1] = 0.0; cs[2 * j] = 1.0; }
      else {
        double coef = 1.0 / std::sqrt(h(j, j) * h(j, j) + h(j + 1, j) * h(j + 1, j));
        cs[2 * j + 1] = std::sqrt(h(j, j) * h(j, j)) * coef;
        cs[2 * j] = cs[2 * j + 1] * h(j + 1, j) / h(j, j);
      }
      h(j, j) = cs[2 * j + 1] * h(j, j) + cs[2 * j] * h(j + 1, j);
      h(j + 1, j) = 0.0;
      g[j + 1] = -cs[2 * j] * g[j];
      g[j] = cs[2 * j + 1] * g[j];
      ++iter;
      if (breakdown) { exitLoop = 1; break; }
      l2res = std::fabs(g[j + 1]);
      if (l2res <= target || iter >= maxits) { exitLoop = 1; break; }
    }
    if (j == numVec) --j;
    for (int i = j; i >= 0; --i) {
      y[i] = g[i];
      for (int k = j; k >= i + 1; --k) y[i] -= h(i, k) * y[k];
      y[i] /= h(i, i);
    }
    AEROF_CUDA(cudaMemcpyAsync(yd, y.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice, s));
    k_combine<double><<<gv, kIB, 0, s>>>(n, j + 1, yd, Z, ld, w);
    AEROF_LAUNCH_CHECK();
    k_add<double><<<gv, kIB, 0, s>>>(n, w, x);
    AEROF_LAUNCH_CHECK();
  } while (exitLoop == 0);
  AEROF_CUDA(cudaStreamSynchronize(s));
  if (final_res) *final_res = l2res;
  return iter;
}

// Lockstep GMRES over R right-hand sides (batched sensitivities): every
// system runs the algorithm of gmres_t (FLEX = false: FP32 Krylov vectors,
// right-preconditioned, products with H1 batched over the running systems)
// or of fgmres_exact (FLEX = true: FP64, the preconditioner one inner
// lockstep solve of all running systems, exact products), the iterations of
// all systems together; a system that converges stops, the others go on.
// B[q] / X[q] are the right-hand sides and solutions (device, [N][5]); X is
// zeroed first.  The inner solve (FLEX = false) runs one cycle: maxits <=
// numVec.
template <class TV, bool FLEX>
static void gmres_lockstep(aerof_gpu_ctx* c, int R, const double* const* B, double* const* X, int numVec, int maxits,
                           double eps, int trans, const double* exactU, int inner_m, int inner_its, double inner_eps,
                           int* its, double* res) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const size_t n = 5 * (size_t)m.N;
  const size_t ld = (n + 63) / 64 * 64;
  const int gv = grid_for(n, kIB);
  cudaStream_t s = c->stream;
  const int M1 = numVec + 1, HS = numVec + 2;
  TV *Vb, *Zb = nullptr, *w, *rr, *pz = nullptr;
  double* hd;
  if constexpr (FLEX) {
    J.bV.ensure((size_t)R * M1 * ld);
    J.bZ.ensure((size_t)R * numVec * ld);
    J.bw.ensure((size_t)R * ld);
    J.br.ensure((size_t)R * ld);
    J.bh.ensure((size_t)R * (HS + M1));
    Vb = J.bV.p; Zb = J.bZ.p; w = J.bw.p; rr = J.br.p; hd = J.bh.p;
  } else {
    J.iV.ensure((size_t)R * M1 * ld);
    J.iw.ensure((size_t)R * ld);
    J.ir.ensure((size_t)R * ld);
    J.iz.ensure((size_t)R * ld);
    J.ih.ensure((size_t)R * (HS + M1));
    J.bptr.ensure(2 * (size_t)R);
    Vb = J.iV.p; w = J.iw.p; rr = J.ir.p; pz = J.iz.p; hd = J.ih.p;
  }
  double* yd = hd + (size_t)R * HS;
  J.ticket.ensure(1);
  c->s.red.ensure(kGB);
  double* part = c->s.red.p;
  unsigned* ticket = J.ticket.p;
  AEROF_CUDA(cudaMemsetAsync(ticket, 0, sizeof(unsigned), s));
  auto V = [&](int q, int j) { return Vb + ((size_t)q * M1 + j) * ld; };
  auto Zv = [&](int q, int j) { return Zb + ((size_t)q * numVec + j) * ld; };
  auto W = [&](int q) { return w + (size_t)q * ld; };
  auto Rv = [&](int q) { return rr + (size_t)q * ld; };
  auto Hq = [&](int q) { return hd + (size_t)q * HS; };
  // host state per system
  std::vector<double> H((size_t)R * M1 * numVec, 0.0), cs((size_t)R * 2 * numVec), g((size_t)R * M1), y(numVec),
      hcol((size_t)R * HS), target(R, 0.0), l2(R, 0.0), bnorm(R);
  std::vector<int> iter(R, 0), jl(R, -1);
  std::vector<char> active(R, 1), run(R, 0), fin(R, 0);
  auto h = [&](int q, int i, int j) -> double& { return H[((size_t)q * M1 + i) * numVec + j]; };
  auto fetch = [&]() {
    AEROF_CUDA(cudaMemcpyAsync(hcol.data(), hd, sizeof(double) * (size_t)R * HS, cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
  };
  // the reductions read 16-byte vectors of the right-hand sides
  for (int q = 0; q < R; ++q)
    if (reinterpret_cast<uintptr_t>(B[q]) % 16 != 0)
      throw ApiError{AEROF_EINVAL, "lockstep GMRES: right-hand side not 16-byte aligned"};
  for (int q = 0; q < R; ++q) {
    AEROF_CUDA(cudaMemsetAsync(X[q], 0, n * sizeof(double), s));
    k_mgs<double, true><<<kGB, kIB, 0, s>>>(n, nullptr, nullptr, nullptr, const_cast<double*>(B[q]), part, ticket,
                                            Hq(q));
    AEROF_LAUNCH_CHECK();
  }
  fetch();
  for (int q = 0; q < R; ++q) bnorm[q] = std::sqrt(hcol[(size_t)q * HS]);
  std::vector<unsigned long long> ptrs(2 * (size_t)R);
  while (true) {
    // residuals of the active systems
    for (int q = 0; q < R; ++q) {
      if (!active[q]) continue;
      if (iter[q] == 0) {
        k_scale<double, TV><<<gv, kIB, 0, s>>>(n, 1.0, B[q], Rv(q));
        AEROF_LAUNCH_CHECK();
      } else {
        TimerScope t(c, AEROF_T_KSP_MATVEC);
        if constexpr (FLEX) {
          exact_product(c, exactU, X[q], W(q), trans);
        } else {
          k_scale<double, TV><<<gv, kIB, 0, s>>>(n, 1.0, X[q], Rv(q));
          AEROF_LAUNCH_CHECK();
          matvec_t<TV, TV>(c, Rv(q), W(q), trans);
        }
        k_sub<TV, TV><<<gv, kIB, 0, s>>>(n, B[q], W(q), Rv(q));
        AEROF_LAUNCH_CHECK();
      }
      k_mgs<TV, true><<<kGB, kIB, 0, s>>>(n, nullptr, nullptr, nullptr, Rv(q), part, ticket, Hq(q));
      AEROF_LAUNCH_CHECK();
    }
    fetch();
    bool any = false;
    for (int q = 0; q < R; ++q) {
      run[q] = 0;
      jl[q] = -1;
      if (!active[q]) continue;
      const double beta = std::sqrt(hcol[(size_t)q * HS]);
      if (iter[q] == 0) target[q] = eps * bnorm[q];
      if (beta == 0.0) {
        active[q] = 0;
        l2[q] = 0.0;
        continue;
      }
      k_scale<TV, TV><<<gv, kIB, 0, s>>>(n, 1.0 / beta, Rv(q), V(q, 0));
      AEROF_LAUNCH_CHECK();
      std::fill(g.begin() + (size_t)q * M1, g.begin() + (size_t)(q + 1) * M1, 0.0);
      g[(size_t)q * M1] = beta;
      run[q] = 1;
      fin[q] = 0;
      any = true;
    }
    if (!any) break;
    for (int j = 0; j < numVec; ++j) {
      std::vector<int> rl;
      for (int q = 0; q < R; ++q)
        if (run[q]) rl.push_back(q);
      if (rl.empty()) break;
      const int nr = (int)rl.size();
      // direction and product of every running system
      if constexpr (FLEX) {
        std::vector<const double*> bi(nr);
        std::vector<double*> xi(nr);
        for (int k = 0; k < nr; ++k) { bi[k] = V(rl[k], j); xi[k] = Zv(rl[k], j); }
        gmres_lockstep<float, false>(c, nr, bi.data(), xi.data(), inner_m, inner_its, inner_eps, trans, nullptr, 0, 0,
                                     0.0, nullptr, nullptr);
        TimerScope t(c, AEROF_T_KSP_MATVEC);
        for (int k = 0; k < nr; ++k) exact_product(c, exactU, Zv(rl[k], j), W(rl[k]), trans);
      } else {
        {
          TimerScope t(c, AEROF_T_KSP_OTHER);
          const int tr = ((trans != 0) != J.transposed) ? 1 : 0;
          if (J.pc == AEROF_PC_ILU0 && J.ilu_ready && J.ilu_tr == tr) {
            // every factor block read once for the running systems
            std::vector<const TV*> xs(nr);
            std::vector<TV*> zs(nr);
            for (int k = 0; k < nr; ++k) { xs[k] = V(rl[k], j); zs[k] = pz + (size_t)rl[k] * ld; }
            ilu_apply_batch<TV, TV>(c, nr, xs.data(), zs.data());
          } else {
            for (int k = 0; k < nr; ++k) prec_apply_t<TV, TV>(c, V(rl[k], j), pz + (size_t)rl[k] * ld, trans);
          }
        }
        TimerScope t(c, AEROF_T_KSP_MATVEC);
        for (int k = 0; k < nr; ++k) {
          ptrs[k] = (unsigned long long)(pz + (size_t)rl[k] * ld);
          ptrs[R + k] = (unsigned long long)W(rl[k]);
        }
        AEROF_CUDA(cudaMemcpyAsync(J.bptr.p, ptrs.data(), sizeof(unsigned long long) * 2 * (size_t)R,
                                   cudaMemcpyHostToDevice, s));
        const TV* const* P = reinterpret_cast<const TV* const*>(J.bptr.p);
        TV* const* Y = reinterpret_cast<TV* const*>(J.bptr.p + R);
        const bool tr = (trans != 0) != J.transposed;
        auto go = [&](auto kern, auto* diag, auto* off) {
          kern<<<grid_for(m.N, kIB), kIB, 0, s>>>(m.N, nr, m.nbr_ptr.p, m.nbr_tpos.p, m.sptr.p, m.scol.p, diag, off,
                                                 P, Y);
          AEROF_LAUNCH_CHECK();
        };
        if (J.precision == AEROF_PREC_FP32) {
          if (tr) go(k_spmv_batch<float, true, TV, 4>, J.diag32.p, J.off32.p);
          else go(k_spmv_batch<float, false, TV, 4>, J.diag32.p, J.off32.p);
        } else {
          if (tr) go(k_spmv_batch<double, true, TV, 4>, J.diag64.p, J.off64.p);
          else go(k_spmv_batch<double, false, TV, 4>, J.diag64.p, J.off64.p);
        }
      }
      TimerScope t(c, AEROF_T_KSP_OTHER);
      for (int q : rl) {
        for (int i = 0; i <= j; ++i) {
          k_mgs<TV, false><<<kGB, kIB, 0, s>>>(n, i ? Hq(q) + (i - 1) : nullptr, i ? V(q, i - 1) : nullptr, V(q, i),
                                               W(q), part, ticket, Hq(q) + i);
          AEROF_LAUNCH_CHECK();
        }
        k_mgs<TV, true><<<kGB, kIB, 0, s>>>(n, Hq(q) + j, V(q, j), nullptr, W(q), part, ticket, Hq(q) + j + 1);
        AEROF_LAUNCH_CHECK();
      }
      fetch();
      for (int q : rl) {
        const double* hc = hcol.data() + (size_t)q * HS;
        double* csq = cs.data() + (size_t)q * 2 * numVec;
        double* gq = g.data() + (size_t)q * M1;
        for (int i = 0; i <= j; ++i) h(q, i, j) = hc[i];
        h(q, j + 1, j) = std::sqrt(hc[j + 1]);
        const bool breakdown = (h(q, j + 1, j) == 0.0);
        if (!breakdown) {
          k_scale<TV, TV><<<gv, kIB, 0, s>>>(n, 1. / h(q, j + 1, j), W(q), V(q, j + 1));
          AEROF_LAUNCH_CHECK();
        }
        for (int i = 0; i < j; ++i) {
          double hj = csq[2 * i + 1] * h(q, i, j) + csq[2 * i] * h(q, i + 1, j);
          double hjp1 = -csq[2 * i] * h(q, i, j) + csq[2 * i + 1] * h(q, i + 1, j);
          h(q, i, j) = hj; h(q, i + 1, j) = hjp1;
        }
        if (h(q, j, j) * h(q, j, j) == 0.0) { csq[2 * j + 1] = 0.0; csq[2 * j] = 1.0; }
        else {
          double coef = 1.0 / std::sqrt(h(q, j, j) * h(q, j, j) + h(q, j + 1, j) * h(q, j + 1, j));
          csq[2 * j + 1] = std::sqrt(h(q, j, j) * h(q, j, j)) * coef;
          csq[2 * j] = csq[2 * j + 1] * h(q, j + 1, j) / h(q, j, j);
        }
        h(q, j, j) = csq[2 * j + 1] * h(q, j, j) + csq[2 * j] * h(q, j + 1, j);
        h(q, j + 1, j) = 0.0;
        gq[j + 1] = -csq[2 * j] * gq[j];
        gq[j] = csq[2 * j + 1] * gq[j];
        ++iter[q];
        jl[q] = j;
        if (breakdown) { run[q] = 0; fin[q] = 1; continue; }
        l2[q] = std::fabs(gq[j + 1]);
        if (l2[q] <= target[q] || iter[q] >= maxits) { run[q] = 0; fin[q] = 1; }
      }
    }
    // solution update of every system that ran in this cycle
    for (int q = 0; q < R; ++q) {
      if (jl[q] < 0) continue;
      const int jj = jl[q];
      const double* gq = g.data() + (size_t)q * M1;
      for (int i = jj; i >= 0; --i) {
        y[i] = gq[i];
        for (int k = jj; k >= i + 1; --k) y[i] -= h(q, i, k) * y[k];
        y[i] /= h(q, i, i);
      }
      double* yq = yd + (size_t)q * M1;
      AEROF_CUDA(cudaMemcpyAsync(yq, y.data(), sizeof(double) * (jj + 1), cudaMemcpyHostToDevice, s));
      if constexpr (FLEX) {
        k_combine<double><<<gv, kIB, 0, s>>>(n, jj + 1, yq, Zv(q, 0), ld, W(q));
        AEROF_LAUNCH_CHECK();
        k_add<double><<<gv, kIB, 0, s>>>(n, W(q), X[q]);
        AEROF_LAUNCH_CHECK();
      } else {
        k_combine<TV><<<gv, kIB, 0, s>>>(n, jj + 1, yq, V(q, 0), ld, W(q));
        AEROF_LAUNCH_CHECK();
        prec_apply_t<TV, TV>(c, W(q), Rv(q), trans);
        k_add<TV><<<gv, kIB, 0, s>>>(n, Rv(q), X[q]);
        AEROF_LAUNCH_CHECK();
      }
      if (fin[q]) active[q] = 0;
    }
    bool left = false;
    for (int q = 0; q < R; ++q) left = left || active[q];
    if (!left) break;
  }
  AEROF_CUDA(cudaStreamSynchronize(s));
  for (int q = 0; q < R; ++q) {
    if (its) its[q] = iter[q];
    if (res) res[q] = l2[q];
  }
}

int gmres_dev(aerof_gpu_ctx* c, const double* b, double* x, int numVec, int maxits, double eps, int trans,
              double* final_res, const double* exactU) {
  if (!exactU && c->imp.precision == AEROF_PREC_FP32)
    return gmres_t<float>(c, b, x, numVec, maxits, eps, trans, final_res, nullptr);
  return gmres_t<double>(c, b, x, numVec, maxits, eps, trans, final_res, exactU);
}

}  // namespace aerof

// ====================================================================== C ABI
using namespace aerof;

extern "C" int aerof_gpu_jacobian(aerof_gpu_ctx* c, const double* U, const double* dt, int precision) {
  return guard(c, [&]() -> int {
    need_mesh_or_throw(c);
    if (!U || (precision != AEROF_PREC_FP32 && precision != AEROF_PREC_FP64)) return AEROF_EINVAL;
    const size_t N = c->mesh.N;
    const double* dU = in_dev(c, U, 5 * N, c->s.Ustage);
    const double* ddt = dt ? in_dev(c, dt, N, c->s.Vstage) : nullptr;
    jacobian_dev(c, dU, ddt, precision, false);
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_get_jacobian(aerof_gpu_ctx* c, double* A) {
  return guard(c, [&]() -> int {
    need_jac(c);
    if (!A) return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    Implicit& J = c->imp;
    const size_t nd = sl_diag_size(m), no = sl_off_size(m);
    std::vector<double> diag(nd), off(no);
    if (J.precision == AEROF_PREC_FP32) {
      std::vector<float> d32(nd), o32(no);
      AEROF_CUDA(cudaMemcpyAsync(d32.data(), J.diag32.p, nd * 4, cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaMemcpyAsync(o32.data(), J.off32.p, no * 4, cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaStreamSynchronize(c->stream));
      std::copy(d32.begin(), d32.end(), diag.begin());
      std::copy(o32.begin(), o32.end(), off.begin());
    } else {
      AEROF_CUDA(cudaMemcpyAsync(diag.data(), J.diag64.p, nd * 8, cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaMemcpyAsync(off.data(), J.off64.p, no * 8, cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaStreamSynchronize(c->stream));
    }
    // MvpMat layout: a[N] diagonal blocks, then per edge l the blocks
    // (i, j) and (j, i); the sliced storage is read back (transposed when
    // it holds H1^T)
    const std::vector<int>& sp = m.h_sptr;
    const std::vector<int>& np = m.h_nbr_ptr;
    const bool T = J.transposed;
    auto el = [&](int e) { return T ? 5 * (e % 5) + e / 5 : e; };
    const bool f32 = J.precision == AEROF_PREC_FP32;
    auto elo = [&](int e, int l) { return f32 ? sl_el<float>(e, l) : sl_el<double>(e, l); };
    for (int r = 0; r < m.N; ++r)
      for (int e = 0; e < 25; ++e) A[25 * (size_t)r + e] = diag[(size_t)(r >> 5) * 800 + elo(el(e), r & 31)];
    auto block = [&](int r, int p, double* dst) {
      // block at CSR position p of row r of H1; with H1^T stored it is the
      // transpose of the mirrored block
      for (int e = 0; e < 25; ++e) dst[e] = off[((size_t)sp[r >> 5] + (p - np[r])) * 800 + elo(e, r & 31)];
    };
    std::vector<int2> epos(m.E);
    AEROF_CUDA(cudaMemcpyAsync(epos.data(), m.edge_pos.p, sizeof(int2) * m.E, cudaMemcpyDeviceToHost, c->stream));
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    const size_t nA = 25 * (size_t)m.N;
    double tmp[25];
    for (int l = 0; l < m.E; ++l) {
      const int i = m.h_edges[2 * (size_t)l], j = m.h_edges[2 * (size_t)l + 1];
      double* aij = A + nA + 50 * (size_t)l;
      double* aji = aij + 25;
      if (!T) {
        block(i, epos[l].x, aij);
        block(j, epos[l].y, aji);
      } else {
        // stored row i, position of j holds A_ji^T; row j, position of i holds A_ij^T
        block(i, epos[l].x, tmp);
        for (int e = 0; e < 25; ++e) aji[e] = tmp[el(e)];
        block(j, epos[l].y, tmp);
        for (int e = 0; e < 25; ++e) aij[e] = tmp[el(e)];
      }
    }
    return AEROF_OK;
  });
}

// ---------------------------------------------------------------------
// MatVecProdFD::apply (MatVecProd.C:262-372): finite-difference products
// of the residual (plus the backward-Euler time term when dt is given)
// with the reference's step computeEpsilon (MatVecProd.C:879-929).

// per block: sum of (1e-6 |U| + 1e-6) and of p^2 over a grid-stride
// range, block tree in a fixed order (the partials are added on the host in
// block order)
__global__ void k_fd_eps_partial(size_t n, const double* __restrict__ U, const double* __restrict__ p,
                                 double* __restrict__ part) {
  __shared__ double su[kIB], sp[kIB];
  double a = 0.0, b = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    a += 1.e-6 * fabs(U[q]) + 1.e-6;
    b += p[q] * p[q];
  }
  su[threadIdx.x] = a;
  sp[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      su[threadIdx.x] += su[threadIdx.x + w];
      sp[threadIdx.x] += sp[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[blockIdx.x] = su[0];
    part[gridDim.x + blockIdx.x] = sp[0];
  }
}
// Q = U + a p
__global__ void k_fd_shift(size_t n, double a, const double* __restrict__ U, const double* __restrict__ p,
                           double* __restrict__ Q) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) Q[q] = U[q] + a * p[q];
}
// F += (Q - U) / dt (the time term of add_dAW_dt with Un = U)
__global__ void k_fd_time(size_t n, const double* __restrict__ Q, const double* __restrict__ U,
                          const double* __restrict__ dt, double* __restrict__ F) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) F[q] += (Q[q] - U[q]) / dt[q / 5];
}
// y = s (Fp - Fm)
__global__ void k_fd_diff(size_t n, double s, const double* __restrict__ Fp, const double* __restrict__ Fm,
                          double* __restrict__ y) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) y[q] = s * (Fp[q] - Fm[q]);
}

// y = finite-difference product at device state dU; dF (R(dU), may be null),
// ddt (may be null).  Returns eps.
double matvec_fd_dev(aerof_gpu_ctx* c, const double* dU, const double* dF, const double* dp, const double* ddt,
                     int fd_order, double* dy) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  cudaStream_t s = c->stream;
  const size_t n = 5 * (size_t)m.N;
  const int gv = grid_for(n, kIB);
  constexpr int kFdBlocks = 296;  // 2 x 148 SMs
  J.fdRed.ensure(2 * kFdBlocks);
  k_fd_eps_partial<<<kFdBlocks, kIB, 0, s>>>(n, dU, dp, J.fdRed.p);
  AEROF_LAUNCH_CHECK();
  std::vector<double> part(2 * kFdBlocks);
  AEROF_CUDA(cudaMemcpyAsync(part.data(), J.fdRed.p, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, s));
  AEROF_CUDA(cudaStreamSynchronize(s));
  double su = 0.0, sp = 0.0;
  for (int b = 0; b < kFdBlocks; ++b) {
    su += part[b];
    sp += part[kFdBlocks + b];
  }
  const double norm = std::sqrt(sp);
  const double eps = norm < 1.0e-14 ? 1.e-6 : su / ((double)n * norm);
  J.fdQ.ensure(n);
  J.fdFp.ensure(n);
  J.fdFm.ensure(n);
  k_fd_shift<<<gv, kIB, 0, s>>>(n, eps, dU, dp, J.fdQ.p);
  AEROF_LAUNCH_CHECK();
  residual_dev(c, J.fdQ.p, J.fdFp.p, true);
  if (ddt) {
    k_fd_time<<<gv, kIB, 0, s>>>(n, J.fdQ.p, dU, ddt, J.fdFp.p);
    AEROF_LAUNCH_CHECK();
  }
  if (fd_order == 2) {
    k_fd_shift<<<gv, kIB, 0, s>>>(n, -eps, dU, dp, J.fdQ.p);
    AEROF_LAUNCH_CHECK();
    residual_dev(c, J.fdQ.p, J.fdFm.p, true);
    if (ddt) {
      k_fd_time<<<gv, kIB, 0, s>>>(n, J.fdQ.p, dU, ddt, J.fdFm.p);
      AEROF_LAUNCH_CHECK();
    }
    k_fd_diff<<<gv, kIB, 0, s>>>(n, 0.5 / eps, J.fdFp.p, J.fdFm.p, dy);
  } else {
    const double* Fm = dF;
    if (!Fm) {
      residual_dev(c, dU, J.fdFm.p, true);
      Fm = J.fdFm.p;
    }
    k_fd_diff<<<gv, kIB, 0, s>>>(n, 1.0 / eps, J.fdFp.p, Fm, dy);
  }
  AEROF_LAUNCH_CHECK();
  return eps;
}

// The reverse of aerof_gpu_get_jacobian: H1 given in the MvpMat layout
// a[N+2E][25] (reference numbering) is stored in the sliced layout in the
// requested precision, as if aerof_gpu_jacobian had assembled it.
extern "C" int aerof_gpu_set_jacobian(aerof_gpu_ctx* c, const double* A, int precision) {
  return guard(c, [&]() -> int {
    need_mesh_or_throw(c);
    if (!A || (precision != AEROF_PREC_FP32 && precision != AEROF_PREC_FP64)) return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    Implicit& J = c->imp;
    const size_t nd = sl_diag_size(m), no = sl_off_size(m);
    const size_t nA = 25 * (size_t)m.N + 50 * (size_t)m.E;
    std::vector<double> hA;
    if (is_device_ptr(A)) {
      hA.resize(nA);
      AEROF_CUDA(cudaMemcpyAsync(hA.data(), A, nA * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaStreamSynchronize(c->stream));
      A = hA.data();
    }
    std::vector<double> diag(nd, 0.0), off(no, 0.0);
    const bool f32 = precision == AEROF_PREC_FP32;
    auto elo = [&](int e, int l) { return f32 ? sl_el<float>(e, l) : sl_el<double>(e, l); };
    for (int r = 0; r < m.N; ++r)
      for (int e = 0; e < 25; ++e) diag[(size_t)(r >> 5) * 800 + elo(e, r & 31)] = A[25 * (size_t)r + e];
    const std::vector<int>& sp = m.h_sptr;
    const std::vector<int>& np = m.h_nbr_ptr;
    std::vector<int2> epos(m.E);
    AEROF_CUDA(cudaMemcpyAsync(epos.data(), m.edge_pos.p, sizeof(int2) * m.E, cudaMemcpyDeviceToHost, c->stream));
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    auto put = [&](int r, int p, const double* src) {
      for (int e = 0; e < 25; ++e) off[((size_t)sp[r >> 5] + (p - np[r])) * 800 + elo(e, r & 31)] = src[e];
    };
    const double* edge_blocks = A + 25 * (size_t)m.N;
    for (int l = 0; l < m.E; ++l) {
      const int i = m.h_edges[2 * (size_t)l], j = m.h_edges[2 * (size_t)l + 1];
      put(i, epos[l].x, edge_blocks + 50 * (size_t)l);
      put(j, epos[l].y, edge_blocks + 50 * (size_t)l + 25);
    }
    if (f32) {
      J.diag64.release(); J.off64.release(); J.dinv64.release();
      std::vector<float> d32(diag.begin(), diag.end()), o32(off.begin(), off.end());
      J.diag32.upload(d32.data(), nd, c->stream);
      J.off32.upload(o32.data(), no, c->stream);
      AEROF_CUDA(cudaStreamSynchronize(c->stream));
    } else {
      J.diag32.release(); J.off32.release(); J.dinv32.release();
      J.diag64.upload(diag.data(), nd, c->stream);
      J.off64.upload(off.data(), no, c->stream);
      AEROF_CUDA(cudaStreamSynchronize(c->stream));
    }
    J.precision = precision;
    J.transposed = false;
    J.prec_ready = false;
    J.ilu_ready = false;
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_set_owned_rows(aerof_gpu_ctx* c, int n_owned) {
  return guard(c, [&]() -> int {
    need_mesh_or_throw(c);
    if (n_owned < 0 || n_owned > c->mesh.N) return AEROF_EINVAL;
    c->n_owned = n_owned;
    c->imp.prec_ready = false;
    c->imp.ilu_ready = false;
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_matvec_fd(aerof_gpu_ctx* c, const double* U, const double* F, const double* p,
                                   const double* dt, int fd_order, double* y, double* eps) {
  return guard(c, [&]() -> int {
    need_mesh_or_throw(c);
    if (!U || !p || !y || (fd_order != 1 && fd_order != 2)) return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    Implicit& J = c->imp;
    const size_t n = 5 * (size_t)m.N;
    // inputs staged side by side: U, p, F, dt
    J.fdIn.ensure(3 * n + (size_t)m.N);
    auto stage = [&](const double* a, size_t cnt, size_t off) -> const double* {
      if (!a) return nullptr;
      if (is_device_ptr(a)) return a;
      AEROF_CUDA(cudaMemcpyAsync(J.fdIn.p + off, a, cnt * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      return J.fdIn.p + off;
    };
    const double* dU = stage(U, n, 0);
    const double* dp = stage(p, n, n);
    const double* dF = stage(F, n, 2 * n);
    const double* ddt = stage(dt, m.N, 3 * n);
    double* dy = out_dev(c, y, n, c->s.Rstage);
    const double e = matvec_fd_dev(c, dU, dF, dp, ddt, fd_order, dy);
    out_finish(c, y, dy, n);
    if (eps) *eps = e;
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_matvec(aerof_gpu_ctx* c, const double* p, double* y, int transpose) {
  return guard(c, [&]() -> int {
    need_jac(c);
    if (!p || !y) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    const double* dp = in_dev(c, p, n, c->s.Ustage);
    double* dy = out_dev(c, y, n, c->s.Rstage);
    matvec_dev(c, dp, dy, transpose);
    out_finish(c, y, dy, n);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_prec_setup(aerof_gpu_ctx* c) {
  return guard(c, [&]() -> int {
    need_jac(c);
    int bad = prec_setup_dev(c);
    if (bad) {
      c->last_error = std::to_string(bad) + " diagonal block(s) with a zero pivot";
      return AEROF_ESINGULAR;
    }
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_prec_apply(aerof_gpu_ctx* c, const double* x, double* y, int transpose) {
  return guard(c, [&]() -> int {
    need_jac(c);
    if (!c->imp.prec_ready) throw ApiError{AEROF_ESTATE, "preconditioner not set up"};
    if (!x || !y) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    const double* dx = in_dev(c, x, n, c->s.Ustage);
    double* dy = out_dev(c, y, n, c->s.Rstage);
    prec_apply_dev(c, dx, dy, transpose);
    out_finish(c, y, dy, n);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_gmres(aerof_gpu_ctx* c, const double* b, double* x, int krylov, int maxits, double eps,
                               int transpose, int* its, double* res) {
  return guard(c, [&]() -> int {
    need_jac(c);
    if (!c->imp.prec_ready) throw ApiError{AEROF_ESTATE, "preconditioner not set up"};
    if (!b || !x || krylov < 1 || maxits < 1 || !(eps >= 0.0)) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    const double* db = in_dev(c, b, n, c->s.Ustage);
    double* dx = out_dev(c, x, n, c->s.Rstage);
    double r = 0.0;
    int it = gmres_dev(c, db, dx, krylov, maxits, eps, transpose, &r, nullptr);
    out_finish(c, x, dx, n);
    if (its) *its = it;
    if (res) *res = r;
    return AEROF_OK;
  });
}

// Steady pseudo-transient Newton: one Newton step per pseudo-time step
// (NewtonSolver.h:106-190 with maxIts = 1): F = R(Q); CFL from the RESIDUAL
// law (TsParameters.C:211-217, 290); local dt; H1 Jacobian + I/dt; block-
// Jacobi; GMRES on -F; Q += dQ.
extern "C" int aerof_gpu_newton(aerof_gpu_ctx* c, double* U, const aerof_newton_params* p,
                                aerof_newton_result* out, double* history) {
  return guard(c, [&]() -> int {
    need_mesh_or_throw(c);
    if (!U || !p || p->max_steps < 0 || p->ksp_krylov < 1 || p->ksp_maxits < 1 ||
        (p->precision != AEROF_PREC_FP32 && p->precision != AEROF_PREC_FP64) || !(p->cfl0 > 0.0))
      return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    const size_t n = 5 * (size_t)m.N;
    cudaStream_t s = c->stream;
    double* dU;
    if (is_device_ptr(U)) dU = U;
    else {
      c->s.Ustage.ensure(n);
      AEROF_CUDA(cudaMemcpyAsync(c->s.Ustage.p, U, n * sizeof(double), cudaMemcpyHostToDevice, s));
      dU = c->s.Ustage.p;
    }
    c->imp.b.ensure(n); c->imp.x.ensure(n); c->s.dt.ensure(m.N); c->s.k1.ensure(n); c->s.U0.ensure(n);
    c->s.counters.ensure(8);
    double* R = c->s.k1.p;
    double* rhs = c->imp.b.p;
    double* dQ = c->imp.x.p;
    double* dt = c->s.dt.p;
    double* Uprev = c->s.U0.p;
    int* nbad_d = c->s.counters.p + 5;
    const int gv = grid_for(n, kIB);
    cudaEvent_t e0, e1;
    AEROF_CUDA(cudaEventCreate(&e0));
    AEROF_CUDA(cudaEventCreate(&e1));
    AEROF_CUDA(cudaEventRecord(e0, s));
    double res0 = 0.0, rel = 1.0, rel_prev = 1.0, cfl = p->cfl0;
    int k = 0, lits = 0, bad = 0, redos = 0;
    bool redo = false;
    while (k <= p->max_steps) {
      if (!redo) {
        bad += residual_dev(c, dU, R);
        double res = norm2_dev(c, R, n);
        // a NaN initial residual would make res0 > 0 false and look converged
        if (!std::isfinite(res)) throw ApiError{AEROF_EINVAL, "non-finite residual in Newton step " + std::to_string(k)};
        if (k == 0) res0 = res;
        rel = res0 > 0.0 ? res / res0 : 0.0;
        if (history) history[k] = rel;
        if (rel <= p->tol || k == p->max_steps) break;
        if (k > 0) cfl = std::min(std::max(cfl * std::pow(rel_prev / rel, p->ser), p->cfl_min), p->cfl_max);
        rel_prev = rel;
      }
      redo = false;
      timestep_dev(c, dU, cfl, dt);
      jacobian_dev(c, dU, dt, p->precision, false);
      if (int nb = prec_setup_dev(c)) {
        c->last_error = std::to_string(nb) + " singular diagonal block(s) at Newton step " + std::to_string(k);
        return AEROF_ESINGULAR;
      }
      k_scale<double, double><<<gv, kIB, 0, s>>>(n, -1.0, R, rhs);
      AEROF_LAUNCH_CHECK();
      lits += gmres_dev(c, rhs, dQ, p->ksp_krylov, p->ksp_maxits, p->ksp_eps, 0, nullptr, nullptr);
      // rhs = Q; Q += dQ, then the physical-solution check
      // (NewtonSolver.h:187-215): on a non-positive density or pressure the
      // state is restored and the step redone with half the CFL number
      // (TsParameters::computeCflNumber, TsParameters.C:187-195), which
      // gives up below cfl0/1000
      AEROF_CUDA(cudaMemcpyAsync(Uprev, dU, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      k_add<double><<<gv, kIB, 0, s>>>(n, dQ, dU);
      AEROF_LAUNCH_CHECK();
      AEROF_CUDA(cudaMemsetAsync(nbad_d, 0, sizeof(int), s));
      k_check_solution<<<grid_for(m.N, kIB), kIB, 0, s>>>(m.N, make_gas(c->cfg.gamma), dU, nbad_d);
      AEROF_LAUNCH_CHECK();
      int nbad = 0;
      AEROF_CUDA(cudaMemcpyAsync(&nbad, nbad_d, sizeof(int), cudaMemcpyDeviceToHost, s));
      AEROF_CUDA(cudaStreamSynchronize(s));
      if (nbad) {
        AEROF_CUDA(cudaMemcpyAsync(dU, Uprev, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ++redos;
        cfl *= 0.5;
        if (cfl < p->cfl0 / 1000.0) {
          AEROF_CUDA(cudaStreamSynchronize(s));
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
          if (dU != U) AEROF_CUDA(cudaMemcpy(U, dU, n * sizeof(double), cudaMemcpyDeviceToHost));
          if (out) {
            out->steps = k;
            out->linear_its = lits;
            out->rel_residual = rel;
            out->seconds = 0.0;
            out->redos = redos;
          }
          c->last_error = "Newton update non-physical at " + std::to_string(nbad) + " node value(s) in step " +
                          std::to_string(k) + "; the CFL number fell below cfl0/1000";
          return AEROF_EDIVERGED;
        }
        redo = true;
        continue;
      }
      ++k;
    }
    AEROF_CUDA(cudaEventRecord(e1, s));
    AEROF_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    AEROF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (dU != U) AEROF_CUDA(cudaMemcpyAsync(U, dU, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    AEROF_CUDA(cudaStreamSynchronize(s));
    if (out) {
      out->steps = k;
      out->linear_its = lits;
      out->rel_residual = rel;
      out->seconds = ms * 1e-3;
      out->redos = redos;
    }
    return bad;
  });
}

// Linearised steady systems with the exact operator (sensitivity analysis,
// FluidShapeOptimizationHandler.C:1557-1624): transpose = 0 solves
// J x = b (direct), transpose = 1 solves J^T x = b (adjoint, GmresSolver::
// solveT, KspSolver.C:752-915).  Preconditioner: block-Jacobi of the
// first-order H1 operator at U without time term, in FP64.
extern "C" int aerof_gpu_linearized_solve(aerof_gpu_ctx* c, const double* U, const double* b, double* x, int krylov,
                                          int maxits, double eps, int transpose, int inner_its, int* its,
                                          double* res) {
  return guard(c, [&]() -> int {
    need_inviscid(c);
    need_mesh_or_throw(c);
    if (!U || !b || !x || krylov < 1 || maxits < 1 || !(eps >= 0.0) || inner_its < 0) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    c->imp.t.ensure(n);
    const double* dU0 = in_dev(c, U, n, c->s.Ustage);
    if (dU0 != c->imp.t.p)
      AEROF_CUDA(cudaMemcpyAsync(c->imp.t.p, dU0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    const double* dU = c->imp.t.p;
    const double* db = in_dev(c, b, n, c->s.Vstage);
    double* dx = out_dev(c, x, n, c->s.Rstage);
    // with the stored operator selected, the exact linearisation at U is
    // evaluated once and every exact product of the solve reads it
    struct UseStored {
      H2Op& h;
      ~UseStored() { h.use = false; }
    } use_stored{c->h2};
    if (c->h2.in_solves) {
      h2_evaluate_dev(c, dU);
      c->h2.use = true;
    }
    jacobian_dev(c, dU, nullptr, inner_its ? AEROF_PREC_FP32 : AEROF_PREC_FP64, inner_its && transpose);
    if (int nb = prec_setup_dev(c, transpose)) {
      c->last_error = std::to_string(nb) + " singular diagonal block(s)";
      return AEROF_ESINGULAR;
    }
    double r = 0.0;
    const int it = inner_its ? fgmres_exact(c, db, dx, krylov, maxits, eps, transpose, &r, dU, std::min(inner_its, 30),
                                            inner_its, 1e-3)
                             : gmres_dev(c, db, dx, krylov, maxits, eps, transpose, &r, dU);
    out_finish(c, x, dx, n);
    if (its) *its = it;
    if (res) *res = r;
    return AEROF_OK;
  });
}

// Several linearised solves sharing one operator set-up (the batched
// direct-sensitivity right-hand sides of a shape optimisation,
// FluidShapeOptimizationHandler.C:2362-2433, one fsoLinearSolver per mode):
// the exact linearisation at U is stored once (MatVecProdH2::evaluate), the
// first-order operator and its block-Jacobi are assembled once, and each
// right-hand side B[k] ([nrhs][N][5]) is solved as aerof_gpu_linearized_solve
// does, its exact products read from the stored operator.
extern "C" int aerof_gpu_linearized_solve_batch(aerof_gpu_ctx* c, const double* U, int nrhs, const double* B,
                                                double* X, int krylov, int maxits, double eps, int transpose,
                                                int inner_its, int* its, double* res) {
  return guard(c, [&]() -> int {
    need_inviscid(c);
    need_mesh_or_throw(c);
    if (!U || !B || !X || nrhs < 0 || krylov < 1 || maxits < 1 || !(eps >= 0.0) || inner_its < 0)
      return AEROF_EINVAL;
    if (nrhs == 0) return AEROF_OK;
    const size_t n = 5 * (size_t)c->mesh.N;
    c->imp.t.ensure(n);
    const double* dU0 = in_dev(c, U, n, c->s.Ustage);
    if (dU0 != c->imp.t.p)
      AEROF_CUDA(cudaMemcpyAsync(c->imp.t.p, dU0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    const double* dU = c->imp.t.p;
    struct UseStored {
      H2Op& h;
      ~UseStored() { h.use = false; }
    } use_stored{c->h2};
    h2_evaluate_dev(c, dU);
    c->h2.use = true;
    jacobian_dev(c, dU, nullptr, inner_its ? AEROF_PREC_FP32 : AEROF_PREC_FP64, inner_its && transpose);
    if (int nb = prec_setup_dev(c, transpose)) {
      c->last_error = std::to_string(nb) + " singular diagonal block(s)";
      return AEROF_ESINGULAR;
    }
    // lockstep flexible GMRES over groups of right-hand sides (the inner
    // FP32 solves of a group share every pass over H1); the group is as
    // large as 70 % of the free device memory allows
    const char* lv = std::getenv("AEROF_LOCKSTEP");
    const bool lockstep = inner_its > 0 && inner_its <= 30 && (!lv || std::atoi(lv) != 0);
    if (lockstep) {
      // right-hand sides and solutions staged at a 512-byte aligned stride
      // (the reductions read 16-byte vectors)
      const size_t ld = (n + 63) / 64 * 64;
      const cudaMemcpyKind kb = is_device_ptr(B) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
      const cudaMemcpyKind kx = is_device_ptr(X) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
      // per right-hand side: the outer FP64 bases and work vectors, the inner
      // FP32 basis and work vectors and, with ILU(0), the sweeps' FP64 work
      // vector (5N doubles)
      const size_t per = ((size_t)2 * krylov + 5 + (c->imp.pc == AEROF_PC_ILU0 ? 1 : 0)) * ld * sizeof(double) +
                         ((size_t)inner_its + 5) * ld * sizeof(float);
      size_t freeb = 0, totalb = 0;
      AEROF_CUDA(cudaMemGetInfo(&freeb, &totalb));
      const int G = (int)std::max<size_t>(1, std::min<size_t>((size_t)nrhs, (size_t)(0.7 * (double)freeb) / per));
      c->imp.bB.ensure((size_t)std::min(G, nrhs) * ld);
      c->imp.bX.ensure((size_t)std::min(G, nrhs) * ld);
      for (int k0 = 0; k0 < nrhs; k0 += G) {
        const int g = std::min(G, nrhs - k0);
        std::vector<const double*> bq(g);
        std::vector<double*> xq(g);
        for (int q = 0; q < g; ++q) {
          AEROF_CUDA(cudaMemcpyAsync(c->imp.bB.p + (size_t)q * ld, B + (size_t)(k0 + q) * n, n * sizeof(double), kb,
                                     c->stream));
          bq[q] = c->imp.bB.p + (size_t)q * ld;
          xq[q] = c->imp.bX.p + (size_t)q * ld;
        }
        gmres_lockstep<double, true>(c, g, bq.data(), xq.data(), krylov, maxits, eps, transpose, dU,
                                     std::min(inner_its, 30), inner_its, 1e-3, its ? its + k0 : nullptr,
                                     res ? res + k0 : nullptr);
        for (int q = 0; q < g; ++q)
          AEROF_CUDA(cudaMemcpyAsync(X + (size_t)(k0 + q) * n, xq[q], n * sizeof(double), kx, c->stream));
        AEROF_CUDA(cudaStreamSynchronize(c->stream));
      }
      return AEROF_OK;
    }
    for (int k = 0; k < nrhs; ++k) {
      const double* db = in_dev(c, B + (size_t)k * n, n, c->s.Vstage);
      double* dx = out_dev(c, X + (size_t)k * n, n, c->s.Rstage);
      double r = 0.0;
      const int it = inner_its ? fgmres_exact(c, db, dx, krylov, maxits, eps, transpose, &r, dU,
                                              std::min(inner_its, 30), inner_its, 1e-3)
                               : gmres_dev(c, db, dx, krylov, maxits, eps, transpose, &r, dU);
      out_finish(c, X + (size_t)k * n, dx, n);
      if (its) its[k] = it;
      if (res) res[k] = r;
    }
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_set_preconditioner(aerof_gpu_ctx* c, int type) {
  return guard(c, [&]() -> int {
    if (type != AEROF_PC_JACOBI && type != AEROF_PC_ILU0) return AEROF_EINVAL;
    if (c->imp.pc != type) {
      c->imp.pc = type;
      c->imp.prec_ready = false;
      c->imp.ilu_ready = false;
    }
    return AEROF_OK;
  });
}
