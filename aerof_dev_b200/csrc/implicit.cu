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
#include <vector>

#include "common.cuh"
#include "physics.cuh"

namespace aerof {

constexpr int kIB = 256;
constexpr int kGB = 1184;  // reduction grid: 8 x 148 SMs

template <class S> __device__ __forceinline__ void store_block(S* dst, const double* v, double scale) {
#pragma unroll
  for (int k = 0; k < 25; ++k) dst[k] = (S)(v[k] * scale);
}

// One thread per edge: approximate Roe Jacobians at the un-reconstructed
// states (roejacappr3Dgas, FluxFcnDescSG.C:155-262), off-diagonal blocks
// A_ij = dF/dU_j / vol_i and A_ji = -dF/dU_i / vol_j (Edge.C:4503-4523),
// and the diagonal contributions +dF/dU_i (row i) and -dF/dU_j (row j) into
// dscr at the same CSR positions, summed per row afterwards.
template <class S>
__global__ void k_jac_edges(int E, Gas g, const int2* __restrict__ edges, const int2* __restrict__ epos,
                            const double* __restrict__ en, const double* __restrict__ P,
                            const double* __restrict__ vol, S* __restrict__ off, double* __restrict__ dscr) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
  const int2 ij = edges[l];
  const int2 pp = epos[l];
  const double n0 = en[l], n1 = en[(size_t)E + l], n2 = en[2 * (size_t)E + l];
  double Vi[5], Vj[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) { Vi[k] = P[8 * (size_t)ij.x + k]; Vj[k] = P[8 * (size_t)ij.y + k]; }
  double ji[25], jj[25];
  if (sqrt(n0 * n0 + n1 * n1 + n2 * n2) < 1e-18) {
#pragma unroll
    for (int k = 0; k < 25; ++k) ji[k] = jj[k] = 0.0;
  } else {
    roe_jac(g, n0, n1, n2, Vi, Vj, 1.0, ji);
    roe_jac(g, n0, n1, n2, Vj, Vi, -1.0, jj);
  }
  const double voli = 1.0 / vol[ij.x], volj = 1.0 / vol[ij.y];
  store_block(off + 25 * (size_t)pp.x, jj, voli);
  store_block(off + 25 * (size_t)pp.y, ji, -volj);
  store_block(dscr + 25 * (size_t)pp.x, ji, 1.0);
  store_block(dscr + 25 * (size_t)pp.y, jj, -1.0);
}

// One thread per node: diagonal block = sum of the row's edge contributions
// (neighbour order), + face blocks (face order, Face.C:814-847), times
// 1/vol (SubDomain.C:1760-1765), + I/dt (TimeState.C:731-756).
template <class S>
__global__ void k_jac_diag(int N, int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ nbr_ptr,
                           const double* __restrict__ dscr, const int* __restrict__ nf_ptr,
                           const int* __restrict__ nf_face, const int* __restrict__ fcode,
                           const double* __restrict__ fn, const double* __restrict__ P,
                           const double* __restrict__ vol, const double* __restrict__ dt, S* __restrict__ diag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double a[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) a[k] = 0.0;
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const double* d = dscr + 25 * (size_t)p;
#pragma unroll
    for (int k = 0; k < 25; ++k) a[k] += d[k];
  }
  const int q1 = nf_ptr[i + 1];
  if (nf_ptr[i] < q1) {
    double V[5], Ub[5], jac[25];
#pragma unroll
    for (int k = 0; k < 5; ++k) { V[k] = P[8 * (size_t)i + k]; Ub[k] = Ub0[k]; }
    const double third = 1.0 / 3.0;
    for (int q = nf_ptr[i]; q < q1; ++q) {
      const int f = nf_face[q];
      face_jac(g, fcode[f], third * fn[f], third * fn[(size_t)F + f], third * fn[2 * (size_t)F + f], V, Ub, jac);
#pragma unroll
      for (int k = 0; k < 25; ++k) a[k] += jac[k];
    }
  }
  const double voli = 1.0 / vol[i];
#pragma unroll
  for (int k = 0; k < 25; ++k) a[k] *= voli;
  if (dt) {
    const double c = 1.0 / dt[i];
#pragma unroll
    for (int k = 0; k < 5; ++k) a[6 * k] += c;
  }
  store_block(diag + 25 * (size_t)i, a, 1.0);
}

// y = A p (or A^T p): per row, diagonal block first, then the row's
// neighbours in ascending order (SubDomain::computeMatVecProdH1 and
// H1transpose, SubDomain.C:3916-3995).  Blocks in S (float or double),
// vectors and accumulation in double.
template <class S, class TX>
__device__ __forceinline__ void gemv_add(const S* __restrict__ a, const TX* __restrict__ x, double* y, bool trans) {
  double xv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) xv[k] = (double)x[k];
  if (!trans) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double s = (double)a[5 * r] * xv[0];
#pragma unroll
      for (int c = 1; c < 5; ++c) s += (double)a[5 * r + c] * xv[c];
      y[r] += s;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
      double s = (double)a[r] * xv[0];
#pragma unroll
      for (int c = 1; c < 5; ++c) s += (double)a[5 * c + r] * xv[c];
      y[r] += s;
    }
  }
}

template <class S, bool TRANS, class TI, class TO>
__global__ void k_spmv(int N, const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_node,
                       const int* __restrict__ nbr_tpos, const S* __restrict__ diag, const S* __restrict__ off,
                       const TI* __restrict__ p, TO* __restrict__ y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double acc[5] = {0, 0, 0, 0, 0};
  gemv_add(diag + 25 * (size_t)i, p + 5 * (size_t)i, acc, TRANS);
  for (int q = nbr_ptr[i]; q < nbr_ptr[i + 1]; ++q) {
    const size_t b = TRANS ? (size_t)nbr_tpos[q] : (size_t)q;
    gemv_add(off + 25 * b, p + 5 * (size_t)nbr_node[q], acc, TRANS);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) y[5 * (size_t)i + k] = (TO)acc[k];
}

// Block-Jacobi set-up (JacobiPrec::setup -> DiagMat::invert, DiagMatrix.C:
// 44-80): blocks with a zero diagonal entry are left as they are (as the
// reference does); a zero pivot counts into bad[0].
template <class S>
__global__ void k_bj_invert(int N, const S* __restrict__ diag, S* __restrict__ dinv, int* __restrict__ bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  S a[25];
#pragma unroll
  for (int k = 0; k < 25; ++k) a[k] = diag[25 * (size_t)i + k];
  bool inv = true;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    if (a[6 * k] == S(0)) inv = false;
  if (inv && invert5<S>(a)) atomicAdd(bad, 1);
#pragma unroll
  for (int k = 0; k < 25; ++k) dinv[25 * (size_t)i + k] = a[k];
}

// z = D^-1 x (or D^-T x): JacobiPrec::apply/applyT (KspPrec.C:86-111)
template <class S, class TI, class TO>
__global__ void k_bj_apply(int N, const S* __restrict__ dinv, const TI* __restrict__ x, TO* __restrict__ z,
                           int trans) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double acc[5] = {0, 0, 0, 0, 0};
  gemv_add(dinv + 25 * (size_t)i, x + 5 * (size_t)i, acc, trans != 0);
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
// Modified Gram-Schmidt step i with the projection of step i-1 fused in:
//   w -= hprev * Vprev   (hprev read from device memory, skipped if null)
//   part[b] = partial sums of w . Vcur      (deterministic block tree)
template <class TV>
__global__ void k_mgs_step(size_t n, const double* __restrict__ hprev, const TV* __restrict__ Vprev,
                           const TV* __restrict__ Vcur, TV* __restrict__ w, double* __restrict__ part) {
  __shared__ double sh[kIB];
  const double h = hprev ? *hprev : 0.0;
  double s = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    double wq = (double)w[q];
    if (hprev) {
      wq = wq - h * (double)Vprev[q];
      w[q] = (TV)wq;
      wq = (double)(TV)wq;
    }
    s += wq * (double)Vcur[q];
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_sum_partials(int nb, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[kIB];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += part[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}
// last projection of the column, then w . w
template <class TV>
__global__ void k_mgs_last(size_t n, const double* __restrict__ hprev, const TV* __restrict__ Vprev,
                           TV* __restrict__ w, double* __restrict__ part) {
  __shared__ double sh[kIB];
  const double h = *hprev;
  double s = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const TV wt = (TV)((double)w[q] - h * (double)Vprev[q]);
    w[q] = wt;
    const double wq = (double)wt;
    s += wq * wq;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
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
template <class TA>
__global__ void k_add(size_t n, const TA* __restrict__ a, double* __restrict__ x) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) x[q] += (double)a[q];
}
// deterministic dot / squared norm of TV vectors, FP64 accumulation
template <class TV>
__global__ void k_dot_tv(size_t n, const TV* __restrict__ x, const TV* __restrict__ y, double* __restrict__ part) {
  __shared__ double sh[kIB];
  double s = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    s += (double)x[q] * (double)y[q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
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
void jacobian_dev(aerof_gpu_ctx* c, const double* dU, const double* ddt, int precision) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const Gas g = make_gas(c->cfg.gamma);
  TimerScope tj(c, AEROF_T_FV_JAC);
  prim_dev(c, dU);
  J.diagscr.ensure(25 * 2 * (size_t)m.E);
  const int ge = grid_for(m.E, kIB), gn = grid_for(m.N, kIB);
  if (precision == AEROF_PREC_FP32) {
    J.diag64.release(); J.off64.release(); J.dinv64.release();
    J.diag32.alloc(25 * (size_t)m.N);
    J.off32.alloc(25 * 2 * (size_t)m.E);
    k_jac_edges<float><<<ge, kIB, 0, c->stream>>>(m.E, g, m.edges.p, m.edge_pos.p, m.en.p, m.P.p, m.vol.p, J.off32.p,
                                                  J.diagscr.p);
    AEROF_LAUNCH_CHECK();
    k_jac_diag<float><<<gn, kIB, 0, c->stream>>>(m.N, m.F, g, m.Ubd.p, m.nbr_ptr.p, J.diagscr.p, m.nf_ptr.p,
                                                 m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, m.vol.p, ddt, J.diag32.p);
    AEROF_LAUNCH_CHECK();
  } else {
    J.diag32.release(); J.off32.release(); J.dinv32.release();
    J.diag64.alloc(25 * (size_t)m.N);
    J.off64.alloc(25 * 2 * (size_t)m.E);
    k_jac_edges<double><<<ge, kIB, 0, c->stream>>>(m.E, g, m.edges.p, m.edge_pos.p, m.en.p, m.P.p, m.vol.p,
                                                   J.off64.p, J.diagscr.p);
    AEROF_LAUNCH_CHECK();
    k_jac_diag<double><<<gn, kIB, 0, c->stream>>>(m.N, m.F, g, m.Ubd.p, m.nbr_ptr.p, J.diagscr.p, m.nf_ptr.p,
                                                  m.nf_face.p, m.fcode.p, m.fnrm.p, m.P.p, m.vol.p, ddt, J.diag64.p);
    AEROF_LAUNCH_CHECK();
  }
  J.precision = precision;
  J.prec_ready = false;
}

template <class TI, class TO>
void matvec_t(aerof_gpu_ctx* c, const TI* p, TO* y, int trans) {
  DeviceMesh& m = c->mesh;
  TimerScope tm(c, AEROF_T_KSP_MATVEC);
  Implicit& J = c->imp;
  const int gn = grid_for(m.N, kIB);
  if (J.precision == AEROF_PREC_FP32) {
    if (trans) k_spmv<float, true, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, m.nbr_ptr.p, m.nbr_node.p, m.nbr_tpos.p, J.diag32.p, J.off32.p, p, y);
    else k_spmv<float, false, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, m.nbr_ptr.p, m.nbr_node.p, m.nbr_tpos.p, J.diag32.p, J.off32.p, p, y);
  } else {
    if (trans) k_spmv<double, true, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, m.nbr_ptr.p, m.nbr_node.p, m.nbr_tpos.p, J.diag64.p, J.off64.p, p, y);
    else k_spmv<double, false, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, m.nbr_ptr.p, m.nbr_node.p, m.nbr_tpos.p, J.diag64.p, J.off64.p, p, y);
  }
  AEROF_LAUNCH_CHECK();
}
void matvec_dev(aerof_gpu_ctx* c, const double* p, double* y, int trans) { matvec_t<double, double>(c, p, y, trans); }

int prec_setup_dev(aerof_gpu_ctx* c) {
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  TimerScope tp(c, AEROF_T_PREC_SETUP);
  c->s.counters.ensure(8);
  int* bad = c->s.counters.p + 4;
  AEROF_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), c->stream));
  const int gn = grid_for(m.N, kIB);
  if (J.precision == AEROF_PREC_FP32) {
    J.dinv32.alloc(25 * (size_t)m.N);
    k_bj_invert<float><<<gn, kIB, 0, c->stream>>>(m.N, J.diag32.p, J.dinv32.p, bad);
  } else {
    J.dinv64.alloc(25 * (size_t)m.N);
    k_bj_invert<double><<<gn, kIB, 0, c->stream>>>(m.N, J.diag64.p, J.dinv64.p, bad);
  }
  AEROF_LAUNCH_CHECK();
  int h = 0;
  AEROF_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  AEROF_CUDA(cudaStreamSynchronize(c->stream));
  J.prec_ready = true;
  return h;
}

template <class TI, class TO>
void prec_apply_t(aerof_gpu_ctx* c, const TI* x, TO* z, int trans) {
  DeviceMesh& m = c->mesh;
  TimerScope tp(c, AEROF_T_KSP_OTHER);
  Implicit& J = c->imp;
  const int gn = grid_for(m.N, kIB);
  if (J.precision == AEROF_PREC_FP32)
    k_bj_apply<float, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, J.dinv32.p, x, z, trans);
  else
    k_bj_apply<double, TI, TO><<<gn, kIB, 0, c->stream>>>(m.N, J.dinv64.p, x, z, trans);
  AEROF_LAUNCH_CHECK();
}
void prec_apply_dev(aerof_gpu_ctx* c, const double* x, double* z, int trans) {
  prec_apply_t<double, double>(c, x, z, trans);
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
  DeviceMesh& m = c->mesh;
  Implicit& J = c->imp;
  const size_t n = 5 * (size_t)m.N;
  const int gv = grid_for(n, kIB);
  cudaStream_t s = c->stream;
  const size_t vbytes = (size_t)(numVec + 1) * n * sizeof(TV);
  J.basis.ensure((vbytes + 7) / 8);
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
    const double* pd = reinterpret_cast<const double*>(p);
    double* yy = reinterpret_cast<double*>(y);
    if (trans) vjp_dev(c, exactU, pd, yy);
    else residual_forward(c, exactU, pd, nullptr, yy, false);
  };
  auto norm2 = [&](const TV* v) -> double {
    k_dot_tv<TV><<<kGB, kIB, 0, s>>>(n, v, v, part);
    AEROF_LAUNCH_CHECK();
    k_sum_partials<<<1, kIB, 0, s>>>(kGB, part, hd);
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
    k_mgs_step<TV><<<kGB, kIB, 0, s>>>(n, hp, vprev, vcur, w, part);
    AEROF_LAUNCH_CHECK();
    k_sum_partials<<<1, kIB, 0, s>>>(kGB, part, out);
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
        prec_apply_t<TV, TV>(c, Vb + (size_t)j * n, r, trans);
      }
      op(r, w);
      // h_ij = w . V_i ; w -= h_ij V_i   (i = 0..j), then ||w||
      TimerScope t(c, AEROF_T_KSP_OTHER);
      for (int i = 0; i <= j; ++i)
        dot_to(i ? hd + (i - 1) : nullptr, i ? Vb + (size_t)(i - 1) * n : nullptr, Vb + (size_t)i * n, hd + i);
      k_mgs_last<TV><<<kGB, kIB, 0, s>>>(n, hd + j, Vb + (size_t)j * n, w, part);
      AEROF_LAUNCH_CHECK();
      k_sum_partials<<<1, kIB, 0, s>>>(kGB, part, hd + j + 1);
      AEROF_LAUNCH_CHECK();
      AEROF_CUDA(cudaMemcpyAsync(hcol.data(), hd, sizeof(double) * (j + 2), cudaMemcpyDeviceToHost, s));
      AEROF_CUDA(cudaStreamSynchronize(s));
      for (int i = 0; i <= j; ++i) h(i, j) = hcol[i];
      h(j + 1, j) = std::sqrt(hcol[j + 1]);
      const bool breakdown = (h(j + 1, j) == 0.0);
      if (!breakdown) {
        k_scale<TV, TV><<<gv, kIB, 0, s>>>(n, 1. / h(j + 1, j), w, Vb + (size_t)(j + 1) * n);
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
    k_combine<TV><<<gv, kIB, 0, s>>>(n, j + 1, yd, Vb, n, w);
    AEROF_LAUNCH_CHECK();
    prec_apply_t<TV, TV>(c, w, r, trans);
    k_add<TV><<<gv, kIB, 0, s>>>(n, r, x);
    AEROF_LAUNCH_CHECK();
  } while (exitLoop == 0);
  AEROF_CUDA(cudaStreamSynchronize(s));
  if (final_res) *final_res = l2res;
  return iter;
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
    jacobian_dev(c, dU, ddt, precision);
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
    const size_t nd = 25 * (size_t)m.N, no = 25 * 2 * (size_t)m.E;
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
    std::vector<int2> epos(m.E);
    AEROF_CUDA(cudaMemcpyAsync(epos.data(), m.edge_pos.p, sizeof(int2) * m.E, cudaMemcpyDeviceToHost, c->stream));
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    std::copy(diag.begin(), diag.end(), A);
    for (int l = 0; l < m.E; ++l) {
      std::copy(&off[25 * (size_t)epos[l].x], &off[25 * (size_t)epos[l].x] + 25, A + nd + 50 * (size_t)l);
      std::copy(&off[25 * (size_t)epos[l].y], &off[25 * (size_t)epos[l].y] + 25, A + nd + 50 * (size_t)l + 25);
    }
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
    c->imp.b.ensure(n); c->imp.x.ensure(n); c->s.dt.ensure(m.N); c->s.k1.ensure(n);
    double* R = c->s.k1.p;
    double* rhs = c->imp.b.p;
    double* dQ = c->imp.x.p;
    double* dt = c->s.dt.p;
    const int gv = grid_for(n, kIB);
    cudaEvent_t e0, e1;
    AEROF_CUDA(cudaEventCreate(&e0));
    AEROF_CUDA(cudaEventCreate(&e1));
    AEROF_CUDA(cudaEventRecord(e0, s));
    double res0 = 0.0, rel = 1.0, rel_prev = 1.0, cfl = p->cfl0;
    int k, lits = 0, bad = 0;
    for (k = 0; k <= p->max_steps; ++k) {
      bad += residual_dev(c, dU, R);
      double res = norm2_dev(c, R, n);
      if (k == 0) res0 = res;
      rel = res0 > 0.0 ? res / res0 : 0.0;
      if (history) history[k] = rel;
      if (!std::isfinite(rel)) throw ApiError{AEROF_EINVAL, "non-finite residual in Newton step " + std::to_string(k)};
      if (rel <= p->tol || k == p->max_steps) break;
      if (k > 0) cfl = std::min(std::max(cfl * std::pow(rel_prev / rel, p->ser), p->cfl_min), p->cfl_max);
      rel_prev = rel;
      timestep_dev(c, dU, cfl, dt);
      jacobian_dev(c, dU, dt, p->precision);
      if (int nb = prec_setup_dev(c)) {
        c->last_error = std::to_string(nb) + " singular diagonal block(s) at Newton step " + std::to_string(k);
        return AEROF_ESINGULAR;
      }
      k_scale<double, double><<<gv, kIB, 0, s>>>(n, -1.0, R, rhs);
      AEROF_LAUNCH_CHECK();
      lits += gmres_dev(c, rhs, dQ, p->ksp_krylov, p->ksp_maxits, p->ksp_eps, 0, nullptr, nullptr);
      k_add<double><<<gv, kIB, 0, s>>>(n, dQ, dU);
      AEROF_LAUNCH_CHECK();
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
                                          int maxits, double eps, int transpose, int* its, double* res) {
  return guard(c, [&]() -> int {
    need_mesh_or_throw(c);
    if (!U || !b || !x || krylov < 1 || maxits < 1 || !(eps >= 0.0)) return AEROF_EINVAL;
    const size_t n = 5 * (size_t)c->mesh.N;
    c->imp.t.ensure(n);
    const double* dU0 = in_dev(c, U, n, c->s.Ustage);
    if (dU0 != c->imp.t.p)
      AEROF_CUDA(cudaMemcpyAsync(c->imp.t.p, dU0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    const double* dU = c->imp.t.p;
    const double* db = in_dev(c, b, n, c->s.Vstage);
    double* dx = out_dev(c, x, n, c->s.Rstage);
    jacobian_dev(c, dU, nullptr, AEROF_PREC_FP64);
    if (int nb = prec_setup_dev(c)) {
      c->last_error = std::to_string(nb) + " singular diagonal block(s)";
      return AEROF_ESINGULAR;
    }
    double r = 0.0;
    int it = gmres_dev(c, db, dx, krylov, maxits, eps, transpose, &r, dU);
    out_finish(c, x, dx, n);
    if (its) *its = it;
    if (res) *res = r;
    return AEROF_OK;
  });
}
