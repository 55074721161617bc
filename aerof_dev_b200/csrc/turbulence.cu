// turbulence.cu -- the Spalart-Allmaras residual (one-equation model
// strongly coupled to the flow: six conserved variables per node, rho nu~
// last) on the GPU, FP64.
//
// Finite-volume term in the edge organisation (caller numbering): primitive
// conversion (VarFcnSGSA::conservativeToPrimitive, VarFcnSGSA.h:210-224),
// LSQ gradients of the six components (the weights of the Euler path,
// SubDomain.C:137-159, 297-374), per edge the componentwise reconstruction,
// the positivity check and the Roe flux with its advected sixth component
// (roeflux7.f:190-196, type 1), per boundary face the slip-wall or
// far-field flux (boundflux5.f:92-103, type 1), then per node the edge
// fluxes in ascending-neighbour order and the subface fluxes in face order,
// times 1/ctrlVol.  Galerkin term (FemEquationTermSA::computeVolumeTerm,
// FemEquationTermDesc.C:669-787, assembled as ElemTet::computeGalerkinTerm,
// ElemTet.C:99-114): one thread per tet forms vol (r . dN_j) - vol/4 s for
// each of its four nodes, then each node sums its tets' shares in tet order
// and adds the sum divided by the control volume.  Every sum is a gather in
// a fixed order (no atomics on doubles).
#include "common.cuh"
#include "physics.cuh"

namespace aerof {

struct SADev {
  int model, fv3;
  double ooreynolds, ooprandtl, bulk, alpha, Ts;
  double cb1, cb2, cw2, cw3_pow6, opcw3_pow, cv1_pow3, oocv2, oosigma, cw1, oovkcst2, oopr_t;
};

__global__ void k_prim6(int N, Gas g, const double* __restrict__ U, double* __restrict__ V) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double* u = U + 6 * (size_t)i;
  double* v = V + 6 * (size_t)i;
  const double invRho = 1.0 / u[0];
  const double v1 = u[1] * invRho, v2 = u[2] * invRho, v3 = u[3] * invRho;
  const double vel2 = v1 * v1 + v2 * v2 + v3 * v3;
  v[0] = u[0];
  v[1] = v1;
  v[2] = v2;
  v[3] = v3;
  v[4] = g.gam1 * (u[4] - 0.5 * u[0] * vel2);
  v[5] = u[5] * invRho;
}

// LSQ gradients of the six components: four lanes per node take the
// neighbours r, r+4, ... of its ascending list; fixed xor-tree lane sum.
// G[18 i + 6 a + k] = d V_k / d x_a.
__global__ void __launch_bounds__(256) k_grad6(int N, const double* __restrict__ V, const double* __restrict__ X,
                                               const double* __restrict__ lsqW, const int* __restrict__ nbr_ptr,
                                               const int* __restrict__ nbr_node, double* __restrict__ G) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t >> 2, r = t & 3;
  const bool act = i < N;
  double g[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) g[k] = 0.0;
  if (act) {
    double w[6], vi[6], xi[3];
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = lsqW[(size_t)k * N + i];
#pragma unroll
    for (int k = 0; k < 6; ++k) vi[k] = V[6 * (size_t)i + k];
#pragma unroll
    for (int a = 0; a < 3; ++a) xi[a] = X[3 * (size_t)i + a];
    for (int p = nbr_ptr[i] + r; p < nbr_ptr[i + 1]; p += 4) {
      const int j = nbr_node[p];
      double W0, W1, W2;
      lsq_weights(w, X[3 * (size_t)j] - xi[0], X[3 * (size_t)j + 1] - xi[1], X[3 * (size_t)j + 2] - xi[2], W0, W1,
                  W2);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double dv = V[6 * (size_t)j + k] - vi[k];
        g[k] += W0 * dv;
        g[6 + k] += W1 * dv;
        g[12 + k] += W2 * dv;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 18; ++k) {
    g[k] += __shfl_xor_sync(0xffffffffu, g[k], 1);
    g[k] += __shfl_xor_sync(0xffffffffu, g[k], 2);
  }
  if (!act || r != 0) return;
#pragma unroll
  for (int k = 0; k < 18; ++k) G[18 * (size_t)i + k] = g[k];
}

// upwinded sixth flux component of roeflux7 / boundflux5 with type 1:
// phi6 = phi1 (updir a + (1 - updir) b), updir = 0.5 + sign(0.5, phi1)
__device__ __forceinline__ double sa_upwind(double phi1, double a, double b) {
  const double updir = 0.5 + copysign(0.5, phi1);
  return phi1 * (updir * a + (1.0 - updir) * b);
}

// Roe flux of every edge into flux[E][6] (one 48-byte record per edge);
// non-positive reconstructed densities or pressures skip the edge and are
// counted.
__global__ void k_edge_flux6(int E, Gas g, int rec, double beta, const int2* __restrict__ edges,
                             const double* __restrict__ en, const double* __restrict__ V,
                             const double* __restrict__ X, const double* __restrict__ G,
                             double* __restrict__ flux, int* __restrict__ counter) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= E) return;
  const int2 ij = edges[l];
  const double* vi = V + 6 * (size_t)ij.x;
  const double* vj = V + 6 * (size_t)ij.y;
  double Vi[6], Vj[6];
  if (rec == AEROF_REC_CONSTANT) {
#pragma unroll
    for (int k = 0; k < 6; ++k) { Vi[k] = vi[k]; Vj[k] = vj[k]; }
  } else {
    const double dx0 = X[3 * (size_t)ij.y] - X[3 * (size_t)ij.x];
    const double dx1 = X[3 * (size_t)ij.y + 1] - X[3 * (size_t)ij.x + 1];
    const double dx2 = X[3 * (size_t)ij.y + 2] - X[3 * (size_t)ij.x + 2];
    const double* gi = G + 18 * (size_t)ij.x;
    const double* gj = G + 18 * (size_t)ij.y;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double ddVij = dx0 * gi[k] + dx1 * gi[6 + k] + dx2 * gi[12 + k];
      const double ddVji = dx0 * gj[k] + dx1 * gj[6 + k] + dx2 * gj[12 + k];
      if (rec == AEROF_REC_VANALBADA) vanalbada(beta, vi[k], ddVij, vj[k], ddVji, Vi[k], Vj[k]);
      else linear_rec(beta, vi[k], ddVij, vj[k], ddVji, Vi[k], Vj[k]);
    }
  }
  double f[6] = {0, 0, 0, 0, 0, 0};
  const bool bi = !(Vi[0] > 0.0) || !(Vi[4] > 0.0);
  const bool bj = !(Vj[0] > 0.0) || !(Vj[4] > 0.0);
  const double n0 = en[l], n1 = en[(size_t)E + l], n2 = en[2 * (size_t)E + l];
  if (bi || bj) {
    atomicAdd(counter, (int)bi + (int)bj);
  } else if (n0 * n0 + n1 * n1 + n2 * n2 >= 1e-36) {
    roe_flux(g, n0, n1, n2, Vi, Vj, f);
    f[5] = sa_upwind(f[0], Vi[5], Vj[5]);
  }
  double2* o = reinterpret_cast<double2*>(flux + 6 * (size_t)l);
  o[0] = make_double2(f[0], f[1]);
  o[1] = make_double2(f[2], f[3]);
  o[2] = make_double2(f[4], f[5]);
}

// Boundary subface fluxes (normal n_f / 3) into fbuf[3F][6].
__global__ void k_face_flux6(int F, Gas g, const double* __restrict__ Ub0, const int* __restrict__ faces,
                             const int* __restrict__ fcode, const double* __restrict__ fn,
                             const double* __restrict__ V, double* __restrict__ fbuf) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  const double third = 1.0 / 3.0;
  double Ub[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) Ub[k] = Ub0[k];
  const double nx = third * fn[f], ny = third * fn[(size_t)F + f], nz = third * fn[2 * (size_t)F + f];
  const int code = fcode[f];
  for (int l = 0; l < 3; ++l) {
    const double* v = V + 6 * (size_t)faces[3 * (size_t)f + l];
    double Vn[5], ff[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) Vn[k] = v[k];
    face_flux(g, code, nx, ny, nz, Vn, Ub, ff);
    double* out = fbuf + 6 * (3 * (size_t)f + l);
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = ff[k];
    out[5] = code == AEROF_BC_SLIP_WALL_MOVING ? 0.0 : sa_upwind(ff[0], v[5], Ub[5] * (1.0 / Ub[0]));
  }
}

// Per node: edges in ascending-neighbour order (+ first endpoint, -
// second), boundary subfaces in face order, times 1/ctrlVol; three lanes
// per node, lane c summing components 2c and 2c + 1 (16-byte loads of the
// 48-byte edge and subface records)
__global__ void k_node_residual6(int N, const int* __restrict__ nbr_ptr, const int* __restrict__ nbr_edge,
                                 const double* __restrict__ flux, const int* __restrict__ nf_ptr,
                                 const int* __restrict__ nf_face, const int* __restrict__ faces,
                                 const double* __restrict__ fbuf, const double* __restrict__ vol,
                                 double* __restrict__ R) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= 3 * (long long)N) return;
  const int i = (int)(j / 3), c = (int)(j - 3 * (long long)i);
  double a0 = 0.0, a1 = 0.0;
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    const int e = nbr_edge[p];
    const size_t l = (size_t)(e & 0x7fffffff);
    const double sg = e < 0 ? -1.0 : 1.0;
    const double2 v = reinterpret_cast<const double2*>(flux + 6 * l)[c];
    a0 += sg * v.x;
    a1 += sg * v.y;
  }
  for (int q = nf_ptr[i]; q < nf_ptr[i + 1]; ++q) {
    const int f = nf_face[q];
    const int* fd = faces + 3 * (size_t)f;
    const int l = fd[0] == i ? 0 : (fd[1] == i ? 1 : 2);
    const double2 v = reinterpret_cast<const double2*>(fbuf + 6 * (3 * (size_t)f + l))[c];
    a0 += v.x;
    a1 += v.y;
  }
  const double invcv = 1.0 / vol[i];
  // R is the caller's array: 8-byte stores (no alignment beyond a double's)
  R[6 * (size_t)i + 2 * c] = a0 * invcv;
  R[6 * (size_t)i + 2 * c + 1] = a1 * invcv;
}

// P1 shape-function gradients of tet nd (ElemTet::computeGradientP1Function,
// ElemTetCore.C:1961-2010); returns the volume.
__device__ __forceinline__ double p1_grad6(const double x[4][3], double g[4][3]) {
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

// One thread per tet: node k's share of the tet's SA Galerkin term,
// vol (r_1..5 . dN_k) - vol/4 s in the last component (component 0 of r
// is zero), written as the record C[5 (4t + k) .. +4]; the block's records
// are staged in shared memory (row stride 21 doubles: conflict-free) and
// stored contiguously with evict-first stores (each record is read once,
// by k_tet_gather).  Q: per-node records of k_sa_records
template <int TB>
__global__ void __launch_bounds__(TB) k_galerkin_sa_tets(int T, Gas gs, SADev sp, const int* __restrict__ tets,
                                                         const double* __restrict__ Q, double* __restrict__ C) {
  constexpr int REC = 20, RS = REC + 1;
  __shared__ double st[TB * RS];
  const int t0 = blockIdx.x * TB, t = t0 + threadIdx.x;
  if (t < T) {
    const double cp = gs.gam * gs.invgam1;
    const double twothird = 2.0 / 3.0, sixth = 1.0 / 6.0;
    const int4 q4 = *reinterpret_cast<const int4*>(tets + 4 * (size_t)t);
    const int nd[4] = {q4.x, q4.y, q4.z, q4.w};
    double u[4][3], Tn[4], rh[4], nu[4], dw[4], x[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double2* q = reinterpret_cast<const double2*>(Q + 12 * (size_t)nd[k]);
      const double2 a = q[0], b = q[1], c = q[2], d = q[3], e = q[4];
      rh[k] = a.x; u[k][0] = a.y; u[k][1] = b.x; u[k][2] = b.y;
      Tn[k] = c.x; nu[k] = c.y; dw[k] = d.x;
      x[k][0] = d.y; x[k][1] = e.x; x[k][2] = e.y;
    }
    double g[4][3];
    const double tv = p1_grad6(x, g);
    double ucg[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ucg[a] = 0.25 * (u[0][a] + u[1][a] + u[2][a] + u[3][a]);
    const double Tcg = 0.25 * (Tn[0] + Tn[1] + Tn[2] + Tn[3]);
    double du[3][3], dT[3], dnu[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int j = 0; j < 3; ++j) du[a][j] = g[0][j] * u[0][a] + g[1][j] * u[1][a] + g[2][j] * u[2][a] + g[3][j] * u[3][a];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      dT[j] = g[0][j] * Tn[0] + g[1][j] * Tn[1] + g[2][j] * Tn[2] + g[3][j] * Tn[3];
      dnu[j] = g[0][j] * nu[0] + g[1][j] * nu[1] + g[2][j] * nu[2] + g[3][j] * nu[3];
    }
    // laminar coefficients at the mean temperature (before 1/Re)
    double mul, lambdal;
    if (sp.model == 2) {
      const double Ta = sp.alpha * Tcg;
      mul = Ta * sqrt(Ta) * (1.0 + sp.Ts) / (Ta + sp.Ts);
      lambdal = -twothird * mul;
    } else {
      mul = 1.0;
      lambdal = sp.bulk - twothird * mul;
    }
    const double kappal = sp.ooprandtl * cp * mul;
    // eddy viscosity (SATerm::computeTurbulentViscosity)
    const double mutilde = 0.25 * (rh[0] * nu[0] + rh[1] * nu[1] + rh[2] * nu[2] + rh[3] * nu[3]);
    const double chi0 = mutilde / mul;
    const double chi03 = chi0 * chi0 * chi0;
    const double mut = mutilde * (chi03 / (chi03 + sp.cv1_pow3));
    const double lambdat = -2.0 * mut / 3.0;
    const double kappat = cp * mut * sp.oopr_t;
    const double absmutilde = fabs(mutilde), maxmutilde = fmax(mutilde, 0.0);
    const double mu5 = sp.oosigma * (mul + absmutilde);
    double s5 = 0.0;
    const double d2w = 0.25 * (dw[0] + dw[1] + dw[2] + dw[3]);
    if (d2w >= 1.e-15) {
      const double chi = fmax(mutilde / mul, 0.001);
      const double chi3 = chi * chi * chi;
      const double fv1 = chi3 / (chi3 + sp.cv1_pow3);
      double fv2 = 1. - chi / (1. + chi * fv1);
      double fv3 = 1.0;
      if (sp.fv3) {
        fv2 = 1.0 + sp.oocv2 * chi;
        fv2 = 1.0 / (fv2 * fv2 * fv2);
        fv3 = (1.0 + chi * fv1) * (1.0 - fv2) / chi;
      }
      const double ood2wall2 = 1.0 / (d2w * d2w);
      const double rho = 0.25 * (rh[0] + rh[1] + rh[2] + rh[3]);
      const double oorho = 1.0 / rho;
      const double zz = sp.ooreynolds * sp.oovkcst2 * maxmutilde * oorho * ood2wall2;
      const double s12 = du[0][1] - du[1][0];
      const double s23 = du[1][2] - du[2][1];
      const double s31 = du[2][0] - du[0][2];
      const double sv = sqrt(s12 * s12 + s23 * s23 + s31 * s31);
      const double Stilde = fmax(sv * fv3 + zz * fv2, 1.0e-12);
      const double rr = fmin(zz / Stilde, 2.0);
      const double rr2 = rr * rr;
      const double gg = rr + sp.cw2 * (rr2 * rr2 * rr2 - rr);
      const double gg2 = gg * gg;
      const double fw = sp.opcw3_pow * gg * pow(gg2 * gg2 * gg2 + sp.cw3_pow6, -sixth);
      const double AA = sp.oosigma * sp.cb2 * rho * (dnu[0] * dnu[0] + dnu[1] * dnu[1] + dnu[2] * dnu[2]);
      const double BB = sp.cb1 * Stilde * absmutilde;
      const double CC = -sp.cw1 * fw * oorho * maxmutilde * maxmutilde * ood2wall2;
      s5 = AA + BB + CC;
    }
    const double mu = sp.ooreynolds * (mul + mut), lambda = sp.ooreynolds * (lambdal + lambdat);
    const double kappa = sp.ooreynolds * (kappal + kappat);
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
      r[j][0] = tij[0][j];
      r[j][1] = tij[1][j];
      r[j][2] = tij[2][j];
      r[j][3] = ucg[0] * tij[0][j] + ucg[1] * tij[1][j] + ucg[2] * tij[2][j] - (-kappa * dT[j]);
      r[j][4] = mu5 * dnu[j];
    }
    double* row = st + threadIdx.x * RS;
#pragma unroll
    for (int kj = 0; kj < 4; ++kj) {
#pragma unroll
      for (int k = 0; k < 4; ++k) row[5 * kj + k] = tv * (r[0][k] * g[kj][0] + r[1][k] * g[kj][1] + r[2][k] * g[kj][2]);
      row[5 * kj + 4] = tv * ((r[0][4] * g[kj][0] + r[1][4] * g[kj][1] + r[2][4] * g[kj][2]) - 0.25 * s5);
    }
  }
  __syncthreads();
  const int cnt = min(TB, T - t0) * REC;
  double* out = C + (size_t)t0 * REC;
  for (int f = threadIdx.x; f < cnt; f += TB) __stcs(out + f, st[(f / REC) * RS + (f % REC)]);
}

// Per-node records of the SA Galerkin term: (rho, u, v, w, T, nu~, d2wall,
// x, y, z, 0, 0) with T = p / ((gamma - 1) rho), formed once per node
// instead of once per (tet, vertex); V: primitive records of k_prim6
__global__ void k_sa_records(int N, Gas g, const double* __restrict__ V, const double* __restrict__ X,
                             const double* __restrict__ d2wall, double* __restrict__ Q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double* v = V + 6 * (size_t)i;
  const double* xi = X + 3 * (size_t)i;
  double2* q = reinterpret_cast<double2*>(Q + 12 * (size_t)i);
  q[0] = make_double2(v[0], v[1]);
  q[1] = make_double2(v[2], v[3]);
  q[2] = make_double2(g.invgam1 * v[4] / v[0], v[5]);
  q[3] = make_double2(d2wall[i], xi[0]);
  q[4] = make_double2(xi[1], xi[2]);
  q[5] = make_double2(0.0, 0.0);
}

static SADev sa_dev(const aerof_gpu_ctx* c) {
  const aerof_sa_params& p = c->turb.p;
  SADev d;
  d.model = c->visc.model;
  d.fv3 = p.fv3;
  d.ooreynolds = c->visc.model ? 1.0 / c->visc.reynolds_mu : 0.0;
  d.ooprandtl = c->visc.model ? 1.0 / c->visc.prandtl : 0.0;
  d.bulk = c->visc.bulk_viscosity;
  d.alpha = c->visc.sutherland_alpha;
  d.Ts = c->visc.sutherland_Ts;
  d.cb1 = p.cb1;
  d.cb2 = p.cb2;
  d.cw2 = p.cw2;
  d.cw3_pow6 = p.cw3 * p.cw3 * p.cw3 * p.cw3 * p.cw3 * p.cw3;
  d.opcw3_pow = std::pow(1.0 + d.cw3_pow6, 1.0 / 6.0);
  d.cv1_pow3 = p.cv1 * p.cv1 * p.cv1;
  d.oocv2 = 1.0 / p.cv2;
  d.oovkcst2 = 1.0 / (p.vkcst * p.vkcst);
  // SATerm::SATerm: cw1 and 1/sigma carry the 1/Re of the viscosity
  d.cw1 = (p.cb1 * d.oovkcst2 + (1.0 + p.cb2) * (1.0 / p.sigma)) * d.ooreynolds;
  d.oosigma = (1.0 / p.sigma) * d.ooreynolds;
  d.oopr_t = 1.0 / p.prandtl_turbulent;
  return d;
}

// SA residual of the device state dU [N][6] into dR [N][6]; returns the
// number of non-positive reconstructed states (synchronous)
static int residual_sa_dev(aerof_gpu_ctx* c, const double* dU, double* dR) {
  DeviceMesh& m = c->mesh;
  TurbWork& t = c->turb;
  cudaStream_t s = c->stream;
  const Gas g = make_gas(c->cfg.gamma);
  const int rec = c->cfg.reconstruction;
  t.V6.ensure(6 * (size_t)m.N);
  t.G6.ensure(18 * (size_t)m.N);
  t.flux6.ensure(6 * (size_t)std::max(m.E, 1));
  t.fbuf6.ensure(18 * (size_t)std::max(m.F, 1));
  c->s.counters.ensure(8);
  int* cnt = c->s.counters.p;
  AEROF_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
  k_prim6<<<grid_for(m.N, 256), 256, 0, s>>>(m.N, g, dU, t.V6.p);
  AEROF_LAUNCH_CHECK();
  if (rec != AEROF_REC_CONSTANT) {
    k_grad6<<<grid_for(4 * (size_t)m.N, 256), 256, 0, s>>>(m.N, t.V6.p, m.X.p, m.lsqW.p, m.nbr_ptr.p, m.nbr_node.p,
                                                          t.G6.p);
    AEROF_LAUNCH_CHECK();
  }
  k_edge_flux6<<<grid_for(m.E, 256), 256, 0, s>>>(m.E, g, rec, c->cfg.beta, m.edges.p, m.en.p, t.V6.p, m.X.p, t.G6.p,
                                                  t.flux6.p, cnt);
  AEROF_LAUNCH_CHECK();
  if (m.F) {
    k_face_flux6<<<grid_for(m.F, 256), 256, 0, s>>>(m.F, g, t.Ubd.p, m.faces.p, m.fcode.p, m.fnrm.p, t.V6.p,
                                                    t.fbuf6.p);
    AEROF_LAUNCH_CHECK();
  }
  k_node_residual6<<<grid_for(3 * (size_t)m.N, 256), 256, 0, s>>>(m.N, m.nbr_ptr.p, m.nbr_edge.p, t.flux6.p,
                                                                  m.nf_ptr.p, m.nf_face.p, m.faces.p, t.fbuf6.p,
                                                                  m.vol.p, dR);
  AEROF_LAUNCH_CHECK();
  if (c->visc.model != 0) {
    t.tetc.ensure(20 * (size_t)std::max(m.T, 1));
    t.q.ensure(12 * (size_t)m.N);
    k_sa_records<<<grid_for(m.N, 256), 256, 0, s>>>(m.N, g, t.V6.p, m.X.p, t.d2wall.p, t.q.p);
    AEROF_LAUNCH_CHECK();
    if (m.T) {
      k_galerkin_sa_tets<128><<<grid_for(m.T, 128), 128, 0, s>>>(m.T, g, sa_dev(c), m.tets.p, t.q.p, t.tetc.p);
      AEROF_LAUNCH_CHECK();
    }
    k_tet_gather<5, 6, 1><<<grid_for(5 * (size_t)m.N, 256), 256, 0, s>>>(m.N, m.nt_ptr.p, m.nt_tet.p, t.tetc.p,
                                                                        m.vol.p, dR);
    AEROF_LAUNCH_CHECK();
  }
  int bad = 0;
  AEROF_CUDA(cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
  AEROF_CUDA(cudaStreamSynchronize(s));
  return bad;
}

}  // namespace aerof

using namespace aerof;

extern "C" int aerof_gpu_set_turbulence(aerof_gpu_ctx* c, const aerof_sa_params* p, const double* d2wall,
                                        const double* Ub) {
  return guard(c, [&]() -> int {
    if (!c->has_mesh) {
      c->last_error = "no mesh: call aerof_gpu_set_mesh first";
      return AEROF_ESTATE;
    }
    TurbWork& t = c->turb;
    if (!p) {
      t.on = false;
      return AEROF_OK;
    }
    if (!d2wall || !Ub) return AEROF_EINVAL;
    if (!(p->sigma > 0.0 && p->vkcst > 0.0 && p->cv1 > 0.0 && p->cv2 > 0.0 && p->prandtl_turbulent > 0.0 &&
          p->cw3 >= 0.0 && Ub[0] > 0.0)) {
      c->last_error = "Spalart-Allmaras constants must be positive, and the free-stream density too";
      return AEROF_EINVAL;
    }
    const DeviceMesh& m = c->mesh;
    std::vector<double> d(m.N);
    if (is_device_ptr(d2wall))
      AEROF_CUDA(cudaMemcpy(d.data(), d2wall, sizeof(double) * m.N, cudaMemcpyDeviceToHost));
    else
      std::copy(d2wall, d2wall + m.N, d.begin());
    for (double x : d)
      if (!(x >= 0.0) || !std::isfinite(x)) {
        c->last_error = "wall distances must be finite and non-negative";
        return AEROF_EINVAL;
      }
    t.p = *p;
    for (int k = 0; k < 6; ++k) t.Ub[k] = Ub[k];
    t.Ubd.upload(t.Ub, 6, c->stream);
    t.d2wall.upload(d.data(), d.size(), c->stream);
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    t.on = true;
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_residual_sa(aerof_gpu_ctx* c, const double* U, double* R) {
  return guard(c, [&]() -> int {
    if (!c->has_mesh) {
      c->last_error = "no mesh: call aerof_gpu_set_mesh first";
      return AEROF_ESTATE;
    }
    if (!c->turb.on) {
      c->last_error = "the Spalart-Allmaras model is off: call aerof_gpu_set_turbulence first";
      return AEROF_ESTATE;
    }
    if (!U || !R) return AEROF_EINVAL;
    const size_t n6 = 6 * (size_t)c->mesh.N;
    const double* dU = in_dev(c, U, n6, c->turb.Ustage);
    double* dR = out_dev(c, R, n6, c->turb.Rstage);
    const int bad = residual_sa_dev(c, dU, dR);
    out_finish(c, R, dR, n6);
    return bad;
  });
}
