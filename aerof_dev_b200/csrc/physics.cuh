// physics.cuh -- pointwise device functions of the Euler finite-volume path.
//
// Each function states the reference routine whose arithmetic it keeps
// (file:line in the AERO-F tree).  They are templated on the scalar type so
// the same source yields the primal kernels (double) and the exact
// forward-mode linearisation (Dual, adjoint.cu).
#pragma once

#include <cuda_runtime.h>

namespace aerof {

#define AEROF_HD __host__ __device__ __forceinline__

// ------------------------------------------------------------ dual numbers
struct Dual {
  double v, d;
  AEROF_HD Dual() : v(0), d(0) {}
  AEROF_HD Dual(double a) : v(a), d(0) {}
  AEROF_HD Dual(double a, double b) : v(a), d(b) {}
};
AEROF_HD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
AEROF_HD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
AEROF_HD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
AEROF_HD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
AEROF_HD Dual operator/(Dual a, Dual b) {
  double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
AEROF_HD Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
AEROF_HD Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
AEROF_HD Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }
AEROF_HD Dual dsqrt(Dual a) { double s = sqrt(a.v); return Dual(s, a.d / (2.0 * s)); }
AEROF_HD double dsqrt(double a) { return sqrt(a); }
AEROF_HD double vof(double a) { return a; }
AEROF_HD double vof(Dual a) { return a.v; }
template <class T> AEROF_HD T tmax0(T a) { return vof(a) < 0.0 ? T(0.0) : a; }
template <class T> AEROF_HD T tmin0(T a) { return vof(a) > 0.0 ? T(0.0) : a; }
template <class T> AEROF_HD T tabs(T a) { return vof(a) < 0.0 ? -a : a; }

// ------------------------------------------------------------ fast reciprocals
// Reciprocal and reciprocal square root for the primal double kernels: the
// hardware approximation (PTX rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64,
// about 23 correct bits) refined by Newton-Raphson iteration.  For 1/x:
// with e = 1 - x r, 1/x = r / (1 - e) = r (1 + e + e^2 + ...), and the step
// r <- r + r (e + e^2) keeps the series to second order, a third-order
// iteration (one step takes 23 correct bits past double precision); this is
// the series-expansion refinement of division described by Markstein
// ("IA-64 and Elementary Functions", 2000) and by Ercegovac and Lang
// ("Digital Arithmetic", 2004).  For 1/sqrt x: Newton's iteration on
// f(y) = y^-2 - x, y <- y + y/2 (1 - x y^2), twice.  Inputs are positive
// normal numbers (densities, pressures, squared norms, positive
// denominators).  tests/test_gpu_fastmath.py bounds the error against the
// correctly rounded values: at most 1 ulp (1/x) and 2 ulp (1/sqrt x) over a
// sweep of inputs.  The dual-number instantiation keeps exact division and
// square root.
AEROF_HD double rcp_(double x) {
#ifdef __CUDA_ARCH__
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  const double e = fma(-x, r, 1.0);
  return fma(r, fma(e, e, e), r);
#else
  return 1.0 / x;
#endif
}
AEROF_HD double rsqrt_(double x) {
#ifdef __CUDA_ARCH__
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x * y, y, 1.0);
  y = fma(0.5 * y, e, y);
  e = fma(-x * y, y, 1.0);
  return fma(0.5 * y, e, y);
#else
  return 1.0 / sqrt(x);
#endif
}
AEROF_HD Dual rcp_(Dual x) { return 1.0 / x; }
AEROF_HD Dual rsqrt_(Dual x) { return 1.0 / dsqrt(x); }
template <class T> AEROF_HD T sel(bool c, T a, T b) { return c ? a : b; }

// ------------------------------------------------------------ gas model
struct Gas {
  double gam, gam1, invgam1;
};
AEROF_HD Gas make_gas(double gam) {
  Gas g;
  g.gam = gam;
  g.gam1 = gam - 1.0;
  g.invgam1 = 1.0 / g.gam1;
  return g;
}

// VarFcnSGEuler::conservativeToPrimitive (VarFcnSGEuler.h:307-327), Pstiff=0
template <class T>
AEROF_HD void cons2prim(const Gas& g, const T* U, T* V) {
  V[0] = U[0];
  T invRho = 1.0 / U[0];
  V[1] = U[1] * invRho;
  V[2] = U[2] * invRho;
  V[3] = U[3] * invRho;
  T vel2 = V[1] * V[1] + V[2] * V[2] + V[3] * V[3];
  V[4] = g.gam1 * (U[4] - 0.5 * U[0] * vel2);
}

// ------------------------------------------------------------ least squares
// Per-node constants of computeLocalWeightsLeastSquares (SubDomain.C:137-159):
// they depend on R_i only, so they are formed once per mesh:
// w = (or11, or22, or33, r12or11, r23or22, psi).
AEROF_HD void lsq_node_constants(const double* R, double* w) {
  double or11 = 1.0 / R[0];
  double or22 = 1.0 / R[3];
  double or33 = 1.0 / R[5];
  w[0] = or11;
  w[1] = or22;
  w[2] = or33;
  w[3] = R[1] * or11;
  w[4] = R[4] * or22;
  w[5] = (R[1] * R[4] - R[2] * R[3]) * or11 * or22;
}
// W(dx) from the per-node constants (same operations as the reference).
template <class T>
AEROF_HD void lsq_weights(const T* w, T dx0, T dx1, T dx2, T& W0, T& W1, T& W2) {
  T alpha1 = dx0 * w[0] * w[0];
  T alpha2 = (dx1 - w[3] * dx0) * w[1] * w[1];
  T alpha3 = (dx2 - w[4] * dx1 + w[5] * dx0) * w[2] * w[2];
  W0 = alpha1 - w[3] * alpha2 + w[5] * alpha3;
  W1 = alpha2 - w[4] * alpha3;
  W2 = alpha3;
}

// ------------------------------------------------------------ reconstruction
// RecFcn::computeVanAlbadaFcn (RecFcn.h:268-281).  For a*b > 0 the
// numerator a(b^2+eps) + b(a^2+eps) equals (a+b)(ab+eps); for a*b == 0 the
// reference's 0.5 eps (a+b) is the same expression with ab+eps replaced by
// eps/2; otherwise the result is 0.  One reciprocal of the denominator,
// branch-free selection.
template <class T>
AEROF_HD T vanalbada_fcn(T a, T b) {
  const double eps = 1.e-16;
  T ab = a * b;
  const double abv = vof(ab);
  T den = a * a + (b * b + 2.0 * eps);
  T t = sel(abv > 0.0, ab + eps, sel(abv == 0.0, T(0.5 * eps), T(0.0)));
  return (a + b) * t * rcp_(den);
}
// RecFcn::vanalbada (RecFcn.h:432-446); beta2 = 1-2 beta
template <class T>
AEROF_HD void vanalbada(double beta, T Vi, T ddVij, T Vj, T ddVji, T& Vij, T& Vji) {
  const double beta2 = 1.0 - 2.0 * beta;
  T dVji = Vj - Vi;
  T dV = beta2 * dVji;
  T dVi = dV + 2.0 * beta * ddVij;
  T dVj = dV + 2.0 * beta * ddVji;
  Vij = Vi + 0.5 * vanalbada_fcn(dVi, dVji);
  Vji = Vj - 0.5 * vanalbada_fcn(dVj, dVji);
}
// RecFcn::linear (RecFcn.h:240-249); beta1 = 1/2 - beta
template <class T>
AEROF_HD void linear_rec(double beta, T Vi, T ddVij, T Vj, T ddVji, T& Vij, T& Vji) {
  const double beta1 = 0.5 - beta;
  T dV = beta1 * (Vj - Vi);
  Vij = Vi + dV + beta * ddVij;
  Vji = Vj - dV - beta * ddVji;
}

// ------------------------------------------------------------ fluxes
// roeflux7.f:1-202 (type 0, pstiff = 0, static mesh vitno = 0): Roe-averaged
// upwind selection of the physical flux plus the one-wave dissipation term.
template <class T>
AEROF_HD void roe_flux(const Gas& g, T n0, T n1, T n2, const T* Ug, const T* Ud, T* phi) {
  const double gam1 = g.gam1, invgam1 = g.invgam1, gog1 = g.gam * g.invgam1;
  T s2 = n0 * n0 + n1 * n1 + n2 * n2;
  T invnorm = rsqrt_(s2);
  T rnorm = s2 * invnorm;
  T nx = n0 * invnorm, ny = n1 * invnorm, nz = n2 * invnorm;
  T vitg2 = Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3];
  T vitd2 = Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3];
  // sqrt(rho) and 1/sqrt(rho) of both sides
  T rs1 = rsqrt_(Ug[0]), rs2 = rsqrt_(Ud[0]);
  T squsr1 = Ug[0] * rs1;
  T squsr2 = Ud[0] * rs2;
  T ener1 = Ug[4] * invgam1 + 0.5 * Ug[0] * vitg2;
  T ener2 = Ud[4] * invgam1 + 0.5 * Ud[0] * vitd2;
  T usro = rcp_(squsr1 + squsr2);
  T uar2 = (squsr1 * Ug[1] + squsr2 * Ud[1]) * usro;
  T uar3 = (squsr1 * Ug[2] + squsr2 * Ud[2]) * usro;
  T uar4 = (squsr1 * Ug[3] + squsr2 * Ud[3]) * usro;
  T uar5 = ((ener1 + Ug[4]) * rs1 + (ener2 + Ud[4]) * rs2) * usro;
  T VdotN = nx * uar2 + ny * uar3 + nz * uar4;
  const bool left = vof(VdotN) > 0.0;
  // centred flux of the upwind side (roeflux7.f:79-98):
  // H = (gam p + 0.5 gam1 rho |u|^2) / (gam1 rho) = gam/gam1 p/rho + |u|^2/2
  T Us0 = sel(left, Ug[0], Ud[0]), Us1 = sel(left, Ug[1], Ud[1]), Us2 = sel(left, Ug[2], Ud[2]);
  T Us3 = sel(left, Ug[3], Ud[3]), Us4 = sel(left, Ug[4], Ud[4]);
  T rss = sel(left, rs1, rs2);
  T vits2 = sel(left, vitg2, vitd2);
  T vn = Us1 * nx + Us2 * ny + Us3 * nz;
  T H = gog1 * Us4 * (rss * rss) + 0.5 * vits2;
  T f0 = Us0 * vn;
  T f1 = f0 * Us1 + Us4 * nx;
  T f2 = f0 * Us2 + Us4 * ny;
  T f3 = f0 * Us3 + Us4 * nz;
  T f4 = f0 * H;
  // one-wave dissipation (roeflux7.f:107-181) with cr2byt = -cr,
  // invtbeta2 = -1/cr: flur4 = max(VdotN+cr,0) (-cr A + gam1 B) when the
  // right side is upwind, flur5 = max(cr-VdotN,0) (cr A + gam1 B) otherwise.
  T qir = 0.5 * (uar2 * uar2 + uar3 * uar3 + uar4 * uar4);
  T c2 = gam1 * (uar5 - qir);
  T rc = rsqrt_(c2);
  T cr = c2 * rc;
  T cr2 = rc * rc;
  T dif1 = Ud[0] - Ug[0];
  T dif2 = Ud[0] * Ud[1] - Ug[0] * Ug[1];
  T dif3 = Ud[0] * Ud[2] - Ug[0] * Ug[2];
  T dif4 = Ud[0] * Ud[3] - Ug[0] * Ug[3];
  T dif5 = ener2 - ener1;
  T A = VdotN * dif1 - nx * dif2 - ny * dif3 - nz * dif4;
  T B = qir * dif1 - uar2 * dif2 - uar3 * dif3 - uar4 * dif4 + dif5;
  T scr = sel(left, cr, -cr);
  T fl = tmax0(cr - (left ? VdotN : -VdotN)) * (scr * A + gam1 * B);
  T rs = -scr * fl;
  T hc = 0.5 * cr2;
  phi[0] = (f0 - hc * fl) * rnorm;
  phi[1] = (f1 - (nx * rs + uar2 * fl) * hc) * rnorm;
  phi[2] = (f2 - (ny * rs + uar3 * fl) * hc) * rnorm;
  phi[3] = (f3 - (nz * rs + uar4 * fl) * hc) * rnorm;
  phi[4] = (f4 - (VdotN * rs + uar5 * fl) * hc) * rnorm;
}

// boundflux5.f:1-111 (type 0, sig = 0): Steger-Warming far-field flux
// A+(V) U(V) + A-(V) Ub with V primitive and Ub conservative.
template <class T>
AEROF_HD void sw_flux(const Gas& g, T vnx, T vny, T vnz, const T* ua, const double* ub, T* flux) {
  const double gam = g.gam, gam1 = g.gam1;
  T cap = dsqrt(vnx * vnx + vny * vny + vnz * vnz);
  T capd1 = vnx / cap, capd2 = vny / cap, capd3 = vnz / cap;
  T ro = ua[0];
  T usro = 1.0 / ro;
  T u = ua[1], v = ua[2], w = ua[3];
  T vit = u * u + v * v + w * w;
  T pm = ua[4];
  T rhoE = pm / gam1 + 0.5 * ro * vit;
  T c2 = gam * pm * usro;
  T c = dsqrt(c2);
  T usc = 1.0 / c;
  T cc = 0.5 * vit + c2 / gam1;
  T unx = capd1 * u + capd2 * v + capd3 * w;
  T l1 = cap * unx, l4 = cap * (unx + c), l5 = cap * (unx - c);
  T vp1 = tmax0(l1), vp4 = tmax0(l4), vp5 = tmax0(l5);
  T vpp = vp4 + vp5;
  T vpm = vp4 - vp5;
  T fgp0 = (gam1 * ro * vp1 + 0.5 * ro * vpp) / gam;
  T fgp1 = fgp0 * u + 0.5 * pm * usc * capd1 * vpm;
  T fgp2 = fgp0 * v + 0.5 * pm * usc * capd2 * vpm;
  T fgp3 = fgp0 * w + 0.5 * pm * usc * capd3 * vpm;
  T fgp4 = 0.5 * ((gam1 / gam) * ro * vit * (vp1 - 0.5 * vpp) + rhoE * vpp + ro * unx * c * vpm / gam);
  vp1 = tmin0(l1); vp4 = tmin0(l4); vp5 = tmin0(l5);
  vpp = vp1 - 0.5 * (vp4 + vp5);
  vpm = 0.5 * (vp5 - vp4);
  T xn1 = gam1 * usc * (-(0.5 * vit * ub[0]) + u * ub[1] + v * ub[2] + w * ub[3] - ub[4]);
  T xn2 = unx * ub[0] - capd1 * ub[1] - capd2 * ub[2] - capd3 * ub[3];
  T ff = usc * (vpp * xn1 + vpm * xn2);
  T gg = vpm * xn1 + vpp * xn2;
  flux[0] = fgp0 + (vp1 * ub[0] + ff);
  flux[1] = fgp1 + (vp1 * ub[1] + u * ff + capd1 * gg);
  flux[2] = fgp2 + (vp1 * ub[2] + v * ff + capd2 * gg);
  flux[3] = fgp3 + (vp1 * ub[3] + w * ff + capd3 * gg);
  flux[4] = fgp4 + (vp1 * ub[4] + cc * ff + unx * gg);
}

// FluxFcnSGWallEuler3D::compute (FluxFcnDescSG.C:779-789), ndot = 0
template <class T>
AEROF_HD void wall_flux(T nx, T ny, T nz, const T* V, T* flux) {
  flux[0] = T(0.0);
  flux[1] = V[4] * nx;
  flux[2] = V[4] * ny;
  flux[3] = V[4] * nz;
  flux[4] = T(0.0);
}

template <class T>
AEROF_HD void face_flux(const Gas& g, int code, T nx, T ny, T nz, const T* V, const double* Ub, T* f) {
  if (code == AEROF_BC_SLIP_WALL_MOVING) wall_flux(nx, ny, nz, V, f);
  else sw_flux(g, nx, ny, nz, V, Ub, f);
}

// ------------------------------------------------------------ Jacobians
// VarFcnBase::postMultiplyBydVdU (VarFcnBase.h:372-400) with
// VarFcnSGEuler::computedVdU (VarFcnSGEuler.h:588-603): res = mat * dV/dU.
AEROF_HD void post_dVdU(const Gas& g, const double* V, const double* mat, double* res) {
  double invrho = 1.0 / V[0];
  double d5 = -invrho * V[1], d10 = -invrho * V[2], d15 = -invrho * V[3];
  double d20 = g.gam1 * 0.5 * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]);
  double d21 = -g.gam1 * V[1], d22 = -g.gam1 * V[2], d23 = -g.gam1 * V[3], d24 = g.gam1;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    const double* m = mat + 5 * r;
    double* o = res + 5 * r;
    o[0] = m[0] + m[1] * d5 + m[2] * d10 + m[3] * d15 + m[4] * d20;
    o[1] = m[1] * invrho + m[4] * d21;
    o[2] = m[2] * invrho + m[4] * d22;
    o[3] = m[3] * invrho + m[4] * d23;
    o[4] = m[4] * d24;
  }
}

// roejac6.f:1-316 (type 0, prec 0 -> beta 1, dissipation coefficient 1):
// approximate Jacobian of the Roe flux w.r.t. the conservative state Ug,
// sw = +1 adds the dissipation matrix, sw = -1 subtracts it.
//
// Convective part of roejac6: the exact flux Jacobian H(U) of state U along
// the unit normal n (roejac6.f, first block).
AEROF_HD void roe_jac_H(const Gas& g, const double* n, const double* Ug, double* H) {
  const double gam = g.gam, gam1 = g.gam1;
  const double VdotN = Ug[1] * n[0] + Ug[2] * n[1] + Ug[3] * n[2];
  const double qir = 0.5 * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]);
  const double enth = (gam * Ug[4] + gam1 * Ug[0] * qir) / (gam1 * Ug[0]);
  H[0] = 0.0; H[1] = n[0]; H[2] = n[1]; H[3] = n[2]; H[4] = 0.0;
  H[5] = gam1 * n[0] * qir - Ug[1] * VdotN;
  H[6] = (1.0 - gam1) * n[0] * Ug[1] + VdotN;
  H[7] = -gam1 * n[0] * Ug[2] + Ug[1] * n[1];
  H[8] = -gam1 * n[0] * Ug[3] + Ug[1] * n[2];
  H[9] = gam1 * n[0];
  H[10] = gam1 * n[1] * qir - Ug[2] * VdotN;
  H[11] = -gam1 * n[1] * Ug[1] + Ug[2] * n[0];
  H[12] = (1.0 - gam1) * n[1] * Ug[2] + VdotN;
  H[13] = -gam1 * n[1] * Ug[3] + Ug[2] * n[2];
  H[14] = gam1 * n[1];
  H[15] = gam1 * n[2] * qir - Ug[3] * VdotN;
  H[16] = -gam1 * n[2] * Ug[1] + Ug[3] * n[0];
  H[17] = -gam1 * n[2] * Ug[2] + Ug[3] * n[1];
  H[18] = (1.0 - gam1) * n[2] * Ug[3] + VdotN;
  H[19] = gam1 * n[2];
  H[20] = (gam1 * qir - enth) * VdotN;
  H[21] = enth * n[0] - gam1 * Ug[1] * VdotN;
  H[22] = enth * n[1] - gam1 * Ug[2] * VdotN;
  H[23] = enth * n[2] - gam1 * Ug[3] * VdotN;
  H[24] = (1.0 + gam1) * VdotN;
}

// Dissipation part of roejac6: |A| at the Roe average of the two states,
// written through its eigenvectors (roejac6.f, second block).  The Roe
// average is symmetric in (Ug, Ud), bit for bit (every sum of the two sides
// is a commutative two-term addition), so one D serves both endpoints.
// RoeAvg holds the scalars of the average; tmw_elem and D_col form the
// eigenvector matrix and D one column at a time, so a caller can stream
// the 5x5 blocks without holding 25-element arrays.
template <class T = double>
struct RoeAvg {
  T uar2, uar3, uar4, enth, VdotN, qir, crsq, gc, usc2, rRT, sRT, tRT, vp1, vp4, vp5;
};
// a*b + c*d with both products rounded (no fused multiply-add), so the
// result does not depend on which pair is named first
AEROF_HD double sym_dot2(double a, double b, double c, double d) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b) + __dmul_rn(c, d);
#else
  return a * b + c * d;
#endif
}
AEROF_HD float sym_dot2(float a, float b, float c, float d) {
#ifdef __CUDA_ARCH__
  return __fmul_rn(a, b) + __fmul_rn(c, d);
#else
  return a * b + c * d;
#endif
}

// T = double: the reference arithmetic; T = float: the same formulas in
// FP32, for the FP32-stored Jacobian of the mixed-precision solver.  The
// Roe average is formed symmetrically in (Ug, Ud) (sym_dot2), so the two
// rows of an edge obtain the same dissipation matrix bit for bit.
template <class T = double>
AEROF_HD RoeAvg<T> roe_avg(const Gas& g, const T* n, const T* Ug, const T* Ud) {
  const T gam1 = (T)g.gam1;
  RoeAvg<T> A;
  T squsr1 = sqrt(Ug[0]), squsr2 = sqrt(Ud[0]);
  T ener1 = Ug[4] / gam1 + T(0.5) * Ug[0] * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]);
  T ener2 = Ud[4] / gam1 + T(0.5) * Ud[0] * (Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3]);
  T usro = T(1.0) / (squsr1 + squsr2);
  A.uar2 = sym_dot2(squsr1, Ug[1], squsr2, Ud[1]) * usro;
  A.uar3 = sym_dot2(squsr1, Ug[2], squsr2, Ud[2]) * usro;
  A.uar4 = sym_dot2(squsr1, Ug[3], squsr2, Ud[3]) * usro;
  T uar5 = ((ener1 + Ug[4]) / squsr1 + (ener2 + Ud[4]) / squsr2) * usro;
  A.enth = uar5;
  A.VdotN = n[0] * A.uar2 + n[1] * A.uar3 + n[2] * A.uar4;
  A.qir = T(0.5) * (A.uar2 * A.uar2 + A.uar3 * A.uar3 + A.uar4 * A.uar4);
  T cr = sqrt(gam1 * (uar5 - A.qir));
  A.crsq = cr * cr;
  A.gc = gam1 / A.crsq;
  A.usc2 = T(0.5) / A.crsq;
  // beta = 1: vp4,vp5 = VdotN +- cr written as the reference's general form
  T sq = sqrt(T(0.0) * A.VdotN * (T(0.0) * A.VdotN) + T(4.0) * A.crsq);
  T vp4 = T(0.5) * (T(2.0) * A.VdotN + sq);
  T vp5 = T(0.5) * (T(2.0) * A.VdotN - sq);
  A.rRT = vp4 - A.VdotN;
  A.sRT = vp5 - A.VdotN;
  A.tRT = T(0.5) * (vp5 - vp4);
  A.vp1 = fabs(A.VdotN);
  A.vp4 = fabs(vp4);
  A.vp5 = fabs(vp5);
  return A;
}
// element e (row-major) of the left eigenvector matrix tmw
template <class T = double>
AEROF_HD T tmw_elem(const Gas& g, const RoeAvg<T>& A, const T* n, int e) {
  const T gam1 = (T)g.gam1;
  switch (e) {
    case 0: return n[0] + n[1] * A.uar4 - A.uar3 * n[2] - A.gc * n[0] * A.qir;
    case 1: return A.gc * n[0] * A.uar2;
    case 2: return A.gc * n[0] * A.uar3 + n[2];
    case 3: return A.gc * n[0] * A.uar4 - n[1];
    case 4: return -A.gc * n[0];
    case 5: return n[1] + n[2] * A.uar2 - A.uar4 * n[0] - A.gc * n[1] * A.qir;
    case 6: return A.gc * n[1] * A.uar2 - n[2];
    case 7: return A.gc * n[1] * A.uar3;
    case 8: return A.gc * n[1] * A.uar4 + n[0];
    case 9: return -A.gc * n[1];
    case 10: return n[2] + n[0] * A.uar3 - A.uar2 * n[1] - A.gc * n[2] * A.qir;
    case 11: return A.gc * n[2] * A.uar2 + n[1];
    case 12: return A.gc * n[2] * A.uar3 - n[0];
    case 13: return A.gc * n[2] * A.uar4;
    case 14: return -A.gc * n[2];
    case 15: return gam1 * A.qir * A.sRT / A.tRT + A.VdotN * A.crsq / A.tRT;
    case 16: return -gam1 * A.uar2 * A.sRT / A.tRT - A.crsq * n[0] / A.tRT;
    case 17: return -gam1 * A.uar3 * A.sRT / A.tRT - A.crsq * n[1] / A.tRT;
    case 18: return -gam1 * A.uar4 * A.sRT / A.tRT - A.crsq * n[2] / A.tRT;
    case 19: return gam1 * A.sRT / A.tRT;
    case 20: return -gam1 * A.qir * A.rRT / A.tRT - A.VdotN * A.crsq / A.tRT;
    case 21: return gam1 * A.uar2 * A.rRT / A.tRT + A.crsq * n[0] / A.tRT;
    case 22: return gam1 * A.uar3 * A.rRT / A.tRT + A.crsq * n[1] / A.tRT;
    case 23: return gam1 * A.uar4 * A.rRT / A.tRT + A.crsq * n[2] / A.tRT;
    default: return -gam1 * A.rRT / A.tRT;
  }
}
// column j of D: d[m] = D[5 m + j]
template <class T = double>
AEROF_HD void D_col(const Gas& g, const RoeAvg<T>& A, const T* n, int j, T* d) {
  const T t0 = tmw_elem(g, A, n, j), t1 = tmw_elem(g, A, n, 5 + j), t2 = tmw_elem(g, A, n, 10 + j);
  const T t3 = tmw_elem(g, A, n, 15 + j), t4 = tmw_elem(g, A, n, 20 + j);
  const T uar2 = A.uar2, uar3 = A.uar3, uar4 = A.uar4, qir = A.qir, usc2 = A.usc2, rRT = A.rRT, sRT = A.sRT;
  const T vp1 = A.vp1, vp4 = A.vp4, vp5 = A.vp5, enth = A.enth, VdotN = A.VdotN;
  d[0] = vp1 * (n[0] * t0 + n[1] * t1 + n[2] * t2) + vp4 * usc2 * t3 + vp5 * usc2 * t4;
  d[1] = vp1 * (n[0] * uar2 * t0 + (n[1] * uar2 - n[2]) * t1 + (n[2] * uar2 + n[1]) * t2) +
         vp4 * (usc2 * (uar2 + rRT * n[0])) * t3 + vp5 * (usc2 * (uar2 + sRT * n[0])) * t4;
  d[2] = vp1 * (n[1] * uar3 * t1 + (n[0] * uar3 + n[2]) * t0 + (n[2] * uar3 - n[0]) * t2) +
         vp4 * (usc2 * (uar3 + rRT * n[1])) * t3 + vp5 * (usc2 * (uar3 + sRT * n[1])) * t4;
  d[3] = vp1 * (n[2] * uar4 * t2 + (n[0] * uar4 - n[1]) * t0 + (n[1] * uar4 + n[0]) * t1) +
         vp4 * (usc2 * (uar4 + rRT * n[2])) * t3 + vp5 * (usc2 * (uar4 + sRT * n[2])) * t4;
  d[4] = vp1 * ((n[0] * qir + (n[2] * uar3 - n[1] * uar4)) * t0 + (n[1] * qir + (n[0] * uar4 - n[2] * uar2)) * t1 +
                (n[2] * qir + (n[1] * uar2 - n[0] * uar3)) * t2) +
         vp4 * (usc2 * (enth + VdotN * rRT)) * t3 + vp5 * (usc2 * (enth + VdotN * sRT)) * t4;
}
AEROF_HD void roe_jac_D(const Gas& g, const double* n, const double* Ug, const double* Ud, double* D) {
  const RoeAvg<double> A = roe_avg(g, n, Ug, Ud);
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    double d[5];
    D_col(g, A, n, j, d);
#pragma unroll
    for (int m = 0; m < 5; ++m) D[5 * m + j] = d[m];
  }
}

// Scalars of the convective Jacobian H(U) (see roe_jac_H) and its element
// e (row-major), for streaming use.
template <class T = double>
struct HState {
  T U1, U2, U3, VdotN, qir, enth;
};
template <class T = double>
AEROF_HD HState<T> h_state(const Gas& g, const T* n, const T* Ug) {
  HState<T> h;
  h.U1 = Ug[1]; h.U2 = Ug[2]; h.U3 = Ug[3];
  h.VdotN = Ug[1] * n[0] + Ug[2] * n[1] + Ug[3] * n[2];
  h.qir = T(0.5) * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]);
  h.enth = ((T)g.gam * Ug[4] + (T)g.gam1 * Ug[0] * h.qir) / ((T)g.gam1 * Ug[0]);
  return h;
}
template <class T = double>
AEROF_HD T H_elem(const Gas& g, const HState<T>& h, const T* n, int e) {
  const T gam1 = (T)g.gam1;
  switch (e) {
    case 0: return T(0.0);
    case 1: return n[0];
    case 2: return n[1];
    case 3: return n[2];
    case 4: return T(0.0);
    case 5: return gam1 * n[0] * h.qir - h.U1 * h.VdotN;
    case 6: return (T(1.0) - gam1) * n[0] * h.U1 + h.VdotN;
    case 7: return -gam1 * n[0] * h.U2 + h.U1 * n[1];
    case 8: return -gam1 * n[0] * h.U3 + h.U1 * n[2];
    case 9: return gam1 * n[0];
    case 10: return gam1 * n[1] * h.qir - h.U2 * h.VdotN;
    case 11: return -gam1 * n[1] * h.U1 + h.U2 * n[0];
    case 12: return (T(1.0) - gam1) * n[1] * h.U2 + h.VdotN;
    case 13: return -gam1 * n[1] * h.U3 + h.U2 * n[2];
    case 14: return gam1 * n[1];
    case 15: return gam1 * n[2] * h.qir - h.U3 * h.VdotN;
    case 16: return -gam1 * n[2] * h.U1 + h.U3 * n[0];
    case 17: return -gam1 * n[2] * h.U2 + h.U3 * n[1];
    case 18: return (T(1.0) - gam1) * n[2] * h.U3 + h.VdotN;
    case 19: return gam1 * n[2];
    case 20: return (gam1 * h.qir - h.enth) * h.VdotN;
    case 21: return h.enth * n[0] - gam1 * h.U1 * h.VdotN;
    case 22: return h.enth * n[1] - gam1 * h.U2 * h.VdotN;
    case 23: return h.enth * n[2] - gam1 * h.U3 * h.VdotN;
    default: return (T(1.0) + gam1) * h.VdotN;
  }
}

// jac = (H(Ug) + sw |A|_Roe) |n| / 2: the derivative of the Roe flux with
// respect to the first state (sw = +1) or, called with the states swapped,
// the second (sw = -1).
AEROF_HD void roe_jac(const Gas& g, double n0, double n1, double n2, const double* Ug, const double* Ud,
                      double sw, double* jac) {
  double rnorm = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  double invnorm = 1.0 / rnorm;
  double n[3] = {n0 * invnorm, n1 * invnorm, n2 * invnorm};
  double H[25], D[25];
  roe_jac_H(g, n, Ug, H);
  roe_jac_D(g, n, Ug, Ud, D);
  const double half_rn = 0.5 * rnorm;
#pragma unroll
  for (int k = 0; k < 25; ++k) jac[k] = (H[k] + sw * D[k]) * half_rn;
}

// Face blocks: FluxFcnFD<5>::computeJacobian (FluxFcnBase.h:112-159) for the
// Steger-Warming faces, FluxFcnSGWallEuler3D::computeJacobian
// (FluxFcnDescSG.C:838-886) for slip walls, both post-multiplied by dV/dU.
AEROF_HD void face_jac(const Gas& g, int code, double nx, double ny, double nz, const double* V,
                       const double* Ub, double* jac) {
  double dfdV[25];
  if (code == AEROF_BC_SLIP_WALL_MOVING) {
#pragma unroll
    for (int k = 0; k < 25; ++k) dfdV[k] = 0.0;
    dfdV[9] = nx; dfdV[14] = ny; dfdV[19] = nz; dfdV[24] = 0.0;
  } else {
    const double eps0 = 1.e-6;
    double f0[5], fe[5], Ve[5];
    sw_flux(g, nx, ny, nz, V, Ub, f0);
    for (int k = 0; k < 5; ++k) {
#pragma unroll
      for (int q = 0; q < 5; ++q) Ve[q] = V[q];
      double eps = (fabs(V[k]) < 1.e-10) ? eps0 : eps0 * V[k];
      double inveps = 1.0 / eps;
      Ve[k] += eps;
      sw_flux(g, nx, ny, nz, Ve, Ub, fe);
#pragma unroll
      for (int j = 0; j < 5; ++j) dfdV[5 * j + k] = (fe[j] - f0[j]) * inveps;
    }
  }
  post_dVdU(g, V, dfdV, jac);
}

// ------------------------------------------------------------ 5x5 inverse
// invertDenseMatrix (DenseMatrixOps.h:1006-1185): LINPACK dgefa (partial
// pivoting) + dgedi, here on a row-major block viewed as column-major
// transpose.  Returns 0 or the 1-based step with a zero pivot.
template <class S>
AEROF_HD int invert5(S* a) {
  // t(r,c) = a[c*5 + r] : the transpose in column-major is a itself read
  // row-major, so operate on a directly with A(r,c) = a[r + 5*c]^T ...
  S t[25];
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) t[r + 5 * c] = a[5 * r + c];
#define AEROF_A(r, c) t[(r) + 5 * (c)]
  int ipvt[5];
  for (int k = 0; k < 4; ++k) {
    int l = k;
    S mx = AEROF_A(k, k) < S(0) ? -AEROF_A(k, k) : AEROF_A(k, k);
    for (int r = k + 1; r < 5; ++r) {
      S v = AEROF_A(r, k) < S(0) ? -AEROF_A(r, k) : AEROF_A(r, k);
      if (v > mx) { mx = v; l = r; }
    }
    ipvt[k] = l;
    if (AEROF_A(l, k) == S(0)) return k + 1;
    if (l != k) { S tmp = AEROF_A(l, k); AEROF_A(l, k) = AEROF_A(k, k); AEROF_A(k, k) = tmp; }
    S tt = S(-1.0) / AEROF_A(k, k);
    for (int r = k + 1; r < 5; ++r) AEROF_A(r, k) *= tt;
    for (int j = k + 1; j < 5; ++j) {
      S u = AEROF_A(l, j);
      if (l != k) { AEROF_A(l, j) = AEROF_A(k, j); AEROF_A(k, j) = u; }
      for (int r = k + 1; r < 5; ++r) AEROF_A(r, j) += u * AEROF_A(r, k);
    }
  }
  ipvt[4] = 4;
  if (AEROF_A(4, 4) == S(0)) return 5;
  for (int k = 0; k < 5; ++k) {
    AEROF_A(k, k) = S(1.0) / AEROF_A(k, k);
    S tt = -AEROF_A(k, k);
    for (int r = 0; r < k; ++r) AEROF_A(r, k) *= tt;
    for (int j = k + 1; j < 5; ++j) {
      S u = AEROF_A(k, j);
      AEROF_A(k, j) = S(0);
      for (int r = 0; r <= k; ++r) AEROF_A(r, j) += u * AEROF_A(r, k);
    }
  }
  S work[5];
  for (int kb = 1; kb <= 4; ++kb) {
    int k = 4 - kb;
    for (int i = k + 1; i < 5; ++i) { work[i] = AEROF_A(i, k); AEROF_A(i, k) = S(0); }
    for (int j = k + 1; j < 5; ++j) {
      S u = work[j];
      for (int r = 0; r < 5; ++r) AEROF_A(r, k) += u * AEROF_A(r, j);
    }
    int l = ipvt[k];
    if (l != k)
      for (int r = 0; r < 5; ++r) { S tmp = AEROF_A(r, k); AEROF_A(r, k) = AEROF_A(r, l); AEROF_A(r, l) = tmp; }
  }
#undef AEROF_A
#pragma unroll
  for (int r = 0; r < 5; ++r)
#pragma unroll
    for (int c = 0; c < 5; ++c) a[5 * r + c] = t[r + 5 * c];
  return 0;
}

}  // namespace aerof

namespace aerof {

// ------------------------------------------------------------ adjoints
// Reverse mode of roe_flux: recomputes the forward values, then
// accumulates the cotangents gUg += (dphi/dUg)^T gphi, gUd += (dphi/dUd)^T
// gphi and gn += (dphi/dn)^T gphi.  The dissipation term is differentiated
// in its algebraically simplified form fl = lam (s cr A + gam1 B), s = -1
// (right side upwind) or +1 (left side), which is the same function as the
// reference's cr2byt / invtbeta2 form.
__device__ __forceinline__ void roe_flux_adj(const Gas& g, double n0, double n1, double n2, const double* Ug,
                                             const double* Ud, const double* gphi, double* gUg, double* gUd,
                                             double* gn) {
  const double gam = g.gam, gam1 = g.gam1, invgam1 = g.invgam1;
  // ---- forward
  const double s2 = n0 * n0 + n1 * n1 + n2 * n2;
  const double rnorm = sqrt(s2);
  const double invnorm = 1.0 / rnorm;
  const double nx = n0 * invnorm, ny = n1 * invnorm, nz = n2 * invnorm;
  const double vitg2 = Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3];
  const double vitd2 = Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3];
  const double sq1 = sqrt(Ug[0]), sq2 = sqrt(Ud[0]);
  const double ener1 = Ug[4] * invgam1 + 0.5 * Ug[0] * vitg2;
  const double ener2 = Ud[4] * invgam1 + 0.5 * Ud[0] * vitd2;
  const double usro = 1.0 / (sq1 + sq2);
  const double m2 = sq1 * Ug[1] + sq2 * Ud[1], m3 = sq1 * Ug[2] + sq2 * Ud[2], m4 = sq1 * Ug[3] + sq2 * Ud[3];
  const double uar2 = m2 * usro, uar3 = m3 * usro, uar4 = m4 * usro;
  const double a1 = (ener1 + Ug[4]) / sq1, a2 = (ener2 + Ud[4]) / sq2;
  const double uar5 = (a1 + a2) * usro;
  const double VdotN = nx * uar2 + ny * uar3 + nz * uar4;
  const bool left = VdotN > 0.0;
  const double* Us = left ? Ug : Ud;
  const double vits2 = left ? vitg2 : vitd2;
  const double vn = Us[1] * nx + Us[2] * ny + Us[3] * nz;
  const double H = (gam * Us[4] + 0.5 * gam1 * Us[0] * vits2) / (gam1 * Us[0]);
  const double f0 = Us[0] * vn;
  const double f1 = f0 * Us[1] + Us[4] * nx, f2 = f0 * Us[2] + Us[4] * ny, f3 = f0 * Us[3] + Us[4] * nz;
  const double f4 = f0 * H;
  const double qir = 0.5 * (uar2 * uar2 + uar3 * uar3 + uar4 * uar4);
  const double c2 = gam1 * (uar5 - qir);
  const double cr = sqrt(c2);
  const double cr2 = 1.0 / c2;
  const double dif1 = Ud[0] - Ug[0];
  const double dif2 = Ud[0] * Ud[1] - Ug[0] * Ug[1];
  const double dif3 = Ud[0] * Ud[2] - Ug[0] * Ug[2];
  const double dif4 = Ud[0] * Ud[3] - Ug[0] * Ug[3];
  const double dif5 = ener2 - ener1;
  const double A = VdotN * dif1 - nx * dif2 - ny * dif3 - nz * dif4;
  const double B = qir * dif1 - uar2 * dif2 - uar3 * dif3 - uar4 * dif4 + dif5;
  const double sg = left ? 1.0 : -1.0;
  const double lamarg = cr - sg * VdotN;
  const bool lam_on = lamarg > 0.0;
  const double lam = lam_on ? lamarg : 0.0;
  const double K = sg * cr * A + gam1 * B;
  const double fl = lam * K;
  const double rs = -sg * cr * fl;
  const double t1 = nx * rs + uar2 * fl, t2 = ny * rs + uar3 * fl, t3 = nz * rs + uar4 * fl;
  const double t4 = VdotN * rs + uar5 * fl;
  const double q0 = f0 - 0.5 * fl * cr2;
  const double q1 = f1 - t1 * 0.5 * cr2, q2 = f2 - t2 * 0.5 * cr2, q3 = f3 - t3 * 0.5 * cr2;
  const double q4 = f4 - t4 * 0.5 * cr2;
  // ---- reverse
  double g_rnorm = gphi[0] * q0 + gphi[1] * q1 + gphi[2] * q2 + gphi[3] * q3 + gphi[4] * q4;
  const double gq0 = gphi[0] * rnorm, gq1 = gphi[1] * rnorm, gq2 = gphi[2] * rnorm, gq3 = gphi[3] * rnorm,
               gq4 = gphi[4] * rnorm;
  double g_f0 = gq0, g_f1 = gq1, g_f2 = gq2, g_f3 = gq3, g_f4 = gq4;
  double g_fl = -0.5 * cr2 * gq0;
  double g_cr2 = -0.5 * (fl * gq0 + t1 * gq1 + t2 * gq2 + t3 * gq3 + t4 * gq4);
  const double gt1 = -0.5 * cr2 * gq1, gt2 = -0.5 * cr2 * gq2, gt3 = -0.5 * cr2 * gq3, gt4 = -0.5 * cr2 * gq4;
  double g_nx = rs * gt1, g_ny = rs * gt2, g_nz = rs * gt3;
  double g_rs = nx * gt1 + ny * gt2 + nz * gt3 + VdotN * gt4;
  double g_uar2 = fl * gt1, g_uar3 = fl * gt2, g_uar4 = fl * gt3, g_uar5 = fl * gt4;
  double g_VdotN = rs * gt4;
  g_fl += uar2 * gt1 + uar3 * gt2 + uar4 * gt3 + uar5 * gt4;
  // rs = -sg cr fl
  double g_cr = -sg * fl * g_rs;
  g_fl += -sg * cr * g_rs;
  // fl = lam K
  const double g_lam = K * g_fl;
  const double g_K = lam * g_fl;
  g_cr += sg * A * g_K;
  const double g_A = sg * cr * g_K;
  const double g_B = gam1 * g_K;
  if (lam_on) {
    g_cr += g_lam;
    g_VdotN += -sg * g_lam;
  }
  // A, B
  g_VdotN += dif1 * g_A;
  double g_dif1 = VdotN * g_A + qir * g_B;
  double g_dif2 = -nx * g_A - uar2 * g_B;
  double g_dif3 = -ny * g_A - uar3 * g_B;
  double g_dif4 = -nz * g_A - uar4 * g_B;
  const double g_dif5 = g_B;
  g_nx -= dif2 * g_A; g_ny -= dif3 * g_A; g_nz -= dif4 * g_A;
  double g_qir = dif1 * g_B;
  g_uar2 -= dif2 * g_B; g_uar3 -= dif3 * g_B; g_uar4 -= dif4 * g_B;
  // cr2 = 1/c2 ; cr = sqrt(c2) ; c2 = gam1 (uar5 - qir)
  double g_c2 = -cr2 * cr2 * g_cr2 + 0.5 / cr * g_cr;
  g_uar5 += gam1 * g_c2;
  g_qir -= gam1 * g_c2;
  g_uar2 += uar2 * g_qir; g_uar3 += uar3 * g_qir; g_uar4 += uar4 * g_qir;
  // differences
  double gL[5] = {0, 0, 0, 0, 0}, gR[5] = {0, 0, 0, 0, 0};
  gR[0] += g_dif1 + Ud[1] * g_dif2 + Ud[2] * g_dif3 + Ud[3] * g_dif4;
  gL[0] -= g_dif1 + Ug[1] * g_dif2 + Ug[2] * g_dif3 + Ug[3] * g_dif4;
  gR[1] += Ud[0] * g_dif2; gR[2] += Ud[0] * g_dif3; gR[3] += Ud[0] * g_dif4;
  gL[1] -= Ug[0] * g_dif2; gL[2] -= Ug[0] * g_dif3; gL[3] -= Ug[0] * g_dif4;
  double g_ener2 = g_dif5, g_ener1 = -g_dif5;
  // centred flux of the upwind side
  {
    double gs[5] = {0, 0, 0, 0, 0};
    const double g_f0t = g_f0 + Us[1] * g_f1 + Us[2] * g_f2 + Us[3] * g_f3 + H * g_f4;
    gs[1] += f0 * g_f1; gs[2] += f0 * g_f2; gs[3] += f0 * g_f3;
    gs[4] += nx * g_f1 + ny * g_f2 + nz * g_f3;
    g_nx += Us[4] * g_f1; g_ny += Us[4] * g_f2; g_nz += Us[4] * g_f3;
    const double g_H = f0 * g_f4;
    gs[0] += vn * g_f0t;
    const double g_vn = Us[0] * g_f0t;
    gs[4] += gam / (gam1 * Us[0]) * g_H;
    gs[0] += -gam * Us[4] / (gam1 * Us[0] * Us[0]) * g_H;
    const double g_vits2 = 0.5 * g_H;
    gs[1] += 2.0 * Us[1] * g_vits2 + nx * g_vn;
    gs[2] += 2.0 * Us[2] * g_vits2 + ny * g_vn;
    gs[3] += 2.0 * Us[3] * g_vits2 + nz * g_vn;
    g_nx += Us[1] * g_vn; g_ny += Us[2] * g_vn; g_nz += Us[3] * g_vn;
    double* gt = left ? gL : gR;
#pragma unroll
    for (int k = 0; k < 5; ++k) gt[k] += gs[k];
  }
  // VdotN = n . uar
  g_nx += uar2 * g_VdotN; g_ny += uar3 * g_VdotN; g_nz += uar4 * g_VdotN;
  g_uar2 += nx * g_VdotN; g_uar3 += ny * g_VdotN; g_uar4 += nz * g_VdotN;
  // Roe averages
  const double g_S = usro * g_uar5;
  double g_usro = (a1 + a2) * g_uar5;
  g_ener1 += g_S / sq1; gL[4] += g_S / sq1;
  g_ener2 += g_S / sq2; gR[4] += g_S / sq2;
  double g_sq1 = -a1 / sq1 * g_S, g_sq2 = -a2 / sq2 * g_S;
  const double gm2 = usro * g_uar2, gm3 = usro * g_uar3, gm4 = usro * g_uar4;
  g_usro += m2 * g_uar2 + m3 * g_uar3 + m4 * g_uar4;
  g_sq1 += Ug[1] * gm2 + Ug[2] * gm3 + Ug[3] * gm4;
  g_sq2 += Ud[1] * gm2 + Ud[2] * gm3 + Ud[3] * gm4;
  gL[1] += sq1 * gm2; gL[2] += sq1 * gm3; gL[3] += sq1 * gm4;
  gR[1] += sq2 * gm2; gR[2] += sq2 * gm3; gR[3] += sq2 * gm4;
  g_sq1 += -usro * usro * g_usro;
  g_sq2 += -usro * usro * g_usro;
  // energies
  gL[4] += invgam1 * g_ener1; gL[0] += 0.5 * vitg2 * g_ener1;
  const double g_vitg2 = 0.5 * Ug[0] * g_ener1;
  gR[4] += invgam1 * g_ener2; gR[0] += 0.5 * vitd2 * g_ener2;
  const double g_vitd2 = 0.5 * Ud[0] * g_ener2;
  gL[1] += 2.0 * Ug[1] * g_vitg2; gL[2] += 2.0 * Ug[2] * g_vitg2; gL[3] += 2.0 * Ug[3] * g_vitg2;
  gR[1] += 2.0 * Ud[1] * g_vitd2; gR[2] += 2.0 * Ud[2] * g_vitd2; gR[3] += 2.0 * Ud[3] * g_vitd2;
  gL[0] += 0.5 / sq1 * g_sq1;
  gR[0] += 0.5 / sq2 * g_sq2;
#pragma unroll
  for (int k = 0; k < 5; ++k) { gUg[k] += gL[k]; gUd[k] += gR[k]; }
  if (gn) {
    // nx = n0 / rnorm ...
    const double g_inv = n0 * g_nx + n1 * g_ny + n2 * g_nz;
    g_rnorm += -invnorm * invnorm * g_inv;
    const double g_s2 = 0.5 / rnorm * g_rnorm;
    gn[0] += invnorm * g_nx + 2.0 * n0 * g_s2;
    gn[1] += invnorm * g_ny + 2.0 * n1 * g_s2;
    gn[2] += invnorm * g_nz + 2.0 * n2 * g_s2;
  }
}

// Partial derivatives of RecFcn::computeVanAlbadaFcn (RecFcn.h:268-281)
// w.r.t. its two arguments, branch by branch.
__device__ __forceinline__ void vanalbada_fcn_partials(double a, double b, double& da, double& db) {
  // one reciprocal of the denominator D (rcp_), branch-free selection
  const double eps = 1.e-16;
  const double ab = a * b;
  const double D = a * a + b * b + 2.0 * eps;
  const double iD = rcp_(D);
  const double iD2 = iD * iD;
  const bool pos = ab > 0.0;
  const double Nn = pos ? a * (b * b + eps) + b * (a * a + eps) : 0.5 * eps * (a + b);
  const double ta = pos ? (b * b + eps) + 2.0 * a * b : 0.5 * eps;
  const double tb = pos ? 2.0 * a * b + (a * a + eps) : 0.5 * eps;
  const bool live = ab >= 0.0;
  da = live ? ta * iD - Nn * 2.0 * a * iD2 : 0.0;
  db = live ? tb * iD - Nn * 2.0 * b * iD2 : 0.0;
}

// Reverse of the per-component reconstruction (vanalbada / linear /
// constant): given cotangents of (Vij, Vji), accumulate those of Vi, Vj and
// of the projected slopes ddVij, ddVji.
__device__ __forceinline__ void reconstruct_adj(int rec, double beta, double Vi, double ddVij, double Vj,
                                                double ddVji, double gVij, double gVji, double& gVi, double& gVj,
                                                double& gddij, double& gddji) {
  if (rec == AEROF_REC_CONSTANT) {
    gVi += gVij; gVj += gVji; gddij = 0.0; gddji = 0.0;
    return;
  }
  if (rec == AEROF_REC_LINEAR) {
    const double b1 = 0.5 - beta;
    gVi += gVij * (1.0 - b1) + gVji * b1;
    gVj += gVij * b1 + gVji * (1.0 - b1);
    gddij = beta * gVij;
    gddji = -beta * gVji;
    return;
  }
  const double b2 = 1.0 - 2.0 * beta;
  const double dVji = Vj - Vi;
  const double dV = b2 * dVji;
  const double dVi = dV + 2.0 * beta * ddVij;
  const double dVj = dV + 2.0 * beta * ddVji;
  double A1, B1, A2, B2;
  vanalbada_fcn_partials(dVi, dVji, A1, B1);
  vanalbada_fcn_partials(dVj, dVji, A2, B2);
  const double g_dVi = 0.5 * A1 * gVij;
  const double g_dVj = -0.5 * A2 * gVji;
  double g_dVji = 0.5 * B1 * gVij - 0.5 * B2 * gVji;
  const double g_dV = g_dVi + g_dVj;
  gddij = 2.0 * beta * g_dVi;
  gddji = 2.0 * beta * g_dVj;
  g_dVji += b2 * g_dV;
  gVi += gVij - g_dVji;
  gVj += gVji + g_dVji;
}

// (dV/dU)^T gV for V = prim(U) (VarFcnSGEuler.h:307-327)
__device__ __forceinline__ void prim_adj(const Gas& g, const double* U, const double* gV, double* gU) {
  const double ir = 1.0 / U[0];
  const double u = U[1] * ir, v = U[2] * ir, w = U[3] * ir;
  gU[0] = gV[0] - (u * gV[1] + v * gV[2] + w * gV[3]) * ir + g.gam1 * 0.5 * (u * u + v * v + w * w) * gV[4];
  gU[1] = gV[1] * ir - g.gam1 * u * gV[4];
  gU[2] = gV[2] * ir - g.gam1 * v * gV[4];
  gU[3] = gV[3] * ir - g.gam1 * w * gV[4];
  gU[4] = g.gam1 * gV[4];
}

}  // namespace aerof
