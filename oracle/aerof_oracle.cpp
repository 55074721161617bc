// aerof_oracle.cpp -- CPU restatement of AERO-F's implicit edge-based
// finite-volume hot path, used ONLY as test infrastructure: the checker in
// tests/, the CPU baseline leg of bench.py and __graft_entry__.smoke().
// Nothing in the product links, loads or calls this file.
//
// Parity status: the reconstruction (RecFcnVanAlbada/RecFcnLinear) and gas
// conversions (VarFcnSGEuler) are pinned against golden vectors produced by
// the reference's own headers (oracle/ref_golden.cpp -> tests/golden/).  The
// Fortran kernels (roeflux7.f, boundflux5.f, roejac6.f) cannot be compiled
// here (no Fortran compiler), so they are pinned by self-consistency only:
// free-stream preservation, flux antisymmetry/consistency and FD checks.
//
// Every function follows one reference routine, cited as file:line (paths
// relative to the AERO-F source tree).  Operation order follows the
// reference's source order, including Fortran left-to-right evaluation, so
// that a double instantiation reproduces the reference's arithmetic.
// Everything is templated on the scalar type: T=double is the reference
// arithmetic, T=Dual gives exact forward-mode derivatives of the same code
// (used to check the GPU's Jacobian-vector and dR/dX kernels).
//
// Build: g++ -O3 -march=native -fopenmp -ffp-contract=off -shared -fPIC
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- dual type
struct Dual {
  double v, d;
  Dual() : v(0), d(0) {}
  Dual(double a) : v(a), d(0) {}
  Dual(double a, double b) : v(a), d(b) {}
};
inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) {
  double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
inline Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
inline Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline Dual sqrt(Dual a) { double s = std::sqrt(a.v); return Dual(s, a.d / (2.0 * s)); }
inline Dual fabs(Dual a) { return a.v < 0 ? -a : a; }
inline double val(double a) { return a; }
inline double val(Dual a) { return a.v; }
using std::sqrt;
using std::fabs;
template <class T> inline T tmax(T a, T b) { return val(a) < val(b) ? b : a; }
template <class T> inline T tmin(T a, T b) { return val(b) < val(a) ? b : a; }

// ---------------------------------------------------------------- constants
constexpr int BC_SLIP_WALL_MOVING = -2;
constexpr int BC_INLET_MOVING = -4;
constexpr int BC_OUTLET_MOVING = -5;
static const double third = 1.0 / 3.0;
static const double twelfth = 1.0 / 12.0;
static const double sixth = 1.0 / 6.0;

// ElemTet tables (ElemTetCore.C:19-21)
static const int edgeEndTet[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
static const int edgeFaceTet[6][2] = {{0, 1}, {2, 0}, {1, 2}, {0, 3}, {3, 1}, {2, 3}};

// ---------------------------------------------------------------- vec3 helpers
template <class T> struct V3 {
  T x[3];
  V3() { x[0] = x[1] = x[2] = T(0.0); }
  V3(T a, T b, T c) { x[0] = a; x[1] = b; x[2] = c; }
  T& operator[](int i) { return x[i]; }
  const T& operator[](int i) const { return x[i]; }
};
template <class T> inline V3<T> operator+(const V3<T>& a, const V3<T>& b) { return V3<T>(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <class T> inline V3<T> operator-(const V3<T>& a, const V3<T>& b) { return V3<T>(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <class T> inline V3<T> operator*(double c, const V3<T>& a) { return V3<T>(c * a[0], c * a[1], c * a[2]); }
// Vec3D::operator^ (Vector3D.h:266-274)
template <class T> inline V3<T> cross(const V3<T>& a, const V3<T>& b) {
  return V3<T>(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}
template <class T> inline T dot(const V3<T>& a, const V3<T>& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// ---------------------------------------------------------------- mesh
struct Mesh {
  int N = 0, T = 0, F = 0, E = 0;
  double gam = 1.4;
  std::vector<double> X;       // [N][3]
  std::vector<int> tets;       // [T][4]
  std::vector<int> faces;      // [F][3]
  std::vector<int> codes;      // [F]
  std::vector<int> edges;      // [E][2], i<j, lexicographic
  std::vector<int> tetEdge;    // [T][6]
  std::vector<int> nodeEdgePtr, nodeEdgeIdx;  // node -> incident edges, ascending
  // geometry (double instantiation)
  std::vector<double> edgeNorm, faceNorm, ctrlVol, Rlsq;
};

// EdgeSet::find + createPointers (EdgeCore.C:55-117): edges are the unique
// (min,max) node pairs of the elements, numbered lexicographically.
static void build_edges(Mesh& m) {
  std::vector<uint64_t> keys;
  keys.reserve((size_t)m.T * 6);
  for (int t = 0; t < m.T; ++t)
    for (int l = 0; l < 6; ++l) {
      uint64_t a = (uint32_t)m.tets[4 * t + edgeEndTet[l][0]];
      uint64_t b = (uint32_t)m.tets[4 * t + edgeEndTet[l][1]];
      if (a > b) std::swap(a, b);
      keys.push_back((a << 32) | b);
    }
  std::vector<uint64_t> u(keys);
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  m.E = (int)u.size();
  m.edges.resize(2 * (size_t)m.E);
  for (int l = 0; l < m.E; ++l) {
    m.edges[2 * l] = (int)(u[l] >> 32);
    m.edges[2 * l + 1] = (int)(u[l] & 0xffffffffu);
  }
  m.tetEdge.resize((size_t)m.T * 6);
  for (size_t k = 0; k < keys.size(); ++k)
    m.tetEdge[k] = (int)(std::lower_bound(u.begin(), u.end(), keys[k]) - u.begin());
  std::vector<int> cnt(m.N + 1, 0);
  for (int l = 0; l < m.E; ++l) { cnt[m.edges[2 * l] + 1]++; cnt[m.edges[2 * l + 1] + 1]++; }
  for (int i = 0; i < m.N; ++i) cnt[i + 1] += cnt[i];
  m.nodeEdgePtr = cnt;
  m.nodeEdgeIdx.resize(2 * (size_t)m.E);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int l = 0; l < m.E; ++l) {
    m.nodeEdgeIdx[pos[m.edges[2 * l]]++] = l;
    m.nodeEdgeIdx[pos[m.edges[2 * l + 1]]++] = l;
  }
}

// ---------------------------------------------------------------- geometry
// Control volumes: ElemTet::computeVolume + computeControlVolumes
// (ElemTetCore.C:24-39, 102-112).
// Edge normals: ElemTet::computeEdgeNormalsGCL1 (ElemTetCore.C:281-330) with
// Xn = Xnp1 = X, the form a static mesh takes (GeoData.C:32, DistGeoState.C:
// 565-568): n = 0.5*((xg1^xg0)+(xg1^xg0)) + 0.25*((xg1^xg0)+(xg1^xg0)).
// Face normals: FaceTria::computeNormalGCL1 (FaceTriaCore.C:65-82), Xn=Xnp1.
// Edge/face normal velocities are zero (DGCL IMPLICIT_ZERO velocities).
template <class T>
static void compute_geometry(const Mesh& m, const T* X, std::vector<T>& edgeNorm,
                             std::vector<T>& faceNorm, std::vector<T>& ctrlVol) {
  edgeNorm.assign(3 * (size_t)m.E, T(0.0));
  faceNorm.assign(3 * (size_t)m.F, T(0.0));
  ctrlVol.assign(m.N, T(0.0));
  auto P = [&](int n) { return V3<T>(X[3 * n], X[3 * n + 1], X[3 * n + 2]); };
  for (int t = 0; t < m.T; ++t) {
    const int* nd = &m.tets[4 * t];
    V3<T> x[4] = {P(nd[0]), P(nd[1]), P(nd[2]), P(nd[3])};
    V3<T> v1 = x[1] - x[0], v2 = x[2] - x[0], v3 = x[3] - x[0];
    T volume = sixth * dot(v3, cross(v1, v2));
    for (int j = 0; j < 4; ++j) ctrlVol[nd[j]] += 0.25 * volume;
  }
  for (int t = 0; t < m.T; ++t) {
    const int* nd = &m.tets[4 * t];
    V3<T> x[4] = {P(nd[0]), P(nd[1]), P(nd[2]), P(nd[3])};
    V3<T> f[4];
    f[0] = third * (x[0] + x[1] + x[2]);
    f[1] = third * (x[0] + x[1] + x[3]);
    f[2] = third * (x[0] + x[2] + x[3]);
    f[3] = third * (x[1] + x[2] + x[3]);
    V3<T> g = 0.25 * (x[0] + x[1] + x[2] + x[3]);
    for (int l = 0; l < 6; ++l) {
      V3<T> xg0 = f[edgeFaceTet[l][0]] - g;
      V3<T> xg1 = f[edgeFaceTet[l][1]] - g;
      V3<T> c = cross(xg1, xg0);
      V3<T> n = 0.5 * (c + c) + 0.25 * (c + c);
      int e = m.tetEdge[6 * t + l];
      if (nd[edgeEndTet[l][0]] < nd[edgeEndTet[l][1]]) {
        for (int k = 0; k < 3; ++k) edgeNorm[3 * e + k] += n[k];
      } else {
        for (int k = 0; k < 3; ++k) edgeNorm[3 * e + k] -= n[k];
      }
    }
  }
  for (int f = 0; f < m.F; ++f) {
    const int* nd = &m.faces[3 * f];
    V3<T> x0 = P(nd[0]), x1 = P(nd[1]), x2 = P(nd[2]);
    V3<T> x01 = x1 - x0, x02 = x2 - x0;
    V3<T> a = 2.0 * x02 + x02;
    V3<T> s = cross(a, x01) + cross(a, x01);
    V3<T> n = twelfth * s;
    for (int k = 0; k < 3; ++k) faceNorm[3 * f + k] = n[k];
  }
}

// SubDomain::computeWeightsLeastSquaresEdgePart (SubDomainCore.C:1334-1381)
// and NodePart (SubDomainCore.C:1755-1777): R = upper Cholesky factor of
// sum_j dx dx^T, stored (r11,r12,r13,r22,r23,r33).
template <class T>
static void compute_lsq_R(const Mesh& m, const T* X, std::vector<T>& R) {
  R.assign(6 * (size_t)m.N, T(0.0));
  for (int l = 0; l < m.E; ++l) {
    int i = m.edges[2 * l], j = m.edges[2 * l + 1];
    T dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
    T dxdx = dx[0] * dx[0], dydy = dx[1] * dx[1], dzdz = dx[2] * dx[2];
    T dxdy = dx[0] * dx[1], dxdz = dx[0] * dx[2], dydz = dx[1] * dx[2];
    R[6 * i + 0] += dxdx; R[6 * j + 0] += dxdx;
    R[6 * i + 1] += dxdy; R[6 * j + 1] += dxdy;
    R[6 * i + 2] += dxdz; R[6 * j + 2] += dxdz;
    R[6 * i + 3] += dydy; R[6 * j + 3] += dydy;
    R[6 * i + 4] += dydz; R[6 * j + 4] += dydz;
    R[6 * i + 5] += dzdz; R[6 * j + 5] += dzdz;
  }
  for (int i = 0; i < m.N; ++i) {
    T* r = &R[6 * i];
    T r11 = sqrt(r[0]);
    T or11 = 1.0 / r11;
    T r12 = r[1] * or11;
    T r13 = r[2] * or11;
    T r22 = sqrt(r[3] - r12 * r12);
    T r23 = (r[4] - r12 * r13) / r22;
    T r33 = sqrt(r[5] - (r13 * r13 + r23 * r23));
    r[0] = r11; r[1] = r12; r[2] = r13; r[3] = r22; r[4] = r23; r[5] = r33;
  }
}

// computeLocalWeightsLeastSquares (SubDomain.C:137-159)
template <class T>
static inline void lsq_weights(const T dx[3], const T* R, T W[3]) {
  T or11 = 1.0 / R[0];
  T or22 = 1.0 / R[3];
  T or33 = 1.0 / R[5];
  T r12or11 = R[1] * or11;
  T r23or22 = R[4] * or22;
  T psi = (R[1] * R[4] - R[2] * R[3]) * or11 * or22;
  T alpha1 = dx[0] * or11 * or11;
  T alpha2 = (dx[1] - r12or11 * dx[0]) * or22 * or22;
  T alpha3 = (dx[2] - r23or22 * dx[1] + psi * dx[0]) * or33 * or33;
  W[0] = alpha1 - r12or11 * alpha2 + psi * alpha3;
  W[1] = alpha2 - r23or22 * alpha3;
  W[2] = alpha3;
}

// VarFcnSGEuler::conservativeToPrimitive (VarFcnSGEuler.h:307-327), Pstiff=0
template <class T>
static inline void cons2prim(double gam, const T* U, T* V) {
  V[0] = U[0];
  T invRho = 1.0 / U[0];
  V[1] = U[1] * invRho;
  V[2] = U[2] * invRho;
  V[3] = U[3] * invRho;
  T vel2 = V[1] * V[1] + V[2] * V[2] + V[3] * V[3];
  V[4] = (gam - 1.0) * (U[4] - 0.5 * U[0] * vel2) - gam * 0.0;
}

// SubDomain::computeGradientsLeastSquares (SubDomain.C:297-374)
template <class T>
static void compute_gradients(const Mesh& m, const T* X, const T* R, const T* V,
                              T* ddx, T* ddy, T* ddz) {
  for (size_t k = 0; k < 5 * (size_t)m.N; ++k) ddx[k] = ddy[k] = ddz[k] = T(0.0);
  for (int l = 0; l < m.E; ++l) {
    int i = m.edges[2 * l], j = m.edges[2 * l + 1];
    T Wi[3], Wj[3];
    T dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
    lsq_weights(dx, &R[6 * i], Wi);
    dx[0] = -dx[0]; dx[1] = -dx[1]; dx[2] = -dx[2];
    lsq_weights(dx, &R[6 * j], Wj);
    for (int k = 0; k < 5; ++k) {
      T dv = V[5 * j + k] - V[5 * i + k];
      ddx[5 * i + k] += Wi[0] * dv;
      ddy[5 * i + k] += Wi[1] * dv;
      ddz[5 * i + k] += Wi[2] * dv;
      ddx[5 * j + k] -= Wj[0] * dv;
      ddy[5 * j + k] -= Wj[1] * dv;
      ddz[5 * j + k] -= Wj[2] * dv;
    }
  }
}

// RecFcn::computeVanAlbadaFcn (RecFcn.h:268-281)
template <class T>
static inline T vanalbada_fcn(double eps, T a, T b) {
  T a2 = a * a;
  T b2 = b * b;
  if (val(a * b) > 0.0) return (a * (b2 + eps) + b * (a2 + eps)) / (a2 + b2 + 2.0 * eps);
  else if (val(a * b) == 0.0) return 0.5 * eps * (a + b) / (a2 + b2 + 2.0 * eps);
  else return T(0.0);
}

// RecFcn constructor (RecFcn.h:40-49) and vanalbada (RecFcn.h:432-446),
// linear (RecFcn.h:240-249); beta = 1/3 (IoDataCore.C:2425).
struct RecParams {
  double beta, beta1, beta2, eps0;
};
static inline RecParams rec_params(double beta) {
  RecParams p;
  p.beta = beta;
  p.beta1 = 0.5 - beta;
  p.beta2 = 1.0 - 2.0 * beta;
  p.eps0 = 1.e-16;
  return p;
}
template <class T>
static inline void vanalbada(const RecParams& p, T Vi, T ddVij, T Vj, T ddVji, T& Vij, T& Vji) {
  T dVji = Vj - Vi;
  T dV = p.beta2 * dVji;
  T dVi = dV + 2.0 * p.beta * ddVij;
  T dVj = dV + 2.0 * p.beta * ddVji;
  Vij = Vi + 0.5 * vanalbada_fcn(p.eps0, dVi, dVji);
  Vji = Vj - 0.5 * vanalbada_fcn(p.eps0, dVj, dVji);
}
template <class T>
static inline void linear_rec(const RecParams& p, T Vi, T ddVij, T Vj, T ddVji, T& Vij, T& Vji) {
  T dV = p.beta1 * (Vj - Vi);
  Vij = Vi + dV + p.beta * ddVij;
  Vji = Vj - dV - p.beta * ddVji;
}

// roeflux7.f:1-202 (type 0): Roe flux with one-wave dissipation, gamma=1.
template <class T>
static void roeflux7(double gam, double pstiff, const T* enormal, T evitno, const T* Ug,
                     const T* Ud, T* phi) {
  double gam1 = gam - 1.0;
  double invgam1 = 1.0 / gam1;
  T rnorm = sqrt(enormal[0] * enormal[0] + enormal[1] * enormal[1] + enormal[2] * enormal[2]);
  T invnorm = 1.0 / rnorm;
  T normal[3] = {enormal[0] * invnorm, enormal[1] * invnorm, enormal[2] * invnorm};
  T vitno = evitno * invnorm;
  T vitg2 = Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3];
  T vitd2 = Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3];
  T squsr1 = sqrt(Ug[0]);
  T squsr2 = sqrt(Ud[0]);
  T ener1 = (Ug[4] + gam * pstiff) * invgam1 + 0.5 * Ug[0] * vitg2;
  T ener2 = (Ud[4] + gam * pstiff) * invgam1 + 0.5 * Ud[0] * vitd2;
  T usro = 1.0 / (squsr1 + squsr2);
  T uar2 = (squsr1 * Ug[1] + squsr2 * Ud[1]) * usro;
  T uar3 = (squsr1 * Ug[2] + squsr2 * Ud[2]) * usro;
  T uar4 = (squsr1 * Ug[3] + squsr2 * Ud[3]) * usro;
  T uar5 = ((ener1 + Ug[4]) / squsr1 + (ener2 + Ud[4]) / squsr2) * usro;
  T VdotNt = normal[0] * uar2 + normal[1] * uar3 + normal[2] * uar4;
  T VdotN, H;
  if (val(VdotNt - vitno) > 0) {
    VdotN = Ug[1] * normal[0] + Ug[2] * normal[1] + Ug[3] * normal[2];
    H = gam * (Ug[4] + pstiff) + 0.5 * gam1 * Ug[0] * vitg2;
    H = H / (gam1 * Ug[0]);
    phi[0] = Ug[0] * (VdotN - vitno);
    phi[1] = phi[0] * Ug[1] + Ug[4] * normal[0];
    phi[2] = phi[0] * Ug[2] + Ug[4] * normal[1];
    phi[3] = phi[0] * Ug[3] + Ug[4] * normal[2];
    phi[4] = phi[0] * H + Ug[4] * vitno;
  } else {
    VdotN = Ud[1] * normal[0] + Ud[2] * normal[1] + Ud[3] * normal[2];
    H = gam * (Ud[4] + pstiff) + 0.5 * gam1 * Ud[0] * vitd2;
    H = H / (gam1 * Ud[0]);
    phi[0] = Ud[0] * (VdotN - vitno);
    phi[1] = phi[0] * Ud[1] + Ud[4] * normal[0];
    phi[2] = phi[0] * Ud[2] + Ud[4] * normal[1];
    phi[3] = phi[0] * Ud[3] + Ud[4] * normal[2];
    phi[4] = phi[0] * H + Ud[4] * vitno;
  }
  VdotN = VdotNt;
  T qir = 0.5 * (uar2 * uar2 + uar3 * uar3 + uar4 * uar4);
  T cr2 = gam1 * (uar5 - qir);
  T cr = sqrt(cr2);
  cr2 = 1.0 / cr2;
  T vp1 = VdotN;
  T vp4 = VdotN + cr;
  T vp5 = VdotN - cr;
  T r = cr;
  T s = -cr;
  T cr2byt = -cr;
  T invtbeta2 = -1.0 / cr;
  T dif1 = -Ug[0] + Ud[0];
  T dif2 = -Ug[0] * Ug[1] + Ud[0] * Ud[1];
  T dif3 = -Ug[0] * Ug[2] + Ud[0] * Ud[2];
  T dif4 = -Ug[0] * Ug[3] + Ud[0] * Ud[3];
  T dif5 = -ener1 + ener2;
  vp1 = vp1 - vitno;
  vp4 = vp4 - vitno;
  vp5 = vp5 - vitno;
  (void)vp1;
  T flur4, flur5;
  if (val(VdotNt - vitno) <= 0) {
    flur4 = tmax(vp4, T(0.0)) *
            (cr2byt * (VdotN * dif1 - normal[0] * dif2 - normal[1] * dif3 - normal[2] * dif4) +
             gam1 * s * invtbeta2 * (qir * dif1 - uar2 * dif2 - uar3 * dif3 - uar4 * dif4 + dif5));
    flur5 = T(0.0);
  } else {
    flur4 = T(0.0);
    flur5 = -tmin(vp5, T(0.0)) *
            (-cr2byt * (VdotN * dif1 - normal[0] * dif2 - normal[1] * dif3 - normal[2] * dif4) +
             (-gam1 * r * invtbeta2 * (qir * dif1 - uar2 * dif2 - uar3 * dif3 - uar4 * dif4 + dif5)));
  }
  phi[0] = phi[0] - 0.5 * (flur4 + flur5) * cr2;
  phi[1] = phi[1] - (normal[0] * (r * flur4 + s * flur5) + uar2 * (flur4 + flur5)) * 0.5 * cr2;
  phi[2] = phi[2] - (normal[1] * (r * flur4 + s * flur5) + uar3 * (flur4 + flur5)) * 0.5 * cr2;
  phi[3] = phi[3] - (normal[2] * (r * flur4 + s * flur5) + uar4 * (flur4 + flur5)) * 0.5 * cr2;
  phi[4] = phi[4] - (VdotN * (r * flur4 + s * flur5) + uar5 * (flur4 + flur5)) * 0.5 * cr2;
  for (int k = 0; k < 5; ++k) phi[k] = phi[k] * rnorm;
}

// boundflux5.f:1-111 (type 0): Steger-Warming far-field flux
// A+(V)U + A-(V)Ub; ua primitive, ub conservative.
template <class T>
static void boundflux5(double gam, const T* normal, T sig, const T* ua, const double* ub, T* flux) {
  double gam1 = gam - 1.0;
  T vnx = normal[0], vny = normal[1], vnz = normal[2];
  T cap = sqrt(vnx * vnx + vny * vny + vnz * vnz);
  T capd1 = vnx / cap, capd2 = vny / cap, capd3 = vnz / cap;
  T ro = ua[0];
  T usro = 1.0 / ro;
  T u = ua[1], v = ua[2], w = ua[3];
  T vit = u * u + v * v + w * w;
  T pm = ua[4];
  T rhoE = pm / gam1 + 0.5 * ro * vit;
  T c2 = gam * pm * usro;
  T c = sqrt(c2);
  T usc = 1.0 / c;
  T cc = 0.5 * vit + c2 / gam1;
  T unx = capd1 * u + capd2 * v + capd3 * w;
  T vp1 = tmax(cap * unx - sig, T(0.0));
  T vp4 = tmax(cap * (unx + c) - sig, T(0.0));
  T vp5 = tmax(cap * (unx - c) - sig, T(0.0));
  T vpp = vp4 + vp5;
  T vpm = vp4 - vp5;
  T fgp[5];
  fgp[0] = (gam1 * ro * vp1 + 0.5 * ro * vpp) / gam;
  fgp[1] = fgp[0] * u + 0.5 * pm * usc * capd1 * vpm;
  fgp[2] = fgp[0] * v + 0.5 * pm * usc * capd2 * vpm;
  fgp[3] = fgp[0] * w + 0.5 * pm * usc * capd3 * vpm;
  fgp[4] = 0.5 * ((gam1 / gam) * ro * vit * (vp1 - 0.5 * vpp) + rhoE * vpp + ro * unx * c * vpm / gam);
  vp1 = tmin(cap * unx - sig, T(0.0));
  vp4 = tmin(cap * (unx + c) - sig, T(0.0));
  vp5 = tmin(cap * (unx - c) - sig, T(0.0));
  vpp = vp1 - 0.5 * (vp4 + vp5);
  vpm = 0.5 * (vp5 - vp4);
  T xn1 = gam1 * usc * (-(0.5 * vit * ub[0]) + u * ub[1] + v * ub[2] + w * ub[3] - ub[4]);
  T xn2 = unx * ub[0] - capd1 * ub[1] - capd2 * ub[2] - capd3 * ub[3];
  T ff = usc * (vpp * xn1 + vpm * xn2);
  T gg = vpm * xn1 + vpp * xn2;
  T fgm[5];
  fgm[0] = vp1 * ub[0] + ff;
  fgm[1] = vp1 * ub[1] + u * ff + capd1 * gg;
  fgm[2] = vp1 * ub[2] + v * ff + capd2 * gg;
  fgm[3] = vp1 * ub[3] + w * ff + capd3 * gg;
  fgm[4] = vp1 * ub[4] + cc * ff + unx * gg;
  for (int k = 0; k < 5; ++k) flux[k] = fgp[k] + fgm[k];
}

// FluxFcnSGWallEuler3D::compute (FluxFcnDescSG.C:779-789)
template <class T>
static inline void wallflux(const T* normal, T normalVel, const T* V, T* flux) {
  flux[0] = T(0.0);
  flux[1] = V[4] * normal[0];
  flux[2] = V[4] * normal[1];
  flux[3] = V[4] * normal[2];
  flux[4] = V[4] * normalVel;
}

template <class T>
static inline void face_flux(double gam, int code, const T* n3, const T* V, const double* Ub, T* flux) {
  if (code == BC_SLIP_WALL_MOVING) wallflux(n3, T(0.0), V, flux);
  else boundflux5(gam, n3, T(0.0), V, Ub, flux);
}

// ---------------------------------------------------------------- residual
// SpaceOperator::computeResidual (SpaceOperator.C:524-634) restricted to the
// Euler / finite-volume / NONDESCRIPTOR path:
//   R=0; V=prim(U); [LSQ gradients]; edge loop (Edge.C:371-439) with
//   reconstruction, positivity check (EdgeCore.C:137-168), Roe flux; face
//   loop (Face.C:354-389, 1185-1215) with subface normals n_f/3
//   (FaceTriaCore.C:288-308); R *= 1/ctrlVol (SpaceOperator.C:614-620).
// order: 1 = RecFcnConstant, 2 = LSQ + van Albada, 3 = LSQ + linear.
// Failsafe (Domain.C:876-918): when failsafe != 0 and a reconstructed
// density/pressure is non-positive, the offending nodes are tagged, their
// gradients zeroed, and the edge loop is re-run.  Returns the number of
// non-positive reconstructed states of the first pass.
template <class T>
struct Work {
  std::vector<T> V, ddx, ddy, ddz;
};

template <class T>
static int residual_t(const Mesh& m, const T* X, const std::vector<T>& edgeNorm,
                      const std::vector<T>& faceNorm, const std::vector<T>& ctrlVol,
                      const std::vector<T>& Rlsq, const T* U, const double* Ub, int order,
                      double beta, int failsafe, T* R, Work<T>& w) {
  const double gam = m.gam;
  const int N = m.N;
  w.V.resize(5 * (size_t)N);
  for (int i = 0; i < N; ++i) cons2prim(gam, &U[5 * i], &w.V[5 * i]);
  const T* V = w.V.data();
  if (order > 1) {
    w.ddx.resize(5 * (size_t)N); w.ddy.resize(5 * (size_t)N); w.ddz.resize(5 * (size_t)N);
    compute_gradients(m, X, Rlsq.data(), V, w.ddx.data(), w.ddy.data(), w.ddz.data());
  }
  RecParams rp = rec_params(order == 1 ? 0.0 : beta);
  std::vector<char> tag;
  int ierr_first = 0;
  for (int pass = 0; pass < 2; ++pass) {
    for (size_t k = 0; k < 5 * (size_t)N; ++k) R[k] = T(0.0);
    int ierr = 0;
    for (int l = 0; l < m.E; ++l) {
      int i = m.edges[2 * l], j = m.edges[2 * l + 1];
      T dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
      T Vi[5], Vj[5];
      if (order == 1) {
        for (int k = 0; k < 5; ++k) { Vi[k] = V[5 * i + k]; Vj[k] = V[5 * j + k]; }
      } else {
        for (int k = 0; k < 5; ++k) {
          T ddVij = dx[0] * w.ddx[5 * i + k] + dx[1] * w.ddy[5 * i + k] + dx[2] * w.ddz[5 * i + k];
          T ddVji = dx[0] * w.ddx[5 * j + k] + dx[1] * w.ddy[5 * j + k] + dx[2] * w.ddz[5 * j + k];
          if (order == 2) vanalbada(rp, V[5 * i + k], ddVij, V[5 * j + k], ddVji, Vi[k], Vj[k]);
          else linear_rec(rp, V[5 * i + k], ddVij, V[5 * j + k], ddVji, Vi[k], Vj[k]);
        }
      }
      // VarFcnSGEuler::checkReconstructedValues (VarFcnSGEuler.h:90-110)
      bool bi = val(Vi[0]) <= 0.0 || val(Vi[4]) + 0.0 <= 0.0;
      bool bj = val(Vj[0]) <= 0.0 || val(Vj[4]) + 0.0 <= 0.0;
      if (bi || bj) {
        ierr += (int)bi + (int)bj;
        if (pass == 0 && failsafe) {
          if (tag.empty()) tag.assign(N, 0);
          if (bi) tag[i] = 1;
          if (bj) tag[j] = 1;
        }
        continue;
      }
      const T* nl = &edgeNorm[3 * l];
      T nn = sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
      if (val(nn) < 1e-18) continue;
      T flux[5];
      roeflux7(gam, 0.0, nl, T(0.0), Vi, Vj, flux);
      for (int k = 0; k < 5; ++k) { R[5 * i + k] += flux[k]; R[5 * j + k] -= flux[k]; }
    }
    if (pass == 0) ierr_first = ierr;
    if (pass == 0 && ierr && failsafe && order > 1) {
      for (int i = 0; i < N; ++i)
        if (tag[i])
          for (int k = 0; k < 5; ++k) w.ddx[5 * i + k] = w.ddy[5 * i + k] = w.ddz[5 * i + k] = T(0.0);
      continue;
    }
    break;
  }
  for (int f = 0; f < m.F; ++f) {
    T n3[3] = {third * faceNorm[3 * f], third * faceNorm[3 * f + 1], third * faceNorm[3 * f + 2]};
    for (int l = 0; l < 3; ++l) {
      int nd = m.faces[3 * f + l];
      T flux[5];
      face_flux(gam, m.codes[f], n3, &V[5 * nd], Ub, flux);
      for (int k = 0; k < 5; ++k) R[5 * nd + k] += flux[k];
    }
  }
  for (int i = 0; i < N; ++i) {
    T invcv = 1.0 / ctrlVol[i];
    for (int k = 0; k < 5; ++k) R[5 * i + k] *= invcv;
  }
  return ierr_first;
}

// Threaded second-order residual for the CPU baseline timing: the edge list
// is cut into nthreads contiguous chunks, each accumulated into a private
// array and summed in chunk order, the way AERO-F's OpenMP loop over
// subdomains accumulates per-subdomain arrays that CommPattern then adds
// (Domain.C:868-928).
static void residual_threaded(const Mesh& m, const double* U, const double* Ub, int order,
                              double beta, int nthreads, double* R,
                              std::vector<double>& V, std::vector<double>& G,
                              std::vector<double>& priv) {
  const int N = m.N, E = m.E;
  const double gam = m.gam;
  V.resize(5 * (size_t)N);
  G.resize(15 * (size_t)N);
  priv.resize((size_t)nthreads * 15 * N);
  const double* X = m.X.data();
  RecParams rp = rec_params(order == 1 ? 0.0 : beta);
#pragma omp parallel num_threads(nthreads)
  {
#ifdef _OPENMP
    int t = omp_get_thread_num();
#else
    int t = 0;
#endif
    int l0 = (int)((int64_t)E * t / nthreads), l1 = (int)((int64_t)E * (t + 1) / nthreads);
#pragma omp for schedule(static)
    for (int i = 0; i < N; ++i) cons2prim(gam, &U[5 * i], &V[5 * i]);
    if (order > 1) {
      double* g = &priv[(size_t)t * 15 * N];
      std::memset(g, 0, sizeof(double) * 15 * (size_t)N);
      for (int l = l0; l < l1; ++l) {
        int i = m.edges[2 * l], j = m.edges[2 * l + 1];
        double Wi[3], Wj[3];
        double dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        lsq_weights(dx, &m.Rlsq[6 * i], Wi);
        dx[0] = -dx[0]; dx[1] = -dx[1]; dx[2] = -dx[2];
        lsq_weights(dx, &m.Rlsq[6 * j], Wj);
        for (int k = 0; k < 5; ++k) {
          double dv = V[5 * j + k] - V[5 * i + k];
          g[15 * i + k] += Wi[0] * dv; g[15 * i + 5 + k] += Wi[1] * dv; g[15 * i + 10 + k] += Wi[2] * dv;
          g[15 * j + k] -= Wj[0] * dv; g[15 * j + 5 + k] -= Wj[1] * dv; g[15 * j + 10 + k] -= Wj[2] * dv;
        }
      }
#pragma omp barrier
#pragma omp for schedule(static)
      for (int i = 0; i < N; ++i)
        for (int k = 0; k < 15; ++k) {
          double s = 0.0;
          for (int q = 0; q < nthreads; ++q) s += priv[(size_t)q * 15 * N + 15 * i + k];
          G[15 * i + k] = s;
        }
    }
    double* r = &priv[(size_t)t * 15 * N];
#pragma omp barrier
    std::memset(r, 0, sizeof(double) * 5 * (size_t)N);
    for (int l = l0; l < l1; ++l) {
      int i = m.edges[2 * l], j = m.edges[2 * l + 1];
      double Vi[5], Vj[5];
      if (order == 1) {
        for (int k = 0; k < 5; ++k) { Vi[k] = V[5 * i + k]; Vj[k] = V[5 * j + k]; }
      } else {
        double dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
        for (int k = 0; k < 5; ++k) {
          double ddVij = dx[0] * G[15 * i + k] + dx[1] * G[15 * i + 5 + k] + dx[2] * G[15 * i + 10 + k];
          double ddVji = dx[0] * G[15 * j + k] + dx[1] * G[15 * j + 5 + k] + dx[2] * G[15 * j + 10 + k];
          vanalbada(rp, V[5 * i + k], ddVij, V[5 * j + k], ddVji, Vi[k], Vj[k]);
        }
      }
      double flux[5];
      roeflux7(gam, 0.0, &m.edgeNorm[3 * l], 0.0, Vi, Vj, flux);
      for (int k = 0; k < 5; ++k) { r[5 * i + k] += flux[k]; r[5 * j + k] -= flux[k]; }
    }
    if (t == 0) {
      for (int f = 0; f < m.F; ++f) {
        double n3[3] = {third * m.faceNorm[3 * f], third * m.faceNorm[3 * f + 1], third * m.faceNorm[3 * f + 2]};
        for (int l = 0; l < 3; ++l) {
          int nd = m.faces[3 * f + l];
          double flux[5];
          face_flux(gam, m.codes[f], n3, &V[5 * nd], Ub, flux);
          for (int k = 0; k < 5; ++k) r[5 * nd + k] += flux[k];
        }
      }
    }
#pragma omp barrier
#pragma omp for schedule(static)
    for (int i = 0; i < N; ++i) {
      double invcv = 1.0 / m.ctrlVol[i];
      for (int k = 0; k < 5; ++k) {
        double s = 0.0;
        for (int q = 0; q < nthreads; ++q) s += priv[(size_t)q * 15 * N + 5 * i + k];
        R[5 * i + k] = s * invcv;
      }
    }
  }
}

// ---------------------------------------------------------------- time step
// EdgeSet::computeTimeStep (Edge.C:87-143), Face::computeTimeStep
// (Face.C:242-289) and the dt formula of Domain::computeTimeStep
// (Domain.C:70-96): dt_i = cfl*vol_i / (-idti_i), beta = 1 (no low-Mach
// preconditioning, LowMachPrec.h:89-92).
static void timestep(const Mesh& m, const double* U, double cfl, double* dt) {
  const double gam = m.gam;
  std::vector<double> V(5 * (size_t)m.N), idti(m.N, 0.0);
  for (int i = 0; i < m.N; ++i) cons2prim(gam, &U[5 * i], &V[5 * i]);
  const double locbeta = 1.0, beta2 = locbeta * locbeta;
  for (int l = 0; l < m.E; ++l) {
    int i = m.edges[2 * l], j = m.edges[2 * l + 1];
    const double* nl = &m.edgeNorm[3 * l];
    double S = std::sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
    double invS = 1.0 / S;
    double n[3] = {invS * nl[0], invS * nl[1], invS * nl[2]};
    double ndot = invS * 0.0;
    double Vmid[5];
    for (int k = 0; k < 5; ++k) Vmid[k] = 0.5 * (V[5 * i + k] + V[5 * j + k]);
    double a = std::sqrt(gam * (Vmid[4] + 0.0) / Vmid[0]);
    double un = Vmid[1] * n[0] + Vmid[2] * n[1] + Vmid[3] * n[2] - ndot;
    double coeff1 = (1.0 + beta2) * un;
    double coeff2 = std::pow(std::pow((1.0 - beta2) * un, 2.0) + std::pow(2.0 * locbeta * a, 2.0), 0.5);
    idti[i] += std::min(0.5 * (coeff1 - coeff2), 0.0) * S;
    idti[j] += std::min(0.5 * (-coeff1 - coeff2), 0.0) * S;
  }
  for (int f = 0; f < m.F; ++f) {
    const double* nf = &m.faceNorm[3 * f];
    double S = std::sqrt(nf[0] * nf[0] + nf[1] * nf[1] + nf[2] * nf[2]);
    double invS = 1.0 / S;
    double n[3] = {invS * nf[0], invS * nf[1], invS * nf[2]};
    double ndot = invS * 0.0;
    for (int l = 0; l < 3; ++l) {
      int nd = m.faces[3 * f + l];
      const double* v = &V[5 * nd];
      double a = std::sqrt(gam * (v[4] + 0.0) / v[0]);
      double un = v[1] * n[0] + v[2] * n[1] + v[3] * n[2] - ndot;
      double coeff1 = (1.0 + beta2) * un;
      double coeff2 = std::pow(std::pow((1.0 - beta2) * un, 2.0) + std::pow(2.0 * locbeta * a, 2.0), 0.5);
      idti[nd] += std::min(0.5 * (coeff1 - coeff2), 0.0) * S / 3;
    }
  }
  for (int i = 0; i < m.N; ++i) dt[i] = cfl * m.ctrlVol[i] / (-1.0 * idti[i] + 0.0 * 0.0);
}

// ---------------------------------------------------------------- Jacobians
// VarFcnSGEuler::computedVdU (VarFcnSGEuler.h:588-603) and
// VarFcnBase::postMultiplyBydVdU (VarFcnBase.h:372-400).
static void post_dVdU(double gam, const double* V, const double* mat, double* res) {
  double gam1 = gam - 1.0;
  double d[25] = {0};
  double invrho = 1.0 / V[0];
  d[0] = 1.0;
  d[5] = -invrho * V[1]; d[6] = invrho;
  d[10] = -invrho * V[2]; d[12] = invrho;
  d[15] = -invrho * V[3]; d[18] = invrho;
  d[20] = gam1 * 0.5 * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]);
  d[21] = -gam1 * V[1]; d[22] = -gam1 * V[2]; d[23] = -gam1 * V[3]; d[24] = gam1;
  for (int r = 0; r < 5; ++r) {
    const double* m = &mat[5 * r];
    double* o = &res[5 * r];
    o[0] = m[0] * d[0] + m[1] * d[5] + m[2] * d[10] + m[3] * d[15] + m[4] * d[20];
    o[1] = m[1] * d[6] + m[4] * d[21];
    o[2] = m[2] * d[12] + m[4] * d[22];
    o[3] = m[3] * d[18] + m[4] * d[23];
    o[4] = m[4] * d[24];
  }
}

// roejac6.f:1-316 with type=0, prec=0 (beta=1), dissipation gamma=1.
static void roejac6(double gamma, double gam, double pstiff, const double* enormal, double evitno,
                    const double* Ug, const double* Ud, double* jac, int sw) {
  double gam1 = gam - 1.0;
  double rnorm = std::sqrt(enormal[0] * enormal[0] + enormal[1] * enormal[1] + enormal[2] * enormal[2]);
  double invnorm = 1.0 / rnorm;
  double normal[3] = {enormal[0] * invnorm, enormal[1] * invnorm, enormal[2] * invnorm};
  double vitno = evitno * invnorm;
  double H[5][5], tmw[5][5], dmat[5][5];
  double VdotN = Ug[1] * normal[0] + Ug[2] * normal[1] + Ug[3] * normal[2];
  double qir = 0.5 * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]);
  double enth = gam * (Ug[4] + pstiff) + gam1 * Ug[0] * qir;
  enth = enth / (gam1 * Ug[0]);
  H[0][0] = -vitno; H[0][1] = normal[0]; H[0][2] = normal[1]; H[0][3] = normal[2]; H[0][4] = 0.0;
  H[1][0] = gam1 * normal[0] * qir - Ug[1] * VdotN;
  H[1][1] = (1.0 - gam1) * normal[0] * Ug[1] + VdotN - vitno;
  H[1][2] = -gam1 * normal[0] * Ug[2] + Ug[1] * normal[1];
  H[1][3] = -gam1 * normal[0] * Ug[3] + Ug[1] * normal[2];
  H[1][4] = gam1 * normal[0];
  H[2][0] = gam1 * normal[1] * qir - Ug[2] * VdotN;
  H[2][1] = -gam1 * normal[1] * Ug[1] + Ug[2] * normal[0];
  H[2][2] = (1.0 - gam1) * normal[1] * Ug[2] + VdotN - vitno;
  H[2][3] = -gam1 * normal[1] * Ug[3] + Ug[2] * normal[2];
  H[2][4] = gam1 * normal[1];
  H[3][0] = gam1 * normal[2] * qir - Ug[3] * VdotN;
  H[3][1] = -gam1 * normal[2] * Ug[1] + Ug[3] * normal[0];
  H[3][2] = -gam1 * normal[2] * Ug[2] + Ug[3] * normal[1];
  H[3][3] = (1.0 - gam1) * normal[2] * Ug[3] + VdotN - vitno;
  H[3][4] = gam1 * normal[2];
  H[4][0] = (gam1 * qir - enth) * VdotN;
  H[4][1] = enth * normal[0] - gam1 * Ug[1] * VdotN;
  H[4][2] = enth * normal[1] - gam1 * Ug[2] * VdotN;
  H[4][3] = enth * normal[2] - gam1 * Ug[3] * VdotN;
  H[4][4] = (1.0 + gam1) * VdotN - vitno;
  double squsr1 = std::sqrt(Ug[0]);
  double squsr2 = std::sqrt(Ud[0]);
  double ener1 = (Ug[4] + gam * pstiff) / gam1 + 0.5 * Ug[0] * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]);
  double ener2 = (Ud[4] + gam * pstiff) / gam1 + 0.5 * Ud[0] * (Ud[1] * Ud[1] + Ud[2] * Ud[2] + Ud[3] * Ud[3]);
  double usro = 1.0 / (squsr1 + squsr2);
  double uar2 = (squsr1 * Ug[1] + squsr2 * Ud[1]) * usro;
  double uar3 = (squsr1 * Ug[2] + squsr2 * Ud[2]) * usro;
  double uar4 = (squsr1 * Ug[3] + squsr2 * Ud[3]) * usro;
  double uar5 = ((ener1 + Ug[4]) / squsr1 + (ener2 + Ud[4]) / squsr2) * usro;
  enth = uar5;
  VdotN = normal[0] * uar2 + normal[1] * uar3 + normal[2] * uar4;
  qir = 0.5 * (uar2 * uar2 + uar3 * uar3 + uar4 * uar4);
  double cr2 = gam1 * (uar5 - qir);
  double cr = std::sqrt(cr2);
  cr2 = 1.0 / cr2;
  double gc = gam1 / (cr * cr);
  double usc2 = 0.5 / (cr * cr);
  double beta = 1.0;
  double betaRT2 = beta * beta;
  double vp1 = VdotN;
  double sq = std::sqrt(((1.0 - betaRT2) * VdotN) * ((1.0 - betaRT2) * VdotN) + 4.0 * betaRT2 * (cr * cr));
  double vp4 = 0.5 * ((1.0 + betaRT2) * VdotN + sq);
  double vp5 = 0.5 * ((1.0 + betaRT2) * VdotN - sq);
  double rRT = vp4 - vp1 * betaRT2;
  double sRT = vp5 - vp1 * betaRT2;
  double tRT = 0.5 * (vp5 - vp4);
  vp1 = std::fabs(vp1 - vitno) * gamma;
  vp4 = std::fabs(vp4 - vitno) * gamma;
  vp5 = std::fabs(vp5 - vitno) * gamma;
  const double* n = normal;
  tmw[0][0] = n[0] + n[1] * uar4 - uar3 * n[2] - gc * n[0] * qir;
  tmw[0][1] = gc * n[0] * uar2;
  tmw[0][2] = gc * n[0] * uar3 + n[2];
  tmw[0][3] = gc * n[0] * uar4 - n[1];
  tmw[0][4] = -gc * n[0];
  tmw[1][0] = n[1] + n[2] * uar2 - uar4 * n[0] - gc * n[1] * qir;
  tmw[1][1] = gc * n[1] * uar2 - n[2];
  tmw[1][2] = gc * n[1] * uar3;
  tmw[1][3] = gc * n[1] * uar4 + n[0];
  tmw[1][4] = -gc * n[1];
  tmw[2][0] = n[2] + n[0] * uar3 - uar2 * n[1] - gc * n[2] * qir;
  tmw[2][1] = gc * n[2] * uar2 + n[1];
  tmw[2][2] = gc * n[2] * uar3 - n[0];
  tmw[2][3] = gc * n[2] * uar4;
  tmw[2][4] = -gc * n[2];
  double crsq = cr * cr;
  tmw[3][0] = gam1 * qir * sRT / (betaRT2 * tRT) + VdotN * crsq / tRT;
  tmw[3][1] = -gam1 * uar2 * sRT / (betaRT2 * tRT) - crsq * n[0] / tRT;
  tmw[3][2] = -gam1 * uar3 * sRT / (betaRT2 * tRT) - crsq * n[1] / tRT;
  tmw[3][3] = -gam1 * uar4 * sRT / (betaRT2 * tRT) - crsq * n[2] / tRT;
  tmw[3][4] = gam1 * sRT / (betaRT2 * tRT);
  tmw[4][0] = -gam1 * qir * rRT / (betaRT2 * tRT) - VdotN * crsq / tRT;
  tmw[4][1] = gam1 * uar2 * rRT / (betaRT2 * tRT) + crsq * n[0] / tRT;
  tmw[4][2] = gam1 * uar3 * rRT / (betaRT2 * tRT) + crsq * n[1] / tRT;
  tmw[4][3] = gam1 * uar4 * rRT / (betaRT2 * tRT) + crsq * n[2] / tRT;
  tmw[4][4] = -gam1 * rRT / (betaRT2 * tRT);
  for (int j = 0; j < 5; ++j) {
    dmat[0][j] = vp1 * (n[0] * tmw[0][j] + n[1] * tmw[1][j] + n[2] * tmw[2][j]) + vp4 * usc2 * tmw[3][j] +
                 vp5 * usc2 * tmw[4][j];
    dmat[1][j] = vp1 * (n[0] * uar2 * tmw[0][j] + (n[1] * uar2 - n[2]) * tmw[1][j] + (n[2] * uar2 + n[1]) * tmw[2][j]) +
                 vp4 * (usc2 * (uar2 + rRT * n[0])) * tmw[3][j] + vp5 * (usc2 * (uar2 + sRT * n[0])) * tmw[4][j];
    dmat[2][j] = vp1 * (n[1] * uar3 * tmw[1][j] + (n[0] * uar3 + n[2]) * tmw[0][j] + (n[2] * uar3 - n[0]) * tmw[2][j]) +
                 vp4 * (usc2 * (uar3 + rRT * n[1])) * tmw[3][j] + vp5 * (usc2 * (uar3 + sRT * n[1])) * tmw[4][j];
    dmat[3][j] = vp1 * (n[2] * uar4 * tmw[2][j] + (n[0] * uar4 - n[1]) * tmw[0][j] + (n[1] * uar4 + n[0]) * tmw[1][j]) +
                 vp4 * (usc2 * (uar4 + rRT * n[2])) * tmw[3][j] + vp5 * (usc2 * (uar4 + sRT * n[2])) * tmw[4][j];
    dmat[4][j] = vp1 * ((n[0] * qir + (n[2] * uar3 - n[1] * uar4)) * tmw[0][j] +
                        (n[1] * qir + (n[0] * uar4 - n[2] * uar2)) * tmw[1][j] +
                        (n[2] * qir + (n[1] * uar2 - n[0] * uar3)) * tmw[2][j]) +
                 vp4 * (usc2 * (enth + VdotN * rRT)) * tmw[3][j] + vp5 * (usc2 * (enth + VdotN * sRT)) * tmw[4][j];
  }
  (void)cr2;
  for (int i = 0; i < 5; ++i)
    for (int k = 0; k < 5; ++k) {
      if (sw == 1) H[i][k] = H[i][k] + dmat[i][k];
      if (sw == 2) H[i][k] = H[i][k] - dmat[i][k];
    }
  for (int i = 0; i < 5; ++i)
    for (int k = 0; k < 5; ++k) jac[5 * i + k] = 0.5 * H[i][k] * rnorm;
}

// FluxFcnFD<5>::computeJacobian (FluxFcnBase.h:112-159) around a face flux,
// then postMultiplyBydVdU (CONSERVATIVE Jacobian type).
static void face_jac_fd(double gam, int code, const double* n3, const double* VL, const double* Ub,
                        double* jac) {
  const double eps0 = 1.e-6;
  double Veps[5], flux[5], fluxeps[5], dfdV[25];
  face_flux(gam, code, n3, VL, Ub, flux);
  for (int k = 0; k < 5; ++k) Veps[k] = VL[k];
  for (int k = 0; k < 5; ++k) {
    double eps = (std::fabs(Veps[k]) < 1.e-10) ? eps0 : eps0 * Veps[k];
    double inveps = 1.0 / eps;
    Veps[k] += eps;
    if (k != 0) Veps[k - 1] = VL[k - 1];
    face_flux(gam, code, n3, Veps, Ub, fluxeps);
    for (int j = 0; j < 5; ++j) dfdV[5 * j + k] = (fluxeps[j] - flux[j]) * inveps;
  }
  post_dVdU(gam, VL, dfdV, jac);
}

// FluxFcnSGWallEuler3D::computeJacobian (FluxFcnDescSG.C:838-886)
static void wall_jac(double gam, const double* n3, double ndot, const double* V, double* jac) {
  double dfdV[25] = {0};
  dfdV[9] = n3[0]; dfdV[14] = n3[1]; dfdV[19] = n3[2]; dfdV[24] = ndot;
  post_dVdU(gam, V, dfdV, jac);
}

// H1 Jacobian in MvpMat layout a[N + 2E][25] (MvpMatrix.h:10-80):
// EdgeSet::computeJacobianFiniteVolumeTerm (Edge.C:4472-4526) with the
// approximate Roe Jacobians roejacappr3Dgas (FluxFcnDescSG.C:155-262),
// Face::computeJacobianFiniteVolumeTerm (Face.C:814-847), diag *= 1/vol
// (SubDomain.C:1760-1765), then TimeState::addToJacobianNoPrecLocal
// (TimeState.C:731-756): A_ii += 1/dt_i (backward Euler, NONDESCRIPTOR).
static void jacobian(const Mesh& m, const double* U, const double* Ub, const double* dt, double* A) {
  const double gam = m.gam;
  const int N = m.N;
  std::vector<double> V(5 * (size_t)N);
  for (int i = 0; i < N; ++i) cons2prim(gam, &U[5 * i], &V[5 * i]);
  std::memset(A, 0, sizeof(double) * 25 * ((size_t)N + 2 * (size_t)m.E));
  for (int l = 0; l < m.E; ++l) {
    int i = m.edges[2 * l], j = m.edges[2 * l + 1];
    const double* nl = &m.edgeNorm[3 * l];
    double nn = std::sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
    if (nn < 1e-18) continue;
    double n[3] = {nl[0], nl[1], nl[2]};
    double dfdUi[25], dfdUj[25];
    roejac6(1.0, gam, 0.0, n, 0.0, &V[5 * i], &V[5 * j], dfdUi, 1);
    roejac6(1.0, gam, 0.0, n, 0.0, &V[5 * j], &V[5 * i], dfdUj, 2);
    double* Aii = &A[25 * (size_t)i];
    double* Ajj = &A[25 * (size_t)j];
    for (int k = 0; k < 25; ++k) { Aii[k] += dfdUi[k]; Ajj[k] -= dfdUj[k]; }
    double* Aij = &A[25 * ((size_t)N + 2 * (size_t)l)];
    double* Aji = &A[25 * ((size_t)N + 2 * (size_t)l + 1)];
    double voli = 1.0 / m.ctrlVol[i];
    double volj = 1.0 / m.ctrlVol[j];
    for (int k = 0; k < 25; ++k) { Aij[k] += dfdUj[k] * voli; Aji[k] -= dfdUi[k] * volj; }
  }
  for (int f = 0; f < m.F; ++f) {
    double n3[3] = {third * m.faceNorm[3 * f], third * m.faceNorm[3 * f + 1], third * m.faceNorm[3 * f + 2]};
    for (int l = 0; l < 3; ++l) {
      int nd = m.faces[3 * f + l];
      double jac[25];
      if (m.codes[f] == BC_SLIP_WALL_MOVING) wall_jac(gam, n3, third * 0.0, &V[5 * nd], jac);
      else face_jac_fd(gam, m.codes[f], n3, &V[5 * nd], Ub, jac);
      double* Aii = &A[25 * (size_t)nd];
      for (int k = 0; k < 25; ++k) Aii[k] += jac[k];
    }
  }
  for (int i = 0; i < N; ++i) {
    double voli = 1.0 / m.ctrlVol[i];
    double* Aii = &A[25 * (size_t)i];
    for (int k = 0; k < 25; ++k) Aii[k] *= voli;
  }
  if (dt) {
    for (int i = 0; i < N; ++i) {
      double c_np1 = 1.0 / dt[i];
      for (int k = 0; k < 5; ++k) A[25 * (size_t)i + 6 * k] += c_np1;
    }
  }
}

// SubDomain::computeMatVecProdH1 / H1transpose (SubDomain.C:3916-3995) with
// DenseMatrixOp::applyAndAddToVector (DenseMatrixOps.h:670-773).
static void matvec(const Mesh& m, const double* A, const double* p, double* y, int transpose) {
  const int N = m.N;
  for (size_t k = 0; k < 5 * (size_t)N; ++k) y[k] = 0.0;
  auto apply = [&](const double* a, const double* x, double* o) {
    for (int r = 0; r < 5; ++r) {
      double s = 0.0;
      for (int c = 0; c < 5; ++c) s += a[5 * r + c] * x[c];
      o[r] += s;
    }
  };
  auto applyT = [&](const double* a, const double* x, double* o) {
    for (int r = 0; r < 5; ++r) {
      double s = 0.0;
      for (int c = 0; c < 5; ++c) s += a[5 * c + r] * x[c];
      o[r] += s;
    }
  };
  for (int i = 0; i < N; ++i) {
    if (!transpose) apply(&A[25 * (size_t)i], &p[5 * i], &y[5 * i]);
    else applyT(&A[25 * (size_t)i], &p[5 * i], &y[5 * i]);
  }
  for (int l = 0; l < m.E; ++l) {
    int i = m.edges[2 * l], j = m.edges[2 * l + 1];
    const double* aij = &A[25 * ((size_t)N + 2 * (size_t)l)];
    const double* aji = &A[25 * ((size_t)N + 2 * (size_t)l + 1)];
    if (!transpose) {
      apply(aij, &p[5 * j], &y[5 * i]);
      apply(aji, &p[5 * i], &y[5 * j]);
    } else {
      applyT(aij, &p[5 * i], &y[5 * j]);
      applyT(aji, &p[5 * j], &y[5 * i]);
    }
  }
}

// invertDenseMatrix (DenseMatrixOps.h:1164-1185): LINPACK dgefa (Gaussian
// elimination, partial pivoting) + dgedi (inverse) on the transposed block.
// Returns the LINPACK info code (k>0: zero pivot at step k).
template <class S>
static int invert5(S* a) {
  const int n = 5;
  S t_[25];
  for (int r = 0; r < 5; ++r)
    for (int c = 0; c < 5; ++c) t_[5 * c + r] = a[5 * r + c];
  // column-major view: A(r,c) = t_[r + 5*c]
  auto A = [&](int r, int c) -> S& { return t_[r + 5 * c]; };
  int ipvt[5];
  for (int k = 0; k < n - 1; ++k) {
    int l = k;
    S mx = std::fabs(A(k, k));
    for (int r = k + 1; r < n; ++r)
      if (std::fabs(A(r, k)) > mx) { mx = std::fabs(A(r, k)); l = r; }
    ipvt[k] = l;
    if (A(l, k) == S(0)) return k + 1;
    if (l != k) std::swap(A(l, k), A(k, k));
    S t = S(-1.0) / A(k, k);
    for (int r = k + 1; r < n; ++r) A(r, k) *= t;
    for (int j = k + 1; j < n; ++j) {
      S tt = A(l, j);
      if (l != k) { A(l, j) = A(k, j); A(k, j) = tt; }
      for (int r = k + 1; r < n; ++r) A(r, j) += tt * A(r, k);
    }
  }
  ipvt[n - 1] = n - 1;
  if (A(n - 1, n - 1) == S(0)) return n;
  // inverse(U)
  for (int k = 0; k < n; ++k) {
    A(k, k) = S(1.0) / A(k, k);
    S t = -A(k, k);
    for (int r = 0; r < k; ++r) A(r, k) *= t;
    for (int j = k + 1; j < n; ++j) {
      S tt = A(k, j);
      A(k, j) = S(0);
      for (int r = 0; r <= k; ++r) A(r, j) += tt * A(r, k);
    }
  }
  // inverse(U) * inverse(L)
  S work[5];
  for (int kb = 1; kb <= n - 1; ++kb) {
    int k = n - 1 - kb;
    for (int i = k + 1; i < n; ++i) { work[i] = A(i, k); A(i, k) = S(0); }
    for (int j = k + 1; j < n; ++j) {
      S tt = work[j];
      for (int r = 0; r < n; ++r) A(r, k) += tt * A(r, j);
    }
    int l = ipvt[k];
    if (l != k)
      for (int r = 0; r < n; ++r) std::swap(A(r, k), A(r, l));
  }
  for (int r = 0; r < 5; ++r)
    for (int c = 0; c < 5; ++c) a[5 * r + c] = t_[5 * c + r];
  return 0;
}

// ---------------------------------------------------------------- GMRES
// GmresSolver::solve (KspSolver.C:351-492) with right preconditioning
// (typePrec = 2), modified Gram-Schmidt and Givens rotations
// (KspSolver.C:917-982).  x starts at 0 (ImplicitCoupledTsDesc.C:292).
// Factors of the block ILU(0) of one operator on one node ordering
// (SparseMat after numericILU): rows in the order perm (perm[i] = node of
// row i), CSR pattern ia/ja of the node graph plus the diagonal, ju the
// diagonal's position, a the L\U blocks with the inverted diagonal.
struct IluFactors {
  int N = 0, bad = 0;
  std::vector<int> perm, ia, ja, ju;
  std::vector<double> a;
};

// Block ILU(0) preconditioner (IluPrec, KspPrec.C:138-330, fill 0):
// SparseMat::numericILU and lusol (SparseMatrix.C:353-450) restated on a
// node ordering: by default the multicolour ordering the GPU uses (greedy
// colouring of the node graph in ascending node order, smallest colour not
// taken by an already coloured neighbour, rows sorted by (colour, node)),
// or the given order; columns of each row ascending in that order.  A is
// the MvpMat layout a[N + 2E][25]; the factored operator is A (transpose =
// 0) or A^T (1).  fp32 != 0 rounds every stored block to float
// (PrecScalar = float), arithmetic in double.  ilu_solve: y = (LU)^-1 x in
// the caller's numbering.  F->bad counts singular diagonal blocks.
static IluFactors* ilu_factor(const Mesh* m, const double* A, int fp32, int transpose, const int* order,
                              int* ncolor_out, int* colour_out) {
  const int N = m->N;
  // neighbours ascending (edges are lexicographic: node -> incident edges
  // ascending gives ascending neighbours)
  std::vector<int> col(N, -1);
  int nc = 0;
  auto nbr = [&](int i, int k) {
    const int l = m->nodeEdgeIdx[k];
    return m->edges[2 * l] == i ? m->edges[2 * l + 1] : m->edges[2 * l];
  };
  for (int i = 0; i < N; ++i) {
    std::vector<char> seen(nc + 1, 0);
    for (int k = m->nodeEdgePtr[i]; k < m->nodeEdgePtr[i + 1]; ++k) {
      const int c = col[nbr(i, k)];
      if (c >= 0) seen[c] = 1;
    }
    int c = 0;
    while (seen[c]) ++c;
    col[i] = c;
    nc = std::max(nc, c + 1);
  }
  if (ncolor_out) *ncolor_out = nc;
  if (colour_out) std::memcpy(colour_out, col.data(), sizeof(int) * N);
  std::vector<int> perm, iperm(N);
  if (order) {
    perm.assign(order, order + N);
  } else {
    for (int c = 0; c < nc; ++c)
      for (int i = 0; i < N; ++i)
        if (col[i] == c) perm.push_back(i);
  }
  for (int i = 0; i < N; ++i) iperm[perm[i]] = i;
  // pattern and blocks in colour order
  std::vector<int> ia(N + 1), ja, ju(N);
  std::vector<double> a;
  auto block = [&](int r, int cnode, double* out) {
    // block (r, cnode) of the operator
    const double* src;
    bool tr = transpose != 0;
    int rr = r, cc = cnode;
    if (tr) std::swap(rr, cc);
    if (rr == cc) {
      src = &A[25 * (size_t)rr];
    } else {
      const int lo = std::min(rr, cc), hi = std::max(rr, cc);
      int l = -1;
      for (int k = m->nodeEdgePtr[lo]; k < m->nodeEdgePtr[lo + 1]; ++k)
        if (nbr(lo, k) == hi) l = m->nodeEdgeIdx[k];
      src = &A[25 * ((size_t)N + 2 * (size_t)l + (rr < cc ? 0 : 1))];
    }
    for (int e = 0; e < 25; ++e) {
      double v = tr ? src[5 * (e % 5) + e / 5] : src[e];
      out[e] = fp32 ? (double)(float)v : v;
    }
  };
  for (int i = 0; i < N; ++i) {
    const int r = perm[i];
    std::vector<int> cols{i};
    for (int k = m->nodeEdgePtr[r]; k < m->nodeEdgePtr[r + 1]; ++k) cols.push_back(iperm[nbr(r, k)]);
    std::sort(cols.begin(), cols.end());
    ia[i] = (int)ja.size();
    for (int c : cols) {
      if (c == i) ju[i] = (int)ja.size();
      ja.push_back(c);
      a.resize(a.size() + 25);
      block(r, perm[c], &a[a.size() - 25]);
    }
  }
  ia[N] = (int)ja.size();
  auto rnd = [&](double v) { return fp32 ? (double)(float)v : v; };
  // numericILU
  int bad = 0;
  std::vector<int> marker(N, -1);
  for (int i = 0; i < N; ++i) {
    for (int k = ia[i]; k < ia[i + 1]; ++k) marker[ja[k]] = k;
    for (int k = ia[i]; k < ju[i]; ++k) {
      const int l = ja[k];
      double mult[25];
      for (int r = 0; r < 5; ++r)
        for (int c = 0; c < 5; ++c) {
          double t = 0.0;
          for (int q = 0; q < 5; ++q) t += a[25 * (size_t)k + 5 * r + q] * a[25 * (size_t)ju[l] + 5 * q + c];
          mult[5 * r + c] = t;
        }
      for (int e = 0; e < 25; ++e) a[25 * (size_t)k + e] = rnd(mult[e]);
      for (int j = ju[l] + 1; j < ia[l + 1]; ++j) {
        const int mm = marker[ja[j]];
        if (mm == -1) continue;
        for (int r = 0; r < 5; ++r)
          for (int c = 0; c < 5; ++c) {
            double t = a[25 * (size_t)mm + 5 * r + c];
            for (int q = 0; q < 5; ++q) t -= mult[5 * r + q] * a[25 * (size_t)j + 5 * q + c];
            a[25 * (size_t)mm + 5 * r + c] = rnd(t);
          }
      }
    }
    for (int k = ia[i]; k < ia[i + 1]; ++k) marker[ja[k]] = -1;
    double d[25];
    for (int e = 0; e < 25; ++e) d[e] = a[25 * (size_t)ju[i] + e];
    if (invert5<double>(d)) ++bad;
    for (int e = 0; e < 25; ++e) a[25 * (size_t)ju[i] + e] = rnd(d[e]);
  }
  IluFactors* F = new IluFactors;
  F->N = N;
  F->bad = bad;
  F->perm = std::move(perm);
  F->ia = std::move(ia);
  F->ja = std::move(ja);
  F->ju = std::move(ju);
  F->a = std::move(a);
  return F;
}

static void ilu_solve(const IluFactors& F, const double* x, double* y) {
  const int N = F.N;
  const std::vector<int>& perm = F.perm;
  const std::vector<int>& ia = F.ia;
  const std::vector<int>& ja = F.ja;
  const std::vector<int>& ju = F.ju;
  const std::vector<double>& a = F.a;
  std::vector<double> w(5 * (size_t)N);
  for (int i = 0; i < N; ++i) {
    double acc[5];
    for (int c = 0; c < 5; ++c) acc[c] = x[5 * (size_t)perm[i] + c];
    for (int k = ia[i]; k < ju[i]; ++k)
      for (int r = 0; r < 5; ++r)
        for (int c = 0; c < 5; ++c) acc[r] -= a[25 * (size_t)k + 5 * r + c] * w[5 * (size_t)ja[k] + c];
    for (int c = 0; c < 5; ++c) w[5 * (size_t)i + c] = acc[c];
  }
  for (int i = N - 1; i >= 0; --i) {
    double acc[5];
    for (int c = 0; c < 5; ++c) acc[c] = w[5 * (size_t)i + c];
    for (int k = ju[i] + 1; k < ia[i + 1]; ++k)
      for (int r = 0; r < 5; ++r)
        for (int c = 0; c < 5; ++c) acc[r] -= a[25 * (size_t)k + 5 * r + c] * w[5 * (size_t)ja[k] + c];
    for (int r = 0; r < 5; ++r) {
      double t = 0.0;
      for (int c = 0; c < 5; ++c) t += a[25 * (size_t)ju[i] + 5 * r + c] * acc[c];
      w[5 * (size_t)i + r] = t;
      y[5 * (size_t)perm[i] + r] = t;
    }
  }
}

struct Operator {
  const Mesh* m;
  const double* A;           // H1 Jacobian (MvpMat layout)
  std::vector<double> Dinv;  // block-Jacobi inverses (FP64 or rounded FP32)
  int transpose = 0;
  const IluFactors* ilu = nullptr;  // when set, the preconditioner instead of Dinv
};

static double dotv(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  for (size_t k = 0; k < a.size(); ++k) s += a[k] * b[k];
  return s;
}

static void bj_apply(const Operator& op, const std::vector<double>& x, std::vector<double>& y) {
  if (op.ilu) {
    ilu_solve(*op.ilu, x.data(), y.data());
    return;
  }
  const int N = op.m->N;
  for (int i = 0; i < N; ++i) {
    const double* d = &op.Dinv[25 * (size_t)i];
    for (int r = 0; r < 5; ++r) {
      double s = 0.0;
      for (int c = 0; c < 5; ++c) s += (op.transpose ? d[5 * c + r] : d[5 * r + c]) * x[5 * i + c];
      y[5 * i + r] = s;
    }
  }
}

static int gmres(const Operator& op, const std::vector<double>& b, std::vector<double>& x, int numVec,
                 int maxits, double eps, double* final_res) {
  const size_t n = b.size();
  std::vector<std::vector<double>> Vb(numVec + 1, std::vector<double>(n));
  std::vector<double> w(n), r(n);
  std::vector<double> H((numVec + 1) * numVec, 0.0), cs(2 * numVec), g(numVec + 1), y(numVec);
  auto h = [&](int i, int j) -> double& { return H[(size_t)i * numVec + j]; };
  int iter = 0, exitLoop = 0;
  double target = 0.0, l2res = 0.0;
  do {
    matvec(*op.m, op.A, x.data(), w.data(), op.transpose);
    for (size_t k = 0; k < n; ++k) r[k] = b[k] - w[k];
    double beta = std::sqrt(dotv(r, r));
    if (iter == 0) target = eps * std::sqrt(dotv(b, b));
    if (beta == 0.0) { if (final_res) *final_res = 0.0; return 0; }
    for (size_t k = 0; k < n; ++k) Vb[0][k] = (1.0 / beta) * r[k];
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int j;
    for (j = 0; j < numVec; ++j) {
      bj_apply(op, Vb[j], r);
      matvec(*op.m, op.A, r.data(), w.data(), op.transpose);
      for (int i = 0; i <= j; ++i) {
        h(i, j) = dotv(w, Vb[i]);
        for (size_t k = 0; k < n; ++k) w[k] -= h(i, j) * Vb[i][k];
      }
      h(j + 1, j) = std::sqrt(dotv(w, w));
      bool breakdown = (h(j + 1, j) == 0.0);
      if (!breakdown)
        for (size_t k = 0; k < n; ++k) Vb[j + 1][k] = (1. / h(j + 1, j)) * w[k];
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
    std::fill(w.begin(), w.end(), 0.0);
    for (int mm = 0; mm <= j; ++mm)
      for (size_t k = 0; k < n; ++k) w[k] += y[mm] * Vb[mm][k];
    bj_apply(op, w, r);
    for (size_t k = 0; k < n; ++k) x[k] += r[k];
  } while (exitLoop == 0);
  if (final_res) *final_res = l2res;
  return iter;
}

}  // namespace orc

using namespace orc;

// ============================================================== C interface
extern "C" {

void* orc_create(int N, int T, int F, const double* X, const int* tets, const int* faces,
                 const int* codes, double gam) {
  Mesh* m = new Mesh();
  m->N = N; m->T = T; m->F = F; m->gam = gam;
  m->X.assign(X, X + 3 * (size_t)N);
  m->tets.assign(tets, tets + 4 * (size_t)T);
  m->faces.assign(faces, faces + 3 * (size_t)F);
  m->codes.assign(codes, codes + F);
  build_edges(*m);
  compute_geometry<double>(*m, m->X.data(), m->edgeNorm, m->faceNorm, m->ctrlVol);
  compute_lsq_R<double>(*m, m->X.data(), m->Rlsq);
  return m;
}

void orc_destroy(void* h) { delete (Mesh*)h; }
int orc_num_edges(void* h) { return ((Mesh*)h)->E; }
void orc_get_edges(void* h, int* e) {
  Mesh* m = (Mesh*)h;
  std::memcpy(e, m->edges.data(), sizeof(int) * 2 * (size_t)m->E);
}
void orc_get_geometry(void* h, double* edgeNorm, double* faceNorm, double* ctrlVol, double* Rlsq) {
  Mesh* m = (Mesh*)h;
  if (edgeNorm) std::memcpy(edgeNorm, m->edgeNorm.data(), sizeof(double) * 3 * (size_t)m->E);
  if (faceNorm) std::memcpy(faceNorm, m->faceNorm.data(), sizeof(double) * 3 * (size_t)m->F);
  if (ctrlVol) std::memcpy(ctrlVol, m->ctrlVol.data(), sizeof(double) * (size_t)m->N);
  if (Rlsq) std::memcpy(Rlsq, m->Rlsq.data(), sizeof(double) * 6 * (size_t)m->N);
}

void orc_prim(void* h, const double* U, double* V) {
  Mesh* m = (Mesh*)h;
  for (int i = 0; i < m->N; ++i) cons2prim(m->gam, &U[5 * i], &V[5 * i]);
}

void orc_gradients(void* h, const double* V, double* ddx, double* ddy, double* ddz) {
  Mesh* m = (Mesh*)h;
  compute_gradients<double>(*m, m->X.data(), m->Rlsq.data(), V, ddx, ddy, ddz);
}

int orc_residual(void* h, const double* U, const double* Ub, int order, double beta, int failsafe,
                 double* R) {
  Mesh* m = (Mesh*)h;
  Work<double> w;
  return residual_t<double>(*m, m->X.data(), m->edgeNorm, m->faceNorm, m->ctrlVol, m->Rlsq, U, Ub,
                            order, beta, failsafe, R, w);
}

// ---------------------------------------------------------------------------
// Viscous (laminar Navier-Stokes) Galerkin term, the SpaceOperator's
// computeGalerkinTerm (SpaceOperator.C:570-573) for tets:
// ElemTet::computeGalerkinTerm (ElemTet.C:24-127, the non-embedded branch)
// with FemEquationTermNS::computeVolumeTerm (FemEquationTermDesc.C:98-160):
// per tet the P1 shape-function gradients (ElemTet::computeGradientP1Function,
// ElemTetCore.C:1961-2010), the velocity and temperature at the nodes and
// their means (NavierStokesTerm.h:205-295), their P1 gradients
// (NavierStokesTerm.h:357-497), the transport coefficients at the mean
// temperature (constant viscosity or Sutherland, ViscoFcn.h:46-103; constant
// Prandtl conductivity kappa = cp mu / Pr, ThermalCondFcn.h:52-75) scaled by
// 1/Re_mu, the stress tensor and heat flux (NavierStokesTerm.h:561-576,
// 647-654), r = (0, tau_kj, u_i tau_ij - q_j) for j = x, y, z
// (NavierStokesTerm.h:690-724), then R[node] += vol (r_0 dN_x + r_1 dN_y +
// r_2 dN_z) for the tet's four nodes in tet order.  Temperature
// T = p/(rho (gamma - 1)) (VarFcnSGEuler.h:120-126, Pstiff = 0).
struct Visc {
  int model = 0;              // 0 inviscid, 1 constant viscosity, 2 Sutherland
  double ooreynolds = 0.0;    // 1 / Re_mu
  double ooprandtl = 0.0;     // 1 / Pr
  double bulk = 0.0;          // bulk viscosity (constant model)
  double alpha = 0.0, Ts = 0.0;  // Sutherland: T = alpha T_adim, Ts
};

static double p1_gradients(const double* X, const int* t, double g[4][3]) {
  const double* x0 = X + 3 * (size_t)t[0];
  const double* x1 = X + 3 * (size_t)t[1];
  const double* x2 = X + 3 * (size_t)t[2];
  const double* x3 = X + 3 * (size_t)t[3];
  double jac[3][3];
  for (int a = 0; a < 3; ++a) {
    jac[a][0] = x1[a] - x0[a];
    jac[a][1] = x2[a] - x0[a];
    jac[a][2] = x3[a] - x0[a];
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
  for (int a = 0; a < 3; ++a) g[0][a] = -(g[1][a] + g[2][a] + g[3][a]);
  return (1.0 / 6.0) * dOmega;
}

static void galerkin_term(const Mesh& m, const double* V, const Visc& vp, double* R) {
  const double gam1 = m.gam - 1.0, invgam1 = 1.0 / gam1, cp = m.gam * invgam1;
  const double fourth = 0.25, twothird = 2.0 / 3.0;
  for (int t = 0; t < m.T; ++t) {
    const int* nd = &m.tets[4 * (size_t)t];
    double g[4][3];
    const double vol = p1_gradients(m.X.data(), nd, g);
    double u[4][3], T[4];
    for (int k = 0; k < 4; ++k) {
      const double* v = V + 5 * (size_t)nd[k];
      u[k][0] = v[1]; u[k][1] = v[2]; u[k][2] = v[3];
      T[k] = invgam1 * (v[4] + 0.0) / v[0];
    }
    double ucg[3];
    for (int a = 0; a < 3; ++a) ucg[a] = fourth * (u[0][a] + u[1][a] + u[2][a] + u[3][a]);
    const double Tcg = fourth * (T[0] + T[1] + T[2] + T[3]);
    double dudxj[3][3], dTdxj[3];
    for (int a = 0; a < 3; ++a)
      for (int j = 0; j < 3; ++j)
        dudxj[a][j] = g[0][j] * u[0][a] + g[1][j] * u[1][a] + g[2][j] * u[2][a] + g[3][j] * u[3][a];
    for (int j = 0; j < 3; ++j) dTdxj[j] = g[0][j] * T[0] + g[1][j] * T[1] + g[2][j] * T[2] + g[3][j] * T[3];
    double mu, lambda;
    if (vp.model == 2) {
      const double Ta = vp.alpha * Tcg;
      mu = Ta * std::sqrt(Ta) * (1.0 + vp.Ts) / (Ta + vp.Ts);
      lambda = -twothird * mu;
    } else {
      mu = 1.0;
      lambda = vp.bulk - twothird * mu;
    }
    double kappa = vp.ooprandtl * cp * mu;
    mu *= vp.ooreynolds;
    lambda *= vp.ooreynolds;
    kappa *= vp.ooreynolds;
    const double div = dudxj[0][0] + dudxj[1][1] + dudxj[2][2];
    double tij[3][3];
    tij[0][0] = lambda * div + 2.0 * mu * dudxj[0][0];
    tij[1][1] = lambda * div + 2.0 * mu * dudxj[1][1];
    tij[2][2] = lambda * div + 2.0 * mu * dudxj[2][2];
    tij[0][1] = mu * (dudxj[1][0] + dudxj[0][1]);
    tij[0][2] = mu * (dudxj[2][0] + dudxj[0][2]);
    tij[1][2] = mu * (dudxj[2][1] + dudxj[1][2]);
    tij[1][0] = tij[0][1];
    tij[2][0] = tij[0][2];
    tij[2][1] = tij[1][2];
    const double qj[3] = {-kappa * dTdxj[0], -kappa * dTdxj[1], -kappa * dTdxj[2]};
    double r[3][5];
    for (int j = 0; j < 3; ++j) {
      r[j][0] = 0.0;
      r[j][1] = tij[0][j];
      r[j][2] = tij[1][j];
      r[j][3] = tij[2][j];
      r[j][4] = ucg[0] * tij[0][j] + ucg[1] * tij[1][j] + ucg[2] * tij[2][j] - qj[j];
    }
    for (int j = 0; j < 4; ++j) {
      double* Rj = R + 5 * (size_t)nd[j];
      for (int k = 0; k < 5; ++k)
        Rj[k] += vol * (r[0][k] * g[j][0] + r[1][k] * g[j][1] + r[2][k] * g[j][2]);
    }
  }
}

// Timed CPU baseline: threaded residual (order 1 or 2, van Albada).
struct Baseline {
  std::vector<double> V, G, priv;
};
void* orc_baseline_create() { return new Baseline(); }
void orc_baseline_destroy(void* b) { delete (Baseline*)b; }
void orc_residual_threaded(void* h, void* b, const double* U, const double* Ub, int order, int nthreads,
                           double* R) {
  Mesh* m = (Mesh*)h;
  Baseline* bl = (Baseline*)b;
  residual_threaded(*m, U, Ub, order, 1.0 / 3.0, nthreads, R, bl->V, bl->G, bl->priv);
}

// Residual with the viscous Galerkin term: (R_fv + G) / ctrlVol, evaluated
// as R_fv / ctrlVol + G / ctrlVol.  model, ooreynolds, ooprandtl, bulk,
// alpha, Ts as in Visc.
int orc_residual_visc(void* h, const double* U, const double* Ub, int order, int model, double ooreynolds,
                      double ooprandtl, double bulk, double alpha, double Ts, double* R) {
  Mesh* m = (Mesh*)h;
  const int bad = orc_residual(h, U, Ub, order, 1.0 / 3.0, 0, R);
  if (model == 0) return bad;
  Visc vp;
  vp.model = model; vp.ooreynolds = ooreynolds; vp.ooprandtl = ooprandtl; vp.bulk = bulk;
  vp.alpha = alpha; vp.Ts = Ts;
  std::vector<double> V(5 * (size_t)m->N), G(5 * (size_t)m->N, 0.0);
  for (int i = 0; i < m->N; ++i) cons2prim(m->gam, &U[5 * (size_t)i], &V[5 * (size_t)i]);
  galerkin_term(*m, V.data(), vp, G.data());
  for (int i = 0; i < m->N; ++i)
    for (int k = 0; k < 5; ++k) R[5 * (size_t)i + k] += G[5 * (size_t)i + k] / m->ctrlVol[i];
  return bad;
}

// ---------------------------------------------------------------------------
// Spalart-Allmaras turbulence model, strongly coupled (state U = (rho, rho
// u, rho v, rho w, E, rho nu~), dim 6).  The finite-volume term is the
// Euler path's on six components:
// * VarFcnSGSA::conservativeToPrimitive (VarFcnSGSA.h:210-224): V[5] =
//   U[5] / rho;
// * LSQ gradients and the reconstruction componentwise (the same
//   SubDomain::computeGradientsLeastSquares and RecFcn functions on dim
//   6), the positivity check on the reconstructed density and pressure;
// * the Roe flux FluxFcnSGApprJacRoeSA3D::compute (FluxFcnDescSG.C:
//   1886-1901) = roeflux7.f with type 1: phi(6) = phi(1) (updir nu~_L +
//   (1 - updir) nu~_R), updir = 0.5 + sign(0.5, phi(1)) (roeflux7.f:
//   190-196);
// * slip walls FluxFcnSGWallSA3D::compute (FluxFcnDescSG.C:2024-2035:
//   flux[5] = 0); inlet and outlet both FluxFcnSGOutflowSA3D (FluxFcn.h:
//   246-262) = boundflux5.f with type 1: flux(6) = phiro (updir nu~ + (1 -
//   updir) (rho nu~)_b / rho_b), phiro = flux(1) (boundflux5.f:92-103).
// The Galerkin term is FemEquationTermSA::computeVolumeTerm
// (FemEquationTermDesc.C:669-787) assembled by ElemTet::computeGalerkinTerm
// (ElemTet.C:99-114, R += vol (r . dN_j) - vol/4 s): the laminar
// coefficients at the tet's mean temperature, mu~ = mean(rho nu~),
// mu_t = mu~ fv1 (SATerm::computeTurbulentViscosity,
// SpalartAllmarasTerm.h:139-151), lambda_t = -2/3 mu_t, kappa_t = cp mu_t /
// Pr_t (ConstantPrandtlThermalCondFcn::turbulentConductivity,
// ThermalCondFcn.h:84-87), the Navier-Stokes stress and heat flux with mu
// + mu_t, lambda + lambda_t, kappa + kappa_t scaled by 1/Re, the SA
// diffusion r[j][5] = (mul + |mu~|) / (sigma Re) dnu~/dx_j and the source
// s[5] = cb2/(sigma Re) rho |grad nu~|^2 + cb1 S~ |mu~| - cw1/Re fw
// max(mu~,0)^2 / (rho d^2) (production with S~ = max(s fv3 + zz fv2,
// 1e-12), zz = max(mu~,0) / (Re kappa^2 rho d^2); destruction with r =
// min(zz / S~, 2), g = r + cw2 (r^6 - r), fw = g ((1 + cw3^6) / (g^6 +
// cw3^6))^(1/6)), applied when the tet's mean wall distance is >= 1e-15
// (constants as SATerm::SATerm, SpalartAllmarasTerm.h:77-112).  No trip
// (its box is empty by default), no porous media, no wall functions.
struct SAParams {
  double cb1, cb2, cw2, cw3, cv1, cv2, sigma, vkcst, prandtl_t;
  int fv3;
};

// roeflux7 with type 1 (six components)
static void roeflux7_sa(double gam, const double* n, const double* Vg, const double* Vd, double* phi) {
  roeflux7<double>(gam, 0.0, n, 0.0, Vg, Vd, phi);
  const double updir = 0.5 + std::copysign(0.5, phi[0]);
  phi[5] = phi[0] * (updir * Vg[5] + (1.0 - updir) * Vd[5]);
}

// the SA boundary fluxes (wall, or boundflux5 with type 1)
static void face_flux_sa(double gam, int code, const double* n3, const double* V, const double* Ub, double* flux) {
  face_flux<double>(gam, code, n3, V, Ub, flux);
  if (code == BC_SLIP_WALL_MOVING) {
    flux[5] = 0.0;
  } else {
    const double phiro = flux[0];
    const double updir = 0.5 + std::copysign(0.5, phiro);
    const double usro = 1.0 / Ub[0];
    flux[5] = phiro * (updir * V[5] + (1.0 - updir) * Ub[5] * usro);
  }
}

static void galerkin_term_sa(const Mesh& m, const double* V, const Visc& vp, const SAParams& sa,
                             const double* d2wall, double* R) {
  const double gam1 = m.gam - 1.0, invgam1 = 1.0 / gam1, cp = m.gam * invgam1;
  const double fourth = 0.25, twothird = 2.0 / 3.0, sixth_ = 1.0 / 6.0;
  const double oorey = vp.ooreynolds;
  const double oovkcst2 = 1.0 / (sa.vkcst * sa.vkcst);
  const double cw3_pow6 = std::pow(sa.cw3, 6.0);
  const double opcw3_pow = std::pow(1.0 + cw3_pow6, 1.0 / 6.0);
  const double cv1_pow3 = sa.cv1 * sa.cv1 * sa.cv1;
  const double oocv2 = 1.0 / sa.cv2;
  const double oosigma = 1.0 / sa.sigma * oorey;
  const double cw1 = (sa.cb1 * oovkcst2 + (1.0 + sa.cb2) / sa.sigma) * oorey;
  for (int t = 0; t < m.T; ++t) {
    const int* nd = &m.tets[4 * (size_t)t];
    double g[4][3];
    const double vol = p1_gradients(m.X.data(), nd, g);
    const double* v[4];
    double u[4][3], T[4];
    for (int k = 0; k < 4; ++k) {
      v[k] = V + 6 * (size_t)nd[k];
      u[k][0] = v[k][1]; u[k][1] = v[k][2]; u[k][2] = v[k][3];
      T[k] = invgam1 * v[k][4] / v[k][0];
    }
    double ucg[3];
    for (int a = 0; a < 3; ++a) ucg[a] = fourth * (u[0][a] + u[1][a] + u[2][a] + u[3][a]);
    const double Tcg = fourth * (T[0] + T[1] + T[2] + T[3]);
    double dudxj[3][3], dTdxj[3];
    for (int a = 0; a < 3; ++a)
      for (int j = 0; j < 3; ++j)
        dudxj[a][j] = g[0][j] * u[0][a] + g[1][j] * u[1][a] + g[2][j] * u[2][a] + g[3][j] * u[3][a];
    for (int j = 0; j < 3; ++j) dTdxj[j] = g[0][j] * T[0] + g[1][j] * T[1] + g[2][j] * T[2] + g[3][j] * T[3];
    // laminar coefficients (not yet scaled by 1/Re)
    double mul, lambdal;
    if (vp.model == 2) {
      const double Ta = vp.alpha * Tcg;
      mul = Ta * std::sqrt(Ta) * (1.0 + vp.Ts) / (Ta + vp.Ts);
      lambdal = -twothird * mul;
    } else {
      mul = 1.0;
      lambdal = vp.bulk - twothird * mul;
    }
    const double kappal = vp.ooprandtl * cp * mul;
    // turbulent coefficients
    const double mutilde = 0.25 * (v[0][0] * v[0][5] + v[1][0] * v[1][5] + v[2][0] * v[2][5] + v[3][0] * v[3][5]);
    const double chi0 = mutilde / mul;
    const double chi03 = chi0 * chi0 * chi0;
    const double mut = mutilde * (chi03 / (chi03 + cv1_pow3));
    const double lambdat = -2.0 * mut / 3.0;
    const double kappat = cp * mut / sa.prandtl_t;
    double r[3][6], s5 = 0.0;
    const double absmutilde = std::fabs(mutilde), maxmutilde = std::max(mutilde, 0.0);
    const double mu5 = oosigma * (mul + absmutilde);
    double dnu[3];
    for (int j = 0; j < 3; ++j) dnu[j] = g[0][j] * v[0][5] + g[1][j] * v[1][5] + g[2][j] * v[2][5] + g[3][j] * v[3][5];
    for (int j = 0; j < 3; ++j) r[j][5] = mu5 * dnu[j];
    const double d2w = 0.25 * (d2wall[nd[0]] + d2wall[nd[1]] + d2wall[nd[2]] + d2wall[nd[3]]);
    if (d2w >= 1.e-15) {
      const double chi = std::max(mutilde / mul, 0.001);
      const double chi3 = chi * chi * chi;
      const double fv1 = chi3 / (chi3 + cv1_pow3);
      double fv2 = 1. - chi / (1. + chi * fv1);
      double fv3 = 1.0;
      if (sa.fv3) {
        fv2 = 1.0 + oocv2 * chi;
        fv2 = 1.0 / (fv2 * fv2 * fv2);
        fv3 = (1.0 + chi * fv1) * (1.0 - fv2) / chi;
      }
      const double ood2wall2 = 1.0 / (d2w * d2w);
      const double rho = 0.25 * (v[0][0] + v[1][0] + v[2][0] + v[3][0]);
      const double oorho = 1.0 / rho;
      const double zz = oorey * oovkcst2 * maxmutilde * oorho * ood2wall2;
      const double s12 = dudxj[0][1] - dudxj[1][0];
      const double s23 = dudxj[1][2] - dudxj[2][1];
      const double s31 = dudxj[2][0] - dudxj[0][2];
      const double sv = std::sqrt(s12 * s12 + s23 * s23 + s31 * s31);
      const double Stilde = std::max(sv * fv3 + zz * fv2, 1.0e-12);
      const double rr = std::min(zz / Stilde, 2.0);
      const double rr2 = rr * rr;
      const double gg = rr + sa.cw2 * (rr2 * rr2 * rr2 - rr);
      const double gg2 = gg * gg;
      const double fw = opcw3_pow * gg * std::pow(gg2 * gg2 * gg2 + cw3_pow6, -sixth_);
      const double AA = oosigma * sa.cb2 * rho * (dnu[0] * dnu[0] + dnu[1] * dnu[1] + dnu[2] * dnu[2]);
      const double BB = sa.cb1 * Stilde * absmutilde;
      const double CC = -cw1 * fw * oorho * maxmutilde * maxmutilde * ood2wall2;
      s5 = AA + BB + CC;
    }
    // NavierStokesTerm::computeVolumeTermNS with the summed coefficients
    const double mu = oorey * (mul + mut), lambda = oorey * (lambdal + lambdat), kappa = oorey * (kappal + kappat);
    const double div = dudxj[0][0] + dudxj[1][1] + dudxj[2][2];
    double tij[3][3];
    tij[0][0] = lambda * div + 2.0 * mu * dudxj[0][0];
    tij[1][1] = lambda * div + 2.0 * mu * dudxj[1][1];
    tij[2][2] = lambda * div + 2.0 * mu * dudxj[2][2];
    tij[0][1] = mu * (dudxj[1][0] + dudxj[0][1]);
    tij[0][2] = mu * (dudxj[2][0] + dudxj[0][2]);
    tij[1][2] = mu * (dudxj[2][1] + dudxj[1][2]);
    tij[1][0] = tij[0][1];
    tij[2][0] = tij[0][2];
    tij[2][1] = tij[1][2];
    for (int j = 0; j < 3; ++j) {
      r[j][0] = 0.0;
      r[j][1] = tij[0][j];
      r[j][2] = tij[1][j];
      r[j][3] = tij[2][j];
      r[j][4] = ucg[0] * tij[0][j] + ucg[1] * tij[1][j] + ucg[2] * tij[2][j] - (-kappa * dTdxj[j]);
    }
    for (int j = 0; j < 4; ++j) {
      double* Rj = R + 6 * (size_t)nd[j];
      for (int k = 0; k < 6; ++k)
        Rj[k] += vol * ((r[0][k] * g[j][0] + r[1][k] * g[j][1] + r[2][k] * g[j][2]) - (k == 5 ? fourth * s5 : 0.0));
    }
  }
}

// Spalart-Allmaras residual (R_fv + G) / ctrlVol of U [N][6], evaluated as
// R_fv / ctrlVol + G / ctrlVol; Ub [6] conservative free stream; sa = (cb1,
// cb2, cw2, cw3, cv1, cv2, sigma, vkcst, Pr_t); d2wall [N].  Returns the
// number of non-positive reconstructed states.
int orc_residual_sa(void* h, const double* U, const double* Ub, int order, int model, double ooreynolds,
                    double ooprandtl, double bulk, double alpha, double Ts, const double* sa, int fv3,
                    const double* d2wall, double* R) {
  Mesh* mp = (Mesh*)h;
  const Mesh& m = *mp;
  const int N = m.N;
  const double gam = m.gam;
  std::vector<double> V(6 * (size_t)N);
  for (int i = 0; i < N; ++i) {
    const double* u = U + 6 * (size_t)i;
    double* v = &V[6 * (size_t)i];
    v[0] = u[0];
    const double invRho = 1.0 / u[0];
    v[1] = u[1] * invRho;
    v[2] = u[2] * invRho;
    v[3] = u[3] * invRho;
    const double vel2 = v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
    v[4] = (gam - 1.0) * (u[4] - 0.5 * u[0] * vel2) - gam * 0.0;
    v[5] = u[5] * invRho;
  }
  const double* X = m.X.data();
  std::vector<double> ddx(6 * (size_t)N, 0.0), ddy(6 * (size_t)N, 0.0), ddz(6 * (size_t)N, 0.0);
  if (order > 1)
    for (int l = 0; l < m.E; ++l) {
      const int i = m.edges[2 * l], j = m.edges[2 * l + 1];
      double Wi[3], Wj[3];
      double dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
      lsq_weights(dx, &m.Rlsq[6 * (size_t)i], Wi);
      dx[0] = -dx[0]; dx[1] = -dx[1]; dx[2] = -dx[2];
      lsq_weights(dx, &m.Rlsq[6 * (size_t)j], Wj);
      for (int k = 0; k < 6; ++k) {
        const double dv = V[6 * (size_t)j + k] - V[6 * (size_t)i + k];
        ddx[6 * (size_t)i + k] += Wi[0] * dv;
        ddy[6 * (size_t)i + k] += Wi[1] * dv;
        ddz[6 * (size_t)i + k] += Wi[2] * dv;
        ddx[6 * (size_t)j + k] -= Wj[0] * dv;
        ddy[6 * (size_t)j + k] -= Wj[1] * dv;
        ddz[6 * (size_t)j + k] -= Wj[2] * dv;
      }
    }
  RecParams rp = rec_params(order == 1 ? 0.0 : 1.0 / 3.0);
  std::fill(R, R + 6 * (size_t)N, 0.0);
  int ierr = 0;
  for (int l = 0; l < m.E; ++l) {
    const int i = m.edges[2 * l], j = m.edges[2 * l + 1];
    const double dx[3] = {X[3 * j] - X[3 * i], X[3 * j + 1] - X[3 * i + 1], X[3 * j + 2] - X[3 * i + 2]};
    double Vi[6], Vj[6];
    for (int k = 0; k < 6; ++k) {
      const double vi = V[6 * (size_t)i + k], vj = V[6 * (size_t)j + k];
      if (order == 1) { Vi[k] = vi; Vj[k] = vj; continue; }
      const double ddVij = dx[0] * ddx[6 * (size_t)i + k] + dx[1] * ddy[6 * (size_t)i + k] + dx[2] * ddz[6 * (size_t)i + k];
      const double ddVji = dx[0] * ddx[6 * (size_t)j + k] + dx[1] * ddy[6 * (size_t)j + k] + dx[2] * ddz[6 * (size_t)j + k];
      if (order == 2) vanalbada(rp, vi, ddVij, vj, ddVji, Vi[k], Vj[k]);
      else linear_rec(rp, vi, ddVij, vj, ddVji, Vi[k], Vj[k]);
    }
    const bool bi = Vi[0] <= 0.0 || Vi[4] <= 0.0;
    const bool bj = Vj[0] <= 0.0 || Vj[4] <= 0.0;
    if (bi || bj) { ierr += (int)bi + (int)bj; continue; }
    const double* nl = &m.edgeNorm[3 * (size_t)l];
    if (std::sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]) < 1e-18) continue;
    double flux[6];
    roeflux7_sa(gam, nl, Vi, Vj, flux);
    for (int k = 0; k < 6; ++k) { R[6 * (size_t)i + k] += flux[k]; R[6 * (size_t)j + k] -= flux[k]; }
  }
  for (int f = 0; f < m.F; ++f) {
    const double n3[3] = {third * m.faceNorm[3 * f], third * m.faceNorm[3 * f + 1], third * m.faceNorm[3 * f + 2]};
    for (int l = 0; l < 3; ++l) {
      const int nd = m.faces[3 * f + l];
      double flux[6];
      face_flux_sa(gam, m.codes[f], n3, &V[6 * (size_t)nd], Ub, flux);
      for (int k = 0; k < 6; ++k) R[6 * (size_t)nd + k] += flux[k];
    }
  }
  for (int i = 0; i < N; ++i) {
    const double invcv = 1.0 / m.ctrlVol[i];
    for (int k = 0; k < 6; ++k) R[6 * (size_t)i + k] *= invcv;
  }
  if (model == 0) return ierr;
  Visc vp;
  vp.model = model; vp.ooreynolds = ooreynolds; vp.ooprandtl = ooprandtl; vp.bulk = bulk;
  vp.alpha = alpha; vp.Ts = Ts;
  SAParams sp{sa[0], sa[1], sa[2], sa[3], sa[4], sa[5], sa[6], sa[7], sa[8], fv3};
  std::vector<double> G(6 * (size_t)N, 0.0);
  galerkin_term_sa(m, V.data(), vp, sp, d2wall, G.data());
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 6; ++k) R[6 * (size_t)i + k] += G[6 * (size_t)i + k] / m.ctrlVol[i];
  return ierr;
}

void orc_roeflux7_sa(double gam, const double* n, const double* Vi, const double* Vj, double* phi) {
  roeflux7_sa(gam, n, Vi, Vj, phi);
}
void orc_face_flux_sa(double gam, int code, const double* n3, const double* V, const double* Ub, double* flux) {
  face_flux_sa(gam, code, n3, V, Ub, flux);
}

void orc_timestep(void* h, const double* U, double cfl, double* dt) { timestep(*(Mesh*)h, U, cfl, dt); }

// ExplicitTsDesc::computeRKSecondOrder (ExplicitTsDesc.C:98-117) with local
// time stepping (TimeData.C:11-18 for a steady problem):
// k1 = dt R(U); U0 = U - k1; k2 = dt R(U0); U = U - 1/2 (k1 + k2).
void orc_rk2(void* h, double* U, const double* Ub, int order, double cfl, int nsteps) {
  Mesh* m = (Mesh*)h;
  const size_t n5 = 5 * (size_t)m->N;
  std::vector<double> dt(m->N), k1(n5), k2(n5), U0(n5);
  for (int s = 0; s < nsteps; ++s) {
    timestep(*m, U, cfl, dt.data());
    orc_residual(h, U, Ub, order, 1.0 / 3.0, 0, k1.data());
    for (int i = 0; i < m->N; ++i)
      for (int k = 0; k < 5; ++k) k1[5 * i + k] *= dt[i];
    for (size_t k = 0; k < n5; ++k) U0[k] = U[k] - k1[k];
    orc_residual(h, U0.data(), Ub, order, 1.0 / 3.0, 0, k2.data());
    for (int i = 0; i < m->N; ++i)
      for (int k = 0; k < 5; ++k) k2[5 * i + k] *= dt[i];
    for (size_t k = 0; k < n5; ++k) U[k] = U[k] - 1.0 / 2.0 * (k1[k] + k2[k]);
  }
}

void orc_roeflux7(double gam, const double* n, double ndot, const double* Vi, const double* Vj,
                  double* phi) {
  roeflux7<double>(gam, 0.0, n, ndot, Vi, Vj, phi);
}
void orc_boundflux5(double gam, const double* n, double sig, const double* V, const double* Ub,
                    double* flux) {
  boundflux5<double>(gam, n, sig, V, Ub, flux);
}
void orc_roejac6(double gam, const double* n, const double* Vi, const double* Vj, double* jacL,
                 double* jacR) {
  double nn[3] = {n[0], n[1], n[2]};
  roejac6(1.0, gam, 0.0, nn, 0.0, Vi, Vj, jacL, 1);
  roejac6(1.0, gam, 0.0, nn, 0.0, Vj, Vi, jacR, 2);
}
void orc_vanalbada(double beta, const double* Vi, const double* ddVij, const double* Vj,
                   const double* ddVji, double* Vij, double* Vji) {
  RecParams p = rec_params(beta);
  for (int k = 0; k < 5; ++k) vanalbada(p, Vi[k], ddVij[k], Vj[k], ddVji[k], Vij[k], Vji[k]);
}
void orc_linear_rec(double beta, const double* Vi, const double* ddVij, const double* Vj,
                    const double* ddVji, double* Vij, double* Vji) {
  RecParams p = rec_params(beta);
  for (int k = 0; k < 5; ++k) linear_rec(p, Vi[k], ddVij[k], Vj[k], ddVji[k], Vij[k], Vji[k]);
}
void orc_cons2prim(double gam, const double* U, double* V) { cons2prim<double>(gam, U, V); }
void orc_post_dVdU(double gam, const double* V, const double* mat, double* res) { post_dVdU(gam, V, mat, res); }
int orc_invert5(double* a) { return invert5<double>(a); }
int orc_invert5f(float* a) { return invert5<float>(a); }

void orc_jacobian(void* h, const double* U, const double* Ub, const double* dt, double* A) {
  jacobian(*(Mesh*)h, U, Ub, dt, A);
}
void orc_matvec(void* h, const double* A, const double* p, double* y, int transpose) {
  matvec(*(Mesh*)h, A, p, y, transpose);
}

// Block-Jacobi inverses of the diagonal blocks (JacobiPrec::setup,
// KspPrec.C:75-82; DiagMat::invert, DiagMatrix.C:44-80). fp32 != 0 stores
// the blocks as float before inverting (PrecScalar = float,
// CMakeLists.txt:654).  Returns the number of singular blocks.
int orc_bj_invert(void* h, const double* A, double* Dinv, int fp32) {
  Mesh* m = (Mesh*)h;
  int bad = 0;
  for (int i = 0; i < m->N; ++i) {
    if (fp32) {
      float a[25];
      for (int k = 0; k < 25; ++k) a[k] = (float)A[25 * (size_t)i + k];
      if (invert5<float>(a)) ++bad;
      for (int k = 0; k < 25; ++k) Dinv[25 * (size_t)i + k] = a[k];
    } else {
      double a[25];
      for (int k = 0; k < 25; ++k) a[k] = A[25 * (size_t)i + k];
      if (invert5<double>(a)) ++bad;
      for (int k = 0; k < 25; ++k) Dinv[25 * (size_t)i + k] = a[k];
    }
  }
  return bad;
}

int orc_ilu0(void* h, const double* A, int fp32, int transpose, const double* x, double* y, int* ncolor_out,
             int* colour_out) {
  IluFactors* F = ilu_factor((Mesh*)h, A, fp32, transpose, nullptr, ncolor_out, colour_out);
  if (!F) return -1;
  ilu_solve(*F, x, y);
  const int bad = F->bad;
  delete F;
  return bad;
}

// The same factorisation kept for repeated solves, on the multicolour
// order (order == null) or on a given node order (order[i] = node of row
// i, e.g. the reverse Cuthill-McKee order of orc_rcm_order).
void* orc_ilu_factor(void* h, const double* A, int fp32, int transpose, const int* order, int* bad) {
  IluFactors* F = ilu_factor((Mesh*)h, A, fp32, transpose, order, nullptr, nullptr);
  if (bad) *bad = F ? F->bad : -1;
  return F;
}
void orc_ilu_apply(void* f, const double* x, double* y) { ilu_solve(*(IluFactors*)f, x, y); }
void orc_ilu_free(void* f) { delete (IluFactors*)f; }

// Reverse Cuthill-McKee order of the ILU(0) rows, as the reference
// renumbers a subdomain's ILU matrix (PcData::renumbering = RCM,
// IoDataCore.C:2744-2745; SubDomain::createMaskILU, SubDomain.C:3371-3390):
// the node graph with each node's own entry, neighbours ascending
// (SubDomain::createEdgeBasedConnectivity, SubDomainCore.C:253-318), one
// connected component after another from the lowest-numbered unvisited node
// (Connectivity::renumByComponent), each renumbered by renumRCM
// (ConnectivityCore.C:582-626): a pseudo-peripheral end node from
// findPseudoDiam (:324-383, rooted level structures of rootLS, :386-420),
// breadth-first from it with neighbours in ascending order, then reversed.
// renumRCM's sort of each new level segment by degree swaps nothing
// (order[k] is written twice), so neighbours keep their ascending order, as
// in the reference.  order[r] = node of row r.
namespace {
struct NodeGraph {
  int n;
  std::vector<int> ptr, tgt;  // with the node's own entry, ascending
  int num(int i, const std::vector<int>& mask) const {
    int r = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k)
      if (mask[tgt[k]]) ++r;
    return r;
  }
  // rooted level structure: ls (levels xls[0..h]), width w; returns h
  int rootLS(int root, std::vector<int>& xls, std::vector<int>& ls, int& w, const std::vector<int>& mask) const {
    std::vector<int> loc(mask);
    w = 0;
    loc[root] = 0;
    ls[0] = root;
    xls[0] = 0;
    int nlvl = 1, nf = 1;
    while (nf > xls[nlvl - 1]) {
      xls[nlvl] = nf;
      const int lb = xls[nlvl - 1], le = xls[nlvl];
      for (int i = lb; i < le; ++i) {
        const int n1 = ls[i];
        for (int k = ptr[n1]; k < ptr[n1 + 1]; ++k) {
          const int n2 = tgt[k];
          if (loc[n2]) { loc[n2] = 0; ls[nf++] = n2; }
        }
      }
      if (nf - xls[nlvl] > w) w = nf - xls[nlvl];
      ++nlvl;
    }
    return nlvl - 1;
  }
};
}  // namespace

void orc_rcm_order(void* h, int* order) {
  Mesh* m = (Mesh*)h;
  const int N = m->N;
  NodeGraph G;
  G.n = N;
  G.ptr.assign(N + 1, 0);
  for (int i = 0; i < N; ++i) G.ptr[i + 1] = G.ptr[i] + 1 + (m->nodeEdgePtr[i + 1] - m->nodeEdgePtr[i]);
  G.tgt.resize(G.ptr[N]);
  for (int i = 0; i < N; ++i) {
    int q = G.ptr[i];
    G.tgt[q++] = i;
    for (int k = m->nodeEdgePtr[i]; k < m->nodeEdgePtr[i + 1]; ++k) {
      const int l = m->nodeEdgeIdx[k];
      G.tgt[q++] = m->edges[2 * l] == i ? m->edges[2 * l + 1] : m->edges[2 * l];
    }
    std::stable_sort(G.tgt.begin() + G.ptr[i], G.tgt.begin() + G.ptr[i + 1]);
  }
  std::vector<int> mark(N, 1), renum(N, -1), ls(N), xls(N + 1), loc(N, 0), all(N, 1);
  int next = 0;
  for (int inode = 0; inode < N; ++inode) {
    if (!mark[inode]) continue;
    int w;
    const int hc = G.rootLS(inode, xls, ls, w, all);  // the component of inode
    for (int j = 0; j < xls[hc]; ++j) { loc[ls[j]] = 1; mark[ls[j]] = 0; }
    // findPseudoDiam on the component
    int s = 0, e = 0, cmin = G.ptr[N] + 1, cmax = 0;
    for (int i = 0; i < N; ++i)
      if (loc[i]) {
        const int nw = G.num(i, loc);
        if (nw < cmin) { cmin = nw; s = i; }
        if (nw > cmax) cmax = nw;
      }
    int hh = G.rootLS(s, xls, ls, w, loc);
    const int sub = xls[hh];
    e = ls[xls[hh - 1]];
    std::vector<int> sorted(cmax + 1);
    while (hh < sub) {
      std::fill(sorted.begin(), sorted.end(), -1);
      for (int k = xls[hh - 1]; k < xls[hh]; ++k) sorted[G.num(ls[k], loc)] = ls[k];
      int w_e = sub, k;
      for (k = 0; k <= cmax; ++k)
        if (sorted[k] >= 0) {
          const int nh = G.rootLS(sorted[k], xls, ls, w, loc);
          if (w < w_e) {
            if (nh > hh) { s = sorted[k]; hh = nh; break; }
            e = sorted[k];
            w_e = w;
          }
        }
      if (k > cmax) break;
    }
    // renumRCM from e
    std::vector<int> sign(loc), ord;
    ord.push_back(e);
    sign[e] = -sign[e];
    for (size_t i = 0; i < ord.size(); ++i) {
      const int cur = ord[i];
      for (int k = G.ptr[cur]; k < G.ptr[cur + 1]; ++k) {
        const int nb = G.tgt[k];
        if (sign[nb] > 0) { ord.push_back(nb); sign[nb] = -sign[nb]; }
      }
    }
    for (size_t i = ord.size(); i--;) renum[ord[i]] = next++;
    for (int j = 0; j < N; ++j) loc[j] = 0;
  }
  for (int i = 0; i < N; ++i) order[renum[i]] = i;
}

// Right-preconditioned GMRES with the block ILU(0) factors f (orc_ilu_factor)
// as the preconditioner, otherwise as orc_gmres.
int orc_gmres_ilu(void* h, const double* A, void* f, const double* b, double* x, int numVec, int maxits,
                  double eps, int transpose, double* final_res) {
  Mesh* m = (Mesh*)h;
  Operator op;
  op.m = m; op.A = A; op.transpose = transpose;
  op.ilu = (const IluFactors*)f;
  std::vector<double> bb(b, b + 5 * (size_t)m->N), xx(5 * (size_t)m->N, 0.0);
  int its = gmres(op, bb, xx, numVec, maxits, eps, final_res);
  std::memcpy(x, xx.data(), sizeof(double) * xx.size());
  return its;
}

int orc_gmres(void* h, const double* A, const double* Dinv, const double* b, double* x, int numVec,
              int maxits, double eps, int transpose, double* final_res) {
  Mesh* m = (Mesh*)h;
  Operator op;
  op.m = m; op.A = A; op.transpose = transpose;
  op.Dinv.assign(Dinv, Dinv + 25 * (size_t)m->N);
  std::vector<double> bb(b, b + 5 * (size_t)m->N), xx(5 * (size_t)m->N, 0.0);
  int its = gmres(op, bb, xx, numVec, maxits, eps, final_res);
  std::memcpy(x, xx.data(), sizeof(double) * xx.size());
  return its;
}

// Pseudo-transient Newton (TsSolver::resolve, TsSolver.h:231-380;
// NewtonSolver::solve with maxIts=1, NewtonSolver.h:70-231;
// ImplicitCoupledTsDesc::computeJacobian/setOperators/solveLinearSystem,
// ImplicitCoupledTsDesc.C:85-300) with the RESIDUAL CFL law
// (TsParameters.C:182-217,290): cfl *= (res_{k-1}/res_k)^ser, clipped to
// [cflMin, cflMax].  The Jacobian is the first-order H1 approximation in
// FP64; block-Jacobi in FP32 (fp32_prec) or FP64.  Stops when
// ||R(Q)||/||R(Q0)|| <= tol or after max_steps.  history (max_steps+1
// entries) receives the relative residuals; returns the steps taken.
//
// After every update the physical-solution check (NewtonSolver.h:187-215,
// SubDomain::checkSolution SubDomain.C:6746-6806): a node value with a
// non-positive density or pressure restores the state and the step is
// redone at half the CFL number (TsParameters::computeCflNumber,
// TsParameters.C:187-195); below cfl0/1000 the reference aborts, here the
// call returns -7.  *redos (optional) counts the redone steps.
int orc_newton(void* h, double* U, const double* Ub, int order, double cfl0, double cflMin,
               double cflMax, double ser, int numVec, int maxits, double eps, double tol,
               int max_steps, int fp32_prec, double* history, int* lin_its, int* redos) {
  Mesh* m = (Mesh*)h;
  const int N = m->N;
  const size_t n5 = 5 * (size_t)N;
  std::vector<double> R(n5), rhs(n5), dt(N), A(25 * ((size_t)N + 2 * (size_t)m->E)), Dinv(25 * (size_t)N),
      dQ(n5), Uprev(n5);
  double res0 = 0.0, cfl = cfl0, rel_prev = 1.0;
  int k = 0, nredo = 0;
  bool redo = false;
  if (redos) *redos = 0;
  while (k <= max_steps) {
    if (!redo) {
      orc_residual(h, U, Ub, order, 1.0 / 3.0, 0, R.data());
      double res = std::sqrt(std::inner_product(R.begin(), R.end(), R.begin(), 0.0));
      if (k == 0) res0 = res;
      double rel = res / res0;
      if (history) history[k] = rel;
      if (rel <= tol || k == max_steps) break;
      if (k > 0) cfl = std::min(std::max(cfl * std::pow(rel_prev / rel, ser), cflMin), cflMax);
      rel_prev = rel;
    }
    redo = false;
    timestep(*m, U, cfl, dt.data());
    jacobian(*m, U, Ub, dt.data(), A.data());
    orc_bj_invert(h, A.data(), Dinv.data(), fp32_prec);
    for (size_t q = 0; q < n5; ++q) rhs[q] = -1.0 * R[q];
    int its = orc_gmres(h, A.data(), Dinv.data(), rhs.data(), dQ.data(), numVec, maxits, eps, 0, nullptr);
    if (lin_its) lin_its[k] = its;
    std::copy(U, U + n5, Uprev.begin());
    for (size_t q = 0; q < n5; ++q) U[q] += dQ[q];
    int bad = 0;
    for (int i = 0; i < N; ++i) {
      double V[5];
      cons2prim<double>(m->gam, U + 5 * (size_t)i, V);
      bad += (V[0] <= 0.0 || std::isnan(V[0])) + (V[4] <= 0.0 || std::isnan(V[4]));
    }
    if (bad) {
      std::copy(Uprev.begin(), Uprev.end(), U);
      ++nredo;
      if (redos) *redos = nredo;
      cfl *= 0.5;
      if (cfl < cfl0 / 1000.0) return -7;
      redo = true;
      continue;
    }
    ++k;
  }
  return k;
}

// MatVecProdFD::apply (MatVecProd.C:262-372) with computeEpsilon
// (MatVecProd.C:879-929): eps = sum over the state entries of
// (1e-6 |U| + 1e-6) / (5 N ||p||), or 1e-6 when ||p|| < 1e-14; first order
// prod = (F(U + eps p) - F(U)) / eps, second order (F(U + eps p) -
// F(U - eps p)) / (2 eps), with F = R + (U - Un)/dt when dt is given (the
// backward-Euler time term add_dAW_dt, TimeState.C:40-73, with Un = U).
// F (optional) is R(U), as MatVecProdFD::evaluate keeps it.
double orc_matvec_fd(void* h, const double* U, const double* Ub, int order, const double* F, const double* p,
                     const double* dt, int fd_order, double* prod) {
  Mesh* m = (Mesh*)h;
  const size_t n5 = 5 * (size_t)m->N;
  const double eps0 = 1.e-6;
  double pp = 0.0;
  for (size_t q = 0; q < n5; ++q) pp += p[q] * p[q];
  const double norm = std::sqrt(pp);
  double eps = eps0;
  if (!(norm < 1.0e-14)) {
    double loceps = 0.0;
    for (size_t q = 0; q < n5; ++q) loceps += eps0 * std::fabs(U[q]) + eps0;
    eps = loceps / (double(n5) * norm);
  }
  std::vector<double> Qp(n5), Qm(n5), Fp(n5), Fm(n5);
  for (size_t q = 0; q < n5; ++q) Qp[q] = U[q] + eps * p[q];
  orc_residual(h, Qp.data(), Ub, order, 1.0 / 3.0, 0, Fp.data());
  if (dt)
    for (size_t q = 0; q < n5; ++q) Fp[q] += (Qp[q] - U[q]) / dt[q / 5];
  if (fd_order == 2) {
    for (size_t q = 0; q < n5; ++q) Qm[q] = U[q] - eps * p[q];
    orc_residual(h, Qm.data(), Ub, order, 1.0 / 3.0, 0, Fm.data());
    if (dt)
      for (size_t q = 0; q < n5; ++q) Fm[q] += (Qm[q] - U[q]) / dt[q / 5];
    for (size_t q = 0; q < n5; ++q) prod[q] = (0.5 / eps) * (Fp[q] - Fm[q]);
  } else {
    if (F) std::copy(F, F + n5, Fm.begin());
    else orc_residual(h, U, Ub, order, 1.0 / 3.0, 0, Fm.data());
    for (size_t q = 0; q < n5; ++q) prod[q] = (1.0 / eps) * (Fp[q] - Fm[q]);
  }
  return eps;
}

// Exact forward-mode linearisation of the residual (T = Dual):
// Jv = dR/dU . v  (the operator MatVecProdH2 applies, MatVecProd.C:1462-1704)
int orc_jvp(void* h, const double* U, const double* Ub, int order, const double* v, double* Jv) {
  Mesh* m = (Mesh*)h;
  const size_t n5 = 5 * (size_t)m->N;
  std::vector<Dual> Ud(n5), Rd(n5), Xd(3 * (size_t)m->N);
  for (size_t k = 0; k < n5; ++k) Ud[k] = Dual(U[k], v[k]);
  for (size_t k = 0; k < 3 * (size_t)m->N; ++k) Xd[k] = Dual(m->X[k]);
  std::vector<Dual> en, fn, cv, Rl;
  compute_geometry<Dual>(*m, Xd.data(), en, fn, cv);
  compute_lsq_R<Dual>(*m, Xd.data(), Rl);
  Work<Dual> w;
  int ierr = residual_t<Dual>(*m, Xd.data(), en, fn, cv, Rl, Ud.data(), Ub, order, 1.0 / 3.0, 0, Rd.data(), w);
  for (size_t k = 0; k < n5; ++k) Jv[k] = Rd[k].d;
  return ierr;
}

// Exact forward-mode derivative of the residual w.r.t. node coordinates:
// dR = dR/dX . Xdot, through edge/face normals, control volumes, LSQ R and
// dx (the quantities SpaceOperator::computeDerivativeOfResidual differentiates).
int orc_dRdX(void* h, const double* U, const double* Ub, int order, const double* Xdot, double* dR,
             double* R) {
  Mesh* m = (Mesh*)h;
  const size_t n5 = 5 * (size_t)m->N;
  std::vector<Dual> Ud(n5), Rd(n5), Xd(3 * (size_t)m->N);
  for (size_t k = 0; k < n5; ++k) Ud[k] = Dual(U[k]);
  for (size_t k = 0; k < 3 * (size_t)m->N; ++k) Xd[k] = Dual(m->X[k], Xdot[k]);
  std::vector<Dual> en, fn, cv, Rl;
  compute_geometry<Dual>(*m, Xd.data(), en, fn, cv);
  compute_lsq_R<Dual>(*m, Xd.data(), Rl);
  Work<Dual> w;
  int ierr = residual_t<Dual>(*m, Xd.data(), en, fn, cv, Rl, Ud.data(), Ub, order, 1.0 / 3.0, 0, Rd.data(), w);
  for (size_t k = 0; k < n5; ++k) { dR[k] = Rd[k].d; if (R) R[k] = Rd[k].v; }
  return ierr;
}

// Residual on displaced coordinates X (geometry recomputed), for central
// finite differences of shape sensitivities.
int orc_residual_at(void* h, const double* X, const double* U, const double* Ub, int order, double* R) {
  Mesh* m = (Mesh*)h;
  std::vector<double> en, fn, cv, Rl;
  compute_geometry<double>(*m, X, en, fn, cv);
  compute_lsq_R<double>(*m, X, Rl);
  Work<double> w;
  return residual_t<double>(*m, X, en, fn, cv, Rl, U, Ub, order, 1.0 / 3.0, 0, R, w);
}

// z-force functional on the z=0 boundary faces: J = sum_f p_f * (-n_z(f)),
// p_f the mean of the 3 node pressures, n_f the outward area normal
// (pressure force along +z on the bottom wall, cf. PostOperator.C:379-).
}  // extern "C"
template <class T>
static T zforce_t(const Mesh& m, const T* X, const T* U, const int* zfaces, int nz) {
  T J(0.0);
  for (int q = 0; q < nz; ++q) {
    int f = zfaces[q];
    const int* nd = &m.faces[3 * f];
    V3<T> x0(X[3 * nd[0]], X[3 * nd[0] + 1], X[3 * nd[0] + 2]);
    V3<T> x1(X[3 * nd[1]], X[3 * nd[1] + 1], X[3 * nd[1] + 2]);
    V3<T> x2(X[3 * nd[2]], X[3 * nd[2] + 1], X[3 * nd[2] + 2]);
    V3<T> n = 0.5 * cross(x2 - x0, x1 - x0);
    T p(0.0);
    for (int l = 0; l < 3; ++l) {
      T V[5];
      cons2prim(m.gam, &U[5 * nd[l]], V);
      p = p + V[4];
    }
    p = third * p;
    J = J + p * (-n[2]);
  }
  return J;
}
extern "C" {
double orc_zforce(void* h, const double* X, const double* U, const int* zfaces, int nz) {
  Mesh* m = (Mesh*)h;
  return zforce_t<double>(*m, X ? X : m->X.data(), U, zfaces, nz);
}
// dJ/dU (gradient, [N][5]): J depends on U only through the face-node
// pressures p = (gam-1)(E - |m|^2/(2 rho)), so
// dJ/dU_i = sum_{faces f at i} third*(-n_z(f)) * dp/dU_i.
void orc_zforce_dU(void* h, const double* U, const int* zfaces, int nz, double* g) {
  Mesh* m = (Mesh*)h;
  const size_t n5 = 5 * (size_t)m->N;
  std::fill(g, g + n5, 0.0);
  const double* X = m->X.data();
  for (int q = 0; q < nz; ++q) {
    int f = zfaces[q];
    const int* nd = &m->faces[3 * f];
    V3<double> x0(X[3 * nd[0]], X[3 * nd[0] + 1], X[3 * nd[0] + 2]);
    V3<double> x1(X[3 * nd[1]], X[3 * nd[1] + 1], X[3 * nd[1] + 2]);
    V3<double> x2(X[3 * nd[2]], X[3 * nd[2] + 1], X[3 * nd[2] + 2]);
    V3<double> n = 0.5 * cross(x2 - x0, x1 - x0);
    double w = third * (-n[2]);
    for (int l = 0; l < 3; ++l) {
      const double* u = &U[5 * nd[l]];
      double ux = u[1] / u[0], uy = u[2] / u[0], uz = u[3] / u[0];
      double gm1 = m->gam - 1.0;
      double* gi = &g[5 * nd[l]];
      gi[0] += w * gm1 * 0.5 * (ux * ux + uy * uy + uz * uz);
      gi[1] += w * (-gm1 * ux);
      gi[2] += w * (-gm1 * uy);
      gi[3] += w * (-gm1 * uz);
      gi[4] += w * gm1;
    }
  }
}
double orc_zforce_dX(void* h, const double* U, const int* zfaces, int nz, const double* Xdot) {
  Mesh* m = (Mesh*)h;
  const size_t n5 = 5 * (size_t)m->N;
  std::vector<Dual> Xd(3 * (size_t)m->N), Ud(n5);
  for (size_t k = 0; k < 3 * (size_t)m->N; ++k) Xd[k] = Dual(m->X[k], Xdot[k]);
  for (size_t k = 0; k < n5; ++k) Ud[k] = Dual(U[k]);
  return zforce_t<Dual>(*m, Xd.data(), Ud.data(), zfaces, nz).d;
}

}  // extern "C"
