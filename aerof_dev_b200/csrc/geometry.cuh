// geometry.cuh -- dual-cell geometry of tetrahedra and boundary triangles,
// templated on the scalar type (double for the set-up, Dual for the shape
// derivatives).
#pragma once

#include "physics.cuh"

namespace aerof {

// ElemTet tables (ElemTetCore.C:19-21)
__device__ __forceinline__ int tet_edge_end(int l, int s) {
  // {0,1} {0,2} {0,3} {1,2} {1,3} {2,3}
  return s == 0 ? (l < 3 ? 0 : (l < 5 ? 1 : 2)) : (l < 3 ? l + 1 : (l == 3 ? 2 : 3));
}
__device__ __forceinline__ int tet_edge_face(int l, int s) {
  // {0,1} {2,0} {1,2} {0,3} {3,1} {2,3}
  const int t0[6] = {0, 2, 1, 0, 3, 2}, t1[6] = {1, 0, 2, 3, 1, 3};
  return s == 0 ? t0[l] : t1[l];
}

template <class T>
struct Vec3 {
  T x, y, z;
};
template <class T> __device__ __forceinline__ Vec3<T> v3(T a, T b, T c) { return Vec3<T>{a, b, c}; }
template <class T> __device__ __forceinline__ Vec3<T> operator+(Vec3<T> a, Vec3<T> b) {
  return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <class T> __device__ __forceinline__ Vec3<T> operator-(Vec3<T> a, Vec3<T> b) {
  return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <class T> __device__ __forceinline__ Vec3<T> scale(double c, Vec3<T> a) {
  return v3(c * a.x, c * a.y, c * a.z);
}
// Vec3D::operator^ (Vector3D.h:266-274)
template <class T> __device__ __forceinline__ Vec3<T> cross(Vec3<T> a, Vec3<T> b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> __device__ __forceinline__ Vec3<T> node_x(const T* X, int n) {
  return v3(X[3 * (size_t)n], X[3 * (size_t)n + 1], X[3 * (size_t)n + 2]);
}

// Signed tet volume (ElemTetCore.C:24-39): sixth * v3 . (v1 ^ v2)
template <class T>
__device__ __forceinline__ T tet_volume(const T* X, const int* nd) {
  Vec3<T> x0 = node_x(X, nd[0]);
  Vec3<T> v1 = node_x(X, nd[1]) - x0, v2 = node_x(X, nd[2]) - x0, v3_ = node_x(X, nd[3]) - x0;
  Vec3<T> c = cross(v1, v2);
  const double sixth = 1.0 / 6.0;
  return sixth * (v3_.x * c.x + v3_.y * c.y + v3_.z * c.z);
}

// Dual-cell facet normal of local edge l of a tet, oriented from the lower
// to the higher global node id: ElemTet::computeEdgeNormalsGCL1
// (ElemTetCore.C:281-330) with Xn = Xnp1.
template <class T>
__device__ __forceinline__ Vec3<T> tet_edge_normal(const T* X, const int* nd, int l) {
  const double third = 1.0 / 3.0;
  Vec3<T> x[4] = {node_x(X, nd[0]), node_x(X, nd[1]), node_x(X, nd[2]), node_x(X, nd[3])};
  Vec3<T> f[4];
  f[0] = scale(third, x[0] + x[1] + x[2]);
  f[1] = scale(third, x[0] + x[1] + x[3]);
  f[2] = scale(third, x[0] + x[2] + x[3]);
  f[3] = scale(third, x[1] + x[2] + x[3]);
  Vec3<T> g = scale(0.25, x[0] + x[1] + x[2] + x[3]);
  Vec3<T> xg0 = f[tet_edge_face(l, 0)] - g;
  Vec3<T> xg1 = f[tet_edge_face(l, 1)] - g;
  Vec3<T> c = cross(xg1, xg0);
  Vec3<T> n = scale(0.5, c + c) + scale(0.25, c + c);
  if (nd[tet_edge_end(l, 0)] < nd[tet_edge_end(l, 1)]) return n;
  return v3(-n.x, -n.y, -n.z);
}

// Same normal with the vertices' coordinates given locally (xs[4][3]) and
// the orientation taken from the global node ids nd.
template <class T>
__device__ __forceinline__ Vec3<T> tet_edge_normal_local(const T* xs, const int* nd, int l) {
  const int loc[4] = {0, 1, 2, 3};
  Vec3<T> n = tet_edge_normal(xs, loc, l);
  // tet_edge_normal orients by the local ids (always ascending): reorient
  if (nd[tet_edge_end(l, 0)] < nd[tet_edge_end(l, 1)]) return n;
  return v3(-n.x, -n.y, -n.z);
}

// FaceTria::computeNormalGCL1 (FaceTriaCore.C:65-82) with Xn = Xnp1:
// twelfth * ((3 x02) ^ x01 + (3 x02) ^ x01), outward for the face ordering.
template <class T>
__device__ __forceinline__ Vec3<T> face_normal(const T* X, const int* nd) {
  const double twelfth = 1.0 / 12.0;
  Vec3<T> x0 = node_x(X, nd[0]);
  Vec3<T> x01 = node_x(X, nd[1]) - x0, x02 = node_x(X, nd[2]) - x0;
  Vec3<T> a = scale(2.0, x02) + x02;
  Vec3<T> s = cross(a, x01) + cross(a, x01);
  return scale(twelfth, s);
}

}  // namespace aerof
