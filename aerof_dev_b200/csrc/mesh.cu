// mesh.cu -- mesh set-up: integer preprocessing on the host (edge list,
// incidence lists; all bit-exact integer work) and the static geometry on
// the device (control volumes, dual-cell edge normals, boundary face
// normals, least-squares factors), each accumulated per output item in the
// reference's element/edge order so the sums are deterministic.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <numeric>
#include <utility>

#include "common.cuh"
#include "physics.cuh"
#include "geometry.cuh"

namespace aerof {

constexpr int kMBlock = 256;

static const int h_edgeEnd[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

template <class T>
__global__ void k_ctrl_vol(int N, const T* __restrict__ X, const int* __restrict__ tets,
                           const int* __restrict__ nt_ptr, const int* __restrict__ nt_tet, T* __restrict__ vol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T v(0.0);
  for (int p = nt_ptr[i]; p < nt_ptr[i + 1]; ++p) {
    int t = nt_tet[p] >> 2;
    v += 0.25 * tet_volume(X, tets + 4 * (size_t)t);
  }
  vol[i] = v;
}

template <class T>
__global__ void k_edge_normals(int E, const T* __restrict__ X, const int* __restrict__ tets,
                               const int* __restrict__ et_ptr, const int* __restrict__ et_tet, T* __restrict__ en) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  T a(0.0), b(0.0), c(0.0);
  for (int p = et_ptr[e]; p < et_ptr[e + 1]; ++p) {
    int t = et_tet[p] >> 3, l = et_tet[p] & 7;
    Vec3<T> n = tet_edge_normal(X, tets + 4 * (size_t)t, l);
    a += n.x; b += n.y; c += n.z;
  }
  en[e] = a; en[(size_t)E + e] = b; en[2 * (size_t)E + e] = c;
}

template <class T>
__global__ void k_face_normals(int F, const T* __restrict__ X, const int* __restrict__ faces, T* __restrict__ fn) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  Vec3<T> n = face_normal(X, faces + 3 * (size_t)f);
  fn[f] = n.x; fn[(size_t)F + f] = n.y; fn[2 * (size_t)F + f] = n.z;
}

// SubDomain::computeWeightsLeastSquaresEdgePart/NodePart
// (SubDomainCore.C:1334-1381, 1755-1777), per node over its neighbours in
// ascending order (the reference's edge order for that node).
template <class T>
__global__ void k_lsq_R(int N, const T* __restrict__ X, const int* __restrict__ nbr_ptr,
                        const int* __restrict__ nbr_node, T* __restrict__ R) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T s[6] = {T(0.0), T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
  Vec3<T> xi = node_x(X, i);
  for (int p = nbr_ptr[i]; p < nbr_ptr[i + 1]; ++p) {
    Vec3<T> d = node_x(X, nbr_node[p]) - xi;
    s[0] += d.x * d.x; s[1] += d.x * d.y; s[2] += d.x * d.z;
    s[3] += d.y * d.y; s[4] += d.y * d.z; s[5] += d.z * d.z;
  }
  T r11 = dsqrt(s[0]);
  T or11 = 1.0 / r11;
  T r12 = s[1] * or11;
  T r13 = s[2] * or11;
  T r22 = dsqrt(s[3] - r12 * r12);
  T r23 = (s[4] - r12 * r13) / r22;
  T r33 = dsqrt(s[5] - (r13 * r13 + r23 * r23));
  R[i] = r11; R[(size_t)N + i] = r12; R[2 * (size_t)N + i] = r13;
  R[3 * (size_t)N + i] = r22; R[4 * (size_t)N + i] = r23; R[5 * (size_t)N + i] = r33;
}

__global__ void k_lsq_W(int N, const double* __restrict__ R, double* __restrict__ W) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double r[6], w[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) r[k] = R[(size_t)k * N + i];
  lsq_node_constants(r, w);
#pragma unroll
  for (int k = 0; k < 6; ++k) W[(size_t)k * N + i] = w[k];
}

__global__ void k_setX(int N, const double* __restrict__ X, double* __restrict__ P) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  P[8 * (size_t)i + 5] = X[3 * (size_t)i];
  P[8 * (size_t)i + 6] = X[3 * (size_t)i + 1];
  P[8 * (size_t)i + 7] = X[3 * (size_t)i + 2];
}


// ------------------------------------------------------------------ host
struct HostMesh {
  std::vector<int> edge_pos;
  std::vector<int> edges, tet_edge, nbr_ptr, nbr_node, nbr_edge, nbr_tpos, nf_ptr, nf_face, et_ptr, et_tet,
      nt_ptr, nt_tet;
};

// EdgeSet::find + createPointers (EdgeCore.C:55-117): unique (min,max)
// pairs of the tet edges, numbered lexicographically.
static void build_host(int N, int T, int F, const int* tets, const int* faces, HostMesh& h, int& E) {
  std::vector<uint64_t> keys((size_t)T * 6);
  for (int t = 0; t < T; ++t)
    for (int l = 0; l < 6; ++l) {
      uint64_t a = (uint32_t)tets[4 * (size_t)t + h_edgeEnd[l][0]];
      uint64_t b = (uint32_t)tets[4 * (size_t)t + h_edgeEnd[l][1]];
      if (a > b) std::swap(a, b);
      keys[6 * (size_t)t + l] = (a << 32) | b;
    }
  std::vector<uint64_t> u(keys);
  std::sort(u.begin(), u.end());
  u.erase(std::unique(u.begin(), u.end()), u.end());
  if (u.size() > (size_t)0x3fffffff) throw ApiError{AEROF_EINVAL, "too many edges"};
  E = (int)u.size();
  h.edges.resize(2 * (size_t)E);
  for (int l = 0; l < E; ++l) {
    h.edges[2 * (size_t)l] = (int)(u[l] >> 32);
    h.edges[2 * (size_t)l + 1] = (int)(u[l] & 0xffffffffu);
  }
  h.tet_edge.resize((size_t)T * 6);
  for (size_t k = 0; k < keys.size(); ++k)
    h.tet_edge[k] = (int)(std::lower_bound(u.begin(), u.end(), keys[k]) - u.begin());
  // node -> neighbours ascending: appending edges in lexicographic order
  // gives, per node, incoming edges (k<i) by k then outgoing (i<j) by j.
  h.nbr_ptr.assign(N + 1, 0);
  for (int l = 0; l < E; ++l) { h.nbr_ptr[h.edges[2 * l] + 1]++; h.nbr_ptr[h.edges[2 * l + 1] + 1]++; }
  for (int i = 0; i < N; ++i) h.nbr_ptr[i + 1] += h.nbr_ptr[i];
  h.nbr_node.resize(2 * (size_t)E);
  h.nbr_edge.resize(2 * (size_t)E);
  h.nbr_tpos.resize(2 * (size_t)E);
  h.edge_pos.resize(2 * (size_t)E);
  std::vector<int> pos(h.nbr_ptr.begin(), h.nbr_ptr.end() - 1);
  for (int l = 0; l < E; ++l) {
    int i = h.edges[2 * l], j = h.edges[2 * l + 1];
    int pi = pos[i]++, pj = pos[j]++;
    h.nbr_node[pi] = j; h.nbr_edge[pi] = l;
    h.nbr_node[pj] = i; h.nbr_edge[pj] = (int)((unsigned)l | 0x80000000u);
    h.nbr_tpos[pi] = pj; h.nbr_tpos[pj] = pi;
    h.edge_pos[2 * (size_t)l] = pi; h.edge_pos[2 * (size_t)l + 1] = pj;
  }
  // node -> faces (ascending face id)
  h.nf_ptr.assign(N + 1, 0);
  for (size_t q = 0; q < 3 * (size_t)F; ++q) h.nf_ptr[faces[q] + 1]++;
  for (int i = 0; i < N; ++i) h.nf_ptr[i + 1] += h.nf_ptr[i];
  h.nf_face.resize(3 * (size_t)F);
  pos.assign(h.nf_ptr.begin(), h.nf_ptr.end() - 1);
  for (int f = 0; f < F; ++f)
    for (int l = 0; l < 3; ++l) h.nf_face[pos[faces[3 * (size_t)f + l]]++] = f;
  // edge -> tets (ascending tet id)
  h.et_ptr.assign(E + 1, 0);
  for (size_t k = 0; k < h.tet_edge.size(); ++k) h.et_ptr[h.tet_edge[k] + 1]++;
  for (int l = 0; l < E; ++l) h.et_ptr[l + 1] += h.et_ptr[l];
  h.et_tet.resize((size_t)T * 6);
  pos.assign(h.et_ptr.begin(), h.et_ptr.end() - 1);
  for (int t = 0; t < T; ++t)
    for (int l = 0; l < 6; ++l) h.et_tet[pos[h.tet_edge[6 * (size_t)t + l]]++] = t * 8 + l;
  // node -> tets (ascending tet id)
  h.nt_ptr.assign(N + 1, 0);
  for (size_t q = 0; q < 4 * (size_t)T; ++q) h.nt_ptr[tets[q] + 1]++;
  for (int i = 0; i < N; ++i) h.nt_ptr[i + 1] += h.nt_ptr[i];
  h.nt_tet.resize(4 * (size_t)T);
  pos.assign(h.nt_ptr.begin(), h.nt_ptr.end() - 1);
  for (int t = 0; t < T; ++t)
    for (int l = 0; l < 4; ++l) h.nt_tet[pos[tets[4 * (size_t)t + l]]++] = t * 4 + l;
}

// ------------------------------------------------------------------ blocked
// Morton (Z-order) renumbering of the nodes and the per-block edge lists of
// the blocked residual kernel.  Integer work only; deterministic.
struct HostBlocked {
  std::vector<int> n2o, o2n, nb2_ptr, nb2_node, bsrc, beptr, lptr, lidx, xslot, xin_ptr, hptr, hnode,
      hfptr, hfnode;
  std::vector<unsigned short> lnb, lpad;
  std::vector<int> hpad, hfpad;
  std::vector<ushort2> bl;
  std::vector<int2> bedges;
  int nblk = 0, maxE = 0, nX = 0, maxH = 0, maxL = 0, maxHf = 0, maxLp = 0;
};

static inline uint64_t spread3(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}

static void build_blocked(int N, int E, int NB, const double* X, const std::vector<int>& edges, HostBlocked& b) {
  double lo[3] = {X[0], X[1], X[2]}, hi[3] = {X[0], X[1], X[2]};
  for (int i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], X[3 * (size_t)i + k]);
      hi[k] = std::max(hi[k], X[3 * (size_t)i + k]);
    }
  double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  double sc = ext > 0 ? (double)((1 << 21) - 1) / ext : 0.0;
  std::vector<std::pair<uint64_t, int>> key(N);
  for (int i = 0; i < N; ++i) {
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) q[k] = (uint64_t)((X[3 * (size_t)i + k] - lo[k]) * sc);
    key[i] = {spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2, i};
  }
  std::sort(key.begin(), key.end());
  b.n2o.resize(N);
  b.o2n.resize(N);
  for (int n = 0; n < N; ++n) { b.n2o[n] = key[n].second; b.o2n[key[n].second] = n; }
  // edges in the new numbering, oriented first < second, sorted
  std::vector<std::pair<uint64_t, int>> ek(E);
  for (int l = 0; l < E; ++l) {
    uint32_t a = (uint32_t)b.o2n[edges[2 * (size_t)l]], c = (uint32_t)b.o2n[edges[2 * (size_t)l + 1]];
    const bool rev = a > c;
    if (rev) std::swap(a, c);
    ek[l] = {((uint64_t)a << 32) | c, (int)((unsigned)l | (rev ? 0x80000000u : 0u))};
  }
  std::sort(ek.begin(), ek.end());
  b.bedges.resize(E);
  b.bsrc.resize(E);
  for (int q = 0; q < E; ++q) {
    b.bedges[q] = make_int2((int)(ek[q].first >> 32), (int)(ek[q].first & 0xffffffffu));
    b.bsrc[q] = ek[q].second;
  }
  ek.clear();
  ek.shrink_to_fit();
  b.nblk = (N + NB - 1) / NB;
  b.beptr.assign(b.nblk + 1, E);
  {
    int q = 0;
    for (int blk = 0; blk < b.nblk; ++blk) {
      while (q < E && b.bedges[q].x < blk * NB) ++q;
      b.beptr[blk] = q;
    }
    b.beptr[b.nblk] = E;
  }
  b.maxE = 0;
  for (int blk = 0; blk < b.nblk; ++blk) b.maxE = std::max(b.maxE, b.beptr[blk + 1] - b.beptr[blk]);
  // neighbour CSR (ascending new ids), local assembly lists, spill slots
  b.nb2_ptr.assign(N + 1, 0);
  b.lptr.assign(N + 1, 0);
  b.xin_ptr.assign(N + 1, 0);
  b.xslot.assign(E, -1);
  b.nX = 0;
  for (int q = 0; q < E; ++q) {
    const int f = b.bedges[q].x, sd = b.bedges[q].y;
    b.nb2_ptr[f + 1]++; b.nb2_ptr[sd + 1]++;
    b.lptr[f + 1]++;
    if (sd / NB == f / NB) b.lptr[sd + 1]++;
    else { b.xslot[q] = 0; b.nX++; b.xin_ptr[sd + 1]++; }
  }
  for (int n = 0; n < N; ++n) {
    b.nb2_ptr[n + 1] += b.nb2_ptr[n];
    b.lptr[n + 1] += b.lptr[n];
    b.xin_ptr[n + 1] += b.xin_ptr[n];
  }
  b.nb2_node.resize(2 * (size_t)E);
  b.lidx.resize(b.lptr[N]);
  std::vector<int> pn(b.nb2_ptr.begin(), b.nb2_ptr.end() - 1), pl(b.lptr.begin(), b.lptr.end() - 1),
      px(b.xin_ptr.begin(), b.xin_ptr.end() - 1);
  for (int q = 0; q < E; ++q) {
    const int f = b.bedges[q].x, sd = b.bedges[q].y;
    const int blk = f / NB, slot = q - b.beptr[blk];
    b.nb2_node[pn[f]++] = sd;
    b.nb2_node[pn[sd]++] = f;
    b.lidx[pl[f]++] = slot;
    // spill slots numbered by destination node (then edge), so the
    // destination's incoming fluxes are contiguous
    if (b.xslot[q] < 0) b.lidx[pl[sd]++] = (int)((unsigned)slot | 0x80000000u);
    else b.xslot[q] = px[sd]++;
  }
  // halo of every block (neighbours outside it, ascending) and each
  // neighbour-CSR entry as a slot of the block's staged node set: slots
  // [0, nn) are the block's own nodes, [nn, nn + halo) its halo.
  b.hptr.assign(b.nblk + 1, 0);
  b.hnode.clear();
  b.lnb.assign(2 * (size_t)E, 0);
  b.maxH = 0;
  std::vector<int> h;
  for (int blk = 0; blk < b.nblk; ++blk) {
    const int n0 = blk * NB, n1 = std::min(N, n0 + NB), nn = n1 - n0;
    h.clear();
    for (int p = b.nb2_ptr[n0]; p < b.nb2_ptr[n1]; ++p) {
      const int j = b.nb2_node[p];
      if (j < n0 || j >= n1) h.push_back(j);
    }
    std::sort(h.begin(), h.end());
    h.erase(std::unique(h.begin(), h.end()), h.end());
    if (nn + h.size() > 65535) throw ApiError{AEROF_EINVAL, "a node block's halo exceeds 65535 nodes"};
    b.maxH = std::max(b.maxH, (int)h.size());
    b.maxL = std::max(b.maxL, b.nb2_ptr[n1] - b.nb2_ptr[n0]);
    for (int p = b.nb2_ptr[n0]; p < b.nb2_ptr[n1]; ++p) {
      const int j = b.nb2_node[p];
      b.lnb[p] = (unsigned short)(j >= n0 && j < n1 ? j - n0
                                                    : nn + (std::lower_bound(h.begin(), h.end(), j) - h.begin()));
    }
    b.hnode.insert(b.hnode.end(), h.begin(), h.end());
    b.hptr[blk + 1] = (int)b.hnode.size();
  }
  // the same in fixed-stride per-block segments (halo ids padded with -1 to
  // maxH, local slots padded to a multiple of 8 entries), so a block's
  // staging addresses follow from its index alone
  b.maxLp = (b.maxL + 7) / 8 * 8;
  b.hpad.assign((size_t)b.nblk * std::max(b.maxH, 1), -1);
  b.lpad.assign((size_t)b.nblk * std::max(b.maxLp, 8), 0);
  for (int blk = 0; blk < b.nblk; ++blk) {
    const int n0 = blk * NB, n1 = std::min(N, n0 + NB);
    std::copy(b.hnode.begin() + b.hptr[blk], b.hnode.begin() + b.hptr[blk + 1], b.hpad.begin() + (size_t)blk * b.maxH);
    std::copy(b.lnb.begin() + b.nb2_ptr[n0], b.lnb.begin() + b.nb2_ptr[n1], b.lpad.begin() + (size_t)blk * b.maxLp);
  }
  // forward halo of every block (second endpoints of its edges lying in
  // later blocks, ascending) and each edge's endpoints as staged slots
  b.hfptr.assign(b.nblk + 1, 0);
  b.hfnode.clear();
  b.bl.resize(E);
  b.maxHf = 0;
  for (int blk = 0; blk < b.nblk; ++blk) {
    const int n0 = blk * NB, n1 = std::min(N, n0 + NB), nn = n1 - n0;
    h.clear();
    for (int q = b.beptr[blk]; q < b.beptr[blk + 1]; ++q)
      if (b.bedges[q].y >= n1) h.push_back(b.bedges[q].y);
    std::sort(h.begin(), h.end());
    h.erase(std::unique(h.begin(), h.end()), h.end());
    if (nn + h.size() > 65535) throw ApiError{AEROF_EINVAL, "a node block's forward halo exceeds 65535 nodes"};
    b.maxHf = std::max(b.maxHf, (int)h.size());
    for (int q = b.beptr[blk]; q < b.beptr[blk + 1]; ++q) {
      const int j = b.bedges[q].y;
      const int lj = j < n1 ? j - n0 : nn + (int)(std::lower_bound(h.begin(), h.end(), j) - h.begin());
      b.bl[q] = make_ushort2((unsigned short)(b.bedges[q].x - n0), (unsigned short)lj);
    }
    b.hfnode.insert(b.hfnode.end(), h.begin(), h.end());
    b.hfptr[blk + 1] = (int)b.hfnode.size();
  }
  // fixed-stride copy of the forward halo ids (-1 padded to maxHf)
  b.hfpad.assign((size_t)b.nblk * std::max(b.maxHf, 1), -1);
  for (int blk = 0; blk < b.nblk; ++blk)
    std::copy(b.hfnode.begin() + b.hfptr[blk], b.hfnode.begin() + b.hfptr[blk + 1],
              b.hfpad.begin() + (size_t)blk * b.maxHf);
}

// blocked copies of the node geometry and oriented edge normals
__global__ void k_blocked_nodes(int N, const int* __restrict__ n2o, const double* __restrict__ X,
                                const double* __restrict__ W, const double* __restrict__ vol,
                                double* __restrict__ P2, double* __restrict__ W2, double* __restrict__ vol2) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int o = n2o[n];
#pragma unroll
  for (int k = 0; k < 5; ++k) P2[8 * (size_t)n + k] = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) P2[8 * (size_t)n + 5 + k] = X[3 * (size_t)o + k];
#pragma unroll
  for (int k = 0; k < 6; ++k) W2[(size_t)k * N + n] = W[(size_t)k * N + o];
  vol2[n] = vol[o];
}
__global__ void k_blocked_normals(int E, const int* __restrict__ bsrc, const double* __restrict__ en,
                                  double* __restrict__ bn) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= E) return;
  const int src = bsrc[q];
  const size_t l = (size_t)(src & 0x7fffffff);
  const double sg = src < 0 ? -1.0 : 1.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) bn[(size_t)k * E + q] = sg * en[(size_t)k * E + l];
}

void compute_blocked_geometry(aerof_gpu_ctx* c) {
  DeviceMesh& m = c->mesh;
  cudaStream_t s = c->stream;
  m.P2.alloc(8 * (size_t)m.N);
  m.W2.alloc(6 * (size_t)m.N);
  m.vol2.alloc(m.N);
  m.bnorm.alloc(3 * (size_t)m.E);
  k_blocked_nodes<<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, m.n2o.p, m.X.p, m.lsqW.p, m.vol.p, m.P2.p, m.W2.p,
                                                              m.vol2.p);
  AEROF_LAUNCH_CHECK();
  k_blocked_normals<<<grid_for(m.E, kMBlock), kMBlock, 0, s>>>(m.E, m.bsrc.p, m.en.p, m.bnorm.p);
  AEROF_LAUNCH_CHECK();
}

void compute_geometry(aerof_gpu_ctx* c) {
  DeviceMesh& m = c->mesh;
  cudaStream_t s = c->stream;
  m.vol.alloc(m.N);
  m.en.alloc(3 * (size_t)m.E);
  m.fnrm.alloc(3 * (size_t)std::max(m.F, 1));
  m.lsqR.alloc(6 * (size_t)m.N);
  m.lsqW.alloc(6 * (size_t)m.N);
  k_ctrl_vol<double><<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, m.X.p, m.tets.p, m.nt_ptr.p, m.nt_tet.p, m.vol.p);
  AEROF_LAUNCH_CHECK();
  k_edge_normals<double><<<grid_for(m.E, kMBlock), kMBlock, 0, s>>>(m.E, m.X.p, m.tets.p, m.et_ptr.p, m.et_tet.p,
                                                                      m.en.p);
  AEROF_LAUNCH_CHECK();
  if (m.F) {
    k_face_normals<double><<<grid_for(m.F, kMBlock), kMBlock, 0, s>>>(m.F, m.X.p, m.faces.p, m.fnrm.p);
    AEROF_LAUNCH_CHECK();
  }
  k_lsq_R<double><<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, m.X.p, m.nbr_ptr.p, m.nbr_node.p, m.lsqR.p);
  AEROF_LAUNCH_CHECK();
  k_lsq_W<<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, m.lsqR.p, m.lsqW.p);
  AEROF_LAUNCH_CHECK();
  k_setX<<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, m.X.p, m.P.p);
  AEROF_LAUNCH_CHECK();
  compute_blocked_geometry(c);
}

void geometry_dual(aerof_gpu_ctx* c, const Dual* XD, Dual* volD, Dual* enD, Dual* fnD, Dual* RD) {
  DeviceMesh& m = c->mesh;
  cudaStream_t s = c->stream;
  k_ctrl_vol<Dual><<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, XD, m.tets.p, m.nt_ptr.p, m.nt_tet.p, volD);
  AEROF_LAUNCH_CHECK();
  k_edge_normals<Dual><<<grid_for(m.E, kMBlock), kMBlock, 0, s>>>(m.E, XD, m.tets.p, m.et_ptr.p, m.et_tet.p, enD);
  AEROF_LAUNCH_CHECK();
  if (m.F) {
    k_face_normals<Dual><<<grid_for(m.F, kMBlock), kMBlock, 0, s>>>(m.F, XD, m.faces.p, fnD);
    AEROF_LAUNCH_CHECK();
  }
  k_lsq_R<Dual><<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, XD, m.nbr_ptr.p, m.nbr_node.p, RD);
  AEROF_LAUNCH_CHECK();
}

// Rejects non-finite coordinates.
static int check_coordinates(aerof_gpu_ctx* c, int N, const double* X) {
  for (size_t q = 0; q < 3 * (size_t)N; ++q)
    if (!std::isfinite(X[q])) {
      c->last_error = "non-finite coordinate of node " + std::to_string(q / 3);
      return AEROF_EINVAL;
    }
  return AEROF_OK;
}

// Counts nodes whose dual control volume (ElemTetCore.C:102-112) is zero or
// not finite: the residual divides by it (SpaceOperator.C:614-620).
// Inverted tets are accepted, as the reference accepts them (the signed tet
// volumes around an interior node add up to the volume of its star), and
// so are negative volumes, which the outer ghost nodes of a subdomain mesh
// can have (their rows are not used).
__global__ void k_check_vol(int N, const double* __restrict__ vol, int* __restrict__ nbad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N && !(vol[i] != 0.0 && fabs(vol[i]) < INFINITY)) atomicAdd(nbad, 1);
}

}  // namespace aerof

using namespace aerof;

extern "C" int aerof_gpu_set_mesh(aerof_gpu_ctx* c, int N, int T, int F, const double* X, const int* tets,
                                  const int* faces, const int* codes, const double* Ub) {
  return guard(c, [&]() -> int {
    if (N <= 0 || T <= 0 || F < 0 || !X || !tets || (F && (!faces || !codes)) || !Ub) return AEROF_EINVAL;
    for (size_t q = 0; q < 4 * (size_t)T; ++q)
      if (tets[q] < 0 || tets[q] >= N) { c->last_error = "tet node index out of range"; return AEROF_EINVAL; }
    for (size_t q = 0; q < 3 * (size_t)F; ++q)
      if (faces[q] < 0 || faces[q] >= N) { c->last_error = "face node index out of range"; return AEROF_EINVAL; }
    for (int f = 0; f < F; ++f)
      if (codes[f] != AEROF_BC_SLIP_WALL_MOVING && codes[f] != AEROF_BC_INLET_MOVING &&
          codes[f] != AEROF_BC_OUTLET_MOVING) {
        c->last_error = "unsupported boundary code " + std::to_string(codes[f]);
        return AEROF_EINVAL;
      }
    if (int e = check_coordinates(c, N, X)) return e;
    c->has_mesh = false;
    c->pipe.reset();
    c->turb.on = false;
    c->imp.precision = 0;
    c->imp.prec_ready = false;
    c->imp.ilu_ready = false;
    c->h2.ready = false;
    HostMesh h;
    int E = 0;
    build_host(N, T, F, tets, faces, h, E);
    DeviceMesh& m = c->mesh;
    cudaStream_t s = c->stream;
    m.N = N; m.T = T; m.F = F; m.E = E;
    for (int k = 0; k < 5; ++k) m.Ub[k] = Ub[k];
    m.Ubd.upload(Ub, 5, s);
    m.X.upload(X, 3 * (size_t)N, s);
    m.P.alloc(8 * (size_t)N);
    m.P.zero(s);
    m.tets.upload(tets, 4 * (size_t)T, s);
    m.tet_edge.upload(h.tet_edge.data(), h.tet_edge.size(), s);
    m.edges.upload(reinterpret_cast<const int2*>(h.edges.data()), (size_t)E, s);
    if (F) {
      m.faces.upload(faces, 3 * (size_t)F, s);
      m.fcode.upload(codes, (size_t)F, s);
    } else {
      m.faces.alloc(3); m.fcode.alloc(1);
    }
    m.nbr_ptr.upload(h.nbr_ptr.data(), h.nbr_ptr.size(), s);
    m.nbr_node.upload(h.nbr_node.data(), h.nbr_node.size(), s);
    m.nbr_edge.upload(h.nbr_edge.data(), h.nbr_edge.size(), s);
    m.nbr_tpos.upload(h.nbr_tpos.data(), h.nbr_tpos.size(), s);
    m.edge_pos.upload(reinterpret_cast<const int2*>(h.edge_pos.data()), (size_t)E, s);
    m.nf_ptr.upload(h.nf_ptr.data(), h.nf_ptr.size(), s);
    if (F) m.nf_face.upload(h.nf_face.data(), h.nf_face.size(), s);
    else m.nf_face.alloc(1);
    m.et_ptr.upload(h.et_ptr.data(), h.et_ptr.size(), s);
    m.et_tet.upload(h.et_tet.data(), h.et_tet.size(), s);
    m.nt_ptr.upload(h.nt_ptr.data(), h.nt_ptr.size(), s);
    m.nt_tet.upload(h.nt_tet.data(), h.nt_tet.size(), s);
    {
      // nodes per block of the blocked residual kernel (tuning knob; the
      // shared-memory footprint is NB*192 B + owned edges * 40 B)
      m.NB = 128;
      if (const char* env = std::getenv("AEROF_BLOCK_NODES")) {
        const int v = std::atoi(env);
        if (v == 64 || v == 128 || v == 256) m.NB = v;
      }
      HostBlocked hb;
      build_blocked(N, E, m.NB, X, h.edges, hb);
      m.nblk = hb.nblk; m.maxE = hb.maxE; m.nX = hb.nX;
      m.maxH = hb.maxH; m.maxL = hb.maxL; m.maxHf = hb.maxHf; m.maxLp = hb.maxLp;
      m.hpad.upload(hb.hpad.data(), hb.hpad.size(), s);
      m.lpad.upload(hb.lpad.data(), hb.lpad.size(), s);
      m.hfpad.upload(hb.hfpad.data(), hb.hfpad.size(), s);
      m.hfptr.upload(hb.hfptr.data(), hb.hfptr.size(), s);
      if (hb.hfnode.empty()) m.hfnode.alloc(1);
      else m.hfnode.upload(hb.hfnode.data(), hb.hfnode.size(), s);
      if (hb.bl.empty()) m.bl.alloc(1);
      else m.bl.upload(hb.bl.data(), hb.bl.size(), s);
      m.hptr.upload(hb.hptr.data(), hb.hptr.size(), s);
      if (hb.hnode.empty()) m.hnode.alloc(1);
      else m.hnode.upload(hb.hnode.data(), hb.hnode.size(), s);
      if (hb.lnb.empty()) m.lnb.alloc(1);
      else m.lnb.upload(hb.lnb.data(), hb.lnb.size(), s);
      m.n2o.upload(hb.n2o.data(), N, s);
      m.o2n.upload(hb.o2n.data(), N, s);
      const int last = hb.nb2_ptr[N];
      hb.nb2_ptr.resize(N + 1 + 4, last);  // padding read by the 16-byte staging of the last block
      m.nb2_ptr.upload(hb.nb2_ptr.data(), hb.nb2_ptr.size(), s);
      m.nb2_node.upload(hb.nb2_node.data(), hb.nb2_node.size(), s);
      m.bsrc.upload(hb.bsrc.data(), (size_t)E, s);
      m.beptr.upload(hb.beptr.data(), hb.beptr.size(), s);
      m.lptr.upload(hb.lptr.data(), N + 1, s);
      if (hb.lidx.empty()) m.lidx.alloc(1);
      else m.lidx.upload(hb.lidx.data(), hb.lidx.size(), s);
      m.xslot.upload(hb.xslot.data(), (size_t)E, s);
      m.xin_ptr.upload(hb.xin_ptr.data(), N + 1, s);
      {
        // boundary subface fluxes of each node, blocked numbering
        std::vector<int> bp(N + 1, 0), be;
        for (int n = 0; n < N; ++n) {
          const int o = hb.n2o[n];
          for (int q = h.nf_ptr[o]; q < h.nf_ptr[o + 1]; ++q) {
            const int f = h.nf_face[q];
            const int l = faces[3 * (size_t)f] == o ? 0 : (faces[3 * (size_t)f + 1] == o ? 1 : 2);
            be.push_back(3 * f + l);
          }
          bp[n + 1] = (int)be.size();
        }
        if (be.empty()) be.push_back(0);
        m.bnf_ptr.upload(bp.data(), bp.size(), s);
        m.bnf_ent.upload(be.data(), be.size(), s);
      }
      {
        // stages of the residual of host arrays with overlapped copies
        // (DeviceMesh::h_st_*): K chunks of consecutive caller rows, their
        // sizes in proportion to the weights w_k.  Short first chunks let
        // the copies of R start early, short last ones shorten what remains
        // after the last copy of U.  Default K = 8 equal chunks (tuning
        // knobs AEROF_PIPE_CHUNKS, 2-32 equal chunks, or AEROF_PIPE_WEIGHTS,
        // 2-32 comma-separated positive weights)
        std::vector<double> w(8, 1.0);
        if (const char* env = std::getenv("AEROF_PIPE_CHUNKS")) {
          const int v = std::atoi(env);
          if (v >= 2 && v <= 32) w.assign(v, 1.0);
        }
        if (const char* env = std::getenv("AEROF_PIPE_WEIGHTS")) {
          std::vector<double> v;
          for (const char* q = env; *q;) {
            char* e = nullptr;
            const double x = std::strtod(q, &e);
            if (e == q || !(x > 0.0)) { v.clear(); break; }
            v.push_back(x);
            q = *e == ',' ? e + 1 : e;
            if (*e && *e != ',') { v.clear(); break; }
          }
          if (v.size() >= 2 && v.size() <= 32) w = v;
        }
        m.pipeK = (int)w.size();
        const int nb = hb.nblk, NBk = m.NB, K = m.pipeK;
        {
          double tot = 0.0, acc = 0.0;
          for (double x : w) tot += x;
          m.pipe_rows.assign(K + 1, N);
          m.pipe_rows[0] = 0;
          for (int k = 1; k < K; ++k) {
            acc += w[k - 1];
            m.pipe_rows[k] = std::max(m.pipe_rows[k - 1], std::min(N, (int)std::llround(acc / tot * N)));
          }
        }
        std::vector<unsigned char> row_chunk(N);
        for (int k = 0; k < K; ++k)
          for (int o = m.pipe_rows[k]; o < m.pipe_rows[k + 1]; ++o) row_chunk[o] = (unsigned char)k;
        m.h_st_prim.resize(N);
        for (int n = 0; n < N; ++n) m.h_st_prim[n] = row_chunk[hb.n2o[n]];
        m.h_st_grad = m.h_st_prim;
        for (int n = 0; n < N; ++n)
          for (int q = hb.nb2_ptr[n]; q < hb.nb2_ptr[n + 1]; ++q)
            m.h_st_grad[n] = std::max(m.h_st_grad[n], m.h_st_prim[hb.nb2_node[q]]);
        m.h_st_flux.assign(nb, 0);
        for (int n = 0; n < N; ++n) m.h_st_flux[n / NBk] = std::max(m.h_st_flux[n / NBk], m.h_st_grad[n]);
        for (int b = 0; b < nb; ++b)
          for (int q = hb.hfptr[b]; q < hb.hfptr[b + 1]; ++q)
            m.h_st_flux[b] = std::max(m.h_st_flux[b], m.h_st_grad[hb.hfnode[q]]);
        m.h_st_node = m.h_st_flux;
        for (int q = 0; q < E; ++q)
          if (hb.xslot[q] >= 0) {
            const int bs = hb.bedges[q].y / NBk;
            m.h_st_node[bs] = std::max(m.h_st_node[bs], m.h_st_flux[hb.bedges[q].x / NBk]);
          }
        m.h_o2n = hb.o2n;
      }
      AEROF_CUDA(cudaStreamSynchronize(s));  // host vectors die at scope end
    }
    // rows with boundary faces (their face blocks are formed apart)
    {
      std::vector<int> br(N, -1), bls;
      for (int r = 0; r < N; ++r)
        if (h.nf_ptr[r] < h.nf_ptr[r + 1]) { br[r] = (int)bls.size(); bls.push_back(r); }
      m.nbrow = (int)bls.size();
      m.brow.upload(br.data(), (size_t)N, s);
      if (bls.empty()) m.blist.alloc(1);
      else m.blist.upload(bls.data(), bls.size(), s);
      AEROF_CUDA(cudaStreamSynchronize(s));
    }
    // multicolour ordering and the ILU(0) pattern in it
    {
      std::vector<int> col(N, -1), seen;
      int nc = 0;
      for (int r = 0; r < N; ++r) {
        seen.assign(nc + 1, 0);
        for (int q = h.nbr_ptr[r]; q < h.nbr_ptr[r + 1]; ++q) {
          const int cq = col[h.nbr_node[q]];
          if (cq >= 0) seen[cq] = 1;
        }
        int c0 = 0;
        while (seen[c0]) ++c0;
        col[r] = c0;
        nc = std::max(nc, c0 + 1);
      }
      std::vector<int> cptr(nc + 1, 0), perm(N), iperm(N);
      for (int r = 0; r < N; ++r) ++cptr[col[r] + 1];
      for (int c0 = 0; c0 < nc; ++c0) cptr[c0 + 1] += cptr[c0];
      {
        std::vector<int> fill(cptr.begin(), cptr.end() - 1);
        for (int r = 0; r < N; ++r) perm[fill[col[r]]++] = r;
      }
      for (int i = 0; i < N; ++i) iperm[perm[i]] = i;
      // slices of 32 rows inside each colour
      std::vector<int> cslice(nc + 1, 0);
      for (int c0 = 0; c0 < nc; ++c0) cslice[c0 + 1] = cslice[c0] + (cptr[c0 + 1] - cptr[c0] + 31) / 32;
      const int nsl = cslice[nc];
      std::vector<int> rsl(N), sr0(std::max(nsl, 1)), rlen(N), rju(N), isp(nsl + 1, 0);
      for (int c0 = 0; c0 < nc; ++c0)
        for (int t = 0; t < cptr[c0 + 1] - cptr[c0]; ++t) {
          const int sl = cslice[c0] + t / 32;
          rsl[cptr[c0] + t] = sl;
          if (t % 32 == 0) sr0[sl] = cptr[c0] + t;
        }
      // rows: diagonal + neighbours in colour order, ascending
      std::vector<std::vector<std::pair<int, int>>> rows(N);
      for (int i = 0; i < N; ++i) {
        const int r = perm[i];
        auto& row = rows[i];
        row.emplace_back(i, -1);
        for (int q = h.nbr_ptr[r]; q < h.nbr_ptr[r + 1]; ++q) row.emplace_back(iperm[h.nbr_node[q]], q - h.nbr_ptr[r]);
        std::sort(row.begin(), row.end());
        rlen[i] = (int)row.size();
        for (int k = 0; k < rlen[i]; ++k)
          if (row[k].second < 0) rju[i] = k;
      }
      for (int sl = 0; sl < nsl; ++sl) {
        int kmax = 0;
        for (int i = sr0[sl]; i < N && rsl[i] == sl; ++i) kmax = std::max(kmax, rlen[i]);
        isp[sl + 1] = isp[sl] + kmax;
      }
      const size_t nb = (size_t)isp[nsl];
      std::vector<int> jc(nb * 32, -1), jsrc(nb * 32, -2);
      for (int i = 0; i < N; ++i) {
        const int sl = rsl[i], lane = i - sr0[sl];
        for (int k = 0; k < rlen[i]; ++k) {
          jc[((size_t)isp[sl] + k) * 32 + lane] = rows[i][k].first;
          jsrc[((size_t)isp[sl] + k) * 32 + lane] = rows[i][k].second;
        }
      }
      // numericILU schedule: entry id of (row i, position k)
      auto eid = [&](int i, int k) { return (isp[rsl[i]] + k) * 32 + (i - sr0[rsl[i]]); };
      std::vector<int> lo_ptr(N + 1, 0), up_ptr(1, 0);
      std::vector<int2> lo, up;
      for (int i = 0; i < N; ++i) {
        const auto& ri = rows[i];
        for (int k = 0; k < rju[i]; ++k) {
          const int l = ri[k].first;
          const auto& rl = rows[l];
          lo.push_back(make_int2(eid(i, k), eid(l, rju[l])));
          int mm = k + 1;
          for (int j = rju[l] + 1; j < rlen[l]; ++j) {
            while (mm < rlen[i] && ri[mm].first < rl[j].first) ++mm;
            if (mm >= rlen[i]) break;
            if (ri[mm].first == rl[j].first) up.push_back(make_int2(eid(l, j), eid(i, mm)));
          }
          up_ptr.push_back((int)up.size());
        }
        lo_ptr[i + 1] = (int)lo.size();
      }
      if (lo.empty()) lo.push_back(make_int2(0, 0));
      if (up.empty()) up.push_back(make_int2(0, 0));
      m.lo_ptr.upload(lo_ptr.data(), lo_ptr.size(), s);
      m.up_ptr.upload(up_ptr.data(), up_ptr.size(), s);
      m.lo.upload(lo.data(), lo.size(), s);
      m.up.upload(up.data(), up.size(), s);
      m.ncolor = nc;
      m.ilu_blocks = nb;
      m.h_cptr.swap(cptr);
      m.h_cslice.swap(cslice);
      m.cperm.upload(perm.data(), (size_t)N, s);
      m.rlen.upload(rlen.data(), (size_t)N, s);
      m.rju.upload(rju.data(), (size_t)N, s);
      m.rsl.upload(rsl.data(), (size_t)N, s);
      m.sr0.upload(sr0.data(), sr0.size(), s);
      m.isp.upload(isp.data(), isp.size(), s);
      m.jc.upload(jc.data(), jc.size(), s);
      m.jsrc.upload(jsrc.data(), jsrc.size(), s);
      AEROF_CUDA(cudaStreamSynchronize(s));
    }
    // sliced layout of the implicit operator
    {
      const int nsl = (N + 31) / 32;
      std::vector<int> sp(nsl + 1, 0);
      for (int sl = 0; sl < nsl; ++sl) {
        int ks = 0;
        for (int r = 32 * sl; r < std::min(N, 32 * sl + 32); ++r) ks = std::max(ks, h.nbr_ptr[r + 1] - h.nbr_ptr[r]);
        sp[sl + 1] = sp[sl] + ks;
      }
      std::vector<int> sc((size_t)sp[nsl] * 32);
      for (int r = 0; r < N; ++r) {
        const int sl = r >> 5, l = r & 31, cnt = h.nbr_ptr[r + 1] - h.nbr_ptr[r];
        for (int k = 0; k < sp[sl + 1] - sp[sl]; ++k)
          sc[((size_t)sp[sl] + k) * 32 + l] = k < cnt ? h.nbr_node[h.nbr_ptr[r] + k] : r;
      }
      for (int r = N; r < 32 * nsl; ++r) {
        const int sl = r >> 5, l = r & 31;
        for (int k = 0; k < sp[sl + 1] - sp[sl]; ++k) sc[((size_t)sp[sl] + k) * 32 + l] = 32 * sl;
      }
      m.nsl = nsl;
      m.sptr.upload(sp.data(), sp.size(), s);
      if (sc.empty()) m.scol.alloc(1);
      else m.scol.upload(sc.data(), sc.size(), s);
      AEROF_CUDA(cudaStreamSynchronize(s));
      m.h_sptr.swap(sp);
      m.h_nbr_ptr = h.nbr_ptr;
    }
    m.h_edges.swap(h.edges);
    compute_geometry(c);
    c->dual.geom_static = false;
    {
      DBuf<int> nb;
      nb.alloc(1);
      nb.zero(s);
      k_check_vol<<<grid_for(m.N, kMBlock), kMBlock, 0, s>>>(m.N, m.vol.p, nb.p);
      AEROF_LAUNCH_CHECK();
      int bad = 0;
      AEROF_CUDA(cudaMemcpyAsync(&bad, nb.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      AEROF_CUDA(cudaStreamSynchronize(s));
      if (bad) {
        c->last_error = std::to_string(bad) + " node(s) with a zero or non-finite control volume "
                        "(degenerate tets)";
        return AEROF_EINVAL;
      }
    }
    AEROF_CUDA(cudaStreamSynchronize(s));
    c->n_owned = N;
    c->has_mesh = true;
    galerkin_reserve(c, c->visc.model);
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_update_coordinates(aerof_gpu_ctx* c, const double* X) {
  return guard(c, [&]() -> int {
    if (!c->has_mesh) return AEROF_ESTATE;
    if (!X) return AEROF_EINVAL;
    DeviceMesh& m = c->mesh;
    if (is_device_ptr(X))
      AEROF_CUDA(cudaMemcpyAsync(m.X.p, X, 3 * (size_t)m.N * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    else
      AEROF_CUDA(cudaMemcpyAsync(m.X.p, X, 3 * (size_t)m.N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    compute_geometry(c);
    c->dual.geom_static = false;
    c->imp.precision = 0;
    c->imp.prec_ready = false;
    c->h2.ready = false;
    AEROF_CUDA(cudaStreamSynchronize(c->stream));
    return AEROF_OK;
  });
}

extern "C" int aerof_gpu_mesh_sizes(aerof_gpu_ctx* c, int* N, int* E, int* F) {
  if (!c) return AEROF_EINVAL;
  if (N) *N = c->mesh.N;
  if (E) *E = c->mesh.E;
  if (F) *F = c->mesh.F;
  return c->has_mesh ? AEROF_OK : AEROF_ESTATE;
}

extern "C" int aerof_gpu_get_edges(aerof_gpu_ctx* c, int* edges) {
  if (!c || !edges) return AEROF_EINVAL;
  if (!c->has_mesh) return AEROF_ESTATE;
  std::copy(c->mesh.h_edges.begin(), c->mesh.h_edges.end(), edges);
  return AEROF_OK;
}

extern "C" int aerof_gpu_get_geometry(aerof_gpu_ctx* c, double* edge_normal, double* face_normal, double* ctrl_vol,
                                      double* lsq_R) {
  return guard(c, [&]() -> int {
    if (!c->has_mesh) return AEROF_ESTATE;
    DeviceMesh& m = c->mesh;
    auto soa_to_aos = [&](const DBuf<double>& src, int n, int w, double* dst) {
      std::vector<double> h((size_t)n * w);
      AEROF_CUDA(cudaMemcpyAsync(h.data(), src.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      AEROF_CUDA(cudaStreamSynchronize(c->stream));
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < w; ++k) dst[(size_t)w * i + k] = h[(size_t)k * n + i];
    };
    if (edge_normal) soa_to_aos(m.en, m.E, 3, edge_normal);
    if (face_normal && m.F) soa_to_aos(m.fnrm, m.F, 3, face_normal);
    if (ctrl_vol) soa_to_aos(m.vol, m.N, 1, ctrl_vol);
    if (lsq_R) soa_to_aos(m.lsqR, m.N, 6, lsq_R);
    return AEROF_OK;
  });
}
