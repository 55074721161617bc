// sower.cu -- reader of AERO-F's pre-partitioned binary mesh files (the
// files the reference's GeoSource reads: a connectivity file, and per
// cluster a geometry and a decomposition file), host code only.
//
// Format (restated from the reference's readers):
//  - every file starts with BinFileHandler's header (BinFileHandler.h:
//    the int 1, whose byte order tells whether the file must be swapped,
//    then a double version); offsets stored in the files count from the
//    end of that header;
//  - connectivity file: two Connectivity records (ConnectivityCore.C:869-
//    882: size, numtarget, pointer[size+1], target[numtarget]):
//    cluster -> subdomains and subdomain -> subdomains
//    (GeoSource::readConnectivityInfo, GeoSource.C:94-141);
//  - decomposition file of a cluster: number of subdomains, then one
//    offset per subdomain; at a subdomain's offset its node, element and
//    face ranges (GeoSource::getRangeInfo, GeoSource.C:218-252: the numbers
//    of ranges and singles, the ranges, the singles), its neighbour
//    subdomains and the nodes it shares with each (a Connectivity)
//    (GeoSource::getSubDomain, GeoSource.C:256-333);
//  - geometry file of a cluster: three table-of-contents offsets (nodes,
//    elements, faces) and the offset of the boundary conditions; nodes:
//    count, offset of the first, then per node its global number and x,y,z
//    (NodeSet::read, Node.C:7-50); elements: count, offset, a table of
//    per-element offsets, then type (TET = 5), global number, volume id and
//    4 nodes (ElemSet::read, ElemCore.C:135-199); faces: count, offset, a
//    table of offsets, then type (TRIA = 4), global number, 3 nodes, code
//    (6 means symmetry) and surface id (FaceSet::read, FaceCore.C:270-330);
//    boundary conditions: count, then node, dof and value
//    (BCondSet::read, BCond.C:6-19).
// Cluster suffixes are the cluster number (from 1) padded with zeros to the
// width of the number of clusters (computeClusterSuffix, BinFileHandler.h).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/aerof_gpu.h"

namespace {

struct ReadError {
  int code;
  std::string msg;
};

// BinFileHandler's reading side
class BinFile {
 public:
  explicit BinFile(const std::string& name) : name_(name) {
    f_ = std::fopen(name.c_str(), "rb");
    if (!f_) throw ReadError{AEROF_EINVAL, "cannot open " + name};
    int one = 0;
    raw(&one, sizeof(int), 1);
    if (one != 1) {
      swap_ = true;
      swap_bytes(&one, sizeof(int), 1);
      if (one != 1) throw ReadError{AEROF_EINVAL, name + ": not a BinFileHandler file"};
    }
    read(&version_, 1);
  }
  ~BinFile() {
    if (f_) std::fclose(f_);
  }
  BinFile(const BinFile&) = delete;
  BinFile& operator=(const BinFile&) = delete;

  template <class T>
  void read(T* p, size_t n) {
    raw(p, sizeof(T), n);
    if (swap_) swap_bytes(p, sizeof(T), n);
  }
  template <class T>
  T get() {
    T v;
    read(&v, 1);
    return v;
  }
  // offsets count from the end of the header
  void seek(int64_t off) {
    if (off < 0 || fseeko(f_, (off_t)(off + kHeader), SEEK_SET) != 0)
      throw ReadError{AEROF_EINVAL, name_ + ": bad offset"};
  }
  int64_t tell() { return (int64_t)ftello(f_) - kHeader; }

 private:
  static constexpr int64_t kHeader = sizeof(int) + sizeof(double);
  void raw(void* p, size_t sz, size_t n) {
    if (n && std::fread(p, sz, n, f_) != n) throw ReadError{AEROF_EINVAL, name_ + ": unexpected end of file"};
  }
  static void swap_bytes(void* p, size_t sz, size_t n) {
    unsigned char* c = static_cast<unsigned char*>(p);
    for (size_t k = 0; k < n; ++k, c += sz)
      for (size_t a = 0, b = sz - 1; a < b; ++a, --b) std::swap(c[a], c[b]);
  }
  std::string name_;
  FILE* f_ = nullptr;
  bool swap_ = false;
  double version_ = 0.0;
};

struct Conn {  // Connectivity: pointer[size+1], target[numtarget]
  std::vector<int> ptr, tgt;
  int size() const { return (int)ptr.size() - 1; }
  void read(BinFile& f) {
    const int size = f.get<int>(), numtarget = f.get<int>();
    if (size < 0 || numtarget < 0) throw ReadError{AEROF_EINVAL, "bad connectivity record"};
    ptr.resize((size_t)size + 1);
    tgt.resize((size_t)numtarget);
    f.read(ptr.data(), ptr.size());
    f.read(tgt.data(), tgt.size());
    if (ptr[0] != 0 || ptr[size] != numtarget) throw ReadError{AEROF_EINVAL, "bad connectivity pointers"};
  }
};

// ranges then singles, as inclusive [first, last] pairs
std::vector<std::pair<int, int>> read_ranges(BinFile& f) {
  const int nr = f.get<int>(), ns = f.get<int>();
  if (nr < 0 || ns < 0) throw ReadError{AEROF_EINVAL, "bad range record"};
  std::vector<int> r(2 * (size_t)nr), s((size_t)ns);
  f.read(r.data(), r.size());
  f.read(s.data(), s.size());
  std::vector<std::pair<int, int>> out;
  for (int i = 0; i < nr; ++i) out.emplace_back(r[2 * i], r[2 * i + 1]);
  for (int i = 0; i < ns; ++i) out.emplace_back(s[i], s[i]);
  return out;
}

size_t count_of(const std::vector<std::pair<int, int>>& rg) {
  size_t n = 0;
  for (auto& p : rg) n += (size_t)(p.second - p.first + 1);
  return n;
}

std::string cluster_suffix(int num, int max_num) {
  auto digits = [](int v) {
    int d = 1;
    while (v >= 10) { v /= 10; ++d; }
    return d;
  };
  return std::string((size_t)std::max(0, digits(max_num) - digits(num)), '0') + std::to_string(num);
}

}  // namespace

struct aerof_sower {
  std::string geo, dec;
  Conn cluster_to_sub, sub_to_sub;
  std::vector<int> sub_cluster, sub_index;  // cluster and position in it of every subdomain
  int num_clusters = 0;
  std::string last_error;
  // the last subdomain read, kept for the sizes-then-read protocol
  int cached = -1;
  std::vector<double> X;
  std::vector<int> node_l2g, tets, elem_l2g, faces, codes, face_l2g, neighb, shared_ptr, shared;
  std::vector<int> node_l2c;  // local -> cluster node number
};

namespace {

void load_subdomain(aerof_sower* s, int iSub) {
  if (s->cached == iSub) return;
  const int clus = s->sub_cluster[iSub], pos = s->sub_index[iSub];
  const std::string suffix = cluster_suffix(clus + 1, s->num_clusters);
  // decomposition: ranges, neighbours, shared nodes
  BinFile dec(s->dec + suffix);
  dec.get<int>();  // subdomains in the cluster
  dec.seek((int64_t)sizeof(int) + (int64_t)pos * (int64_t)sizeof(int64_t));
  dec.seek(dec.get<int64_t>());
  const auto nrg = read_ranges(dec), erg = read_ranges(dec), frg = read_ranges(dec);
  const int nnb = dec.get<int>();
  std::vector<int> nb((size_t)std::max(nnb, 0));
  Conn sh;
  if (nnb > 0) {
    dec.read(nb.data(), nb.size());
    sh.read(dec);
  } else {
    sh.ptr = {0};
  }
  // geometry
  BinFile geo(s->geo + suffix);
  int64_t toc[3], bcs;
  geo.read(toc, 3);
  geo.read(&bcs, 1);
  (void)bcs;
  const size_t nn = count_of(nrg), ne = count_of(erg), nf = count_of(frg);
  s->X.assign(3 * nn, 0.0);
  s->node_l2g.assign(nn, 0);
  s->node_l2c.assign(nn, 0);
  geo.seek(toc[0]);
  geo.get<int>();                   // nodes in the cluster
  const int64_t nstart = geo.get<int64_t>();
  size_t c = 0;
  for (auto& r : nrg) {
    geo.seek(nstart + (int64_t)r.first * (int64_t)(sizeof(int) + 3 * sizeof(double)));
    for (int k = r.first; k <= r.second; ++k, ++c) {
      s->node_l2g[c] = geo.get<int>();
      s->node_l2c[c] = k;
      geo.read(&s->X[3 * c], 3);
    }
  }
  std::map<int, int> c2l;
  for (size_t i = 0; i < nn; ++i) c2l[s->node_l2c[i]] = (int)i;
  auto local = [&](int cn) {
    auto it = c2l.find(cn);
    if (it == c2l.end()) throw ReadError{AEROF_EINVAL, "element or face node outside the subdomain"};
    return it->second;
  };
  // elements
  s->tets.assign(4 * ne, 0);
  s->elem_l2g.assign(ne, 0);
  geo.seek(toc[1]);
  geo.get<int>();
  int64_t estart = geo.get<int64_t>();
  int64_t etoc = geo.tell();
  c = 0;
  for (auto& r : erg) {
    geo.seek(etoc + (int64_t)sizeof(int) * r.first);
    const int t = geo.get<int>();
    geo.seek(estart + (int64_t)sizeof(int) * t);
    for (int k = r.first; k <= r.second; ++k, ++c) {
      const int type = geo.get<int>();
      if (type != 5) throw ReadError{AEROF_EINVAL, "element type " + std::to_string(type) + " (only tets, 5)"};
      s->elem_l2g[c] = geo.get<int>();
      geo.get<int>();  // volume id
      int nd[4];
      geo.read(nd, 4);
      for (int q = 0; q < 4; ++q) s->tets[4 * c + q] = local(nd[q]);
    }
  }
  // faces
  s->faces.assign(3 * nf, 0);
  s->codes.assign(nf, 0);
  s->face_l2g.assign(nf, 0);
  geo.seek(toc[2]);
  geo.get<int>();
  const int64_t fstart = geo.get<int64_t>();
  const int64_t ftoc = geo.tell();
  c = 0;
  for (auto& r : frg) {
    geo.seek(ftoc + (int64_t)sizeof(int) * r.first);
    const int t = geo.get<int>();
    geo.seek(fstart + (int64_t)sizeof(int) * t);
    for (int k = r.first; k <= r.second; ++k, ++c) {
      const int type = geo.get<int>();
      if (type != 4) throw ReadError{AEROF_EINVAL, "face type " + std::to_string(type) + " (only triangles, 4)"};
      s->face_l2g[c] = geo.get<int>();
      int nd[3];
      geo.read(nd, 3);
      for (int q = 0; q < 3; ++q) s->faces[3 * c + q] = local(nd[q]);
      int code = geo.get<int>();
      if (code == 6) code = 11;  // BC_SYMMETRY (FaceCore.C:318-321)
      s->codes[c] = code;
      geo.get<int>();  // surface id
    }
  }
  s->neighb = nb;
  s->shared_ptr = sh.ptr;
  s->shared.resize(sh.tgt.size());
  for (size_t k = 0; k < sh.tgt.size(); ++k) s->shared[k] = local(sh.tgt[k]);
  s->cached = iSub;
}

template <class F>
int sower_guard(aerof_sower* s, F&& f) {
  if (!s) return AEROF_EINVAL;
  try {
    return f();
  } catch (const ReadError& e) {
    s->last_error = e.msg;
    s->cached = -1;
    return e.code;
  } catch (const std::exception& e) {
    s->last_error = e.what();
    s->cached = -1;
    return AEROF_EINVAL;
  }
}

}  // namespace

extern "C" int aerof_sower_open(const char* con_file, const char* geo_prefix, const char* dec_prefix,
                                aerof_sower** out) {
  if (!con_file || !geo_prefix || !dec_prefix || !out) return AEROF_EINVAL;
  *out = nullptr;
  aerof_sower* s = new aerof_sower();
  s->geo = geo_prefix;
  s->dec = dec_prefix;
  try {
    BinFile con(con_file);
    s->cluster_to_sub.read(con);
    s->sub_to_sub.read(con);
    s->num_clusters = s->cluster_to_sub.size();
    const int nsub = (int)s->cluster_to_sub.tgt.size();
    s->sub_cluster.assign((size_t)nsub, -1);
    s->sub_index.assign((size_t)nsub, -1);
    for (int cl = 0; cl < s->num_clusters; ++cl)
      for (int p = s->cluster_to_sub.ptr[cl]; p < s->cluster_to_sub.ptr[cl + 1]; ++p) {
        const int g = s->cluster_to_sub.tgt[p];
        if (g < 0 || g >= nsub) throw ReadError{AEROF_EINVAL, "subdomain number out of range"};
        s->sub_cluster[g] = cl;
        s->sub_index[g] = p - s->cluster_to_sub.ptr[cl];
      }
  } catch (const ReadError&) {
    delete s;
    return AEROF_EINVAL;
  }
  *out = s;
  return AEROF_OK;
}

extern "C" int aerof_sower_close(aerof_sower* s) {
  if (!s) return AEROF_EINVAL;
  delete s;
  return AEROF_OK;
}

extern "C" int aerof_sower_num_subdomains(aerof_sower* s, int* nsub, int* nclusters) {
  return sower_guard(s, [&]() -> int {
    if (nsub) *nsub = (int)s->sub_cluster.size();
    if (nclusters) *nclusters = s->num_clusters;
    return AEROF_OK;
  });
}

extern "C" int aerof_sower_subdomain_sizes(aerof_sower* s, int iSub, int* nnodes, int* nelems, int* nfaces,
                                           int* nneighb, int* nshared) {
  return sower_guard(s, [&]() -> int {
    if (iSub < 0 || iSub >= (int)s->sub_cluster.size()) return AEROF_EINVAL;
    load_subdomain(s, iSub);
    if (nnodes) *nnodes = (int)s->node_l2g.size();
    if (nelems) *nelems = (int)s->elem_l2g.size();
    if (nfaces) *nfaces = (int)s->face_l2g.size();
    if (nneighb) *nneighb = (int)s->neighb.size();
    if (nshared) *nshared = (int)s->shared.size();
    return AEROF_OK;
  });
}

extern "C" int aerof_sower_read_subdomain(aerof_sower* s, int iSub, double* X, int* node_l2g, int* tets,
                                          int* elem_l2g, int* faces, int* codes, int* face_l2g, int* neighb,
                                          int* shared_ptr, int* shared) {
  return sower_guard(s, [&]() -> int {
    if (iSub < 0 || iSub >= (int)s->sub_cluster.size()) return AEROF_EINVAL;
    load_subdomain(s, iSub);
    auto put = [](auto* dst, const auto& src) {
      if (dst && !src.empty()) std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
    };
    put(X, s->X);
    put(node_l2g, s->node_l2g);
    put(tets, s->tets);
    put(elem_l2g, s->elem_l2g);
    put(faces, s->faces);
    put(codes, s->codes);
    put(face_l2g, s->face_l2g);
    put(neighb, s->neighb);
    put(shared_ptr, s->shared_ptr);
    put(shared, s->shared);
    return AEROF_OK;
  });
}

extern "C" int aerof_sower_last_error(aerof_sower* s, char* buf, int len) {
  if (!s || !buf || len <= 0) return AEROF_EINVAL;
  std::strncpy(buf, s->last_error.c_str(), (size_t)len - 1);
  buf[len - 1] = 0;
  return AEROF_OK;
}
