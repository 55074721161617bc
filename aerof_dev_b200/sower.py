"""AERO-F's pre-partitioned binary mesh files (the files sower writes and
GeoSource reads): reading through the library's C ABI, and writing.

``GeoSource`` mirrors the reference's reader (GeoSource.C:94-444): the
connectivity file names the clusters and their subdomains; every cluster
has a geometry file (nodes, tets, boundary triangles) and a decomposition
file (each subdomain's node, element and face ranges, its neighbour
subdomains and the nodes it shares with each).  A subdomain comes back in
its local numbering with its local-to-global maps, as GeoSource::
getSubDomain builds it; ``global_mesh`` reassembles the whole mesh and
``owners`` applies the reference's rule for the node that several
subdomains share (the lowest-numbered one owns it), which
``decomposition.decompose`` turns into ghost-layer subdomains for several
GPUs.

``write`` produces the same files from a mesh and an element partition
(native or swapped byte order), so meshes made here can be read by the
reference, and the reader can be checked on round trips.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import AerofError, library

TET, TRIA = 5, 4
BC_SYMMETRY_FILE = 6


class GeoSource:
    def __init__(self, con_file: str, geo_prefix: str, dec_prefix: str):
        L = library()
        vp = C.c_void_p
        L.aerof_sower_open.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(vp)]
        L.aerof_sower_close.argtypes = [vp]
        L.aerof_sower_num_subdomains.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.aerof_sower_subdomain_sizes.argtypes = [vp, C.c_int] + [C.POINTER(C.c_int)] * 5
        L.aerof_sower_read_subdomain.argtypes = [vp, C.c_int] + [vp] * 10
        L.aerof_sower_last_error.argtypes = [vp, C.c_char_p, C.c_int]
        self.L = L
        self.h = vp()
        rc = L.aerof_sower_open(con_file.encode(), geo_prefix.encode(), dec_prefix.encode(), C.byref(self.h))
        if rc != 0:
            raise AerofError(rc, f"cannot read the connectivity file {con_file}")
        n, nc = C.c_int(), C.c_int()
        self._check(L.aerof_sower_num_subdomains(self.h, C.byref(n), C.byref(nc)))
        self.num_subdomains, self.num_clusters = n.value, nc.value

    def _check(self, rc):
        if rc < 0:
            buf = C.create_string_buffer(512)
            self.L.aerof_sower_last_error(self.h, buf, 512)
            raise AerofError(rc, buf.value.decode())
        return rc

    def close(self):
        if self.h:
            self.L.aerof_sower_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read_subdomain(self, i: int) -> dict:
        """Subdomain i (0-based global subdomain number) in local numbering:
        X, tets, faces, codes, node/elem/face local-to-global maps,
        neighbours and the shared nodes with each (local ids, CSR)."""
        s = [C.c_int() for _ in range(5)]
        self._check(self.L.aerof_sower_subdomain_sizes(self.h, i, *[C.byref(v) for v in s]))
        nn, ne, nf, nb, ns = (v.value for v in s)
        out = {"X": np.empty((nn, 3)), "node_l2g": np.empty(nn, np.int32), "tets": np.empty((ne, 4), np.int32),
               "elem_l2g": np.empty(ne, np.int32), "faces": np.empty((nf, 3), np.int32),
               "codes": np.empty(nf, np.int32), "face_l2g": np.empty(nf, np.int32),
               "neighb": np.empty(nb, np.int32), "shared_ptr": np.empty(nb + 1, np.int32),
               "shared": np.empty(ns, np.int32)}
        keys = ["X", "node_l2g", "tets", "elem_l2g", "faces", "codes", "face_l2g", "neighb", "shared_ptr",
                "shared"]
        self._check(self.L.aerof_sower_read_subdomain(self.h, i, *[C.c_void_p(out[k].ctypes.data) for k in keys]))
        return out

    def global_mesh(self) -> dict:
        """The whole mesh from all subdomains, in global numbering."""
        subs = [self.read_subdomain(i) for i in range(self.num_subdomains)]
        N = 1 + max(int(s["node_l2g"].max()) for s in subs if s["node_l2g"].size)
        T = 1 + max(int(s["elem_l2g"].max()) for s in subs if s["elem_l2g"].size)
        F = 1 + max((int(s["face_l2g"].max()) for s in subs if s["face_l2g"].size), default=-1)
        X = np.empty((N, 3))
        tets = np.empty((T, 4), np.int32)
        faces = np.empty((F, 3), np.int32)
        codes = np.empty(F, np.int32)
        for s in subs:
            X[s["node_l2g"]] = s["X"]
            tets[s["elem_l2g"]] = s["node_l2g"][s["tets"]]
            if s["face_l2g"].size:
                faces[s["face_l2g"]] = s["node_l2g"][s["faces"]]
                codes[s["face_l2g"]] = s["codes"]
        return {"X": X, "tets": tets, "faces": faces, "codes": codes}

    def owners(self) -> np.ndarray:
        """owner[N]: the lowest-numbered subdomain holding each node (the
        reference's masterFlag rule, GeoSource.C:400-405)."""
        owner = None
        for i in range(self.num_subdomains):
            s = self.read_subdomain(i)
            if owner is None:
                owner = {}
            for g in s["node_l2g"].tolist():
                if g not in owner:
                    owner[g] = i
        N = 1 + max(owner)
        out = np.empty(N, np.int32)
        for g, i in owner.items():
            out[g] = i
        return out


# --------------------------------------------------------------------- write
def _ranges(ids: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Sorted ids as inclusive ranges (runs of two or more) and singles."""
    if ids.size == 0:
        return np.empty((0, 2), np.int32), np.empty(0, np.int32)
    br = np.nonzero(np.diff(ids) != 1)[0]
    starts = np.concatenate([[0], br + 1])
    ends = np.concatenate([br, [ids.size - 1]])
    runs = np.stack([ids[starts], ids[ends]], 1)
    single = runs[:, 0] == runs[:, 1]
    return runs[~single].astype(np.int32), runs[single, 0].astype(np.int32)


class _Writer:
    def __init__(self, path: str, swap: bool):
        self.f = open(path, "wb")
        self.e = ">" if swap else "<"
        self.i4(1)
        self.f8(1.0)
        self.header = 12

    def i4(self, *v):
        np.asarray(v, dtype=self.e + "i4").tofile(self.f)

    def i4a(self, a):
        np.asarray(a, dtype=self.e + "i4").tofile(self.f)

    def i8(self, *v):
        np.asarray(v, dtype=self.e + "i8").tofile(self.f)

    def f8(self, *v):
        np.asarray(v, dtype=self.e + "f8").tofile(self.f)

    def tell(self) -> int:
        return self.f.tell() - self.header

    def seek(self, off: int):
        self.f.seek(off + self.header)

    def conn(self, ptr, tgt):
        self.i4(len(ptr) - 1, len(tgt))
        self.i4a(ptr)
        self.i4a(tgt)

    def close(self):
        self.f.close()


def _suffix(num: int, max_num: int) -> str:
    return str(num).zfill(len(str(max_num)))


def write(prefix: str, mesh: dict, elem_part: np.ndarray, nclusters: int = 1, swap: bool = False) -> dict:
    """Writes prefix.con, prefix.geo<suffix>, prefix.dec<suffix> for the
    mesh {X, tets, faces, codes} and the subdomain of every tet
    (elem_part[T], 0..P-1); subdomains go to clusters in contiguous groups.
    Each boundary triangle belongs to the subdomain of a tet that holds its
    three nodes.  Returns the file names for GeoSource."""
    X, tets, faces, codes = mesh["X"], np.asarray(mesh["tets"]), np.asarray(mesh["faces"]), np.asarray(mesh["codes"])
    P = int(elem_part.max()) + 1
    # boundary triangle -> subdomain of a tet that contains it
    key = lambda a: tuple(sorted(a))
    tri_owner = {}
    for t, p in zip(tets.tolist(), elem_part.tolist()):
        for fc in ((t[0], t[1], t[2]), (t[0], t[1], t[3]), (t[0], t[2], t[3]), (t[1], t[2], t[3])):
            tri_owner.setdefault(key(fc), p)
    face_part = np.array([tri_owner[key(f)] for f in faces.tolist()], dtype=np.int32)
    sub_elems = [np.nonzero(elem_part == p)[0] for p in range(P)]
    sub_faces = [np.nonzero(face_part == p)[0] for p in range(P)]
    sub_nodes = [np.unique(tets[e].ravel()) for e in sub_elems]
    clusters = np.array_split(np.arange(P), nclusters)
    names = {"con": prefix + ".con", "geo": prefix + ".geo", "dec": prefix + ".dec"}
    # shared nodes between subdomains (ascending global id)
    holders = {}
    for p, nodes in enumerate(sub_nodes):
        for g in nodes.tolist():
            holders.setdefault(g, []).append(p)
    shared = {p: {} for p in range(P)}
    for g, hs in holders.items():
        for a in hs:
            for b in hs:
                if a != b:
                    shared[a].setdefault(b, []).append(g)
    # connectivity file
    w = _Writer(names["con"], swap)
    cptr = np.concatenate([[0], np.cumsum([len(c) for c in clusters])])
    w.conn(cptr, np.concatenate(clusters))
    sptr, stgt = [0], []
    for p in range(P):
        nb = sorted(shared[p])
        stgt += nb
        sptr.append(len(stgt))
    w.conn(sptr, stgt)
    w.close()
    for ci, cl in enumerate(clusters):
        sfx = _suffix(ci + 1, nclusters)
        cnodes = np.unique(np.concatenate([sub_nodes[p] for p in cl]))
        celems = np.unique(np.concatenate([sub_elems[p] for p in cl]))
        cfaces = np.unique(np.concatenate([sub_faces[p] for p in cl])) if len(cl) else np.empty(0, int)
        n_g2c = {int(g): k for k, g in enumerate(cnodes)}
        e_g2c = {int(g): k for k, g in enumerate(celems)}
        f_g2c = {int(g): k for k, g in enumerate(cfaces)}
        # geometry file: TOC, BC offset, nodes, elements, faces, BCs
        w = _Writer(names["geo"] + sfx, swap)
        w.i8(0, 0, 0)
        w.i8(0)
        toc = []
        toc.append(w.tell())
        w.i4(len(cnodes))
        w.i8(w.tell() + 8)
        for g in cnodes.tolist():
            w.i4(g)
            w.f8(*X[g])
        toc.append(w.tell())
        w.i4(len(celems))
        start = w.tell() + 8 + 4 * len(celems)
        w.i8(start)
        w.i4a(7 * np.arange(len(celems)))
        for g in celems.tolist():
            w.i4(TET, g, 0, *[n_g2c[int(v)] for v in tets[g]])
        toc.append(w.tell())
        w.i4(len(cfaces))
        start = w.tell() + 8 + 4 * len(cfaces)
        w.i8(start)
        w.i4a(7 * np.arange(len(cfaces)))
        for g in cfaces.tolist():
            code = int(codes[g])
            w.i4(TRIA, g, *[n_g2c[int(v)] for v in faces[g]], BC_SYMMETRY_FILE if code == 11 else code, 0)
        bcs = w.tell()
        w.i4(0)
        w.seek(0)
        w.i8(*toc)
        w.i8(bcs)
        w.close()
        # decomposition file
        w = _Writer(names["dec"] + sfx, swap)
        w.i4(len(cl))
        w.i8(*([0] * len(cl)))
        offs = []
        for p in cl:
            offs.append(w.tell())
            for ids, g2c in ((sub_nodes[p], n_g2c), (sub_elems[p], e_g2c), (sub_faces[p], f_g2c)):
                r, s = _ranges(np.array(sorted(g2c[int(g)] for g in ids), dtype=np.int64))
                w.i4(len(r), len(s))
                w.i4a(r.ravel())
                w.i4a(s)
            nb = sorted(shared[p])
            w.i4(len(nb))
            if nb:
                w.i4a(nb)
                ptr, tgt = [0], []
                for q in nb:
                    tgt += [n_g2c[g] for g in sorted(shared[p][q])]
                    ptr.append(len(tgt))
                w.conn(ptr, tgt)
        w.seek(4)
        w.i8(*offs)
        w.close()
    return names


def element_partition(mesh: dict, nparts: int) -> np.ndarray:
    """Subdomain of every tet by recursive coordinate bisection of the tet
    centroids (a stand-in for the partitioner that made the files)."""
    from .decomposition import rcb
    cen = mesh["X"][np.asarray(mesh["tets"])].mean(1)
    return rcb(cen, nparts)
