// common.cuh -- context, device buffers and error plumbing shared by the
// kernels of the edge-based FV path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <atomic>
#include <memory>
#include <string>
#include <vector>

#include "../../include/aerof_gpu.h"
#include "physics.cuh"

namespace aerof {
extern std::atomic<long long> g_launch_count;

// ------------------------------------------------------------------ errors
struct CudaError {
  cudaError_t err;
  const char* where;
};

#define AEROF_CUDA(call)                                                  \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) throw ::aerof::CudaError{e_, #call};           \
  } while (0)

// Every kernel launch of the library is followed by this check, which also
// counts the launch (aerof_gpu_launch_count).
#define AEROF_LAUNCH_CHECK()                                            \
  do {                                                                  \
    ::aerof::g_launch_count.fetch_add(1, std::memory_order_relaxed);    \
    AEROF_CUDA(cudaGetLastError());                                     \
  } while (0)

struct ApiError {
  int code;
  std::string msg;
};

// ------------------------------------------------------------------ buffers
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      throw ApiError{AEROF_ENOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed"};
    }
    n = count;
  }
  void ensure(size_t count) {
    if (count > n) alloc(count);
  }
  void upload(const T* h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) AEROF_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s) {
    if (n) AEROF_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------------ mesh
// Device-resident mesh in the kernels' numbering.  Nodes are kept in the
// caller's numbering; edges are the reference's lexicographic list.
struct DeviceMesh {
  int N = 0, T = 0, F = 0, E = 0;
  double Ub[5] = {0, 0, 0, 0, 0};
  DBuf<double> Ubd;        // [5] free-stream conservative state on the device
  // node record: V (5) + X (3), 64 bytes per node
  DBuf<double> P;
  DBuf<double> X;          // [N][3] (copy used by geometry/derivative kernels)
  DBuf<int> tets;          // [T][4]
  DBuf<int> tet_edge;      // [T][6]
  DBuf<int2> edges;        // [E] (i, j), i < j
  DBuf<double> en;         // [3][E] edge normals, SoA
  DBuf<double> fnrm;       // [3][F] face normals, SoA
  DBuf<int> faces;         // [F][3]
  DBuf<int> fcode;         // [F]
  DBuf<double> vol;        // [N]
  DBuf<double> lsqR;       // [6][N] Cholesky factors (r11 r12 r13 r22 r23 r33)
  DBuf<double> lsqW;       // [6][N] or11 or22 or33 r12or11 r23or22 psi
  // node -> incident edges in the reference's accumulation order (neighbour
  // ascending).  nbr_edge holds edge id, sign bit set when the node is the
  // edge's second endpoint.
  DBuf<int> nbr_ptr;       // [N+1]
  DBuf<int> nbr_node;      // [2E]
  DBuf<int> nbr_edge;      // [2E]  (edge id) | (0x80000000 if node is j)
  DBuf<int> nbr_tpos;      // [2E]  position of the mirrored entry (row nbr, col node)
  DBuf<int2> edge_pos;     // [E]   CSR positions of (i,j) in row i and (j,i) in row j
  // node -> incident boundary faces, ascending face id
  DBuf<int> nf_ptr;        // [N+1]
  DBuf<int> nf_face;       // [3F]
  // edge -> incident tets (ascending) with local edge index
  DBuf<int> et_ptr;        // [E+1]
  DBuf<int> et_tet;        // [6T]  tet*8 + local edge
  // node -> incident tets (ascending) with local vertex index
  DBuf<int> nt_ptr;        // [N+1]
  DBuf<int> nt_tet;        // [4T]  tet*4 + local vertex
  // host copies for queries
  std::vector<int> h_edges;
  // Sliced block layout of the H1 operator (rows in slices of 32; block k of
  // row r = 32 s + l stored element-interleaved: element e at
  // ((sptr[s] + k) * 25 + e) * 32 + l; diagonal and its inverse at
  // (s * 25 + e) * 32 + l).  scol: column of block (s, k, l); rows with
  // fewer than ks[s] blocks are padded with their own index.
  int nsl = 0;
  int nbrow = 0;           // rows with boundary faces
  DBuf<int> brow, blist;   // [N] index among the boundary rows (-1: none); [nbrow] those rows
  // multicolour ordering for the block ILU(0) preconditioner: greedy
  // colouring of the node graph (ascending node order, smallest free
  // colour), rows sorted by (colour, node).  ILU pattern in that order:
  // row i holds its diagonal and its neighbours, columns ascending, in a
  // sliced layout as H1's: each colour's rows in slices of 32 (a slice never
  // spans two colours), entry k of the slice's rows at block (isp[s] + k).
  int ncolor = 0;
  size_t ilu_blocks = 0;         // isp[number of slices]
  std::vector<int> h_cptr;       // [ncolor+1] first row of each colour
  std::vector<int> h_cslice;     // [ncolor+1] first slice of each colour
  DBuf<int> cperm;               // [N] colour-order row -> caller row
  DBuf<int> rlen, rju, rsl;      // [N] entries of the row, diagonal position, slice
  DBuf<int> sr0, isp;            // [slices] first row, [slices+1] blocks before the slice
  DBuf<int> jc, jsrc;            // [ilu_blocks*32] column (colour order; -1 padding), neighbour slot (-1 diagonal)
  // factorisation schedule, as entry ids (block * 32 + lane): per row its
  // lower entries (A_ik, inverted U_kk) and, per lower entry, the updates
  // (U_kj, A_ij) of numericILU
  DBuf<int> lo_ptr, up_ptr;      // [N+1], [lower entries + 1]
  DBuf<int2> lo, up;
  DBuf<int> sptr;          // [nsl+1] block columns before slice s
  DBuf<int> scol;          // [sptr[nsl] * 32]
  std::vector<int> h_sptr, h_nbr_ptr;

  // ---- blocked residual: Morton-renumbered copy of the node data ----
  int NB = 256;            // nodes per block
  int nblk = 0, maxE = 0, nX = 0, maxH = 0, maxL = 0, maxHf = 0, maxLp = 0;
  DBuf<int> n2o, o2n;      // [N] new -> old and old -> new node ids
  DBuf<double> P2;         // [N][8] node records in new numbering
  DBuf<double> W2;         // [6][N] LSQ constants, new numbering
  DBuf<double> vol2;       // [N]
  DBuf<int> nb2_ptr, nb2_node;  // neighbour CSR in new numbering (ascending)
  DBuf<int> hptr, hnode;        // per block: halo nodes (outside the block, ascending)
  DBuf<unsigned short> lnb;     // nb2_node entries as slots of the block's staged nodes
  DBuf<int> hpad;               // [nblk][maxH] halo ids, -1 padded
  DBuf<unsigned short> lpad;    // [nblk][maxLp] the block's lnb segment, 0 padded
  DBuf<int> hfptr, hfnode;      // per block: forward halo (second endpoints in later blocks)
  DBuf<int> hfpad;              // [nblk][maxHf] forward halo ids, -1 padded
  DBuf<ushort2> bl;             // per blocked edge: (first, second) as slots of the staged nodes
  DBuf<int> bsrc;          // [E] reference edge id | (1<<31 if reversed)
  DBuf<double> bnorm;      // [3][E] normals oriented first -> second
  DBuf<int> beptr;         // [nblk+1] owned-edge range of each block
  DBuf<int> lptr, lidx;    // per node (new): owned local edge slots, sign bit = second endpoint
  DBuf<int> xslot;         // [E] spill slot of a block-crossing edge, -1 otherwise
  DBuf<int> xin_ptr;       // per node (new): its incoming spill slots [xin_ptr[n], xin_ptr[n+1])
  DBuf<int> bnf_ptr, bnf_ent;   // per node (new): its boundary subface fluxes, rows 3 f + l of fbuf, face order
  // schedule of the residual of host arrays with its copies overlapped
  // (residual.cu), for pipeK chunks of caller rows: the stage (the
  // chunk after whose arrival it can run) of every blocked node's
  // primitive conversion (its own row) and gradient (its and its
  // neighbours' rows), of every block's edge fluxes (the gradients of its
  // nodes and forward halo) and node assembly (its edge fluxes, those of
  // the blocks that spill into it, and its boundary fluxes)
  int pipeK = 8;                                    // chunks of caller rows
  std::vector<int> pipe_rows;                       // [pipeK + 1] first caller row of each chunk
  std::vector<unsigned char> h_st_prim, h_st_grad;  // [N] blocked nodes
  std::vector<unsigned char> h_st_flux, h_st_node;  // [nblk]
  std::vector<int> h_o2n;       // [N] caller row -> blocked node
};

// Residual of host arrays in K chunks of caller rows: the copy of chunk s
// of U, then the blocks whose stages it completes, while the next chunk is
// copied in and finished chunks of R are copied out (residual.cu).
struct ResidualPipe {
  int K = 0;
  int ggrid = 1;                     // CTAs of the persistent gradient kernel
  cudaStream_t sin = nullptr, sout = nullptr;
  std::vector<cudaEvent_t> ev_in, ev_stage;  // [K] chunk of U on the device; [K] stage s computed
  cudaEvent_t ev_go = nullptr, ev_out = nullptr;
  DBuf<int> lists;                   // node or block lists of every (kind, stage)
  std::vector<int> off;              // [5 kinds][K + 1] offsets into lists
  std::vector<int> out_stage;        // [K] stage after which caller chunk c of R is copied out
  // caller rows of R still being written when their chunk is copied out:
  // after the last stage (and after that chunk's copy has landed) a kernel
  // writes their final values into the page-locked R through its device
  // address
  DBuf<int> late;                    // [nlate] caller rows
  std::vector<int> h_late;
  int* h_bad = nullptr;              // page-locked unphysical count
  cudaEvent_t ev_pre = nullptr;      // the copies before the last stage's
  // each stage's kernels captured once as a graph, with its kernel count
  std::vector<cudaGraphExec_t> stage_exec;
  std::vector<const void*> graph_key;   // the device buffers they were recorded with
  std::vector<long long> stage_launches;
  ~ResidualPipe() {
    for (auto e : stage_exec) cudaGraphExecDestroy(e);
    if (h_bad) cudaFreeHost(h_bad);
    if (ev_pre) cudaEventDestroy(ev_pre);
    for (auto e : ev_in) cudaEventDestroy(e);
    for (auto e : ev_stage) cudaEventDestroy(e);
    if (ev_go) cudaEventDestroy(ev_go);
    if (ev_out) cudaEventDestroy(ev_out);
    if (sin) cudaStreamDestroy(sin);
    if (sout) cudaStreamDestroy(sout);
  }
};

struct Scratch {
  DBuf<double> G;          // [N][16] gradients ddx(5) ddy(5) ddz(5) pad
  DBuf<double> flux;       // [5][E] per-edge fluxes
  DBuf<double> fbuf;       // [3F][5] boundary subface fluxes
  DBuf<double> G2;         // [N][16] gradients, blocked numbering
  DBuf<double> part;       // [N][5] block-local flux sums, blocked numbering
  DBuf<double> spill;      // [nX][5] fluxes of block-crossing edges
  DBuf<double> Ustage, Rstage, Vstage, Xstage;  // staging for host arrays
  DBuf<double> dt, k1, k2, U0;
  DBuf<int> tag;           // [N] failsafe tags
  DBuf<int> counters;      // [8] device counters
  DBuf<double> red;        // reduction partials
  DBuf<double> tetc;       // [4T][4] Galerkin shares of each (tet, vertex)
  DBuf<double> viscq;      // [N][8] node records of the Galerkin term
  // set by the blocked residual: P2 / G2 hold the untagged primitive
  // records and gradients of the state it evaluated
  bool p2g2_valid = false;
  DBuf<double> redout;     // reduction results
};

// Implicit operator: BSR-by-rows of the H1 Jacobian.
struct Implicit {
  int precision = 0;       // 32 or 64, 0 = not assembled
  bool transposed = false; // blocks hold H1^T (row r = column r of H1)
  DBuf<double> diag64, off64, dinv64;   // [N][25], [2E][25], [N][25]
  DBuf<float> diag32, off32, dinv32;
  bool prec_ready = false;
  // Krylov workspace
  DBuf<double> basis;      // [(m+1)][5N]
  DBuf<double> w, r, x, b, t;
  DBuf<double> hcol;       // device scratch for one Hessenberg column
  // device-driven GMRES: Hessenberg matrix, rotations, g, y, estimate and
  // target, per-CTA partials; counters and barrier arrivals
  DBuf<double> gst;
  DBuf<int> gsti;
  // pinned copy of its done flag and the event that marks it current, for
  // the host's non-blocking polls inside a cycle
  struct Poll {
    int* done = nullptr;
    cudaEvent_t ev = nullptr;
    ~Poll() {
      if (done) cudaFreeHost(done);
      if (ev) cudaEventDestroy(ev);
    }
  } poll;
  DBuf<unsigned> ticket;   // grid-reduction ticket of the fused Gram-Schmidt kernels
  DBuf<double> fsum;       // [nbrow][25] boundary-face blocks of the boundary rows
  // preconditioner: AEROF_PC_JACOBI or AEROF_PC_ILU0 (block ILU(0) in the
  // multicolour ordering, factors in the sliced layout of the colour-ordered
  // rows with the diagonal inverted; factored for the operator read plainly
  // (ilu_tr = 0) or transposed (1)); iluw: the sweeps' work vectors
  int pc = 0;
  bool ilu_ready = false;
  int ilu_tr = 0;
  DBuf<double> ilu64, iluw;
  DBuf<float> ilu32;
  // flexible GMRES on the exact linearisation (outer FP64 vectors)
  DBuf<double> fV, fZ, fw, fr, fh;
  // finite-difference products (MatVecProdFD): perturbed states and
  // residuals, staged inputs, reduction partials
  DBuf<double> fdQ, fdFp, fdFm, fdIn, fdRed;
  // lockstep solves of several right-hand sides: outer (FP64) and inner
  // (FP32) bases and work vectors, Hessenberg columns, pointer arrays of the
  // batched kernels
  DBuf<double> bV, bZ, bw, br, bh, ih, bB, bX;
  DBuf<float> iV, iw, ir, iz;
  DBuf<unsigned long long> bptr, iptr;
};

// Dual-number work arrays of the forward-mode linearisation.
struct DualWork {
  DBuf<Dual> XD, PD, GD, WD, RD, volD, enD, fnD, fluxD;
  bool geom_static = false;  // dual geometry holds the primal with zero tangents
};

// Reverse-mode work arrays.
struct AdjWork {
  DBuf<double> edge;       // [E][20] per-edge cotangent contributions
  DBuf<double> gG;         // [N][16] gradient cotangents
  DBuf<double> gV;         // [N][5] direct state cotangents
  DBuf<double> lam;        // [N][5] w / vol
  DBuf<double> gd;         // [2E][3] least-squares offset cotangents
  DBuf<double> gvol;       // [N] control-volume cotangents
  DBuf<double> gfn;        // [F][3] face-normal cotangents
  // blocked reverse sweep
  DBuf<double> lam2;       // [N][6] w / vol in the blocked numbering (16-byte records)
  DBuf<double> gVp, gGp;   // [N][5], [N][16] in-block partial sums (blocked numbering)
  DBuf<double> spill;      // [nX][13] second-endpoint parts of block-crossing edges
  DBuf<double> geo;        // [E][6] cotangents of edge normal and dx per edge (original edge order)
  DBuf<double> tg;         // [T][12] per-tet vertex coordinate cotangents
  DBuf<double> gV2, gG2;   // [N][5], [N][16] assembled cotangents, blocked numbering
};

// Stored exact linearisation of the residual (the operator MatVecProdH2
// holds between evaluate and apply).  Per edge of the blocked organisation,
// kH2Rec doubles as 16-byte pairs, SoA by pair ([kH2Rec / 2][E] double2):
// (d phi_r / d Vij_c, d phi_r / d Vji_c) for r, c < 5, then (p1_c, p2_c)
// and (q1_c, q2_c), the partials of the reconstruction:
// dVij = (1-p1) dVi + p1 dVj + q1 dddij, dVji = p2 dVi + (1-p2) dVj -
// q2 dddji.  Per boundary row, SoA [25][nbrow]: the summed face-flux
// Jacobian d F / d V of its faces.
constexpr int kH2Rec = 70;
// Spalart-Allmaras model (turbulence.cu): constants, wall distances and
// the work arrays of its six-component residual
struct TurbWork {
  bool on = false;
  aerof_sa_params p = {};
  double Ub[6] = {0, 0, 0, 0, 0, 0};
  DBuf<double> Ubd;        // [6]
  DBuf<double> d2wall;     // [N]
  DBuf<double> V6;         // [N][6] primitive
  DBuf<double> G6;         // [N][18] LSQ gradients (x, y, z of the six components)
  DBuf<double> flux6;      // [E][6]
  DBuf<double> fbuf6;      // [3F][6]
  DBuf<double> tetc;       // [4T][5] SA Galerkin shares of each (tet, vertex)
  DBuf<double> q;          // [N][12] node records of the SA Galerkin term
  DBuf<double> Ustage, Rstage;
};

struct H2Op {
  bool ready = false;      // evaluated for the current mesh and coordinates
  bool use = false;        // exact products of linearised solves read it
  bool in_solves = false;  // linearised solves evaluate and use it
  int rec = 0;             // reconstruction it was evaluated with
  DBuf<double> a;          // [kH2Rec / 2][E] pairs
  DBuf<double> fj;         // [25][nbrow]
  DBuf<double> U;          // [N][5] state of the linearisation
  DBuf<double> dP2;        // [N][8] tangent records (dV, X), blocked numbering
  DBuf<double> dG2;        // [N][16] tangent gradients, blocked numbering
  DBuf<double> part;       // [N][5] block-local tangent flux sums
  DBuf<double> spill;      // [nX][5] tangent fluxes of block-crossing edges
};

// CUDA-event timers per category (AEROF_T_*), recorded without host sync.
struct Timers {
  bool on = false;
  int depth = 0;           // open scopes (only the outermost records)
  struct Rec { int cat; cudaEvent_t a, b; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double ms[AEROF_T_COUNT] = {0};
  long long cnt[AEROF_T_COUNT] = {0};
  ~Timers() {
    for (auto& r : recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

}  // namespace aerof

struct aerof_gpu_ctx {
  aerof_gpu_config cfg;
  int dev = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  bool has_mesh = false;
  aerof::DeviceMesh mesh;
  aerof::Scratch s;
  aerof::Implicit imp;
  aerof::DualWork dual;
  aerof::AdjWork adj;
  aerof::H2Op h2;
  aerof::TurbWork turb;
  aerof::Timers timers;
  std::string last_error;
  // device address of the allocation-free residual's fixed scratch array,
  // looked up at context creation (residual.cu)
  double* noalloc_scratch = nullptr;
  std::string noalloc_error;
  // rows [n_owned, N) are ghost rows of a subdomain mesh (set-up only)
  int n_owned = 0;
  // viscous Galerkin term (model 0: inviscid)
  aerof_viscous_params visc = {};
  // schedule and streams of the residual of host arrays (built on first use
  // for the current mesh)
  std::unique_ptr<aerof::ResidualPipe> pipe;
};

namespace aerof {

// Staging: return a device pointer holding the contents of `p` (count
// doubles); host arrays are copied into `stage`.
bool is_device_ptr(const void* p);
const double* in_dev(aerof_gpu_ctx* c, const double* p, size_t count, DBuf<double>& stage);
double* out_dev(aerof_gpu_ctx* c, double* p, size_t count, DBuf<double>& stage);
void out_finish(aerof_gpu_ctx* c, double* user, const double* dev, size_t count);

template <class F>
int guard(aerof_gpu_ctx* c, F&& f) {
  if (!c) return AEROF_EINVAL;
  try {
    cudaSetDevice(c->dev);
    return f();
  } catch (const CudaError& e) {
    c->last_error = std::string(e.where) + ": " + cudaGetErrorString(e.err);
    return AEROF_ECUDA;
  } catch (const ApiError& e) {
    c->last_error = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    c->last_error = e.what();
    return AEROF_EINVAL;
  }
}

inline int grid_for(size_t n, int block) { return (int)((n + block - 1) / block); }

// implemented in mesh.cu: geometry of coordinates XD ([N][3]) in dual
// numbers, same kernels and order as the primal set-up
void geometry_dual(aerof_gpu_ctx* c, const Dual* XD, Dual* volD, Dual* enD, Dual* fnD, Dual* RD);

// Timer scope: records start/stop events around the enclosed launches.
int timer_begin(aerof_gpu_ctx* c, int cat);
void timer_end(aerof_gpu_ctx* c, int handle);
struct TimerScope {
  aerof_gpu_ctx* c;
  int h;
  TimerScope(aerof_gpu_ctx* cc, int cat) : c(cc), h(timer_begin(cc, cat)) {}
  ~TimerScope() { timer_end(c, h); }
};

// ---- shared-memory staging helpers (residual and adjoint kernels)
// Strides (in doubles) of the node records staged in shared memory: 80 B
// for (V, X) and 144 B for the gradients, so that the 16-byte loads of 8
// lanes reading 8 different records fall into disjoint banks.
constexpr int kPS = 10;
constexpr int kGS = 18;

// 16-byte global -> shared copy that completes asynchronously (cp.async,
// cached in L2 only); cp_async_wait_all() waits for this thread's copies.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// 8-byte variant (cached in L1 and L2)
__device__ __forceinline__ void cp_async8(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
// Bulk prefetch of a contiguous global range into L2 (no destination, no
// completion to wait for): src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void prefetch_l2_bulk(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
// The stored operator's pairs of edges [e0, e1): one bulk L2 prefetch per
// pair array ([npair][E] double2), issued by the first npair threads.
__device__ __forceinline__ void prefetch_pairs_l2(const double2* h2, size_t E, int e0, int e1, int npair) {
  const int k = threadIdx.x;
  if (k < npair && e1 > e0) prefetch_l2_bulk(h2 + (size_t)k * E + e0, 16u * (unsigned)(e1 - e0));
}

// implemented in residual.cu (used by implicit.cu and adjoint.cu).  With
// sync == false the unphysical count is left on the device (counters[2]).
int residual_dev(aerof_gpu_ctx* c, const double* dU, double* dR, bool sync = true);
void prim_dev(aerof_gpu_ctx* c, const double* dU);
void prim_grad_blocked_dev(aerof_gpu_ctx* c, const double* dU, const int* tag);
void grad_records_blocked_dev(aerof_gpu_ctx* c, const double* P2src, double* G2dst);
void gradients_dev(aerof_gpu_ctx* c);
void timestep_dev(aerof_gpu_ctx* c, const double* dU, double cfl, double* ddt);
double norm2_dev(aerof_gpu_ctx* c, const double* x, size_t n);
double dot_dev(aerof_gpu_ctx* c, const double* x, const double* y, size_t n);

// implemented in adjoint.cu
int residual_forward(aerof_gpu_ctx* c, const double* dU, const double* dv, const double* dXdot, double* ddR,
                     bool sync = true);
void vjp_dev(aerof_gpu_ctx* c, const double* dU, const double* dw, double* dout);
// exact product of the linearised solves: the stored operator when h2.use,
// else the matrix-free sweeps at dU
void exact_product(aerof_gpu_ctx* c, const double* dU, const double* p, double* y, bool trans);
// the stored operator at dU (h2.ready on return)
void h2_evaluate_dev(aerof_gpu_ctx* c, const double* dU);
// implemented in mesh.cu: recompute the geometry for new coordinates
void compute_geometry(aerof_gpu_ctx* c);
// implemented in viscous.cu: R += (viscous Galerkin term of U) / ctrlVol
// when a viscous model is set (no allocation: the per-tet buffer is sized
// by galerkin_reserve, which set_mesh and set_viscosity call)
void galerkin_add(aerof_gpu_ctx* c, const double* dU, double* dR);
void galerkin_reserve(aerof_gpu_ctx* c, int model);

// Node side of a Galerkin term evaluated once per tet: the tet kernel wrote
// node k's share of tet t as the W-double record C[W (4t + k)]; thread
// (i, k) sums component k of the records of node i's tets in ascending tet
// order (nt_tet holds 4t + k, ascending in t) and adds the sum / vol[i] to
// R[RS i + R0 + k].  W consecutive threads read one record.
template <int W, int RS, int R0>
__global__ void k_tet_gather(int N, const int* __restrict__ nt_ptr, const int* __restrict__ nt_tet,
                             const double* __restrict__ C, const double* __restrict__ vol, double* __restrict__ R) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (long long)N * W) return;
  const int i = (int)(j / W), k = (int)(j - (long long)i * W);
  double acc = 0.0;
  int q = nt_ptr[i];
  const int qe = nt_ptr[i + 1];
  // four records in flight per step; the sum keeps ascending tet order
  for (; q + 4 <= qe; q += 4) {
    const int4 tl = make_int4(nt_tet[q], nt_tet[q + 1], nt_tet[q + 2], nt_tet[q + 3]);
    const double c0 = __ldcs(C + W * (size_t)tl.x + k), c1 = __ldcs(C + W * (size_t)tl.y + k);
    const double c2 = __ldcs(C + W * (size_t)tl.z + k), c3 = __ldcs(C + W * (size_t)tl.w + k);
    acc += c0;
    acc += c1;
    acc += c2;
    acc += c3;
  }
  for (; q < qe; ++q) acc += __ldcs(C + W * (size_t)nt_tet[q] + k);
  const double iv = 1.0 / vol[i];
  R[RS * (size_t)i + R0 + k] += acc * iv;
}
// the exact linearisations cover the inviscid residual only
inline void need_inviscid(aerof_gpu_ctx* c) {
  if (c->visc.model != 0)
    throw ApiError{AEROF_EINVAL, "the exact linearisation of the viscous term is not built: set model 0"};
}
// implemented in residual.cu: device address of the allocation-free
// residual's scratch array for the current device, kept in the context
void noalloc_attach(aerof_gpu_ctx* c);

}  // namespace aerof
