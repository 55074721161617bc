/*
 * aerof_gpu.h -- C ABI of the B200 (sm_100a) implementation of AERO-F's
 * implicit edge-based finite-volume hot path.
 *
 * AERO-F has no plugin or FFI layer: the hot path is reached through C++
 * template classes (SpaceOperator<dim>, MatVecProd<dim,neq>,
 * KspPrec<dim,Scalar>, KspSolver<...>).  Each entry point below replaces one
 * member of that call surface; the citation names the reference function
 * (file:line in the AERO-F tree) whose contract it keeps.  A C++ shim
 * subclasses those classes and forwards to these entry points.
 *
 * Conventions
 *  - Every function returns int: 0 = AEROF_OK, > 0 = number of unphysical
 *    states detected (a warning, the result is still written), < 0 = error.
 *  - State and residual vectors use the reference's layout: double[N][5]
 *    (AoS, one node after the other, node numbering of the mesh passed to
 *    aerof_gpu_set_mesh), conservative (rho, rho u, rho v, rho w, E) for U.
 *  - Any array argument may be host memory (pageable or pinned) or device
 *    memory of the context's GPU; the library detects which and stages host
 *    arrays through its own device buffers on the context's stream.  All
 *    calls are synchronous with respect to the host on return.
 *  - One context is used by one host thread at a time.
 *  - No call spins on device flags; device-side failures are counted into a
 *    device error word and returned as status codes.
 */
#ifndef AEROF_GPU_H
#define AEROF_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AEROF_OK 0
#define AEROF_EINVAL -1    /* bad argument */
#define AEROF_ENOMEM -2    /* device allocation failed */
#define AEROF_ECUDA -3     /* CUDA runtime error */
#define AEROF_ETIMEDOUT -4 /* bounded wait expired */
#define AEROF_ESINGULAR -5 /* zero pivot in a 5x5 diagonal block */
#define AEROF_ESTATE -6    /* call order violated (e.g. no mesh set) */
#define AEROF_EDIVERGED -7 /* Newton updates stayed non-physical down to
                              CFL cfl0/1000 (TsParameters.C:187-195)      */

/* Boundary codes (BcDef.h:5-28) understood by the face kernels. */
#define AEROF_BC_SLIP_WALL_MOVING -2
#define AEROF_BC_INLET_MOVING -4
#define AEROF_BC_OUTLET_MOVING -5

/* Reconstruction (SchemeData, IoDataCore.C:2415-2435). */
#define AEROF_REC_CONSTANT 1  /* first order: RecFcnConstant                     */
#define AEROF_REC_VANALBADA 2 /* LSQ gradients + van Albada, RecFcnVanAlbada<5>   */
#define AEROF_REC_LINEAR 3    /* LSQ gradients + unlimited MUSCL, RecFcnLinear<5> */

/* Preconditioner of the Krylov solvers (PcData::type, IoDataCore.C:2735-2760):
 * block-Jacobi (JacobiPrec), or block ILU(0) (IluPrec with fill 0,
 * SparseMat::numericILU / lusol, SparseMatrix.C:353-450) of the same
 * operator on a colour-major node ordering (greedy colouring of the node
 * graph) instead of the reference's RCM order, so that every colour
 * factors and solves in parallel.                                         */
#define AEROF_PC_JACOBI 0
#define AEROF_PC_ILU0 1

/* Precision of the assembled H1 Jacobian and block-Jacobi preconditioner. */
#define AEROF_PREC_FP64 64
#define AEROF_PREC_FP32 32 /* FP32 blocks, FP64 vectors and accumulation */

typedef struct aerof_gpu_ctx aerof_gpu_ctx;

/* The few IoData fields the path uses (IoDataCore.C:2415-2435, 3160). */
typedef struct aerof_gpu_config {
  double gamma;      /* ratio of specific heats (GasModelData), 1.4        */
  double beta;       /* MUSCL beta (SchemeData::beta), 1/3                 */
  int reconstruction;/* AEROF_REC_*                                          */
  int failsafe;      /* 1: tag nodes with non-positive reconstructed rho/p,
                        zero their gradients and recompute (Domain.C:876-918) */
  int device;        /* CUDA device ordinal                                  */
  int residual_kernel;/* AEROF_KERNEL_* (0: blocked, the default)           */
  int reserved[4];
} aerof_gpu_config;

/* Residual kernel organisation (same result within rounding):
 * BLOCKED: nodes renumbered along a Morton curve, one thread block per 256
 *   nodes evaluates the fluxes of the edges it owns into shared memory and
 *   assembles them there; only edges that cross blocks go through global
 *   memory.  Per-node sums run in a fixed order, not the reference's.
 * EDGE: one thread per edge writes its flux to global memory, every node
 *   then sums its edges in the reference's order (ascending neighbour).   */
#define AEROF_KERNEL_BLOCKED 0
#define AEROF_KERNEL_EDGE 1

/* Steady pseudo-transient Newton-Krylov parameters (TsData/CFLData/KspData,
 * IoDataCore.C:2896-2911, 3067-3089; IoData.C:9-20). */
typedef struct aerof_newton_params {
  double cfl0, cfl_min, cfl_max, ser; /* RESIDUAL CFL law (TsParameters.C:211-217) */
  double ksp_eps;                     /* GMRES relative tolerance (1e-2)            */
  double tol;                         /* stop at ||R(Q)||/||R(Q0)|| <= tol          */
  int ksp_krylov;                     /* GMRES restart length (30)                  */
  int ksp_maxits;                     /* GMRES max iterations (30)                  */
  int max_steps;                      /* pseudo-time steps                          */
  int precision;                      /* AEROF_PREC_FP32 or AEROF_PREC_FP64         */
  int reserved[4];
} aerof_newton_params;

typedef struct aerof_newton_result {
  int steps;            /* pseudo-time steps taken                   */
  int linear_its;       /* total GMRES iterations                    */
  double rel_residual;  /* final ||R||/||R0||                        */
  double seconds;       /* device time of the solve (CUDA events)    */
  int redos;            /* steps redone at half the CFL number after a
                           non-physical update (NewtonSolver.h:195-205) */
  int reserved[3];
} aerof_newton_result;

/* ---- context ---------------------------------------------------------- */
int aerof_gpu_create(const aerof_gpu_config* cfg, aerof_gpu_ctx** out);
int aerof_gpu_destroy(aerof_gpu_ctx* ctx);
/* Run subsequent work on this cudaStream_t (NULL: the context's own stream). */
int aerof_gpu_set_stream(aerof_gpu_ctx* ctx, void* stream);
/* Number of kernels the library has launched (all contexts of the process)
 * since the previous call; the counter restarts at 0.  Diagnostics only, no
 * reference counterpart. */
int aerof_gpu_launch_count(long long* count);
/* Last error message of this context (NUL-terminated, truncated to len). */
int aerof_gpu_last_error(aerof_gpu_ctx* ctx, char* buf, int len);

/* ---- mesh -------------------------------------------------------------
 * Replaces GeoSource/SubDomain construction plus the static-mesh geometry
 * DistGeoState::compute (DistGeoState.C:542-600): edges are the unique node
 * pairs of the tets numbered lexicographically (EdgeSet::createPointers,
 * EdgeCore.C:92-117); edge normals ElemTet::computeEdgeNormalsGCL1
 * (ElemTetCore.C:281-330), face normals FaceTria::computeNormalGCL1
 * (FaceTriaCore.C:65-82), control volumes (ElemTetCore.C:102-112) and the
 * least-squares factors (SubDomainCore.C:1334-1381, 1755-1777).
 * X[N][3], tets[T][4] (positively oriented), faces[F][3] (outward by
 * 0.5*((x2-x0)^(x1-x0))), codes[F] (AEROF_BC_*), Ub[5] the conservative
 * free-stream state of every far-field face (DistBcData.C:652-730).       */
int aerof_gpu_set_mesh(aerof_gpu_ctx* ctx, int N, int T, int F, const double* X, const int* tets,
                       const int* faces, const int* codes, const double* Ub);
/* New node coordinates X[N][3] for the same topology: recomputes the
 * static geometry (DistGeoState::compute with a moved mesh, as the shape
 * finite differences of fsoSemiAnalytical do, FluidShapeOptimizationHandler.C:
 * 1216-1363).                                                               */
int aerof_gpu_update_coordinates(aerof_gpu_ctx* ctx, const double* X);
int aerof_gpu_mesh_sizes(aerof_gpu_ctx* ctx, int* N, int* E, int* F);
/* Edge list [E][2] (i<j), lexicographic: EdgeSet::getPtr (Edge.h). */
int aerof_gpu_get_edges(aerof_gpu_ctx* ctx, int* edges);
/* Geometry in reference numbering: edge normals [E][3], face normals [F][3],
 * control volumes [N], least-squares factors [N][6] (r11 r12 r13 r22 r23 r33). */
int aerof_gpu_get_geometry(aerof_gpu_ctx* ctx, double* edge_normal, double* face_normal,
                           double* ctrl_vol, double* lsq_R);

/* ---- residual ---------------------------------------------------------
 * SpaceOperator<5>::computeResidual(X, ctrlVol, U, R, timeState)
 * (SpaceOperator.h:171-173, SpaceOperator.C:524-634): R = (sum of Roe edge
 * fluxes + boundary fluxes)/ctrlVol for the configured reconstruction.
 * Returns the number of non-positive reconstructed densities/pressures
 * (EdgeCore.C:137-168) -- 0 on a healthy state.                          */
int aerof_gpu_residual(aerof_gpu_ctx* ctx, const double* U, double* R);
/* Same as aerof_gpu_residual for device-resident U and R, without waiting
 * for the GPU: the call only enqueues work on the context's stream.  The
 * count of non-positive reconstructed states accumulates on the device and
 * is returned (and reset) by aerof_gpu_status.  Requires failsafe == 0
 * (the failsafe re-run needs the count on the host), AEROF_EINVAL otherwise. */
int aerof_gpu_residual_async(aerof_gpu_ctx* ctx, const double* U, double* R);
/* Waits for the context's stream; returns the accumulated unphysical count
 * of asynchronous calls since the previous aerof_gpu_status (>= 0) or an
 * error code.                                                              */
int aerof_gpu_status(aerof_gpu_ctx* ctx);
/* Same result as aerof_gpu_residual, but the call allocates no memory: it is
 * for callers that cannot allocate device memory while they run (an
 * application that has handed all device memory to its own pool, a thread
 * that must not take the allocator's locks).  This entry point has no
 * counterpart in the reference; it is an addition of this library.
 * - U and R must be device pointers (host arrays would need staging buffers).
 * - Scratch (per-edge fluxes, gradients, tags, counters) lives in one fixed
 *   16 MiB array of device memory inside the library.  aerof_gpu_create
 *   claims it on the context's device (it loads the library's residual
 *   module and looks up the array's device address there), so the 16 MiB
 *   are taken at context set-up, before the caller hands the rest of the
 *   device to its own pool, and stay taken until the process exits.
 *   Meshes needing more than a(a(5E) + 16N) + (N + 8)/2 <= 2,097,152 doubles
 *   (a(x): x rounded up to a multiple of 32; about 40,000 nodes) are
 *   rejected with AEROF_EINVAL and a message in aerof_gpu_last_error.
 * - Every call shares the array and the previous call's contents stay in it
 *   (the call clears what must start at zero).  Calls that overlap on the GPU
 *   -- on other streams or from other contexts on the same device -- race.
 * Returns the unphysical-state count like aerof_gpu_residual.              */
int aerof_gpu_residual_noalloc(aerof_gpu_ctx* ctx, const double* U, double* R);
/* DistNodalGrad::compute, least squares (DistNodalGrad.C:790-806,
 * SubDomain.C:297-374) of primitive V[N][5]; ddx/ddy/ddz [N][5].        */
int aerof_gpu_gradients(aerof_gpu_ctx* ctx, const double* V, double* ddx, double* ddy, double* ddz);
/* DistTimeState::computeTimeStep with local time stepping
 * (DistTimeState.C:746-801, Domain.C:30-100, Edge.C:87-143, Face.C:242-289):
 * dt[N] = cfl*vol/(-sum of wave-speed terms).                             */
int aerof_gpu_timestep(aerof_gpu_ctx* ctx, const double* U, double cfl, double* dt);
/* ExplicitTsDesc::computeRKSecondOrder (ExplicitTsDesc.C:98-117), nsteps
 * local-time-step Heun steps at fixed cfl, U[N][5] updated in place.     */
int aerof_gpu_rk2(aerof_gpu_ctx* ctx, double* U, double cfl, int nsteps);

/* ---- viscous term -----------------------------------------------------
 * The laminar Navier-Stokes Galerkin term that SpaceOperator::
 * computeResidual adds when a FemEquationTerm is present (SpaceOperator.C:
 * 570-573; ElemTet::computeGalerkinTerm, ElemTet.C:24-127;
 * FemEquationTermNS::computeVolumeTerm, FemEquationTermDesc.C:98-160):
 * model 0 inviscid (default), 1 constant viscosity (ConstantViscoFcn,
 * mu = 1, lambda = bulk_viscosity - 2/3 mu), 2 Sutherland (mu = T^1.5
 * (1 + Ts)/(T + Ts) with T = sutherland_alpha * T_adim, alpha =
 * gamma (gamma - 1) M^2, Ts = sutherlandReferenceTemperature / reference
 * temperature; lambda = -2/3 mu), conductivity cp mu / prandtl, all scaled
 * by 1/reynolds_mu (ViscoFcn.h:46-103, ThermalCondFcn.h:52-75).  Every
 * residual evaluation (aerof_gpu_residual and its variants, RK2, Newton)
 * then includes it.  The local time step keeps the inviscid spectral
 * radius (the reference's default, TsData::viscousCst = 0), and the H1
 * operator of the Newton solves stays the first-order inviscid one (a
 * defect correction); the exact linearisations (jvp, vjp, dR/dX, the stored
 * operator, linearised solves) return AEROF_EINVAL with a viscous model.   */
typedef struct aerof_viscous_params {
  int model;               /* 0, 1 or 2 as above                              */
  double reynolds_mu;      /* Reynolds number of the viscosity               */
  double prandtl;          /* Prandtl number                                  */
  double bulk_viscosity;   /* constant model                                  */
  double sutherland_alpha; /* gamma (gamma - 1) M^2                           */
  double sutherland_Ts;    /* Sutherland temperature / reference temperature */
  int reserved[4];
} aerof_viscous_params;
int aerof_gpu_set_viscosity(aerof_gpu_ctx* ctx, const aerof_viscous_params* p);

/* ---- Spalart-Allmaras turbulence model ---------------------------------
 * The one-equation model strongly coupled to the flow, state U = (rho,
 * rho u, rho v, rho w, E, rho nu~) per node (dim 6; VarFcnSGSA.h:210-224).
 * Finite-volume term: the second-order edge loop on six components with
 * the Roe flux's advected sixth component (FluxFcnSGApprJacRoeSA3D::compute,
 * FluxFcnDescSG.C:1886-1901 -> roeflux7.f type 1), slip walls
 * (FluxFcnSGWallSA3D, FluxFcnDescSG.C:2024-2035) and far field
 * (FluxFcnSGOutflowSA3D for inlet and outlet, FluxFcn.h:246-262 ->
 * boundflux5.f type 1).  Galerkin term (with the viscous model of
 * aerof_gpu_set_viscosity; model 0 leaves it out):
 * FemEquationTermSA::computeVolumeTerm (FemEquationTermDesc.C:669-787):
 * eddy viscosity mu_t = mu~ fv1, lambda_t = -2/3 mu_t, kappa_t = cp mu_t /
 * prandtl_turbulent in the Navier-Stokes stress and heat flux, SA
 * diffusion and source (production, destruction with the wall distance,
 * cb2 gradient term) per tet; constants as SATerm::SATerm
 * (SpalartAllmarasTerm.h:77-112).                                         */
typedef struct aerof_sa_params {
  double cb1, cb2, cw2, cw3, cv1, cv2, sigma, vkcst; /* reference defaults
                             0.1355 0.622 0.3 2.0 7.1 5.0 2/3 0.41        */
  double prandtl_turbulent;  /* 0.9                                          */
  int fv3;                   /* 1: the fv3 form (SAModelData::FV3)           */
  int reserved[3];
} aerof_sa_params;
/* Turns the model on: constants, the wall distance of every node d2wall
 * [N] (caller numbering) and the conservative free stream Ub [6] of the
 * far-field boundaries (rho nu~ last).  p == NULL turns it off.             */
int aerof_gpu_set_turbulence(aerof_gpu_ctx* ctx, const aerof_sa_params* p, const double* d2wall,
                             const double* Ub);
/* R = residual(U) / ctrlVol for U, R [N][6] (host or device).  Returns the
 * number of non-positive reconstructed states (>= 0) or an error.          */
int aerof_gpu_residual_sa(aerof_gpu_ctx* ctx, const double* U, double* R);

/* ---- implicit operator ------------------------------------------------
 * MatVecProdH1<5,MatScalar,5>::evaluate (MatVecProd.C:1074-1160) =
 * SpaceOperator::computeJacobian (SpaceOperator.C:2088-2150) +
 * TimeState::addToJacobian (TimeState.C:731-756): first-order approximate
 * Roe Jacobian (roejac6.f), FD far-field and analytic wall face blocks,
 * diag/ctrlVol, + I/dt.  dt may be NULL (no time term).  precision selects
 * FP32 or FP64 block storage.                                              */
int aerof_gpu_jacobian(aerof_gpu_ctx* ctx, const double* U, const double* dt, int precision);
/* The assembled H1 operator in MvpMat layout a[N+2E][25] (MvpMatrix.h:10-80),
 * reference numbering, as double.                                          */
int aerof_gpu_get_jacobian(aerof_gpu_ctx* ctx, double* A);
/* The reverse of aerof_gpu_get_jacobian: an H1 operator assembled by the
 * caller, in the MvpMat layout a[N+2E][25] (reference numbering, as
 * MvpMat<Scalar,5> holds it, MvpMatrix.h:10-80), becomes the context's
 * operator in the given precision, as if aerof_gpu_jacobian had assembled it
 * (a caller that adds terms of its own to the matrix, or one that keeps
 * the reference's assembly).                                              */
int aerof_gpu_set_jacobian(aerof_gpu_ctx* ctx, const double* A, int precision);
/* MatVecProdH1::apply / applyTranspose (MatVecProd.C:1165-1208,
 * SubDomain.C:3916-3995): y = A p or A^T p, p,y [N][5].                   */
int aerof_gpu_matvec(aerof_gpu_ctx* ctx, const double* p, double* y, int transpose);
/* MatVecProdFD::apply (MatVecProd.C:262-372): finite-difference product of
 * the configured residual, prod = (F(U + eps p) - F(U)) / eps (fd_order 1)
 * or (F(U + eps p) - F(U - eps p)) / (2 eps) (fd_order 2), with
 * F = R + (U' - U)/dt when dt[N] is given (the backward-Euler time term,
 * TimeState::add_dAW_dt, TimeState.C:40-73) and the reference's step
 * (computeEpsilon, MatVecProd.C:879-929): eps = sum over the 5N state
 * entries of (1e-6 |U| + 1e-6) / (5N ||p||), or 1e-6 when ||p|| < 1e-14.
 * F (optional, first order only) is R(U) as MatVecProdFD::evaluate keeps
 * it; without it R(U) is evaluated.  eps (optional) receives the step.    */
int aerof_gpu_matvec_fd(aerof_gpu_ctx* ctx, const double* U, const double* F, const double* p, const double* dt,
                        int fd_order, double* prod, double* eps);
/* JacobiPrec::getData + setup (KspPrec.C:75-82,115-124; DiagMatrix.C:44-80):
 * invert the 5x5 diagonal blocks (LINPACK dgefa/dgedi) in the Jacobian's
 * precision.  Returns AEROF_ESINGULAR on a zero pivot.                    */
int aerof_gpu_prec_setup(aerof_gpu_ctx* ctx);
/* JacobiPrec::apply / applyT (KspPrec.C:86-111): y = D^-1 x or D^-T x;
 * with AEROF_PC_ILU0, IluPrec::apply (y = (LU)^-1 x, factors of H1 or, for
 * transpose = 1, of H1^T).                                                 */
int aerof_gpu_prec_apply(aerof_gpu_ctx* ctx, const double* x, double* y, int transpose);
/* Subdomain meshes (one per rank of a decomposed mesh, owned nodes first,
 * then the ghost nodes whose states the caller exchanges between ranks,
 * the role of DistInfo::masterFlag, DistVector.h:1435-1452): rows
 * [n_owned, N) are ghost rows, whose block-Jacobi blocks are taken as the
 * identity (their partial diagonal blocks are not used and may be
 * singular).  Default after aerof_gpu_set_mesh: n_owned = N.              */
int aerof_gpu_set_owned_rows(aerof_gpu_ctx* ctx, int n_owned);
/* Selects the preconditioner of aerof_gpu_prec_setup / _apply, the GMRES,
 * Newton and linearised solves: AEROF_PC_JACOBI (default) or
 * AEROF_PC_ILU0 (IluPrec::setup / apply, KspPrec.C:220-260).               */
int aerof_gpu_set_preconditioner(aerof_gpu_ctx* ctx, int type);
/* GmresSolver::solve / solveT (KspSolver.C:351-492, 752-915): right-
 * preconditioned GMRES(krylov) with modified Gram-Schmidt in FP64, x0 = 0.
 * its receives the iteration count (== maxits means saturation, the
 * reference's SATURATED_LS), res the final estimated residual norm.       */
int aerof_gpu_gmres(aerof_gpu_ctx* ctx, const double* b, double* x, int krylov, int maxits,
                    double eps, int transpose, int* its, double* res);
/* TsSolver::resolve + NewtonSolver::solve (maxIts=1) for a steady problem
 * (TsSolver.h:231-380, NewtonSolver.h:70-231, ImplicitCoupledTsDesc.C:
 * 85-300): U[N][5] updated in place; history (optional, max_steps+1
 * entries) receives ||R||/||R0|| per step.  After every update the state
 * is checked (SubDomain::checkSolution, SubDomain.C:6746-6806): if a node
 * has a non-positive (or non-finite) density or pressure, U is restored and
 * the step redone at half the CFL number (NewtonSolver.h:195-205,
 * TsParameters.C:187-195); out->redos counts those.  When the CFL number
 * falls below cfl0/1000 the call returns AEROF_EDIVERGED with U restored to
 * the last physical state.  A non-finite residual returns AEROF_EINVAL.    */
int aerof_gpu_newton(aerof_gpu_ctx* ctx, double* U, const aerof_newton_params* p,
                     aerof_newton_result* out, double* history);

/* ---- timers ------------------------------------------------------------
 * The reference's Timer categories (Timer.h:12-70: addNodalGradTime,
 * addFiniteVolumeTermTime, addTimeStepTime, addFiniteVolumeJacTime,
 * addPrecSetupTime, addKspTime) measured with CUDA events on the context's
 * stream while profiling is enabled.                                        */
#define AEROF_T_NODAL_GRAD 0    /* conservative->primitive + LSQ gradients   */
#define AEROF_T_FV_TERM 1       /* boundary fluxes + node assembly; edge
                                   fluxes too outside the blocked kernel    */
#define AEROF_T_TIME_STEP 2
#define AEROF_T_FV_JAC 3
#define AEROF_T_PREC_SETUP 4
#define AEROF_T_KSP_MATVEC 5
#define AEROF_T_KSP_OTHER 6     /* orthogonalisation, preconditioner apply   */
#define AEROF_T_FV_EDGES 7      /* edge fluxes of the blocked residual kernel
                                   (with AEROF_T_FV_TERM: the whole term)   */
#define AEROF_T_COUNT 8
int aerof_gpu_profile(aerof_gpu_ctx* ctx, int enable);
/* Waits for the stream, then returns per category the summed device time
 * in milliseconds and the number of timed intervals, and resets them.     */
int aerof_gpu_timers(aerof_gpu_ctx* ctx, double* ms, long long* count, int n);

/* ---- sensitivities ----------------------------------------------------
 * Exact linearisation of the configured residual (the operator
 * MatVecProdH2 applies, MatVecProd.C:1462-1704; derivative routines
 * Edge.C:1451-1573, RecFcn.h:451-526, g_roeflux*.f, g_boundflux5.f):     */
/* Jv = dR/dU . v                                                            */
int aerof_gpu_jvp(aerof_gpu_ctx* ctx, const double* U, const double* v, double* Jv);
/* JTw = (dR/dU)^T . w  (MatVecProdH2::applyTranspose, MatVecProd.C:1685-1704) */
int aerof_gpu_vjp(aerof_gpu_ctx* ctx, const double* U, const double* w, double* JTw);
/* dR = dR/dX . Xdot, Xdot[N][3] (SpaceOperator::computeDerivativeOfResidual
 * through normals, ctrlVol, LSQ factors and dx; fsoAnalytical,
 * FluidShapeOptimizationHandler.C:1368-1430)                               */
int aerof_gpu_dRdX(aerof_gpu_ctx* ctx, const double* U, const double* Xdot, double* dR);
/* gX = (dR/dX)^T . lambda, gX[N][3] (fsoApply_dFdXtranspose,
 * FluidShapeOptimizationHandler.C:1434-1448)                               */
int aerof_gpu_dRdX_T(aerof_gpu_ctx* ctx, const double* U, const double* lambda, double* gX);
/* Both products of the adjoint gradient from one reverse sweep over the
 * edges: JTl = (dR/dU)^T . lambda and gX = (dR/dX)^T . lambda (the two
 * operators fsoComputeAdjoint and fsoApply_dFdXtranspose apply,
 * FluidShapeOptimizationHandler.C:1434-1448, 2475-2502).                  */
int aerof_gpu_adjoint_products(aerof_gpu_ctx* ctx, const double* U, const double* lambda, double* JTl,
                               double* gX);

/* Stored exact linearisation (MatVecProdH2, MatVecProd.C:1462-1704).
 * evaluate (MatVecProd.C:1498-1520; SubDomain::precomputeRec
 * SubDomain.C:3836-3865 and computeH2): linearises the residual at U and
 * keeps, per edge, the flux Jacobians with respect to both reconstructed
 * states and the partials of the reconstruction, and per boundary node the
 * face-flux Jacobian: 560 bytes per edge + 200 per boundary node + 40 per
 * node of device memory.  apply (transpose = 0: y = J p) and
 * applyTranspose (transpose = 1: y = J^T p) (MatVecProd.C:1622-1704;
 * SubDomain::computeMatVecProdH2, SubDomain.C:4076-4190) read it; the
 * results equal aerof_gpu_jvp / aerof_gpu_vjp at U within rounding.  The
 * operator stays valid until the mesh or its coordinates change.         */
int aerof_gpu_h2_evaluate(aerof_gpu_ctx* ctx, const double* U);
int aerof_gpu_h2_apply(aerof_gpu_ctx* ctx, const double* p, double* y, int transpose);
/* Frees the stored operator's device memory.                              */
int aerof_gpu_h2_release(aerof_gpu_ctx* ctx);
/* Exact products of aerof_gpu_linearized_solve: stored = 0 (default)
 * re-evaluates the linearisation per product (no operator storage);
 * stored = 1 evaluates the stored operator at U once per solve and applies
 * it to every Krylov vector (the reference's MatVecProdH2 path).          */
int aerof_gpu_set_exact_operator(aerof_gpu_ctx* ctx, int stored);

/* Linearised steady solves with the exact Jacobian applied matrix-free
 * (fsoLinearSolver / fsoAdjointLinearSolver, FluidShapeOptimizationHandler.C:
 * 1557-1624; GmresSolver::solve / solveT): transpose = 0 solves J x = b,
 * transpose = 1 solves J^T x = b to ||r|| <= eps ||b||.
 * inner_its = 0: GMRES(krylov) right-preconditioned by the block-Jacobi of
 * the FP64 first-order operator at U (no time term).
 * inner_its > 0: flexible GMRES(krylov) whose preconditioner is inner_its
 * iterations of the mixed-precision GMRES on the first-order operator (FP32
 * blocks and Krylov vectors, block-Jacobi); the outer iteration and the
 * exact products stay FP64.  its = outer iterations.                       */
int aerof_gpu_linearized_solve(aerof_gpu_ctx* ctx, const double* U, const double* b, double* x, int krylov,
                               int maxits, double eps, int transpose, int inner_its, int* its, double* res);

/* Batched linearised solves sharing one operator set-up (the direct
 * sensitivities of several shape modes, FluidShapeOptimizationHandler.C:
 * 2362-2433, one fsoLinearSolver per mode): B and X are [nrhs][N][5]; the
 * stored exact linearisation at U is evaluated once (as
 * aerof_gpu_h2_evaluate), the first-order operator and its preconditioner
 * are assembled once, and every right-hand side is solved as
 * aerof_gpu_linearized_solve does with the stored operator's products; with
 * 0 < inner_its <= 30 the right-hand sides run in lockstep groups whose
 * inner FP32 solves share the passes over H1 and its preconditioner.
 * its[k], res[k]: outer iterations and final residual norm of each.       */
int aerof_gpu_linearized_solve_batch(aerof_gpu_ctx* ctx, const double* U, int nrhs, const double* B, double* X,
                                     int krylov, int maxits, double eps, int transpose, int inner_its, int* its,
                                     double* res);

/* ---- pre-partitioned mesh files ---------------------------------------
 * Reader of AERO-F's binary mesh and decomposition files (host only):
 * GeoSource::readConnectivityInfo (GeoSource.C:94-141) opens the
 * connectivity file and names the clusters' geometry and decomposition
 * files (prefix + cluster suffix, computeClusterSuffix in
 * BinFileHandler.h); GeoSource::getSubDomain (GeoSource.C:256-444) reads
 * one subdomain: nodes (NodeSet::read, Node.C:7-50), tets
 * (ElemSet::read, ElemCore.C:135-199), boundary triangles
 * (FaceSet::read, FaceCore.C:270-330; file code 6 becomes symmetry, 11),
 * neighbour subdomains and shared nodes.  Both byte orders are read
 * (BinFileHandler's header).  Arrays come back in the subdomain's local
 * node numbering (cluster order), with local-to-global maps (0-based).
 * aerof_sower_subdomain_sizes then aerof_sower_read_subdomain with arrays
 * of those sizes: X[nn][3], node_l2g[nn], tets[ne][4], elem_l2g[ne],
 * faces[nf][3], codes[nf], face_l2g[nf], neighb[nb], shared_ptr[nb+1],
 * shared[ns]; any array may be NULL.                                      */
typedef struct aerof_sower aerof_sower;
int aerof_sower_open(const char* con_file, const char* geo_prefix, const char* dec_prefix, aerof_sower** out);
int aerof_sower_close(aerof_sower* s);
int aerof_sower_num_subdomains(aerof_sower* s, int* nsub, int* nclusters);
int aerof_sower_subdomain_sizes(aerof_sower* s, int isub, int* nnodes, int* nelems, int* nfaces, int* nneighb,
                                int* nshared);
int aerof_sower_read_subdomain(aerof_sower* s, int isub, double* X, int* node_l2g, int* tets, int* elem_l2g,
                               int* faces, int* codes, int* face_l2g, int* neighb, int* shared_ptr, int* shared);
int aerof_sower_last_error(aerof_sower* s, char* buf, int len);

#ifdef __cplusplus
}
#endif

#endif /* AEROF_GPU_H */
