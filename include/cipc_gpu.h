/*
 * cipc_gpu.h - C ABI of the B200 IPC Newton pipeline.
 *
 * A host that today calls the CPU simulator's per-step solver binds these
 * plain-C entry points instead.  All arrays are host pointers with sizes given
 * explicitly; positions are AoS xyz doubles, indices are 0-based int32.
 * Every function returns CIPC_OK (0) or an error code; the message of the
 * last failure is available from cipc_gpu_last_error().  A context is used
 * from one host thread at a time and enqueues all device work on one stream.
 *
 * Reference interfaces each entry point replaces are cited as
 * path:line within the CPU-IPC project.
 */
#ifndef CIPC_GPU_H
#define CIPC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (the reference throws std::invalid_argument / std::runtime_error,
 * NewtonLinearSystem.cpp:30-36, PardisoSolver.cpp:175-179, IPCSolver.cpp:585-587). */
enum {
    CIPC_OK = 0,
    CIPC_ERR_INVALID_ARGUMENT = 1,
    CIPC_ERR_RUNTIME = 2,        /* non-finite values, iteration caps, line-search failure */
    CIPC_ERR_CUDA = 3,
    CIPC_ERR_NOT_CONVERGED = 4,  /* PCG iteration limit */
    CIPC_ERR_DEVICE_STATUS = 5   /* a kernel raised a status bit (stack, capacity, CCD cap) */
};

/* LinearSolverBackend (LinearSolverOptions.h:3-7) extended with the GPU PCG. */
enum {
    CIPC_LINEAR_CHOLMOD = 0,
    CIPC_LINEAR_PARDISO = 1,
    CIPC_LINEAR_EIGEN_CG = 2,
    CIPC_LINEAR_GPU_PCG = 3
};
enum { CIPC_PRECISION_FP64 = 0, CIPC_PRECISION_MIXED = 1 };
enum { CIPC_PRECOND_BLOCK_JACOBI = 0, CIPC_PRECOND_LEARNED = 1, CIPC_PRECOND_FSAI = 2 };
/* Prescribed motions of boundary vertices (twistingBoundaryDirection,
 * Simulator.cpp:24-46, with the angular rate as a parameter). */
enum { CIPC_MOTION_NONE = 0, CIPC_MOTION_TWIST_X = 1 };

/* LinearSolverOptions (LinearSolverOptions.h:9-19) plus precision and
 * preconditioner selection for the GPU backend. */
typedef struct {
    int backend;               /* must be CIPC_LINEAR_GPU_PCG */
    int precision;             /* CIPC_PRECISION_* */
    int preconditioner;        /* CIPC_PRECOND_* */
    double relativeTolerance;  /* default 1e-6 */
    int maximumIterations;     /* default 10000 */
} cipc_linear_options;

/* Scene description: the mesh3D fields the Newton pipeline reads
 * (SimulationMesh.h:37-129) and the parameters loadSettings/updateMaterial
 * derive (Simulator.cpp:128-263).  Optional arrays may be NULL, in which case
 * the library computes them exactly as FEMSimulator::buildModels does
 * (initMesh3D, prepareQuadraticBending, getSurface). */
typedef struct {
    int nv, nt, nf;
    const double* x;        /* 3*nv rest (= initial) positions */
    const double* vel;      /* 3*nv initial velocities or NULL */
    const int* tets;        /* 4*nt */
    const int* tris;        /* 3*nf cloth triangles */
    const int* btype;       /* nv: 0 free, 1 Dirichlet, >=2 external collider */
    const double* tetE;     /* nt per-tet Young's modulus or NULL */
    double density, cloth_density, thickness, E, nu, clothE, shearE, bendE, strainRate, friction;
    double dt, drag, newtonThr, relDhat;
    int use_barrier, apply_gravity, quasi_static;
    int quad_bending;       /* bending model: 1 quadratic (USE_QUADRATIC_BENDING), 2 dihedral-angle
                               hinges (the reference's build without it), 0 none */
    double bboxMin[3], bboxMax[3];
    int nsoft; const int* softIdx; double softW; int softMotion; double softRate;
    int ndir; const int* dirIdx; int dirMotion; double dirRate;
    /* optional precomputed surface (getSurface order) */
    int nsf, nsv, nse;
    const int* surfFaces;   /* 3*nsf */
    const int* surfVerts;   /* nsv */
    const int* surfEdges;   /* 2*nse */
} cipc_scene_desc;

/* IPCStepStats (IPCSolver.h:12-44) plus the PCG figures of the GPU backend. */
typedef struct {
    int frame, newtonIterations, kappaIterations, lineSearchBacktracks, energyBacktracks, intersectionBacktracks;
    int maximumEnergyBacktracksPerNewton, newtonStepsWithMoreThanTwoBacktracks;
    double stepMilliseconds, assemblyMilliseconds, linearSolveMilliseconds, ccdMilliseconds, lineSearchMilliseconds,
        postLineSearchMilliseconds;
    double collisions, kappa, minConstraintDistance2, acceptedStepSum, minimumAcceptedStep, maximumAcceptedStep;
    long long groundContacts, selfContacts, mollifiedContacts, matrixBlocks;
    long long pcgIterations;
    double pcgRelativeResidual;
} cipc_step_stats;

typedef struct cipc_gpu_context cipc_gpu_context;

/* Context life cycle: replaces FEMSimulator::buildModels' set-up of mesh3D,
 * SpatialHash and NewtonLinearSystem (Simulator.cpp:426-529,
 * IPCSolver.cpp:1157-1160).  Uploads topology and rest data once. */
int cipc_gpu_create(const cipc_scene_desc* scene, const cipc_linear_options* options, cipc_gpu_context** out);
void cipc_gpu_destroy(cipc_gpu_context* ctx);
const char* cipc_gpu_last_error(const cipc_gpu_context* ctx);
/* Message of the last cipc_gpu_create failure (no context exists then). */
const char* cipc_gpu_create_error(void);

/* One time step: solveIPCStep (IPCSolver.cpp:1079-1336) - kappa loop around
 * the barrier sub-problem Newton loop (IPCSolver.cpp:890-1064), all stages on
 * the GPU; fills the IPCStepStats fields. */
int cipc_gpu_step(cipc_gpu_context* ctx, cipc_step_stats* stats);

/* State access.  which: 0 positions x, 1 velocities, 2 previous positions
 * (V_prev), 3 inertial target, 4 rest positions; 3*nv doubles. */
int cipc_gpu_get_state(cipc_gpu_context* ctx, int which, double* out);
int cipc_gpu_set_state(cipc_gpu_context* ctx, int which, const double* in);
/* scalars: kappa, Hhat, Fhat, dTol, bboxDiag2, meanMass, avgEdge, lengthRate,
 * volumeRate, stretchS, shearS, plateRigidity, dt, newtonThr */
int cipc_gpu_get_scalars(cipc_gpu_context* ctx, double* out14);
int cipc_gpu_set_kappa(cipc_gpu_context* ctx, double kappa);
/* Segment-triangle test of the intersection check (isIntersected /
 * IglUtils::segTriIntersect, IPCSolver.cpp:476-542, ContactMechanics.h:47-71).
 * CIPC_INTERSECT_TOLERANT (default) also skips a segment whose two plane
 * distances are both within 1e-12 of zero relative to |n| times its reach
 * (near-coplanar through rounding on rotated meshes);
 * CIPC_INTERSECT_REFERENCE is the reference's exact rule (signs and
 * det == 0 only). */
enum { CIPC_INTERSECT_TOLERANT = 0, CIPC_INTERSECT_REFERENCE = 1 };
int cipc_gpu_set_intersection_rule(cipc_gpu_context* ctx, int rule);
/* Broad-phase backend (cipc_headless --broad-phase, the reference's
 * SpatialHash or LBVH, CollisionBroadPhase.cpp:11-763, LBVH.cpp:163-282):
 * both report the same candidate sets after the same exact box test; the
 * LBVH is the default. */
enum { CIPC_BROAD_PHASE_LBVH = 0, CIPC_BROAD_PHASE_SPATIAL_HASH = 1 };
int cipc_gpu_set_broad_phase(cipc_gpu_context* ctx, int backend);
/* counts: nv, nsf, nsv, nse, nbend, nt, nf, nnzb (static BSR blocks),
 * contact BSR blocks of the last assembly */
int cipc_gpu_get_counts(cipc_gpu_context* ctx, long long* out9);
int cipc_gpu_get_surface(cipc_gpu_context* ctx, int* faces, int* verts, int* edges);

/* Broad phase + active sets at the current positions:
 * SpatialHash::build + calculateActivateSet + Ground::calculateActivateSet
 * (CollisionBroadPhase.cpp:765-1092, IPCSolver.cpp:544-556).
 * counts: self active, mollified, partial-CCD pairs, ground contacts. */
int cipc_gpu_build_collision_sets(cipc_gpu_context* ctx, long long* out4);
/* Copies the sets in the reference's encoding (EncodedContact.h, 4 ints per
 * contact; Self_CCD_ActiveSet pairs; Environment_ActiveSet vertices). */
int cipc_gpu_get_active_sets(cipc_gpu_context* ctx, int* selfActive, int* selfEE, int* eeIe, int* ccdPairs, int* ground);
/* Friction::initialize (Friction.cpp:81-156) at the current state. */
int cipc_gpu_friction_init(cipc_gpu_context* ctx);

/* computeGradientAndHessian (IPCSolver.cpp:108-319) + assembly into the
 * Newton matrix (NewtonLinearSystem::assemble, NewtonLinearSystem.cpp:126-154).
 * grad: 3*nv.  Returns the collision count in *collisions if non-NULL. */
int cipc_gpu_assemble(cipc_gpu_context* ctx, double* grad, int* collisions);
/* Exports the last assembled matrix as a full symmetric scalar COO on free
 * vertices plus the mass/ground/soft diagonal: call with rows == NULL to get
 * the entry count. */
int cipc_gpu_export_matrix(cipc_gpu_context* ctx, long long* count, int* rows, int* cols, double* vals);
/* NewtonLinearSystem::solve (NewtonLinearSystem.h:22-28) on the last
 * assembled system: direction (3*nv) solves A p = g (g zeroed off free DOFs). */
int cipc_gpu_solve(cipc_gpu_context* ctx, double* direction, int* iterations, double* relResidual);
/* computeEnergy (IPCSolver.cpp:322-456) at the current state with the given kappa. */
int cipc_gpu_energy(cipc_gpu_context* ctx, double kappa, double* energy);
/* Feasible step bounds along dir: out[0] limitStepByGround (FeasibleStep.cpp:8-40),
 * out[1] Self_largestFeasibleStepSize (ContactMechanics.cpp:3704-3752) from
 * alpha_in, out[2] the CFL bound (IPCSolver.cpp:960-975), out[3]
 * Self_largestFeasibleStepSize_CCD (ContactMechanics.cpp:3754-3867) from alpha_in. */
int cipc_gpu_step_bounds(cipc_gpu_context* ctx, const double* dir, double alpha_in, double* out4);
/* isIntersected (IPCSolver.cpp:520-542) at the current positions; *result 0/1. */
int cipc_gpu_intersected(cipc_gpu_context* ctx, int* result);

/* Runs nsteps time steps (cipc_gpu_step each) with CUDA events recorded on
 * the context's stream before and after; *deviceMs is the elapsed device
 * time, *last the last step's statistics. */
int cipc_gpu_timed_steps(cipc_gpu_context* ctx, int nsteps, cipc_step_stats* last, double* deviceMs);
/* Kernel timing for measurement: kind selects one kernel family
 * (1 PCG SpMV, 2 tetrahedra, 3 cloth triangles, 4 BSR slot reduction,
 * 5 self-contact barrier, 6 active-set traversal, 7 full CCD, 8 persistent
 * PCG solve); its launches are bracketed by CUDA events on the context's
 * stream (up to `capacity` launches).  kind 0 disables.  _read returns the
 * number of timed launches and their summed device time. */
int cipc_gpu_profile(cipc_gpu_context* ctx, int kind, int capacity);
int cipc_gpu_profile_read(cipc_gpu_context* ctx, long long* launches, double* totalMs);
/* Kernel launches this library has issued since it was loaded (library
 * sorts/scans excluded). */
long long cipc_gpu_kernel_launches(void);

/* System dump at the NewtonLinearSystem::solve seam (NewtonLinearSystem.cpp:39,
 * after assembly): the last assembled Newton matrix in the device layout.
 * sizes[0] = static blocks, sizes[1] = contact blocks; call with rowPtr NULL
 * to get the sizes.  rowPtr nv+1, col and val (9 per block, row-major) for
 * the full symmetric static pattern; dynRowStart/dynRowEnd nv, dynCol and
 * dynVal for the contact pattern; diagExtra 9 per vertex (inertia, ground
 * and soft-target terms on the diagonal).  A = static + contact + diagExtra. */
int cipc_gpu_export_bsr(cipc_gpu_context* ctx, int* sizes, int* rowPtr, int* col, double* val, int* dynRowStart, int* dynRowEnd, int* dynCol,
                        double* dynVal, double* diagExtra);

/* Learned preconditioner (no counterpart in the reference; the closest is
 * the Eigen IncompleteCholesky option, NewtonLinearSystem.cpp:186-192).  A
 * 3-layer width-32 message-passing network over the matrix block graph
 * emits a lower-triangular factor G on the IC(0) pattern of the
 * block-Jacobi-scaled matrix; PCG applies M^-1 = S^T G^T G S.  Selected by
 * CIPC_PRECOND_LEARNED; block-Jacobi takes over when the true FP64 residual
 * rejects a learned solve.  CIPC_PRECOND_FSAI applies the exact
 * factorised sparse approximate inverse of the same pattern instead (the
 * optimum of the network's loss).  Weights are FP32 arrays of
 * cipc_gpu_precond_num_params() values. */
int cipc_gpu_precond_num_params(void);
int cipc_gpu_precond_set_weights(cipc_gpu_context* ctx, const float* weights, int n);
int cipc_gpu_precond_get_weights(cipc_gpu_context* ctx, float* weights, int n);
/* Loss (log Kaporin number of G Â G^T, trace by probes) on the last
 * assembled system and, when grad is not NULL, its gradient with respect to
 * the weights.  probeVectors: probes x 3*nv host floats, or NULL for the
 * device generator seeded by seed. */
int cipc_gpu_precond_loss(cipc_gpu_context* ctx, int probes, const float* probeVectors, unsigned long long seed, double* loss, float* grad);
/* `iterations` Adam steps (rate learningRate) on the last assembled system,
 * `probes` probe vectors per step; losses of the first and last step. */
int cipc_gpu_precond_train(cipc_gpu_context* ctx, int iterations, int probes, double learningRate, unsigned long long seed, double* lossFirst,
                           double* lossLast);
/* Hook at the linear-solve seam of every Newton iteration
 * (NewtonLinearSystem::solve, NewtonLinearSystem.cpp:39; no counterpart in
 * the reference otherwise).  With iterations > 0 the network takes that many
 * Adam steps on each assembled Newton system before it is solved (the
 * systems the simulator produces train the network as they arise; 0 turns
 * it off). */
int cipc_gpu_set_online_training(cipc_gpu_context* ctx, int iterations, int probes, double learningRate, unsigned long long seed);
/* With a directory, every Newton system is written there before its solve,
 * one file per system (system_<frame>_<newton>.bin: magic "CIPCSYS1", int32
 * nv, nnzb, ndyn, value bytes, frame, Newton index; static BSR row pointers,
 * columns, values; contact BSR row starts, ends, columns, values; FP64
 * diagonal extras, right-hand side, positions; int32 boundary types).  NULL
 * or "" turns it off. */
int cipc_gpu_set_system_dump(cipc_gpu_context* ctx, const char* directory);
/* Times the host has waited for the context's stream since creation (the
 * Newton driver's host round trips; no counterpart in the reference). */
int cipc_gpu_host_syncs(cipc_gpu_context* ctx, long long* count);
/* Newton systems the hook has trained on or written since creation. */
int cipc_gpu_hook_systems(cipc_gpu_context* ctx, long long* count);

/* Builds the factor of preconditioner `which` (CIPC_PRECOND_LEARNED: the
 * network forward; CIPC_PRECOND_FSAI: the exact factorised sparse
 * approximate inverse of the same pattern) on the last assembled system and
 * copies it out slot-aligned with cipc_gpu_export_bsr: 9 floats per static
 * block (lower slots G_ij, upper slots G_ji^T, diagonal slots G_ii) and per
 * contact block.  Either pointer may be NULL. */
int cipc_gpu_precond_factor(cipc_gpu_context* ctx, int which, float* gStatic, float* gContact);
/* out[0] block-Jacobi fallbacks taken, out[1] Adam steps since the weights
 * were set, out[2] iterations of the last PCG launch. */
int cipc_gpu_precond_stats(cipc_gpu_context* ctx, long long* out3);

/* Additive CCD (AdditiveCCD.cpp:221-329, the per-pair time of impact of
 * Self_largestFeasibleStepSize, ContactMechanics.cpp:3704-3752) on n
 * independent candidate pairs, host arrays: kind[k] 0 point-triangle
 * (positions point, t0, t1, t2), 1 edge-edge (a0, a1, b0, b1); 12 positions
 * and 12 displacements per pair; eta = 1 - slackness (the reference uses 0.2).
 * toi[k] in [0, 1] is the conservative step along the displacements. */
int cipc_gpu_accd(int n, const int* kind, const double* positions, const double* displacements, double eta, double* toi, char* err,
                  int errlen);

/* Stand-alone GPU PCG on a caller-given matrix (full symmetric 3x3-block CSR,
 * FP64 values, 9 per block row-major) - the backend switch of
 * NewtonLinearSystem::solve (NewtonLinearSystem.cpp:41-53) without a scene.
 * Row pointers must be non-negative and non-decreasing, column indices in
 * [0, nv), and every block row must hold exactly one diagonal block;
 * otherwise CIPC_ERR_INVALID_ARGUMENT. */
int cipc_gpu_pcg_bsr(int nv, const int* rowPtr, const int* colIdx, const double* vals, const double* rhs, double* sol,
                     const cipc_linear_options* options, int* iterations, double* relResidual, char* err, int errlen);

/* Allocation-free variant of cipc_gpu_pcg_bsr (no counterpart in the
 * reference).  For callers that cannot or must not allocate device memory -
 * e.g. a host whose device memory belongs to its own allocator, or a loop
 * that must not pay cudaMalloc latency.  All array arguments are DEVICE
 * pointers the caller owns (rowPtr nv+1, colIdx and vals as in
 * cipc_gpu_pcg_bsr, rhs and sol 3*nv); the function allocates nothing and
 * keeps its scratch vectors in a fixed array inside the library, sized for at
 * most CIPC_NOALLOC_MAX_ROWS block rows (8,008,064 bytes, 7.6 MiB, held on
 * every GPU that loads the library until the process exits); larger nv
 * returns CIPC_ERR_INVALID_ARGUMENT.  The matrix structure is checked on the
 * device with the rules cipc_gpu_pcg_bsr applies on the host (same error
 * code) before any block is read.  The first call on a device resolves that array's
 * device address with the device current, so make the first call on each
 * device outside any stream capture.  Every call shares the array: calls
 * that overlap on the GPU (other streams or threads) race and must be
 * serialised.  stream is a cudaStream_t (NULL = legacy default stream). */
#define CIPC_NOALLOC_MAX_ROWS 32768
int cipc_gpu_pcg_bsr_noalloc(int nv, const int* rowPtr, const int* colIdx, const double* vals, const double* rhs, double* sol,
                             double relativeTolerance, int maximumIterations, void* stream, int* iterations, double* relResidual);

#ifdef __cplusplus
}
#endif

#endif /* CIPC_GPU_H */
