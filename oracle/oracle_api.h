/* Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * liboracle.so; the shipped library never links it.
 *
 * C ABI of the oracle, used through ctypes by the test-suite. */
#ifndef CIPC_ORACLE_API_H
#define CIPC_ORACLE_API_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nv, nt, nf;
    const double* x;      /* 3*nv rest (= initial) positions */
    const double* vel;    /* 3*nv initial velocities, may be NULL */
    const int* tets;      /* 4*nt */
    const int* tris;      /* 3*nf cloth triangles */
    const int* btype;     /* nv boundary codes: 0 free, 1 Dirichlet, >=2 external collider */
    const double* tetE;   /* nt per-tet Young's modulus, may be NULL (uniform E) */
    double density, cloth_density, thickness, E, nu, clothE, shearE, bendE, strainRate, friction;
    double dt, drag, newtonThr, relDhat;
    int use_barrier, apply_gravity, quasi_static, quad_bending;  /* bending model: 0 none, 1 quadratic, 2 hinge */
    double bboxMin[3], bboxMax[3];
    int nsoft; const int* softIdx; double softW; int softMotion; double softRate;
    int ndir; const int* dirIdx; int dirMotion; double dirRate;
    int linear;           /* 0 envelope Cholesky, 1 block-Jacobi PCG, 2 multifrontal Cholesky */
    double pcgRelTol;
    int threads;
} cipc_oracle_scene;

typedef struct {
    int frame, newton, kappaIters, backtracks, energyBacktracks, intersectionBacktracks;
    int maxEnergyBacktracksPerNewton, newtonOverTwo;
    double collisions, kappa, minDist2, acceptedStepSum, minStep, maxStep;
    long long groundContacts, selfContacts, mollifiedContacts, matrixNnz, pcgIterations, linearSolves;
} cipc_oracle_stats;

void* cipc_oracle_create(const cipc_oracle_scene* s, char* err, int errlen);
void cipc_oracle_destroy(void* h);
int cipc_oracle_step(void* h, cipc_oracle_stats* st, char* err, int errlen);
/* counts: nv, nsurfFaces, nsurfVerts, nsurfEdges, nbend, ntets, ntris */
void cipc_oracle_info(void* h, long long* counts);
/* scalars: kappa, Hhat, Fhat, dTol, bboxDiag2, meanMass, avgEdge, lengthRate, volumeRate,
 * stretchS, shearS, plateRigidity, dt, newtonThr */
void cipc_oracle_scalars(void* h, double* out);
void cipc_oracle_set_kappa(void* h, double kappa);
/* segment-triangle test of the intersection check: 0 skips near-coplanar
 * segments within a 1e-12 relative tolerance (default), 1 is the
 * reference's exact rule (ContactMechanics.h:47-71) */
void cipc_oracle_set_intersection_rule(void* h, int rule);
/* which: 0 x, 1 vel, 2 vprev, 3 xtilde, 4 rest, 5 mass(nv) */
void cipc_oracle_get(void* h, int which, double* out);
void cipc_oracle_set(void* h, int which, const double* in);
void cipc_oracle_surface(void* h, int* faces, int* verts, int* edges);
/* rest data: DmInv (9*nt row-major), vol (nt), DmInv2 (4*nf), area (nf), bend verts (4*nb), bend Q (16*nb) */
void cipc_oracle_rest(void* h, double* dminv, double* vol, double* dminv2, double* area, int* bendv, double* bendq);
/* rebuild broad phase + active sets at the current positions; returns counts
 * [nSelfActive, nSelfEE, nCCD, nGround] */
void cipc_oracle_collision_sets(void* h, long long* counts);
void cipc_oracle_get_sets(void* h, int* selfActive, int* selfEE, int* eeIe, int* ccd, int* ground);
void cipc_oracle_friction_init(void* h);
/* gradient (3*nv) and lower free-only scalar CSR of the Newton matrix; call
 * with rowptr == NULL to get nnz first (returned) */
long long cipc_oracle_system(void* h, double* grad, int* rowptr, int* col, double* val, double* rhs);
double cipc_oracle_energy(void* h, double kappa);
/* feasible-step bounds along dir (3*nv): out[0] ground, out[1] partial CCD,
 * out[2] CFL, out[3] full CCD (entry step alpha_in) */
void cipc_oracle_step_bounds(void* h, const double* dir, double alpha_in, double* out);
int cipc_oracle_intersected(void* h);
double cipc_oracle_pt_ccd(const double* p12, const double* d12, double eta);
double cipc_oracle_ee_ccd(const double* p12, const double* d12, double eta);
/* element-level kernels for unit parity: snh (F 9 row-major, u, r) -> P 9, H 81 */
void cipc_oracle_snh(const double* F, double u, double r, double* P, double* H, double* psi);
/* distance kind 0 PP,1 PE,2 PT,3 EE,4 crossSqNorm: value, gradient, Hessian */
double cipc_oracle_distance(int kind, const double* pts, double* g, double* H);
/* one hinge bending element (HingeBending.cpp:76-106 + makePD) */
double cipc_oracle_hinge(const double* x12, const double* rest12, double k, double* g, double* H);
/* linear solve of a given lower CSR system (n scalar rows): method 0 envelope Cholesky, 1 block-Jacobi
   PCG, 2 multifrontal Cholesky on `threads` threads (xyz: vertex positions for its ordering, or null) */
int cipc_oracle_linear_solve(int nv, const int* rowptr, const int* col, const double* val, const double* rhs,
                             double* sol, int method, double tol, int maxIter, int* iters, double* relres, int threads,
                             const double* xyz);
double cipc_oracle_total_energy(void* h);

#ifdef __cplusplus
}
#endif
#endif
