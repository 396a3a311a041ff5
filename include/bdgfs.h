/*
 * bdgfs: B200-native DGFS hot path (fast-spectral Boltzmann collision
 * operator and flux-reconstruction advection) behind a plain C ABI.
 *
 * Every entry point takes device pointers, sizes and a CUDA stream passed
 * as void*, returns an int32 status (0 = ok, negative = error), never
 * allocates device memory and never synchronises the host, so a sequence
 * of calls can be captured in a CUDA graph.  Buffers and scratch are owned
 * by the caller.
 */
#ifndef BDGFS_H
#define BDGFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BDGFS_OK 0
#define BDGFS_EINVAL (-1)       /* bad argument / size / layout             */
#define BDGFS_ECUDA (-2)        /* a CUDA runtime call failed               */
#define BDGFS_EUNSUPPORTED (-3) /* grid size / precision not compiled in    */
#define BDGFS_ETIMEOUT (-4)     /* a bounded device wait gave up            */
#define BDGFS_ESCRATCH (-5)     /* caller-provided scratch is too small     */

/* ------------------------------------------------------------------------
 * Fast-spectral VHS collision operator Q(f, f)
 * ---------------------------------------------------------------------- */

/* One velocity grid (Nv^3 cube) with its precomputed tables.  All table
 * pointers are device pointers; "real" means float when fp64 == 0 and
 * double when fp64 == 1, "complex" the matching (re, im) pair. */
typedef struct bdgfs_vhs_grid {
    int32_t Nv;          /* points per axis: 8, 12, 16, 24 or 32            */
    int32_t Nrho;        /* radial Gauss-Jacobi points                      */
    int32_t M;           /* half-sphere directions                          */
    int32_t fp64;        /* 0: FP32 state/tables, 1: FP64                   */
    int32_t tile;        /* kernel variant (threads per CTA), 0 = default;
                            see bdgfs_vhs_tiles                             */
    int32_t pad_;
    double prefac;       /* VHS prefactor                                   */
    double cw;           /* velocity cell volume (2L/Nv)^3                  */
    const void* phase;   /* complex [Nrho][M][3][Nv]:
                            exp(i*(pi/L)*(qz_p/2)*s_{q,a}*l0[k])            */
    const void* gw;      /* real [Nrho][Nv][Nv/2+1][Nv], index [p][kz][kx][ky]:
                            (2*qw_p*sw/Nv^3) * bb1_p(k)                     */
    const void* bb2;     /* real [Nv][Nv][Nv], index [kz][kx][ky]            */
    const double* c0;    /* [Nv] cell-centre velocities                     */
    const double* ginv;  /* [5][5] inverse Gram matrix of {1,cx,cy,cz,|c|^2} */
} bdgfs_vhs_grid;

/* A batch of distributions living on one grid. */
typedef struct bdgfs_vhs_batch {
    int32_t grid;        /* index into the grids array                      */
    int32_t pad_;
    int64_t ndof;        /* number of distributions                         */
    const void* f;       /* real [ndof][Nv^3], velocity index (x*Nv+y)*Nv+z  */
    void* Q;             /* real [ndof][Nv^3]                               */
    double* moments;     /* optional [ndof][10]: C.Q before (0..4) and after
                            (5..9) the projection, in FP64, C = cw*{1,c,|c|^2} */
    const int32_t* index;  /* optional: distribution i is f[index[i]] (and
                              Q/moments at the same position)              */
    const int64_t* count;  /* optional device count of distributions to
                              process (<= ndof), read by the kernel          */
} bdgfs_vhs_batch;

/* Number of kernel variants compiled for this grid set (tile values
 * 0..n-1, 0 being the default); threads[i] receives each variant's CTA size
 * when threads is not NULL (capacity n).  Returns 0 for an unsupported set. */
int32_t bdgfs_vhs_tiles(const bdgfs_vhs_grid* grids, int32_t ngrids,
                        int32_t* threads, int32_t capacity);

/* Bytes of device scratch bdgfs_vhs_collide needs for nctas resident CTAs
 * (nctas <= 0: one per SM of the current device). */
size_t bdgfs_vhs_scratch_bytes(const bdgfs_vhs_grid* grids, int32_t ngrids,
                               int32_t nctas);

#define BDGFS_PROJECT 1  /* FP64 minimal-norm conservation projection      */
#define BDGFS_EXACT 2    /* also carry the second-order Nyquist-plane term  */

/* Q for every distribution of every batch, in one persistent launch.
 * flags & BDGFS_PROJECT applies the FP64 minimal-norm conservation
 * projection Q <- Q - phi^T G^{-1} (phi Q); flags & BDGFS_EXACT runs a
 * second transform per (p, q) so that the result equals the reference's
 * complex-square form to rounding (2x the work).  work_counter: one device uint64 that this
 * call resets (stream-ordered) and uses to hand out distributions.
 * Replaces DGFSVHSGLLScatteringModel.fs (frfs/solvers/dgfs/scattering.py:227)
 * called for every (elem, upt) by DGFSSystem.collide
 * (frfs/solvers/dgfs/system.py:199-218). */
int32_t bdgfs_vhs_collide(const bdgfs_vhs_grid* grids, int32_t ngrids,
                          const bdgfs_vhs_batch* batches, int32_t nbatch,
                          int32_t flags, void* scratch, size_t scratch_bytes,
                          uint64_t* work_counter, void* stream);

/* Same as bdgfs_vhs_collide, for callers that cannot allocate device memory
 * (their device memory belongs to another allocator or a fixed arena, or they
 * must not allocate once running): scratch and work counter come from one
 * file-scope device array of 16 MiB held by every GPU that loads the library.
 * No counterpart in the reference.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  Returns BDGFS_ESCRATCH if one CTA's scratch for these
 * grids exceeds the array; calls that overlap on the GPU race on the array. */
int32_t bdgfs_vhs_collide_static(const bdgfs_vhs_grid* grids, int32_t ngrids,
                                 const bdgfs_vhs_batch* batches, int32_t nbatch,
                                 int32_t flags, void* stream);

/* Bounded-wait probe: one thread waits on an mbarrier with the polling
 * loop the tensor-core kernels use for their waits, at most `limit` polls.
 * arrive = 0: nothing arrives, the wait runs out and *status (device) is set
 * to BDGFS_ETIMEOUT; arrive = 1: the barrier completes and *status is
 * BDGFS_OK.  Tests the timeout path without a device fault.  No counterpart
 * in the reference. */
int32_t bdgfs_wait_probe(uint32_t limit, int32_t arrive, int32_t* status, void* stream);

/* Measured FP32 FMA throughput probe: runs iters dependent-free FMA chains
 * per thread on nblocks x 256 threads and writes a checksum to out[0]. */
int32_t bdgfs_fma_probe(float* out, int32_t nblocks, int32_t iters,
                        void* stream);

/* ------------------------------------------------------------------------
 * Flux-reconstruction advection (all Nv^3 velocities per launch)
 * ---------------------------------------------------------------------- */

/* One element type.  State u[e][upt][v], face values uf[e][fpt][v],
 * v = (x*Nv + y)*Nv + z.  "real" is float (fp64 == 0) or double. */
typedef struct bdgfs_fr_eles {
    int32_t ndims;       /* 2 (quad) or 3 (hex)                            */
    int32_t nupts;       /* solution points per element                    */
    int32_t nfpts;       /* flux points per element                        */
    int32_t neles;
    int64_t nv;          /* Nv^3                                           */
    int32_t Nv;
    int32_t fp64;
    const void* m0;      /* real [nfpts][nupts]        M0                  */
    const void* dcorr;   /* real [nupts][ndims*nupts]  M1 - M3*M2          */
    const void* m3;      /* real [nupts][nfpts]        M3                  */
    const void* smats;   /* real [neles][nupts][ndims][ndims]              */
    const void* rcpdjac; /* real [neles][nupts]                            */
    const void* pnorm;   /* real [neles][nfpts][ndims] unit outward normal */
    const void* magn;    /* real [neles][nfpts]        |J J^-T n|          */
    const int32_t* nbr;  /* [neles][nfpts]: e'*nfpts+f' of the neighbour
                            face point, or -1 - (wall face-point index)     */
    const void* c0;      /* real [Nv] cell-centre velocities               */
    int32_t engine;      /* bdgfs_fr_rhs: 0 = CUDA cores (default);
                            1 = tensor cores (tcgen05 kind::tf32, 3xTF32
                            products keep FP32 accuracy; FP32 state and the
                            tabulated shapes only, else CUDA cores)        */
    int32_t pad_;
} bdgfs_fr_eles;

/* Boundary face points (walls, inlets, outlets, symmetry planes).  The
 * ghost state u_R of a boundary face point, by the kind of its boundary
 * condition (frfs/solvers/dgfs/kernels/bcs/<type>.mako):
 *   BDGFS_BC_DIFFUSE   u_R = f_w (-bc0/bc1) where (c - U).n < 0, else u_L
 *                      (dgfs-wall-diffuse, dgfs-wall-diffuse-cyl)
 *   BDGFS_BC_INLET     u_R = f_w where (c - U).n < 0, else u_L (dgfs-inlet;
 *                      dgfs-inlet-normalshock with U = 0; dgfs-vanish with
 *                      U = 0 and f_w = 0)
 *   BDGFS_BC_OUTLET    u_R = u_L (dgfs-outlet)
 *   BDGFS_BC_SPECULAR_X/Y/Z  u_R(c) = u_L(c mirrored in the plane normal to
 *                      that axis) (dgfs-wall-specular on axis-aligned walls;
 *                      the velocity grid is symmetric about 0)
 * with U = uwall[bid] and f_w = fw[bid]. */
#define BDGFS_BC_DIFFUSE 0
#define BDGFS_BC_INLET 1
#define BDGFS_BC_OUTLET 2
#define BDGFS_BC_SPECULAR_X 3
#define BDGFS_BC_SPECULAR_Y 4
#define BDGFS_BC_SPECULAR_Z 5
typedef struct bdgfs_fr_walls {
    int32_t nwall;       /* boundary face points                           */
    int32_t nbc;         /* boundary conditions                            */
    const int32_t* fpt;  /* [nwall][2] (element, flux point)               */
    const int32_t* bcid; /* [nwall] boundary condition of each point       */
    const void* uwall;   /* real [nbc][3] wall / inlet velocity U          */
    const void* fw;      /* real [nbc][nv] wall / inlet Maxwellian f_w     */
    void* bcv;           /* real [nwall][2] bc0, bc1 (written by bc_update;
                            diffuse walls only)                            */
    double cw;           /* velocity cell volume                           */
    const int32_t* kind; /* [nbc] BDGFS_BC_* of each condition (device);
                            NULL: every condition is a diffuse wall        */
    int32_t kinds_used;  /* bit (1 << kind) set for every kind in kind[]   */
    int32_t pad_;
} bdgfs_fr_walls;

/* uf = M0 u.  Replaces kernels['eles', 'disu'] (solvers/dgfs/elements.py:56-59). */
int32_t bdgfs_fr_disu(const bdgfs_fr_eles* el, const void* u, void* uf,
                      void* stream);

/* out = minv u per element, minv real [nupts][nupts] in el's precision: the
 * inverse mass matrix M12 (frfs/shapes.py:163-166).  out must not alias u.
 * Replaces kernels['eles', 'invmass'] (solvers/dgfs/elements.py:161-164),
 * which system.invmass (solvers/dgfs/system.py:221-231) launches. */
int32_t bdgfs_fr_invmass(const bdgfs_fr_eles* el, const void* minv,
                         const void* u, void* out, void* stream);

/* bc0/bc1 of every diffuse-wall face point from uf.  Replaces
 * kernels['bcint', 'update_bc'] (solvers/dgfs/inters.py:221-229,
 * kernels/bccupdate.mako, kernels/bcs/dgfs-wall-diffuse-update.mako),
 * summed over all velocities in one pass. */
int32_t bdgfs_fr_bc_update(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                           const void* uf, void* stream);

/* out = a*u + b*L(u) + c1*x1 + c2*x2 with L(u) = -div F (FR, upwind
 * interfaces, diffuse walls).  x1/x2 may be NULL; out may alias u, x1 or
 * x2.  Replaces kernels ('eles','tdisf'), ('eles','tdivtpcorf'),
 * ('iint','comm_flux'), ('bcint','comm_flux'), ('eles','tdivtconf'),
 * ('eles','negdivconf') of DGFSSystem.rhs (solvers/dgfs/system.py:140-177)
 * and the stepper's axnpby (backends/cuda/blasext.py:14-43). */
int32_t bdgfs_fr_rhs(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                     const void* u, const void* uf, void* out, double a,
                     double b, const void* x1, double c1, const void* x2,
                     double c2, void* stream);

/* Face points on solution points (every row of M0 a unit vector, as with
 * GLL points): fsel[f] (int32 [nfpts], device) is the solution point of
 * flux point f, and the face values are read from u itself, so no uf array
 * and no bdgfs_fr_disu are needed.  bdgfs_fr_rhs_gather computes what
 * bdgfs_fr_disu + bdgfs_fr_rhs compute (bitwise); nbr entries e'*nfpts + f'
 * read u[e'][fsel[f']] (entries past the state, e.g. halo rows of a
 * partitioned mesh, are not supported and read as the element's own face
 * value).  out must not alias u (BDGFS_EINVAL): other
 * elements read u's face rows during the launch.  bdgfs_fr_bc_update_gather
 * is bdgfs_fr_disu + bdgfs_fr_bc_update. */
int32_t bdgfs_fr_rhs_gather(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                            const int32_t* fsel, const void* u, void* out,
                            double a, double b, const void* x1, double c1,
                            const void* x2, double c2, void* stream);
int32_t bdgfs_fr_bc_update_gather(const bdgfs_fr_eles* el,
                                  const bdgfs_fr_walls* wl,
                                  const int32_t* fsel, const void* u,
                                  void* stream);

/* Tensor-product points (nupts = p^ndims, point index fastest in the first
 * reference coordinate) with flux points on solution points: the residual
 * factored as R = M1 F~ + M3 (F^n - M2 F~) instead of the dense
 * (M1 - M3 M2) F~ + M3 F^n of the shape's operators. */
typedef struct bdgfs_fr_tensor {
    const int32_t* fsel;  /* [nfpts] solution point of flux point f (M0's 1)  */
    const int32_t* fdim;  /* [nfpts] reference direction d of M2's only
                             nonzero in row f, at column d*nupts + fsel[f]   */
    const void* fsgn;     /* real [nfpts] that nonzero                       */
    const void* m1line;   /* real [ndims][nupts][4]: M1 on the d-line through
                             point j: M1[j + (t - j_d) p^d][d*nupts + j] for
                             t < p (j_d the d-th coordinate index of j), 0
                             for p <= t < 4; every other entry of M1 is 0    */
    int32_t p;            /* points per line, 2..4                           */
    int32_t pad_;
} bdgfs_fr_tensor;

/* bdgfs_fr_rhs (uf = the face values of bdgfs_fr_disu) or, with uf NULL,
 * bdgfs_fr_rhs_gather (out must not alias u then), with the factored
 * residual: equal to rounding, and bitwise the same with or without uf. */
int32_t bdgfs_fr_rhs_tensor(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                            const bdgfs_fr_tensor* tp, const void* u,
                            const void* uf, void* out, double a, double b,
                            const void* x1, double c1, const void* x2,
                            double c2, void* stream);

/* FP64 raw velocity moments of ndof distributions, out[ndof][13]:
 * cw*sum{f, c f (3), c_i c_j f (xx xy xz yy yz zz), |c|^2 c f (3)}.
 * Feeds the macroscopic fields of plugins/dgfsmomwriterstd.py:14-313. */
int32_t bdgfs_moments(const void* f, int64_t ndof, int32_t Nv, int32_t fp64,
                      const double* c0, double cw, double* out, void* stream);

/* out2[0] = sum (a-b)^2, out2[1] = sum b^2 in FP64 (residual norm of
 * plugins/dgfsresidualstd.py:34-80). */
int32_t bdgfs_residual(const void* a, const void* b, int64_t n, int32_t fp64,
                       double* out2, void* stream);

/* *status |= 1 if any of the n values is NaN or Inf (plugins/nancheck.py). */
int32_t bdgfs_status_check(const void* a, int64_t n, int32_t fp64,
                           int32_t* status, void* stream);

/* ------------------------------------------------------------------------
 * GEMMs of the learned collision-operator surrogate (no counterpart in the
 * reference, whose collision operator is spectral only)
 * ---------------------------------------------------------------------- */

/* C[m][n] = alpha * sum_k A(m,k) B(n,k) [+ beta*C] [+ bias[n]] -> act,
 * A(m,k) = A[m*sam + k*sak], B(n,k) = B[n*sbn + k*sbk].
 * engine 0: tcgen05 tensor cores, bf16 operands (float sources are rounded
 *           to bf16), FP32 accumulation, beta must be 0.  bf16 A and B with
 *           unit K stride, K, sam, sbn multiples of 8, 16-byte aligned and
 *           no arow run on the persistent TMA-fed engine (128x256 tiles);
 *           everything else on the general loader (128x128 tiles);
 * engine 1: FP32 CUDA cores (float sources only, no bias/act);
 * engine 2: the general tcgen05 loader only (same results as engine 0 up
 *           to FP32 summation order).
 * act 0: none; 1: GELU (erf form); 2: multiply by GELU'(zin[m][n]).
 * zout (optional, float, leading dim ldz) receives the pre-activation. */
typedef struct bdgfs_gemm_args {
    int64_t M, N, K;
    const void* A;
    int64_t sam, sak;
    const void* B;
    int64_t sbn, sbk;
    int32_t a_bf16, b_bf16;
    float alpha, beta;
    const void* bias;    /* float [N] or NULL                            */
    int32_t act;
    int32_t engine;
    void* cf32;          /* float output or NULL                         */
    void* cbf16;         /* bf16 output or NULL                          */
    int64_t ldc;
    void* zout;          /* float pre-activation output or NULL          */
    const void* zin;     /* float pre-activation input (act == 2)        */
    int64_t ldz;
    int32_t* status;     /* receives BDGFS_ETIMEOUT if a wait expired    */
    int32_t pad_;
    const int32_t* arow; /* optional: row m of A is row arow[m] (gather) */
    const int32_t* crow; /* optional: row m of C/zout is crow[m] (scatter) */
    const float* row_scale;   /* optional: acc of row m scaled by row_scale[m] */
    const int64_t* mcount;    /* optional device row count (<= M)        */
} bdgfs_gemm_args;

int32_t bdgfs_gemm(const bdgfs_gemm_args* args, void* stream);

/* out[n] = sum_m X[m][n] (bias gradients). */
int32_t bdgfs_colsum(const float* X, int64_t M, int64_t N, float* out,
                     void* stream);

/* Mean per-row relative squared error of y against t and its gradient dy
 * (loss of the surrogate's training). */
int32_t bdgfs_relmse(const float* y, const float* t, int64_t M, int64_t N,
                     float delta, float* dy, double* loss, void* stream);

/* AdamW step on FP32 master weights p (n values) with moments m1, m2;
 * writes a bf16 copy to p_bf16 when not NULL.  step counts from 1. */
int32_t bdgfs_adamw(float* p, const float* grad, float* m1, float* m2,
                    void* p_bf16, int64_t n, float lr, float beta1,
                    float beta2, float eps, float weight_decay, int64_t step,
                    void* stream);

/* ------------------------------------------------------------------------
 * Surrogate/spectral hybrid collision step (no counterpart in the reference)
 * ---------------------------------------------------------------------- */
typedef struct bdgfs_hybrid_args {
    int64_t ndof;            /* distributions of the state (rows)          */
    int32_t Nv;              /* 1..64                                      */
    int32_t fp64;
    const double* c0;        /* [Nv] cell-centre velocities                */
    const double* ginv;      /* [5][5] inverse Gram matrix of {1,c,|c|^2}  */
    double cw;
    float threshold;         /* Maxwellian deviation below which the
                                surrogate is used                          */
    float recheck;           /* fraction of surrogate cells re-checked     */
    uint64_t seed;           /* re-check sampling seed (e.g. step number)  */
    int64_t* counts;         /* [3] device: surrogate, spectral (incl.
                                re-checks), re-checked; [4] with fb_idx:
                                + fallback                                 */
    int32_t* sur_idx;        /* [ndof] surrogate cells                     */
    float* sur_inv_rho;      /* [ndof] 1/rho of each surrogate row         */
    float* sur_rho2;         /* [ndof] rho^2 of each surrogate row         */
    int32_t* spec_idx;       /* [ndof] spectral cells                      */
    uint8_t* flag;           /* [ndof] 0 spectral, 1 surrogate, 2 re-checked */
    float* eps;              /* optional [ndof] indicator values           */
    double* recheck_err;     /* optional [2]: sum |Qs-Qspec|^2, sum |Qspec|^2 */
    uint64_t* seed_dev;      /* optional device step counter: used instead of
                                seed, advanced by bdgfs_hybrid_scatter      */
    void* dev_rows;          /* optional bf16 [ndof][Nv^3]: for surrogate row p,
                                d / |d|_2 with d = f/rho - M[f]/rho (the
                                deviation from the local Maxwellian at unit
                                density; zero when d = 0)                   */
    void* feat;              /* optional bf16 rows with stride feat_ld: row p
                                gets (u_x, u_y, u_z, T - 1) at columns 0..3 */
    int64_t feat_ld;
    float* sur_s;            /* optional [ndof]: |d|_2 of surrogate row p   */
    int32_t* fb_idx;         /* optional [ndof]: the scatter lists here the
                                surrogate cells whose row is not finite
                                (NaN / Inf) and writes nothing for them;
                                counts[3] their number -- the caller runs
                                the spectral operator on that list         */
    float* sur_uT;           /* optional [ndof][4]: (u_x, u_y, u_z, T) of
                                surrogate row p (FP32)                      */
    int32_t center;          /* nonzero (needs sur_uT and dev_rows): the
                                surrogate works at zero drift --
                                bdgfs_hybrid_classify writes the deviation
                                rows re-centred at zero velocity and the
                                features (0, 0, 0, T - 1); the scatter
                                entries move each compact row of Qc back to
                                its cell's drift first (FP32 rows: fused with
                                the projection, Qc unchanged; otherwise Qc
                                is shifted in place)                        */
    int32_t pad2_;
} bdgfs_hybrid_args;

/* Indicator eps = |f - M[f]| / |f| per distribution and device-side lists. */
int32_t bdgfs_hybrid_classify(const bdgfs_hybrid_args* h, const void* f,
                              void* stream);
/* FP64 conservation projection of the first counts[0] compact rows of Qc. */
int32_t bdgfs_hybrid_project(const bdgfs_hybrid_args* h, void* Qc,
                             void* stream);
/* Compact surrogate rows -> Q[sur_idx[m]], except re-checked cells (kept
 * spectral; their surrogate error is accumulated in recheck_err). */
int32_t bdgfs_hybrid_scatter(const bdgfs_hybrid_args* h, const void* Qc,
                             void* Q, void* stream);
/* bdgfs_hybrid_project and bdgfs_hybrid_scatter in one pass (Qc is read,
 * projected on the fly and written to Q; Qc itself is left unchanged). */
int32_t bdgfs_hybrid_project_scatter(const bdgfs_hybrid_args* h,
                                     const void* Qc, void* Q, void* stream);
/* bdgfs_hybrid_heads with each value split into bf16 hi and lo parts,
 * written as [hi | hi | lo] column blocks of width nheads*k (ldo >=
 * 3*nheads*k): against an output basis stored as [B_hi | B_lo | B_hi], one
 * bf16 GEMM reconstructs Q to about FP32 accuracy. */
int32_t bdgfs_hybrid_heads_split(const bdgfs_hybrid_args* h, const float* Y, int64_t ldy,
                                 int64_t k, int32_t nheads, void* out, int64_t ldo,
                                 void* stream);
/* Spectral velocity shift of the first counts[0] compact rows: row p of out
 * is row p of in evaluated at the velocities c + sign * u_p, u_p =
 * sur_uT[p][0..2], by trigonometric interpolation on the periodic Nv^3 grid
 * of spacing c0[1] - c0[0] (one circulant pass along each axis; exact for
 * band-limited rows, its own inverse with the opposite sign up to the
 * Nyquist terms).  sign = +1 centres a row at zero velocity, -1 moves it
 * back.  in / out: bf16 (flag 1) or the state's real type, [rows][Nv^3];
 * they may be the same array.  Nv in {8, 12, 16, 24, 32}.  No counterpart
 * in the reference (the surrogate works on rows centred at zero velocity,
 * where the collision operator's dependence on the drift is removed
 * exactly). */
int32_t bdgfs_hybrid_shift(const bdgfs_hybrid_args* h, const void* in, int32_t in_bf16,
                           void* out, int32_t out_bf16, float sign, void* stream);
/* Features of the first counts[0] rows of the bf16 network input xc
 * (leading dimension ld) from its deviation modes x = columns [x0, x0+k):
 * columns [x1, x1+k) <- (T-1) x and [x1+k, x1+2k) <- (T-1)^2 x (T =
 * sur_uT[p][3]; the linearised operator's temperature dependence), and the
 * k2 (k2+1)/2 products x_i x_j, i <= j < k2, row-major over the upper
 * triangle, at columns [xq, ...) (the quadratic term of the collision
 * operator in the deviation; k2 <= 64, 0 for none). */
int32_t bdgfs_hybrid_tfeatures(const bdgfs_hybrid_args* h, void* xc, int64_t ld, int64_t x0,
                               int64_t x1, int64_t k, int32_t k2, int64_t xq, void* stream);
/* Scale the network's output heads of the first counts[0] rows:
 * out[m][i*k + j] = sur_s[m]^i * Y[m][i*k + j], i < nheads, j < k
 * (Y float, leading dimension ldy; out bf16, leading dimension ldo). */
int32_t bdgfs_hybrid_heads(const bdgfs_hybrid_args* h, const float* Y,
                           int64_t ldy, int64_t k, int32_t nheads,
                           void* out, int64_t ldo, void* stream);

/* ------------------------------------------------------------------------
 * BGK relaxation ('bgk-direct-gll') and the ARS IMEX stage update of the
 * 'adgfs' system (frfs/solvers/adgfs/scattering.py,
 * frfs/solvers/adgfs/kernels/scattering/bgk-direct-gll.mako,
 * linear-common-direct-gll.mako, frfs/integrators/std/steppers.py:489-670).
 * Moment rows U[dof][5] = (rho, rho u_x, rho u_y, rho u_z, E), FP64,
 * E = sum |c|^2 f cw; T = (E - |rho u|^2/rho) / (1.5 rho);
 * nu = prefac * rho * T^(1 - omega); M = rho/(pi T)^1.5 exp(-|c-u|^2/T).
 * ---------------------------------------------------------------------- */
#define BDGFS_ARS_MOM0 1   /* U[0]      <- moments of f[0]                  */
#define BDGFS_ARS_MOML 2   /* LU[ar-1]  <- moments of L[ar-1]               */
#define BDGFS_ARS_MOMU 4   /* U[ar]     <- U[0] + dt sum_j ae[j] LU[j]      */
#define BDGFS_ARS_DIST 8   /* fout      <- (f0 + sum_j ae[j] dt L_j
                                + sum_{j=1}^{ar-1} ai[j-1] dt nu_j (M_j - f_j)
                                + ai[ar-1] dt nu_ar M_ar)
                               / (1 + ai[ar-1] dt nu_ar)                    */

typedef struct bdgfs_ars_args {
    int64_t ndof;            /* distributions (rows)                        */
    int32_t Nv;              /* 1..64                                       */
    int32_t fp64;
    const double* c0;        /* [Nv]                                        */
    double cw;
    double prefac, omega, dt;
    int32_t stage;           /* ar = 1..4                                   */
    int32_t flags;           /* BDGFS_ARS_*                                 */
    double ae[4];            /* explicit row _A[ar][0..ar-1]                */
    double ai[4];            /* implicit row A[ar][1..ar]                   */
    const void* f[4];        /* f_0 .. f_{ar-1}                             */
    void* fout;              /* f_ar (may be f_0: updated in place)         */
    const void* L[4];        /* L_0 .. L_{ar-1} (explicit FR parts)          */
    double* U[5];            /* moment rows U_0 .. U_ar (5, 11 or 14)       */
    double* LU[4];           /* moment rows of L_0 .. L_{ar-1}              */
    int32_t model;           /* BDGFS_ARS_BGK (5 moments, Maxwellian),
                                BDGFS_ARS_ESBGK (11 moments, ES Gaussian) or
                                BDGFS_ARS_SHAKOV (14 moments, Shakov)       */
    int32_t pad_;
    double Pr;               /* Prandtl number (ES-BGK, Shakov)             */
} bdgfs_ars_args;

#define BDGFS_ARS_BGK 0
#define BDGFS_ARS_ESBGK 1
#define BDGFS_ARS_SHAKOV 2

/* U[dof] = moments of f[dof]: ADGFSBGKDirectGLLScatteringModel.moment. */
int32_t bdgfs_bgk_moments(const void* f, int64_t ndof, int32_t Nv, int32_t fp64,
                          const double* c0, double cw, double* U, void* stream);
/* M[dof] = Maxwellian of U[dof]: cmaxwellian (bgk-direct-gll.mako:4-50). */
int32_t bdgfs_bgk_maxwellian(const double* U, int64_t ndof, int32_t Nv,
                             int32_t fp64, const double* c0, void* M,
                             void* stream);
/* ES-BGK ('esbgk-direct-gll', frfs/solvers/adgfs/scattering.py,
 * ADGFSESBGKDirectGLLScatteringModel): U[dof][11] = moments of f[dof]
 * {1, c, |c|^2, cx^2, cy^2, cz^2, cx cy, cy cz, cz cx} cw (the moment
 * method), and M[dof] = the Gaussian of the ES tensor of U[dof]
 * (momentNorm + cmaxwellian, esbgk-direct-gll.mako:4-120). */
int32_t bdgfs_esbgk_moments(const void* f, int64_t ndof, int32_t Nv,
                            int32_t fp64, const double* c0, double cw,
                            double* U, void* stream);
int32_t bdgfs_esbgk_gaussian(const double* U, int64_t ndof, int32_t Nv,
                             int32_t fp64, const double* c0, double Pr,
                             void* M, void* stream);
/* ------------------------------------------------------------------------
 * Gas mixtures: fast-spectral VSS collision operator on one velocity grid
 * ---------------------------------------------------------------------- */

/* Q_p = sum_q Q_pq(f_p, f_q) for every species p and distribution
 * (DGFSBiVSSGLLScatteringModel.fs, frfs/solvers/dgfsbi/scattering.py:
 * 229-330; kernels/scattering/vss-gll.mako:100-300).  Tables (built on the
 * host from the reference's precompute_a / precompute_bc_pq):
 *   rfac[r] = pi/L qz_r, rw[r] = qw_r sw / Nv^3, sz = the M full-sphere
 *   directions, mfrac[p*S+q] = m_q/(m_p+m_q), prefac[p*S+q],
 *   b[p*S+q][r*M+s][Nv^3] and c[p*S+q][Nv^3] complex in the state's
 *   precision (interleaved re, im). */
typedef struct bdgfs_vss_args {
    int32_t Nv;              /* 8, 12, 16, 24 or 32                          */
    int32_t nspcs;           /* species, 1..4                                */
    int32_t Nrho;
    int32_t M;
    int64_t ndof;            /* distributions per species                    */
    int32_t fp64;
    int32_t pad_;
    const void* f[4];        /* real [ndof][Nv^3] per species                */
    void* Q[4];              /* real [ndof][Nv^3] per species (written)      */
    const double* mfrac;
    const double* prefac;
    const double* rfac;
    const double* rw;
    const double* sz;        /* [M][3]                                       */
    const void* b;
    const void* c;
} bdgfs_vss_args;
/* Scratch for nctas persistent CTAs: 6 complex Nv^3 arrays each.  The
 * launch uses as many CTAs as the scratch holds (at most ndof * nspcs). */
size_t bdgfs_vss_scratch_bytes(int32_t Nv, int32_t fp64, int32_t nctas);
int32_t bdgfs_vss_collide(const bdgfs_vss_args* a, void* scratch, size_t bytes,
                          void* stream);

/* FP64 conservation projection of a mixture's Q, in place, per
 * distribution: the minimal-norm change of (Q_0 .. Q_{S-1}) that zeroes each
 * species' mass and the total momentum and energy (species weighted by
 * their masses).  ginv is the inverse (S+4) x (S+4) Gram matrix of the
 * constraint functions (1 per species; m_p c; m_p |c|^2) over the grid.
 * New relative to the reference's vss-gll operator (it has no projection);
 * the counterpart of the VHS kernel's BDGFS_PROJECT for mixtures. */
typedef struct bdgfs_vss_proj_args {
    int32_t Nv;
    int32_t nspcs;           /* 1..4                                          */
    int64_t ndof;
    int32_t fp64;
    int32_t pad_;
    void* Q[4];              /* real [ndof][Nv^3] per species (updated)       */
    const double* c0;        /* [Nv]                                          */
    const double* mass;      /* [nspcs] molar masses / molarMass0             */
    const double* ginv;      /* [(nspcs+4)^2], row-major                      */
} bdgfs_vss_proj_args;
int32_t bdgfs_vss_project(const bdgfs_vss_proj_args* a, void* stream);

/* One IMEX-BDF step of the 'adgfs' system (BDF2/BDF3AstdStepper.step,
 * frfs/integrators/std/steppers.py:680-860: updateMom{q}_BDF,
 * constructMaxwellian and updateDistribution{q}_BDF of
 * kernels/scattering/{bgk,esbgk,shakov}-direct-gll.mako and
 * linear-common-direct-gll.mako:40-88).  With X_0..X_{q-1} oldest to
 * newest: N = -sum_i (a_i X_i + g_i dt LX_i); the new moments U = N/a_q for
 * the conserved five (higher ones relax implicitly as in the reference) and
 * f = (N_f + b dt nu M[U]) / (a_q + b dt nu).  g_i are the reference's
 * arguments (the negated G coefficients). */
#define BDGFS_BDF_MOMN 1     /* reduce U[q-1], LU[q-1] from f[q-1], L[q-1]  */
#define BDGFS_BDF_MOMU 2     /* form Unew                                    */
#define BDGFS_BDF_DIST 4     /* write fout                                   */
typedef struct bdgfs_bdf_args {
    int64_t ndof;
    int32_t Nv;
    int32_t fp64;
    const double* c0;        /* [Nv] (FP64)                                  */
    double cw;
    double prefac;           /* nu = prefac rho T^(1 - omega)                */
    double omega;
    double dt;
    int32_t q;               /* history length 1..3                          */
    int32_t model;           /* BDGFS_ARS_BGK / _ESBGK / _SHAKOV             */
    double Pr;
    double a[4];             /* a_0..a_q                                     */
    double g[3];             /* g_0..g_{q-1}                                 */
    double b;
    const void* f[3];        /* distributions f_0..f_{q-1} ([ndof][Nv^3])    */
    const void* L[3];        /* explicit parts L_0..L_{q-1}                  */
    double* U[3];            /* moment rows of f_i ([ndof][5, 11 or 14])     */
    double* LU[3];           /* moment rows of L_i                           */
    double* Unew;            /* new moment rows (written with MOMU, read
                                otherwise)                                   */
    void* fout;              /* new distribution (may alias f[0])            */
    int32_t flags;
    int32_t pad_;
} bdgfs_bdf_args;
int32_t bdgfs_bdf_step(const bdgfs_bdf_args* a, void* stream);

/* Shakov ('shakov-direct-gll', frfs/solvers/adgfs/scattering.py,
 * ADGFSShakovDirectGLLScatteringModel): U[dof][14] = the 11 ES-BGK moments
 * followed by {|c|^2 c} cw, and S[dof] = M (1 + 2 (1 - Pr)/5 (q.d)/(rho T^2)
 * (2 |d|^2/T - 5)) with q the heat flux of U[dof] (momentNorm + cmaxwellian,
 * shakov-direct-gll.mako:4-95). */
int32_t bdgfs_shakov_moments(const void* f, int64_t ndof, int32_t Nv,
                             int32_t fp64, const double* c0, double cw,
                             double* U, void* stream);
int32_t bdgfs_shakov_target(const double* U, int64_t ndof, int32_t Nv,
                            int32_t fp64, const double* c0, double Pr,
                            void* S, void* stream);
/* One ARS stage (the flagged parts, in the order MOM0, MOML, MOMU, DIST):
 * updateMom{ar}_ARS + cmaxwellian + updateDistribution{ar}_ARS in one
 * launch, the Maxwellians computed on the fly. */
int32_t bdgfs_ars_stage(const bdgfs_ars_args* a, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BDGFS_H */
