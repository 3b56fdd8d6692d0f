/*
 * fea_b200 — C ABI of the B200 (sm_100a) element / assembly / solver library.
 *
 * Plain C: integers, raw pointers and sizes, no framework types.  Every entry
 * point returns an int status: 0 = ok, negative = bad argument / size /
 * plan (see FEA_E*), positive = a CUDA error code from the launch.  Device
 * entry points are asynchronous on the given stream unless stated; pointers
 * named *_dev are device memory, the others host memory.
 *
 * The library replaces the hot path of the reference package sssnnn7119/FEA:
 *   - Element_3D.initialize COO pattern + element-to-slot map
 *       (FEA/assemble/elements/C3/C3base.py:109-153) and the Dirichlet
 *       reduction/relabelling (FEA/assemble/assembly.py:357-387)
 *         -> fea_plan_build / fea_plan_get  (host, once per mesh)
 *   - Element_3D.structural_Force R + K + slot scatter (C3base.py:413-452),
 *       NeoHookean.material_Constitutive_C3 (materials/hyperelastic.py:35-84),
 *       Assembly._assemble_generalized_Matrix (assembly.py:311-355)
 *         -> fea_assemble_volume
 *   - Pressure.get_stiffness (FEA/assemble/loads/pressure.py:80-132)
 *         -> fea_assemble_pressure
 *   - Element_3D.potential_Energy (C3base.py:387-411) and
 *       Pressure.get_potential_energy (pressure.py:134-159)
 *         -> fea_energy_volume / fea_energy_pressure
 *   - Element_3D.get_mass_matrix + row-sum lumping (C3base.py:348-384,
 *       FEA/solver/dynamic_explicit.py:147-167) -> fea_lumped_mass
 *   - _linear_solver.conjugate_gradient with the symmetric Jacobi scaling of
 *       StaticImplicitSolver._solve_linear_equation
 *       (FEA/solver/_linear_solver.py:6-42, FEA/solver/static_implicit.py:352-405)
 *         -> fea_pcg_solve / fea_pcg_solve_mixed
 *   - DynamicExplicitSolver.solve time loop (dynamic_explicit.py:97-140)
 *         -> fea_explicit_run
 */
#ifndef FEA_B200_H
#define FEA_B200_H

#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FEA_OK 0
#define FEA_EINVAL -1      /* bad argument (null pointer, negative size, bad kind) */
#define FEA_ERANGE -2      /* index out of range in the inputs (node id >= n_nodes) */
#define FEA_ECHUNK -3      /* one node needs more threads / shared memory than a chunk holds */
#define FEA_ESMEM -4       /* requested shared memory exceeds the device limit */
#define FEA_EWORK -5       /* caller-provided work buffer too small */
#define FEA_ENOTCONV -6    /* iterative solver hit its iteration cap */
#define FEA_EBREAKDOWN -7  /* PCG breakdown (p.Ap <= 0 or non-finite) */
#define FEA_ETOOBIG -8     /* size beyond a fixed limit: of an allocation-free entry point, or a
                              group of more than FEA_PLAN_MAX_ELEMS elements or faces */

/* element kinds (reference class names) */
#define FEA_C3D4 4
#define FEA_C3D8 8
/* surface kinds for the follower pressure */
#define FEA_T3 3
#define FEA_Q4 40

/* ---------------------------------------------------------------------------
 * Host-side plan: reduced pattern, node adjacency and per-node gather lists.
 * ------------------------------------------------------------------------- */
typedef struct fea_plan fea_plan;

/* Build the plan for one assembly.
 *   n_nodes          nodes of the (single) instance
 *   free_mask[n]     bit k set <=> DOF (n, k) is free (not Dirichlet, and the
 *                    node belongs to an element); 0 = node has no rows
 *   groups           n_groups element groups: kind (FEA_C3D4 / FEA_C3D8),
 *                    element count, connectivity int32 [ne, nn] (host)
 *   faces            n_faces pressure face groups: kind (FEA_T3 / FEA_Q4),
 *                    face count, node lists int32 [nf, 3|4] (host)
 *   vol_threads      incidences per gather chunk for the element kernels
 *                    (0 = default: 32 for C3D8 (8 lanes each), 256 for C3D4)
 *   smem_doubles     per-chunk shared-memory budget in doubles (0 = default)
 * The reduced DOF numbering is node-major over free DOFs, as GC in the
 * reference (assembly.py:170-183); the CSR pattern equals the reference's
 * coalesced reduced K pattern.  A group of more than FEA_PLAN_MAX_ELEMS
 * elements (faces) returns FEA_ETOOBIG: incidences are coded e * 16 + a in
 * 32 bits; split larger meshes into several groups. */
#define FEA_PLAN_MAX_ELEMS 134217727
int fea_plan_build(int64_t n_nodes, const uint8_t* free_mask,
                   int32_t n_groups, const int32_t* group_kind, const int64_t* group_ne,
                   const int32_t* const* group_conn,
                   int32_t n_faces, const int32_t* face_kind, const int64_t* face_nf,
                   const int32_t* const* face_conn,
                   int32_t vol_threads, int64_t smem_doubles, fea_plan** out);
void fea_plan_free(fea_plan* plan);

/* Array / scalar ids for fea_plan_get. "group" selects the element group
 * (FEA_A_G_*) or the face group (FEA_A_F_*); ignored otherwise. */
enum {
  FEA_S_NDOF = 0,        /* int64 scalar: reduced DOF count n            */
  FEA_S_NNZ = 1,         /* int64 scalar: nonzeros of the reduced K       */
  FEA_S_NNZB = 2,        /* int64 scalar: node-level adjacency entries    */
  FEA_A_RDOF = 10,       /* int32 [N]   first reduced DOF of node, -1 none */
  FEA_A_MASK = 11,       /* uint8 [N]   free-DOF bits                      */
  FEA_A_DBASE = 12,      /* int32 [N+1] prefix of free-DOF counts          */
  FEA_A_VBASE = 13,      /* int64 [N+1] first K value of the node's rows   */
  FEA_A_ROWLEN = 14,     /* int32 [N]   scalar row length of the node      */
  FEA_A_INDPTR = 15,     /* int64 [n+1] CSR row pointer                    */
  FEA_A_INDICES = 16,    /* int32 [nnz] CSR column indices                 */
  FEA_A_ADJPTR = 17,     /* int64 [N+1] node adjacency row pointer         */
  FEA_A_ADJCOL = 18,     /* int32 [nnzb] neighbour node                    */
  FEA_A_ADJOFF = 19,     /* int32 [nnzb] value offset of neighbour in row  */
  FEA_A_MOFF = 20,       /* int32 [nnzb] value offset of the row node in the neighbour's row */
  FEA_A_G_INC = 30,      /* int32 [ninc] element*16 + local node           */
  FEA_A_G_BOFF = 31,     /* uint16 [ninc, nn] row offset per element node  */
  FEA_A_G_NODEINC = 32,  /* int32 [N+1] first incidence of each node       */
  FEA_A_G_CHUNKPTR = 33, /* int32 [nchunk+1] chunk -> range of CHUNKLIST   */
  FEA_A_G_CHUNKINC = 34, /* int32 [nchunk+1] first incidence of each chunk */
  FEA_S_G_NCHUNK = 35,   /* int64 scalar */
  FEA_S_G_MAXVAL = 36,   /* int64 scalar: max incidences of one node       */
  FEA_S_G_THREADS = 37,  /* int64 scalar: threads per chunk                */
  FEA_S_G_SMEM = 38,     /* int64 scalar: max shared doubles of a chunk    */
  FEA_A_G_CHUNKLIST = 39,/* int32 nodes with incidences, chunk by chunk   */
  FEA_A_G_CHUNKDIM = 40, /* int32 [nchunk,3] values, residual entries, contiguous */
  FEA_A_G_SOFF = 41,     /* int32 [N] shared offset of the node's values   */
  FEA_A_G_ROFF = 42,     /* int32 [N] offset of its residual entries       */
  FEA_A_G_UPTR = 43,     /* int64 [N+1] first upper-block record of each node (C3D8)      */
  FEA_A_G_UBLK = 44,     /* int64 [nu, 4] upper-block records (fea_ublk_t layout, C3D8)   */
  FEA_A_G_ALLPTR = 45,   /* int32 [N+1] incidences of every node (all nodes) */
  FEA_A_G_ALLINC = 46,   /* int32 element*16 + a                           */
  FEA_A_G_INCPOS = 47,   /* int32 [ne, nn] incidence index of (e, a), -1: node without rows */
  FEA_A_G_STAGEPOS = 48, /* int32 [ne, 36] staged block of each element block, -1: none  */
  FEA_A_G_REGION = 49,   /* int64 [N+1] first staged block of each node's region (even)   */
  FEA_S_G_HXSTRIDE = 70, /* int64 scalar: C3D8 fixed region stride in blocks, 0 = packed  */
  FEA_A_F_INC = 50,      /* the same arrays / scalars for face groups      */
  FEA_A_F_BOFF = 51,
  FEA_A_F_NODEINC = 52,
  FEA_A_F_CHUNKPTR = 53,
  FEA_A_F_CHUNKINC = 54,
  FEA_S_F_NCHUNK = 55,
  FEA_S_F_MAXVAL = 56,
  FEA_S_F_THREADS = 57,
  FEA_S_F_SMEM = 58,
  FEA_A_F_CHUNKLIST = 59,
  FEA_A_F_CHUNKDIM = 60,
  FEA_A_F_SOFF = 61,
  FEA_A_F_ROFF = 62,
  FEA_A_F_ALLPTR = 65,
  FEA_A_F_ALLINC = 66
};

/* Copy array `id` (of element/face group `group`) into dst (host memory),
 * or, for FEA_S_* ids, write the scalar to *count.  With dst == NULL only
 * *count (number of entries) is set. */
int fea_plan_get(const fea_plan* plan, int32_t id, int32_t group, void* dst, int64_t* count);

/* ---------------------------------------------------------------------------
 * Device-side descriptors (device pointers; filled from the plan's arrays).
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t n_nodes;
  int64_t ndof;
  int64_t nnz;
  const double* X_dev;        /* [N,3] reference coordinates of the part     */
  const int32_t* rdof_dev;    /* FEA_A_RDOF   */
  const uint8_t* mask_dev;    /* FEA_A_MASK   */
  const int64_t* vbase_dev;   /* FEA_A_VBASE  */
  const int32_t* rowlen_dev;  /* FEA_A_ROWLEN */
  const int32_t* dbase_dev;   /* FEA_A_DBASE  */
  const int64_t* adjptr_dev;  /* FEA_A_ADJPTR */
  const int32_t* adjcol_dev;  /* FEA_A_ADJCOL */
  const int32_t* adjoff_dev;  /* FEA_A_ADJOFF */
  const int32_t* moff_dev;    /* FEA_A_MOFF   */
} fea_nodes_t;

/* C3D8 staging.  Element block {i, j} of element e (the 36 unordered local
 * pairs, in the slot order of the element kernel's lanes: lane a < 4 holds
 * (a, a + d mod 8) for d = 0..4 at slots 5a + d, lane a >= 4 holds d = 0..3 at
 * 20 + 4(a - 4) + d) is staged at block STAGEPOS[e, slot], oriented as the
 * upper node block (row node min(n_i, n_j), column node max): a node's
 * region REGION[n] .. REGION[n+1] holds, block-major, the contributions to
 * its upper blocks in adjacency order, each block's in ascending element
 * order.  One record per upper block (row n, column c >= n), from UPTR[n].
 * In the fixed layout of a regular mesh (FEA_S_G_HXSTRIDE > 0) REGION[n] =
 * n * stride, UPTR[n] = 16 n (record slots past the node's own hold row =
 * col = -1) and the residual slot of incidence (e, a) (INCPOS) is n * maxval
 * + its rank among the node's incidences: */
typedef struct {
  int64_t row;                /* value index of (first free row of n, first free column of c)  */
  int64_t col;                /* value index of the transpose in c's rows; -1 on the diagonal  */
  int32_t rowlen_c;           /* values per row of c                                           */
  int32_t mask_c;             /* free-DOF mask of c                                            */
  int32_t first;              /* first contribution, relative to REGION[n]                     */
  int32_t count;              /* contributions (0: the block is written as zero)               */
} fea_ublk_t;

typedef struct {
  int32_t kind;               /* FEA_C3D4 / FEA_C3D8, or FEA_T3 / FEA_Q4      */
  int32_t nn;                 /* nodes per element / face                     */
  int64_t ne;                 /* elements / faces                             */
  const int32_t* conn_dev;    /* [ne, nn]                                     */
  const int32_t* inc_dev;     /* FEA_A_*_INC                                  */
  const uint16_t* boff_dev;   /* FEA_A_*_BOFF                                 */
  const int32_t* nodeinc_dev; /* FEA_A_*_NODEINC                              */
  const int32_t* chunkptr_dev;
  const int32_t* chunkinc_dev;
  const int32_t* chunklist_dev;
  const int32_t* chunkdim_dev;
  const int32_t* soff_dev;
  const int32_t* roff_dev;
  const int64_t* uptr_dev;    /* FEA_A_G_UPTR (C3D8 only) */
  const fea_ublk_t* ublk_dev; /* FEA_A_G_UBLK (C3D8 only) */
  const int32_t* allptr_dev;  /* FEA_A_*_ALLPTR (adjoint kernels) */
  const int32_t* allinc_dev;
  int64_t nchunk;
  int32_t maxval;
  int32_t threads;
  int64_t smem_doubles;
  const int32_t* incpos_dev;  /* FEA_A_G_INCPOS (C3D8 only) */
  const int32_t* stagepos_dev;/* FEA_A_G_STAGEPOS (C3D8 only) */
  const int64_t* region_dev;  /* FEA_A_G_REGION (C3D8 only) */
  int64_t nblk;               /* staged blocks: REGION[N] (C3D8 only)         */
  int32_t maxblk;             /* largest region, in blocks (C3D8 only)        */
  int32_t hx_stride;          /* FEA_S_G_HXSTRIDE: > 0 when the C3D8 staging has
                                 the fixed layout (regions at n * hx_stride =
                                 n * maxblk, records at 16 n, residual slots at
                                 n * maxval); 0: packed (REGION, UPTR, NODEINC) */
} fea_group_t;

/* Element residual and tangent of one Neo-Hookean group, gathered per node
 * row and written once into the reduced CSR values (store mode) or added to
 * them (accumulate != 0).  gc_dev: reduced displacement [ndof] (NULL allowed
 * when ndof == 0).  Any of K_dev / R_dev / elemR_dev may be NULL.  A group
 * without elements writes nothing in either mode and needs no work (its
 * INCPOS and STAGEPOS may be NULL).  elemR_dev receives the unassembled
 * element residual in the reference's (a, j, e) order [nn*3*ne]; it is only
 * meaningful for a plan whose every element node is active.
 * work_dev: fea_assemble_work_len(group) doubles of scratch, 16-byte
 * aligned (C3D8 stages there the upper blocks of every element row, 9
 * doubles each, node by node (nblk blocks), then R_a of every incidence, 4
 * doubles each; C3D4 needs none). */
int64_t fea_assemble_work_len(const fea_group_t* group);
int fea_assemble_volume(const fea_nodes_t* nodes, const fea_group_t* group, double mu, double kappa,
                        const double* gc_dev, double* K_dev, double* R_dev, double* elemR_dev,
                        int32_t accumulate, double* work_dev, int64_t work_len, cudaStream_t stream);

/* Follower pressure p on a face group: adds -p dV/dx to R and -p d2V/dx2 to
 * K (always accumulate).  Xinst_dev: instance node coordinates [N,3]. */
int fea_assemble_pressure(const fea_nodes_t* nodes, const fea_group_t* faces, double p,
                          const double* Xinst_dev, const double* gc_dev,
                          double* K_dev, double* R_dev, cudaStream_t stream);

/* Strain energy sum_{g,e} W(F) w of a group, written to out_dev[0]
 * (deterministic two-stage reduction; scratch_dev needs
 * fea_reduce_scratch_len(ne) doubles). */
int64_t fea_reduce_scratch_len(int64_t n_items);
int fea_energy_volume(const fea_nodes_t* nodes, const fea_group_t* group, double mu, double kappa,
                      const double* gc_dev, double* out_dev, double* scratch_dev, int64_t scratch_len,
                      cudaStream_t stream);
/* Allocation-free variant of fea_energy_volume (no counterpart in the
 * reference).  For callers that cannot allocate device memory when they call
 * the library — e.g. a host that reserves all device memory for its own pool
 * allocator, or a foreign-language host that only passes pointers it already
 * owns — and so cannot provide the scratch buffer fea_energy_volume needs.
 * The scratch is a fixed array inside the library's device image, sized for
 * at most FEA_NOALLOC_MAX_ELEMS elements per group; larger groups return
 * FEA_ETOOBIG without launching.  Nothing is allocated (no cudaMalloc /
 * cudaFree, no allocating library routine).  The first call on each device
 * resolves the array's device address (cudaGetSymbolAddress) with that device
 * current, so make that first call before any stream capture.  Every call
 * shares the one array: calls that may overlap on the GPU (different streams
 * or threads) race and must be serialised by the caller.  Same result as
 * fea_energy_volume (same kernels and summation order). */
#define FEA_NOALLOC_MAX_ELEMS 4194304
int fea_energy_volume_noalloc(const fea_nodes_t* nodes, const fea_group_t* group, double mu, double kappa,
                              const double* gc_dev, double* out_dev, cudaStream_t stream);

/* Enclosed-volume functional V of a face group -> out_dev[0]. */
int fea_energy_pressure(const fea_nodes_t* nodes, const fea_group_t* faces, const double* Xinst_dev,
                        const double* gc_dev, double* out_dev, double* scratch_dev, int64_t scratch_len,
                        cudaStream_t stream);

/* Row-sum lumped mass over free DOFs, added into m_dev [ndof] (call once per
 * group on a zeroed vector, then fea_invert_mass). */
int fea_lumped_mass(const fea_nodes_t* nodes, const fea_group_t* group, double rho,
                    double* m_dev, cudaStream_t stream);
int fea_invert_mass(int64_t ndof, double* m_dev, cudaStream_t stream);

/* Consistent mass of one element group added into Mv_dev [nnz], the values
 * of the plan's reduced CSR pattern (the mass couples like directions of two
 * nodes, a subset of the stiffness pattern; other entries are left as they
 * are).  Replaces Element_3D.get_mass_matrix (FEA/assemble/elements/C3/
 * C3base.py:348-384) with the reduction of Assembly.assemble_mass_matrix
 * (FEA/assemble/assembly.py:421-443), whose duplicates this sums. */
int fea_mass_csr(const fea_nodes_t* nodes, const fea_group_t* group, double rho, double* Mv_dev,
                 cudaStream_t stream);

/* y += alpha x over n doubles (the effective tangent K + M / (beta dt^2) of
 * FEA/solver/dynamic_implicit.py:120-146 on CSR values of one pattern). */
int fea_axpy(int64_t n, double alpha, const double* x_dev, double* y_dev, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Jacobi-preconditioned CG on the reduced CSR matrix.
 *   stop test: (r.D^-1 r) / (b.D^-1 b) < tol  — the reference's
 *   ||r~||^2/||b~||^2 < tol on the symmetrically scaled system.
 *   x_dev holds the initial guess on entry (warm start) and the solution on
 *   exit.  work_dev: fea_pcg_work_len(n) doubles.  iters / relres: host outs.
 *   check_every: iterations between host-side convergence checks.
 *   jacobi: 1 = Jacobi preconditioner (the solver's scaled CG), 0 = plain CG
 *   (the reference's conjugate_gradient on an unscaled matrix).
 * Returns FEA_OK, FEA_ENOTCONV (cap reached) or FEA_EBREAKDOWN.
 * ------------------------------------------------------------------------- */
int64_t fea_pcg_work_len(int64_t n);
int fea_pcg_solve(int64_t n, const int64_t* indptr_dev, const int32_t* indices_dev, const double* values_dev,
                  const double* b_dev, double* x_dev, double tol, int32_t max_iter, int32_t check_every,
                  int32_t jacobi, double* work_dev, int64_t work_len, int32_t* iters, double* relres,
                  cudaStream_t stream);
/* FP32-SpMV CG with FP64 refinement of the residual: the iterations run in
 * FP32 (float values, vectors and SpMV; FP64 accumulation of the dot
 * products) on the correction since the last refinement; every check_every
 * iterations the correction is added to the FP64 solution, the true residual
 * b - A x is formed in FP64 and replaces the FP32 one, and the recurrence
 * continues with the same search direction (residual replacement, no
 * restart).  The stop test is fea_pcg_solve's, on the FP64 residual.
 * values32_dev: float copy of values.  inner_tol > 0: a batch of
 * check_every iterations ends in a replacement only once the FP32 r.D^-1 r
 * has fallen below inner_tol times its value at the last replacement (or
 * the stop test may pass, the FP32 recurrence broke down, or the cap is
 * reached); inner_tol <= 0 replaces after every batch.  outer: number of
 * refinements.  work: fea_pcg_mixed_work_len(n) doubles. */
int64_t fea_pcg_mixed_work_len(int64_t n);
int fea_pcg_solve_mixed(int64_t n, const int64_t* indptr_dev, const int32_t* indices_dev,
                        const double* values_dev, const float* values32_dev,
                        const double* b_dev, double* x_dev, double tol, double inner_tol,
                        int32_t max_iter, int32_t check_every,
                        double* work_dev, int64_t work_len, int32_t* iters, int32_t* outer,
                        double* relres, cudaStream_t stream);
/* y = K x (FP64) */
int fea_spmv(int64_t n, const int64_t* indptr_dev, const int32_t* indices_dev, const double* values_dev,
             const double* x_dev, double* y_dev, cudaStream_t stream);

/* The same solvers and SpMV on a matrix in the plan's reduced layout (the
 * values written by fea_assemble_volume / fea_assemble_pressure; indices_dev
 * = FEA_A_INDICES).  The f free rows of node n share one column list of
 * length rowlen[n] and start at vbase[n] + j * rowlen[n], so one warp per
 * node reads the column indices and gathers x once for all f rows.  Always
 * Jacobi-preconditioned (the path of StaticImplicitSolver._solve_linear_equation,
 * static_implicit.py:352-405); work lengths as fea_pcg_work_len(ndof) /
 * fea_pcg_mixed_work_len(ndof); results equal those of fea_pcg_solve /
 * fea_pcg_solve_mixed on the same CSR up to the order of the row sums. */
int fea_spmv_nodes(const fea_nodes_t* nodes, const int32_t* indices_dev, const double* values_dev,
                   const double* x_dev, double* y_dev, cudaStream_t stream);
int fea_pcg_solve_nodes(const fea_nodes_t* nodes, const int32_t* indices_dev, const double* values_dev,
                        const double* b_dev, double* x_dev, double tol, int32_t max_iter, int32_t check_every,
                        double* work_dev, int64_t work_len, int32_t* iters, double* relres, cudaStream_t stream);
int fea_pcg_solve_mixed_nodes(const fea_nodes_t* nodes, const int32_t* indices_dev, const double* values_dev,
                              const float* values32_dev, const double* b_dev, double* x_dev, double tol,
                              double inner_tol, int32_t max_iter, int32_t check_every, double* work_dev,
                              int64_t work_len, int32_t* iters, int32_t* outer, double* relres,
                              cudaStream_t stream);
/* The mixed solver on an FP32 copy of the plan's matrix in a padded layout:
 * node n's column list starts at cbase[n] and its row j at qbase[n] + j *
 * (cbase[n+1] - cbase[n]); both are multiples of 4 and every list is padded
 * to a multiple of 4 entries (column 0, value 0), so that the FP32 SpMV
 * reads 4 columns and 4 values of each row with 128-bit loads, one warp per
 * node.  cbase / qbase are prefix sums over the nodes of L4 = rowlen rounded
 * up to 4 (0 for a node without free DOFs) and of popcount(mask) * L4.
 * fea_f32_layout_fill writes vals_dev (and cols_dev when with_cols != 0)
 * from the FP64 values in the plan's layout.  No counterpart in the
 * reference (its solves are FP64 throughout). */
typedef struct {
  const int64_t* cbase_dev;   /* [N+1] */
  const int64_t* qbase_dev;   /* [N+1] */
  int32_t* cols_dev;          /* [cbase[N]] */
  float* vals_dev;            /* [qbase[N]] */
} fea_f32_layout_t;
int fea_f32_layout_fill(const fea_nodes_t* nodes, const int32_t* indices_dev, const double* values_dev,
                        fea_f32_layout_t* layout, int32_t with_cols, cudaStream_t stream);
int fea_pcg_solve_mixed_nodes32(const fea_nodes_t* nodes, const int32_t* indices_dev, const double* values_dev,
                                const fea_f32_layout_t* layout, const double* b_dev, double* x_dev, double tol,
                                double inner_tol, int32_t max_iter, int32_t check_every, double* work_dev,
                                int64_t work_len, int32_t* iters, int32_t* outer, double* relres,
                                cudaStream_t stream);
/* ---------------------------------------------------------------------------
 * Batched Jacobi-PCG over independent systems ("slots"), for serving many
 * static solves at once (no counterpart in the reference, which solves one
 * system at a time with _linear_solver.conjugate_gradient,
 * _linear_solver.py:6-42).  Work items are warp-sized and fixed per slot:
 * SpMV items of 16 nodes (plan layout) or 16 rows (CSR), update items of 256
 * rows; every kernel walks the item lists of all active slots, and each slot
 * keeps its own scalars, per-item partial sums and stop test (same test and
 * status codes as fea_pcg_solve with jacobi = 1).  A slot's iterates do not
 * depend on the other slots: alone or in a batch, it computes the same bits.
 *   table: fea_pcgb_table_bytes(max_slots, max_items) bytes of device memory;
 *     max_items bounds the items of all active slots in each list.
 *   fea_pcgb_set: loads the slot table (host array of nslots descriptors;
 *     work == NULL marks an empty slot) and the item lists of the active
 *     slots; synchronises `stream`.  Every descriptor is checked before
 *     the first device call: a call that returns FEA_EINVAL, FEA_EWORK or
 *     FEA_ERANGE has changed neither the table nor any work buffer.
 *   fea_pcgb_start: initial residual, Jacobi scaling and state of one slot
 *     (x holds the initial guess).  n and nnz are the slot's own (they size
 *     the launch; chunks beyond the slot's rows exit without writing).
 *   fea_pcgb_iterate: `iters` iterations of every active, unfinished slot;
 *     a fixed launch sequence that reads the table from device memory, so it
 *     can be captured once and replayed while slots come and go.
 *   fea_pcgb_state: out_dev[4*slot + {0,1,2,3}] = done, iterations, status,
 *     (r.D^-1 r) / (b.D^-1 b).
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t n;                   /* rows                                        */
  int64_t nnz;
  const int64_t* indptr_dev;
  const int32_t* indices_dev;
  const double* values_dev;
  const double* b_dev;
  double* x_dev;               /* initial guess in, iterate out               */
  double* work_dev;            /* fea_pcgb_work_len(n, n_nodes) doubles; NULL: empty */
  int64_t work_len;
  double tol;
  int32_t max_iter;
  int32_t active;              /* 0: kept in the table, not iterated          */
  /* Optional plan layout of the matrix (vbase_dev NULL: plain CSR rows): the
   * fea_nodes_t arrays, so that the SpMV runs node rows. */
  int64_t n_nodes;
  const int64_t* vbase_dev;
  const int32_t* rowlen_dev;
  const int32_t* dbase_dev;
  const uint8_t* mask_dev;
} fea_pcgb_slot_t;
int64_t fea_pcgb_work_len(int64_t n, int64_t n_nodes);
int64_t fea_pcgb_table_bytes(int32_t max_slots, int64_t max_items);
int fea_pcgb_set(void* table_dev, int32_t max_slots, int64_t max_items, int32_t nslots,
                 const fea_pcgb_slot_t* slots, cudaStream_t stream);
int fea_pcgb_start(void* table_dev, int32_t max_slots, int64_t max_items, int32_t slot, int64_t n, int64_t nnz,
                   cudaStream_t stream);
int fea_pcgb_iterate(void* table_dev, int32_t max_slots, int64_t max_items, int32_t iters, cudaStream_t stream);
int fea_pcgb_state(void* table_dev, int32_t max_slots, int64_t max_items, int32_t nslots, double* out_dev,
                   cudaStream_t stream);

/* values32 = (float) values */
int fea_convert_f32(int64_t nnz, const double* values_dev, float* values32_dev, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Device line search of the Newton solver.  Replaces the host loop of
 * StaticImplicitSolver._line_search (static_implicit.py:97-169: Armijo with
 * c1, step halving from 1, no step below 1e-12, step-length cap) by trial
 * energies evaluated on the device a ladder at a time.
 *   state_dev: FEA_LS_NSTATE doubles.  fea_ls_prepare writes
 *     [DE] = -|dgc.R|, [E0] = *e0_dev (energy at gc), [SMAX] = max|dgc|,
 *     [SIGN] = -1 when dgc.R > 0 (the direction is turned around, as the
 *     reference does), +1 otherwise; [FOUND] = 0; [ROUND] = 1 when
 *     |dgc.R| <= 1e-10 |E0| (the energy test carries no information; the
 *     caller decides that step itself).  scratch: 2 * min(ceil(n/256), 1024).
 *   fea_ls_energy_volume / _pressure: out[k] (+)= the group's energy (or
 *     p V of the face group) at gc + SIGN 2^-(k0+k) dgc, k < FEA_LS_M;
 *     scratch: fea_ls_scratch_len(ne).
 *   fea_ls_select: the first k of the ladder with
 *     E[k] <= E0 + c1 DE 2^-(k0+k) and 2^-(k0+k) SMAX <= max_step sets
 *     [ALPHA] = SIGN 2^-(k0+k), [ENEW] = E[k], [FOUND] = 1 and adds
 *     ALPHA dgc to gc; a step below 1e-12 sets [FOUND] = -1.  Nothing
 *     happens once FOUND != 0 or ROUND != 0.
 * ------------------------------------------------------------------------- */
#define FEA_LS_M 8
#define FEA_LS_DE 0
#define FEA_LS_E0 1
#define FEA_LS_SMAX 2
#define FEA_LS_SIGN 3
#define FEA_LS_ALPHA 4
#define FEA_LS_ENEW 5
#define FEA_LS_FOUND 6
#define FEA_LS_ROUND 7
#define FEA_LS_NSTATE 8
int32_t fea_ls_ladder_len(void);
int64_t fea_ls_scratch_len(int64_t n_items);
int fea_ls_prepare(int64_t n, const double* dgc_dev, const double* R_dev, const double* e0_dev,
                   double* state_dev, double* scratch_dev, int64_t scratch_len, cudaStream_t stream);
int fea_ls_energy_volume(const fea_nodes_t* nodes, const fea_group_t* group, double mu, double kappa,
                         const double* gc_dev, const double* dgc_dev, const double* state_dev, int32_t k0,
                         int32_t accumulate, double* out_dev, double* scratch_dev, int64_t scratch_len,
                         cudaStream_t stream);
int fea_ls_energy_pressure(const fea_nodes_t* nodes, const fea_group_t* faces, double p, const double* Xi_dev,
                           const double* gc_dev, const double* dgc_dev, const double* state_dev, int32_t k0,
                           int32_t accumulate, double* out_dev, double* scratch_dev, int64_t scratch_len,
                           cudaStream_t stream);
int fea_ls_select(int64_t n, const double* E_dev, int32_t k0, double c1, double max_step, double* state_dev,
                  const double* dgc_dev, double* gc_dev, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Explicit central difference (lumped mass), one element group, no loads.
 * One reference time step (dynamic_explicit.py:103-117) is
 *   vh += dt a;  u += dt vh;  a = minv * (-f_int(u));  v = (vh_new + vh_old)/2.
 * init != 0: on entry u = u_0 and v = v_0; a_0 and vh_{-1/2} = v_0 - dt/2 a_0
 *            are computed first (dynamic_explicit.py:80-91).
 * init == 0: on entry u = u_k, vh = vh_{k-1/2}, a = a_k.
 * Runs `steps` steps and leaves u, vh, a, v at the final step.
 * fp32 != 0 evaluates the element force in FP32 with FP64 nodal sums.
 * work_dev: fea_explicit_work_len(nodes) doubles, 16-byte aligned (a second
 * u buffer and two node-major copies of the coordinates and u, which the
 * element math reads with 16-byte loads).
 * ------------------------------------------------------------------------- */
int64_t fea_explicit_work_len(const fea_nodes_t* nodes);

/* One stage of the same central-difference step around a residual R that
 * the caller assembles (all element groups and loads: the reference's
 * assemble_force call inside its loop, dynamic_explicit.py:80-117), n reduced DOFs:
 *   stage 0 (before the force pass): vhp = vh; vh += dt a; u += dt vh
 *   stage 1 (R = reduced residual at u): a = -minv R; v = (vh + vhp)/2
 *   stage 2 (start, R at u_0, v = v_0): a = -minv R; vh = v - dt/2 a
 * Pointers not used by a stage may be null. */
int fea_explicit_stage(int64_t n, int32_t stage, double dt, const double* minv_dev, const double* R_dev,
                       double* u_dev, double* vh_dev, double* vhp_dev, double* a_dev, double* v_dev,
                       cudaStream_t stream);
int fea_explicit_run(const fea_nodes_t* nodes, const fea_group_t* group, double mu, double kappa,
                     const double* minv_dev, double dt, int64_t steps, int32_t fp32, int32_t init,
                     double* u_dev, double* vh_dev, double* a_dev, double* v_dev,
                     double* work_dev, int64_t work_len, cudaStream_t stream);

/* ---------------------------------------------------------------------------
 * Adjoint (sensitivities of the equilibrium; no kernel counterpart in the
 * reference, which differentiates its torch graph: tests/gradient_test/
 * test_grad.py:87-99).
 *   fea_adjoint_vjp_volume: for the adjoint field lam [N,3] (all nodes,
 *     zero on Dirichlet DOFs) adds d(lam . R_e)/dX [N,3] to dX_dev (every
 *     node, constrained ones included) and writes d(lam . R_e)/dmu to
 *     dmu_dev[0].  scratch: fea_reduce_scratch_len(ne) doubles.
 *   fea_adjoint_hvp_pressure: adds p d2V/dx2 v (all nodes) to out_dev, the
 *     X-derivative of v . (p dV/dx) of a pressure face group.
 * ------------------------------------------------------------------------- */
int fea_adjoint_vjp_volume(const fea_nodes_t* nodes, const fea_group_t* group, double mu, double kappa,
                           const double* gc_dev, const double* lam_dev, double* dX_dev, double* dmu_dev,
                           double* scratch_dev, int64_t scratch_len, cudaStream_t stream);
int fea_adjoint_hvp_pressure(const fea_nodes_t* nodes, const fea_group_t* faces, double p,
                             const double* Xinst_dev, const double* gc_dev, const double* v_dev,
                             double* out_dev, cudaStream_t stream);

/* Library version and the number of kernels this library has launched
 * (a host-side counter, for instrumentation). */
int32_t fea_version(void);
int64_t fea_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* FEA_B200_H */
