/*
 * fem_b200.h -- C ABI of libfem_b200, the B200 (sm_100a) matrix-free mass
 * operator behind the fe-demo-cpp API.
 *
 * Plain C: pointers and sizes only, no C++ or torch types.  Every function
 * returns a status (FEM_B200_SUCCESS = 0); on failure fem_b200_last_error()
 * returns the message of the calling thread's last failure.  The C++ drop-in
 * (the headers under include/fem/) turns FEM_B200_ERROR_ARGUMENT into
 * std::invalid_argument and every other failure into std::runtime_error,
 * the exception split of the reference.
 *
 * Memory: "device" arrays are CUDA global memory of the current device,
 * "host" arrays are ordinary (preferably pinned) host memory.  A `stream`
 * argument is a cudaStream_t (NULL = the legacy default stream); device work
 * is asynchronous on it, like the reference's CUDA restriction
 * (include/cuda/cuda-elem-restriction.hpp:106-111).
 *
 * Layouts are the reference's:
 *   L-vector   node n, component k at offsets[...] + k*comp_stride
 *   E-vector   E[(k*elem_size + i)*num_elem + e]      (include/elem-restriction.hpp:49-51)
 *   Q-vector   [comp][q][e]; Grad output [d][comp][q][e]  (include/tensor-contract.hpp:30-33)
 *   qdata      backend-strided [q][e]                  (include/elem-restriction.hpp:53-56)
 * Local nodes and quadrature points are lexicographic with x fastest.
 */
#ifndef FEM_B200_H
#define FEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define FEM_B200_SUCCESS 0
#define FEM_B200_ERROR_ARGUMENT 1    /* bad size / index / mode (std::invalid_argument) */
#define FEM_B200_ERROR_CUDA 2        /* a CUDA call or a device status failed */
#define FEM_B200_ERROR_UNSUPPORTED 3 /* valid, but not on the device path (no CPU fallback) */
#define FEM_B200_NOT_READY 4         /* fem_b200_server_wait: not finished within the timeout */

/* ---- enums, numbered as the reference's ---------------------------------- */
/* ContractMode, include/transpose-mode.hpp:13 */
#define FEM_B200_NOTRANSPOSE 0
#define FEM_B200_TRANSPOSE 1
/* EvalMode, include/eval-mode.hpp:11 */
#define FEM_B200_EVAL_NONE 0
#define FEM_B200_EVAL_INTERP 1
#define FEM_B200_EVAL_GRAD 2
#define FEM_B200_EVAL_WEIGHT 3
/* QuadMode, include/basis.hpp:21 */
#define FEM_B200_QUAD_GAUSS 0
#define FEM_B200_QUAD_GAUSS_LOBATTO 1
/* fem::cuda::ScatterMode, include/cuda/cuda-elem-restriction.hpp:10-21 */
#define FEM_B200_SCATTER_ATOMIC 0
#define FEM_B200_SCATTER_DETERMINISTIC 1
/* Device QFunctions (the host side matches fem::qfunctions by pointer) */
#define FEM_B200_QF_APPLY_MASS 0        /* include/qfunctions/mass.hpp:45-51: component 0 only */
#define FEM_B200_QF_APPLY_MASS_VECTOR 1 /* every component: v_k = qdata * u_k (no reference counterpart) */
/* Kernel variants of the fused 3D mass apply (fem_b200_mass_set_kernel) */
#define FEM_B200_KERNEL_AUTO 0      /* the autotuned variant for the shape (fem_b200_mass_autotune), else a measured per-order default (3D, Q = P+1: ELEMENT at P <= 3, PIPELINED at P = 6 with a centro-symmetric basis; SIMPLE otherwise) */
#define FEM_B200_KERNEL_SIMPLE 1    /* one CTA per 8-element tile, one element per thread */
#define FEM_B200_KERNEL_PIPELINED 2 /* persistent CTAs, next tile staged by bulk copies during this one */
#define FEM_B200_KERNEL_PAIRED 3    /* one CTA per 16 elements, two adjacent elements per thread */
#define FEM_B200_KERNEL_PREFETCH 4  /* persistent CTAs, qdata bulk-copied two tiles ahead, offsets/u one ahead */
#define FEM_B200_KERNEL_OCCUPANCY 5 /* as SIMPLE, registers capped for up to 5 resident CTAs per SM */
#define FEM_B200_KERNEL_NARROW 6    /* half-tile CTAs of 4 elements: twice the registers a thread (high order) */
#define FEM_B200_KERNEL_ELEMENT 7   /* one element per thread in registers (P <= 3); the CTA's qdata and offsets bulk-copied into shared memory first */

typedef struct fem_b200_restriction_s *fem_b200_restriction;
typedef struct fem_b200_basis_s *fem_b200_basis;
typedef struct fem_b200_mass_s *fem_b200_mass;
typedef struct fem_b200_batch_s *fem_b200_batch;
typedef struct fem_b200_server_s *fem_b200_server;

/* Message of this thread's last failure ("" if none). */
const char *fem_b200_last_error(void);
/* Library version, major*10000 + minor*100 + patch. */
int fem_b200_version(void);
/* Number of visible CUDA devices (0 without a usable GPU; never fails). */
int fem_b200_device_count(void);

/* ========================================================================= */
/* Host set-up (no GPU needed)                                                */
/* ========================================================================= */

/* Gauss-Legendre points/weights on [-1,1], Q >= 1.
 * Replaces fem::gauss_legendre_quadrature, src/basis.cpp:16-68. */
int fem_b200_gauss_legendre(int Q, double *x, double *w);

/* Gauss-Lobatto points on [-1,1] (ascending), Q >= 2; w may be NULL.
 * Replaces fem::gauss_lobatto_points, src/basis.cpp:81-144. */
int fem_b200_gauss_lobatto(int Q, double *x, double *w);

/* Lagrange interpolation / derivative matrices [M][P] of the basis on
 * `nodes` (P) evaluated at `pts` (M).
 * Replaces fem::lagrange_basis_matrix, src/basis.cpp:156-186. */
int fem_b200_lagrange_basis_matrix(int P, const double *nodes, int M, const double *pts, double *interp,
                                   double *grad);

/* 1D data of the tensor-product H1 Lagrange basis (GLL nodes): q_ref[Q],
 * q_weight[Q], interp[Q*P], grad[Q*P]; dim 1..3, num_comp 1..3, P >= 2, Q >= 1.
 * Replaces fem::TensorBasis::create_tensor_H1_lagrange, src/basis.cpp:202-228. */
int fem_b200_tensor_h1_lagrange(int dim, int num_comp, int P, int Q, int quad_mode, double *q_ref, double *q_weight,
                                double *interp, double *grad);

/* Validation of an offset restriction (n_offsets = entries given).
 * Replaces the checks of fem::elem_restriction_create, src/elem-restriction.cpp:102-138. */
int fem_b200_restriction_check_offset(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size,
                                      const int *offsets, int64_t n_offsets);

/* Validation of a strided restriction; strides NULL = backend strides
 * {num_elem, elem_size*num_elem, 1}.
 * Replaces the checks of fem::elem_restriction_create_strided, src/elem-restriction.cpp:155-204. */
int fem_b200_restriction_check_strided(int num_elem, int elem_size, int num_comp, int l_size, const int *strides);

/* Transpose map (CSR inverse of the offsets) on the host.  Sizes: l_vec_indices
 * and t_offsets at least l_size and l_size+1, t_indices num_elem*elem_size;
 * *num_nodes receives the number of used L-nodes.
 * Replaces fem::cuda::build_transpose_map, src/cuda/cuda-elem-restriction.cu:149-177. */
int fem_b200_transpose_map(int num_elem, int elem_size, int l_size, const int *offsets, int *l_vec_indices,
                           int *t_offsets, int *t_indices, int *num_nodes);

/* ========================================================================= */
/* Element restriction on the device                                          */
/* ========================================================================= */

/* Offset restriction from host offsets [num_elem][elem_size]; validated as
 * above, uploaded once.  SCATTER_DETERMINISTIC also builds the transpose map.
 * Replaces fem::cuda::elem_restriction_create, src/cuda/cuda-elem-restriction.cu:188-215. */
int fem_b200_restriction_create_offset(int num_elem, int elem_size, int num_comp, int comp_stride, int l_size,
                                       const int *offsets, int scatter_mode, fem_b200_restriction *out);

/* Strided restriction; strides NULL = backend strides.
 * Replaces fem::cuda::elem_restriction_create on a strided restriction. */
int fem_b200_restriction_create_strided(int num_elem, int elem_size, int num_comp, int l_size, const int *strides,
                                        fem_b200_restriction *out);

int fem_b200_restriction_destroy(fem_b200_restriction r);

/* Sizes of a restriction (any pointer may be NULL). */
int fem_b200_restriction_sizes(fem_b200_restriction r, int *num_elem, int *elem_size, int *num_comp, int *l_size,
                               int64_t *e_size);

/* Device transpose map (deterministic offset restrictions): copies it into
 * host arrays sized as for fem_b200_transpose_map. */
int fem_b200_restriction_transpose_map(fem_b200_restriction r, int *l_vec_indices, int *t_offsets, int *t_indices,
                                       int *num_nodes);

/* NoTranspose: out (device, e_size) = gather of in (device, l_size).
 * Transpose:   out (device, l_size) += scatter of in (device, e_size).
 * Replaces fem::cuda::elem_restriction_apply, src/cuda/cuda-elem-restriction.cu:230-273,
 * and fem::elem_restriction_apply, src/elem-restriction.cpp:34-83. */
int fem_b200_restriction_apply(fem_b200_restriction r, int t_mode, const double *in, int64_t n_in, double *out,
                               int64_t n_out, void *stream);

/* mult (device, l_size) = E^T(E 1), overwritten.
 * Replaces fem::elem_restriction_get_multiplicity, src/elem-restriction.cpp:215-227. */
int fem_b200_restriction_multiplicity(fem_b200_restriction r, double *mult, int64_t n, void *stream);

/* ========================================================================= */
/* Tensor basis on the device                                                 */
/* ========================================================================= */

int fem_b200_basis_create(int dim, int num_comp, int P, int Q, int quad_mode, fem_b200_basis *out);

/* A device basis from explicit 1D data (q_weight[Q], interp[Q*P], grad[Q*P]),
 * e.g. the arrays of a TensorBasis the caller built or changed itself
 * (include/basis.hpp:28-40 is a plain aggregate). */
int fem_b200_basis_create_from(int dim, int num_comp, int P, int Q, const double *q_weight, const double *interp,
                               const double *grad, fem_b200_basis *out);
int fem_b200_basis_destroy(fem_b200_basis b);

/* v (device) = basis action on u (device) for num_elem elements.  Interp and
 * Grad in both directions, Weight NoTranspose (u ignored).  v is overwritten
 * in every mode (the reference's Grad Transpose adds into a stale v,
 * src/tensor-contract.cpp:115-145; on a zeroed v both agree).
 * Replaces fem::tensor_basis_apply, src/tensor-contract.cpp:207-222. */
int fem_b200_basis_apply(fem_b200_basis b, int num_elem, int t_mode, int eval_mode, const double *u, int64_t n_u,
                         double *v, int64_t n_v, void *stream);

/* Allocation-free form of fem_b200_basis_apply (no counterpart in the
 * reference).  fem_b200_basis_apply keeps its pass buffers in device memory
 * that it allocates with cudaMalloc on its first call and whenever num_elem
 * grows.  Some callers cannot allow that: code that is being captured into a
 * CUDA graph (cudaMalloc is not permitted during a global-mode capture), hosts
 * whose device memory is owned by another allocator or a fixed budget, and
 * loops that must not stall on the allocator.  This entry point takes the same
 * arguments and computes the same result without allocating.  Dimension 3 runs
 * the fused one-pass kernels, which use no scratch (no size limit).  Other
 * shapes run the generic passes with their buffers in a fixed array compiled
 * into the library: 2,097,152 doubles (16 MiB), which every GPU that loads the
 * library holds until the process exits.  A call needing more
 * (2 * num_comp * max(P,Q)^dim * num_elem doubles for dim 2, or dim 3 without a
 * fused kernel) fails with FEM_B200_ERROR_ARGUMENT; split the elements over
 * several calls.  The first call on a device that uses the array looks up its
 * device address (set-up that may load the module), so make that first call
 * before any stream capture.  All calls
 * share the one array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.  Each pass
 * overwrites the scratch it uses, so nothing needs clearing between calls. */
int fem_b200_basis_apply_static(fem_b200_basis b, int num_elem, int t_mode, int eval_mode, const double *u,
                                int64_t n_u, double *v, int64_t n_v, void *stream);

/* ========================================================================= */
/* Device memory and raw launchers                                            */
/* (caller-owned device arrays; used by the C++ drop-in's DeviceArray and     */
/* fem::cuda restriction, which own their index arrays like the reference's)  */
/* ========================================================================= */

/* cudaMalloc / cudaFree / copies (kind 0 H2D, 1 D2H, 2 D2D; H2D and D2H
 * synchronise `stream`) / zero fill / stream synchronise.
 * Replace the CUDA calls of fem::cuda::DeviceArray, include/cuda/device-array.hpp:18-95. */
int fem_b200_malloc(void **ptr, size_t bytes);
int fem_b200_free(void *ptr);
int fem_b200_memcpy(void *dst, const void *src, size_t bytes, int kind, void *stream);
int fem_b200_memset_zero(void *ptr, size_t bytes, void *stream);
int fem_b200_synchronize(void *stream);

/* Device limits: name (NUL-terminated, name_len bytes), ints[6] = {cc_major,
 * cc_minor, sm_count, warp_size, max_threads_per_block, regs_per_block},
 * sizes[5] = {shared_mem_per_block, ..._optin, shared_mem_per_sm,
 * total_global_mem, free_global_mem}.
 * Replaces fem::cuda::device_info, src/cuda/device-info.cpp:28-56. */
int fem_b200_device_info(int device, char *name, int name_len, int *ints, int64_t *sizes);

/* Restriction kernels on caller-owned device arrays (offsets [num_elem][elem_size]):
 * gather (e_out overwritten), atomic scatter-add, transpose-map (deterministic)
 * scatter-add, strided gather (t_mode 0) / scatter-add (t_mode 1) with host strides[3].
 * Replace the five kernels of src/cuda/cuda-elem-restriction.cu:37-127. */
int fem_b200_offset_gather(int num_elem, int elem_size, int num_comp, int comp_stride, const int *offsets,
                           const double *l_in, double *e_out, void *stream);
int fem_b200_offset_scatter_add(int num_elem, int elem_size, int num_comp, int comp_stride, const int *offsets,
                                const double *e_in, double *l_out, void *stream);
int fem_b200_transpose_scatter_add(int num_nodes, int num_elem, int elem_size, int num_comp, int comp_stride,
                                   const int *l_vec_indices, const int *t_offsets, const int *t_indices,
                                   const double *e_in, double *l_out, void *stream);
int fem_b200_strided_apply(int t_mode, int num_elem, int elem_size, int num_comp, const int *strides,
                           const double *in, double *out, void *stream);

/* v (+)= t(j,b) u over one tensor mode, device arrays (t is J x B row-major,
 * read transposed for t_mode = TRANSPOSE).
 * Replaces fem::tensor_contract_apply, src/tensor-contract.cpp:35-59. */
int fem_b200_contract(int64_t A, int B, int64_t C, int J, const double *t, int t_mode, int add, const double *u,
                      double *v, void *stream);

/* The two mass QFunctions pointwise over Q points (device arrays, [size][Q]):
 * v = qdata * u, and qdata = det(J) * w with J [dim][dim][Q].
 * Replace apply_mass / build_mass, include/qfunctions/mass.hpp:17-51, when
 * run through qfunction_apply. */
int fem_b200_qfunction_apply_mass(int64_t Q, const double *u, const double *qdata, double *v, void *stream);
int fem_b200_qfunction_build_mass(int dim, int64_t Q, const double *J, const double *w, double *qdata, void *stream);

/* ========================================================================= */
/* Mass operator                                                              */
/* ========================================================================= */

/* qdata (device, Q^dim*num_elem, [q][e]) = det(dx/dX) * w from the coordinate
 * L-vector x (device) of restriction rx (num_comp = dim) and basis bx
 * (num_comp = dim): the build operator of the reference, fused.
 * Replaces operator_apply on the build_mass operator, src/operator.cpp:148-182
 * with include/qfunctions/mass.hpp:17-40. */
int fem_b200_mass_build(fem_b200_restriction rx, fem_b200_basis bx, const double *x, int64_t n_x, double *qdata,
                        int64_t n_qdata, void *stream);

/* Mass operator v = E^T B^T D B E u on restriction ru / basis bu with the
 * backend-strided qdata (device, [q][e]); the plan keeps its own copy of
 * qdata (laid out for the kernel), as the reference Operator copies passive
 * vectors (include/operator.hpp:33-47).  qf: FEM_B200_QF_APPLY_MASS or
 * FEM_B200_QF_APPLY_MASS_VECTOR.  The scatter mode is ru's.
 * Replaces operator_create + operator_set_field on the mass QFunction,
 * src/operator.cpp:21-117. */
int fem_b200_mass_create(fem_b200_restriction ru, fem_b200_basis bu, const double *qdata, int64_t n_qdata, int qf,
                         fem_b200_mass *out);
int fem_b200_mass_destroy(fem_b200_mass op);

/* v (device, l_size) = M u (device, l_size): zeroed, then summed into.
 * Replaces fem::operator_apply, src/operator.cpp:148-182. */
int fem_b200_mass_apply(fem_b200_mass op, const double *u, int64_t n_u, double *v, int64_t n_v, void *stream);

/* v += M u (device arrays), no zeroing. */
int fem_b200_mass_apply_add(fem_b200_mass op, const double *u, int64_t n_u, double *v, int64_t n_v, void *stream);

/* Host-memory form of fem_b200_mass_apply: copies u in, applies, copies v out
 * through plan-owned device buffers, and returns with v_host written.  The
 * call a host std::vector user makes (operator_apply(op, in, out)).  With the
 * atomic scatter and at least 1024 tiles of elements the copies are
 * pipelined: u comes in by node span on a plan-owned stream, the kernels run
 * per element chunk on `stream` as their span arrives, and v goes out on a
 * second plan-owned stream as each range becomes final, so the two PCIe
 * directions overlap (page-locked or pageable host memory; the plan is not
 * to be used from two threads at once).  Otherwise: copy in, apply, copy out
 * on `stream`. */
int fem_b200_mass_apply_host(fem_b200_mass op, const double *u_host, int64_t n_u, double *v_host, int64_t n_v,
                             void *stream);

/* Chunks of the host-memory apply's pipeline: 0 the default (about 24), 1 no
 * pipelining (copy in, apply, copy out), n >= 2 about n chunks (each at least
 * 512 tiles).  Takes effect at the next fem_b200_mass_apply_host. */
int fem_b200_mass_set_host_chunks(fem_b200_mass op, int chunks);

/* Number of kernel launches one fem_b200_mass_apply makes, the plan's
 * element-tile size, device footprint in bytes and the kernel variant in use
 * (any pointer may be NULL). */
int fem_b200_mass_info(fem_b200_mass op, int *launches_per_apply, int *tile_elems, int64_t *device_bytes,
                       int *kernel_variant);

/* Select the fused kernel variant (FEM_B200_KERNEL_*).  PIPELINED and PAIRED
 * are dim-3 kernels; each is FEM_B200_ERROR_UNSUPPORTED where its shared
 * memory or thread count does not fit a CTA. */
int fem_b200_mass_set_kernel(fem_b200_mass op, int variant);

/* Autotuner: run every fused kernel variant the plan supports `reps` times
 * on (u, v) -- device arrays of l_size; v is overwritten as scratch -- keep
 * the fastest for this plan (CUDA-event timing on `stream`) and remember it
 * for later plans with the same device, dim, P, Q, components, scatter mode
 * and log2(num_elem) (FEM_B200_KERNEL_AUTO then starts from it).  *chosen
 * receives the variant, *best_ms its time per apply (either may be NULL).
 * Synchronises the stream. */
int fem_b200_mass_autotune(fem_b200_mass op, const double *u, int64_t n_u, double *v, int64_t n_v, int reps,
                           int *chosen, float *best_ms, void *stream);

/* Assembled diagonal of the mass operator, diag (device, l_size), overwritten:
 * diag_i = sum over elements and quadrature points of qdata * (phi_i)^2, one
 * fused kernel (interp^T with the squared 1D matrix applied to qdata, then
 * the scatter-add); every component of a vector plan gets the same diagonal.
 * The Jacobi preconditioner of fem_b200_mass_solve.  No reference counterpart
 * (its survey verifies it against e_i^T M e_i on small meshes). */
int fem_b200_mass_diagonal(fem_b200_mass op, double *diag, int64_t n, void *stream);

/* Solve M u = f (device arrays, l_size) by Jacobi-preconditioned CG from u = 0
 * (Chronopoulos-Gear form: one grid reduction point per iteration, scalars kept
 * on the device, the host checking convergence between batches of queued
 * iterations; reductions in FP64, in a fixed order).
 *   FEM_B200_SOLVE_FP64     FP64 PCG to ||r|| <= rtol ||f|| (recursive residual);
 *   FEM_B200_SOLVE_FP32_IR  FP64 iterative refinement: r = f - M u in FP64, a
 *                           correction from FP32 PCG (FP32 qdata, vectors and
 *                           fused apply; FP64 reductions) on r / ||r||, each
 *                           inner solve to what the target still needs (not
 *                           below 5e-6), until ||f - M u|| <= rtol ||f||;
 *   FEM_B200_SOLVE_BF16_IR  the same refinement with a BF16-storage inner PCG:
 *                           BF16 qdata and Krylov vectors r, p, s, FP32
 *                           x, dinv, M z and arithmetic, FP64 reductions; each
 *                           inner solve to at most 1e-2 (BF16's attainable
 *                           level), so more refinement steps.
 * max_iter bounds the CG iterations (all inner ones for the _IR forms).  Outputs (any
 * may be NULL): total CG iterations, refinement steps, and the true FP64
 * relative residual ||f - M u|| / ||f||.  Plans with the deterministic scatter
 * reproduce every bit of u from run to run.  Synchronises the stream.  Plans of the reference apply_mass with num_comp > 1 are
 * singular (components 1.. are left out) and return FEM_B200_ERROR_UNSUPPORTED.
 * No reference counterpart (the reference has no solver). */
#define FEM_B200_SOLVE_FP64 0
#define FEM_B200_SOLVE_FP32_IR 1
#define FEM_B200_SOLVE_BF16_IR 2
int fem_b200_mass_solve(fem_b200_mass op, const double *f, int64_t n_f, double *u, int64_t n_u, double rtol,
                        int max_iter, int precision, int *iterations, int *refinements, double *rel_residual,
                        void *stream);

/* ---- batched apply over many meshes (no reference counterpart) ------------
 * One batch = many mass operators (any dim, P, Q, num_comp; atomic scatter)
 * applied together: v_i = M_i u_i for all i, as ONE captured CUDA graph.
 * Two forms: the one-launch form -- a single persistent kernel taking work
 * items from a ticket: the zeroing of every v_i, then the tiles of every
 * class, heaviest first, several low-order tiles a block at once; it covers
 * dim 2 and 3, P = 2..6, Q = P + 1 with one basis a P -- and the per-class
 * form (a kernel zeroing every v_i, then one kernel per class of equal dim,
 * P, Q, components and basis over a device table of (mesh, tile) pairs,
 * classes on parallel graph branches).  The operators must outlive the
 * batch. */
#define FEM_B200_BATCH_AUTO 0       /* the one-launch form where it applies, unless autotuning preferred the other */
#define FEM_B200_BATCH_CLASSES 1    /* one kernel per class */
#define FEM_B200_BATCH_PERSISTENT 2 /* one persistent launch (FEM_B200_ERROR_UNSUPPORTED where it does not apply) */
/* Precision and layout as below.
 * Precision FEM_B200_PRECISION_FP32 applies FP32 u_i / v_i with FP32 qdata
 * (converted once from each operator's FP64 qdata). */
#define FEM_B200_PRECISION_FP64 0
#define FEM_B200_PRECISION_FP32 1
int fem_b200_batch_create(const fem_b200_mass *ops, int num_ops, int precision, fem_b200_batch *out);
/* Device pointers u[i], v[i] (double or float per the batch's precision, each
 * of operator i's l_size), written into the batch's device descriptor table
 * in `stream` order; the captured graph reads them at launch, so rebinding
 * needs no new capture. */
int fem_b200_batch_bind(fem_b200_batch b, const void *const *u, void *const *v, void *stream);
/* v_i = M_i u_i for every i.  use_graph != 0: launch the captured graph
 * (captured on the first call, from streams of the batch's own); 0: the same
 * kernels launched one by one into `stream`. */
int fem_b200_batch_apply(fem_b200_batch b, int use_graph, void *stream);
/* Time each class's schedules (one CTA per tile; a persistent grid of
 * resident CTAs) over `reps` launches and keep the faster; then time the
 * graph with 1, 2 and 4 parallel branches and keep the fastest capture; in
 * mode FEM_B200_BATCH_AUTO also the one-launch form against that graph, and
 * keep the faster.  Leaves v_i = M_i u_i.  Synchronises the stream. */
int fem_b200_batch_autotune(fem_b200_batch b, int reps, void *stream);
/* Choose the batch's form (FEM_B200_BATCH_*); drops the captured graph. */
int fem_b200_batch_set_mode(fem_b200_batch b, int mode);
/* Synchronise `stream` and report a bounded wait of the one-launch kernel
 * that ran out as FEM_B200_ERROR_CUDA. */
int fem_b200_batch_check(fem_b200_batch b, void *stream);
/* Any output may be NULL: classes, tiles, sum of l_size (DoFs), kernels per
 * graph launch, classes on the persistent schedule, parallel graph branches. */
int fem_b200_batch_info(fem_b200_batch b, int *num_classes, int64_t *total_tiles, int64_t *total_dofs,
                        int *graph_kernels, int *persistent_classes, int *graph_branches);
int fem_b200_batch_destroy(fem_b200_batch b);

/* ---- served solves (no reference counterpart) ------------------------------
 * A request loop over a device-memory budget: each request is one mass solve
 * M u = f (vector mass, num_comp 1..3) on its own mesh.  Requests are admitted
 * in arrival order as soon as one of `slots` workers is free and the
 * request's device-memory estimate (mesh, qdata, Krylov vectors, set-up
 * temporaries) fits in what the budget has left; admitted requests keep
 * their data resident until they finish and run concurrently, each worker on
 * its own CUDA stream with stream-ordered allocation, so their kernels
 * overlap.  A result does not depend on the mix it ran in (bitwise so with
 * the deterministic scatter). */
#define FEM_B200_REQUEST_BOX 0  /* box [0,1]^dim generated on the device */
#define FEM_B200_REQUEST_MESH 1 /* offsets / coordinates / f from the host */
typedef struct {
  int kind;
  int dim, P, Q, num_comp;
  /* BOX: elements per direction, interior vertices moved by U[-perturb h,
   * perturb h] per coordinate, f ~ U[-1, 1]; mesh and f from `seed` */
  int shape[3];
  double perturb;
  uint64_t seed;
  /* MESH (host arrays, valid until the request completes): offsets
   * [num_elem][P^dim], coordinates blocked [dim][num_nodes], f blocked
   * [num_comp][num_nodes] */
  int num_elem, num_nodes;
  const int *offsets;
  const double *coords;
  const double *f;
  /* the solve: as fem_b200_mass_solve */
  double rtol;
  int max_iter, precision, scatter_mode;
  /* optional host outputs (num_comp * num_nodes doubles, valid until the
   * request completes): the solution, and the right-hand side used */
  double *u_out;
  double *f_out;
} fem_b200_request;
typedef struct {
  int status; /* FEM_B200_SUCCESS or the error of this request (message) */
  int iterations, refinements;
  double rel_residual; /* ||f - M u|| / ||f||, FP64 */
  double t_submit, t_start, t_end; /* seconds on the server's clock */
  int64_t dofs;         /* num_comp * num_nodes */
  int64_t device_bytes; /* reserved from the budget while it ran */
  char message[256];
} fem_b200_result;
int fem_b200_server_create(int slots, int64_t hbm_budget_bytes, fem_b200_server *out);
/* Queue a request; ARGUMENT error if it alone exceeds the budget. */
int fem_b200_server_submit(fem_b200_server s, const fem_b200_request *req, int64_t *id);
/* Wait up to timeout_s seconds (< 0: no limit) for request `id`; on success
 * the result is written and the id forgotten; FEM_B200_NOT_READY on timeout. */
int fem_b200_server_wait(fem_b200_server s, int64_t id, double timeout_s, fem_b200_result *result);
/* Any output may be NULL. */
int fem_b200_server_stats(fem_b200_server s, int64_t *submitted, int64_t *completed, int *running, int64_t *pending,
                          int64_t *bytes_in_use, int64_t *bytes_peak);
/* Finishes every queued request, then stops the workers. */
int fem_b200_server_destroy(fem_b200_server s);

/* operator_apply in reduced storage (src/operator.cpp:148-182 is FP64 only):
 * _f32: u, v and qdata in FP32 (qdata converted once from the plan's FP64
 * copy), FP32 arithmetic; _bf16: u and qdata in BF16 (bfloat16 bit patterns,
 * 2 bytes an entry), FP32 arithmetic and FP32 v.  v is overwritten; both
 * scatter modes; device pointers, `stream` order. */
int fem_b200_mass_apply_f32(fem_b200_mass op, const float *u, int64_t n_u, float *v, int64_t n_v, void *stream);
int fem_b200_mass_apply_bf16(fem_b200_mass op, const void *u_bf16, int64_t n_u, float *v, int64_t n_v,
                             void *stream);

/* operator_apply with its 1D contractions on the tensor cores (tcgen05.mma,
 * TF32 inputs, FP32 accumulation; src/operator.cpp:148-182 computes in FP64
 * with scalar loops, src/tensor-contract.cpp:35-91).  3D plans with P = 6..8,
 * Q = P..8 and atomic scatter (else FEM_B200_ERROR_UNSUPPORTED).
 * _f32_tc: u, v, qdata FP32; split = 1 stages every operand as two TF32
 * parts (3xTF32: FP32-level accuracy), split = 0 as one (relative rounding
 * 2^-11 per contraction).  _bf16_tc: u and qdata BF16, one TF32 part.  v is
 * overwritten; device pointers, `stream` order. */
int fem_b200_mass_apply_f32_tc(fem_b200_mass op, const float *u, int64_t n_u, float *v, int64_t n_v, int split,
                               void *stream);
int fem_b200_mass_apply_bf16_tc(fem_b200_mass op, const void *u_bf16, int64_t n_u, float *v, int64_t n_v,
                                void *stream);

/* Self-test of the tensor-core layer behind the _tc applies (no counterpart
 * in the reference): one M = 128, N = 16, K = 8 TF32 tcgen05.mma with the
 * operands staged as the applies stage them, read back from tensor memory;
 * writes max |D - A B^T| / max |A B^T| against the host product of the
 * TF32-rounded inputs (FP32 rounding of the sums, ~1e-7, when the
 * descriptors and layouts are right). */
int fem_b200_tc_selftest(double *max_rel_err);

/* ---- one mesh over several ranks (no reference counterpart; the reference
 * is single-process, src/operator.cpp:148-182) ---------------------------------
 * The elements are split into `world` contiguous ranges; rank `rank` holds
 * elements [e0, e1) with its nodes renumbered compactly in ascending global
 * id (l2g), applies the mass operator to them (an operator over
 * local_offsets), then sums the values of the nodes it shares with other
 * ranks.  The sum needs one exchange per apply: fem_b200_shard_pack puts the
 * shared values, for every peer, into one send buffer (peer i's segment is
 * contiguous: count_i x num_comp values from offset num_comp x (the counts
 * of peers before i)); the caller moves each segment to its peer and fills
 * the receive buffer in the same layout (NCCL send/recv, MPI, a copy);
 * fem_b200_shard_unpack_add then sets every shared value to the sum of all
 * ranks' values in rank order, from 0, so a shared node ends with the same
 * bits on every rank.  A node is owned by the lowest rank that touches it
 * (for dot products over the whole mesh).  Vectors are blocked
 * [num_comp][num_nodes]; pack / unpack take device pointers.  The set-up
 * reads the whole mesh's offsets on the host and needs no GPU. */
typedef struct fem_b200_shard_s *fem_b200_shard;
int fem_b200_shard_create(int num_elem, int elem_size, const int *offsets, int world, int rank,
                          fem_b200_shard *out);
/* Any output may be NULL.  shared_total: the sum of the peers' counts. */
int fem_b200_shard_sizes(fem_b200_shard s, int *e0, int *e1, int *num_nodes, int *num_peers,
                         int64_t *shared_total);
/* local_offsets [(e1 - e0) * elem_size], l2g [num_nodes], owned [num_nodes]
 * (1 where this rank owns the node); any may be NULL. */
int fem_b200_shard_local(fem_b200_shard s, int *local_offsets, int64_t *l2g, unsigned char *owned);
/* Peer i (ascending rank): its rank, the number of shared nodes, their local
 * indices (ascending; may be NULL). */
int fem_b200_shard_peer(fem_b200_shard s, int i, int *peer, int64_t *count, int64_t *local_idx);
int fem_b200_shard_pack(fem_b200_shard s, const double *v, int64_t n_v, int num_comp, double *send, int64_t n_send,
                        void *stream);
int fem_b200_shard_unpack_add(fem_b200_shard s, const double *recv, int64_t n_recv, int num_comp, double *v,
                              int64_t n_v, void *stream);
int fem_b200_shard_destroy(fem_b200_shard s);

/* Synchronise `stream` and report a device-side failure of the plan's kernels
 * (a bounded wait that ran out) as FEM_B200_ERROR_CUDA.  fem_b200_mass_apply_host
 * does this check itself. */
int fem_b200_mass_check(fem_b200_mass op, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* FEM_B200_H */
