/*
 * psierra_b200: C ABI of the B200 (sm_100a) Tet4/Tet10 Total-Lagrangian NeoHookean
 * element-evaluation and global-assembly library.
 *
 * Every entry point takes plain pointers and sizes, returns an int status (PSX_OK
 * on success) and never allocates device memory: the caller owns every buffer.
 * Pointers documented as "device" must be CUDA device (or managed) memory of the
 * current device; "host" pointers are ordinary host memory.  Work is enqueued on
 * the given stream and is asynchronous unless stated otherwise.
 *
 * Reference interfaces replaced (tanadul-s/psierra, file:line):
 *   psx_graph_count / psx_graph_fill / psx_csr_pattern
 *       -> utility/indexing.py:35-59 compute_element_dofs,
 *          utility/assembly.py:6-34 create_coo_sparsity_indices and the index
 *          structure of utility/assembly.py:75-76 coo_matrix(...).tocsr()
 *   psx_tet4_assemble (PSX_WANT_F)  -> domain/solid.py:230-274 assemble_internal_forces
 *          (element/tet4_total_lagrangian.py:77-139 + utility/assembly.py:79-108)
 *   psx_tet4_assemble (PSX_WANT_K)  -> domain/solid.py:280-325 assemble_tangent_stiffness_matrix
 *          (element/tet4_total_lagrangian.py:77-139 + utility/assembly.py:37-76)
 *   psx_tet4_assemble (PSX_LINEAR)  -> domain/solid.py:172-207 assemble_stiffness_matrix
 *          (element/tet4_base.py:129-136)
 *   psx_tet10_assemble              -> the same three, element/tet10_total_lagrangian.py:63-136
 *          and element/tet10_base.py:310-342
 *   psx_tet4_kv                     -> K_T(u) @ v with the assembled reference K_T
 *   psx_pcg                         -> solver/sparse_linear_solver.py:37-68
 *          ConjugateGradientSolver.solve (Jacobi-preconditioned CG)
 */
#ifndef PSIERRA_B200_H
#define PSIERRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes */
#define PSX_OK 0
#define PSX_ERR_ARG 1           /* invalid argument (null pointer, bad size) */
#define PSX_ERR_CUDA 2          /* a CUDA launch or copy failed */
#define PSX_ERR_LIMIT 3         /* mesh exceeds a documented kernel limit */

/* Assembly request bits (psx_tet4_assemble / psx_tet10_assemble `mode`) */
#define PSX_WANT_F 1            /* internal force vector f_int(u) */
#define PSX_WANT_K 2            /* tangent stiffness K_T(u) values in the CSR pattern */
#define PSX_LINEAR 4            /* small-strain stiffness from (lambda, mu); ignores u */
#define PSX_KV 8                /* matrix-free product y = K_T(u) v (psx_tet4_kv) */
#define PSX_MASS 32             /* consistent mass matrix; `lam` carries the density */

/* Precision of the element tangent (`precision`) */
#define PSX_FP64 0              /* everything in FP64, K values stored as double */
#define PSX_FP32_MIXED 1        /* f_int, det F and ln J in FP64; K_T in FP32, stored as float */

/*
 * Status block written by the element kernels (device memory, psx_status_bytes()
 * bytes, zero it before a call).  Layout: int32 n_inverted, int32 n_bad_volume,
 * int32 first_bad_key (INT32_MAX - lowest bad element index, 0 if none),
 * int32 n_not_finite, int32 iters, int32 flags, double value.  The assembly kernels
 * put the number of spin iterations of their bounded waits in `iters`.
 * An element is "bad" when its reference volume det is <= 0 (n_bad_volume) or
 * det F <= 0 (n_inverted): the two conditions on which the reference raises
 * ValueError (element/tet4_base.py:56-61, element/tet4_total_lagrangian.py:110-112).
 */
size_t psx_status_bytes(void);

/* ---- Sparsity pattern (host memory, once per mesh) ------------------------- */

/*
 * Node graph of a mesh with `npe` nodes per element (4 or 10), connectivity
 * `conn` (host, E x npe, row-major, int64, node ids in [0, N)).
 *   nbr_ptr (host, N+1): prefix sums of node degrees (distinct neighbours incl. self)
 *   inc_ptr (host, N+1): prefix sums of node -> element incidences
 * Returns PSX_ERR_LIMIT if 9 * sum(deg) does not fit int32.
 */
int psx_graph_count(const int64_t* conn, int64_t E, int npe, int64_t N,
                    int32_t* nbr_ptr, int32_t* inc_ptr);

/*
 * Fill the node graph (host): nbr (sum deg) sorted neighbour lists; inc_elem
 * (E*npe) incident elements of each node in ascending element order; inc_code
 * (E*npe): for Tet4, bits 0-1 = local index of the node in the element and bits
 * 2+7b..8+7b = rank of element node b in the node's neighbour list (ranks < 128);
 * for Tet10 the local index only.
 */
int psx_graph_fill(const int64_t* conn, int64_t E, int npe, int64_t N,
                   const int32_t* nbr_ptr, const int32_t* inc_ptr,
                   int32_t* nbr, int32_t* inc_elem, uint32_t* inc_code);

/*
 * Canonical CSR pattern of the assembled 3N x 3N matrix (host): indptr (3N+1),
 * indices (9*sum deg), identical to scipy's coo_matrix((data,(rows,cols))).tocsr()
 * index arrays for the reference's rows/cols (sorted columns, duplicates merged).
 * Row 3i+k of node i starts at 9*nbr_ptr[i] + 3*deg_i*k.
 */
int psx_csr_pattern(int64_t N, const int32_t* nbr_ptr, const int32_t* nbr,
                    int32_t* indptr, int32_t* indices);

/*
 * Per neighbour-block gather lists (host) used by the Tet10 path: for the block
 * (node i, neighbour rank r) at entry q = nbr_ptr[i] + r, blk_src[blk_ptr[q] ..
 * blk_ptr[q+1]) lists (e*npe + a)*npe + b for every element e containing node i at
 * local index a and the neighbour at local index b, in ascending element order.
 * blk_ptr has sum(deg)+1 entries, blk_src E*npe*npe.  PSX_ERR_LIMIT if E*npe*npe
 * does not fit int32.
 */
int psx_block_lists(const int64_t* conn, int64_t E, int npe, int64_t N,
                    const int32_t* nbr_ptr, const int32_t* nbr,
                    int32_t* blk_ptr, int32_t* blk_src);

/* ---- Gather plan (host, once per mesh) ------------------------------------- */

/*
 * Plan of the element-record / owner-gather assembly.  Items are the node pairs
 * (i < j) of the node graph and the nodes; every item lists the element slots that
 * contribute to it (ascending element order) and the items are sorted by the last
 * element they need, so the items completed by element chunk k can be gathered right
 * after chunk k has been evaluated.  Pointers marked device/host as noted.
 */
typedef struct psx_plan {
  int32_t npe;              /* nodes per element: 4 or 10 */
  int32_t n_granules;       /* ceil(n_elements / granule) */
  int64_t n_elements;
  int64_t n_nodes;
  int64_t n_pairs;          /* node pairs i < j */
  int64_t granule;          /* plan resolution in elements (power of two) */
  int64_t max_span;         /* max over items of (last - first contributing element) */
  const int32_t* conn;      /* device, E x npe int32 */
  const int32_t* pair_info; /* device, 4 per pair: pos_up, stride_up, pos_lo, stride_lo */
  const int32_t* pair_ptr;  /* device, n_pairs + 1 */
  const int32_t* pair_src;  /* device, e * 64 + local pair slot */
  const int32_t* node_info; /* device, 4 per node item: pos_diag, stride, node, 0 */
  const int32_t* node_ptr;  /* device, N + 1 */
  const int32_t* node_src;  /* device, e * 16 + local node index */
  const int32_t* pair_gptr; /* host, n_granules + 1: pair items ready in each granule */
  const int32_t* node_gptr; /* host, n_granules + 1 */
  int32_t tile;             /* elements per element task (psx_task_fill) */
  int32_t lag;              /* granules between an element tile and the gathers it completes */
  int32_t tile_items;       /* items per gather task */
  int32_t blocks_per_sm;    /* persistent blocks launched per SM; 0 = the kernel's register target */
  int64_t n_tasks_k;        /* task queue with pair tiles (any request involving K) */
  int64_t n_tasks_f;        /* task queue without pair tiles (f only) */
  const int32_t* tasks_k;   /* device, 4 per task: kind, granule, begin, end */
  const int32_t* tasks_f;   /* device */
  const int32_t* btiles_k;  /* device, n_granules: gather tiles per granule in tasks_k */
  const int32_t* btiles_f;  /* device, n_granules: gather tiles per granule in tasks_f */
  int32_t ring_slack;       /* ring granules beyond span + lag (>= 6; 0 = 6): room for tiles in flight */
  int32_t lag_f;            /* lag of tasks_f (0 = lag); `lag` is the lag of tasks_k */
  /* Tet4 tile records (psx_tile_plan_fill; required when npe == 4, device arrays) */
  int32_t tile_cap_pairs;   /* most distinct node pairs in one element tile */
  int32_t tile_cap_nodes;   /* most distinct nodes in one element tile */
  const uint8_t* tile_meta; /* n_tiles x psx_tile_meta_stride(tile) bytes (psx_tile_plan_fill) */
  const int32_t* pair_ptr_t; /* n_pairs + 1 */
  const int32_t* pair_src_t; /* tile * 256 + local pair, ascending tile */
  const int32_t* node_ptr_t; /* N + 1 */
  const int32_t* node_src_t; /* tile * 128 + local node, ascending tile */
  /* Warp-specialised FP32 tangent sweeps (Tet4; optional, NULL = the mixed kernel): the
     gather tasks of tasks_k (kinds 1 and 2) in queue order.  With them, f+K and K-only
     FP32 sweeps run element tiles and gathers in separate warps of one block per SM. */
  int64_t n_gtasks_k;
  const int32_t* gtasks_k;  /* device, 4 per task like tasks_k */
  /* Polls of one bounded wait of the persistent kernels before it gives up (status flag
     bit 0, which the host turns into an error; every later wait of the launch then
     returns at once).  0 = the default, 1 << 22 polls (about a second).  A small value
     lets a test make a wait run out without faulting the GPU. */
  int32_t wait_spins;
  int32_t reserved0;        /* 0 */
} psx_plan_t;

/* n_pairs = (sum deg - N) / 2 and the pair_src length E * npe (npe - 1) / 2 (host). */
int psx_plan_count(const int64_t* conn, int64_t E, int npe, int64_t N, const int32_t* nbr_ptr,
                   int64_t* n_pairs, int64_t* n_pair_src);

/*
 * Fill the plan arrays (host memory; the caller uploads the device ones):
 * pair_info (4 n_pairs), pair_ptr (n_pairs+1), pair_src (E npe (npe-1)/2),
 * pair_gptr (n_granules+1), node_info (4 N), node_ptr (N+1), node_src (E npe),
 * node_gptr (n_granules+1), max_span (1).  PSX_ERR_LIMIT if E > 2^25.
 */
int psx_plan_fill(const int64_t* conn, int64_t E, int npe, int64_t N, const int32_t* nbr_ptr,
                  const int32_t* nbr, int64_t granule, int32_t* pair_info, int32_t* pair_ptr,
                  int32_t* pair_src, int32_t* pair_gptr, int32_t* node_info, int32_t* node_ptr,
                  int32_t* node_src, int32_t* node_gptr, int64_t* max_span);

/*
 * 1 when the warp-specialised Tet4 FP32 tangent kernel can run on the current device
 * (its compiled register count matches the register split it moves between its element
 * and gather warps), else 0; FP32 tangent sweeps of a plan with gtasks_k then use the
 * mixed kernel.  No counterpart in the reference (no GPU path).
 */
int psx_tet4_split_ready(void);

/*
 * Tile plan of the Tet4 kernels (host; no counterpart in the reference, which has no
 * element tiles): the element tile of one warp (tile consecutive elements, tile <= 32,
 * a power of two; the plan's `tile`) sums the blocks its elements share in shared
 * memory and writes one record per distinct pair / node.  Inputs: conn (E x 4), the
 * element-code item lists of psx_plan_fill.  Outputs (host buffers, n_tiles =
 * ceil(E / tile)): meta (n_tiles x psx_tile_meta_stride(tile) bytes; per tile: pair and
 * node counts, then the node offsets and codes, then the pair offsets and codes, laid
 * out as psx_pattern.cpp describes), pair_ptr_t
 * (n_pairs + 1), pair_src_t (<= len pair_src), node_ptr_t (N + 1), node_src_t (<= len
 * node_src), caps[2] = {most pairs, most nodes in a tile}.  Contributions keep
 * ascending element order inside a tile and ascending tile order across tiles (a
 * fixed, reproducible summation order).
 */
int64_t psx_tile_meta_stride(int32_t tile);
int psx_tile_plan_fill(const int64_t* conn, int64_t E, int npe, int32_t tile, const int32_t* pair_ptr,
                       const int32_t* pair_src, int64_t n_pairs, const int32_t* node_ptr, const int32_t* node_src,
                       int64_t N, uint8_t* meta, int32_t* pair_ptr_t, int32_t* pair_src_t, int32_t* node_ptr_t,
                       int32_t* node_src_t, int32_t* caps);

/*
 * F-bar plan (host; Tet4Fbar, element/tet4_fbar.py:53-118, 420-459): the two-ring graph
 * of the one-ring graph nbr_ptr/nbr (sorted lists, self included; its CSR pattern is
 * psx_csr_pattern(N, nbr2_ptr, nbr2, ...)), the one-ring gather items' positions in that
 * CSR (pair_info2 4 n_pairs, node_info2 4 N, from psx_plan_fill's pair_info/node_info)
 * and, per two-ring entry, the nodes a whose patch holds both ends with the one-ring
 * entries of g_a at both ends (vol_ptr n_nbr2 + 1, vol_src 3 per entry: a, entry of
 * (a, b), entry of (a, c); a ascending).  _count gives n_nbr2 and n_vol.
 */
int psx_fbar_plan_count(int64_t N, const int32_t* nbr_ptr, const int32_t* nbr, int64_t* n_nbr2, int64_t* n_vol);
int psx_fbar_plan_fill(int64_t N, const int32_t* nbr_ptr, const int32_t* nbr, int64_t n_pairs,
                       const int32_t* pair_info, const int32_t* node_info, int32_t* nbr2_ptr, int32_t* nbr2,
                       int32_t* pair_info2, int32_t* node_info2, int32_t* vol_ptr, int32_t* vol_src);

/*
 * Task queue of the persistent assembly kernel (host): for each granule g, the
 * element tiles of g followed by the gather tiles made ready by granule g-1-lag
 * (pairs when with_pairs, then nodes).  Each task is 4 int32 {kind, granule, begin, end};
 * b_tiles_per_granule (n_granules) counts the gather tiles of each granule.  Element
 * tasks hold `tile` elements (dividing the plan granule), gather tasks `tile_items`
 * items.  Uses only the host fields of `plan`.
 */
int psx_task_count(const psx_plan_t* plan, int with_pairs, int32_t tile, int32_t tile_items, int32_t lag,
                   int64_t* n_tasks);
int psx_task_fill(const psx_plan_t* plan, int with_pairs, int32_t tile, int32_t tile_items, int32_t lag,
                  int32_t* tasks, int32_t* b_tiles_per_granule);

/*
 * Workspace bytes of one assembly call on the current device: task counters and a
 * ring of *ring_elems element records (K part in the precision's type, f in double).
 */
int psx_work_bytes(const psx_plan_t* plan, int precision, int64_t* ring_elems, int64_t* bytes);

/* ---- Tet4 element kernels (device) ----------------------------------------- */

/*
 * Tet4 Total-Lagrangian NeoHookean assembly (replaces the element loops of
 * domain/solid.py:172-207, 230-325 and the COO->CSR / np.add.at scatter).
 *   X, u (device, N x 3 double; u ignored for PSX_LINEAR)
 *   mu_e, kappa_e (device, E doubles) per-element moduli, or NULL to use mu, kappa
 *   lam: Lame lambda for PSX_LINEAR (with mu); the mass density for PSX_MASS
 *        (element/tet4_base.py:138-151: rho V / 20 (1 + delta_ab) I per block)
 *   f_out (device, 3N doubles) when mode has PSX_WANT_F
 *   k_out (device, nnz values in psx_csr_pattern order: double for PSX_FP64, float
 *          for PSX_FP32_MIXED) when mode has PSX_WANT_K or PSX_LINEAR
 *   work (device, >= psx_work_bytes, 256-byte aligned) scratch ring of element records
 *   status (device, psx_status_bytes(), zeroed by the caller); flags bit 0 is set if a
 *          bounded wait of the persistent kernel gave up (the results are then invalid)
 * One launch of a persistent kernel; the call also clears the task counters.
 * Deterministic: every output value is a fixed-order sum; no atomics touch f or K.
 */
int psx_tet4_assemble(const psx_plan_t* plan, const double* X, const double* u,
                      const double* mu_e, const double* kappa_e, double mu, double kappa, double lam,
                      int mode, int precision, double* f_out, void* k_out, void* work,
                      int64_t work_bytes, void* status, void* stream);

/* ---- Tet10 element kernels (device) ---------------------------------------- */

/*
 * Tet10 Total-Lagrangian NeoHookean assembly, 4-point rule (replaces the element loops of
 * domain/solid.py:172-207, 230-325 around element/tet10_total_lagrangian.py:63-136 and
 * element/tet10_base.py:310-342).  Same arguments and outputs as psx_tet4_assemble;
 * modes PSX_WANT_F, PSX_WANT_K, PSX_LINEAR and PSX_MASS (the consistent mass of
 * element/tet10_base.py:344-372 with the corner tetrahedron's |det| / 6 as the element
 * volume, density in `lam`).  The plan must be built with npe = 10 and an element task
 * tile of 8.
 */
int psx_tet10_assemble(const psx_plan_t* plan, const double* X, const double* u,
                       const double* mu_e, const double* kappa_e, double mu, double kappa, double lam,
                       int mode, int precision, double* f_out, void* k_out, void* work,
                       int64_t work_bytes, void* status, void* stream);

/* det J and det F at the 4 quadrature points of element e: out8 (device, 8 doubles). */
int psx_tet10_element_dets(const int32_t* conn, const double* X, const double* u, int64_t e,
                           double* out8, void* stream);

/*
 * Dynamic effective tangent in one sweep: K_eff = c_t K_T(u) + c_m M + c_0 K_0 with M the
 * consistent mass of density rho (element/tet4_base.py:138-151) and K_0 the small-strain
 * stiffness (lam, mu; or lambda_e = kappa_e - 2/3 mu_e, mu_e per element) -- the
 * combination NonlinearDynamicAnalysis forms on the host (analysis/nonlinear_dynamic.py:
 * 640-644, with Rayleigh damping C = alpha M + beta K_0 folded into c_m and c_0).  mode:
 * PSX_WANT_K, optionally | PSX_WANT_F (f_out = f_int(u)).  Same CSR order, workspace and
 * status as psx_tet4_assemble.
 */
int psx_tet4_assemble_effective(const psx_plan_t* plan, const double* X, const double* u, const double* mu_e,
                                const double* kappa_e, double mu, double kappa, double lam, double rho, double c_t,
                                double c_m, double c_0, int mode, int precision, double* f_out, void* k_out,
                                void* work, int64_t work_bytes, void* status, void* stream);

/*
 * Tet4Fbar f_int and tangent (replaces Tet4Fbar.assemble_internal_forces /
 * assemble_tangent_stiffness_matrix, element/tet4_fbar.py:248-459) on the two-ring CSR
 * (k_out: nnz2 doubles, zero where the reference's sum K_dev + K_vol has no entry).
 * Device inputs: conn (E x 4), X, u (N x 3), the node -> element incidences (inc_ptr,
 * inc_elem, psx_graph_fill), the one-ring graph and its block lists (psx_block_lists),
 * the gather items of psx_plan_fill with psx_fbar_plan_fill positions, the two-ring
 * vol lists; jbar_in (E, optional) replaces the nodal average, jbar_out (E, optional)
 * receives the J_bar used.  work: psx_fbar_work_doubles(E, N, n_nbr) doubles.
 * Scalar moduli only (the volumetric blocks use one bulk modulus, as the reference).
 */
int64_t psx_fbar_work_doubles(int64_t E, int64_t N, int64_t n_nbr);
/*
 * Independent Tet4Fbar elements with given J_bar (Tet4Fbar.compute_nonlinear_force_and_
 * tangent_stiffness, element/tet4_fbar.py:147-211): X_elem, u_elem (device, n x 4 x 3),
 * jbar (n) -> k_out (n x 12 x 12), f_out (n x 12).
 */
int psx_fbar_element(int64_t n, const double* X_elem, const double* u_elem, const double* jbar, double mu,
                     double kappa, double* k_out, double* f_out, void* status, void* stream);
int psx_fbar_assemble(const int32_t* conn, int64_t E, int64_t N, const double* X, const double* u, double mu,
                      double kappa, const int32_t* inc_ptr, const int32_t* inc_elem, const int32_t* nbr_ptr,
                      const int32_t* nbr, int64_t n_nbr, const int32_t* blk_ptr, const int32_t* blk_src,
                      int64_t n_pairs, const int32_t* pair_info2, const int32_t* pair_ptr, const int32_t* pair_src,
                      const int32_t* node_info2, const int32_t* node_ptr, const int32_t* node_src,
                      const int32_t* nbr2_ptr, const int32_t* vol_ptr, const int32_t* vol_src, const double* jbar_in,
                      double* f_out, double* k_out, int64_t nnz2, double* jbar_out, double* work,
                      int64_t work_doubles, void* status, void* stream);

/*
 * Hyper-reduced (ECSW) Tet4 evaluation (replaces HyperReducedECSWModel.
 * evaluate_forces_and_stiffness, hyperreduction/model.py:254-318): for the n elements of
 * the reduced integration domain -- reference coordinates X_elem (n x 4 x 3), modal
 * sub-bases phi_elem (n x 12 x r, row-major), cubature weights (n), optional per-element
 * moduli (n) -- and reduced coordinates u_r (r): f_r (r) = sum_e w_e Phi_e^T f_e(Phi_e u_r)
 * and K_r (r x r) = sym(sum_e w_e Phi_e^T k_e(Phi_e u_r) Phi_e), summed in element order.
 * work: psx_ecsw_work_doubles(n, r) doubles.  Status as psx_tet4_assemble.
 */
int64_t psx_ecsw_work_doubles(int64_t n, int32_t r);
int psx_ecsw_evaluate(int64_t n, int32_t r, const double* X_elem, const double* phi_elem, const double* weights,
                      const double* u_r, const double* mu_e, const double* kappa_e, double mu, double kappa,
                      double* f_r, double* K_r, double* work, int64_t work_doubles, void* status, void* stream);

/*
 * Matrix-free tangent product y = K_T(u) v (no matrix is formed): each element
 * evaluates K_e v_e from its kinematics in closed form and the node gather sums the
 * contributions in fixed order, so y equals the assembled K_T @ v of the reference
 * (domain/solid.py:280-325 followed by a CSR product) to rounding.
 *   v, y_out (device, 3N doubles); work as for psx_tet4_assemble.
 */
int psx_tet4_kv(const psx_plan_t* plan, const double* X, const double* u,
                const double* mu_e, const double* kappa_e, double mu, double kappa, int precision,
                const double* v, double* y_out, void* work, int64_t work_bytes, void* status,
                void* stream);

/*
 * Vector-Jacobian product of the internal force (no counterpart in the reference, which
 * is gradient-free): for a cotangent w (3N), gX_out (3N) = w^T df_int/dX, and, when not
 * null, gmu_out / gkappa_out (E) = w^T df_int/dmu_e, w^T df_int/dkappa_e.  F is
 * recomputed from (X, u); FP64 throughout; gX is gathered per node in fixed order.
 * w^T df_int/du = K_T(u) w is psx_tet4_kv.  work as for psx_tet4_assemble (FP64).
 */
int psx_tet4_adjoint(const psx_plan_t* plan, const double* X, const double* u,
                     const double* mu_e, const double* kappa_e, double mu, double kappa,
                     const double* w, double* gX_out, double* gmu_out, double* gkappa_out,
                     void* work, int64_t work_bytes, void* status, void* stream);

/*
 * One dynamic-relaxation pseudo-step on the linearised system K_T(u) x = b, fused into
 * a single pass (the viscous update of analysis/dynamic_relaxation.py:296-299,378-382):
 *   r = b - K_T(u) x,  a = minv * r,  vel = c1 vel + c2 a,  x += dt vel   (in place)
 * minv (device, 3N) is the inverse lumped mass, 0 on prescribed DOFs; r_out (device,
 * 3N, optional) receives the residual r of the incoming x.
 */
int psx_tet4_dr_step(const psx_plan_t* plan, const double* X, const double* u,
                     const double* mu_e, const double* kappa_e, double mu, double kappa, int precision,
                     const double* b, const double* minv, double c1, double c2, double dt,
                     double* x, double* vel, double* r_out, void* work, int64_t work_bytes,
                     void* status, void* stream);

/* ---- Preconditioned CG (device) ---------------------------------------------- */

#define PSX_PRECOND_NONE 0
#define PSX_PRECOND_JACOBI 1     /* 1/diag where |diag| > 1e-14, else 1 (the reference's) */
#define PSX_PRECOND_BJACOBI 2    /* inverse 3x3 diagonal block per node (n % 3 == 0) */
/* OR'd into `precond` of the PCG entry points (no counterpart in the reference): the
   caller guarantees a node-blocked CSR, as psx_csr_pattern builds it -- the three rows of
   node i have the same columns, in triples 3j, 3j+1, 3j+2 per neighbour j, and row 3i+k
   starts k * (length of row 3i) after row 3i (n % 3 == 0).  The SpMVs then read each
   neighbour's columns and x once per node instead of once per row. */
#define PSX_PCG_NODAL 0x100

/* Workspace bytes of psx_pcg for an n x n system. */
int psx_pcg_work_bytes(int64_t n, int precond, int64_t* bytes);

/*
 * Preconditioned CG on a CSR matrix (replaces solver/sparse_linear_solver.py:37-68,
 * scipy.sparse.linalg.cg with the Jacobi operator).  indptr (n+1), indices (nnz,
 * sorted per row), values (nnz; double for PSX_FP64, float for PSX_FP32_MIXED) on the
 * device; b (n) and x (n, in: initial guess -- zero for the reference's behaviour --,
 * out: solution) double.  Stops when ||r|| < max(atol, rtol ||b||), as scipy does;
 * after maxiter updates without that it stops unconverged.  Writes to status:
 * iters = iterations, flags = 0 converged / 2 max iterations reached / 4 breakdown,
 * value = final ||r||.  Dot products are reduced in a fixed order (bitwise
 * reproducible).  Synchronises the stream every 16 iterations to test convergence.
 */
int psx_pcg(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
            int value_precision, const double* b, double* x, double rtol, double atol, int32_t maxiter,
            int precond, void* work, int64_t work_bytes, void* status, void* stream);

/*
 * psx_pcg with a fixed trip count and no host synchronisation (no counterpart in the
 * reference, whose solves always return to Python): exactly maxiter iterations are
 * enqueued on the stream and become no-ops once converged, so the call can be captured
 * in a CUDA graph.  Same arguments, results and status as psx_pcg.
 */
int psx_pcg_enqueue(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                    int value_precision, const double* b, double* x, double rtol, double atol, int32_t maxiter,
                    int precond, void* work, int64_t work_bytes, void* status, void* stream);

/* ---- Two-level preconditioner (no counterpart in the reference) -------------------
 * A coarse space of rigid-body modes: the nodes are grouped into aggregates, and each
 * aggregate a contributes six columns of the prolongation P (three translations and
 * three rotations about its centroid: the column of rotation e at node i is
 * e x (X_i - c_a)); P is zero on eliminated unknowns.  The preconditioner is
 *   M^-1 r = B^-1 r + P A_c^-1 P^T r,    A_c = P^T A P,
 * with B the 3x3 diagonal blocks of A (block-Jacobi).  The aggregates are grouped into
 * independent blocks (the instances of a batch of meshes, whose A is block diagonal), and
 * the caller supplies A_c^-1 of every block as a dense matrix (psx_coarse_probe and
 * psx_coarse_restrict assemble A_c from products with A). */
typedef struct psx_coarse_t {
  int64_t n_nodes;           /* N: the system has 3N unknowns */
  int64_t n_agg;             /* aggregates */
  const int32_t* node_agg;   /* N: aggregate of each node, or -1 */
  const int32_t* agg_ptr;    /* n_agg + 1: nodes of aggregate a are agg_nodes[agg_ptr[a] .. agg_ptr[a+1]) */
  const int32_t* agg_nodes;  /* ascending within each aggregate */
  const double* d;           /* N x 3: node coordinates minus the centroid of its aggregate */
  const uint8_t* fixed;      /* 3N: nonzero on eliminated unknowns */
  int32_t n_blocks;          /* independent coarse blocks */
  int32_t nc;                /* padded coarse size: >= 6 x the aggregates of any block */
  const int32_t* block_agg;  /* n_blocks + 1: block b holds aggregates [block_agg[b], block_agg[b+1]); a block with
                                6 x its aggregates > nc gets no coarse correction */
  const double* ainv;        /* n_blocks x nc x nc, row-major: A_c^-1 of each block (6 (a - block_agg[b]) + t) */
  double* rc;                /* 6 n_agg scratch */
  double* yc;                /* 6 n_agg scratch */
} psx_coarse_t;

/* v (3N, device) = sum over the aggregates a with agg_color[a] == color of column
 * 6 a + mode of P (mode 0-2 translations, 3-5 rotations). */
int psx_coarse_probe(const psx_coarse_t* coarse, const int32_t* agg_color, int32_t color, int32_t mode, double* v,
                     void* stream);

/* out (6 n_agg, device) = P^T w, each aggregate's six sums in a fixed order. */
int psx_coarse_restrict(const psx_coarse_t* coarse, const double* w, double* out, void* stream);

/*
 * psx_pcg / psx_pcg_enqueue with the two-level preconditioner: precond must be
 * PSX_PRECOND_BJACOBI (optionally | PSX_PCG_NODAL); the coarse correction is added to
 * every block-Jacobi application.  host_checks = 1 behaves as psx_pcg (a stream
 * synchronisation every 16 iterations), 0 as psx_pcg_enqueue (capturable).
 */
int psx_pcg_coarse(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                   int value_precision, const double* b, double* x, double rtol, double atol, int32_t maxiter,
                   int precond, const psx_coarse_t* coarse, void* work, int64_t work_bytes, void* status,
                   void* stream, int host_checks);

/*
 * Batched CG (no counterpart in the reference, which solves one mesh at a time): a
 * block-diagonal system of n_seg independent segments (the meshes of a batch stored back
 * to back; segment s owns unknowns seg_offsets[s] .. seg_offsets[s+1], whole nodes) is
 * solved as n_seg independent preconditioned CGs run in the same launches, each with its
 * own step lengths, residual test max(atol, rtol ||b_s||) and iteration count, so every
 * instance converges at its own rate.  precond must be PSX_PRECOND_BJACOBI (optionally |
 * PSX_PCG_NODAL); coarse (or NULL) adds the two-level correction.  seg_offsets (int64,
 * n_seg + 1) and node_seg (int32, N: segment of each node) on the device.  Exactly
 * maxiter iterations are enqueued (finished segments stop updating), nothing is read
 * back.  status: iters = most iterations of a segment, flags = 0 if every segment
 * converged (2: a segment hit maxiter, 4: a breakdown); seg_iters (device, n_seg, or
 * NULL) receives each segment's iterations, as -(iterations + 1) if it did not converge.
 * Workspace: psx_pcg_batched_work_bytes.
 */
int psx_pcg_batched_work_bytes(int64_t n, int32_t n_seg, int64_t* bytes);
int psx_pcg_batched(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                    int value_precision, const double* b, double* x, double rtol, double atol, int32_t maxiter,
                    int precond, int32_t n_seg, const int64_t* seg_offsets, const int32_t* node_seg,
                    const psx_coarse_t* coarse, void* work, int64_t work_bytes, void* status, int32_t* seg_iters,
                    void* stream);

/*
 * y = alpha A x + beta y for a CSR matrix (values double for PSX_FP64, float for
 * PSX_FP32_MIXED; x, y double, device), rows summed in a fixed order: the products with
 * the constant mass and stiffness matrices in the dynamic residual
 * (analysis/nonlinear_dynamic.py:602-611).
 */
int psx_csr_spmv(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values, int value_precision,
                 const double* x, double alpha, double beta, double* y, void* stream);

/*
 * out[s] = sum of x[i]^2 for offsets[s] <= i < offsets[s+1] (device arrays; offsets int64,
 * n_seg + 1 entries), reduced in a fixed order: the per-mesh residual norms of a batch of
 * meshes stored back to back (the per-instance ||R_free|| test of
 * analysis/nonlinear_static.py:321-345 for every mesh at once).
 */
int psx_segment_sumsq(int64_t n_seg, const int64_t* offsets, const double* x, double* out, void* stream);

/*
 * Symmetric elimination of prescribed DOFs in a CSR matrix, in place: rows and columns
 * of DOFs with fixed[d] != 0 are zeroed and their diagonal set to 1 (the pattern and
 * symmetry are kept).  fixed (device, n bytes).
 */
int psx_csr_dirichlet(int64_t n, const int32_t* indptr, const int32_t* indices, void* values,
                      int value_precision, const uint8_t* fixed, void* stream);

/*
 * psx_pcg without a workspace argument: no counterpart in the reference.  For callers
 * that cannot allocate device memory when they solve (their device memory belongs to
 * their own pool allocator, or their run reserves all memory up front), the solve runs
 * on a fixed 32 MiB scratch array that is part of this library and is reserved on every
 * GPU that loads it until the process exits (psx_pcg_static_max_bytes() returns the
 * size).  It allocates nothing.  Systems whose psx_pcg_work_bytes exceeds the scratch
 * are rejected with PSX_ERR_LIMIT: about n <= 838,000 unknowns with the Jacobi
 * preconditioner and n <= 599,000 with block-Jacobi.  The array is reserved when the CUDA
 * runtime loads this library's CG module on a device: at context creation when the
 * process runs with CUDA_MODULE_LOADING=EAGER, otherwise (lazy loading, the CUDA 12
 * default) at the first call that uses the module on that device, which a
 * psx_pcg_static call does.  A caller that must have all its device memory reserved
 * before its run either sets CUDA_MODULE_LOADING=EAGER or makes one psx_pcg_static call
 * on each device during its set-up; later calls reserve nothing more.  The first call on
 * a device also looks up the scratch address on that device; make that first call before
 * any stream capture.  Like psx_pcg, the solve reads its convergence test back to the
 * host every 16 iterations (a device-to-host copy and a synchronisation of `stream`).
 * Every call on a device shares the one array, so calls that overlap on the GPU (other
 * streams, other host threads) race; the scalars the solve needs at zero are cleared at
 * the start of every call.  Arguments and results are those of psx_pcg.
 */
size_t psx_pcg_static_max_bytes(void);
int psx_pcg_static(int64_t n, const int32_t* indptr, const int32_t* indices, const void* values,
                   int value_precision, const double* b, double* x, double rtol, double atol,
                   int32_t maxiter, int precond, void* status, void* stream);

/*
 * CUDA-core compute roofs (no counterpart in the reference; measurement support): one
 * launch of `blocks` x 256 threads, each running 8 independent FMA chains for `iters`
 * steps in FP64 (precision PSX_FP64) or FP32 (PSX_FP32_MIXED).  *flops receives the
 * FLOPs of the launch (2 per FMA); the caller times it.  sink: device scratch of
 * psx_fma_roof_sink_bytes(blocks) bytes (one value per thread, so nothing is dead code).
 */
int psx_fma_roof(int precision, int64_t iters, int blocks, void* sink, double* flops, void* stream);
int64_t psx_fma_roof_sink_bytes(int blocks);

/*
 * Reference det (of [1 X], = 6 V) and det F of one element, written to out2
 * (device, 2 doubles).  Used to word the inversion error of a failed call.
 */
int psx_tet4_element_dets(const int32_t* conn, const double* X, const double* u,
                          int64_t e, double* out2, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PSIERRA_B200_H */
