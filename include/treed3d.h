/*
 * treed3d.h -- C ABI of libtreed3d.so, the sm_100a field solver of charges in a plane
 * (B200-native implementation of tree-d-3d's FlatQuadtree, Barnes-Hut walk, FMM and
 * direct sums).
 *
 * Conventions (those of the reference's kernel boundary, src/tree_d_3d/kernels/
 * __init__.py:99-114, where every kernel takes contiguous float64 / int64 arrays and
 * writes caller-allocated outputs in place):
 *   - every pointer is a DEVICE pointer to caller-owned memory, unless marked "host";
 *   - points are component-major (2, n) float64 arrays (x row, then y row);
 *   - node arrays are node-major: center (nodes, 2), moments (nodes, order + 1);
 *   - indices are int64;
 *   - `stream` is a cudaStream_t (0: the legacy default stream); work is enqueued on it;
 *   - `status` is an int64 device word the caller zeroes: a kernel that meets an
 *     unsoftened coincident charged pair writes 1 + an index there (the first thread
 *     to report wins, as tree_d_3d_report, src/tree_d_3d/kernels/barnes_hut.cuh:15-20);
 *   - scratch memory is a caller-provided `workspace` of at least the size returned
 *     by the matching *_workspace_size query; the library allocates nothing;
 *   - return value: TD3_OK, or an error code below (launch errors are TD3_ECUDA with
 *     the CUDA error kept for td3_last_error).
 * Entry points are re-entrant and keep no state between calls, with one exception:
 * td3_direct_sum_noalloc keeps its scratch in one fixed device array shared by all of
 * its calls (and caches that array's address per device), so its calls must not
 * overlap on the GPU; its block below gives the details.
 */
#ifndef TREED3D_H
#define TREED3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TD3_OK 0
#define TD3_EINVAL 1      /* an argument is out of range */
#define TD3_ECUDA 2       /* a CUDA call failed (td3_last_error) */
#define TD3_ENEEDMORE 3   /* an output buffer is too small; the needed size is reported */
#define TD3_EWORKSPACE 4  /* the workspace is smaller than its size query */
#define TD3_EDEPTH 5      /* the tree is too deep for the walk (depth > 190) */
#define TD3_ETOOLARGE 6   /* the call needs more than a no-allocation entry's fixed scratch */

#define TD3_KERNEL_COULOMB 0
#define TD3_KERNEL_LOG 1

/* Highest expansion order (MAX_ORDER, src/tree_d_3d/flat_tree.py:46). */
#define TD3_MAX_ORDER 64

/* Library version (major * 10000 + minor * 100 + patch). */
int td3_version(void);

/* The last CUDA error seen by this thread, as a string ("" when none). */
const char* td3_last_error(void);

/* ------------------------------------------------------------------ direct sums */

/* Exact all-pairs potential (n_targets) and field (2, n_targets) at `targets` of the
 * sources `pos` (2, n_sources) with `charge`, without k_e.  kernel: TD3_KERNEL_COULOMB
 * (phi = sum q / sqrt(r^2 + eps^2)) or TD3_KERNEL_LOG (phi = -sum q ln(r^2 + eps^2),
 * E = 2 sum q d / (r^2 + eps^2)).  exclude[i] is a source index skipped for target i
 * (-1: none); zero charges are skipped.  with_potential = 0 writes phi = 0 and, for
 * the log kernel, skips the logarithms.
 * Replaces the reference kernels direct_sum (src/tree_d_3d/kernels/direct_sum/
 * direct_sum_cuda.cu:7-44) and direct_log_sum (kernels/direct_log_sum/
 * direct_log_sum_cuda.cu:7-42), called by direct_field (src/tree_d_3d/flat_tree.py:157-158). */
size_t td3_direct_sum_workspace_size(int64_t n_targets, int64_t n_sources);
int td3_direct_sum(int kernel, const double* targets, int64_t n_targets, const int64_t* exclude,
                   const double* pos, const double* charge, int64_t n_sources, double softening,
                   int with_potential, double* phi, double* field, int64_t* status,
                   void* workspace, size_t workspace_bytes, void* stream);

/* td3_direct_sum without a workspace, for callers that cannot allocate device memory
 * (a host application that owns all device memory and passes only inputs and outputs,
 * a loop where an allocation could block).  No counterpart in the reference.  Its
 * scratch is a fixed device array of the library (4.6 MiB on every device that loads
 * it, kept until exit), enough for at most TD3_DIRECT_NOALLOC_MAX_TARGETS targets and
 * any number of sources; more targets return TD3_ETOOLARGE (td3_last_error says why).
 * The first call on a device looks up the array's device address (once per device,
 * with that device current); make that first call before any stream capture.  The
 * address stays cached until the process exits: do not reset a device
 * (cudaDeviceReset) between calls of this entry point.  Every call shares the array:
 * calls that overlap on the GPU (other streams, other threads) race on it, so
 * serialise them.  Results equal td3_direct_sum's. */
#define TD3_DIRECT_NOALLOC_MAX_TARGETS 65536
int td3_direct_sum_noalloc(int kernel, const double* targets, int64_t n_targets,
                           const int64_t* exclude, const double* pos, const double* charge,
                           int64_t n_sources, double softening, int with_potential,
                           double* phi, double* field, int64_t* status, void* stream);

/* Exact pair energy sum_{i<j} q_i q_j / sqrt(r^2 + eps^2) of the Coulomb kernel, added
 * to energy[0] (device).  Replaces pair_energy (src/tree_d_3d/kernels/pair_energy/
 * pair_energy_cuda.cu:11-38), used by ElectrostaticSimulation.get_potential_energy
 * (src/tree_d_3d/simulation.py:905-915). */
size_t td3_pair_energy_workspace_size(int64_t n);
int td3_pair_energy(const double* pos, const double* charge, int64_t n, double softening,
                    double* energy, int64_t* status, void* workspace, size_t workspace_bytes,
                    void* stream);

/* ------------------------------------------------------------------ tree build */

/* Build the quadtree of the n particles at `pos` (2, n) in the root cell (xmid, ymid,
 * half): nodes with more than leaf_capacity particles above max_depth split into four
 * children (upper left, upper right, lower left, lower right), numbered breadth first
 * in the order of their parents; a particle on a dividing line goes left or up; the
 * particles of a cell keep their input order.  Writes the node arrays (capacity rows:
 * node_center (capacity, 2), node_half, node_start, node_end, node_child (-1 for
 * leaves), node_depth), perm (n; the particles in tree order) and sorted_pos (2, n;
 * pos[:, perm]).  levels (HOST, min(capacity, max_depth + 1) + 1) receives the first
 * node of each depth;
 * sizes (HOST, 4) receives node count, number of levels and 1 if capacity was too
 * small (then TD3_ENEEDMORE is returned, the tree is unfinished and sizes[0] is the
 * node count needed, or a lower bound of it: retry with a larger capacity, as the
 * reference doubles it); sizes[3] is 1 if a position is not finite, 2 if one lies
 * outside the root cell (the inputs FlatQuadtree rejects, src/tree_d_3d/flat_tree.py:
 * 788-794), and TD3_EINVAL is returned.  Synchronises `stream` once (twice for trees deeper than 16
 * levels; once per level for trees deeper than 32 levels).
 * Replaces quadtree_build (src/tree_d_3d/kernels/quadtree_build/quadtree_build_pyccel.py:
 * 12-137) and the GPU level kernels quadtree_quadrants / quadtree_scatter
 * (kernels/quadtree_quadrants/quadtree_quadrants_cuda.cu:7-26, kernels/quadtree_scatter/
 * quadtree_scatter_cuda.cu:8-34) driven by FlatQuadtree._build (src/tree_d_3d/flat_tree.py:
 * 483-625); identical node arrays, perm and levels. */
size_t td3_quadtree_build_workspace_size(int64_t n, int64_t capacity);
int td3_quadtree_build(const double* pos, int64_t n, double xmid, double ymid, double half,
                       int64_t leaf_capacity, int64_t max_depth, int64_t capacity,
                       double* node_center, double* node_half, int64_t* node_start,
                       int64_t* node_end, int64_t* node_child, int64_t* node_depth,
                       int64_t* perm, double* sorted_pos, int64_t* levels, int64_t* sizes,
                       void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ moments */

/* Coulomb cell moments about each node centre: node_q, node_qabs (sum |q|), node_p
 * (nodes, 2) and the raw second moment node_s (nodes, 3: xx, xy, yy); leaves from their
 * particles (sorted_pos (2, n), sorted_charge in tree order), parents by M2M, deepest
 * level first.  levels (HOST, n_levels + 1).  Replaces quadtree_moments_upward
 * (src/tree_d_3d/kernels/quadtree_moments_upward/quadtree_moments_upward_pyccel.py:13-83)
 * and quadtree_moments (kernels/quadtree_moments/quadtree_moments_cuda.cu:7-46), called
 * by FlatQuadtree._moments (src/tree_d_3d/flat_tree.py:720-743). */
int td3_quadtree_moments(const int64_t* levels, int64_t n_levels, const double* sorted_pos,
                         const double* sorted_charge, int64_t n, const double* node_center,
                         const int64_t* node_start, const int64_t* node_end,
                         const int64_t* node_child, double* node_q, double* node_qabs,
                         double* node_p, double* node_s, void* stream);

/* Complex multipole moments a_n = sum q (z - c)^n, n = 0..order, of every node
 * (moment_re / moment_im (nodes, order + 1)) and node_qabs; binomial is the
 * (binomial_size, binomial_size) table C(n, m) of the reference (_binomial_table,
 * src/tree_d_3d/flat_tree.py:224-231).  Replaces log_moments_upward
 * (src/tree_d_3d/kernels/log_moments_upward/log_moments_upward_pyccel.py:14-93) and
 * log_quadtree_moments (kernels/log_quadtree_moments/log_quadtree_moments_cuda.cu:7-46),
 * called at src/tree_d_3d/flat_tree.py:689-713. */
int td3_log_moments(const int64_t* levels, int64_t n_levels, int order,
                    const double* sorted_pos, const double* sorted_charge, int64_t n,
                    const double* node_center, const int64_t* node_start,
                    const int64_t* node_end, const int64_t* node_child,
                    const double* binomial, int binomial_size, double* node_qabs,
                    double* moment_re, double* moment_im, void* stream);

/* td3_log_moments (sorted_dipole null) or td3_log_moments_adjoint (sorted_dipole the
 * (2, n) point dipoles) in one launch, orders up to 12: a thread per node forms its
 * leaf's moments, and the last of four children to finish forms their parent by M2M
 * (an atomic arrival counter per node in `arrive`, count int32, zeroed by the call),
 * with the operations of the level-by-level pass: the same bits.  node_parent from
 * td3_node_parents.  Replaces the per-level loop of log_moments_upward
 * (src/tree_d_3d/kernels/log_moments_upward/log_moments_upward_pyccel.py:14-93,
 * src/tree_d_3d/flat_tree.py:689-713) in one launch. */
int td3_log_moments_tree(int64_t count, int order, const double* sorted_pos,
                         const double* sorted_charge, const double* sorted_dipole, int64_t n,
                         const double* node_center, const int64_t* node_start,
                         const int64_t* node_end, const int64_t* node_child,
                         const int32_t* node_parent, const double* binomial, int binomial_size,
                         double* node_qabs, double* moment_re, double* moment_im,
                         int32_t* arrive, void* stream);

/* Cartesian multipole moments m_g = sum q (r - c)^g, |g| <= order, of every node
 * (moments (nodes, n_coef)), with the index tables of the reference's _cartesian.tables
 * (src/tree_d_3d/_cartesian.py:40-107): ex, ey (n_coef), shift (n_shift, 3) rows
 * (g, b, g - b) sorted by g with shift_coef, and shift_start (n_coef + 1) the first
 * row of each g (ex, ey are accepted for the reference's argument list; the powers of a
 * coefficient follow from its index).  Bit-identical to the reference; orders up to 66.
 * Replaces cart_moments_upward (src/tree_d_3d/kernels/
 * cart_moments_upward/cart_moments_upward_pyccel.py:14-82), called by
 * FlatQuadtree._cartesian_moments (src/tree_d_3d/flat_tree.py:1063-1084). */
int td3_cart_moments(const int64_t* levels, int64_t n_levels, const double* sorted_pos,
                     const double* sorted_charge, int64_t n, const double* node_center,
                     const int64_t* node_start, const int64_t* node_end,
                     const int64_t* node_child, const int64_t* ex, const int64_t* ey,
                     const int64_t* shift, const double* shift_coef, const int64_t* shift_start,
                     int n_coef, double* moments, void* stream);

/* ------------------------------------------------------------------ Barnes-Hut walk */

/* An order of the m targets (2, m) in which consecutive ones are close: the stable
 * sort of the reference's 16-bit Morton keys ((t - lo) * 65535 / span, x bits odd,
 * y bits even), written to order (m, int64).  Replaces FlatQuadtree._target_order
 * (src/tree_d_3d/flat_tree.py:891-912). */
size_t td3_target_order_workspace_size(int64_t m);
int td3_target_order(const double* targets, int64_t m, int64_t* order, void* workspace,
                     size_t workspace_bytes, void* stream);

/* Potential (m) and field (2, m) at `targets` by the Barnes-Hut walk, without k_e.
 * kernel TD3_KERNEL_COULOMB uses node_q, node_p, node_s (monopole through quadrupole,
 * softened far field); TD3_KERNEL_LOG uses moment_re / moment_im (nodes, order_p + 1)
 * (unsoftened series).  A cell containing the target is always opened; otherwise it is
 * accepted when 2h < theta |r - c| (Coulomb) or (4h) h < theta^2 |r - c|^2 (log), as in
 * the reference.  Cells with node_qabs == 0 are skipped; leaves are summed directly
 * (sorted_pos, sorted_charge in tree order, perm = source index of each slot), skipping
 * source exclude[i] for target i.  order (m, may be NULL) is the processing order of
 * the targets (warps take 32 consecutive ones).  tree_depth is the deepest node depth;
 * above 190 the call returns TD3_EDEPTH.  with_potential = 0 writes phi = 0 and skips
 * the log kernel's logarithms.  mixed = 1 keeps the FP64 opening decisions and evaluates
 * leaf pairs and far-field terms in FP32 with compensated sums; the log kernel then
 * reads moment_hat (td3_scale_moments' layout), hat_k = a_k / h^k
 * instead of moment_re / moment_im.  mixed = 0 ignores moment_hat (may be NULL).
 * Replaces evaluate_quadtree (src/tree_d_3d/kernels/evaluate_quadtree/
 * evaluate_quadtree_cuda.cu:9-107), evaluate_log_quadtree (kernels/evaluate_log_quadtree/
 * evaluate_log_quadtree_cuda.cu:9-104) and the CPU walk evaluate_groups
 * (kernels/evaluate_groups/evaluate_groups_pyccel.py:16-297), called by
 * FlatQuadtree.evaluate (src/tree_d_3d/flat_tree.py:987-1061). */
size_t td3_walk_workspace_size(int64_t node_count, int kernel);
int td3_evaluate_quadtree(int kernel, const double* targets, int64_t m, const int64_t* exclude,
                          const int64_t* order, const double* sorted_pos,
                          const double* sorted_charge, const int64_t* perm, int64_t n,
                          int64_t node_count, const double* node_center, const double* node_half,
                          const int64_t* node_start, const int64_t* node_end,
                          const int64_t* node_child, const int64_t* node_depth,
                          int64_t tree_depth, const double* node_q, const double* node_qabs,
                          const double* node_p, const double* node_s, const double* moment_re,
                          const double* moment_im, const float* moment_hat, int order_p,
                          double theta, double softening, int with_potential, int mixed,
                          double* phi, double* field, int64_t* status, void* workspace,
                          size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ FMM lists */

/* The mutual dual-tree traversal of one tree from the pair (root, root): a pair of
 * cells becomes an M2L pair if sqrt(2) (h_a + h_b) < theta d (d the centre distance), a
 * P2P pair if both are leaves (or a == b is a leaf), else the pairs of the children
 * of the larger (or the non-leaf) cell, or of a == b the 10 pairs c <= d; empty cells
 * are dropped.  m2l (m2l_capacity, 2) and p2p (p2p_capacity, 2) receive the pairs in
 * the reference's serial order (generation by generation, frontier order); sizes
 * (HOST, 4) = n_m2l, n_p2p, next frontier, -1 on overflow, when TD3_ENEEDMORE is
 * returned (retry with larger buffers).  frontier_capacity bounds one generation.
 * Synchronises `stream` once per 8 generations.  Replaces fmm_traverse
 * (src/tree_d_3d/kernels/fmm_traverse/fmm_traverse_pyccel.py:15-106,
 * fmm_traverse_cuda.cu:14-97) driven by FlatQuadtree._traverse
 * (src/tree_d_3d/flat_tree.py:1318-1358); identical lists.  n_nodes: the node count
 * (the traversal first packs each node into one 32-byte record in the workspace). */
size_t td3_fmm_traverse_workspace_size(int64_t frontier_capacity, int64_t n_nodes);
int td3_fmm_traverse(const double* node_center, const double* node_half,
                     const int64_t* node_start, const int64_t* node_end,
                     const int64_t* node_child, int64_t n_nodes, double theta, int64_t* m2l,
                     int64_t m2l_capacity, int64_t* p2p, int64_t p2p_capacity,
                     int64_t frontier_capacity, int64_t* sizes, void* workspace,
                     size_t workspace_bytes, void* stream);

/* The one-way traversal of a target tree (t_*) against a source tree (s_*) from
 * (root, root), with the predicates of td3_fmm_traverse; pairs are (target cell,
 * source cell), breadth first (the reference walks depth first: the same set of
 * pairs in another order).  Replaces dual_traverse (src/tree_d_3d/kernels/
 * dual_traverse/dual_traverse_pyccel.py:14-86) of FlatQuadtree._dual_lists
 * (src/tree_d_3d/flat_tree.py:1086-1122).  t_nodes, s_nodes: the node counts; the
 * workspace size is td3_fmm_traverse_workspace_size(frontier_capacity, t_nodes + s_nodes). */
int td3_dual_traverse(const double* t_center, const double* t_half, const int64_t* t_start,
                      const int64_t* t_end, const int64_t* t_child, int64_t t_nodes,
                      const double* s_center, const double* s_half, const int64_t* s_start,
                      const int64_t* s_end, const int64_t* s_child, int64_t s_nodes,
                      double theta, int64_t* m2l, int64_t m2l_capacity, int64_t* p2p,
                      int64_t p2p_capacity, int64_t frontier_capacity, int64_t* sizes,
                      void* workspace, size_t workspace_bytes, void* stream);

/* Rows by node of the pairs (count, 2): row_start (n_nodes + 1) and partners, in pair
 * order; mutual != 0 lists b under a and a under b (once if a == b).  partners holds
 * count (mutual: 2 count) slots; those past row_start[n_nodes] are scratch.  entry_row
 * (may be NULL; as many slots as partners) receives the row of every entry (n_nodes in
 * the scratch slots), for kernels that walk the entries rather than the rows.  Replaces pair_csr
 * (src/tree_d_3d/kernels/pair_csr/pair_csr_pyccel.py:12-45); identical rows. */
size_t td3_pair_csr_workspace_size(int64_t count, int mutual, int64_t n_nodes);
int td3_pair_csr(const int64_t* pairs, int64_t count, int mutual, int64_t n_nodes,
                 int64_t* row_start, int64_t* partners, int32_t* entry_row, void* workspace,
                 size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ log-kernel FMM */

/* M2L of the log kernel, FP64: adds to the local expansions (local_re / local_im
 * (n_dst, order + 1)) of every destination cell n the translated multipoles of the
 * source cells partners[row_start[n]:row_start[n + 1]]: with t = c_dst - c_src,
 * w = 1/t and a'_k = a_k w^k, s_l = sum_k coeff[k, l] a'_k (coeff the reference's real
 * M2L matrix, (order + 1)^2, _m2l_coefficients, src/tree_d_3d/flat_tree.py:234-245),
 * b_0 += a_0 ln|t| - s_0, b_l += -(-1)^l s_l w^l.  (Im ln t, which only moves Im b_0,
 * is dropped: Im b_0 never reaches the potential or the field.)  Replaces
 * fmm_m2l_host (src/tree_d_3d/kernels/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105) and
 * fmm_m2l (kernels/fmm_m2l/fmm_m2l_cuda.cu:12-80). */
int td3_fmm_m2l(const int64_t* row_start, const int64_t* partners, int64_t n_dst,
                const double* dst_center, const double* src_center, const double* moment_re,
                const double* moment_im, int order, const double* coeff, double* local_re,
                double* local_im, void* stream);

/* Mixed-precision M2L of the log kernel: moments scaled by the cell size, hat_k =
 * a_k / h^k (td3_scale_moments: rows of order + 1 complex float pairs rounded up to an
 * even count, so each row is 16-byte aligned, the pad pair zero), translated
 * in FP32 with ws = h_src / t and wd = h_dst / t (|ws|, |wd| < 1 for separated cells):
 * s_l = sum_k coeff[k, l] hat_k ws^k, bhat_0 = a_0 ln|t| - s_0, bhat_l = -(-1)^l s_l wd^l,
 * and local_re / local_im (FP64) += bhat_l / h_dst^l.  ln|t| is formed as ln|t / unit|
 * in FP32 plus ln(unit) sum a_0 in FP64 (unit > 0: a length of the problem, e.g. the
 * root half-width).  coeff is a HOST (order + 1)^2 array (the reference's M2L matrix);
 * order <= 20.  entry_row: the row of every entry of partners (td3_pair_csr); a warp
 * takes 32 consecutive entries at a time across row boundaries.  tensor_cores != 0
 * (orders <= 15) takes the matrix products s_l on the tensor cores (tcgen05.mma, 3xTF32 with FP32 accumulation) and needs status, a device
 * int64 the caller zeroed: it becomes nonzero if a wait for the tensor cores ran out (the
 * locals are then incomplete); otherwise FP32 CUDA-core arithmetic, status unused.  The
 * rows of one destination are summed in row order either way (deterministic).  The
 * FP32 counterpart of td3_fmm_m2l (reference: fmm_m2l_host,
 * src/tree_d_3d/kernels/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105). */
int td3_scale_moments(int64_t count, int order, const double* moment_re,
                      const double* moment_im, const double* node_half, float* hat, void* stream);
int td3_fmm_m2l_mixed(const int64_t* row_start, const int32_t* entry_row,
                      const int64_t* partners, int64_t n_dst,
                      const double* dst_center, const double* dst_half, const double* src_center,
                      const double* src_half, const float* hat, int order, const double* coeff,
                      double unit, int tensor_cores, double* local_re, double* local_im,
                      int64_t* status, void* stream);

/* The same mixed-precision log M2L (same formula, arguments and accuracy as
 * td3_fmm_m2l_mixed with tensor_cores = 0) with a group of 8 lanes per destination row:
 * each lane keeps its partial sums of the row in FP32 registers, the group's 8 partial
 * rows are summed pairwise at the row's end and added to local_re / local_im (FP64);
 * rows above 96 entries are taken by a whole warp (32 partial rows).  Every destination
 * is summed by one group in a fixed order (deterministic).  The sources come as packed
 * records (td3_pack_m2l_sources: td3_m2l_record_floats(order) floats per node, 16-byte
 * aligned: the centre as two doubles, hat_k = a_k / h^k as FP32 pairs, h / unit; 128
 * bytes at order 12, one cache line per gathered partner) written from the source tree's
 * FP64 moments, centres and half-widths.  A warp's rows are an even share of entries + 8
 * per row (a row takes a group at least one round), so runs of empty or short rows, as
 * in fmm_at's one-way target rows, spread over the warps.  Orders <= 20; coeff HOST.
 * Replaces fmm_m2l_host (src/tree_d_3d/kernels/fmm_m2l_host/fmm_m2l_host_pyccel.py:16-105)
 * in FP32 for fmm / fmm_at (src/tree_d_3d/flat_tree.py:1505-1539, :1151-1316). */
int td3_m2l_record_floats(int order);
int td3_pack_m2l_sources(int64_t count, int order, const double* moment_re,
                         const double* moment_im, const double* node_center,
                         const double* node_half, double unit, float* records, void* stream);
int td3_fmm_m2l_mixed_rows(const int64_t* row_start, const int64_t* partners, int64_t n_dst,
                           const double* dst_center, const double* dst_half,
                           const float* records, int order, const double* coeff, double unit,
                           double* local_re, double* local_im, void* stream);

/* The mixed-precision log M2L of the mutual lists of one tree as dense tensor-core
 * products grouped by translation (tcgen05.mma, 3xTF32 with FP32 accumulation), orders
 * up to TD3_M2L_GROUPED_MAX_ORDER.  A translation between cells whose depths differ by
 * dl = -1, 0, 1 and whose centres differ by t = u h_min (u an integer vector with
 * |u_x|, |u_y| <= span, h_min the smaller half-width) is the fixed matrix of the key
 * (dl, u) on size-scaled expansions; the other translations take the per-translation
 * formula in FP64.  Three calls:
 *   td3_m2l_operators: the 3 (2 span + 1)^2 keys' matrices into `ops`
 *     (td3_m2l_operators_size(span) bytes, float; coeff the reference's M2L matrix,
 *     DEVICE, (order + 1)^2); depends on (order, coeff, span) only;
 *   td3_m2l_groups: the directed translations of `pairs` (n_pairs, 2) sorted by
 *     (tile of 128 destinations, key; an off-table translation's key is
 *     3 (2 span + 1)^2 + its row in the tile) into keys / values (2 n_pairs each), the run
 *     starts run_start (2 n_pairs + 1) and the first run of every tile tile_run
 *     (ceil(n_nodes / 128) + 1); levels HOST (n_levels + 1, the first node of each
 *     depth, then n_nodes); n_nodes < 2^25; depends on the tree and the lists only;
 *   td3_fmm_m2l_grouped: the products into local_re / local_im (FP64, added), from the
 *     scaled moments `hat` of td3_scale_moments; the products of up to 4 runs of a tile
 *     are summed in FP32 on the tensor cores, then per destination in FP64, in the runs'
 *     order (deterministic); coeff HOST.
 * `status` (zeroed by the caller) receives 1 if a wait for the copies or the tensor
 * cores ran out.  Replaces fmm_m2l_host (src/tree_d_3d/kernels/fmm_m2l_host/
 * fmm_m2l_host_pyccel.py:16-105) for fmm (src/tree_d_3d/flat_tree.py:1505-1539). */
#define TD3_M2L_GROUPED_MAX_ORDER 14
size_t td3_m2l_operators_size(int span);
int td3_m2l_operators(int order, const double* coeff, int span, float* ops, void* stream);
size_t td3_m2l_groups_workspace_size(int64_t n_pairs);
int td3_m2l_groups(const int64_t* pairs, int64_t n_pairs, const double* node_center,
                   const double* node_half, const int64_t* node_depth, const int64_t* levels,
                   int64_t n_levels, int64_t n_nodes, int span, uint32_t* keys, uint32_t* values,
                   int32_t* tile_run, int32_t* run_start, void* workspace,
                   size_t workspace_bytes, void* stream);
int td3_fmm_m2l_grouped(const int32_t* tile_run, const int32_t* run_start,
                        const uint32_t* keys, const uint32_t* values, int64_t n_nodes,
                        const int64_t* levels, int64_t n_levels, const double* node_center,
                        const double* node_half, const float* hat, int order, const float* ops,
                        int span, const double* coeff, double* local_re, double* local_im,
                        int64_t* status, void* stream);

/* The parent of every node (node_parent (count), int32; -1 for the root), from
 * node_child.  No reference counterpart (its walks keep explicit stacks). */
int td3_node_parents(int64_t count, const int64_t* node_child, int32_t* node_parent,
                     void* stream);

/* L2L from the root down, level by level (levels HOST, n_levels + 1): every local
 * expansion shifted into its children, b_m(child) += sum_{l>=m} C(l, m) b_l s^(l-m),
 * over the children of each level (node_parent from td3_node_parents); empty cells
 * (node_start == node_end) are left as they are, nothing reads their locals.
 * Replaces fmm_downward (src/tree_d_3d/kernels/fmm_downward/fmm_downward_pyccel.py:15-64,
 * fmm_downward_cuda.cu:10-51) and its per-level loop (src/tree_d_3d/flat_tree.py:1540-1552). */
int td3_fmm_downward(const int64_t* levels, int64_t n_levels, const double* node_center,
                     const int32_t* node_parent, const int64_t* node_start,
                     const int64_t* node_end, int order, const double* binomial,
                     int binomial_size, double* local_re, double* local_im, void* stream);

/* The downward pass in one launch: every non-empty leaf's local becomes its own M2L
 * local plus the own M2L local of each ancestor shifted straight to the leaf's centre
 * (the L2L shift above, an exact re-expansion: equal to the level-by-level pass up to
 * rounding).  Internal cells keep their own M2L locals: only leaves feed L2P.
 * Replaces fmm_downward's per-level loop (src/tree_d_3d/flat_tree.py:1540-1552,
 * src/tree_d_3d/kernels/fmm_downward/fmm_downward_pyccel.py:15-64) for the FMM. */
int td3_fmm_downward_leaves(int64_t count, int order, const double* node_center,
                            const int32_t* node_parent, const int64_t* node_start,
                            const int64_t* node_end, const int64_t* node_child,
                            const double* binomial, int binomial_size, double* local_re,
                            double* local_im, void* stream);

/* ------------------------------------------------------------------ Coulomb FMM */

/* M2L of the softened Coulomb kernel with Cartesian expansions, FP64: for every
 * destination cell n and source cell partners[row_start[n]:row_start[n + 1]], the
 * Taylor coefficients A_g(t) of (|r|^2 + eps^2)^(-1/2) at t = c_dst - c_src by the
 * reference's recurrence, then local[n, b] += coef * m_a * A_{a+b} over the M2L rows
 * (b, a, a + b) of _cartesian.tables (src/tree_d_3d/_cartesian.py:40-107): row_a,
 * row_g (int32), row_coef, b_start (int32, n_coef + 1: first row of each b).  moments
 * (src cells, n_coef), local (n_dst, n_coef).  Orders up to 16 use the scaled form
 * T_b = (1 / b!) sum_a ((-1)^|a| m_a / a!) (g! A_g), g = a + b, with computed indices
 * (the row tables are then not read); higher orders read the rows.  Replaces cart_m2l_host
 * (src/tree_d_3d/kernels/cart_m2l_host/cart_m2l_host_pyccel.py:16-80). */
int td3_cart_m2l(const int64_t* row_start, const int64_t* partners, int64_t n_dst,
                 const double* dst_center, const double* src_center, const double* moments,
                 int order, double softening, const int* row_a, const int* row_g,
                 const double* row_coef, const int* b_start, double* local, void* stream);

/* The mixed-precision td3_cart_m2l for orders up to 16: the same translations in FP32
 * on expansions scaled by the source cell's half-width (t / h_src, eps / h_src,
 * m_a / h_src^|a|), the partners' sums brought to the destination's scale by exact
 * powers of two and added to the FP64 locals with h_dst^(-1-|b|) in FP64; dst_half and
 * src_half the cells' half-widths.  Replaces cart_m2l_host (src/tree_d_3d/kernels/
 * cart_m2l_host/cart_m2l_host_pyccel.py:16-80) in the mixed form. */
int td3_cart_m2l_mixed(const int64_t* row_start, const int64_t* partners, int64_t n_dst,
                       const double* dst_center, const double* dst_half,
                       const double* src_center, const double* src_half,
                       const double* moments, int order, double softening, double* local,
                       void* stream);

/* L2L of the Cartesian local expansions from the root down (levels HOST, n_levels + 1):
 * T_b(child) += C(g, b) T_g s^(g - b) over the shift rows regrouped by b (l2l_start
 * (n_coef + 1), l2l_g, l2l_d = g - b, l2l_coef; int32 indices); ex / ey are accepted for
 * the reference's argument list.  Replaces cart_downward (src/tree_d_3d/kernels/cart_downward/
 * cart_downward_pyccel.py:14-55). */
int td3_cart_downward(const int64_t* levels, int64_t n_levels, const double* node_center,
                      const int64_t* node_child, int order, const int64_t* ex, const int64_t* ey,
                      const int* l2l_start, const int* l2l_g, const int* l2l_d,
                      const double* l2l_coef, double* local, void* stream);

/* ------------------------------------------------------------------ near field */

/* The work plan of the near field: every non-empty leaf's row of P2P partners
 * (rows: n_nodes + 1 offsets, td3_pair_csr) cut into segments of at most `segment`
 * partners.  seg_leaf (int32), seg_range (e0, e1 pairs) and seg_out (-1: the leaf has
 * one segment and writes its final values; else the offset, in targets, of the
 * segment's partial sums) receive n_seg entries; sizes (HOST, 2) = n_seg and the
 * partial length (the caller allocates 3 * partial length doubles for the evaluation).
 * TD3_ENEEDMORE when seg_capacity < n_seg (n_seg is still reported).  Synchronises
 * `stream` once.  No reference counterpart (the reference's near field is serial on
 * the CPU and one thread per pair with atomics on the GPU). */
size_t td3_nearfield_plan_workspace_size(int64_t n_nodes);
int td3_nearfield_plan(const int64_t* rows, int64_t n_nodes, const int64_t* node_child,
                       const int64_t* node_start, const int64_t* node_end, int segment,
                       int* seg_leaf, int64_t* seg_range, int64_t* seg_out, int64_t seg_capacity,
                       int64_t* sizes, void* workspace, size_t workspace_bytes, void* stream);

/* L2P at the particles of every leaf plus the exact near field over the leaf's P2P
 * partners (the mutual P2P pairs as rows, cut by td3_nearfield_plan), softened,
 * excluding each particle itself; phi (n) and field (2, n) in input order (perm).
 * kernel TD3_KERNEL_LOG: complex local expansion local_a / local_b = local_re /
 * local_im (nodes, order + 1), phi += -2 Re W, Ex - i Ey += 2 W' (W' skipped logs when
 * with_potential = 0); TD3_KERNEL_COULOMB: Cartesian local expansion local_a (nodes,
 * (order + 1)(order + 2)/2), softened Coulomb pairs.  A coincident pair of two nonzero
 * charges reports 1 + a particle index.  partial: 3 * partial length doubles.
 * mixed != 0: the pair arithmetic in FP32 (pair differences taken in FP64, divided by
 * `unit` > 0, a length of the problem such as the root half-width, then rounded) with
 * compensated (Kahan) accumulation, rescaled in FP64 (the log kernel's ln unit^2 times
 * the charge sum added in FP64); the local expansions in FP64.  mixed = 0 ignores unit.
 * Replaces fmm_evaluate_host (src/tree_d_3d/kernels/fmm_evaluate_host/
 * fmm_evaluate_host_pyccel.py:14-100), fmm_evaluate (kernels/fmm_evaluate/
 * fmm_evaluate_cuda.cu:11-87) and cart_evaluate_host (kernels/cart_evaluate_host/
 * cart_evaluate_host_pyccel.py:16-110). */
int td3_fmm_evaluate(int kernel, const double* sorted_pos, const double* sorted_charge,
                     const int64_t* perm, int64_t n, const double* node_center,
                     const int64_t* node_start, const int64_t* node_end, int order,
                     const double* local_a, const double* local_b, const int64_t* p2p_partners,
                     const int* seg_leaf, const int64_t* seg_range, const int64_t* seg_out,
                     int64_t n_seg, double* partial, double softening, int with_potential,
                     int mixed, double unit, double* phi, double* field, int64_t* status,
                     void* stream);

/* The mixed-precision form of td3_fmm_evaluate (same arguments, outputs, status and
 * accuracy contract as mixed = 1) in three launches: the local expansions at every
 * particle in FP64, one thread per slot (slot_leaf: the leaf of every particle slot,
 * td3_slot_leaves), then the pair sums added to them, one warp per plan segment, then
 * the partial sums of leaves with several segments.  Pair arithmetic without FP64:
 * positions relative to the target leaf's centre in units of the power of two u with
 * unit <= u < 2 unit, held as FP32 hi + lo pairs, a pair's difference
 * (hi_i - hi_j) + (lo_i - lo_j); compensated sums as td3_fmm_evaluate.  slot_leaf is
 * required.  Replaces fmm_evaluate_host (src/tree_d_3d/kernels/fmm_evaluate_host/
 * fmm_evaluate_host_pyccel.py:14-100) and cart_evaluate_host (kernels/cart_evaluate_host/
 * cart_evaluate_host_pyccel.py:16-110) in FP32.  slot_leaf[k] = -1 leaves slot k out of
 * the far field (its outputs untouched), as the plan's emptied leaves leave it out of the
 * pair sums: one rank's share of the leaves. */
int td3_slot_leaves(int64_t n_nodes, const int64_t* node_child, const int64_t* node_start,
                    const int64_t* node_end, int32_t* slot_leaf, void* stream);
int td3_fmm_evaluate_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
                           const int64_t* perm, int64_t n, const double* node_center,
                           const int64_t* node_start, const int64_t* node_end, int order,
                           const double* local_a, const double* local_b,
                           const int32_t* slot_leaf, const int64_t* p2p_partners,
                           const int* seg_leaf, const int64_t* seg_range, const int64_t* seg_out,
                           int64_t n_seg, double* partial, double softening, int with_potential,
                           double unit, double* phi, double* field, int64_t* status,
                           void* stream);

/* td3_fmm_evaluate_mixed in its two parts, for callers that overlap them with other work:
 * td3_fmm_near_mixed WRITES the near field alone into phi and field (the pair sums, then
 * the leaves with several segments; every slot of a planned leaf; it reads no expansion,
 * so it can run on another stream while the M2M, M2L and L2L run), and
 * td3_fmm_far_mixed then ADDS the local expansions at the slots whose slot_leaf is not
 * -1.  td3_fmm_evaluate_mixed is the two in a row on one stream (the same bits). */
int td3_fmm_near_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
                       const int64_t* perm, int64_t n, const double* node_center,
                       const int64_t* node_start, const int64_t* node_end,
                       const int64_t* p2p_partners, const int* seg_leaf, const int64_t* seg_range,
                       const int64_t* seg_out, int64_t n_seg, double* partial, double softening,
                       int with_potential, double unit, double* phi, double* field,
                       int64_t* status, void* stream);
int td3_fmm_far_mixed(int kernel, const double* sorted_pos, const int64_t* perm, int64_t n,
                      const double* node_center, int order, const double* local_a,
                      const double* local_b, const int32_t* slot_leaf, int with_potential,
                      double* phi, double* field, void* stream);

/* fmm_at: L2P at the m targets (sorted_targets (2, m) in target-tree order, target_perm
 * their input indices, sorted_exclude their excluded source index) plus exact sums over
 * the partner source leaves of each target leaf (the one-way P2P rows cut by
 * td3_nearfield_plan on the target tree) of the source tree (sorted_pos, sorted_charge,
 * perm, s_start, s_end), skipping zero charges and the excluded source; results at the
 * targets' input indices; a coincident charge reports 1 + the target index.  mixed and
 * unit as in td3_fmm_evaluate.  Replaces
 * log_targets_host (src/tree_d_3d/kernels/log_targets_host/log_targets_host_pyccel.py:14-94)
 * and cart_targets_host (kernels/cart_targets_host/cart_targets_host_pyccel.py:16-98). */
int td3_fmm_targets(int kernel, const double* sorted_targets, const int64_t* sorted_exclude,
                    const int64_t* target_perm, int64_t m, const double* t_center,
                    const int64_t* t_start, const int64_t* t_end, int order,
                    const double* local_a, const double* local_b, const int64_t* p2p_partners,
                    const int* seg_leaf, const int64_t* seg_range, const int64_t* seg_out,
                    int64_t n_seg, double* partial, const double* sorted_pos,
                    const double* sorted_charge, const int64_t* perm, int64_t n,
                    const int64_t* s_start, const int64_t* s_end, double softening,
                    int with_potential, int mixed, double unit, double* phi, double* field,
                    int64_t* status, void* stream);

/* ------------------------------------------------------------------ adjoint (backward) */

/* Multipole moments of the adjoint FMM pass: monopoles sorted_weight (n) and point
 * dipoles sorted_dipole (2, n) at the particles (tree order).  Log kernel: a_n = sum
 * [w (z - c)^n - n e (z - c)^(n-1)], e = ex + i ey (moment_re / moment_im, node_wabs =
 * sum |w|); Cartesian: m_g = sum [w (r - c)^g - e . grad (r - c)^g] (tables as
 * td3_cart_moments).  No reference counterpart (the reference has no backward). */
int td3_log_moments_adjoint(const int64_t* levels, int64_t n_levels, int order,
                            const double* sorted_pos, const double* sorted_weight,
                            const double* sorted_dipole, int64_t n, const double* node_center,
                            const int64_t* node_start, const int64_t* node_end,
                            const int64_t* node_child, const double* binomial,
                            int binomial_size, double* node_wabs, double* moment_re,
                            double* moment_im, void* stream);
int td3_cart_moments_adjoint(const int64_t* levels, int64_t n_levels, const double* sorted_pos,
                             const double* sorted_weight, const double* sorted_dipole, int64_t n,
                             const double* node_center, const int64_t* node_start,
                             const int64_t* node_end, const int64_t* node_child,
                             const int64_t* ex, const int64_t* ey, const int64_t* shift,
                             const double* shift_coef, const int64_t* shift_start, int n_coef,
                             double* moments, void* stream);

/* Backward of the FMM field at the sources: for upstream gradients w = dL/dphi and
 * e = dL/dE (sorted_weight (n), sorted_dipole (2, n) in tree order) and the forward
 * field efield (2, n, input order), writes qbar = dL/dq (n) and xbar = dL/dx (2, n) in
 * input order:  qbar_k = Psi(x_k),  xbar_k = -w_k E_k + q_k grad Psi(x_k) - M_k e_k,
 * with Psi(y) = sum_j [w_j G(y - x_j) + e_j . grad G(y - x_j)] (j != k) and M_k =
 * sum_j q_j Hess G(x_k - x_j).  Far parts come from the adjoint local expansions
 * adj_a / adj_b (value and gradient) and the forward ones fwd_a / fwd_b (Hessian),
 * near parts pair by pair over the near-field plan (softened kernel; kernel as in
 * td3_fmm_evaluate, mixed and unit too).  partial: 6 * partial length doubles.  No
 * reference counterpart. */
int td3_fmm_adjoint(int kernel, const double* sorted_pos, const double* sorted_charge,
                    const int64_t* perm, int64_t n, const double* node_center,
                    const int64_t* node_start, const int64_t* node_end, int order,
                    const double* fwd_a, const double* fwd_b, const double* adj_a,
                    const double* adj_b, const int64_t* p2p_partners, const int* seg_leaf,
                    const int64_t* seg_range, const int64_t* seg_out, int64_t n_seg,
                    double* partial, const double* sorted_weight, const double* sorted_dipole,
                    const double* efield, double softening, int mixed, double unit,
                    double* qbar, double* xbar, void* stream);

/* The mixed-precision form of td3_fmm_adjoint (mixed = 1 implied) laid out as
 * td3_fmm_evaluate_mixed: the far parts of qbar and xbar at every particle in FP64, one
 * thread per slot (slot_leaf required), then the near parts added pair by pair without
 * FP64 arithmetic (qbar and xbar are linear in the near sums), then the partial sums of
 * multi-segment leaves.  No reference counterpart. */
int td3_fmm_adjoint_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
                          const int64_t* perm, int64_t n, const double* node_center,
                          const int64_t* node_start, const int64_t* node_end, int order,
                          const double* fwd_a, const double* fwd_b, const double* adj_a,
                          const double* adj_b, const int32_t* slot_leaf,
                          const int64_t* p2p_partners, const int* seg_leaf,
                          const int64_t* seg_range, const int64_t* seg_out, int64_t n_seg,
                          double* partial, const double* sorted_weight,
                          const double* sorted_dipole, const double* efield, double softening,
                          double unit, double* qbar, double* xbar, void* stream);

/* td3_fmm_adjoint_mixed in its two parts, as td3_fmm_near_mixed / td3_fmm_far_mixed:
 * td3_fmm_adjoint_near_mixed WRITES the near parts of qbar and xbar (it reads no
 * expansion), td3_fmm_adjoint_far_mixed then ADDS the far parts. */
int td3_fmm_adjoint_near_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
                               const int64_t* perm, int64_t n, const double* node_center,
                               const int64_t* node_start, const int64_t* node_end,
                               const int64_t* p2p_partners, const int* seg_leaf,
                               const int64_t* seg_range, const int64_t* seg_out, int64_t n_seg,
                               double* partial, const double* sorted_weight,
                               const double* sorted_dipole, double softening, double unit,
                               double* qbar, double* xbar, void* stream);
int td3_fmm_adjoint_far_mixed(int kernel, const double* sorted_pos, const double* sorted_charge,
                              const int64_t* perm, int64_t n, const double* node_center, int order,
                              const double* fwd_a, const double* fwd_b, const double* adj_a,
                              const double* adj_b, const int32_t* slot_leaf,
                              const double* sorted_weight, const double* sorted_dipole,
                              const double* efield, double* qbar, double* xbar, void* stream);

/* ------------------------------------------------------------------ grounded strip */

/* The conformal map zeta = exp(i pi (x + i y) / width) of the strip 0 < x < width
 * (src/tree_d_3d/strip.py:147-163, GroundedStripField.to_plane / _sources).  pos
 * (2, n).  With charge (n) given: sources (2, 2n) receive the n mapped charges then
 * their images conj(zeta), source_charge (2n) receives q then -q; without: sources
 * (2, n) receive the mapped points.  A point not strictly between the plates reports
 * 1 + its index in status (the caller raises the reference's ValueError). */
int td3_strip_map(const double* pos, int64_t n, double width, const double* charge,
                  double* sources, double* source_charge, int64_t* status, void* stream);

/* Field and potential in the strip from the mapped-plane sums (strip.py:228-246 and
 * :289-293): zeta (2, m) with row stride zeta_stride, phi_raw (m) and field_raw (2, m)
 * with row stride field_stride (raw E_x - i E_y = 2 W'(zeta)).  E_x - i E_y = raw (i pi /
 * width) zeta; with charge (m) given (the charges themselves) plus the own regular term
 * 2 q (i pi / 2 width) and phi = phi_raw - 2 q ln(pi |zeta| / width); without (probes)
 * phi = phi_raw.  phi is 0 when with_potential is 0.  Not yet scaled by k_e. */
int td3_strip_assemble(const double* zeta, int64_t zeta_stride, int64_t m, double width,
                       const double* charge, const double* phi_raw, const double* field_raw,
                       int64_t field_stride, int with_potential, double* phi, double* field,
                       void* stream);

/* Softening of close pairs in the physical plane, then scaling: for every target
 * (targets (2, m)) the sources (sources (2, n), charge (n)) within `radius` get the
 * softened log kernel instead of the bare one, phi += q ln(r^2 / (r^2 + eps^2)) and
 * E += q (2 / (r^2 + eps^2) - 2 / r^2) d, and then phi, field (2, m) are multiplied by
 * `scale` (phi set to 0 when with_potential is 0).  same != 0: targets are the sources
 * (a target skips itself).  A zero separation reports 1 + the target's index in status.
 * softening = 0 only scales.  Replaces soften_pairs (src/tree_d_3d/kernels/soften_pairs/
 * soften_pairs_pyccel.py:16-52) over the k-d tree pairs of strip.py:172-201, and the
 * probe correction of strip.py:296-326. */
size_t td3_soften_workspace_size(int64_t n);
int td3_soften(const double* targets, int64_t m, const double* sources, const double* charge,
               int64_t n, int same, double radius, double softening, int with_potential,
               double scale, double* phi, double* field, int64_t* status, void* workspace,
               size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ utilities */

/* Stable radix sort of (key, value) uint32 pairs by the low `bits` bits of the key.
 * The buffers ping-pong; *result_in_alt (host) tells whether the sorted pairs ended in
 * the *_alt buffers.  No reference counterpart (the reference sorts Morton keys on
 * the host with numpy.argsort, src/tree_d_3d/flat_tree.py:891-912). */
size_t td3_radix_sort_workspace_size(int64_t n);
int td3_radix_sort_pairs(uint32_t* keys, uint32_t* keys_alt, uint32_t* values,
                         uint32_t* values_alt, int64_t n, int bits, int* result_in_alt,
                         void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TREED3D_H */
