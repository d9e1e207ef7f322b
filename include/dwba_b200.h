/*
 * dwba_b200.h -- C ABI of the B200 engine for the DWBA radial matrix elements
 *
 *     I_L = sum_{i<n_rows} sum_{j<n_cols} a_i K_L(r_i, r_j) b_j ,
 *     K_L(r, r') = (1/r_>) (r_</r_>)^L      (diagonal: (1/r) (1-1e-12)^L)
 *
 * The reference (StaryPasterz/DWBA) is pure Python; its hot path is
 * dwba_matrix_elements.py:radial_ME_all_L (CPU, :780-1300) and
 * radial_ME_all_L_gpu (CuPy, :1563-2549), whose 2-D quadrature lives in
 * oscillatory_integrals.py:oscillatory_kernel_integral_2d (:2385-2777).
 * Each entry point below replaces one stage of that path; the host binding
 * (dwba_b200/dwba_matrix_elements.py) keeps the reference call signatures.
 *
 * Conventions: every pointer named *_dev is device memory; descriptor arrays
 * are device arrays of the structs below. All entry points are asynchronous
 * on the given stream, return a dwba_status code, throw nothing, and never
 * allocate device memory (scratch buffers are passed in by the caller).
 */
#ifndef DWBA_B200_H
#define DWBA_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dwba_stream_t; /* == cudaStream_t */

enum dwba_status {
  DWBA_OK = 0,
  DWBA_ERR_INVALID_ARG = 1, /* null pointer, bad size, L_max out of range (reference: ValueError) */
  DWBA_ERR_CUDA = 2,        /* CUDA launch or runtime failure */
  DWBA_ERR_NO_DEVICE = 3,   /* no usable sm_100 device (reference: RuntimeError without a GPU runtime) */
  DWBA_ERR_WORKSPACE = 4,   /* caller-provided scratch too small */
  DWBA_ERR_UNSUPPORTED = 5, /* request outside the kernel's numeric range (e.g. r^-(L+1) overflow) */
  DWBA_ERR_RANGE = 6        /* a device-side consistency check failed (status word set by a kernel) */
};

#define DWBA_ABI_VERSION 1
#define DWBA_MAX_L 63

/* ---------------------------------------------------------------------------
 * Node set: the phase-split Clenshaw-Curtis quadrature of one (k_total, n1,
 * eta, phase step) combination, folded into banded operators on the grid.
 *
 * Replaces the CC node / interpolation construction of
 *   oscillatory_integrals.py:2578-2601 (filon) and :2681-2742 (filon_exchange),
 *   oscillatory_integrals.py:279-302 (_interp_on_radial_grid).
 * Outputs:
 *   ta[3*i + d+1], i < n1, d in {-1,0,1}:  T = P1^T diag(W) P1   (outer fold, both terms)
 *   bx[5*k + d+2], k < n_grid, d in -2..2:  B = Q^T diag(W) P2   (exchange inner fold)
 * where P1/P2 interpolate (log-r on log grids) onto r[:n1] / r[:n_grid] and Q
 * interpolates kernel columns linearly in r.
 * ------------------------------------------------------------------------- */
typedef struct {
  const double* r_dev;      /* grid radii (n_grid), strictly increasing, > 0 */
  const double* logr_dev;   /* log(r) (n_grid) */
  const double* breaks_dev; /* phase breakpoints (n_breaks); NULL => linspace(r[0], r[n1-1], n_breaks) */
  double* ta_dev;           /* out: 3*n1 doubles */
  double* bx_dev;           /* out: 5*n_grid doubles */
  int32_t n_grid;
  int32_t n1;               /* idx_limit */
  int32_t n_breaks;         /* >= 2 */
  int32_t log1;             /* 1: r[:n1] passes the log-spacing test (interpolate in log r) */
  int32_t log2;             /* 1: r[:n_grid] passes the log-spacing test */
  int32_t pad;
} dwba_nodeset_t;

/* Builds the banded quadrature operators of n_sets node sets (one thread per grid
 * interval evaluates the CC nodes in (r_g, r_{g+1}] once; rows add the sums of
 * their three owners; no scratch memory).
 * cc_x_dev/cc_w_dev: Clenshaw-Curtis reference nodes/weights on [-1, 1]
 * (descending nodes, as oscillatory_integrals.py:120-171 builds them), n_cc <= 15.
 * max_grid >= every set's n_grid. status_dev: one int, set non-zero if a band
 * offset falls outside the stored band. */
int dwba_build_nodesets(const dwba_nodeset_t* sets_dev, int n_sets, int max_grid, const double* cc_x_dev,
                        const double* cc_w_dev, int n_cc, int* status_dev, dwba_stream_t stream);

/* ---------------------------------------------------------------------------
 * Fold: out[i] = sum_{d=-h..h} op[(2h+1)*i + d+h] * f[i+d] * g[i+d],  i < n_out
 * (h = 0: op is a weight vector, e.g. Simpson weights; h = 1: ta; h = 2: bx),
 * and zero for n_out <= i < n_clear.
 * Replaces the density products and weights of dwba_matrix_elements.py:1028-1046
 * together with the interpolation/CC-weight folds of the node set.
 * ------------------------------------------------------------------------- */
typedef struct {
  const double* op_dev;
  const double* f_dev;
  const double* g_dev;
  double* out_dev;
  int32_t half_band;   /* 0, 1 or 2 */
  int32_t n_out;       /* rows written with the stencil */
  int32_t n_src;       /* valid length of f, g (stencil taps outside [0, n_src) are skipped) */
  int32_t n_clear;     /* rows [n_out, n_clear) are zeroed */
} dwba_fold_t;

int dwba_fold(const dwba_fold_t* folds_dev, int n_folds, int max_rows, dwba_stream_t stream);

/* Several folds that share the operator and the second factor, in one pass:
 *   out_t[i] = sum_{d=-h..h} op[(2h+1)*i + d+h] * f_t[i+d] * g[i+d],  t < n_f <= DWBA_FOLD_MULTI,
 * with the same n_out / n_src / n_clear rules as dwba_fold. The node-set operator and the
 * continuum wave are read once for every transition of a pair (a_dir with a_ex of each
 * transition; b_ex of each transition). Same products as dwba_fold (the reference's densities,
 * dwba_matrix_elements.py:1028-1046). */
#define DWBA_FOLD_MULTI 8
typedef struct {
  const double* op_dev;
  const double* g_dev;
  const double* f_dev[DWBA_FOLD_MULTI];
  double* out_dev[DWBA_FOLD_MULTI];
  int32_t n_f;
  int32_t half_band;
  int32_t n_out;
  int32_t n_src;
  int32_t n_clear;
  int32_t pad;
} dwba_fold_multi_t;

int dwba_fold_multi(const dwba_fold_multi_t* folds_dev, int n_folds, int max_rows, dwba_stream_t stream);

/* Node sets applied at once: builds the operators of each set as dwba_build_nodesets does, but
 * instead of storing them (ta_dev / bx_dev are not used) applies them row by row to the two
 * multi-folds of the set, folds_dev[2k] (half_band 1, the set's T) and folds_dev[2k + 1]
 * (half_band 2, its B), whose op_dev fields are ignored, and writes the folds' outputs with
 * dwba_fold_multi's arithmetic (the results are bit-identical to building the set, then folding).
 * For node sets that serve a single pair: the operators never reach memory. */
int dwba_build_nodesets_folded(const dwba_nodeset_t* sets_dev, const dwba_fold_multi_t* folds_dev, int n_sets,
                               int max_grid, const double* cc_x_dev, const double* cc_w_dev, int n_cc,
                               int* status_dev, dwba_stream_t stream);

/* ---------------------------------------------------------------------------
 * Bilinear forms in FP64: for each form f and L = 0..L_max,
 *   out[f*(L_max+1) + L] = sum_{i<n_rows} sum_{j<n_cols} a_i K_L(r_i, r_j) b_j.
 * Replaces the inner/outer contractions of dwba_matrix_elements.py:1113-1116 with
 * oscillatory_integrals.py:2571/2644 (filon), :2745-2770 (filon_exchange),
 * :2479-2490 (standard) and the CuPy gemv/dot path of :2324-2513.
 * ------------------------------------------------------------------------- */
typedef struct {
  const double* r_dev;  /* grid radii */
  const double* a_dev;  /* row operand (>= n_rows) */
  const double* b_dev;  /* column operand (>= n_cols) */
  int32_t n_rows;
  int32_t n_cols;
} dwba_form_t;

/* Multipole potentials of column operands (all multipoles at once):
 *   phi[L*stride + p] = sum_{q<n_cols} K_L(r_p, r_q) b_q ,   p < n_rows, L = 0..L_max,
 * the inner integral int_r2 = K[:n1, :N] (rho2 w) of the reference's Filon direct term
 * (oscillatory_integrals.py:2571; dwba_matrix_elements.py:1126-1206 calls it per L), which depends
 * on the bound states only and is shared by every pair of a transition. Exact O(N L) FP64 with
 * forward prefix and backward suffix sums; the same range rule as dwba_bilinear_semisep_fp64. */
typedef struct {
  const double* r_dev;  /* grid radii (>= max(n_rows, n_cols)) */
  const double* b_dev;  /* column operand (n_cols values) */
  double* phi_dev;      /* out: (L_max+1) rows of `stride` doubles; p < n_rows written */
  int32_t n_rows;
  int32_t n_cols;
  int32_t stride;       /* >= n_rows */
  int32_t pad;
} dwba_potential_t;

int dwba_multipole_potentials(const dwba_potential_t* pots_dev, int n, int L_max, const double* diag_scale_host,
                              double r_min_all, double r_max_all, dwba_stream_t stream);

/* Dot forms: out[L] = sum_{i<n_rows} a[i] phi[L*stride + i], L = 0..L_max: the outer CC sum of
 * the Filon direct term (oscillatory_integrals.py:2609-2644, folded into a) against a potential
 * of dwba_multipole_potentials. Each run of 16 consecutive descriptors (descriptors 16k..16k+15)
 * must share phi_dev and stride: the kernel stages the potential's tiles in shared memory once
 * for the run. Pad a run with empty descriptors (n_rows = 0, out_dev = NULL); the first
 * descriptor of a run must not be empty unless the whole run is, and phi must hold at least the
 * largest n_rows of its run. */
typedef struct {
  const double* a_dev;
  const double* phi_dev;
  double* out_dev;      /* L_max+1 values (NULL: empty descriptor) */
  int32_t n_rows;
  int32_t stride;
} dwba_dot_t;

int dwba_dot_forms(const dwba_dot_t* dots_dev, int n, int L_max, dwba_stream_t stream);

/* ---------------------------------------------------------------------------
 * Exchange integrals with the quadrature of the reference's CuPy path (radial_ME_all_L_gpu,
 * dwba_matrix_elements.py:1563-2549; _gpu_filon_exchange :1469-1560, kernel at the CC nodes from
 * interpolated 1/r_> and log-ratio :2072-2091). Node set: linspace phase intervals on [r_0, r_{n1-1}],
 * Clenshaw-Curtis nodes, everything interpolated linearly in r on r[:n1]. The kernel at a node x in
 * (r_j, r_{j+1}] factorises per grid row i into r_i^-(L+1) G^L (i > j) or h r_i^L G^-L (i <= j), G and
 * h the geometric and harmonic interpolations of r_j, r_{j+1}; dwba_cupy_exchange_ops sums, per node
 * set, interval j and multipole, the node weights of those factors against the two interpolation
 * taps of rho2: ops[((L n1) + j) 4 + {0,1,2,3}] = sum W G^L (1-t), W G^L t, W h G^-L (1-t), W h G^-L t.
 * cc_x_dev/cc_w_dev: the CuPy path's reference CC table (:1316-1347). */
typedef struct {
  const double* r_dev;     /* grid radii (>= n1 values) */
  const double* logr_dev;  /* log r */
  double* ops_dev;         /* out: (L_max+1) x n1 x 4 doubles */
  int32_t n1;
  int32_t n_breaks;        /* breakpoints of the linspace on [r_0, r_{n1-1}] (>= 3) */
  int32_t L_max;
  int32_t pad;
} dwba_cupy_set_t;

int dwba_cupy_exchange_ops(const dwba_cupy_set_t* sets_dev, int n_sets, int max_n1, int L_max, const double* cc_x_dev,
                           const double* cc_w_dev, int n_cc, dwba_stream_t stream);

/* out[L] = sum_{i<n1} a_i [r_i^-(L+1) sum_{j<i} A_L(j) + r_i^L sum_{j>=i} B_L(j)], A_L(j), B_L(j) the ops of
 * interval j against rho2_j, rho2_{j+1} (rho2 = f g, the CuPy path's unweighted chi_f u_i on r[:n1]) and a
 * the node set's outer CC fold of rho1 (dwba_fold with the set's T): the CuPy path's exchange I_L. Exact
 * O(n1 L) FP64; the range rule of dwba_bilinear_semisep_fp64. */
typedef struct {
  const double* r_dev;
  const double* a_dev;     /* n1 values */
  const double* f_dev;     /* n1 values */
  const double* g_dev;     /* n1 values */
  const double* ops_dev;   /* the node set's dwba_cupy_exchange_ops output */
  double* out_dev;         /* L_max+1 values */
  int32_t n1;
  int32_t L_max;
} dwba_cupy_form_t;

int dwba_cupy_exchange_forms(const dwba_cupy_form_t* forms_dev, int n, int L_max, double r_min_all, double r_max_all,
                             dwba_stream_t stream);

/* Dense plain form: every K_L element is generated in registers (never stored),
 * operands are staged in shared memory, partial sums are reduced with warp
 * shuffles. Work is split into chunks (CTAs); dwba_dense_chunk_prefix fills
 * prefix_host[0..n_forms] from m_host[f] = max(n_rows, n_cols) and returns the
 * chunk total n_cta; the caller copies the prefix to chunk_prefix_dev. partial_dev
 * needs n_cta*(L_max+1) doubles. diag_scale_host[L] = (1-1e-12)^L, the factor the
 * reference's ratio clamp (dwba_matrix_elements.py:1079) puts on the diagonal. */
int64_t dwba_dense_chunk_prefix(const int32_t* m_host, int n_forms, int64_t* prefix_host);
int dwba_bilinear_dense_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max, const double* diag_scale_host,
                             const int64_t* chunk_prefix_dev, int64_t n_cta, double* partial_dev,
                             int64_t partial_cap, double* out_dev, dwba_stream_t stream);

/* Allocation-free variant of dwba_bilinear_dense_fp64. No counterpart in the
 * reference. For callers that cannot give this library scratch memory: their
 * device memory is owned by another allocator (a framework's caching pool, a
 * pool sized at start-up), or their loop must not call cudaMalloc/cudaFree,
 * which synchronise the device. Inputs and the output are still the caller's;
 * the partial sums live in a fixed array of DWBA_NOALLOC_SCRATCH_DOUBLES doubles
 * (8 MiB) inside the library, held by every GPU that loads it until exit.
 * max_m must be >= max(n_rows, n_cols) of every form (a form above it gets NaN;
 * an empty form, no rows and no columns, gets the empty sum 0); requests needing
 * more than the array, n_forms * ceil(ceil(max_m/128)/2) * (L_max+1) doubles,
 * return DWBA_ERR_WORKSPACE. The first call on a device (and the first after a
 * device reset) looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before any stream capture. All calls share the array: calls that overlap on
 * the GPU race and must be ordered by the caller (e.g. one stream). Results
 * equal dwba_bilinear_dense_fp64's (same tiles and summation order). */
#define DWBA_NOALLOC_SCRATCH_DOUBLES (1 << 20)
int dwba_bilinear_dense_fp64_noalloc(const dwba_form_t* forms_dev, int n_forms, int max_m, int L_max,
                                     const double* diag_scale_host, double* out_dev, dwba_stream_t stream);

/* Semiseparable form (exact in FP64, O(n L) per form): uses
 * K_L(r_i, r_j) = r_j^L / r_i^(L+1) for j < i. Returns DWBA_ERR_UNSUPPORTED if
 * r^-(L_max+1) or r^L could leave the normal FP64 range on [r_min_all, r_max_all]. */
int dwba_bilinear_semisep_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max,
                               const double* diag_scale_host, double r_min_all, double r_max_all,
                               double* out_dev, dwba_stream_t stream);

/* The cancellation scale of each form, S_L = sum_i sum_j |a_i| K_L(r_i, r_j) |b_j| (the same kernel on
 * |a| and |b|), which bounds the rounding error of any evaluation of the form: |dI_L| <= c S_L. No
 * reference counterpart; the split-BF16 engines use it to route forms whose cancellation exceeds
 * their FP32 accumulation to the FP64 form. Same arguments and range rule as
 * dwba_bilinear_semisep_fp64. */
int dwba_bilinear_semisep_abs_fp64(const dwba_form_t* forms_dev, int n_forms, int L_max,
                                   const double* diag_scale_host, double r_min_all, double r_max_all,
                                   double* out_dev, dwba_stream_t stream);

/* Split-BF16 tensor-core form (tcgen05.mma, TMEM accumulators, TMA-loaded operands):
 * for every form of one grid, I_L = sum_i a_i (K_L B)_i with K_L generated on the fly and
 * split into n_terms bf16 terms (2: hi+lo, three products; 3: hi+mid+lo, six products),
 * FP32 accumulation per 64-column block in TMEM and FP64 epilogue sums. Replaces the
 * exchange contraction of oscillatory_integrals.py:2745-2770 / dwba_matrix_elements.py:1469-1560
 * at reduced precision (the error is measured against the FP64 forms). All forms must share
 * r_dev (n_grid points). workspace: dwba_tc_workspace_bytes(...) bytes, 256-byte aligned.
 * status_dev: one int, zero on entry; set to 2 if a bounded wait expired (the call's
 * results are then invalid). */
int64_t dwba_tc_workspace_bytes(int n_forms, int n_grid, int L_max, int n_terms);
int dwba_bilinear_tc_bf16(const dwba_form_t* forms_dev, int n_forms, const double* r_dev, int n_grid, int L_max,
                          int n_terms, const double* diag_scale_host, void* workspace, int64_t workspace_bytes,
                          int* status_dev, double* out_dev, dwba_stream_t stream);

/* The split-BF16 form over forms on several grids in one tensor-core launch (energy points of a
 * sweep, each with its own grid; the per-energy loop of driver.py:907-1029 as one launch). Each
 * segment: its forms (all on its r_dev, n_grid points) and its result array out_dev
 * ((n_forms, L_max+1) doubles). The results of a segment are bit-identical to
 * dwba_bilinear_tc_bf16 on that segment alone, for every tile. tile (NULL: the default):
 *   bn     forms per CTA, 128 or 256 (0: 256);
 *   stages pipeline depth (0: the deepest that fits): n_terms 2: bn 256 -> 3, bn 128 -> 3 or 4;
 *          n_terms 3: bn 256 -> 2, bn 128 -> 2 or 3;
 *   order  0: the CTAs of a segment run its row blocks fastest, 1: its form blocks fastest.
 * Segments run largest grid first. workspace: dwba_tc_ragged_workspace_bytes(...) bytes,
 * 256-byte aligned. status_dev as for dwba_bilinear_tc_bf16. */
typedef struct {
  const dwba_form_t* forms_dev;
  const double* r_dev;
  double* out_dev;
  int32_t n_forms;
  int32_t n_grid;
} dwba_tc_segment_t;

typedef struct {
  int32_t bn;
  int32_t stages;
  int32_t order;
  int32_t pad;
} dwba_tc_tile_t;

int64_t dwba_tc_ragged_workspace_bytes(const dwba_tc_segment_t* segs_host, int n_segs, int L_max, int n_terms,
                                       const dwba_tc_tile_t* tile);
int dwba_bilinear_tc_bf16_ragged(const dwba_tc_segment_t* segs_host, int n_segs, int L_max, int n_terms,
                                 const dwba_tc_tile_t* tile, const double* diag_scale_host, void* workspace,
                                 int64_t workspace_bytes, int* status_dev, dwba_stream_t stream);

/* ---------------------------------------------------------------------------
 * Host helpers (no GPU work)
 * ------------------------------------------------------------------------- */
/* Coulomb-phase breakpoints r_{j+1} = r_j + dphi/|k + eta/r_j| (bounded steps),
 * exactly as oscillatory_integrals.py:1677-1710 (generate_phase_nodes, eta != 0).
 * Writes at most cap values; *n_out = count (<= 10002). */
int dwba_phase_breaks_coulomb(double r_start, double r_end, double k_total, double dphi, double eta_total,
                              double* out_host, int cap, int* n_out);

/* Outer tail of the direct integral for L = 1..L_max of one pair (0 for L = 0):
 * tail[L] = dwba_outer_integral_1d(M_L / r^(L+1), r_m .. r_max) + analytical r_max->inf tail
 * (oscillatory_integrals.py:459-535, :1361-1451, :2064-2184; call site
 * dwba_matrix_elements.py:1213-1241). moments_host[L] = sum w r^L u_f u_i;
 * an entry with |M_L| <= 1e-12 gives 0. mode: 0 = advanced/full_split, 1 = legacy
 * (analytical tail from r_m only). wave_host = {k_i, l_i, delta_i, eta_i, sigma_i,
 * k_f, l_f, delta_f, eta_f, sigma_f}. */
int dwba_outer_tails(const double* wave_host, double r_m, double r_max, int L_max, const double* moments_host,
                     int mode, int max_filon_segments, double max_effective_dphi, double* tail_host);

/* ---------------------------------------------------------------------------
 * Backward (no reference counterpart: the reference computes no gradients).
 * For each form with upstream gradients g[f*(L_max+1) + L] = dLoss/dI_f,L of the forward
 * I_f,L = a_f^T K_L b_f (dwba_bilinear_semisep_fp64 / dwba_bilinear_dense_fp64):
 *   ga_f = K_g b_f  (n_rows values),  gb_f = K_g a_f  (n_cols values),  K_g = sum_L g_L K_L,
 * i.e. dLoss/da_f and dLoss/db_f (K_L is symmetric). Exact O(n L) FP64; the same range rule as
 * dwba_bilinear_semisep_fp64 (DWBA_ERR_UNSUPPORTED when r^L or r^-(L+1) would leave FP64).
 * ------------------------------------------------------------------------- */
typedef struct {
  const double* r_dev;
  const double* a_dev;
  const double* b_dev;
  double* ga_dev;       /* out, n_rows values */
  double* gb_dev;       /* out, n_cols values */
  int32_t n_rows;
  int32_t n_cols;
} dwba_form_grad_t;

int dwba_bilinear_semisep_backward_fp64(const dwba_form_grad_t* forms_dev, int n_forms, int L_max,
                                        const double* diag_scale_host, const double* grad_dev, double r_min_all,
                                        double r_max_all, dwba_stream_t stream);

/* The same gradients through the split-BF16 tensor-core form (no reference counterpart):
 * ga_f = sum_L g_L (K_L b_f), gb_f = sum_L g_L (K_L a_f), each K_L B product on tcgen05 with
 * K_L and the operand split into n_terms bf16 terms and FP32 accumulation (as
 * dwba_bilinear_tc_bf16), the g_L weighting and the sum over L in FP64. All forms share r_dev
 * (n_grid points). workspace: dwba_tc_backward_workspace_bytes(...) bytes, 256-byte aligned.
 * status_dev: one int, zero on entry; set to 2 if a bounded wait expired (the gradients are then
 * invalid). */
int64_t dwba_tc_backward_workspace_bytes(int n_forms, int n_grid, int L_max, int n_terms);
int dwba_bilinear_tc_bf16_backward(const dwba_form_grad_t* forms_dev, int n_forms, const double* r_dev, int n_grid,
                                   int L_max, int n_terms, const double* diag_scale_host, const double* grad_dev,
                                   void* workspace, int64_t workspace_bytes, int* status_dev, dwba_stream_t stream);

/* Bound of every pipeline wait of the tensor-core kernels (dwba_bilinear_tc_bf16, its ragged form
 * and its backward)
 * launched after this call, in SM clock cycles; 0 restores the default (about one second). No
 * reference counterpart: it lets a test make a wait run out on a normal input. A wait that runs
 * out sets the call's status word to 2; its CTA then waits, with the default bound, for its own
 * copies and products in flight, frees its tensor memory and returns, and CTAs that start after
 * the status was set skip their work, so the next call runs normally. The setting is process-wide
 * and read when a call launches. */
int dwba_tc_set_wait_cycles(int64_t cycles);

/* Adjoint of dwba_fold: z = Op^T y for the banded operator of a fold (same op layout), i.e.
 * dLoss/d(f .* g) for y = dLoss/d(out). z gets n_src values. No reference counterpart. */
typedef struct {
  const double* op_dev;
  const double* y_dev;  /* >= n_out values */
  double* z_dev;        /* out, n_src values */
  int32_t half_band;
  int32_t n_out;
  int32_t n_src;
  int32_t pad;
} dwba_fold_adj_t;

int dwba_fold_adjoint(const dwba_fold_adj_t* adj_dev, int n, int max_len, dwba_stream_t stream);

/* Amplitudes -> DCS -> TCS for many partial-wave channels of one transition (replaces the
 * per-channel loop of driver.py:1036-1052 over calculate_amplitude_contribution,
 * dwba_coupling.py:285-505, and dcs_dwba / integrate_dcs_over_angles, sigma_total.py:147-217).
 * cf, cg: complex (re, im) coefficient tables [n_M][P][nl]; yd, ye: angular factors
 * [n_M][P][n_theta]; I_dir, I_exc: [P][nl]; dcs: [n_theta]; tcs: one value (may be NULL). */
int dwba_cross_sections(const double* cf_dev, const double* cg_dev, const double* yd_dev, const double* ye_dev,
                        const double* I_dir_dev, const double* I_exc_dev, const double* theta_dev, int n_M, int P,
                        int nl, int n_theta, double pref, double* dcs_dev, double* tcs_dev, dwba_stream_t stream);

/* Outer tails on the GPU, one warp per (record, L): the same quantity and formulas as
 * dwba_outer_tails (Filon / Levin segments split across the lanes, compensated lane sums).
 * Records whose mid-interval frequency is below 1e-10 take the reference's adaptive-quadrature
 * branch and must go to dwba_outer_tails instead: dwba_outer_tail_on_device returns 0 for them.
 * out_dev[L] of each record receives tail[L] for L = 0..L_max (tail[0] = 0). */
typedef struct {
  double wave[10];            /* k_i, l_i, delta_i, eta_i, sigma_i, k_f, l_f, delta_f, eta_f, sigma_f */
  double r_m, r_max;
  const double* moments_dev;  /* M_L, L = 0..L_max */
  double* out_dev;            /* tail[L], L = 0..L_max */
  int32_t mode;               /* 0: advanced/full_split, 1: legacy */
  int32_t pad;
} dwba_tail_t;

int dwba_outer_tails_batch(const dwba_tail_t* tails_dev, int n, int L_max, int max_filon_segments,
                           double max_effective_dphi, dwba_stream_t stream);
int dwba_outer_tail_on_device(const double* wave_host, double r_m, double r_max);

/* Copy nbytes from page-locked host memory (allocated with cudaHostAlloc / cudaMallocHost, so that
 * the device can address it) into device memory with a kernel on `stream` instead of the copy
 * engines. No counterpart in the reference (its descriptors are CuPy arrays); the engine uses it for
 * the small descriptor arrays a call builds while the call's large wave transfer occupies the copy
 * engines, which would otherwise queue them behind it. Returns DWBA_ERR_INVALID_ARG when the
 * source is not mapped page-locked host memory or the destination not device memory (checked at
 * both ends of each range; like every entry point here, the extents are the caller's to get right).
 * The host memory must stay unchanged until the copy has run on the stream. */
int dwba_copy_from_host(void* dst_dev, const void* src_host, int64_t nbytes, dwba_stream_t stream);

/* Library identity and device probe (the check_cupy_runtime analogue, dwba_matrix_elements.py:178-193). */
int dwba_abi_version(void);
const char* dwba_status_string(int status);
int dwba_device_probe(int* n_devices, int* cc_major, int* cc_minor);
/* sizeof(dwba_nodeset_t), sizeof(dwba_fold_t), sizeof(dwba_form_t), sizeof(dwba_tail_t),
 * sizeof(dwba_form_grad_t), sizeof(dwba_fold_adj_t), sizeof(dwba_fold_multi_t),
 * sizeof(dwba_potential_t), sizeof(dwba_dot_t), sizeof(dwba_cupy_set_t), sizeof(dwba_cupy_form_t),
 * sizeof(dwba_tc_segment_t), sizeof(dwba_tc_tile_t) into sizes[0..12] (the first n of them). */
int dwba_struct_sizes(int64_t* sizes, int n);

#ifdef __cplusplus
}
#endif
#endif /* DWBA_B200_H */
