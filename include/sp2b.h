/*
 * sp2b - B200-native SP2 density-matrix purification (C ABI).
 *
 * Raw-pointer core API.  Every entry point returns an int status (SP2B_OK = 0)
 * instead of terminating the process the way the reference's Fortran `stop` does
 * (src/prg_sp2_mod.F90:118,362).  Matrices are dense FP64, n x n, column-major
 * (the Fortran / BML dense convention), and symmetric (a Hamiltonian): the library
 * relies on H = H^T and returns an exactly symmetric density matrix.  Host-pointer
 * calls copy only the elements at offsets i*n + j with j >= i (in Fortran's column-major
 * terms the lower triangle, H(j+1, i+1) with j >= i) to the device and rebuild the rest
 * from them; device-pointer calls read the whole matrix.  rho is the
 * spin-summed density, 2x the idempotent projector (src/prg_sp2_mod.F90:375).
 *
 * Matrix arguments (H, rho, the CSR arrays and halo lists of the sub-graph call) are
 * host pointers unless sp2b_opts.device_ptrs = 1, in which case they are device
 * pointers on the current CUDA device and the work runs on sp2b_opts.stream.  The
 * short sequence arrays pp, vv and icount are host pointers in every mode.  Calls
 * return after their results are complete.
 *
 * The PROGRESS-named exports (prg_sp2_alg2, ...) with the reference's exact C
 * signatures are declared in prg_sp2b.h.
 */
#ifndef SP2B_H
#define SP2B_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define SP2B_OK 0
#define SP2B_NOT_CONVERGED 1 /* reference: "SP2 purification is not converging: STOP!" */
#define SP2B_BAD_ARG 2
#define SP2B_CUDA_ERROR 3
#define SP2B_TIMEOUT 4       /* a bounded device-side wait ran out */
#define SP2B_BAD_INPUT 5     /* NaN / Inf in the input or during the iteration */
#define SP2B_NO_DEVICE 6

/* Arithmetic of the SP2 squarings. */
#define SP2B_PREC_FP64 0        /* FP64 products and sums: parity form (1e-10) */
#define SP2B_PREC_MIXED_FP16 1  /* FP16 hi+lo split products on tcgen05, FP32 accumulate,
                                   FP64 traces, final FP64 McWeeny step */
#define SP2B_PREC_MIXED_BF16 2  /* same with BF16 hi+lo operands */
#define SP2B_PREC_EXACT_INT8 3  /* every SP2 step's X^2 from exact integer products on the
                                   INT8 tensor cores.  Dense entries: X rounded to 2^-S
                                   (S ~ 35) and squared exactly from residue products, X
                                   kept in FP64; stops on the alg2 rule or when
                                   Tr(X - X^2) stagnates; no McWeeny step.  Sub-graph
                                   entry: X - I/2 held in fixed point on the 2^-31 grid as
                                   four 8-bit digits, X^2 from 13 exact digit products
                                   (terms below ~2^-36 dropped), one rounding per step. */

/* Products of the McWeeny refinement that ends a mixed solve. */
#define SP2B_MCW_INT8 0  /* X^2 exact from INT8 residue products (tcgen05 kind::i8) and CRT,
                            rounded to 2^-S with S ~ 35; correction X (X^2 - X) split
                            precision.  Used for mcweeny = 1 (default). */
#define SP2B_MCW_FP64 1  /* both products FP64 (DMMA).  Always used for mcweeny > 1. */

typedef struct sp2b_opts {
  int precision;     /* SP2B_PREC_* (default FP64) */
  int mcweeny;       /* mixed only: FP64 McWeeny steps after the loop (default 1) */
  double mixed_tol;  /* mixed only: stop after the update whose product gave
                        Tr X - Tr X^2 < mixed_tol (default 1e-3) */
  int device_ptrs;   /* 1: matrix arguments are device pointers */
  void* stream;      /* cudaStream_t to run on (NULL: the per-library stream) */
  int verbose;
  int mcweeny_products; /* mixed only: SP2B_MCW_* (default SP2B_MCW_INT8) */
  double refine_tol; /* sub-graph mixed only: parts whose core rows end with
                        sum (X - X^2)_ii > refine_tol are solved again in FP64
                        (default 1e-3; <= 0 turns this off) */
  int exact_switch;  /* dense mixed only: a nearly gapless input, whose split-precision
                        loop is still running after exact_switch steps or stops on the
                        stagnation test (its products cannot resolve the states at the
                        chemical potential), is solved again from H in the exact INT8
                        form, which follows the FP64 recursion; the outputs are those of
                        the exact solve (default 40; 0 turns this off) */
} sp2b_opts;

/* Fill opts with defaults (FP64, host pointers). */
int sp2b_opts_default(sp2b_opts* opts);

/* Options used by the PROGRESS-named exports (prg_sp2b.h).  Initialised from the
 * environment variable SP2B_PRECISION ("fp64", "mixed", "mixed_bf16", "exact") on
 * first use. */
int sp2b_set_default_opts(const sp2b_opts* opts);
int sp2b_get_default_opts(sp2b_opts* opts);

/* 1 when the last dense solve of this thread started in split precision and was solved
 * again in the exact INT8 form (sp2b_opts.exact_switch), else 0. */
int sp2b_last_exact_switch(void);

/* Message describing the last non-OK status of this thread. */
const char* sp2b_last_error(void);

/* ---- dense SP2 (replaces src/prg_sp2_mod.F90) --------------------------------------- */

/* prg_sp2_alg2, src/prg_sp2_mod.F90:263-380.  iters_out (may be NULL) = SP2 steps taken.
 * `threshold` is accepted for signature parity; dense products are not thresholded. */
int sp2b_sp2_alg2(const double* h, double* rho, int n, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                  int verbose, const sp2b_opts* opts, int* iters_out);

/* prg_sp2_alg2_genseq, src/prg_sp2_mod.F90:395-533.  pp, vv: length >= maxsp2iter. */
int sp2b_sp2_alg2_genseq(const double* h, double* rho, int n, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                         int* pp, int* icount, double* vv, int verbose, const sp2b_opts* opts);

/* prg_sp2_alg2_seq, src/prg_sp2_mod.F90:543-627: replay pp(1:icount). */
int sp2b_sp2_alg2_seq(const double* h, double* rho, int n, double threshold, const int* pp,
                      int icount, double* vv, int verbose, const sp2b_opts* opts);

/* prg_prg_sp2_alg2_seq_inplace, src/prg_sp2_mod.F90:638-722: rho holds H on entry. */
int sp2b_sp2_alg2_seq_inplace(double* rho, int n, double threshold, const int* pp, int icount,
                              double* vv, double mineval, double maxeval, int verbose,
                              const sp2b_opts* opts);

/* prg_sp2_alg1, src/prg_sp2_mod.F90:734-864. */
int sp2b_sp2_alg1(const double* h, double* rho, int n, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                  int verbose, const sp2b_opts* opts, int* iters_out);

/* prg_sp2_alg1_genseq, src/prg_sp2_mod.F90:879-1000. */
int sp2b_sp2_alg1_genseq(const double* h, double* rho, int n, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                         int* pp, int* icount, double* vv, const sp2b_opts* opts);

/* prg_sp2_alg1_seq, src/prg_sp2_mod.F90:1010-1089. */
int sp2b_sp2_alg1_seq(const double* h, double* rho, int n, double threshold, const int* pp,
                      int icount, double* vv, const sp2b_opts* opts);

/* prg_prg_sp2_alg1_seq_inplace, src/prg_sp2_mod.F90:1100-1177. */
int sp2b_sp2_alg1_seq_inplace(double* rho, int n, double threshold, const int* pp, int icount,
                              double* vv, double mineval, double maxeval, const sp2b_opts* opts);

/* prg_sp2_basic, src/prg_sp2_mod.F90:49-135. */
int sp2b_sp2_basic(const double* h, double* rho, int n, double threshold, double bndfil,
                   int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                   int verbose, const sp2b_opts* opts, int* iters_out);

/* prg_sp2_submatrix_inplace, src/prg_sp2_mod.F90:1259-1310: vv(1:icount) is
 * ACCUMULATED with the sum of squares of (X - X^2) over the first core_size rows. */
int sp2b_sp2_submatrix_inplace(double* rho, int n, double threshold, const int* pp, int icount,
                               double* vv, double mineval, double maxeval, int core_size,
                               const sp2b_opts* opts);

/* No counterpart in the reference.  The same SP2 on one core+halo block as
 * sp2b_sp2_submatrix_inplace, for callers that must not allocate GPU memory when they
 * call it: typically a simulation code that reserves its device memory up front in its
 * own pool allocator (a library cudaMalloc would fail or break the pool's accounting),
 * or a time-step loop that may not stall on cudaMalloc / cudaFree, which synchronise
 * the device.  It calls no cudaMalloc / cudaFree / allocating library routine: its
 * working buffers live in one fixed device array (about 4.2 MB, held by every GPU that
 * loads the library until exit).  x_dev is a DEVICE pointer to the n x n block (H in,
 * rho out); pp and vv (accumulated, as in the reference; untouched when core_size is 0)
 * are host arrays; work runs on `stream`.  Limits: n <= 512 and icount <= 100,
 * otherwise SP2B_BAD_ARG.  All calls share the one array and it keeps the last call's
 * contents, so calls whose GPU work overlaps race; the first call on a device looks up
 * the array's address and should come before any stream capture. */
int sp2b_sp2_submatrix_inplace_noalloc(double* x_dev, int n, const int* pp, int icount,
                                       double* vv, double mineval, double maxeval, int core_size,
                                       void* stream);

/* prg_sp2_submatrix, src/prg_sp2_mod.F90:1190-1246 (separate input H). */
int sp2b_sp2_submatrix(const double* ham, double* rho, int n, double threshold, const int* pp,
                       int icount, double* vv, double mineval, double maxeval, int core_size,
                       const sp2b_opts* opts);

/* ---- normalisation and checks ----------------------------------------------------- */

/* bml_gershgorin as used by prg_normalize (src/prg_normalize_mod.F90:41). */
int sp2b_gershgorin(const double* h, int n, double* mineval, double* maxeval,
                    const sp2b_opts* opts);

/* prg_normalize, src/prg_normalize_mod.F90:32-46: h <- (e_max I - h)/(e_max - e_min). */
int sp2b_normalize(double* h, int n, double* mineval, double* maxeval, const sp2b_opts* opts);

/* prg_check_idempotency, src/prg_densitymatrix_mod.F90:862-880: ||A^2 - A||_F. */
int sp2b_check_idempotency(const double* a, int n, double threshold, double* idempotency,
                           const sp2b_opts* opts);

/* ---- host-side graph / sequence logic (no GPU) ------------------------------------ */

/* prg_sp2sequence, src/prg_homolumo_mod.F90:97-147.  pp has room for ppmax (>= 100). */
int sp2b_sp2sequence(int* pp, int* imax, double mineval, double maxeval, double ehomo,
                     double elumo, double errlimit, int ppmax);

/* prg_homolumogap, src/prg_homolumo_mod.F90:22-89 (imax is the 1-based count). */
int sp2b_homolumogap(const double* vv, int imax, const int* pp, double mineval, double maxeval,
                     double* ehomo, double* elumo, double* egap);

/* prg_equalPartition, src/prg_graph_mod.F90:359-399.  part_ptr has nparts+1 entries,
 * nodes has nnodes entries (0-based node ids, part i = nodes[part_ptr[i]:part_ptr[i+1]]).
 * Call with part_ptr = NULL to query nparts. */
int sp2b_equal_partition(int nodes_per_part, int nnodes, int* nparts, int* part_ptr,
                         int* nodes);

/* Core+halo index of each part (bml_matrix2submatrix_index as called at
 * src/prg_subgraphloop_mod.F90:60-63).  Graph and H are CSR (row_ptr n+1 int64,
 * col int32); h_* may be NULL.  Output: halo_ptr (nparts+1) and halo_idx (capacity
 * halo_cap; core nodes first), core sizes in llsize, total sizes in lsize.  Returns
 * SP2B_BAD_ARG with the needed capacity in *halo_needed when halo_cap is too small. */
int sp2b_subgraph_halos(int n, const long long* g_row_ptr, const int* g_col,
                        const long long* h_row_ptr, const int* h_col, int nparts,
                        const int* part_ptr, const int* part_nodes, int double_jump,
                        long long* halo_ptr, int* halo_idx, long long halo_cap,
                        long long* halo_needed, int* lsize, int* llsize);

/* ---- SP2-Fermi (replaces src/prg_sp2_fermi_mod.F90), FP64 ------------------------ */

/* prg_sp2_fermi_init, src/prg_sp2_fermi_mod.F90:43-177.  Gershgorin bounds give
 * h1 = tscale*min, hN = tscale*max and the first mu; each pass normalises
 * X0 = ((hN - mu) I - H)/(hN - h1) and runs nsteps SP2 steps, the first pass choosing
 * sgnlist[i] (1: X <- 2X - X^2, -1: X <- X^2) from the traces, later passes replaying it,
 * with X1 = dX/dmu carried along; Newton steps on mu until |nocc - Tr X| <= occ_err_limit;
 * beta = -Tr X1 / Tr X(I - X) (-1000 when that trace is below trace_limit).  x receives X
 * of the last pass (occupations in [0, 1], not 2X).  Host or device pointers for h and x
 * per opts.device_ptrs; sgnlist (nsteps) and the scalars are host memory. */
int sp2b_sp2_fermi_init(const double* h, int n, int nsteps, double nocc, double tscale,
                        double threshold, double occ_err_limit, double trace_limit, double* x,
                        double* mu, double* beta, double* h1, double* hN, int* sgnlist,
                        const sp2b_opts* opts);

/* prg_sp2_fermi, src/prg_sp2_fermi_mod.F90:388-470: passes of X0 = ((hN - mu) I - H)/
 * (hN - h1) and the nsteps steps of sgnlist, each followed by a Newton step on mu with
 * DX = -beta X (I - X); osteps passes, or (osteps = 0) until |nocc - Tr X| <= eps.
 * x = X + lambda DX with the last pass's lambda; mu is updated in place. */
int sp2b_sp2_fermi(const double* h, int n, int osteps, int nsteps, double nocc, double* mu,
                   double beta, double h1, double hN, const int* sgnlist, double threshold,
                   double eps, double trace_limit, double* x, const sp2b_opts* opts);

/* prg_sp2_fermi_init_norecs, src/prg_sp2_fermi_mod.F90:198-372: as sp2b_sp2_fermi_init,
 * but *beta enters as the target inverse temperature and *nsteps as the most steps; the
 * recursion ends at the first step whose probe temperature (the steepest slope of the
 * sequence applied to the grid 0.999, 0.998, ..., 0, times 4/(max - min), :256-310)
 * exceeds it, which is returned in *nsteps with sgnlist[0 .. *nsteps - 1]. */
int sp2b_sp2_fermi_init_norecs(const double* h, int n, int* nsteps, double nocc, double tscale,
                               double threshold, double occ_err_limit, double trace_limit,
                               double* x, double* mu, double* beta, double* h1, double* hN,
                               int* sgnlist, const sp2b_opts* opts);

/* prg_sp2_entropy_function, src/prg_sp2_fermi_mod.F90:482-532: the SP2 entropy function
 * GG on the mesh ee = 0, 1e-4, ..., 1 (10001 points), the running two-point Gauss-Legendre
 * integral of the inverse SP2 map (sp2_inverse, :592-611) minus GG(end) ee.  Writes the
 * first npoints (1..10001) entries of gg and ee; host memory, host arithmetic (a table of
 * scalars, as in the reference). */
int sp2b_sp2_entropy_function(double mu, double h1, double hN, int nsteps, const int* sgnlist,
                              double* gg, double* ee, int npoints);

/* ---- Launch-configuration autotuner ---------------------------------------------------
 * The first solve of a new shape on a device times the equivalent launch configurations of
 * its step kernel with CUDA events and keeps the fastest:
 *   "f64-step/sm<S>/np<np>"          dense FP64 step tile edge, 128 or 64;
 *   "subgraph/f64/sm<S>/<np>x<k>,..." batched FP64 sub-graph tile edge, 64 or 32;
 *   "subgraph/split/sm<S>/<np>x<k>,..." batched split tile order, 0 (largest parts first) or
 *                                     1 (every other wave reversed: balanced over the CTAs).
 * (<np>x<k>: k parts of padded size np.)  The candidates compute the same products (same k
 * order per element; independent tiles), so a choice changes speed, not results, except
 * the order in which the per-iteration sums vv of a split batch are added.  SP2B_TUNE=0
 * keeps the built-in rules; SP2B_TUNE_FILE=path is read on first use and appended to.
 * sp2b_tune_set records a choice (it applies to solves that start afterwards);
 * sp2b_tune_get returns SP2B_BAD_ARG for an unknown key; sp2b_tune_keys writes the keys,
 * one per line, and returns the length needed including the terminator. */
int sp2b_tune_get(const char* key, int* choice, float* ms, int max_ms, int* nms);
int sp2b_tune_set(const char* key, int choice);
int sp2b_tune_keys(char* buf, int cap);
int sp2b_tune_clear(void);

/* ELLPACK -> CSR, the sparse input of the sub-graph calls and of the graph builder.
 * ELLPACK as BML stores it on the C side (bml_matrix_ellpack): width m, row i's entries
 * at [i*m, i*m + nnz[i]) of idx (0-based columns) and val.  Output: row_ptr (n+1, int64),
 * col (int32) and csr_val, capacity cap.  Returns SP2B_BAD_ARG with the needed capacity
 * in *needed (row_ptr filled) when col / csr_val are NULL or too small, SP2B_BAD_INPUT
 * for nnz[i] outside [0, m] or a column outside [0, n).  Host pointers: converted on the
 * host; device pointers (opts.device_ptrs): one warp per row on the GPU, ordered on
 * opts.stream. */
int sp2b_ellpack_to_csr(int n, int m, const int* nnz, const int* idx, const double* val,
                        long long* row_ptr, int* col, double* csr_val, long long cap,
                        long long* needed, const sp2b_opts* opts);

/* Graph of the sub-graph loop on the GPU: the pattern of |H^2| > gthreshold (the H^2
 * graph the sub-graph benchmark partitions,
 * benchmarks/dmconstruction_graphBased/dmconstruction_graphBased.F90:63-65, formed there
 * with a BML sparse product and a threshold).  H is CSR (row_ptr int64 [n+1], col int32,
 * val FP64); each G_ij = sum_k H_ik H_kj is summed in the order of row i's entries with
 * separately rounded products and sums.  Output: g_row_ptr (n+1) and g_col (capacity
 * g_cap), columns ascending in each row, the diagonal kept when above the threshold.
 * Returns SP2B_BAD_ARG with the needed capacity in *g_needed (g_row_ptr filled) when
 * g_col is NULL or too small, SP2B_BAD_INPUT when a row of H^2 has more than 2048
 * candidate columns.  Host or device pointers per opts.device_ptrs. */
int sp2b_graph_square_threshold(int n, const long long* h_row_ptr, const int* h_col,
                                const double* h_val, double gthreshold, long long* g_row_ptr,
                                int* g_col, long long g_cap, long long* g_needed,
                                const sp2b_opts* opts);

/* ---- graph-partitioned SP2 (replaces prg_subgraphSP2Loop) ------------------------- */

/* prg_subgraphSP2Loop, src/prg_subgraphloop_mod.F90:36-126, flattened (the reference
 * has no C binding: graph_partitioning_t is not interoperable).
 *
 * H is CSR (row_ptr int64 [n+1], col int32, val FP64).  Parts are given by their
 * core+halo index lists (halo_ptr/halo_idx, core first, llsize[p] core nodes).  All
 * parts run the same branch sequence pp(1:maxiter) with the global bounds
 * mineval/maxeval.  Outputs:
 *   rho_core  packed core rows: part p's llsize[p] x lsize[p] block (row-major, row r
 *             = node halo_idx[halo_ptr[p]+r], column c = node halo_idx[halo_ptr[p]+c])
 *             at offset rho_off[p] = sum_{q<p} llsize[q]*lsize[q];
 *   rho_dense optional dense n x n output (may be NULL), core rows filled, rest zero;
 *   vv        maxiter sums over all parts' core rows of (X - X^2)^2, already passed
 *             through sqrt as prg_fnormGraph does (src/prg_graph_mod.F90:933-971).
 * Host or device pointers per opts.device_ptrs.
 *
 * Precisions: FP64 (parity), MIXED_FP16 / MIXED_BF16 (hi + lo split products), and
 * EXACT_INT8 (the INT8 digit form: within ~1e-7 relative Frobenius of FP64 on nearly
 * gapless lattices, where the hi + lo split ends ~1e-5 away).  In the non-FP64 forms a
 * part whose final iterate still has a state half-way between occupied and empty
 * (core-row sum of (X - X^2)_ii above opts.refine_tol) is one whose density depends on
 * rounding far below the products' (a level within ~1e-5 of the chemical potential);
 * those parts are solved again in FP64 and their rows replaced, so they equal the FP64
 * call's.  vv stays that of the first solve.  A part with llsize 0 contributes to
 * neither output and is not solved. */
int sp2b_subgraph_sp2_loop(int n, const long long* h_row_ptr, const int* h_col,
                           const double* h_val, int nparts, const long long* halo_ptr,
                           const int* halo_idx, const int* llsize, const int* pp, int maxiter,
                           double mineval, double maxeval, double* rho_core,
                           double* rho_dense, double* vv, const sp2b_opts* opts);

/* Parts the last sp2b_subgraph_sp2_loop call of this thread solved again in FP64:
 * their number in *count, the first max_parts indices in parts (may be NULL), and the
 * core-row idempotency sums of every part of that call in idem (nparts entries; may be
 * NULL; zeros for FP64 calls). */
int sp2b_last_subgraph_refined(int* count, int* parts, int max_parts, double* idem,
                               int nparts);

/* Assembly step of the multi-rank sub-graph loop (prg_collectMatrixFromParts,
 * src/prg_subgraphloop_mod.F90:132-161), on the device: part p's packed core rows
 * (llsize[p] x lsize[p], lsize[p] = halo_ptr[p+1] - halo_ptr[p], row-major, as
 * sp2b_subgraph_sp2_loop packs them) at src + src_off[p] are written into the dense
 * column-major n x n rho (entry (halo_idx[halo_ptr[p]+r], halo_idx[halo_ptr[p]+c])).
 * All pointers are DEVICE pointers; work runs on `stream`; elements of rho outside the
 * core rows are left as they are. */
int sp2b_place_core_rows(long long n, int nparts, const long long* halo_ptr, const int* halo_idx,
                         const int* llsize, const long long* src_off, const double* src,
                         double* rho, void* stream);

/* ---- device-resident building blocks (used by the torch binding) ------------------ */

/* Split-precision symmetric-operand product on device arrays:
 * C = A * B with A, B symmetric n x n FP32 (row- or column-major, same thing),
 * computed as hi/lo FP16 tcgen05 products with FP32 accumulation. */
int sp2b_dev_sym_gemm_f32(const float* a, const float* b, float* c, int n, void* stream);

/* Row panel of a product with a symmetric right operand, for the row-block distributed
 * dense SP2 (each rank forms its rows of X^2; the reference's DO_MPI_BLOCK loop,
 * src/prg_sp2_mod.F90:263-380 with :312-317 and :365-370): C (m x n, row pitch n) =
 * A_rows (m x n, row pitch n) * B (n x n, symmetric), m <= n, device FP32 arrays on
 * `stream`, hi/lo FP16 tcgen05 products with FP32 accumulation. */
int sp2b_dev_panel_gemm_f32(const float* a_rows, int m, const float* b, int n, float* c,
                            void* stream);

/* Differentiable SP2 (the autograd path), device FP32 n x n arrays on `stream`.  These
 * have no single counterpart in the reference: they are the pieces of a reverse-mode
 * derivative of the SP2 recursion whose forward-mode form is prg_compute_response_SP2
 * (src/prg_response_mod.F90:653-782).
 *   normalize:    x = (maxeval I - h)/(maxeval - mineval)
 *   sp2_step:     y = x^2 (branch 1) or 2x - x^2 (branch 0), split-precision products
 *   adjoint_step: g_out = {g, x} (branch 1) or 2g - {g, x} (branch 0), {g,x} = gx + xg,
 *                 `work` is an n x n scratch array. */
int sp2b_dev_normalize_f32(const float* h, float* x, int n, double mineval, double maxeval,
                           void* stream);
int sp2b_dev_sp2_step_f32(const float* x, float* y, int n, int branch, void* stream);
int sp2b_dev_adjoint_step_f32(const float* g, const float* x, float* g_out, float* work, int n,
                              int branch, void* stream);

/* The same steps with X and G kept in the FP16 hi + lo split form between steps (lo
 * scaled by 2^11; x = hi + 2^-11 lo), so no conversion runs between products.  Each
 * split matrix is two np x np half arrays (hi, lo), np = sp2b_split_dim(n), row pitch
 * np, zeros outside the n x n block (every entry below writes the padding).
 *   normalize_split:    split X_0 = (maxeval I - h)/(maxeval - mineval) from FP32 h
 *   f32_to_split / split_to_f32: conversions; split_to_f32 writes y = scale x (n x n)
 *   sp2_step_split:     y = x^2 (branch 1) or 2x - x^2 (branch 0); one symmetric
 *                       product whose epilogue writes the split y (y must not alias x)
 *   adjoint_step_split: o = {g, x} (branch 1) or 2g - {g, x} (branch 0), g and x
 *                       symmetric, formed as one symmetric product over the
 *                       concatenated K range [g | x][x | g]^T with the branch in its
 *                       epilogue when np is a multiple of 256 (else g x in FP32 and a
 *                       combine pass); o must not alias g or x. */
int sp2b_split_dim(int n);
int sp2b_dev_normalize_split(const float* h, int n, double mineval, double maxeval, void* x_hi,
                             void* x_lo, void* stream);
int sp2b_dev_f32_to_split(const float* a, int n, void* hi, void* lo, void* stream);
int sp2b_dev_split_to_f32(const void* hi, const void* lo, int n, double scale, float* y,
                          void* stream);
int sp2b_dev_sp2_step_split(const void* x_hi, const void* x_lo, void* y_hi, void* y_lo, int n,
                            int branch, void* stream);
int sp2b_dev_adjoint_step_split(const void* g_hi, const void* g_lo, const void* x_hi,
                                const void* x_lo, void* o_hi, void* o_lo, int n, int branch,
                                void* stream);

/* ---- diagnostics ------------------------------------------------------------------ */

/* State of the last dense solve on the current device: SP2 step launches issued by
 * the host, X updates applied, Fortran iteration count, status; and, if recs != NULL,
 * up to max_recs control records as 9 doubles each
 * {trx, trx_data, fro2, idemperr, iter, done, status, last_branch, trp}; record k + 1
 * holds the sums of X_{k+1} and trp = Tr X_k^2 as step k computed it. */
int sp2b_last_solve_info(int* launches, int* nupd, int* iter, int* status, double* recs,
                         int max_recs);

/* Kernel launches issued by this library since load (all kernels, all devices), and
 * the device time of the SP2 step kernels recorded with CUDA events when
 * sp2b_set_step_timing(1) is on (ms, number of timed launches). */
long long sp2b_launch_count(void);

/* First-order density response by SP2 (forward mode): prg_compute_response_SP2
 * (src/prg_response_mod.F90:653-782), in the reference's argument order (ham, prt, rsp,
 * rho, lambda, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol, threshold, verbose).
 * X follows the alg2 branch rule (no iteration decrement on the break branch, as there),
 * Delta_0 = alpha H1, Delta <- {X, Delta} or 2 Delta - {X, Delta} with X's branch;
 * rho = 2 X, rsp = 2 Delta.  FP64 on the DMMA path whatever opts->precision says: each
 * anticommutator is two upper-tile products (3 N^3 flops per iteration with X^2, the
 * reference spends three full products).  lambda and threshold are unused (as in the
 * reference's dense path); pp (length >= maxsp2iter) receives the applied branches and
 * icount their number (either may be NULL). */
int sp2b_compute_response_sp2(const double* h0, const double* h1, double* rsp, double* rho, int n,
                              double lambda, double bndfil, int minsp2iter, int maxsp2iter,
                              const char* sp2conv, double idemtol, double threshold,
                              int verbose, int* pp, int* icount, const sp2b_opts* opts);

/* Scale exponent S and largest squared row norm of X of the last INT8 McWeeny
 * refinement on the current device (the residue products are exact for
 * (2^S sqrt(r2max) + sqrt(np)/2)^2 < prod(moduli)/2). */
int sp2b_last_refinement_info(int* scale_exp, double* r2max);

/* Failure-path self-test (no counterpart in the reference): runs the library's bounded
 * device wait on a barrier that nothing arrives at, limited to spin_limit polls.
 * Returns SP2B_TIMEOUT when the wait ran out and the kernel returned normally, which
 * is the expected outcome; the device stays usable. */
int sp2b_selftest_wait_timeout(int spin_limit);
int sp2b_set_step_timing(int enable);
int sp2b_step_timing(double* ms, long long* launches);
/* With step timing on: summed device time of the INT8 McWeeny refinement phases over
 * the timed solves, ms4 = {residue planes, INT8 products, CRT, combine product}. */
int sp2b_refinement_timing(double* ms4, long long* solves);

#ifdef __cplusplus
}
#endif
#endif /* SP2B_H */
