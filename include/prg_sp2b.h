/*
 * PROGRESS-named C entry points of the SP2 path, served by the sp2b CUDA library.
 *
 * The prototypes are those of the reference's C header
 * (src/prg_progress_mod.h:491-618), which C callers already compile against, and the
 * symbol names are those its Fortran bind(C) wrappers export
 * (src/prg_c_interface.F90:1073-1288).  A caller that links libsp2b.so in place of
 * libprogress gets these routines on the GPU, unchanged.
 *
 * bml_matrix_t.  BML is not part of this library.  It provides a minimal dense handle
 * of the same name: an n x n column-major FP64 array (caller-owned or library-owned).
 * A build that links the real BML converts at the boundary with
 * bml_export_to_dense / bml_import_from_dense.
 *
 * Differences from the reference, all deliberate:
 *  - sp2conv is read as a NUL-terminated string, as the header declares (the
 *    Fortran side binds it as one character(c_char), value; see
 *    src/prg_c_interface.F90:1120 vs src/prg_progress_mod.h:522);
 *  - non-convergence does not `stop` the process: the routine returns and
 *    sp2b_prg_last_status() reports SP2B_NOT_CONVERGED (set SP2B_STRICT_COMPAT=1 in
 *    the environment to print the reference's message and exit(1) instead);
 *  - prg_sp2_submatrix takes the two matrices the Fortran routine needs
 *    (the reference header omits them, src/prg_progress_mod.h:601-608).
 * Precision follows sp2b_get_default_opts (FP64 unless SP2B_PRECISION says otherwise).
 */
#ifndef PRG_SP2B_H
#define PRG_SP2B_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bml_matrix_t bml_matrix_t;

/* Minimal dense handles. */
bml_matrix_t* sp2b_bml_wrap_dense(double* data, int n);  /* caller keeps ownership */
bml_matrix_t* sp2b_bml_zero_dense(int n);                /* library allocates */
double* sp2b_bml_data(bml_matrix_t* a);
int sp2b_bml_n(const bml_matrix_t* a);
void sp2b_bml_free(bml_matrix_t* a);

/* Status of the last PROGRESS-named call of this thread (SP2B_* code). */
int sp2b_prg_last_status(void);

void prg_sp2_basic(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold, double bndfil,
                   int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose);

void prg_sp2_alg2(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose);

void prg_sp2_alg2_genseq(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold,
                         double bndfil, int minsp2iter, int maxsp2iter, char* sp2conv,
                         double idemtol, int* pp, int* icount, double* vv, int verbose);

void prg_sp2_alg2_seq(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold, int* pp,
                      int* icount, double* vv, int verbose);

void prg_sp2_alg1(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose);

void prg_sp2_alg1_genseq(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold,
                         double bndfil, int minsp2iter, int maxsp2iter, char* sp2conv,
                         double idemtol, int* pp, int* icount, double* vv);

void prg_sp2_alg1_seq(bml_matrix_t* h_bml, bml_matrix_t* rho_bml, double threshold, int* pp,
                      int* icount, double* vv);

void prg_prg_sp2_alg2_seq_inplace(bml_matrix_t* rho_bml, double threshold, int ppsize, int* pp,
                                  int* icount, double* vv, double mineval, double maxeval);

void prg_prg_sp2_alg1_seq_inplace(bml_matrix_t* rho_bml, double threshold, int ppsize, int* pp,
                                  int* icount, double* vv, double mineval, double maxeval);

void prg_sp2_submatrix(bml_matrix_t* ham_bml, bml_matrix_t* rho_bml, double threshold, int* pp,
                       int* icount, double* vv, double mineval, double maxeval, int core_size);

void prg_sp2_submatrix_inplace(bml_matrix_t* rho_bml, double threshold, int* pp, int* icount,
                               double* vv, double mineval, double maxeval, int core_size);

/* SP2-Fermi (src/prg_progress_mod.h:433-480; FP64 on the GPU, sp2b_sp2_fermi_init /
 * sp2b_sp2_fermi).  The prototypes follow the reference header; its Fortran binding of
 * prg_sp2_fermi_init (src/prg_c_interface.F90:904-927) takes a trailing `verbose` that
 * the header does not declare and that this export does not read. */
void prg_sp2_fermi_init(bml_matrix_t* h_bml, int nsteps, double nocc, double tscale,
                        double threshold, double occErrLimit, double traceLimit,
                        bml_matrix_t* x_bml, double* mu, double* beta, double* h1, double* hN,
                        int* sgnlist);

void prg_sp2_fermi(bml_matrix_t* h_bml, int osteps, int nsteps, double nocc, double* mu,
                   double* beta, double* h1, double* hN, int* sgnlist, double threshold,
                   double eps, double traceLimit, bml_matrix_t* x_bml);

/* prg_sp2_fermi_init_norecs (src/prg_c_interface.F90:929-952; sp2b_sp2_fermi_init_norecs):
 * *beta in is the target, *nsteps in the most steps; verbose is not read. */
void prg_sp2_fermi_init_norecs(bml_matrix_t* h_bml, int* nsteps, double nocc, double tscale,
                               double threshold, double occErrLimit, double traceLimit,
                               bml_matrix_t* x_bml, double* mu, double* beta, double* h1,
                               double* hN, int* sgnlist, int verbose);

/* prg_sp2_entropy_function (src/prg_c_interface.F90:977-990; sp2b_sp2_entropy_function).
 * The reference header declares sgnlist, GG and ee as scalars; its Fortran binding takes
 * arrays, sgnlist(nsteps), GG(1001) and ee(1001), and assigns the 10001-point results to
 * them, which stores their first 1001 points: this export writes those 1001 entries. */
void prg_sp2_entropy_function(double mu, double h1, double hN, int nsteps, int* sgnlist,
                              double* GG, double* ee);

/* prg_normalize (src/prg_normalize_mod.F90:32-46) and prg_check_idempotency
 * (src/prg_densitymatrix_mod.F90:862-880), the two helpers the SP2 tests call. */
void prg_normalize(bml_matrix_t* h_bml);
void prg_check_idempotency(bml_matrix_t* mat_bml, double threshold, double* idempotency);

#ifdef __cplusplus
}
#endif
#endif /* PRG_SP2B_H */
