// PROGRESS-named exports (src/prg_c_interface.F90:1073-1288 names, the prototypes of
// src/prg_progress_mod.h:491-618) over the minimal dense bml_matrix_t handle.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "../../include/prg_sp2b.h"
#include "../../include/sp2b.h"

struct bml_matrix_t {
  int n;
  double* data;  // n x n, column-major
  bool owned;
};

static thread_local int g_prg_status = SP2B_OK;

static void finish(int status, const char* who) {
  g_prg_status = status;
  if (status == SP2B_OK) return;
  const char* strict = getenv("SP2B_STRICT_COMPAT");
  if (strict && strict[0] == '1') {
    // reference behaviour: print and stop the process (src/prg_sp2_mod.F90:360-363)
    if (status == SP2B_NOT_CONVERGED)
      fprintf(stderr, " SP2 purification is not converging: STOP!\n");
    else
      fprintf(stderr, "%s: %s\n", who, sp2b_last_error());
    exit(1);
  }
}

static sp2b_opts defaults() {
  sp2b_opts o;
  sp2b_get_default_opts(&o);
  o.device_ptrs = 0;
  return o;
}

static bool same_n(const bml_matrix_t* a, const bml_matrix_t* b) {
  return a && b && a->data && b->data && a->n == b->n && a->n > 0;
}

extern "C" {

bml_matrix_t* sp2b_bml_wrap_dense(double* data, int n) {
  if (!data || n <= 0) return nullptr;
  bml_matrix_t* m = new (std::nothrow) bml_matrix_t;
  if (!m) return nullptr;
  m->n = n;
  m->data = data;
  m->owned = false;
  return m;
}

bml_matrix_t* sp2b_bml_zero_dense(int n) {
  if (n <= 0) return nullptr;
  bml_matrix_t* m = new (std::nothrow) bml_matrix_t;
  if (!m) return nullptr;
  m->n = n;
  m->data = static_cast<double*>(calloc((size_t)n * n, sizeof(double)));
  m->owned = true;
  if (!m->data) {
    delete m;
    return nullptr;
  }
  return m;
}

double* sp2b_bml_data(bml_matrix_t* a) { return a ? a->data : nullptr; }
int sp2b_bml_n(const bml_matrix_t* a) { return a ? a->n : 0; }
void sp2b_bml_free(bml_matrix_t* a) {
  if (!a) return;
  if (a->owned) free(a->data);
  delete a;
}

int sp2b_prg_last_status(void) { return g_prg_status; }

void prg_sp2_basic(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                   int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose) {
  if (!same_n(h, rho)) return finish(SP2B_BAD_ARG, "prg_sp2_basic");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_basic(h->data, rho->data, h->n, threshold, bndfil, minsp2iter, maxsp2iter,
                        sp2conv, idemtol, verbose, &o, nullptr),
         "prg_sp2_basic");
}

void prg_sp2_alg2(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose) {
  if (!same_n(h, rho)) return finish(SP2B_BAD_ARG, "prg_sp2_alg2");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg2(h->data, rho->data, h->n, threshold, bndfil, minsp2iter, maxsp2iter,
                       sp2conv, idemtol, verbose, &o, nullptr),
         "prg_sp2_alg2");
}

void prg_sp2_alg2_genseq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int* pp,
                         int* icount, double* vv, int verbose) {
  if (!same_n(h, rho) || !pp || !icount || !vv) return finish(SP2B_BAD_ARG, "prg_sp2_alg2_genseq");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg2_genseq(h->data, rho->data, h->n, threshold, bndfil, minsp2iter, maxsp2iter,
                              sp2conv, idemtol, pp, icount, vv, verbose, &o),
         "prg_sp2_alg2_genseq");
}

void prg_sp2_alg2_seq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, int* pp, int* icount,
                      double* vv, int verbose) {
  if (!same_n(h, rho) || !pp || !icount || !vv) return finish(SP2B_BAD_ARG, "prg_sp2_alg2_seq");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg2_seq(h->data, rho->data, h->n, threshold, pp, *icount, vv, verbose, &o),
         "prg_sp2_alg2_seq");
}

void prg_sp2_alg1(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose) {
  if (!same_n(h, rho)) return finish(SP2B_BAD_ARG, "prg_sp2_alg1");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg1(h->data, rho->data, h->n, threshold, bndfil, minsp2iter, maxsp2iter,
                       sp2conv, idemtol, verbose, &o, nullptr),
         "prg_sp2_alg1");
}

void prg_sp2_alg1_genseq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int* pp,
                         int* icount, double* vv) {
  if (!same_n(h, rho) || !pp || !icount || !vv) return finish(SP2B_BAD_ARG, "prg_sp2_alg1_genseq");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg1_genseq(h->data, rho->data, h->n, threshold, bndfil, minsp2iter, maxsp2iter,
                              sp2conv, idemtol, pp, icount, vv, &o),
         "prg_sp2_alg1_genseq");
}

void prg_sp2_alg1_seq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, int* pp, int* icount,
                      double* vv) {
  if (!same_n(h, rho) || !pp || !icount || !vv) return finish(SP2B_BAD_ARG, "prg_sp2_alg1_seq");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg1_seq(h->data, rho->data, h->n, threshold, pp, *icount, vv, &o),
         "prg_sp2_alg1_seq");
}

void prg_prg_sp2_alg2_seq_inplace(bml_matrix_t* rho, double threshold, int ppsize, int* pp,
                                  int* icount, double* vv, double mineval, double maxeval) {
  if (!rho || !rho->data || !pp || !icount || !vv || *icount > ppsize)
    return finish(SP2B_BAD_ARG, "prg_prg_sp2_alg2_seq_inplace");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg2_seq_inplace(rho->data, rho->n, threshold, pp, *icount, vv, mineval, maxeval,
                                   0, &o),
         "prg_prg_sp2_alg2_seq_inplace");
}

void prg_prg_sp2_alg1_seq_inplace(bml_matrix_t* rho, double threshold, int ppsize, int* pp,
                                  int* icount, double* vv, double mineval, double maxeval) {
  if (!rho || !rho->data || !pp || !icount || !vv || *icount > ppsize)
    return finish(SP2B_BAD_ARG, "prg_prg_sp2_alg1_seq_inplace");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_alg1_seq_inplace(rho->data, rho->n, threshold, pp, *icount, vv, mineval, maxeval,
                                   &o),
         "prg_prg_sp2_alg1_seq_inplace");
}

void prg_sp2_submatrix(bml_matrix_t* ham, bml_matrix_t* rho, double threshold, int* pp,
                       int* icount, double* vv, double mineval, double maxeval, int core_size) {
  if (!same_n(ham, rho) || !pp || !icount || !vv) return finish(SP2B_BAD_ARG, "prg_sp2_submatrix");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_submatrix(ham->data, rho->data, ham->n, threshold, pp, *icount, vv, mineval,
                            maxeval, core_size, &o),
         "prg_sp2_submatrix");
}

void prg_sp2_submatrix_inplace(bml_matrix_t* rho, double threshold, int* pp, int* icount,
                               double* vv, double mineval, double maxeval, int core_size) {
  if (!rho || !rho->data || !pp || !icount || !vv)
    return finish(SP2B_BAD_ARG, "prg_sp2_submatrix_inplace");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_submatrix_inplace(rho->data, rho->n, threshold, pp, *icount, vv, mineval,
                                    maxeval, core_size, &o),
         "prg_sp2_submatrix_inplace");
}

void prg_sp2_fermi_init(bml_matrix_t* h, int nsteps, double nocc, double tscale, double threshold,
                        double occErrLimit, double traceLimit, bml_matrix_t* x, double* mu,
                        double* beta, double* h1, double* hN, int* sgnlist) {
  if (!same_n(h, x) || !mu || !beta || !h1 || !hN || !sgnlist)
    return finish(SP2B_BAD_ARG, "prg_sp2_fermi_init");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_fermi_init(h->data, h->n, nsteps, nocc, tscale, threshold, occErrLimit,
                             traceLimit, x->data, mu, beta, h1, hN, sgnlist, &o),
         "prg_sp2_fermi_init");
}

void prg_sp2_fermi(bml_matrix_t* h, int osteps, int nsteps, double nocc, double* mu, double* beta,
                   double* h1, double* hN, int* sgnlist, double threshold, double eps,
                   double traceLimit, bml_matrix_t* x) {
  if (!same_n(h, x) || !mu || !beta || !h1 || !hN || !sgnlist)
    return finish(SP2B_BAD_ARG, "prg_sp2_fermi");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_fermi(h->data, h->n, osteps, nsteps, nocc, mu, *beta, *h1, *hN, sgnlist,
                        threshold, eps, traceLimit, x->data, &o),
         "prg_sp2_fermi");
}

void prg_sp2_fermi_init_norecs(bml_matrix_t* h, int* nsteps, double nocc, double tscale,
                               double threshold, double occErrLimit, double traceLimit,
                               bml_matrix_t* x, double* mu, double* beta, double* h1, double* hN,
                               int* sgnlist, int verbose) {
  (void)verbose;
  if (!same_n(h, x) || !nsteps || !mu || !beta || !h1 || !hN || !sgnlist)
    return finish(SP2B_BAD_ARG, "prg_sp2_fermi_init_norecs");
  sp2b_opts o = defaults();
  finish(sp2b_sp2_fermi_init_norecs(h->data, h->n, nsteps, nocc, tscale, threshold, occErrLimit,
                                    traceLimit, x->data, mu, beta, h1, hN, sgnlist, &o),
         "prg_sp2_fermi_init_norecs");
}

void prg_sp2_entropy_function(double mu, double h1, double hN, int nsteps, int* sgnlist,
                              double* GG, double* ee) {
  finish(sp2b_sp2_entropy_function(mu, h1, hN, nsteps, sgnlist, GG, ee, 1001),
         "prg_sp2_entropy_function");
}

void prg_normalize(bml_matrix_t* h) {
  if (!h || !h->data) return finish(SP2B_BAD_ARG, "prg_normalize");
  sp2b_opts o = defaults();
  finish(sp2b_normalize(h->data, h->n, nullptr, nullptr, &o), "prg_normalize");
}

void prg_check_idempotency(bml_matrix_t* a, double threshold, double* idempotency) {
  if (!a || !a->data || !idempotency) return finish(SP2B_BAD_ARG, "prg_check_idempotency");
  sp2b_opts o = defaults();
  finish(sp2b_check_idempotency(a->data, a->n, threshold, idempotency, &o), "prg_check_idempotency");
}

}  // extern "C"
