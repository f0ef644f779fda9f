// PROGRESS-named exports (src/prg_c_interface.F90:1073-1288 names, the prototypes of
// src/prg_progress_mod.h:491-618).  Their bml_matrix_t* arguments are either the
// library's own minimal dense handle (sp2b_bml_wrap_dense / sp2b_bml_zero_dense) or a
// real BML matrix of the calling process, the way the reference's C binding receives
// them (h_bml%ptr = h_bml_c, src/prg_c_interface.F90:1113-1129).
//
// BML (github.com/lanl/bml) is not linked: its C API is resolved at call time with
// dlsym(RTLD_DEFAULT, ...), so a caller that links libbml and libsp2b passes its BML
// handles unchanged.  A handle the library did not create is read with
// bml_export_to_dense (column-major; single- or double-precision real) and results are
// written back with bml_import_from_dense of the output handle's own type, precision,
// width and distribution, bml_copy into the handle and bml_deallocate of the temporary,
// with the call's threshold (BML thresholds sparse output; the dense product ignores
// it).  The library's own handles are recognised by a registry, never by reading a
// foreign pointer, so a handle that is neither the library's nor readable through BML
// is rejected with SP2B_BAD_ARG without being dereferenced.
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <unordered_set>
#include <vector>

#include "../../include/prg_sp2b.h"
#include "../../include/sp2b.h"

namespace sp2b {
void set_last_error(const char* fmt, ...);
}

struct bml_matrix_t {
  int n;
  double* data;  // n x n, column-major
  bool owned;
};

static thread_local int g_prg_status = SP2B_OK;

static std::mutex g_handles_mu;
static std::unordered_set<const void*>& own_handles() {
  static std::unordered_set<const void*> s;
  return s;
}
static bool is_own(const bml_matrix_t* a) {
  std::lock_guard<std::mutex> lk(g_handles_mu);
  return own_handles().count(a) != 0;
}

// The part of BML's C API the exports use, with BML's enum values (bml_types.h:
// bml_matrix_precision_t {precision_uninitialized, single_real, double_real, ...},
// bml_dense_order_t {dense_row_major, dense_column_major}).
namespace {
constexpr int kBmlSingleReal = 1, kBmlDoubleReal = 2, kBmlColumnMajor = 1;
struct BmlApi {
  int (*get_N)(void*);
  int (*get_M)(void*);
  int (*get_type)(void*);
  int (*get_precision)(void*);
  int (*get_distribution_mode)(void*);
  void* (*export_to_dense)(void*, int);
  void* (*import_from_dense)(int, int, int, int, int, void*, double, int);
  void (*copy)(void*, void*);
  void (*deallocate)(void**);
  void (*free_memory)(void*);
};

// Resolved from the process's global symbols; null while BML is not loaded.
const BmlApi* bml_api() {
  static std::mutex mu;
  static BmlApi api;
  static bool found = false;
  std::lock_guard<std::mutex> lk(mu);
  if (found) return &api;
  BmlApi a;
  a.get_N = (int (*)(void*))dlsym(RTLD_DEFAULT, "bml_get_N");
  a.get_M = (int (*)(void*))dlsym(RTLD_DEFAULT, "bml_get_M");
  a.get_type = (int (*)(void*))dlsym(RTLD_DEFAULT, "bml_get_type");
  a.get_precision = (int (*)(void*))dlsym(RTLD_DEFAULT, "bml_get_precision");
  a.get_distribution_mode = (int (*)(void*))dlsym(RTLD_DEFAULT, "bml_get_distribution_mode");
  a.export_to_dense = (void* (*)(void*, int))dlsym(RTLD_DEFAULT, "bml_export_to_dense");
  a.import_from_dense =
      (void* (*)(int, int, int, int, int, void*, double, int))dlsym(RTLD_DEFAULT, "bml_import_from_dense");
  a.copy = (void (*)(void*, void*))dlsym(RTLD_DEFAULT, "bml_copy");
  a.deallocate = (void (*)(void**))dlsym(RTLD_DEFAULT, "bml_deallocate");
  a.free_memory = (void (*)(void*))dlsym(RTLD_DEFAULT, "bml_free_memory");
  if (!a.get_N || !a.get_M || !a.get_type || !a.get_precision || !a.get_distribution_mode ||
      !a.export_to_dense || !a.import_from_dense || !a.copy || !a.deallocate)
    return nullptr;
  api = a;
  found = true;
  return &api;
}

// A matrix argument as the dense n x n FP64 array the sp2b ABI takes.
struct Dense {
  bml_matrix_t* h = nullptr;   // the caller's handle
  bool foreign = false;        // a BML matrix (else the library's own handle)
  int n = 0;
  double* data = nullptr;
  std::vector<double> buf;     // BML matrices: the exported values
};

// Reads (or, with read = false, only sizes) a matrix argument.
int dense_in(bml_matrix_t* h, Dense& d, bool read) {
  d.h = h;
  if (!h) return SP2B_BAD_ARG;
  if (is_own(h)) {
    if (!h->data || h->n <= 0) return SP2B_BAD_ARG;
    d.n = h->n;
    d.data = h->data;
    return SP2B_OK;
  }
  const BmlApi* api = bml_api();
  if (!api) {
    sp2b::set_last_error("matrix handle is neither an sp2b handle nor a BML matrix "
                            "(no BML in the process)");
    return SP2B_BAD_ARG;
  }
  d.foreign = true;
  d.n = api->get_N(h);
  if (d.n <= 0) return SP2B_BAD_ARG;
  const int prec = api->get_precision(h);
  if (prec != kBmlDoubleReal && prec != kBmlSingleReal) {
    sp2b::set_last_error("BML matrix precision %d: only real single/double are supported", prec);
    return SP2B_BAD_ARG;
  }
  const size_t nn = (size_t)d.n * d.n;
  d.buf.assign(nn, 0.0);
  d.data = d.buf.data();
  if (!read) return SP2B_OK;
  void* e = api->export_to_dense(h, kBmlColumnMajor);
  if (!e) return SP2B_BAD_ARG;
  if (prec == kBmlDoubleReal) {
    std::memcpy(d.buf.data(), e, nn * sizeof(double));
  } else {
    const float* f = static_cast<const float*>(e);
    for (size_t i = 0; i < nn; ++i) d.buf[i] = (double)f[i];
  }
  if (api->free_memory) api->free_memory(e);
  else free(e);
  return SP2B_OK;
}

// Writes a result back into a BML matrix argument (nothing to do for own handles,
// whose array the ABI call wrote directly).
int dense_out(Dense& d, double threshold) {
  if (!d.foreign) return SP2B_OK;
  const BmlApi* api = bml_api();
  void* h = d.h;
  const int prec = api->get_precision(h);
  std::vector<float> f;
  void* src = d.buf.data();
  if (prec == kBmlSingleReal) {
    f.resize(d.buf.size());
    for (size_t i = 0; i < f.size(); ++i) f[i] = (float)d.buf[i];
    src = f.data();
  }
  void* tmp = api->import_from_dense(api->get_type(h), prec, kBmlColumnMajor, d.n, api->get_M(h),
                                     src, threshold, api->get_distribution_mode(h));
  if (!tmp) return SP2B_BAD_ARG;
  api->copy(tmp, h);
  api->deallocate(&tmp);
  return SP2B_OK;
}
}  // namespace

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

extern "C" {

bml_matrix_t* sp2b_bml_wrap_dense(double* data, int n) {
  if (!data || n <= 0) return nullptr;
  bml_matrix_t* m = new (std::nothrow) bml_matrix_t;
  if (!m) return nullptr;
  m->n = n;
  m->data = data;
  m->owned = false;
  std::lock_guard<std::mutex> lk(g_handles_mu);
  own_handles().insert(m);
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
  std::lock_guard<std::mutex> lk(g_handles_mu);
  own_handles().insert(m);
  return m;
}

double* sp2b_bml_data(bml_matrix_t* a) { return a && is_own(a) ? a->data : nullptr; }
int sp2b_bml_n(const bml_matrix_t* a) { return a && is_own(a) ? a->n : 0; }
void sp2b_bml_free(bml_matrix_t* a) {
  if (!a) return;
  {
    std::lock_guard<std::mutex> lk(g_handles_mu);
    if (own_handles().erase(a) == 0) return;   // not one of ours: leave it alone
  }
  if (a->owned) free(a->data);
  delete a;
}

int sp2b_prg_last_status(void) { return g_prg_status; }

// Each export: read the matrix arguments (in, inout), check the sizes agree, run the
// raw-pointer entry on the dense arrays, write the outputs back (BML handles).
#define SP2B_IN(var, h, read)                         \
  Dense var;                                          \
  if (dense_in((h), var, (read)) != SP2B_OK) return finish(SP2B_BAD_ARG, who);

void prg_sp2_basic(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                   int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose) {
  const char* who = "prg_sp2_basic";
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_basic(H.data, P.data, H.n, threshold, bndfil, minsp2iter, maxsp2iter, sp2conv,
                          idemtol, verbose, &o, nullptr);
  if (st == SP2B_OK || st == SP2B_NOT_CONVERGED) {
    const int wo = dense_out(P, threshold);
    if (wo != SP2B_OK) st = wo;
  }
  finish(st, who);
}

void prg_sp2_alg2(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose) {
  const char* who = "prg_sp2_alg2";
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg2(H.data, P.data, H.n, threshold, bndfil, minsp2iter, maxsp2iter, sp2conv,
                         idemtol, verbose, &o, nullptr);
  if (st == SP2B_OK || st == SP2B_NOT_CONVERGED) {
    const int wo = dense_out(P, threshold);
    if (wo != SP2B_OK) st = wo;
  }
  finish(st, who);
}

void prg_sp2_alg2_genseq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int* pp,
                         int* icount, double* vv, int verbose) {
  const char* who = "prg_sp2_alg2_genseq";
  if (!pp || !icount || !vv) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg2_genseq(H.data, P.data, H.n, threshold, bndfil, minsp2iter, maxsp2iter,
                                sp2conv, idemtol, pp, icount, vv, verbose, &o);
  if (st == SP2B_OK || st == SP2B_NOT_CONVERGED) {
    const int wo = dense_out(P, threshold);
    if (wo != SP2B_OK) st = wo;
  }
  finish(st, who);
}

void prg_sp2_alg2_seq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, int* pp, int* icount,
                      double* vv, int verbose) {
  const char* who = "prg_sp2_alg2_seq";
  if (!pp || !icount || !vv) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg2_seq(H.data, P.data, H.n, threshold, pp, *icount, vv, verbose, &o);
  if (st == SP2B_OK) st = dense_out(P, threshold);
  finish(st, who);
}

void prg_sp2_alg1(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int verbose) {
  const char* who = "prg_sp2_alg1";
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg1(H.data, P.data, H.n, threshold, bndfil, minsp2iter, maxsp2iter, sp2conv,
                         idemtol, verbose, &o, nullptr);
  if (st == SP2B_OK || st == SP2B_NOT_CONVERGED) {
    const int wo = dense_out(P, threshold);
    if (wo != SP2B_OK) st = wo;
  }
  finish(st, who);
}

void prg_sp2_alg1_genseq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, char* sp2conv, double idemtol, int* pp,
                         int* icount, double* vv) {
  const char* who = "prg_sp2_alg1_genseq";
  if (!pp || !icount || !vv) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg1_genseq(H.data, P.data, H.n, threshold, bndfil, minsp2iter, maxsp2iter,
                                sp2conv, idemtol, pp, icount, vv, &o);
  if (st == SP2B_OK || st == SP2B_NOT_CONVERGED) {
    const int wo = dense_out(P, threshold);
    if (wo != SP2B_OK) st = wo;
  }
  finish(st, who);
}

void prg_sp2_alg1_seq(bml_matrix_t* h, bml_matrix_t* rho, double threshold, int* pp, int* icount,
                      double* vv) {
  const char* who = "prg_sp2_alg1_seq";
  if (!pp || !icount || !vv) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg1_seq(H.data, P.data, H.n, threshold, pp, *icount, vv, &o);
  if (st == SP2B_OK) st = dense_out(P, threshold);
  finish(st, who);
}

void prg_prg_sp2_alg2_seq_inplace(bml_matrix_t* rho, double threshold, int ppsize, int* pp,
                                  int* icount, double* vv, double mineval, double maxeval) {
  const char* who = "prg_prg_sp2_alg2_seq_inplace";
  if (!pp || !icount || !vv || *icount > ppsize) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(P, rho, true);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg2_seq_inplace(P.data, P.n, threshold, pp, *icount, vv, mineval, maxeval, 0,
                                     &o);
  if (st == SP2B_OK) st = dense_out(P, threshold);
  finish(st, who);
}

void prg_prg_sp2_alg1_seq_inplace(bml_matrix_t* rho, double threshold, int ppsize, int* pp,
                                  int* icount, double* vv, double mineval, double maxeval) {
  const char* who = "prg_prg_sp2_alg1_seq_inplace";
  if (!pp || !icount || !vv || *icount > ppsize) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(P, rho, true);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_alg1_seq_inplace(P.data, P.n, threshold, pp, *icount, vv, mineval, maxeval, &o);
  if (st == SP2B_OK) st = dense_out(P, threshold);
  finish(st, who);
}

void prg_sp2_submatrix(bml_matrix_t* ham, bml_matrix_t* rho, double threshold, int* pp,
                       int* icount, double* vv, double mineval, double maxeval, int core_size) {
  const char* who = "prg_sp2_submatrix";
  if (!pp || !icount || !vv) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, ham, true);
  SP2B_IN(P, rho, false);
  if (H.n != P.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_submatrix(H.data, P.data, H.n, threshold, pp, *icount, vv, mineval, maxeval,
                              core_size, &o);
  if (st == SP2B_OK) st = dense_out(P, threshold);
  finish(st, who);
}

void prg_sp2_submatrix_inplace(bml_matrix_t* rho, double threshold, int* pp, int* icount,
                               double* vv, double mineval, double maxeval, int core_size) {
  const char* who = "prg_sp2_submatrix_inplace";
  if (!pp || !icount || !vv) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(P, rho, true);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_submatrix_inplace(P.data, P.n, threshold, pp, *icount, vv, mineval, maxeval,
                                      core_size, &o);
  if (st == SP2B_OK) st = dense_out(P, threshold);
  finish(st, who);
}

void prg_sp2_fermi_init(bml_matrix_t* h, int nsteps, double nocc, double tscale, double threshold,
                        double occErrLimit, double traceLimit, bml_matrix_t* x, double* mu,
                        double* beta, double* h1, double* hN, int* sgnlist) {
  const char* who = "prg_sp2_fermi_init";
  if (!mu || !beta || !h1 || !hN || !sgnlist) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(X, x, false);
  if (H.n != X.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_fermi_init(H.data, H.n, nsteps, nocc, tscale, threshold, occErrLimit,
                               traceLimit, X.data, mu, beta, h1, hN, sgnlist, &o);
  if (st == SP2B_OK) st = dense_out(X, threshold);
  finish(st, who);
}

void prg_sp2_fermi(bml_matrix_t* h, int osteps, int nsteps, double nocc, double* mu, double* beta,
                   double* h1, double* hN, int* sgnlist, double threshold, double eps,
                   double traceLimit, bml_matrix_t* x) {
  const char* who = "prg_sp2_fermi";
  if (!mu || !beta || !h1 || !hN || !sgnlist) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(X, x, false);
  if (H.n != X.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_fermi(H.data, H.n, osteps, nsteps, nocc, mu, *beta, *h1, *hN, sgnlist,
                          threshold, eps, traceLimit, X.data, &o);
  if (st == SP2B_OK) st = dense_out(X, threshold);
  finish(st, who);
}

void prg_sp2_fermi_init_norecs(bml_matrix_t* h, int* nsteps, double nocc, double tscale,
                               double threshold, double occErrLimit, double traceLimit,
                               bml_matrix_t* x, double* mu, double* beta, double* h1, double* hN,
                               int* sgnlist, int verbose) {
  (void)verbose;
  const char* who = "prg_sp2_fermi_init_norecs";
  if (!nsteps || !mu || !beta || !h1 || !hN || !sgnlist) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(H, h, true);
  SP2B_IN(X, x, false);
  if (H.n != X.n) return finish(SP2B_BAD_ARG, who);
  sp2b_opts o = defaults();
  int st = sp2b_sp2_fermi_init_norecs(H.data, H.n, nsteps, nocc, tscale, threshold, occErrLimit,
                                      traceLimit, X.data, mu, beta, h1, hN, sgnlist, &o);
  if (st == SP2B_OK) st = dense_out(X, threshold);
  finish(st, who);
}

void prg_sp2_entropy_function(double mu, double h1, double hN, int nsteps, int* sgnlist,
                              double* GG, double* ee) {
  finish(sp2b_sp2_entropy_function(mu, h1, hN, nsteps, sgnlist, GG, ee, 1001),
         "prg_sp2_entropy_function");
}

void prg_normalize(bml_matrix_t* h) {
  const char* who = "prg_normalize";
  SP2B_IN(H, h, true);
  sp2b_opts o = defaults();
  int st = sp2b_normalize(H.data, H.n, nullptr, nullptr, &o);
  if (st == SP2B_OK) st = dense_out(H, 0.0);
  finish(st, who);
}

void prg_check_idempotency(bml_matrix_t* a, double threshold, double* idempotency) {
  const char* who = "prg_check_idempotency";
  if (!idempotency) return finish(SP2B_BAD_ARG, who);
  SP2B_IN(A, a, true);
  sp2b_opts o = defaults();
  finish(sp2b_check_idempotency(A.data, A.n, threshold, idempotency, &o), who);
}

}  // extern "C"
