// SP2-Fermi: the truncated SP2 expansion at finite temperature (src/prg_sp2_fermi_mod.F90),
// FP64 on the GPU.  Each outer pass normalises H with the Fermi bounds, runs the fixed
// number of SP2 steps (the sequence generated on the device in the first pass of the
// init, replayed after), and the host takes one Newton step on mu from the traces the
// last step published.  prg_sp2_fermi_init also carries X1 = dX/dmu through the same
// recursion, as the forward-mode response does (two FP64 products per step following
// the step's branch); prg_sp2_fermi ends with X + lambda DX, DX = -beta X (I - X), as one
// more product: (1 - lambda beta) X + lambda beta X^2.
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "sp2b_ctx.h"

namespace sp2b {

namespace {

struct FermiPass {
  double trx;     // Tr X after the steps
  double fro2;    // ||X||_F^2 (= Tr X^2)
  double trx1;    // Tr X1 (init passes)
};

// One pass: X0 = ((hN - mu) I - H)/(hN - h1) (src/prg_normalize_mod.F90:59-72, as the
// bounds (h1 - mu, hN - mu) of the FP64 normalisation), nsteps SP2 steps (generating the
// branches into c->pp_dev when gen, replaying c->pp_dev otherwise), and with deriv the
// X1 recursion from X1_0 = -I/(hN - h1).  The iterate ends in c->x64[nsteps & 1].
int fermi_pass(Ctx* c, const double* hdev, int n, int nsteps, double nocc, double h1, double hN,
               double mu, bool gen, bool deriv, cudaStream_t st, FermiPass* out) {
  const int np = padded(n);
  double* bounds = c->small;
  double* norm_out = c->small + 4;
  c->h_small[0] = h1 - mu;
  c->h_small[1] = hN - mu;
  SP2B_CUDA_TRY(cudaMemcpyAsync(bounds, c->h_small, 2 * sizeof(double), cudaMemcpyHostToDevice, st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(int), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->sout, 0, sizeof(SolveOut), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->small + 24, 0, 4 * sizeof(double), st));
  SP2B_CUDA_TRY(launch_normalize_f64(hdev, n, n, np, bounds, c->x64[0], c->partials, c->counter,
                                     c->rec, norm_out, st));
  if (deriv) SP2B_CUDA_TRY(launch_resp_init(nullptr, n, n, np, bounds, c->x64[2], st));
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.control = 1;
  a.ctl.algo = gen ? ALGO_FERMI_GEN : ALGO_SEQ;
  a.ctl.icount = nsteps;
  a.ctl.maxit = nsteps + 1;
  a.ctl.occ = nocc;
  a.ctl.n = n;
  a.rec = c->rec;
  a.pp_in = c->pp_dev;
  a.pp_out = gen ? c->pp_dev : nullptr;
  a.sout = c->sout;
  a.partials = c->partials;
  a.counter = c->counter;
  a.err = c->err;
  a.ntiles = f64_ntiles(np);
  for (int k = 0; k < nsteps; ++k) {
    a.k = k;
    const int bin = k & 1, bout = (k + 1) & 1;
    a.A = a.B = a.E = c->x64[bin];
    a.out = c->x64[bout];
    SP2B_CUDA_TRY(launch_sym_gemm_f64(a, st));
    if (deriv) {
      // X1 <- {X, X1} or 2 X1 - {X, X1} with X = X_k (src/prg_sp2_fermi_mod.F90:113-120):
      // P1 = a X X1 + b X1, X1' = a X1 X + P1, (a, b) the step's (1, 0) or (-1, 2)
      StepArgs q = a;
      q.pp_out = nullptr;
      q.sums_out = c->small + 24;
      q.control = 2;
      q.A = c->x64[bin];
      q.B = q.E = c->x64[2 + bin];
      q.out = c->x64[4];
      SP2B_CUDA_TRY(launch_sym_gemm_f64(q, st));
      q.control = 3;
      q.A = c->x64[2 + bin];
      q.B = c->x64[bin];
      q.E = c->x64[4];
      q.out = c->x64[2 + bout];
      SP2B_CUDA_TRY(launch_sym_gemm_f64(q, st));
    }
  }
  SP2Rec r;
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_sout, c->sout, sizeof(SolveOut), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(&r, c->rec + nsteps, sizeof(SP2Rec), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_small + 24, c->small + 24, 4 * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_small + 8, norm_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  int herr = 0;
  SP2B_CUDA_TRY(cudaMemcpy(&herr, c->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (herr) {
    set_last_error("a device-side wait timed out");
    return SP2B_TIMEOUT;
  }
  if (nsteps > 0 && (c->h_sout->nupd != nsteps || c->h_sout->status != SP2B_OK)) {
    set_last_error("SP2-Fermi pass: %d of %d steps applied (status %d)", c->h_sout->nupd, nsteps,
                   c->h_sout->status);
    return c->h_sout->status != SP2B_OK ? c->h_sout->status : SP2B_CUDA_ERROR;
  }
  if (nsteps == 0) {
    SP2B_CUDA_TRY(cudaMemcpy(&r, c->rec, sizeof(SP2Rec), cudaMemcpyDeviceToHost));
  }
  out->trx = r.trx_data;
  out->fro2 = r.fro2;
  // Tr X1: the last control-3 product publishes the trace of its output, X1_nsteps
  out->trx1 = nsteps > 0 ? c->h_small[24 + 1] : -(double)n / (hN - h1);
  if (!(out->trx == out->trx) || !(out->fro2 == out->fro2) || !(out->trx1 == out->trx1)) {
    set_last_error("non-finite values during SP2-Fermi");
    return SP2B_BAD_INPUT;
  }
  return SP2B_OK;
}

// The generated branches as the reference's sgnlist (1: X <- 2X - X^2, -1: X <- X^2)
int fermi_read_sequence(Ctx* c, int nsteps, int* sgnlist) {
  std::vector<int> pp(nsteps);
  SP2B_CUDA_TRY(cudaMemcpy(pp.data(), c->pp_dev, nsteps * sizeof(int), cudaMemcpyDeviceToHost));
  for (int i = 0; i < nsteps; ++i) sgnlist[i] = pp[i] == BR_2X_MINUS_X2 ? 1 : -1;
  return SP2B_OK;
}

struct FermiSetup {
  Ctx* c;
  cudaStream_t st;
  const double* hdev;
  bool dev;
};

int fermi_setup(const double* h, int n, int nsteps, bool deriv, const sp2b_opts* opts,
                FermiSetup* s, std::unique_lock<std::mutex>* lk) {
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  *lk = std::unique_lock<std::mutex>(c->mu);
  s->c = c;
  s->dev = opts->device_ptrs != 0;
  s->st = opts->stream ? (cudaStream_t)opts->stream : (s->dev ? (cudaStream_t)0 : c->stream);
  const int np = padded(n);
  const size_t nn = (size_t)n * n;
  SP2B_CUDA_TRY(c->ensure_common(s->dev ? 0 : nn, np, nsteps + 2, n));
  SP2B_CUDA_TRY(c->ensure_f64(np, deriv ? 5 : 2));
  s->hdev = h;
  if (!s->dev) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->hin, h, nn * sizeof(double), cudaMemcpyHostToDevice, s->st));
    s->hdev = c->hin;
  }
  return SP2B_OK;
}

// X (scale 1) of the last pass, or its final correction, into the caller's x
int fermi_output(FermiSetup& s, int n, int nsteps, double* x, bool correct, double lb) {
  Ctx* c = s.c;
  const int np = padded(n);
  double* src = c->x64[nsteps & 1];
  if (correct) {
    // X + lambda DX = (1 - lambda beta) X + lambda beta X^2 (src/prg_sp2_fermi_mod.F90:460)
    StepArgs q;
    memset(&q, 0, sizeof(q));
    q.np = np;
    q.partials = c->partials;
    q.counter = c->counter;
    q.sums_out = c->small + 16;
    q.A = q.B = q.E = src;
    q.out = c->x64[(nsteps + 1) & 1];
    q.alpha = lb;
    q.beta = 1.0 - lb;
    SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), s.st));
    SP2B_CUDA_TRY(launch_sym_gemm_f64(q, s.st));
    src = c->x64[(nsteps + 1) & 1];
  }
  double* xdev = s.dev ? x : c->hin;
  SP2B_CUDA_TRY(launch_finish_f64(src, np, n, 1.0, xdev, n, s.st));
  if (!s.dev)
    SP2B_CUDA_TRY(cudaMemcpyAsync(x, xdev, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToHost, s.st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(s.st));
  return SP2B_OK;
}

// Newton passes on mu with X1 = dX/dmu until |nocc - Tr X| <= occ_err_limit
// (src/prg_sp2_fermi_mod.F90:89-152): the first pass generates the sequence when gen (into
// sgnlist), later passes replay it; then beta = -Tr X1 / Tr X (I - X) (:157-166) and X.
int fermi_init_passes(FermiSetup& s, int n, int nsteps, double nocc, double h1, double hN,
                      double occ_err_limit, double trace_limit, bool gen, double* mu,
                      double* beta, int* sgnlist, double* x, const char* who) {
  FermiPass f{};
  double occ_err = 1.0;
  int rc;
  for (int pass = 0; occ_err > occ_err_limit; ++pass) {
    if (pass >= 1000) {
      set_last_error("%s: occupation did not converge in 1000 passes", who);
      return SP2B_NOT_CONVERGED;
    }
    const bool g = gen && pass == 0;
    if ((rc = fermi_pass(s.c, s.hdev, n, nsteps, nocc, h1, hN, *mu, g, true, s.st, &f)) != SP2B_OK)
      return rc;
    if (g && (rc = fermi_read_sequence(s.c, nsteps, sgnlist)) != SP2B_OK) return rc;
    occ_err = std::fabs(nocc - f.trx);
    const double lambda = std::fabs(f.trx1) > trace_limit ? (nocc - f.trx) / f.trx1 : 0.0;
    *mu += lambda;
  }
  const double trx = f.trx - f.fro2;
  *beta = std::fabs(trx) > trace_limit ? -f.trx1 / trx : -1000.0;
  return fermi_output(s, n, nsteps, x, false, 0.0);
}

// The step at which prg_sp2_fermi_init_norecs ends the recursion
// (src/prg_sp2_fermi_mod.F90:256-310): the probe p_j = 1 - 0.001 j (j = 1..1000), a grid of
// X0 values, follows the sequence; after step i its steepest slope gives the inverse
// temperature 4 max_j |p_(j+1) - p_j| / 0.001 / (gmax - gmin) (absmaxderivative, :617-630),
// and the first step where that exceeds beta0 is the last.  The probe depends on the
// sequence alone, so every pass of the reference ends at the same step.
int fermi_probe_steps(const int* sgnlist, int nsteps, double gmin, double gmax, double beta0) {
  std::vector<double> p(1000);
  for (int j = 0; j < 1000; ++j) p[j] = 1.0 - (double)(j + 1) * 0.001;
  for (int i = 0; i < nsteps; ++i) {
    for (int j = 0; j < 1000; ++j) {
      const double p2 = p[j] * p[j];
      p[j] = sgnlist[i] == 1 ? 2.0 * p[j] - p2 : p2;
    }
    double maxder = -10000.0;
    for (int j = 0; j < 999; ++j) {
      const double d = std::fabs(p[j + 1] - p[j]) / 0.001;
      if (d > maxder) maxder = d;
    }
    if ((4.0 * maxder) / (gmax - gmin) > beta0) return i + 1;
  }
  return nsteps;
}

// sp2_inverse (src/prg_sp2_fermi_mod.F90:592-611): the energy whose SP2 image is f
double fermi_sp2_inverse(double f, double mu, double h1, double hN, int nsteps, const int* sgnlist) {
  double e = f;
  for (int i = nsteps - 1; i >= 0; --i) {
    const double sgn = (double)sgnlist[i];
    const double c = (1.0 + sgn) / 2.0;
    e = c - sgn * std::sqrt(std::fabs(c - sgn * e));
  }
  return hN - mu - e * (hN - h1);
}

}  // namespace

}  // namespace sp2b

using namespace sp2b;

extern "C" int sp2b_sp2_fermi_init(const double* h, int n, int nsteps, double nocc, double tscale,
                                   double threshold, double occ_err_limit, double trace_limit,
                                   double* x, double* mu, double* beta, double* h1, double* hN,
                                   int* sgnlist, const sp2b_opts* opts) {
  (void)threshold;   // dense products are not thresholded
  if (!h || !x || n <= 0 || nsteps < 1 || !mu || !beta || !h1 || !hN || !sgnlist ||
      !(occ_err_limit >= 0.0)) {
    set_last_error("sp2b_sp2_fermi_init: bad argument");
    return SP2B_BAD_ARG;
  }
  sp2b_opts dflt;
  sp2b_opts_default(&dflt);
  if (!opts) opts = &dflt;
  // Gershgorin bounds (src/prg_sp2_fermi_mod.F90:68-71)
  double gmin = 0.0, gmax = 0.0;
  int rc = sp2b_gershgorin(h, n, &gmin, &gmax, opts);
  if (rc != SP2B_OK) return rc;
  *mu = 0.5 * (gmax + gmin);
  *h1 = tscale * gmin;
  *hN = tscale * gmax;
  FermiSetup s;
  std::unique_lock<std::mutex> lk;
  if ((rc = fermi_setup(h, n, nsteps, true, opts, &s, &lk)) != SP2B_OK) return rc;
  return fermi_init_passes(s, n, nsteps, nocc, *h1, *hN, occ_err_limit, trace_limit, true, mu, beta,
                           sgnlist, x, "sp2b_sp2_fermi_init");
}

extern "C" int sp2b_sp2_fermi(const double* h, int n, int osteps, int nsteps, double nocc,
                              double* mu, double beta, double h1, double hN, const int* sgnlist,
                              double threshold, double eps, double trace_limit, double* x,
                              const sp2b_opts* opts) {
  (void)threshold;
  if (!h || !x || n <= 0 || nsteps < 0 || osteps < 0 || !mu || (nsteps > 0 && !sgnlist) ||
      !(hN - h1 > 0.0)) {
    set_last_error("sp2b_sp2_fermi: bad argument");
    return SP2B_BAD_ARG;
  }
  sp2b_opts dflt;
  sp2b_opts_default(&dflt);
  if (!opts) opts = &dflt;
  FermiSetup s;
  std::unique_lock<std::mutex> lk;
  int rc;
  if ((rc = fermi_setup(h, n, nsteps, false, opts, &s, &lk)) != SP2B_OK) return rc;
  if (nsteps > 0) {
    // the sequence as the step kernels' branches (sgnlist 1: 2X - X^2)
    std::vector<int> pp(nsteps);
    for (int i = 0; i < nsteps; ++i) pp[i] = sgnlist[i] == 1 ? BR_2X_MINUS_X2 : BR_X2;
    SP2B_CUDA_TRY(cudaMemcpy(s.c->pp_dev, pp.data(), nsteps * sizeof(int), cudaMemcpyHostToDevice));
  }
  // osteps passes, or until |nocc - Tr X| <= eps (src/prg_sp2_fermi_mod.F90:416-458)
  double occ_err = 1.0 + eps, lambda = 0.0;
  int it = 0;
  FermiPass f{};
  while ((osteps == 0 && occ_err > eps) || (osteps > 0 && it < osteps)) {
    if (++it > 1000) {
      set_last_error("sp2b_sp2_fermi: occupation did not converge in 1000 passes");
      return SP2B_NOT_CONVERGED;
    }
    if ((rc = fermi_pass(s.c, s.hdev, n, nsteps, nocc, h1, hN, *mu, false, false, s.st, &f)) !=
        SP2B_OK)
      return rc;
    occ_err = std::fabs(nocc - f.trx);
    const double trdx = -beta * (f.trx - f.fro2);   // Tr DX, DX = -beta X (I - X)
    lambda = std::fabs(trdx) > trace_limit ? (nocc - f.trx) / trdx : 0.0;
    *mu += lambda;
  }
  return fermi_output(s, n, nsteps, x, it > 0, lambda * beta);
}

extern "C" int sp2b_sp2_fermi_init_norecs(const double* h, int n, int* nsteps, double nocc,
                                          double tscale, double threshold, double occ_err_limit,
                                          double trace_limit, double* x, double* mu, double* beta,
                                          double* h1, double* hN, int* sgnlist,
                                          const sp2b_opts* opts) {
  (void)threshold;
  if (!h || !x || n <= 0 || !nsteps || *nsteps < 1 || !mu || !beta || !h1 || !hN || !sgnlist ||
      !(occ_err_limit >= 0.0)) {
    set_last_error("sp2b_sp2_fermi_init_norecs: bad argument");
    return SP2B_BAD_ARG;
  }
  sp2b_opts dflt;
  sp2b_opts_default(&dflt);
  if (!opts) opts = &dflt;
  // Gershgorin bounds (src/prg_sp2_fermi_mod.F90:229-232); beta enters as the target
  double gmin = 0.0, gmax = 0.0;
  int rc = sp2b_gershgorin(h, n, &gmin, &gmax, opts);
  if (rc != SP2B_OK) return rc;
  const double beta0 = *beta;
  *mu = 0.5 * (gmax + gmin);
  *h1 = tscale * gmin;
  *hN = tscale * gmax;
  FermiSetup s;
  std::unique_lock<std::mutex> lk;
  if ((rc = fermi_setup(h, n, *nsteps, true, opts, &s, &lk)) != SP2B_OK) return rc;
  // The reference's first pass generates the branches and stops at the probe's step.  Here
  // one pass of X alone generates all nsteps branches at the starting mu (step i's branch
  // depends on the steps before it only), the probe picks the step, and the Newton passes
  // replay that prefix, the first of them at the same mu as the reference's first pass.
  FermiPass f{};
  if ((rc = fermi_pass(s.c, s.hdev, n, *nsteps, nocc, *h1, *hN, *mu, true, false, s.st, &f)) !=
      SP2B_OK)
    return rc;
  std::vector<int> gen(*nsteps);
  if ((rc = fermi_read_sequence(s.c, *nsteps, gen.data())) != SP2B_OK) return rc;
  const int steps = fermi_probe_steps(gen.data(), *nsteps, gmin, gmax, beta0);
  for (int i = 0; i < steps; ++i) sgnlist[i] = gen[i];
  *nsteps = steps;
  return fermi_init_passes(s, n, steps, nocc, *h1, *hN, occ_err_limit, trace_limit, false, mu, beta,
                           sgnlist, x, "sp2b_sp2_fermi_init_norecs");
}

extern "C" int sp2b_sp2_entropy_function(double mu, double h1, double hN, int nsteps,
                                         const int* sgnlist, double* gg, double* ee, int npoints) {
  constexpr int kMesh = 10001;   // ee = 0, 1e-4, ..., 1 (src/prg_sp2_fermi_mod.F90:494-512)
  if (nsteps < 0 || (nsteps > 0 && !sgnlist) || !gg || !ee || npoints < 1 || npoints > kMesh) {
    set_last_error("sp2b_sp2_entropy_function: bad argument");
    return SP2B_BAD_ARG;
  }
  // Running two-point Gauss-Legendre integral of the inverse SP2 map over each mesh interval
  // (:514-525), then GG - GG(end) ee (:528).  A table of 10001 scalars, built on the host as
  // the reference does.
  const double dh = 0.0001, c1 = 1.0, c2 = 1.0;
  const double x1 = 0.5773502691896257, x2 = -x1;
  std::vector<double> e(kMesh), g(kMesh);
  for (int i = 0; i < kMesh; ++i) e[i] = i * dh;
  g[0] = 0.0;
  double iint = 0.0;
  for (int i = 0; i < kMesh - 1; ++i) {
    const double a = e[i], b = e[i + 1];
    const double c_1 = c1 * (b - a) / 2.0, c_2 = c2 * (b - a) / 2.0;
    const double x_1 = ((b - a) * x1 + (b + a)) / 2.0;
    const double x_2 = ((b - a) * x2 + (b + a)) / 2.0;
    iint = iint + c_1 * fermi_sp2_inverse(x_1, mu, h1, hN, nsteps, sgnlist);
    iint = iint + c_2 * fermi_sp2_inverse(x_2, mu, h1, hN, nsteps, sgnlist);
    g[i + 1] = iint;
  }
  const double gend = g[kMesh - 1];
  for (int i = 0; i < npoints; ++i) {
    gg[i] = g[i] - gend * e[i];
    ee[i] = e[i];
  }
  return SP2B_OK;
}
