// Host-side harness for the SP2 control rules (sp2b_common.cuh), built by
// tests/test_control_rules.py with the host C++ compiler.  It runs the recursion on a
// diagonal X (its eigenvalues) with the same record handling as the device's launch
// prologue and last-CTA finalisation (reduce.cuh), and an optional relative bias of
// the products (P = (1 - bias) X^2), the model of the tensor cores' accumulation.
#include <cmath>
#include <cstring>
#include <vector>

#include "sp2b_common.cuh"

using namespace sp2b;

extern "C" int ctl_run(int algo, int conv, int minit, int maxit, double occ, double idemtol,
                       double mixed_tol, double stag_tol, int n, const double* eig0, double bias,
                       int uncorrected, int icount, int* pp_out, int* iters_out, int* nupd_out,
                       int* status_out, double* eig_out) {
  SP2Ctl c;
  std::memset(&c, 0, sizeof(c));
  c.algo = algo;
  c.icount = icount;
  c.conv = conv;
  c.minit = minit;
  c.maxit = maxit;
  c.n = n;
  c.occ = occ;
  c.idemtol = idemtol;
  c.mixed_tol = mixed_tol;
  c.stag_tol = stag_tol;
  std::vector<double> x(eig0, eig0 + n);
  SP2Rec r;
  std::memset(&r, 0, sizeof(r));
  for (double v : x) {
    r.trx += v;
    r.fro2 += v * v;
  }
  r.trx_data = r.trx;
  r.last_branch = -1;
  int k = 0;
  for (; k < maxit + 1; ++k) {
    // launch prologue: stop before updating, or the branch to apply
    SP2Decision d = sp2_decide(c, r, k, nullptr);
    if (d.branch == BR_STOP) {
      r = d.next;
      r.done = 1;
      break;
    }
    double t0 = 0.0, t1 = 0.0, t3 = 0.0;
    for (double& v : x) {
      const double p = (1.0 - bias) * v * v;
      t3 += p;
      v = d.branch == BR_X2 ? p : 2.0 * v - p;
      t0 += v * v;
      t1 += v;
    }
    // last CTA: the record of the next launch
    SP2Rec nx = d.next;
    if (algo == ALGO_MIXED) sp2_mixed_stop(c, r, t3, nx);
    nx.fro2 = t0;
    nx.trx_data = t1;
    nx.trp = t3;
    nx.pbias = uncorrected ? 0.0 : r.fro2 - t3;
    nx.last_branch = d.branch;
    pp_out[k] = d.branch;
    r = nx;
    if (r.done) {
      ++k;
      break;
    }
  }
  *iters_out = r.iter;
  *nupd_out = k;
  *status_out = r.status;
  for (int i = 0; i < n; ++i) eig_out[i] = x[i];
  return 0;
}
