// Host driver of the dense SP2 path and its C-ABI entry points.
#include <atomic>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "sp2b_ctx.h"

namespace sp2b {

static thread_local char g_err[1024] = "";
static std::atomic<long long> g_launches{0};
static std::atomic<int> g_step_timing{0};
static std::mutex g_timing_mu;
static double g_step_ms = 0.0;
static long long g_step_timed = 0;
static double g_ref_ms[4] = {0.0, 0.0, 0.0, 0.0};  // INT8 refinement phases
static long long g_ref_timed = 0;

void note_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(); }
void set_launch_count(long long v) { g_launches.store(v); }

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// ------------------------------------------------------------------------------------
// Per-device context: cached device buffers, one stream, pinned status words.
// Calls on the same device are serialised by the context mutex.
// ------------------------------------------------------------------------------------
static Ctx g_ctx[64];
static std::mutex g_ctx_mu;

template <typename T>
static cudaError_t grow(T*& p, size_t& cap, size_t need) {
  if (need <= cap && p) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)&p, need * sizeof(T));
  if (e == cudaSuccess) cap = need;
  return e;
}

Ctx* get_ctx(int* status) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    set_last_error("no CUDA device available");
    *status = SP2B_NO_DEVICE;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  Ctx& c = g_ctx[dev];
  if (!c.init) {
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void**)&c.h_sout, sizeof(SolveOut)) != cudaSuccess ||
        cudaMallocHost((void**)&c.h_small, 64 * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c.small, 64 * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&c.counter, 4 * sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc((void**)&c.sout, sizeof(SolveOut)) != cudaSuccess ||
        cudaMalloc((void**)&c.err, sizeof(int)) != cudaSuccess ||
        cudaMemset(c.counter, 0, 4 * sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(c.err, 0, sizeof(int)) != cudaSuccess) {
      set_last_error("context setup failed: %s", cudaGetErrorString(cudaGetLastError()));
      *status = SP2B_CUDA_ERROR;
      return nullptr;
    }
    c.dev = dev;
    c.init = true;
  }
  return &c;
}

cudaError_t Ctx::ensure_f64(int np, int nbuf) {
  for (int i = 0; i < nbuf; ++i) {
    cudaError_t e = grow(x64[i], x64_cap[i], (size_t)np * np);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t Ctx::ensure_split(int np) {
  for (int i = 0; i < 2; ++i) {
    cudaError_t e = grow(hi[i], hi_cap[i], (size_t)np * np);
    if (e != cudaSuccess) return e;
    e = grow(lo[i], lo_cap[i], (size_t)np * np);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t Ctx::ensure_common(size_t nin, int np, int maxlaunch, int n) {
  cudaError_t e;
  if (nin) {
    e = grow(hin, hin_cap, nin);
    if (e != cudaSuccess) return e;
  }
  // one partial set per tile of the smallest FP64 edge (64) the step may use
  const long long t64 = np / 64;
  const size_t parts =
      4 * (size_t)std::max<long long>(std::max<long long>(t64 * (t64 + 1) / 2, tc_ntiles(np)), 148 * 8);
  if ((e = grow(partials, partials_cap, parts)) != cudaSuccess) return e;
  if ((e = grow(rec, rec_cap, (size_t)maxlaunch + 2)) != cudaSuccess) return e;
  if ((e = grow(pp_dev, pp_cap, (size_t)maxlaunch + 2)) != cudaSuccess) return e;
  if ((e = grow(vv_dev, vv_cap, (size_t)maxlaunch + 2)) != cudaSuccess) return e;
  const int nsplit = gersh_nsplit(std::max(n, 1));
  if ((e = grow(rowsum, rowsum_cap, (size_t)nsplit * std::max(n, 1))) != cudaSuccess) return e;
  return cudaSuccess;
}

cudaError_t Ctx::ensure_oz(int np, cudaStream_t st) {
  const size_t need = (size_t)oz_nmod() * np * np;
  cudaError_t e;
  if (need > oz_cap || !oz_res) {
    if (oz_res) cudaFree(oz_res);
    if (oz_q) cudaFree(oz_q);
    oz_res = nullptr;
    oz_q = nullptr;
    oz_cap = 0;
    if ((e = cudaMalloc((void**)&oz_res, need)) != cudaSuccess) return e;
    if ((e = cudaMalloc((void**)&oz_q, need)) != cudaSuccess) return e;
    oz_cap = need;
  }
  if (!oz_scale && (e = cudaMalloc(&oz_scale, oz_scale_bytes())) != cudaSuccess) return e;
  if (oz_tiles_np != np) {
    std::vector<int2> t;
    oz_tile_list(np, t);
    if (oz_tiles) cudaFree(oz_tiles);
    oz_tiles = nullptr;
    oz_tiles_np = 0;
    if ((e = cudaMalloc((void**)&oz_tiles, t.size() * sizeof(int2))) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(oz_tiles, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice,
                             st)) != cudaSuccess)
      return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    oz_ntiles = (int)t.size();
    oz_tiles_np = np;
  }
  return cudaSuccess;
}

// Host -> device copy of a symmetric n x n matrix: the upper triangle only, one 2D copy
// per 128-row panel (rows [r0, r0 + 128), columns [r0, n)), ~(n + 128)/(2n) of the bytes;
// the lower triangle is rebuilt on the device from it.
static cudaError_t copy_symmetric_h2d(double* dst, const double* src, int n, cudaStream_t st) {
  for (int r0 = 0; r0 < n; r0 += 128) {
    const int rows = std::min(128, n - r0);
    cudaError_t e = cudaMemcpy2DAsync(dst + (size_t)r0 * n + r0, (size_t)n * sizeof(double),
                                      src + (size_t)r0 * n + r0, (size_t)n * sizeof(double),
                                      (size_t)(n - r0) * sizeof(double), rows,
                                      cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return launch_mirror_lower(dst, n, n, st);
}

// ------------------------------------------------------------------------------------
// Dense solve
// ------------------------------------------------------------------------------------
static int parse_conv(const char* s) {
  if (!s) return CONV_NONE;
  // Fortran blank-padded comparison: "Rel" == "Rel   "; case-sensitive.
  std::string t(s);
  while (!t.empty() && t.back() == ' ') t.pop_back();
  if (t == "Rel") return CONV_REL;
  if (t == "Abs") return CONV_ABS;
  return CONV_NONE;
}

// Device-pointer calls run on the caller's stream, and a NULL stream there means the
// CUDA default stream (the caller's data is ordered on it); host-pointer calls, whose
// data movement is the library's own, run on the library stream unless one is given.
static cudaStream_t pick_stream(const sp2b_opts* o, Ctx* c) {
  if (o && o->stream) return (cudaStream_t)o->stream;
  return (o && o->device_ptrs) ? (cudaStream_t)0 : c->stream;
}

static thread_local int t_exact_switch = 0;   // the last solve restarted in the exact form

// One solve.  A mixed trace-driven solve with exact_switch > 0 sets *want_exact and
// returns without writing its outputs when its loop shows a spectrum the split products
// cannot resolve: still running after exact_switch steps, or stopped on the stagnation
// test (the last step's Tr X - Tr P above mixed_tol) or on maxsp2iter.
static int dense_solve_once(const DenseJob& j, bool* want_exact) {
  if (j.n <= 0 || !j.rho || (!j.h && !j.inplace)) {
    set_last_error("bad argument: n=%d h=%p rho=%p", j.n, (void*)j.h, (void*)j.rho);
    return SP2B_BAD_ARG;
  }
  if (j.ctl.algo == ALGO_SEQ && j.ctl.icount < 0) {
    set_last_error("bad argument: icount=%d", j.ctl.icount);
    return SP2B_BAD_ARG;
  }
  if (j.ctl.algo != ALGO_SEQ && j.ctl.maxit < 1) {
    set_last_error("bad argument: maxsp2iter=%d", j.ctl.maxit);
    return SP2B_BAD_ARG;
  }
  if (j.ctl.algo == ALGO_SEQ && j.ctl.icount > 0 && !j.pp_in) {
    set_last_error("bad argument: pp is NULL");
    return SP2B_BAD_ARG;
  }
  const bool resp = j.h1 != nullptr;   // forward-mode response (FP64 only)
  if (resp && (!j.rsp || j.prec != SP2B_PREC_FP64)) {
    set_last_error("bad argument: response needs rsp and FP64 precision");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = j.stream ? j.stream : (j.dev_ptrs ? (cudaStream_t)0 : c->stream);
  const int n = j.n, np = padded(n);
  const bool split = j.prec == SP2B_PREC_MIXED_FP16 || j.prec == SP2B_PREC_MIXED_BF16;
  const bool exact = j.prec == SP2B_PREC_EXACT_INT8;   // FP64 iterate, INT8 products
  const int bf16 = j.prec == SP2B_PREC_MIXED_BF16;
  if (!split && !exact && j.prec != SP2B_PREC_FP64) {
    set_last_error("bad argument: precision %d", j.prec);
    return SP2B_BAD_ARG;
  }
  int maxlaunch;
  if (j.ctl.algo == ALGO_SEQ) maxlaunch = j.ctl.icount;
  else if (j.ctl.algo == ALGO_BASIC) maxlaunch = j.ctl.maxit + 1;
  else maxlaunch = j.ctl.maxit;

  // one McWeeny step of a split solve runs on the INT8 tensor cores (exact residue
  // products); more steps, or the FP64 choice, use FP64 DMMA products
  const bool oz = split && j.mcweeny == 1 && j.mcweeny_products == SP2B_MCW_INT8 && np <= 65536;
  const bool fallback = split && j.ctl.algo == ALGO_MIXED && j.exact_switch > 0 && want_exact &&
                        np <= 65536;
  const size_t nn = (size_t)n * n;
  SP2B_CUDA_TRY(c->ensure_common(j.dev_ptrs ? 0 : nn, np, maxlaunch, n));
  SP2B_CUDA_TRY(c->ensure_f64(np, split ? (oz ? 1 : 3) : (resp ? 5 : 2)));
  if (split) SP2B_CUDA_TRY(c->ensure_split(np));
  // FP64 steps: the measured tile edge for this size (first solve at np on this device)
  if (!split && !exact) {
    const int trc = tune_f64_tile(np, c->x64[0], c->x64[1], c->partials, c->counter,
                                  c->small + 16, st);
    if (trc != SP2B_OK) {
      set_last_error("FP64 tile tuning failed");
      return trc;
    }
  }
  if (oz || exact) {
    if (np > 65536) {
      set_last_error("bad argument: n=%d above the INT8 products' limit", n);
      return SP2B_BAD_ARG;
    }
    SP2B_CUDA_TRY(c->ensure_oz(np, st));
  }

  // ---- input ----
  const double* hsrc = j.inplace ? j.rho : j.h;
  const double* hdev = hsrc;
  if (!j.dev_ptrs) {
    SP2B_CUDA_TRY(copy_symmetric_h2d(c->hin, hsrc, n, st));
    hdev = c->hin;
  }
  double* bounds = c->small;       // [0..1]
  double* norm_out = c->small + 4; // [4..7]
  if (j.given_bounds) {
    c->h_small[0] = j.mineval;
    c->h_small[1] = j.maxeval;
    SP2B_CUDA_TRY(cudaMemcpyAsync(bounds, c->h_small, 2 * sizeof(double), cudaMemcpyHostToDevice, st));
  } else {
    SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), st));
    SP2B_CUDA_TRY(launch_gersh(hdev, n, n, c->rowsum, gersh_nsplit(n), bounds, c->partials,
                               c->counter, st));
  }
  SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(int), st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->sout, 0, sizeof(SolveOut), st));
  if (split)
    SP2B_CUDA_TRY(launch_normalize_split(hdev, n, n, np, bounds, c->hi[0], c->lo[0], bf16,
                                         c->partials, c->counter, c->rec, norm_out, st));
  else
    SP2B_CUDA_TRY(launch_normalize_f64(hdev, n, n, np, bounds, c->x64[0], c->partials, c->counter,
                                       c->rec, norm_out, st));
  if (resp) {
    // Delta_0 = alpha H1 (src/prg_response_mod.F90:700); a host H1 is staged in x64[4]
    const double* h1dev = j.h1;
    if (!j.dev_ptrs) {
      SP2B_CUDA_TRY(copy_symmetric_h2d(c->x64[4], j.h1, n, st));
      h1dev = c->x64[4];
    }
    SP2B_CUDA_TRY(launch_resp_init(h1dev, n, n, np, bounds, c->x64[2], st));
  }

  // ---- control inputs ----
  // pp / vv / icount are host arrays in every mode (only matrices follow device_ptrs)
  if (j.ctl.algo == ALGO_SEQ && j.ctl.icount > 0)
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->pp_dev, j.pp_in, j.ctl.icount * sizeof(int), cudaMemcpyHostToDevice, st));
  if (j.vv_out && j.vv_accumulate && maxlaunch > 0) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->vv_dev, j.vv_out, maxlaunch * sizeof(double), cudaMemcpyHostToDevice, st));
  } else {
    SP2B_CUDA_TRY(cudaMemsetAsync(c->vv_dev, 0, (maxlaunch + 2) * sizeof(double), st));
  }
  int* pp_out_dev = (j.ctl.algo == ALGO_SEQ) ? nullptr : c->pp_dev;

  // ---- SP2 steps: one launch each, chunked host polling of the device "done" word ----
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.control = 1;
  a.ctl = j.ctl;
  // Stagnation of Tr(X - X^2) counts once it is within 32 x its rounding floor, ~N eps
  // for products with relative error eps (2^-22 FP16 hi+lo, 2^-16 BF16 hi+lo, 2^-35
  // exact INT8 after the 2^-S rounding of X).  The exact mode runs to the alg2 rule or
  // to that stagnation (no mixed_tol, no McWeeny step).
  {
    const double eps = exact ? 0x1p-35 : (bf16 ? 0x1p-16 : 0x1p-22);
    a.ctl.stag_tol = 32.0 * eps * (double)n;
    if (exact) a.ctl.mixed_tol = 0.0;
  }
  a.rec = c->rec;
  a.pp_in = c->pp_dev;
  a.pp_out = pp_out_dev;
  a.vv_out = c->vv_dev;
  a.vv_accumulate = j.vv_accumulate;
  a.core = j.core;
  a.sout = c->sout;
  a.partials = c->partials;
  a.counter = c->counter;
  a.err = c->err;
  int k = 0;
  int chunk = 4;
  bool done = (maxlaunch == 0);
  const bool timing = g_step_timing.load() != 0;
  while (!done && k < maxlaunch) {
    if (fallback && k >= j.exact_switch) {   // still running: a nearly gapless spectrum
      *want_exact = true;
      return SP2B_OK;
    }
    int kend = std::min(maxlaunch, k + chunk);
    if (fallback) kend = std::min(kend, std::max(j.exact_switch, k + 1));
    const int k0 = k;
    if (timing) {
      while ((int)c->ev.size() < 2 * chunk) {
        cudaEvent_t e;
        SP2B_CUDA_TRY(cudaEventCreate(&e));
        c->ev.push_back(e);
      }
    }
    for (; k < kend; ++k) {
      a.k = k;
      if (timing) SP2B_CUDA_TRY(cudaEventRecord(c->ev[2 * (k - k0)], st));
      const int bin = k & 1, bout = (k + 1) & 1;
      if (exact) {
        // X_k^2 exactly: residue planes of rint(2^S X_k), nine INT8 products, then the
        // CRT kernel applies step k's branch and publishes the step's record
        OzStepCtl oc;
        oc.sout = c->sout;
        oc.rec = c->rec;
        oc.pp_in = c->pp_dev;
        oc.ctl = a.ctl;
        oc.k = k;
        oc.active = 1;
        SP2B_CUDA_TRY(launch_oz_planes_f64(c->x64[bin], np, c->oz_scale, c->oz_res, &oc, st));
        SP2B_CUDA_TRY(launch_oz_gemm(c->oz_res, np, c->oz_q, c->oz_tiles, c->oz_ntiles, c->err, st, &oc));
        a.E = c->x64[bin];
        a.out = c->x64[bout];
        SP2B_CUDA_TRY(launch_oz_crt_step(c->oz_q, c->oz_scale, a, st));
      } else if (split) {
        a.A = a.B = a.E = c->hi[bin];
        a.A_lo = a.B_lo = a.E_lo = c->lo[bin];
        a.out = c->hi[bout];
        a.out_lo = c->lo[bout];
        a.ntiles = tc_ntiles(np);
        SP2B_CUDA_TRY(launch_sym_gemm_tc(a, bf16, st));
      } else {
        a.A = a.B = a.E = c->x64[bin];
        a.out = c->x64[bout];
        a.ntiles = f64_ntiles(np);
        SP2B_CUDA_TRY(launch_sym_gemm_f64(a, st));
      }
      if (timing) SP2B_CUDA_TRY(cudaEventRecord(c->ev[2 * (k - k0) + 1], st));
      if (resp) {
        // {X_k, Delta_k} on the upper tiles from two products that follow step k's branch
        // (a, b) = (1, 0) or (-1, 2): P1 = a X Delta + b Delta, Delta' = a Delta X + P1
        // (src/prg_response_mod.F90:725-746); both exactly symmetric by construction
        StepArgs q = a;
        q.pp_out = nullptr;
        q.vv_out = nullptr;
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
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_sout, c->sout, sizeof(SolveOut), cudaMemcpyDeviceToHost, st));
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    done = c->h_sout->done != 0;
    if (timing) {
      // only launches that did work (k < the launch that finished the loop, + itself)
      double ms = 0.0;
      long long cnt = 0;
      const int last = done ? std::max(c->h_sout->nupd, k0) : kend - 1;
      for (int q = k0; q < kend && q <= last; ++q) {
        float t = 0.f;
        SP2B_CUDA_TRY(cudaEventElapsedTime(&t, c->ev[2 * (q - k0)], c->ev[2 * (q - k0) + 1]));
        ms += t;
        ++cnt;
      }
      std::lock_guard<std::mutex> lk2(g_timing_mu);
      g_step_ms += ms;
      g_step_timed += cnt;
    }
    chunk = std::min(chunk * 2, 16);
  }
  c->last_launches = k;
  SolveOut so = *c->h_sout;
  if (maxlaunch == 0) so.nupd = 0;
  if (fallback && so.nupd > 0) {
    // the stop reason: Tr X - Tr P of the last update above mixed_tol means the
    // stagnation test (or maxsp2iter) ended the loop
    SP2Rec last;
    SP2B_CUDA_TRY(cudaMemcpyAsync(&last, c->rec + so.nupd, sizeof(SP2Rec), cudaMemcpyDeviceToHost, st));
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    if (so.status == SP2B_OK && (last.err_hist[1] > j.ctl.mixed_tol ||
                                 !(last.err_hist[1] == last.err_hist[1]))) {
      *want_exact = true;
      return SP2B_OK;
    }
    if (so.status == SP2B_NOT_CONVERGED) {
      *want_exact = true;
      return SP2B_OK;
    }
  }
  // normalisation itself may have flagged bad input
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_small + 8, norm_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  const double emin = c->h_small[8], emax = c->h_small[9];
  if (!(emax - emin > 0.0) || !(emin == emin) || !(emax == emax)) {
    set_last_error("non-finite or degenerate spectral bounds (%g, %g)", emin, emax);
    return SP2B_BAD_INPUT;
  }
  // ||X0||_F^2 of the normalised input: a NaN / Inf in H shows here even when no SP2
  // step runs (icount = 0) to flag it
  if (!(c->h_small[11] == c->h_small[11]) || c->h_small[11] > 1e300) {
    set_last_error("non-finite values in the input matrix");
    return SP2B_BAD_INPUT;
  }
  if (!done && maxlaunch > 0) {
    set_last_error("SP2 loop ended without a final state");
    return SP2B_CUDA_ERROR;
  }

  // ---- final density: D = 2 X (FP64) or McWeeny refinement of the split iterate ----
  const int fb = so.nupd & 1;
  double* rho_dev = j.dev_ptrs ? j.rho : c->hin;
  if (oz) {
    // D = 3X^2 - 2X^3 (times 2) = 2X^2 - 4X(X^2 - X): X^2 from exact INT8 residue
    // products, the small correction X (4R) from one split-precision product.
    const int ob = 1 - fb;
    if (timing) {
      while ((int)c->ev_ref.size() < 5) {
        cudaEvent_t e;
        SP2B_CUDA_TRY(cudaEventCreate(&e));
        c->ev_ref.push_back(e);
      }
      SP2B_CUDA_TRY(cudaEventRecord(c->ev_ref[0], st));
    }
    SP2B_CUDA_TRY(launch_oz_planes(c->hi[fb], c->lo[fb], np, bf16, c->oz_scale, c->oz_res, st));
    if (timing) SP2B_CUDA_TRY(cudaEventRecord(c->ev_ref[1], st));
    SP2B_CUDA_TRY(launch_oz_gemm(c->oz_res, np, c->oz_q, c->oz_tiles, c->oz_ntiles, c->err, st));
    if (timing) SP2B_CUDA_TRY(cudaEventRecord(c->ev_ref[2], st));
    SP2B_CUDA_TRY(launch_oz_crt(c->oz_q, c->hi[fb], c->lo[fb], np, bf16, c->oz_scale, c->x64[0],
                                c->hi[ob], c->lo[ob], st));
    if (timing) SP2B_CUDA_TRY(cudaEventRecord(c->ev_ref[3], st));
    SP2B_CUDA_TRY(launch_mcweeny_tc(c->hi[fb], c->lo[fb], c->hi[ob], c->lo[ob], c->x64[0], np,
                                    bf16, rho_dev, n, n, c->partials, c->counter, c->small + 16,
                                    c->err, st));
    if (timing) SP2B_CUDA_TRY(cudaEventRecord(c->ev_ref[4], st));
  } else {
    double* xfin;
    if (split) {
      SP2B_CUDA_TRY(launch_split_to_f64(c->hi[fb], c->lo[fb], np, bf16, c->x64[0], st));
      double* X = c->x64[0];
      double* P = c->x64[1];
      double* D = c->x64[2];
      for (int m = 0; m < j.mcweeny; ++m) {
        StepArgs q;
        memset(&q, 0, sizeof(q));
        q.np = np;
        q.partials = c->partials;
        q.counter = c->counter;
        q.sums_out = c->small + 16;
        // P = X X
        q.A = q.B = q.E = X;
        q.out = P;
        q.alpha = 1.0;
        q.beta = 0.0;
        SP2B_CUDA_TRY(launch_sym_gemm_f64(q, st));
        // D = 3 P - 2 P X   (McWeeny: 3X^2 - 2X^3)
        q.A = P;
        q.B = X;
        q.E = P;
        q.out = D;
        q.alpha = -2.0;
        q.beta = 3.0;
        SP2B_CUDA_TRY(launch_sym_gemm_f64(q, st));
        std::swap(X, D);
      }
      xfin = X;
    } else {
      xfin = c->x64[fb];
    }
    SP2B_CUDA_TRY(launch_finish_f64(xfin, np, n, 2.0, rho_dev, n, st));
  }
  if (!j.dev_ptrs)
    SP2B_CUDA_TRY(cudaMemcpyAsync(j.rho, rho_dev, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (resp) {
    // rho1 = 2 Delta (src/prg_response_mod.F90:771); host output staged in x64[4]
    double* rsp_dev = j.dev_ptrs ? j.rsp : c->x64[4];
    SP2B_CUDA_TRY(launch_finish_f64(c->x64[2 + fb], np, n, 2.0, rsp_dev, n, st));
    if (!j.dev_ptrs)
      SP2B_CUDA_TRY(cudaMemcpyAsync(j.rsp, rsp_dev, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  if (oz) {
    int S = 0;
    double r2max = 0.0;
    SP2B_CUDA_TRY(oz_read_scale(c->oz_scale, &S, &r2max, st));
    c->oz_last_S = S;
    c->oz_last_r2max = r2max;
    if (timing) {
      std::lock_guard<std::mutex> lk2(g_timing_mu);
      for (int ph = 0; ph < 4; ++ph) {
        float t = 0.f;
        SP2B_CUDA_TRY(cudaEventElapsedTime(&t, c->ev_ref[ph], c->ev_ref[ph + 1]));
        g_ref_ms[ph] += t;
      }
      ++g_ref_timed;
    }
    int herr = 0;
    SP2B_CUDA_TRY(cudaMemcpyAsync(&herr, c->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) {
      set_last_error("a device-side wait timed out in the INT8 McWeeny refinement");
      return SP2B_TIMEOUT;
    }
    if (S < 0) {
      set_last_error("INT8 McWeeny refinement: no valid scale (largest row norm^2 %g)", r2max);
      return SP2B_BAD_INPUT;
    }
  }

  // ---- sequence outputs ----
  // (the response loop counts its break iteration, src/prg_response_mod.F90:751; its
  // icount is the number of applied updates, the length of pp)
  const int iters = (j.ctl.algo == ALGO_RESP) ? so.nupd : so.iter;
  if (j.pp_out && iters > 0)
    SP2B_CUDA_TRY(cudaMemcpyAsync(j.pp_out, c->pp_dev, iters * sizeof(int), cudaMemcpyDeviceToHost, st));
  if (j.vv_out) {
    const int nvv = j.vv_accumulate ? maxlaunch : (j.ctl.algo == ALGO_SEQ ? j.ctl.icount : iters);
    if (nvv > 0)
      SP2B_CUDA_TRY(cudaMemcpyAsync(j.vv_out, c->vv_dev, nvv * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  if (j.icount_out) *j.icount_out = iters;
  if (j.iters_out) *j.iters_out = iters;
  if (j.bounds_out) {
    j.bounds_out[0] = emin;
    j.bounds_out[1] = emax;
  }
  if (so.status != SP2B_OK) {
    if (so.status == SP2B_NOT_CONVERGED)
      set_last_error("SP2 purification is not converging (maxsp2iter=%d)", j.ctl.maxit);
    else if (so.status == SP2B_TIMEOUT)
      set_last_error("a device-side wait timed out");
    else if (so.status == SP2B_BAD_INPUT)
      set_last_error("non-finite values during SP2");
    return so.status;
  }
  return SP2B_OK;
}

int dense_solve(const DenseJob& j) {
  t_exact_switch = 0;
  bool want_exact = false;
  const int st = dense_solve_once(j, &want_exact);
  if (st != SP2B_OK || !want_exact) return st;
  // solved again from the input in the exact INT8 form (the split run wrote no output)
  DenseJob e = j;
  e.prec = SP2B_PREC_EXACT_INT8;
  e.exact_switch = 0;
  t_exact_switch = 1;
  return dense_solve_once(e, nullptr);
}

}  // namespace sp2b

using namespace sp2b;

// ======================================================================================
// C ABI
// ======================================================================================
extern "C" {

const char* sp2b_last_error(void) { return g_err; }

int sp2b_last_refinement_info(int* scale_exp, double* r2max) {
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  if (scale_exp) *scale_exp = c->oz_last_S;
  if (r2max) *r2max = c->oz_last_r2max;
  return SP2B_OK;
}

int sp2b_last_exact_switch(void) { return t_exact_switch; }

int sp2b_opts_default(sp2b_opts* o) {
  if (!o) return SP2B_BAD_ARG;
  memset(o, 0, sizeof(*o));
  o->precision = SP2B_PREC_FP64;
  o->mcweeny = 1;
  o->mixed_tol = 1e-3;
  o->mcweeny_products = SP2B_MCW_INT8;
  o->refine_tol = 1e-3;
  o->exact_switch = 40;
  return SP2B_OK;
}

static std::mutex g_def_mu;
static bool g_def_init = false;
static sp2b_opts g_def;

int sp2b_get_default_opts(sp2b_opts* o) {
  if (!o) return SP2B_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_def_mu);
  if (!g_def_init) {
    sp2b_opts_default(&g_def);
    const char* e = getenv("SP2B_PRECISION");
    if (e) {
      if (!strcmp(e, "mixed") || !strcmp(e, "mixed_fp16")) g_def.precision = SP2B_PREC_MIXED_FP16;
      else if (!strcmp(e, "mixed_bf16")) g_def.precision = SP2B_PREC_MIXED_BF16;
      else if (!strcmp(e, "exact") || !strcmp(e, "exact_int8")) g_def.precision = SP2B_PREC_EXACT_INT8;
    }
    g_def_init = true;
  }
  *o = g_def;
  return SP2B_OK;
}

int sp2b_set_default_opts(const sp2b_opts* o) {
  if (!o) return SP2B_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_def_mu);
  g_def = *o;
  g_def_init = true;
  return SP2B_OK;
}

static DenseJob base_job(const double* h, double* rho, int n, const sp2b_opts* o) {
  DenseJob j;
  memset(&j, 0, sizeof(j));
  sp2b_opts d;
  if (!o) {
    sp2b_opts_default(&d);
    o = &d;
  }
  j.h = h;
  j.rho = rho;
  j.n = n;
  j.prec = o->precision;
  j.dev_ptrs = o->device_ptrs != 0;
  j.stream = (cudaStream_t)o->stream;
  j.mcweeny = o->mcweeny;
  j.mcweeny_products = o->mcweeny_products;
  j.exact_switch = o->exact_switch;
  j.ctl.n = n;
  j.ctl.mixed_tol = o->mixed_tol;
  j.ctl.icount = 0;
  return j;
}

static void set_trace_ctl(DenseJob& j, int algo, double bndfil, int minit, int maxit,
                          const char* conv, double idemtol) {
  j.ctl.algo = algo;
  if (j.prec != SP2B_PREC_FP64 && algo != ALGO_SEQ) j.ctl.algo = ALGO_MIXED;
  j.ctl.minit = minit;
  j.ctl.maxit = maxit;
  j.ctl.conv = parse_conv(conv);
  j.ctl.idemtol = idemtol;
  j.ctl.occ = bndfil * (double)j.n;
}

int sp2b_compute_response_sp2(const double* h0, const double* h1, double* rsp, double* rho, int n,
                              double lambda, double bndfil, int minsp2iter, int maxsp2iter,
                              const char* sp2conv, double idemtol, double threshold,
                              int verbose, int* pp, int* icount, const sp2b_opts* opts) {
  (void)lambda;      // unused by the reference as well (src/prg_response_mod.F90:653)
  (void)threshold;   // dense products are not thresholded
  (void)verbose;
  if (!h0 || !h1 || !rsp || !rho) {
    set_last_error("bad argument: NULL matrix");
    return SP2B_BAD_ARG;
  }
  DenseJob j = base_job(h0, rho, n, opts);
  j.prec = SP2B_PREC_FP64;
  j.h1 = h1;
  j.rsp = rsp;
  set_trace_ctl(j, ALGO_RESP, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol);
  j.pp_out = pp;
  j.icount_out = icount;
  return dense_solve(j);
}

int sp2b_sp2_alg2(const double* h, double* rho, int n, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                  int verbose, const sp2b_opts* opts, int* iters_out) {
  (void)threshold; (void)verbose;
  DenseJob j = base_job(h, rho, n, opts);
  set_trace_ctl(j, ALGO_ALG2, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol);
  j.iters_out = iters_out;
  return dense_solve(j);
}

int sp2b_sp2_alg2_genseq(const double* h, double* rho, int n, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                         int* pp, int* icount, double* vv, int verbose, const sp2b_opts* opts) {
  (void)threshold; (void)verbose;
  DenseJob j = base_job(h, rho, n, opts);
  set_trace_ctl(j, ALGO_ALG2_GENSEQ, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol);
  j.pp_out = pp;
  j.vv_out = vv;
  j.icount_out = icount;
  return dense_solve(j);
}

static int seq_job(const double* h, double* rho, int n, const int* pp, int icount, double* vv,
                   bool inplace, double mineval, double maxeval, int core, int accumulate,
                   const sp2b_opts* opts) {
  DenseJob j = base_job(h, rho, n, opts);
  j.ctl.algo = ALGO_SEQ;
  j.ctl.icount = icount;
  j.pp_in = pp;
  j.vv_out = vv;
  j.inplace = inplace;
  j.given_bounds = inplace;
  j.mineval = mineval;
  j.maxeval = maxeval;
  j.core = core;
  j.vv_accumulate = accumulate;
  return dense_solve(j);
}

int sp2b_sp2_alg2_seq(const double* h, double* rho, int n, double threshold, const int* pp,
                      int icount, double* vv, int verbose, const sp2b_opts* opts) {
  (void)threshold; (void)verbose;
  return seq_job(h, rho, n, pp, icount, vv, false, 0, 0, 0, 0, opts);
}

int sp2b_sp2_alg2_seq_inplace(double* rho, int n, double threshold, const int* pp, int icount,
                              double* vv, double mineval, double maxeval, int verbose,
                              const sp2b_opts* opts) {
  (void)threshold; (void)verbose;
  return seq_job(nullptr, rho, n, pp, icount, vv, true, mineval, maxeval, 0, 0, opts);
}

int sp2b_sp2_alg1(const double* h, double* rho, int n, double threshold, double bndfil,
                  int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                  int verbose, const sp2b_opts* opts, int* iters_out) {
  (void)threshold; (void)verbose;
  DenseJob j = base_job(h, rho, n, opts);
  set_trace_ctl(j, ALGO_ALG1, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol);
  j.iters_out = iters_out;
  return dense_solve(j);
}

int sp2b_sp2_alg1_genseq(const double* h, double* rho, int n, double threshold, double bndfil,
                         int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                         int* pp, int* icount, double* vv, const sp2b_opts* opts) {
  (void)threshold;
  DenseJob j = base_job(h, rho, n, opts);
  set_trace_ctl(j, ALGO_ALG1_GENSEQ, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol);
  j.pp_out = pp;
  j.vv_out = vv;
  j.icount_out = icount;
  return dense_solve(j);
}

int sp2b_sp2_alg1_seq(const double* h, double* rho, int n, double threshold, const int* pp,
                      int icount, double* vv, const sp2b_opts* opts) {
  (void)threshold;
  return seq_job(h, rho, n, pp, icount, vv, false, 0, 0, 0, 0, opts);
}

int sp2b_sp2_alg1_seq_inplace(double* rho, int n, double threshold, const int* pp, int icount,
                              double* vv, double mineval, double maxeval, const sp2b_opts* opts) {
  (void)threshold;
  return seq_job(nullptr, rho, n, pp, icount, vv, true, mineval, maxeval, 0, 0, opts);
}

int sp2b_sp2_basic(const double* h, double* rho, int n, double threshold, double bndfil,
                   int minsp2iter, int maxsp2iter, const char* sp2conv, double idemtol,
                   int verbose, const sp2b_opts* opts, int* iters_out) {
  (void)threshold; (void)verbose;
  DenseJob j = base_job(h, rho, n, opts);
  set_trace_ctl(j, ALGO_BASIC, bndfil, minsp2iter, maxsp2iter, sp2conv, idemtol);
  j.iters_out = iters_out;
  return dense_solve(j);
}

int sp2b_sp2_submatrix_inplace(double* rho, int n, double threshold, const int* pp, int icount,
                               double* vv, double mineval, double maxeval, int core_size,
                               const sp2b_opts* opts) {
  (void)threshold;
  if (core_size < 0 || core_size > n) {
    set_last_error("bad argument: core_size=%d n=%d", core_size, n);
    return SP2B_BAD_ARG;
  }
  // core_size = 0: bml_sum_squares_submatrix over no rows adds nothing, so vv is left
  // as the caller passed it
  return seq_job(nullptr, rho, n, pp, icount, core_size > 0 ? vv : nullptr, true, mineval,
                 maxeval, core_size > 0 ? core_size : -1, 1, opts);
}

int sp2b_sp2_submatrix(const double* ham, double* rho, int n, double threshold, const int* pp,
                       int icount, double* vv, double mineval, double maxeval, int core_size,
                       const sp2b_opts* opts) {
  (void)threshold;
  if (core_size < 0 || core_size > n) {
    set_last_error("bad argument: core_size=%d n=%d", core_size, n);
    return SP2B_BAD_ARG;
  }
  DenseJob j = base_job(ham, rho, n, opts);
  j.ctl.algo = ALGO_SEQ;
  j.ctl.icount = icount;
  j.pp_in = pp;
  j.vv_out = core_size > 0 ? vv : nullptr;   // no core rows: vv gains nothing
  j.given_bounds = true;
  j.mineval = mineval;
  j.maxeval = maxeval;
  j.core = core_size > 0 ? core_size : -1;
  j.vv_accumulate = 1;
  return dense_solve(j);
}

int sp2b_gershgorin(const double* h, int n, double* mineval, double* maxeval,
                    const sp2b_opts* opts) {
  if (n <= 0 || !h || !mineval || !maxeval) {
    set_last_error("bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  const bool dev = opts && opts->device_ptrs;
  cudaStream_t st = pick_stream(opts, c);
  const size_t nn = (size_t)n * n;
  SP2B_CUDA_TRY(c->ensure_common(dev ? 0 : nn, padded(n), 1, n));
  const double* hd = h;
  if (!dev) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->hin, h, nn * sizeof(double), cudaMemcpyHostToDevice, st));
    hd = c->hin;
  }
  SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), st));
  SP2B_CUDA_TRY(launch_gersh(hd, n, n, c->rowsum, gersh_nsplit(n), c->small, c->partials,
                               c->counter, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_small, c->small, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  *mineval = c->h_small[0];
  *maxeval = c->h_small[1];
  if (!(c->h_small[0] == c->h_small[0]) || !(c->h_small[1] == c->h_small[1])) {
    set_last_error("non-finite values in H");
    return SP2B_BAD_INPUT;
  }
  return SP2B_OK;
}

int sp2b_normalize(double* h, int n, double* mineval, double* maxeval, const sp2b_opts* opts) {
  double lo, hi;
  int s = sp2b_gershgorin(h, n, &lo, &hi, opts);
  if (s != SP2B_OK) return s;
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  const bool dev = opts && opts->device_ptrs;
  cudaStream_t st = pick_stream(opts, c);
  const int np = padded(n);
  const size_t nn = (size_t)n * n;
  SP2B_CUDA_TRY(c->ensure_common(dev ? 0 : nn, np, 1, n));
  SP2B_CUDA_TRY(c->ensure_f64(np, 1));
  const double* hd = h;
  if (!dev) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->hin, h, nn * sizeof(double), cudaMemcpyHostToDevice, st));
    hd = c->hin;
  }
  c->h_small[0] = lo;
  c->h_small[1] = hi;
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->small, c->h_small, 2 * sizeof(double), cudaMemcpyHostToDevice, st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), st));
  SP2B_CUDA_TRY(launch_normalize_f64(hd, n, n, np, c->small, c->x64[0], c->partials, c->counter,
                                     c->rec, c->small + 4, st));
  double* out = dev ? h : c->hin;
  SP2B_CUDA_TRY(launch_finish_f64(c->x64[0], np, n, 1.0, out, n, st));
  if (!dev) SP2B_CUDA_TRY(cudaMemcpyAsync(h, out, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  if (mineval) *mineval = lo;
  if (maxeval) *maxeval = hi;
  return SP2B_OK;
}

int sp2b_check_idempotency(const double* a, int n, double threshold, double* idempotency,
                           const sp2b_opts* opts) {
  (void)threshold;
  if (n <= 0 || !a || !idempotency) {
    set_last_error("bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  const bool dev = opts && opts->device_ptrs;
  cudaStream_t st = pick_stream(opts, c);
  const int np = padded(n);
  const size_t nn = (size_t)n * n;
  SP2B_CUDA_TRY(c->ensure_common(dev ? 0 : nn, np, 1, n));
  SP2B_CUDA_TRY(c->ensure_f64(np, 1));
  const double* ad = a;
  if (!dev) {
    SP2B_CUDA_TRY(cudaMemcpyAsync(c->hin, a, nn * sizeof(double), cudaMemcpyHostToDevice, st));
    ad = c->hin;
  }
  SP2B_CUDA_TRY(launch_copy_in(ad, n, n, np, c->x64[0], st));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->counter, 0, 4 * sizeof(unsigned), st));
  StepArgs q;
  memset(&q, 0, sizeof(q));
  q.np = np;
  q.A = q.B = q.E = c->x64[0];
  q.out = nullptr;
  q.alpha = 1.0;
  q.beta = 0.0;
  q.partials = c->partials;
  q.counter = c->counter;
  q.sums_out = c->small + 16;
  SP2B_CUDA_TRY(launch_sym_gemm_f64(q, st));
  SP2B_CUDA_TRY(cudaMemcpyAsync(c->h_small + 16, c->small + 16, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  *idempotency = sqrt(c->h_small[18]);
  return SP2B_OK;
}

int sp2b_selftest_wait_timeout(int spin_limit) {
  if (spin_limit < 1) {
    set_last_error("spin_limit must be positive");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  SP2B_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(int), c->stream));
  SP2B_CUDA_TRY(launch_wait_selftest((uint32_t)spin_limit, c->err, c->stream));
  int herr = 0;
  SP2B_CUDA_TRY(cudaMemcpyAsync(&herr, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  SP2B_CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (herr != 0) {
    set_last_error("self-test: a bounded device wait ran out after %d polls", spin_limit);
    return SP2B_TIMEOUT;
  }
  return SP2B_OK;
}

long long sp2b_launch_count(void) { return g_launches.load(); }

int sp2b_set_step_timing(int enable) {
  std::lock_guard<std::mutex> lk(g_timing_mu);
  g_step_timing.store(enable ? 1 : 0);
  g_step_ms = 0.0;
  g_step_timed = 0;
  for (double& v : g_ref_ms) v = 0.0;
  g_ref_timed = 0;
  return SP2B_OK;
}

int sp2b_refinement_timing(double* ms4, long long* solves) {
  std::lock_guard<std::mutex> lk(g_timing_mu);
  if (ms4)
    for (int i = 0; i < 4; ++i) ms4[i] = g_ref_ms[i];
  if (solves) *solves = g_ref_timed;
  return SP2B_OK;
}

int sp2b_step_timing(double* ms, long long* launches) {
  std::lock_guard<std::mutex> lk(g_timing_mu);
  if (ms) *ms = g_step_ms;
  if (launches) *launches = g_step_timed;
  return SP2B_OK;
}

int sp2b_last_solve_info(int* launches, int* nupd, int* iter, int* status, double* recs,
                         int max_recs) {
  int st = SP2B_OK;
  Ctx* c = get_ctx(&st);
  if (!c) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  if (!c->sout) return SP2B_BAD_ARG;
  SolveOut so;
  SP2B_CUDA_TRY(cudaMemcpy(&so, c->sout, sizeof(so), cudaMemcpyDeviceToHost));
  if (launches) *launches = c->last_launches;
  if (nupd) *nupd = so.nupd;
  if (iter) *iter = so.iter;
  if (status) *status = so.status;
  if (recs && max_recs > 0 && c->rec) {
    const int m = (int)std::min((size_t)max_recs, c->rec_cap);
    std::vector<SP2Rec> r(m);
    SP2B_CUDA_TRY(cudaMemcpy(r.data(), c->rec, m * sizeof(SP2Rec), cudaMemcpyDeviceToHost));
    for (int i = 0; i < m; ++i) {
      double* o = recs + 9 * i;
      o[0] = r[i].trx; o[1] = r[i].trx_data; o[2] = r[i].fro2; o[3] = r[i].idemperr;
      o[4] = r[i].iter; o[5] = r[i].done; o[6] = r[i].status; o[7] = r[i].last_branch;
      o[8] = r[i].trp;
    }
  }
  return SP2B_OK;
}

int sp2b_dev_panel_gemm_f32(const float* a_rows, int m, const float* b, int n, float* cout,
                            void* stream) {
  if (m <= 0 || n <= 0 || m > n || !a_rows || !b || !cout) {
    set_last_error("sp2b_dev_panel_gemm_f32: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = (cudaStream_t)stream;  // device arrays: NULL = the default stream
  const int np = padded(n), mp = padded(m);
  SP2B_CUDA_TRY(c->ensure_split(np));      // mp x np <= np x np
  SP2B_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(int), st));
  SP2B_CUDA_TRY(launch_f32_rows_to_split(a_rows, m, n, mp, np, c->hi[0], c->lo[0], st));
  SP2B_CUDA_TRY(launch_f32_to_split(b, n, np, c->hi[1], c->lo[1], st));
  SP2B_CUDA_TRY(launch_tc_panel(c->hi[0], c->lo[0], mp, c->hi[1], c->lo[1], np, cout, m, n, st,
                                c->err));
  return SP2B_OK;
}

int sp2b_dev_sym_gemm_f32(const float* a, const float* b, float* cout, int n, void* stream) {
  if (n <= 0 || !a || !b || !cout) {
    set_last_error("bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = (cudaStream_t)stream;  // device arrays: NULL = the default stream
  const int np = padded(n);
  SP2B_CUDA_TRY(c->ensure_split(np));
  SP2B_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(int), st));
  SP2B_CUDA_TRY(launch_f32_to_split(a, n, np, c->hi[0], c->lo[0], st));
  SP2B_CUDA_TRY(launch_f32_to_split(b, n, np, c->hi[1], c->lo[1], st));
  SP2B_CUDA_TRY(launch_tc_plain(c->hi[0], c->lo[0], c->hi[1], c->lo[1], np, cout, n, st, c->err));
  return SP2B_OK;
}

}  // extern "C"
