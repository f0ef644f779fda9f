// Per-device library context and the dense-solve job description.
#pragma once
#include <algorithm>
#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace sp2b {

struct Ctx {
  bool init = false;
  int dev = -1;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  // FP64 square buffers (np x np): ping-pong iterates [0, 1]; the FP64-DMMA McWeeny
  // product [2]; the forward-mode response's Delta ping-pong [2, 3] and its first
  // product / host staging [4]
  double* x64[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  size_t x64_cap[5] = {0, 0, 0, 0, 0};
  // split-precision iterates (hi/lo ping-pong)
  __half* hi[2] = {nullptr, nullptr};
  __half* lo[2] = {nullptr, nullptr};
  size_t hi_cap[2] = {0, 0}, lo_cap[2] = {0, 0};
  // host-pointer staging of H / rho (n x n)
  double* hin = nullptr;
  size_t hin_cap = 0;
  // reductions and control
  double* partials = nullptr;
  size_t partials_cap = 0;
  unsigned* counter = nullptr;
  SP2Rec* rec = nullptr;
  size_t rec_cap = 0;
  int* pp_dev = nullptr;
  size_t pp_cap = 0;
  double* vv_dev = nullptr;
  size_t vv_cap = 0;
  double* rowsum = nullptr;
  size_t rowsum_cap = 0;
  double* small = nullptr;      // device scratch scalars
  double* h_small = nullptr;    // pinned host mirror
  SolveOut* sout = nullptr;
  SolveOut* h_sout = nullptr;   // pinned
  int* err = nullptr;
  // INT8 refinement: residue planes, reduced product planes, tile list, scale state
  int8_t* oz_res = nullptr;
  uint8_t* oz_q = nullptr;
  size_t oz_cap = 0;
  int2* oz_tiles = nullptr;
  int oz_tiles_np = 0, oz_ntiles = 0;
  void* oz_scale = nullptr;
  int oz_last_S = 0;            // scale exponent of the last INT8 refinement
  double oz_last_r2max = 0.0;   // its largest squared row norm
  int last_launches = 0;            // SP2 step launches of the last dense solve
  std::vector<cudaEvent_t> ev;      // step timing events (pairs)
  std::vector<cudaEvent_t> ev_ref;  // INT8 refinement phase boundaries

  cudaError_t ensure_f64(int np, int nbuf);
  cudaError_t ensure_split(int np);
  cudaError_t ensure_common(size_t nin, int np, int maxlaunch, int n);
  cudaError_t ensure_oz(int np, cudaStream_t st);
};

Ctx* get_ctx(int* status);

struct DenseJob {
  const double* h;
  double* rho;
  int n;
  int prec;
  bool dev_ptrs;
  cudaStream_t stream;
  bool inplace;        // H read from rho (the *_inplace routines)
  bool given_bounds;   // use mineval/maxeval instead of Gershgorin
  double mineval, maxeval;
  SP2Ctl ctl;
  const int* pp_in;
  int* pp_out;
  double* vv_out;
  int vv_accumulate;
  int core;
  int* icount_out;
  int* iters_out;
  double* bounds_out;
  int mcweeny;
  int mcweeny_products;  // SP2B_MCW_INT8 or SP2B_MCW_FP64
  int exact_switch;      // mixed: steps after which a still-running loop restarts exact
  const double* h1;      // forward-mode response: perturbation H1 (nullptr: plain solve)
  double* rsp;           // ... and its output, the response rho1 = 2 Delta
};

int dense_solve(const DenseJob& j);

}  // namespace sp2b
