// Device building blocks of the differentiable SP2 (the autograd path).
//
// Forward:  X_{k+1} = X_k^2 (pp_k = 1) or 2 X_k - X_k^2 (pp_k = 0), X_0 = a H + b I.
// Reverse:  with G_k = dL/dX_k,
//             G_k = {G_{k+1}, X_k}            (pp_k = 1)
//             G_k = 2 G_{k+1} - {G_{k+1}, X_k} (pp_k = 0),  {G, X} = G X + X G,
//           and dL/dH = a G_0 (bounds held fixed).
// For symmetric G and X, X G = (G X)^T, so one product M = G X and M + M^T give the
// anticommutator.  This is the transpose of the forward-mode recursion of
// prg_compute_response_SP2 (src/prg_response_mod.F90:653-782), which propagates
// Delta_{k+1} = {X_k, Delta_k} or 2 Delta_k - {X_k, Delta_k}.
// All matrices are n x n FP32 on the device; products run as FP16 hi+lo splits on the
// tensor cores (k_tc_gemm), FP32 accumulation.
#include <mutex>

#include "kernels.cuh"
#include "sp2b_ctx.h"

namespace sp2b {

// out = (M + M^T) or 2 G - (M + M^T); 32 x 32 tiles through shared memory so that
// both M and its transpose are read coalesced.
__global__ void k_adjoint_combine(const float* __restrict__ m, const float* __restrict__ g,
                                  float* __restrict__ out, int n, int branch) {
  __shared__ float t[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  // load the transposed block M[bx.., by..] into t
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = bx + j, c = by + threadIdx.x;
    t[j][threadIdx.x] = (r < n && c < n) ? m[(size_t)r * n + c] : 0.f;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = by + j, c = bx + threadIdx.x;
    if (r < n && c < n) {
      const size_t idx = (size_t)r * n + c;
      const float anti = m[idx] + t[threadIdx.x][j];  // M[r][c] + M[c][r]
      out[idx] = branch ? anti : 2.f * g[idx] - anti;
    }
  }
}

__global__ void k_split_to_f32(const __half* __restrict__ hi, const __half* __restrict__ lo,
                               int n, int np, float* __restrict__ y) {
  const size_t total = (size_t)n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i % n);
    const size_t s = (size_t)r * np + c;
    y[i] = (float)((double)__half2float(hi[s]) + (1.0 / 2048.0) * (double)__half2float(lo[s]));
  }
}

__global__ void k_normalize_f32(const float* __restrict__ h, int n, float a, float b,
                                float* __restrict__ x) {
  const size_t total = (size_t)n * n;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / n), c = (int)(i % n);
    x[i] = a * h[i] + (r == c ? b : 0.f);
  }
}

static int grid1d(size_t total) {
  size_t g = (total + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  return (int)(g ? g : 1);
}

}  // namespace sp2b

using namespace sp2b;

extern "C" {

int sp2b_dev_normalize_f32(const float* h, float* x, int n, double mineval, double maxeval,
                           void* stream) {
  if (!h || !x || n <= 0 || !(maxeval - mineval > 0.0)) {
    set_last_error("sp2b_dev_normalize_f32: bad argument");
    return SP2B_BAD_ARG;
  }
  const double mm = maxeval - mineval;
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  (void)c;
  k_normalize_f32<<<grid1d((size_t)n * n), 256, 0, (cudaStream_t)stream>>>(
      h, n, (float)(-1.0 / mm), (float)(maxeval / mm), x);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  return SP2B_OK;
}

int sp2b_dev_sp2_step_f32(const float* x, float* y, int n, int branch, void* stream) {
  if (!x || !y || n <= 0 || (branch != 0 && branch != 1)) {
    set_last_error("sp2b_dev_sp2_step_f32: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = (cudaStream_t)stream;  // device arrays: NULL = the default stream
  const int np = padded(n);
  SP2B_CUDA_TRY(c->ensure_split(np));
  SP2B_CUDA_TRY(c->ensure_common(0, np, 1, n));
  SP2B_CUDA_TRY(launch_f32_to_split(x, n, np, c->hi[0], c->lo[0], st));
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.A = a.B = a.E = c->hi[0];
  a.A_lo = a.B_lo = a.E_lo = c->lo[0];
  a.out = c->hi[1];
  a.out_lo = c->lo[1];
  a.alpha = branch ? 1.0 : -1.0;
  a.beta = branch ? 0.0 : 2.0;
  a.partials = c->partials;
  a.counter = c->counter;
  a.sums_out = c->small + 24;
  a.err = c->err;
  SP2B_CUDA_TRY(launch_sym_gemm_tc(a, 0, st));
  k_split_to_f32<<<grid1d((size_t)n * n), 256, 0, st>>>(c->hi[1], c->lo[1], n, np, y);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  return SP2B_OK;
}

int sp2b_dev_adjoint_step_f32(const float* g, const float* x, float* g_out, float* work, int n,
                              int branch, void* stream) {
  if (!g || !x || !g_out || !work || n <= 0 || (branch != 0 && branch != 1)) {
    set_last_error("sp2b_dev_adjoint_step_f32: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  (void)c;
  cudaStream_t st = (cudaStream_t)stream;  // NULL = the default stream, for both kernels
  int s = sp2b_dev_sym_gemm_f32(g, x, work, n, st);  // M = G X
  if (s != SP2B_OK) return s;
  dim3 grid((n + 31) / 32, (n + 31) / 32), block(32, 8);
  k_adjoint_combine<<<grid, block, 0, st>>>(work, g, g_out, n, branch);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  return SP2B_OK;
}

}  // extern "C"
