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
// The FP32 entries take n x n FP32 matrices and convert to FP16 hi+lo splits around each
// product (FP32 accumulation on the tensor cores).  The split entries keep X and G in
// the split form between steps (np x np hi and lo arrays, np = sp2b_split_dim(n), zeros
// outside the n x n block): a forward step is one symmetric product whose epilogue
// writes the next split iterate, and a reverse step forms {G, X} as one symmetric
// product over the concatenated K range [G | X] [X | G]^T with the branch applied in the
// same epilogue, so neither a conversion nor an M + M^T pass runs between steps.
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

// FP16 hi + lo split with lo scaled by 2^11, as the tensor-core kernels store it
constexpr double kLoScale = 2048.0;
constexpr float kLoInv = 1.0f / 2048.0f;
__device__ __forceinline__ void split_store(double v, __half* hi, __half* lo, size_t i) {
  const __half hv = __double2half(v);
  hi[i] = hv;
  lo[i] = __double2half((v - (double)__half2float(hv)) * kLoScale);
}

// X_0 = a H + b I straight into the split form, one CTA per padded row; the FP32 value is
// formed first and split as k_f32_to_split splits it, so the split X_0 equals the
// FP32 path's.
__global__ void k_normalize_to_split(const float* __restrict__ h, int n, int np, float a, float b,
                                     __half* __restrict__ hi, __half* __restrict__ lo) {
  const int r = blockIdx.x;
  for (int c = threadIdx.x; c < np; c += blockDim.x) {
    float x = 0.f;
    if (r < n && c < n) x = a * h[(size_t)r * n + c] + (r == c ? b : 0.f);
    split_store((double)x, hi, lo, (size_t)r * np + c);
  }
}

// y = scale (hi + 2^-11 lo) over the n x n block, one CTA per row (hi + 2^-11 lo is exact
// in FP32: 22 significant bits).
__global__ void k_split_rows_to_f32(const __half* __restrict__ hi, const __half* __restrict__ lo,
                                    int n, int np, float scale, float* __restrict__ y) {
  const int r = blockIdx.x;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const size_t s = (size_t)r * np + c;
    y[(size_t)r * n + c] = scale * (__half2float(hi[s]) + kLoInv * __half2float(lo[s]));
  }
}

// Split form of out = (M + M^T) or 2 G - (M + M^T) over the padded np x np arrays (M = G X
// in FP32), for sizes the paired anticommutator launch does not take; 32 x 32 tiles
// through shared memory as in k_adjoint_combine.
__global__ void k_adjoint_combine_split(const float* __restrict__ m, const __half* __restrict__ ghi,
                                        const __half* __restrict__ glo, int np, int branch,
                                        __half* __restrict__ ohi, __half* __restrict__ olo) {
  __shared__ float t[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y)
    t[j][threadIdx.x] = m[(size_t)(bx + j) * np + by + threadIdx.x];
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const size_t idx = (size_t)(by + j) * np + bx + threadIdx.x;
    const float anti = m[idx] + t[threadIdx.x][j];
    const float g = __half2float(ghi[idx]) + kLoInv * __half2float(glo[idx]);
    split_store((double)(branch ? anti : 2.f * g - anti), ohi, olo, idx);
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

int sp2b_split_dim(int n) { return n > 0 ? padded(n) : 0; }

int sp2b_dev_normalize_split(const float* h, int n, double mineval, double maxeval, void* x_hi,
                             void* x_lo, void* stream) {
  if (!h || !x_hi || !x_lo || n <= 0 || !(maxeval - mineval > 0.0)) {
    set_last_error("sp2b_dev_normalize_split: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  if (!get_ctx(&status)) return status;
  const double mm = maxeval - mineval;
  const int np = padded(n);
  k_normalize_to_split<<<np, 256, 0, (cudaStream_t)stream>>>(
      h, n, np, (float)(-1.0 / mm), (float)(maxeval / mm), (__half*)x_hi, (__half*)x_lo);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  return SP2B_OK;
}

int sp2b_dev_f32_to_split(const float* a, int n, void* hi, void* lo, void* stream) {
  if (!a || !hi || !lo || n <= 0) {
    set_last_error("sp2b_dev_f32_to_split: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  if (!get_ctx(&status)) return status;
  SP2B_CUDA_TRY(launch_f32_to_split(a, n, padded(n), (__half*)hi, (__half*)lo,
                                    (cudaStream_t)stream));
  return SP2B_OK;
}

int sp2b_dev_split_to_f32(const void* hi, const void* lo, int n, double scale, float* y,
                          void* stream) {
  if (!hi || !lo || !y || n <= 0) {
    set_last_error("sp2b_dev_split_to_f32: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  if (!get_ctx(&status)) return status;
  k_split_rows_to_f32<<<n, 256, 0, (cudaStream_t)stream>>>((const __half*)hi, (const __half*)lo, n,
                                                          padded(n), (float)scale, y);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  return SP2B_OK;
}

int sp2b_dev_sp2_step_split(const void* x_hi, const void* x_lo, void* y_hi, void* y_lo, int n,
                            int branch, void* stream) {
  if (!x_hi || !x_lo || !y_hi || !y_lo || n <= 0 || (branch != 0 && branch != 1) ||
      x_hi == y_hi || x_lo == y_lo) {
    set_last_error("sp2b_dev_sp2_step_split: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = (cudaStream_t)stream;
  const int np = padded(n);
  SP2B_CUDA_TRY(c->ensure_common(0, np, 1, n));
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.A = a.B = a.E = x_hi;
  a.A_lo = a.B_lo = a.E_lo = x_lo;
  a.out = y_hi;
  a.out_lo = y_lo;
  a.alpha = branch ? 1.0 : -1.0;
  a.beta = branch ? 0.0 : 2.0;
  a.err = c->err;   // no partials: the step's traces are not formed
  SP2B_CUDA_TRY(launch_sym_gemm_tc(a, 0, st));
  return SP2B_OK;
}

int sp2b_dev_adjoint_step_split(const void* g_hi, const void* g_lo, const void* x_hi,
                                const void* x_lo, void* o_hi, void* o_lo, int n, int branch,
                                void* stream) {
  if (!g_hi || !g_lo || !x_hi || !x_lo || !o_hi || !o_lo || n <= 0 ||
      (branch != 0 && branch != 1) || o_hi == g_hi || o_hi == x_hi || o_lo == g_lo ||
      o_lo == x_lo) {
    set_last_error("sp2b_dev_adjoint_step_split: bad argument");
    return SP2B_BAD_ARG;
  }
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = (cudaStream_t)stream;
  const int np = padded(n);
  SP2B_CUDA_TRY(c->ensure_common(0, np, 1, n));
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.A = a.E = g_hi;
  a.A_lo = a.E_lo = g_lo;
  a.B = x_hi;
  a.B_lo = x_lo;
  a.out = o_hi;
  a.out_lo = o_lo;
  a.alpha = branch ? 1.0 : -1.0;   // {G, X} or 2 G - {G, X}
  a.beta = branch ? 0.0 : 2.0;
  a.err = c->err;   // no partials: the product's sums are not formed
  cudaError_t e = launch_anti_tc(a, st);
  if (e != cudaErrorNotSupported) {
    SP2B_CUDA_TRY(e);
    return SP2B_OK;
  }
  // np not a multiple of 256: M = G X in FP32 (full product), then the split combine
  SP2B_CUDA_TRY(c->ensure_f64(np, 1));
  float* m = reinterpret_cast<float*>(c->x64[0]);
  SP2B_CUDA_TRY(launch_tc_plain((const __half*)g_hi, (const __half*)g_lo, (const __half*)x_hi,
                                (const __half*)x_lo, np, m, np, st, c->err));
  dim3 grid(np / 32, np / 32), block(32, 8);
  k_adjoint_combine_split<<<grid, block, 0, st>>>(m, (const __half*)g_hi, (const __half*)g_lo, np,
                                                  branch, (__half*)o_hi, (__half*)o_lo);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  return SP2B_OK;
}

}  // extern "C"
