// Graph of the sub-graph loop on the GPU: the pattern of |H^2| > gthreshold from H in
// CSR, the graph the sub-graph benchmark partitions (its H^2 graph,
// benchmarks/dmconstruction_graphBased/dmconstruction_graphBased.F90:63-65; the
// reference forms it with a BML sparse product and a threshold).
//
// One warp per row i of H^2.  The candidate columns of row i are collected in a
// per-warp open-addressing table in shared memory (2048 slots): for each entry (i, k)
// of H in row order, the lanes take the entries (k, j) of row k; the columns j of one
// row are distinct, so within one entry (i, k) no two lanes add into the same slot,
// and each G_ij = sum_k H_ik H_kj is summed in the order of row i's entries, with
// separately rounded products and sums (as a CPU loop over the rows does).  Columns
// with |G_ij| > gthreshold are counted (first pass) or written in ascending order
// (second pass, after a host prefix sum of the counts).
#include <algorithm>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "sp2b_ctx.h"

namespace sp2b {

constexpr int kGraphSlots = 2048;   // candidate columns per row of H^2
constexpr int kGraphWarps = 4;      // rows per CTA

template <bool FILL>
__global__ void __launch_bounds__(kGraphWarps * 32)
    k_square_graph(int n, const long long* __restrict__ rp, const int* __restrict__ col,
                   const double* __restrict__ val, double thr, int* __restrict__ counts,
                   const long long* __restrict__ g_rp, int* __restrict__ g_col,
                   int* __restrict__ overflow) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* keys = reinterpret_cast<int*>(sm_raw) + warp * kGraphSlots;
  double* vals =
      reinterpret_cast<double*>(sm_raw + kGraphWarps * kGraphSlots * sizeof(int)) + warp * kGraphSlots;
  int* list = reinterpret_cast<int*>(sm_raw + kGraphWarps * kGraphSlots * (sizeof(int) + sizeof(double))) +
              warp * kGraphSlots;
  const int i = blockIdx.x * kGraphWarps + warp;
  if (i >= n) return;
  for (int s = lane; s < kGraphSlots; s += 32) {
    keys[s] = -1;
    vals[s] = 0.0;
  }
  __syncwarp();
  bool full = false;
  for (long long e = rp[i]; e < rp[i + 1] && !full; ++e) {
    const int k = col[e];
    const double a = val[e];
    for (long long f = rp[k] + lane; f < rp[k + 1]; f += 32) {
      const int j = col[f];
      const double v = __dmul_rn(a, val[f]);
      unsigned s = ((unsigned)j * 2654435761u) & (kGraphSlots - 1);
      int tries = 0;
      for (;;) {
        const int old = atomicCAS(&keys[s], -1, j);
        if (old == -1 || old == j) break;
        s = (s + 1) & (kGraphSlots - 1);
        if (++tries >= kGraphSlots) {
          full = true;
          break;
        }
      }
      if (tries < kGraphSlots) vals[s] = __dadd_rn(vals[s], v);
    }
    full = __any_sync(0xffffffffu, full);
    __syncwarp();
  }
  if (full) {
    if (lane == 0) atomicExch(overflow, 1);
    if (!FILL) counts[i] = 0;
    return;
  }
  // columns kept: |G_ij| > thr, compacted into list (warp-aggregated)
  int m = 0;
  for (int s0 = 0; s0 < kGraphSlots; s0 += 32) {
    const int s = s0 + lane;
    const bool keep = keys[s] >= 0 && fabs(vals[s]) > thr;
    const unsigned b = __ballot_sync(0xffffffffu, keep);
    if (FILL && keep) list[m + __popc(b & ((1u << lane) - 1))] = keys[s];
    m += __popc(b);
  }
  if (!FILL) {
    if (lane == 0) counts[i] = m;
    return;
  }
  __syncwarp();
  // ascending order: bitonic sort of the list padded to a power of two
  int p2 = 1;
  while (p2 < m) p2 <<= 1;
  for (int s = m + lane; s < p2; s += 32) list[s] = 0x7fffffff;
  __syncwarp();
  for (int size = 2; size <= p2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = lane; t < p2 / 2; t += 32) {
        const int lo = 2 * stride * (t / stride) + (t % stride);
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const int x = list[lo], y = list[hi];
        if ((x > y) == up) {
          list[lo] = y;
          list[hi] = x;
        }
      }
      __syncwarp();
    }
  }
  int* out = g_col + g_rp[i];
  for (int t = lane; t < m; t += 32) out[t] = list[t];
}

static size_t graph_smem() {
  return (size_t)kGraphWarps * kGraphSlots * (2 * sizeof(int) + sizeof(double));
}

// ELLPACK rows to CSR: row i's entries sit at [i*m, i*m + nnz[i]) of idx / val (0-based
// columns; the row-major ELLPACK layout of BML's C storage) and go to [rp[i], rp[i+1]).
// One warp per row.  A column outside [0, n) is flagged in *bad and written as 0.
__global__ void __launch_bounds__(256)
    k_ell_to_csr(int n, int m, const int* __restrict__ nnz, const int* __restrict__ idx,
                 const double* __restrict__ val, const long long* __restrict__ rp,
                 int* __restrict__ col, double* __restrict__ cval, int* __restrict__ bad) {
  const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  const int k = nnz[i];   // 0 <= k <= m, checked by the host
  const long long src = (long long)i * m, dst = rp[i];
  for (int t = lane; t < k; t += 32) {
    const int j = idx[src + t];
    const bool ok = j >= 0 && j < n;
    if (!ok) atomicExch(bad, 1);
    col[dst + t] = ok ? j : 0;
    cval[dst + t] = val[src + t];
  }
}

}  // namespace sp2b

using namespace sp2b;

extern "C" int sp2b_graph_square_threshold(int n, const long long* h_row_ptr, const int* h_col,
                                           const double* h_val, double gthreshold,
                                           long long* g_row_ptr, int* g_col, long long g_cap,
                                           long long* g_needed, const sp2b_opts* opts) {
  if (n <= 0 || !h_row_ptr || !h_col || !h_val || !g_row_ptr || !(gthreshold >= 0.0)) {
    set_last_error("sp2b_graph_square_threshold: bad argument");
    return SP2B_BAD_ARG;
  }
  sp2b_opts dflt;
  sp2b_opts_default(&dflt);
  if (!opts) opts = &dflt;
  const bool dev = opts->device_ptrs != 0;
  int status = SP2B_OK;
  Ctx* c = get_ctx(&status);
  if (!c) return status;
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStream_t st = opts->stream ? (cudaStream_t)opts->stream : (dev ? (cudaStream_t)0 : c->stream);

  long long nnz = 0;
  if (dev) SP2B_CUDA_TRY(cudaMemcpy(&nnz, h_row_ptr + n, sizeof(long long), cudaMemcpyDeviceToHost));
  else nnz = h_row_ptr[n];
  // device copies of H (host-pointer calls) and the working arrays
  long long* rp_d = nullptr;
  int* col_d = nullptr;
  double* val_d = nullptr;
  int* counts = nullptr;
  int* ovf = nullptr;
  long long* grp_d = nullptr;
  int* gcol_d = nullptr;
  auto cleanup = [&]() {
    if (!dev) {
      cudaFree(rp_d);
      cudaFree(col_d);
      cudaFree(val_d);
      cudaFree(gcol_d);
    }
    cudaFree(counts);
    cudaFree(ovf);
    cudaFree(grp_d);
  };
  cudaError_t e = cudaSuccess;
  if (dev) {
    rp_d = const_cast<long long*>(h_row_ptr);
    col_d = const_cast<int*>(h_col);
    val_d = const_cast<double*>(h_val);
  } else {
    if ((e = cudaMalloc(&rp_d, (n + 1) * sizeof(long long))) == cudaSuccess &&
        (e = cudaMalloc(&col_d, std::max<long long>(nnz, 1) * sizeof(int))) == cudaSuccess &&
        (e = cudaMalloc(&val_d, std::max<long long>(nnz, 1) * sizeof(double))) == cudaSuccess &&
        (e = cudaMemcpyAsync(rp_d, h_row_ptr, (n + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                             st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(col_d, h_col, nnz * sizeof(int), cudaMemcpyHostToDevice, st)) ==
            cudaSuccess)
      e = cudaMemcpyAsync(val_d, h_val, nnz * sizeof(double), cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess && (e = cudaMalloc(&counts, n * sizeof(int))) == cudaSuccess &&
      (e = cudaMalloc(&ovf, sizeof(int))) == cudaSuccess)
    e = cudaMemsetAsync(ovf, 0, sizeof(int), st);
  const size_t smem = graph_smem();
  const int grid = (n + kGraphWarps - 1) / kGraphWarps;
  if (e == cudaSuccess) {
    cudaFuncSetAttribute(k_square_graph<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_square_graph<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_square_graph<false><<<grid, kGraphWarps * 32, smem, st>>>(n, rp_d, col_d, val_d, gthreshold,
                                                                counts, nullptr, nullptr, ovf);
    note_launch();
    e = cudaGetLastError();
  }
  std::vector<int> cnt(n);
  int hovf = 0;
  if (e == cudaSuccess && (e = cudaMemcpyAsync(cnt.data(), counts, n * sizeof(int),
                                               cudaMemcpyDeviceToHost, st)) == cudaSuccess &&
      (e = cudaMemcpyAsync(&hovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, st)) == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cleanup();
    set_last_error("sp2b_graph_square_threshold: %s", cudaGetErrorString(e));
    return SP2B_CUDA_ERROR;
  }
  if (hovf) {
    cleanup();
    set_last_error("sp2b_graph_square_threshold: a row of H^2 has more than %d candidate columns",
                   kGraphSlots);
    return SP2B_BAD_INPUT;
  }
  std::vector<long long> grp(n + 1, 0);
  for (int i = 0; i < n; ++i) grp[i + 1] = grp[i] + cnt[i];
  const long long total = grp[n];
  if (g_needed) *g_needed = total;
  if (dev) e = cudaMemcpyAsync(g_row_ptr, grp.data(), (n + 1) * sizeof(long long),
                               cudaMemcpyHostToDevice, st);
  else std::memcpy(g_row_ptr, grp.data(), (n + 1) * sizeof(long long));
  if (e == cudaSuccess && (!g_col || g_cap < total)) {
    cleanup();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    set_last_error("sp2b_graph_square_threshold: g_col needs %lld entries", total);
    return SP2B_BAD_ARG;
  }
  if (e == cudaSuccess && (e = cudaMalloc(&grp_d, (n + 1) * sizeof(long long))) == cudaSuccess)
    e = cudaMemcpyAsync(grp_d, grp.data(), (n + 1) * sizeof(long long), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    if (dev) gcol_d = g_col;
    else e = cudaMalloc(&gcol_d, std::max<long long>(total, 1) * sizeof(int));
  }
  if (e == cudaSuccess) {
    k_square_graph<true><<<grid, kGraphWarps * 32, smem, st>>>(n, rp_d, col_d, val_d, gthreshold,
                                                               nullptr, grp_d, gcol_d, ovf);
    note_launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && !dev)
    e = cudaMemcpyAsync(g_col, gcol_d, total * sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) {
    set_last_error("sp2b_graph_square_threshold: %s", cudaGetErrorString(e));
    return SP2B_CUDA_ERROR;
  }
  return SP2B_OK;
}

extern "C" int sp2b_ellpack_to_csr(int n, int m, const int* nnz, const int* idx, const double* val,
                                   long long* row_ptr, int* col, double* csr_val, long long cap,
                                   long long* needed, const sp2b_opts* opts) {
  if (n <= 0 || m < 0 || !nnz || (m > 0 && (!idx || !val)) || !row_ptr) {
    set_last_error("sp2b_ellpack_to_csr: bad argument");
    return SP2B_BAD_ARG;
  }
  sp2b_opts dflt;
  sp2b_opts_default(&dflt);
  if (!opts) opts = &dflt;
  const bool dev = opts->device_ptrs != 0;
  // row counts (device calls: fetched), checked and summed on the host
  std::vector<int> cnt(n);
  int status = SP2B_OK;
  Ctx* c = nullptr;
  cudaStream_t st = nullptr;
  std::unique_lock<std::mutex> lk;
  if (dev) {
    c = get_ctx(&status);
    if (!c) return status;
    lk = std::unique_lock<std::mutex>(c->mu);
    st = opts->stream ? (cudaStream_t)opts->stream : (cudaStream_t)0;
    SP2B_CUDA_TRY(cudaMemcpyAsync(cnt.data(), nnz, n * sizeof(int), cudaMemcpyDeviceToHost, st));
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  } else {
    std::memcpy(cnt.data(), nnz, n * sizeof(int));
  }
  std::vector<long long> rp(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    if (cnt[i] < 0 || cnt[i] > m) {
      set_last_error("sp2b_ellpack_to_csr: row %d has %d entries (width %d)", i, cnt[i], m);
      return SP2B_BAD_INPUT;
    }
    rp[i + 1] = rp[i] + cnt[i];
  }
  const long long total = rp[n];
  if (needed) *needed = total;
  if (dev) SP2B_CUDA_TRY(cudaMemcpyAsync(row_ptr, rp.data(), (n + 1) * sizeof(long long),
                                         cudaMemcpyHostToDevice, st));
  else std::memcpy(row_ptr, rp.data(), (n + 1) * sizeof(long long));
  if (total > 0 && (!col || !csr_val || cap < total)) {
    if (dev) SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    set_last_error("sp2b_ellpack_to_csr: col / val need %lld entries", total);
    return SP2B_BAD_ARG;
  }
  if (!dev) {
    // host arrays: a host copy (this is input formatting, not SP2 arithmetic)
    for (int i = 0; i < n; ++i)
      for (int t = 0; t < cnt[i]; ++t) {
        const long long s = (long long)i * m + t;
        if (idx[s] < 0 || idx[s] >= n) {
          set_last_error("sp2b_ellpack_to_csr: row %d column %d out of range", i, idx[s]);
          return SP2B_BAD_INPUT;
        }
        col[rp[i] + t] = idx[s];
        csr_val[rp[i] + t] = val[s];
      }
    return SP2B_OK;
  }
  if (total == 0) {
    SP2B_CUDA_TRY(cudaStreamSynchronize(st));
    return SP2B_OK;
  }
  int* bad = c->err;   // the context's device status word, cleared again below
  SP2B_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
  const long long threads = (long long)n * 32;
  const int block = 256;
  k_ell_to_csr<<<(unsigned)((threads + block - 1) / block), block, 0, st>>>(n, m, nnz, idx, val,
                                                                             row_ptr, col, csr_val,
                                                                             bad);
  note_launch();
  SP2B_CUDA_TRY(cudaGetLastError());
  int hbad = 0;
  SP2B_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  SP2B_CUDA_TRY(cudaStreamSynchronize(st));
  SP2B_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), st));
  if (hbad) {
    set_last_error("sp2b_ellpack_to_csr: a column index is outside [0, %d)", n);
    return SP2B_BAD_INPUT;
  }
  return SP2B_OK;
}
