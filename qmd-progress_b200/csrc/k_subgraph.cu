// Kernels of the graph-partitioned SP2 path (prg_subgraphSP2Loop,
// src/prg_subgraphloop_mod.F90:36-126): core+halo extraction from a CSR Hamiltonian
// into a packed buffer of per-part square blocks, per-part normalisation with the
// global bounds, and the core-row scatter of the result.
//
// Packed layout: part p owns rows [row0_p, row0_p + np_p) of an R x ld buffer, np_p =
// its core+halo size padded to 128, ld = the largest np_p; its block is columns
// [0, np_p).  Padding is zero and stays zero under X^2 and 2X - X^2.
#include <cuda_bf16.h>

#include "kernels_subgraph.cuh"

namespace sp2b {

// One CTA per part.  Row r of part p is node halo[r]; each CSR entry (u, val) of that
// node lands at column c where halo[c] = u (binary search in the part's sorted node
// list `skey` with local positions `sval`).  Entries whose column is outside the part
// are dropped, exactly as bml_matrix2submatrix keeps only the core+halo columns.
__global__ void k_extract_csr(const long long* __restrict__ rp, const int* __restrict__ col,
                              const double* __restrict__ val, const PartDesc* __restrict__ parts,
                              const int* __restrict__ halo, const int* __restrict__ skey,
                              const int* __restrict__ sval, int ld, double* __restrict__ xs) {
  const PartDesc P = parts[blockIdx.x];
  const int* hl = halo + P.hoff;
  const int* sk = skey + P.hoff;
  const int* sv = sval + P.hoff;
  double* blk = xs + (size_t)P.row0 * ld;
  for (int r = threadIdx.x; r < P.n; r += blockDim.x) {
    const int v = hl[r];
    for (long long e = rp[v]; e < rp[v + 1]; ++e) {
      const int u = col[e];
      int lo = 0, hi = P.n - 1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int key = sk[mid];
        if (key == u) {
          blk[(size_t)r * ld + sv[mid]] = val[e];
          break;
        }
        if (key < u) lo = mid + 1;
        else hi = mid - 1;
      }
    }
  }
}

template <typename T>
struct SplitOps;
template <>
struct SplitOps<__half> {
  static constexpr double kScale = 2048.0, kInv = 1.0 / 2048.0;
  __device__ static double to_d(__half h) { return (double)__half2float(h); }
  __device__ static __half from_d(double v) { return __double2half(v); }
};
template <>
struct SplitOps<__nv_bfloat16> {
  static constexpr double kScale = 256.0, kInv = 1.0 / 256.0;
  __device__ static double to_d(__nv_bfloat16 h) { return (double)__bfloat162float(h); }
  __device__ static __nv_bfloat16 from_d(double v) { return __double2bfloat16(v); }
};

// X0 = (emax I - Hsub)/(emax - emin) with the GLOBAL bounds (bml_normalize at
// src/prg_sp2_mod.F90:1276), in place on the FP64 packed buffer (prec = FP64) or
// split into hi/lo 16-bit buffers.
template <typename T>
__global__ void k_norm_parts(double* __restrict__ xs, const int* __restrict__ row_part,
                             const PartDesc* __restrict__ parts, long long rows, int ld,
                             double emin, double emax, int split, T* __restrict__ hi,
                             T* __restrict__ lo) {
  const double mm = emax - emin;
  const double alpha = -1.0 / mm, beta = emax / mm;
  const size_t total = (size_t)rows * ld;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const long long gr = (long long)(idx / ld);
    const int c = (int)(idx % ld);
    const PartDesc P = parts[row_part[gr]];
    const int r = (int)(gr - P.row0);
    double v = 0.0;
    if (r < P.n && c < P.n) {
      v = alpha * xs[idx];
      if (r == c) v += beta;
    }
    if (split) {
      const T a = SplitOps<T>::from_d(v);
      hi[idx] = a;
      lo[idx] = SplitOps<T>::from_d((v - SplitOps<T>::to_d(a)) * SplitOps<T>::kScale);
    } else {
      xs[idx] = v;
    }
  }
}

// Extraction and normalisation in one pass (parts up to 512): straight into the hi/lo
// split (split precisions, no FP64 packed block) or into the FP64 packed block, without
// clearing it first.  Grid (part, row group); each warp builds one row of X0 at a
// time in shared memory (zero, scatter the row's CSR entries found in the part's node
// list, add emax/(emax - emin) on the diagonal) and writes its hi/lo halves over the
// part's np columns (rows n..np-1 are zero padding; columns past np are never read).
// The values are those of k_extract_csr followed by k_norm_parts, bit for bit.
template <typename T, bool F64>
__global__ void __launch_bounds__(256) k_extract_split(
    const long long* __restrict__ rp, const int* __restrict__ col, const double* __restrict__ val,
    const PartDesc* __restrict__ parts, const int* __restrict__ halo, const int* __restrict__ skey,
    const int* __restrict__ sval, int ld, double emin, double emax, T* __restrict__ hi,
    T* __restrict__ lo, double* __restrict__ xs) {
  __shared__ double rowbuf[8][512];
  const PartDesc P = parts[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double mm = emax - emin;
  const double alpha = -1.0 / mm, beta = emax / mm;
  const int* hl = halo + P.hoff;
  const int* sk = skey + P.hoff;
  const int* sv = sval + P.hoff;
  double* buf = rowbuf[warp];
  for (int r = blockIdx.y * 8 + warp; r < P.np; r += gridDim.y * 8) {
    for (int c = lane; c < P.np; c += 32) buf[c] = 0.0;
    __syncwarp();
    if (r < P.n) {
      const int v = hl[r];
      for (long long e = rp[v] + lane; e < rp[v + 1]; e += 32) {
        const int u = col[e];
        int a = 0, b = P.n - 1;
        while (a <= b) {
          const int mid = (a + b) >> 1;
          const int key = sk[mid];
          if (key == u) {
            buf[sv[mid]] = val[e];
            break;
          }
          if (key < u) a = mid + 1;
          else b = mid - 1;
        }
      }
    }
    __syncwarp();
    const size_t ro = ((size_t)P.row0 + r) * ld;
    for (int c = lane; c < P.np; c += 32) {
      double x = 0.0;
      if (r < P.n && c < P.n) {
        x = alpha * buf[c];
        if (r == c) x += beta;
      }
      if (F64) {
        xs[ro + c] = x;
      } else {
        const T a = SplitOps<T>::from_d(x);
        hi[ro + c] = a;
        lo[ro + c] = SplitOps<T>::from_d((x - SplitOps<T>::to_d(a)) * SplitOps<T>::kScale);
      }
    }
    __syncwarp();
  }
}

cudaError_t launch_extract_split(const long long* rp, const int* col, const double* val,
                                 const PartDesc* parts, int nparts, const int* halo,
                                 const int* skey, const int* sval, int ld, double emin,
                                 double emax, int prec, void* hi, void* lo, double* xs,
                                 cudaStream_t st) {
  const dim3 grid(nparts, 16);
  if (prec == SP2B_PREC_FP64)
    k_extract_split<__half, true><<<grid, 256, 0, st>>>(rp, col, val, parts, halo, skey, sval, ld,
                                                        emin, emax, nullptr, nullptr, xs);
  else if (prec == SP2B_PREC_MIXED_BF16)
    k_extract_split<__nv_bfloat16, false><<<grid, 256, 0, st>>>(
        rp, col, val, parts, halo, skey, sval, ld, emin, emax, (__nv_bfloat16*)hi,
        (__nv_bfloat16*)lo, nullptr);
  else
    k_extract_split<__half, false><<<grid, 256, 0, st>>>(rp, col, val, parts, halo, skey, sval, ld,
                                                         emin, emax, (__half*)hi, (__half*)lo,
                                                         nullptr);
  note_launch();
  return cudaGetLastError();
}

// rho (core rows) = 2 X: packed per-part output and, optionally, a dense n x n
// column-major matrix (bml_submatrix2matrix, src/prg_subgraphloop_mod.F90:111-113).
template <typename T>
__global__ void k_scatter_parts(const double* __restrict__ x64, const T* __restrict__ hi,
                                const T* __restrict__ lo, int split,
                                const PartDesc* __restrict__ parts,
                                const int* __restrict__ halo, int ld, double* __restrict__ core_out,
                                double* __restrict__ dense, long long n) {
  const PartDesc P = parts[blockIdx.x];
  const int* hl = halo + P.hoff;
  const long long total = (long long)P.ncore * P.n;
  for (long long q = (long long)blockIdx.y * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.y * blockDim.x) {
    const int r = (int)(q / P.n), c = (int)(q % P.n);
    const size_t src = ((size_t)P.row0 + r) * ld + c;
    double v;
    if (split) v = SplitOps<T>::to_d(hi[src]) + SplitOps<T>::kInv * SplitOps<T>::to_d(lo[src]);
    else v = x64[src];
    v *= 2.0;
    if (core_out) core_out[P.coff + q] = v;
    if (dense) dense[(size_t)hl[r] + (size_t)hl[c] * n] = v;
  }
}

// Idempotency error of each part's core rows, sum over core rows i of (X - X^2)_ii =
// X_ii - sum_j X_ij^2 (X symmetric), from the final split iterate.  Grid (part, 16
// row groups); each warp reads whole rows in 16-byte pieces (padding columns are zero);
// out[part * 16 + group] holds the group's partial, summed in a fixed order by the host.
template <typename T>
__global__ void k_part_idem(const T* __restrict__ hi, const T* __restrict__ lo,
                            const PartDesc* __restrict__ parts, int ld, double* __restrict__ out) {
  __shared__ double red[32];
  const PartDesc P = parts[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  double s = 0.0;
  for (int r = blockIdx.y * nw + warp; r < P.ncore; r += gridDim.y * nw) {
    const size_t row = ((size_t)P.row0 + r) * ld;
    for (int c0 = lane * 8; c0 < P.np; c0 += 256) {
      const uint4 vh = *reinterpret_cast<const uint4*>(hi + row + c0);
      const uint4 vl = *reinterpret_cast<const uint4*>(lo + row + c0);
      const T* h8 = reinterpret_cast<const T*>(&vh);
      const T* l8 = reinterpret_cast<const T*>(&vl);
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const double x = SplitOps<T>::to_d(h8[e]) + SplitOps<T>::kInv * SplitOps<T>::to_d(l8[e]);
        s -= x * x;
        if (c0 + e == r) s += x;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w];
    out[(size_t)blockIdx.x * gridDim.y + blockIdx.y] = t;
  }
}

cudaError_t launch_part_idem(const void* hi, const void* lo, int prec, const PartDesc* parts,
                             int nparts, int ld, double* out, cudaStream_t st) {
  const dim3 grid(nparts, kPartIdemGroups);
  if (prec == SP2B_PREC_MIXED_BF16)
    k_part_idem<__nv_bfloat16><<<grid, 256, 0, st>>>((const __nv_bfloat16*)hi,
                                                      (const __nv_bfloat16*)lo, parts, ld, out);
  else
    k_part_idem<__half><<<grid, 256, 0, st>>>((const __half*)hi, (const __half*)lo, parts, ld,
                                              out);
  note_launch();
  return cudaGetLastError();
}

// Packed core-row blocks (as all-gathered from the ranks) into a dense column-major
// n x n density: part p's llsize x lsize block starts at src + off[p], row r = node
// halo[hptr[p] + r], column c = node halo[hptr[p] + c] (prg_collectMatrixFromParts,
// src/prg_subgraphloop_mod.F90:132-161).  One CTA row per part.
__global__ void k_place_core(const long long* __restrict__ hptr, const int* __restrict__ halo,
                             const int* __restrict__ lls, const long long* __restrict__ off,
                             const double* __restrict__ src, double* __restrict__ rho,
                             long long n) {
  const int p = blockIdx.x;
  const long long h0 = hptr[p];
  const int m = (int)(hptr[p + 1] - h0);
  const long long total = (long long)lls[p] * m;
  const int* hl = halo + h0;
  const double* s = src + off[p];
  for (long long q = (long long)blockIdx.y * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.y * blockDim.x) {
    const int r = (int)(q / m), c = (int)(q % m);
    rho[(size_t)hl[r] + (size_t)hl[c] * n] = s[q];
  }
}

cudaError_t launch_place_core(const long long* hptr, const int* halo, const int* lls,
                              const long long* off, int nparts, const double* src, double* rho,
                              long long n, cudaStream_t st) {
  if (nparts <= 0) return cudaSuccess;
  k_place_core<<<dim3(nparts, 8), 256, 0, st>>>(hptr, halo, lls, off, src, rho, n);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_extract_csr(const long long* rp, const int* col, const double* val,
                               const PartDesc* parts, int nparts, const int* halo,
                               const int* skey, const int* sval, int ld, double* xs,
                               cudaStream_t st) {
  k_extract_csr<<<nparts, 256, 0, st>>>(rp, col, val, parts, halo, skey, sval, ld, xs);
  note_launch();
  return cudaGetLastError();
}

static int grid_for(size_t total) {
  size_t g = (total + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  return (int)(g ? g : 1);
}

cudaError_t launch_norm_parts(double* xs, const int* row_part, const PartDesc* parts,
                              long long rows, int ld, double emin, double emax, int prec,
                              void* hi, void* lo, cudaStream_t st) {
  const int g = grid_for((size_t)rows * ld);
  if (prec == SP2B_PREC_MIXED_BF16)
    k_norm_parts<__nv_bfloat16><<<g, 256, 0, st>>>(xs, row_part, parts, rows, ld, emin, emax, 1,
                                                   (__nv_bfloat16*)hi, (__nv_bfloat16*)lo);
  else
    k_norm_parts<__half><<<g, 256, 0, st>>>(xs, row_part, parts, rows, ld, emin, emax,
                                            prec == SP2B_PREC_FP64 ? 0 : 1, (__half*)hi,
                                            (__half*)lo);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_scatter_parts(const double* x64, const void* hi, const void* lo, int prec,
                                 const PartDesc* parts, int nparts, const int* halo, int ld,
                                 double* core_out, double* dense, long long n, cudaStream_t st) {
  dim3 grid(nparts, 16);
  if (prec == SP2B_PREC_MIXED_BF16)
    k_scatter_parts<__nv_bfloat16><<<grid, 256, 0, st>>>(
        x64, (const __nv_bfloat16*)hi, (const __nv_bfloat16*)lo, 1, parts, halo, ld, core_out,
        dense, n);
  else
    k_scatter_parts<__half><<<grid, 256, 0, st>>>(x64, (const __half*)hi, (const __half*)lo,
                                                  prec == SP2B_PREC_FP64 ? 0 : 1, parts, halo, ld,
                                                  core_out, dense, n);
  note_launch();
  return cudaGetLastError();
}

}  // namespace sp2b
