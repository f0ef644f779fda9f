// FP64 kernels: Gershgorin bounds, normalisation, and the symmetric-tile DMMA product
// with the fused SP2 epilogue.  This is the parity form of the SP2 step (1e-10).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "reduce.cuh"
#include "sp2b_tune.h"

namespace sp2b {

// ------------------------------------------------------------------------------------
// Gershgorin bounds (bml_gershgorin as used by prg_normalize, src/prg_normalize_mod.F90:41)
// H is column-major: H(i, j) = h[i + j*ld]; thread i walks row i, so a warp reads 32
// consecutive doubles of one column per step (coalesced).
// ------------------------------------------------------------------------------------
__global__ void k_gersh_partial(const double* __restrict__ h, int n, int ld, int ncol,
                                double* __restrict__ rowsum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j0 = blockIdx.y * ncol;
  const int j1 = min(n, j0 + ncol);
  double s = 0.0;
  for (int j = j0; j < j1; ++j)
    if (j != i) s += fabs(h[i + (size_t)j * ld]);
  rowsum[(size_t)blockIdx.y * n + i] = s;
}

// Row totals, per-block min/max of (h_ii - r_i, h_ii + r_i), and in the last block to
// arrive the min/max over the blocks in block order; a NaN or overflow anywhere makes
// both bounds NaN.
__device__ __forceinline__ double nan_min(double a, double b) {
  return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : fmin(a, b);
}
__device__ __forceinline__ double nan_max(double a, double b) {
  return (a != a || b != b) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(a, b);
}
__global__ void __launch_bounds__(256)
    k_gersh_final(const double* __restrict__ h, int n, int ld, int nsplit,
                  const double* __restrict__ rowsum, double* partials, unsigned* counter,
                  double* __restrict__ bounds) {
  __shared__ double smin[256], smax[256];
  __shared__ int s_last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double mn = 1e308, mx = -1e308;
  if (i < n) {
    double r = 0.0;
    for (int s = 0; s < nsplit; ++s) r += rowsum[(size_t)s * n + i];
    const double d = h[i + (size_t)i * ld];
    if (!(r == r) || !(d == d) || fabs(r) > 1e300 || fabs(d) > 1e300) {
      mn = mx = __longlong_as_double(0x7ff8000000000000ll);
    } else {
      mn = d - r;
      mx = d + r;
    }
  }
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      smin[threadIdx.x] = nan_min(smin[threadIdx.x], smin[threadIdx.x + o]);
      smax[threadIdx.x] = nan_max(smax[threadIdx.x], smax[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = smin[0];
    partials[2 * blockIdx.x + 1] = smax[0];
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  mn = 1e308;
  mx = -1e308;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    mn = nan_min(mn, __ldcg(partials + 2 * b));
    mx = nan_max(mx, __ldcg(partials + 2 * b + 1));
  }
  smin[threadIdx.x] = mn;
  smax[threadIdx.x] = mx;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      smin[threadIdx.x] = nan_min(smin[threadIdx.x], smin[threadIdx.x + o]);
      smax[threadIdx.x] = nan_max(smax[threadIdx.x], smax[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bounds[0] = smin[0];
    bounds[1] = smax[0];
    *counter = 0u;
  }
}

// Delta_0 = alpha H1 (alpha = -1/(e_max - e_min)) into the zero-padded np x np buffer
// (src/prg_response_mod.F90:700: bml_scale(alpha, rsp_bml)).
__global__ void k_resp_init(const double* __restrict__ h1, int n, int ld, int np,
                            const double* __restrict__ bounds, double* __restrict__ d) {
  const double alpha = -1.0 / (bounds[1] - bounds[0]);
  const uint32_t gpr = (uint32_t)np / 8, ngroups = gpr * (uint32_t)np;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
    const int r = (int)(g / gpr), c0 = (int)(g - (uint32_t)r * gpr) * 8;
    double v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int c = c0 + e;
      // h1 == nullptr: the identity (dX0/dmu of the SP2-Fermi normalisation)
      v[e] = (r < n && c < n) ? alpha * (h1 ? h1[(size_t)r * ld + c] : (r == c ? 1.0 : 0.0)) : 0.0;
    }
    double2* dst = reinterpret_cast<double2*>(d + (size_t)r * np + c0);
#pragma unroll
    for (int e = 0; e < 4; ++e) dst[e] = make_double2(v[2 * e], v[2 * e + 1]);
  }
}

cudaError_t launch_resp_init(const double* h1, int n, int ld, int np, const double* bounds,
                             double* d, cudaStream_t st) {
  const size_t groups = (size_t)np * np / 8;
  const int g = (int)std::min<size_t>((groups + 255) / 256, 148 * 8);
  k_resp_init<<<g, 256, 0, st>>>(h1, n, ld, np, bounds, d);
  note_launch();
  return cudaGetLastError();
}

// Lower triangle of a symmetric n x n matrix (row pitch ld) from its upper triangle, by
// 32 x 32 blocks through shared memory (the host-pointer entries copy only the upper
// triangle across PCIe).  One CTA per block pair (ib <= jb).
__global__ void __launch_bounds__(256) k_mirror_lower(double* __restrict__ a, int n, int ld) {
  __shared__ double t[32][33];
  int ib, jb;
  upper_tile(blockIdx.x, ib, jb);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = ib * 32 + ty + 8 * k, c = jb * 32 + tx;
    t[ty + 8 * k][tx] = (r < n && c < n) ? a[(size_t)r * ld + c] : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = jb * 32 + ty + 8 * k, c = ib * 32 + tx;   // (r, c) = mirror of (c, r)
    if (r < n && c < n && r > c) a[(size_t)r * ld + c] = t[tx][ty + 8 * k];
  }
}

cudaError_t launch_mirror_lower(double* a, int n, int ld, cudaStream_t st) {
  const long long nb = (n + 31) / 32;
  k_mirror_lower<<<(unsigned)(nb * (nb + 1) / 2), 256, 0, st>>>(a, n, ld);
  note_launch();
  return cudaGetLastError();
}

int gersh_nsplit(int n) {
  const int rows_blocks = (n + 255) / 256;
  int ns = (4 * 148 + rows_blocks - 1) / rows_blocks;
  if (ns > n) ns = n;
  if (ns < 1) ns = 1;
  return ns;
}

cudaError_t launch_gersh(const double* h, int n, int ld, double* rowsum, int nsplit,
                         double* bounds, double* partials, unsigned* counter, cudaStream_t st) {
  const int ncol = (n + nsplit - 1) / nsplit;
  dim3 grid((n + 255) / 256, nsplit);
  k_gersh_partial<<<grid, 256, 0, st>>>(h, n, ld, ncol, rowsum);
  note_launch();
  k_gersh_final<<<(n + 255) / 256, 256, 0, st>>>(h, n, ld, nsplit, rowsum, partials, counter,
                                                  bounds);
  note_launch();
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Normalisation X0 = alpha H + beta I, alpha = -1/(emax-emin), beta = emax/(emax-emin)
// (src/prg_normalize_mod.F90:27, in the alpha/beta form of src/prg_response_mod.F90:700)
// into the zero-padded np x np buffer, with Tr X0 and ||X0||_F^2 for the first SP2 step.
// ------------------------------------------------------------------------------------
__global__ void k_normalize_f64(const double* __restrict__ h, int n, int ld, int np,
                                const double* __restrict__ bounds, double* __restrict__ x,
                                double* partials, unsigned* counter, SP2Rec* rec0,
                                double* norm_out) {
  __shared__ double red[32 * 4];
  __shared__ int s_last;
  const double emin = bounds[0], emax = bounds[1];
  const double mm = emax - emin;
  const double alpha = -1.0 / mm, beta = emax / mm;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  // groups of 8 consecutive elements of one row (np is a multiple of 128)
  const uint32_t gpr = (uint32_t)np / 8, ngroups = gpr * (uint32_t)np;
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngroups; g += gridDim.x * blockDim.x) {
    const int r = (int)(g / gpr), c0 = (int)(g - (uint32_t)r * gpr) * 8;
    double v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int c = c0 + e;
      v[e] = (r < n && c < n) ? alpha * h[(size_t)r * ld + c] + (r == c ? beta : 0.0) : 0.0;
      s[0] += v[e] * v[e];
      if (r == c) s[1] += v[e];
    }
    double2* dst = reinterpret_cast<double2*>(x + (size_t)r * np + c0);
#pragma unroll
    for (int e = 0; e < 4; ++e) dst[e] = make_double2(v[2 * e], v[2 * e + 1]);
  }
  block_sum<4>(s, red);
  if (threadIdx.x == 0) {
    partials[4 * blockIdx.x] = s[0];
    partials[4 * blockIdx.x + 1] = s[1];
    __threadfence();
    s_last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double t[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) {
    t[0] += __ldcg(partials + 4 * j);
    t[1] += __ldcg(partials + 4 * j + 1);
  }
  block_sum<4>(t, red);
  if (threadIdx.x == 0) {
    *counter = 0u;
    SP2Rec r0;
    memset(&r0, 0, sizeof(r0));
    r0.trx = t[1];
    r0.trx_data = t[1];
    r0.fro2 = t[0];
    r0.last_branch = -1;
    if (!(t[0] == t[0]) || !(mm > 0.0)) {
      r0.status = SP2B_BAD_INPUT;
      r0.done = 1;
    }
    *rec0 = r0;
    norm_out[0] = emin;
    norm_out[1] = emax;
    norm_out[2] = t[1];
    norm_out[3] = t[0];
  }
}

static int norm_grid(int np) {
  const size_t total = (size_t)np * np;
  size_t g = (total + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  return (int)g;
}

cudaError_t launch_normalize_f64(const double* h, int n, int ld, int np, const double* bounds,
                                 double* x, double* partials, unsigned* counter, SP2Rec* rec0,
                                 double* norm_out, cudaStream_t st) {
  k_normalize_f64<<<norm_grid(np), 256, 0, st>>>(h, n, ld, np, bounds, x, partials, counter,
                                                 rec0, norm_out);
  note_launch();
  return cudaGetLastError();
}

__global__ void k_copy_in(const double* __restrict__ src, int n, int ld, int np,
                          double* __restrict__ x) {
  const size_t total = (size_t)np * np;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / np), c = (int)(idx % np);
    x[idx] = (r < n && c < n) ? src[(size_t)r * ld + c] : 0.0;
  }
}

cudaError_t launch_copy_in(const double* src, int n, int ld, int np, double* x,
                           cudaStream_t st) {
  k_copy_in<<<norm_grid(np), 256, 0, st>>>(src, n, ld, np, x);
  note_launch();
  return cudaGetLastError();
}

__global__ void k_finish_f64(const double* __restrict__ x, int np, int n, double scale,
                             double* __restrict__ rho, int ld) {
  const size_t total = (size_t)n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / n), c = (int)(idx % n);
    rho[(size_t)r * ld + c] = scale * x[(size_t)r * np + c];
  }
}

cudaError_t launch_finish_f64(const double* x, int np, int n, double scale, double* rho,
                              int ld, cudaStream_t st) {
  k_finish_f64<<<norm_grid(np), 256, 0, st>>>(x, np, n, scale, rho, ld);
  note_launch();
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Symmetric-tile FP64 product with the SP2 epilogue.
// One CTA per upper tile (bi <= bj) of BT x BT; WM x WN warps, each owning a
// (BT/WM) x (BT/WN) block of m8n8k4 DMMA fragments.  Operand tiles are rows of the
// symmetric inputs: As[k][m] = A[k0+k][i0+m], Bs[k][n] = B[k0+k][j0+n], staged by a
// 3-deep cp.async pipeline with rows padded to BT+4 doubles (conflict-free fragment loads).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <int BT, int WM, int WN>
struct F64Cfg {
  static constexpr int BK = 16;
  static constexpr int NW = WM * WN;
  static constexpr int NT = NW * 32;
  static constexpr int LDS = BT + 4;
  static constexpr int ST = 3;
  static constexpr int TM = BT / WM, TN = BT / WN;
  static constexpr int MI = TM / 8, NI = TN / 8;
  static constexpr size_t SMEM = (size_t)ST * 2 * BK * LDS * sizeof(double);
};

template <int BT, int WM, int WN>
__global__ void __launch_bounds__(WM* WN * 32, 1) k_sym_gemm_f64(const StepArgs p) {
  using C = F64Cfg<BT, WM, WN>;
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[32 * 4];
  __shared__ int s_flag;

  double alpha = p.alpha, beta = p.beta;
  if (p.control) {
    const int br = control_prologue(p);
    if (br < 0) return;
    if (br == BR_X2) { alpha = 1.0; beta = 0.0; }
    else { alpha = -1.0; beta = 2.0; }
    // response products after step k: P1 = a X Delta + b Delta (control 2, the step's
    // own a, b), then Delta' = a Delta X + P1 (control 3)
    if (p.control == 3) beta = 1.0;
  }
  int bi, bj, nloc = p.np, core = p.core;
  size_t row0 = 0;
  if (p.tiles) {
    const int4 t = p.tiles[blockIdx.x];
    row0 = (size_t)t.x;
    bi = t.y >> 16;
    bj = t.y & 0xffff;
    nloc = t.z;
    core = t.w;
  } else {
    upper_tile(blockIdx.x, bi, bj);
  }
  const int i0 = bi * BT, j0 = bj * BT;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = warp / WN, wn = warp % WN;
  const int ld = p.ld;
  // the part's square block starts at row row0 of the packed buffers
  const double* __restrict__ A = (const double*)p.A + row0 * ld;
  const double* __restrict__ B = (const double*)p.B + row0 * ld;

  double acc[C::MI][C::NI][2];
#pragma unroll
  for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
    for (int ni = 0; ni < C::NI; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;

  // every valid tile starts inside its part; anything else contributes nothing
  const bool tile_ok = !p.tiles || (i0 < nloc && j0 < nloc);
  const int KB = tile_ok ? nloc / C::BK : 0;
  auto load = [&](int stage, int kb) {
    double* As = sm + stage * 2 * C::BK * C::LDS;
    double* Bs = As + C::BK * C::LDS;
    const int k0 = kb * C::BK;
    for (int c = tid; c < C::BK * BT / 2; c += C::NT) {
      const int row = c / (BT / 2), col = (c % (BT / 2)) * 2;
      cp_async16(As + row * C::LDS + col, A + (size_t)(k0 + row) * ld + i0 + col);
      cp_async16(Bs + row * C::LDS + col, B + (size_t)(k0 + row) * ld + j0 + col);
    }
  };
#pragma unroll
  for (int s = 0; s < C::ST - 1; ++s) {
    if (s < KB) load(s, s);
    cp_async_commit();
  }
  for (int kb = 0; kb < KB; ++kb) {
    cp_async_wait<C::ST - 2>();
    __syncthreads();
    {
      const int nk = kb + C::ST - 1;
      if (nk < KB) load(nk % C::ST, nk);
      cp_async_commit();
    }
    const double* As = sm + (kb % C::ST) * 2 * C::BK * C::LDS;
    const double* Bs = As + C::BK * C::LDS;
#pragma unroll
    for (int kk = 0; kk < C::BK; kk += 4) {
      double a[C::MI], b[C::NI];
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi) a[mi] = As[(kk + t4) * C::LDS + wm * C::TM + mi * 8 + g];
#pragma unroll
      for (int ni = 0; ni < C::NI; ++ni) b[ni] = Bs[(kk + t4) * C::LDS + wn * C::TN + ni * 8 + g];
#pragma unroll
      for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
        for (int ni = 0; ni < C::NI; ++ni) dmma884(acc[mi][ni], a[mi], b[ni]);
    }
  }
  cp_async_wait<0>();

  // ---- epilogue: out = alpha*acc + beta*E, mirrored store, FP64 sums ----
  const bool diag = (bi == bj);
  const double* __restrict__ E = (const double*)p.E + row0 * ld;
  double* __restrict__ out = p.out ? (double*)p.out + row0 * ld : nullptr;
  double s[4] = {0.0, 0.0, 0.0, 0.0};  // ||out||^2, Tr out, ||E-acc||^2 (core rows), Tr acc
#pragma unroll
  for (int mi = 0; mi < (tile_ok ? C::MI : 0); ++mi) {
#pragma unroll
    for (int ni = 0; ni < C::NI; ++ni) {
      const int r = i0 + wm * C::TM + mi * 8 + g;
      const int c = j0 + wn * C::TN + ni * 8 + 2 * t4;
      const double2 e = *reinterpret_cast<const double2*>(E + (size_t)r * ld + c);
      const double a0 = acc[mi][ni][0], a1 = acc[mi][ni][1];
      const double v0 = alpha * a0 + beta * e.x;
      const double v1 = alpha * a1 + beta * e.y;
      const int w0 = sym_weight(diag, r, c), w1 = sym_weight(diag, r, c + 1);
      const double d0 = e.x - a0, d1 = e.y - a1;
      s[0] += w0 * v0 * v0 + w1 * v1 * v1;
      s[2] += core_weight(w0, r, c, core) * d0 * d0 + core_weight(w1, r, c + 1, core) * d1 * d1;
      if (r == c) { s[1] += v0; s[3] += a0; }
      if (r == c + 1) { s[1] += v1; s[3] += a1; }
      if (out) {
        if (!diag) {
          *reinterpret_cast<double2*>(out + (size_t)r * ld + c) = make_double2(v0, v1);
          out[(size_t)c * ld + r] = v0;
          out[(size_t)(c + 1) * ld + r] = v1;
        } else {
          if (w0) { out[(size_t)r * ld + c] = v0; out[(size_t)c * ld + r] = v0; }
          if (w1) { out[(size_t)r * ld + c + 1] = v1; out[(size_t)(c + 1) * ld + r] = v1; }
        }
      }
    }
  }
  publish_and_finalize(p, s, red, &s_flag);
}

// Tiles of the one-launch form: 32 x 32, 8 warps of 16 x 8, k blocks of 64 in a 3-deep
// pipeline (the k order of every sum is that of F64Cfg<32, 2, 4>: 4 at a time, ascending);
// 110 KB of stages, two CTAs per SM.
struct MsCfg {
  static constexpr int BK = 64, NT = 256, LDS = 36, ST = 3;
  static constexpr int TM = 16, TN = 8, MI = 2, NI = 1;
  static constexpr size_t SMEM = (size_t)ST * 2 * BK * LDS * sizeof(double);
};

// All SP2 steps of a batch of parts in one cooperative launch (see MultiStepArgs).
// Tile math and the order of every sum are those of k_sym_gemm_f64<32, 2, 4>, so each
// part's result equals that of the per-step launches bit for bit; the per-step sums
// (traces, vv) are not formed.  Between steps every CTA of a part adds one to the part's
// counter and waits, with a bounded spin, until the part's tiles have all finished the
// step; operands are read through L2 (cp.async.cg, ld.global.cg), never a stale L1 line.
__global__ void __launch_bounds__(256, 1) k_f64_multistep(const MultiStepArgs a) {
  using C = MsCfg;
  extern __shared__ __align__(16) double sm[];
  const int4 t = a.tiles[blockIdx.x];
  const size_t row0 = (size_t)t.x;
  const int bi = t.y >> 16, bj = t.y & 0xffff, nloc = t.z, part = t.w;
  const unsigned per = (unsigned)a.part_tiles[part];
  const int i0 = bi * 32, j0 = bj * 32;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = warp / 4, wn = warp % 4;   // WM = 2, WN = 4
  const int ld = a.ld;
  const bool tile_ok = i0 < nloc && j0 < nloc;
  const int KB = tile_ok ? nloc / C::BK : 0;
  const bool diag = bi == bj;
  __shared__ int s_bad;
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int k = 0; k < a.maxiter; ++k) {
    const double* __restrict__ X = a.x[k & 1] + row0 * ld;
    double* __restrict__ out = a.x[(k + 1) & 1] + row0 * ld;
    const bool sq = a.pp[k] != 0;
    const double alpha = sq ? 1.0 : -1.0, beta = sq ? 0.0 : 2.0;
    double acc[C::MI][C::NI][2];
#pragma unroll
    for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
      for (int ni = 0; ni < C::NI; ++ni) acc[mi][ni][0] = acc[mi][ni][1] = 0.0;
    auto load = [&](int stage, int kb) {
      double* As = sm + stage * 2 * C::BK * C::LDS;
      double* Bs = As + C::BK * C::LDS;
      const int k0 = kb * C::BK;
      for (int c = tid; c < C::BK * 32 / 2; c += C::NT) {
        const int row = c / 16, col = (c % 16) * 2;   // BT / 2 = 16 pieces per row
        cp_async16(As + row * C::LDS + col, X + (size_t)(k0 + row) * ld + i0 + col);
        cp_async16(Bs + row * C::LDS + col, X + (size_t)(k0 + row) * ld + j0 + col);
      }
    };
#pragma unroll
    for (int s = 0; s < C::ST - 1; ++s) {
      if (s < KB) load(s, s);
      cp_async_commit();
    }
    for (int kb = 0; kb < KB; ++kb) {
      cp_async_wait<C::ST - 2>();
      __syncthreads();
      {
        const int nk = kb + C::ST - 1;
        if (nk < KB) load(nk % C::ST, nk);
        cp_async_commit();
      }
      const double* As = sm + (kb % C::ST) * 2 * C::BK * C::LDS;
      const double* Bs = As + C::BK * C::LDS;
#pragma unroll
      for (int kk = 0; kk < C::BK; kk += 4) {
        double av[C::MI], bv[C::NI];
#pragma unroll
        for (int mi = 0; mi < C::MI; ++mi) av[mi] = As[(kk + t4) * C::LDS + wm * C::TM + mi * 8 + g];
#pragma unroll
        for (int ni = 0; ni < C::NI; ++ni) bv[ni] = Bs[(kk + t4) * C::LDS + wn * C::TN + ni * 8 + g];
#pragma unroll
        for (int mi = 0; mi < C::MI; ++mi)
#pragma unroll
          for (int ni = 0; ni < C::NI; ++ni) dmma884(acc[mi][ni], av[mi], bv[ni]);
      }
    }
    cp_async_wait<0>();
    __syncthreads();   // every warp is done with the stages before the next step reuses them
#pragma unroll
    for (int mi = 0; mi < (tile_ok ? C::MI : 0); ++mi) {
#pragma unroll
      for (int ni = 0; ni < C::NI; ++ni) {
        const int r = i0 + wm * C::TM + mi * 8 + g;
        const int c = j0 + wn * C::TN + ni * 8 + 2 * t4;
        const double ex = __ldcg(X + (size_t)r * ld + c), ey = __ldcg(X + (size_t)r * ld + c + 1);
        const double v0 = alpha * acc[mi][ni][0] + beta * ex;
        const double v1 = alpha * acc[mi][ni][1] + beta * ey;
        if (!diag) {
          *reinterpret_cast<double2*>(out + (size_t)r * ld + c) = make_double2(v0, v1);
          out[(size_t)c * ld + r] = v0;
          out[(size_t)(c + 1) * ld + r] = v1;
        } else {
          if (r <= c) { out[(size_t)r * ld + c] = v0; out[(size_t)c * ld + r] = v0; }
          if (r <= c + 1) { out[(size_t)r * ld + c + 1] = v1; out[(size_t)(c + 1) * ld + r] = v1; }
        }
      }
    }
    // per-part barrier before X_{k+1} is read
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      atomicAdd(a.bar + part, 1u);
      const unsigned target = per * (unsigned)(k + 1);
      bool ok = false;
      for (uint32_t it = 0; it < kSpinLimit; ++it) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(a.bar + part) : "memory");
        if (v >= target) { ok = true; break; }
        if (*(volatile int*)a.err) break;
        __nanosleep(64);
      }
      if (!ok) {
        atomicExch(a.err, 1);
        s_bad = 1;
      }
      __threadfence();
    }
    __syncthreads();
    if (s_bad) return;
  }
}

cudaError_t launch_f64_multistep(const MultiStepArgs& a, cudaStream_t st) {
  using C = MsCfg;
  static int max_blocks = -1;
  if (max_blocks < 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(k_f64_multistep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_f64_multistep, C::NT, C::SMEM);
    max_blocks = sms * per_sm;
  }
  if (a.ntiles <= 0) return cudaSuccess;
  if (a.ntiles > max_blocks) return cudaErrorCooperativeLaunchTooLarge;
  void* args[] = {(void*)&a};
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_f64_multistep, dim3(a.ntiles),
                                                    dim3(C::NT), args, C::SMEM, st);
  note_launch();
  return e;
}

// Tile edge of the dense FP64 step for np: the measured choice when one was made for this
// device and size (tune_f64_tile), else 128 once its tiles fill the SMs twice, else 64.
int f64_tile(int np) {
  int c = 0;
  if (tune_lookup(f64_tune_key(np), &c) && (c == 64 || c == 128)) return c;
  const int t128 = np / 128;
  return (t128 * (t128 + 1) / 2 >= 2 * 148) ? 128 : 64;
}

std::string f64_tune_key(int np) {
  return "f64-step/sm" + std::to_string(device_sms()) + "/np" + std::to_string(np);
}

int f64_ntiles(int np) {
  const int t = np / f64_tile(np);
  return t * (t + 1) / 2;
}

static cudaError_t launch_f64_bt(const StepArgs& a, int bt, int ntiles, cudaStream_t st) {
  if (bt == 128) {
    using C = F64Cfg<128, 2, 4>;
    auto kern = k_sym_gemm_f64<128, 2, 4>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    kern<<<ntiles, C::NT, C::SMEM, st>>>(a);
  } else if (bt == 64) {
    using C = F64Cfg<64, 2, 2>;
    auto kern = k_sym_gemm_f64<64, 2, 2>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    kern<<<ntiles, C::NT, C::SMEM, st>>>(a);
  } else {
    // 32-edge tiles for small batches: 8 warps of 16 x 8 so that a tile's k loop is
    // spread over all four schedulers (each element still sums k in the same order)
    using C = F64Cfg<32, 2, 4>;
    auto kern = k_sym_gemm_f64<32, 2, 4>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    kern<<<ntiles, C::NT, C::SMEM, st>>>(a);
  }
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_sym_gemm_f64(const StepArgs& a0, cudaStream_t st) {
  StepArgs a = a0;
  a.tiles = nullptr;
  if (a.ld == 0) a.ld = a.np;
  const int bt = f64_tile(a.np);
  const int t = a.np / bt;
  a.ntiles = t * (t + 1) / 2;   // the partial sums the last CTA reduces: one per launched tile
  return launch_f64_bt(a, bt, a.ntiles, st);
}

// Measures the dense step's tile edges 128 and 64 at np (one plain product each on
// x_in -> x_out, the same k order per element in both) and records the faster one for
// f64_tile.  partials must hold 4 doubles per 64-edge tile.
int tune_f64_tile(int np, const double* x_in, double* x_out, double* partials, unsigned* counter,
                  double* sums_out, cudaStream_t st) {
  int c = 0;
  const std::string key = f64_tune_key(np);
  if (!tune_enabled() || tune_lookup(key, &c)) return 0;
  const int edges[2] = {128, 64};
  StepArgs q;
  memset(&q, 0, sizeof(q));
  q.np = np;
  q.ld = np;
  q.A = q.B = q.E = x_in;
  q.out = x_out;
  q.alpha = 1.0;
  q.beta = 0.0;
  q.partials = partials;
  q.counter = counter;
  q.sums_out = sums_out;
  // timed on zeros (the buffer may not hold data yet; DMMA time does not depend on values)
  if (cudaMemsetAsync(const_cast<double*>(x_in), 0, (size_t)np * np * sizeof(double), st) !=
      cudaSuccess)
    return 3;   // SP2B_CUDA_ERROR
  std::vector<float> ms;
  int best = 0;
  const int rc = tune_measure(2, 2, st, [&](int cand) -> int {
    const int t = np / edges[cand];
    q.ntiles = t * (t + 1) / 2;
    if (cudaMemsetAsync(counter, 0, 4 * sizeof(unsigned), st) != cudaSuccess ||
        launch_f64_bt(q, edges[cand], q.ntiles, st) != cudaSuccess)
      return 3;   // SP2B_CUDA_ERROR
    return 0;
  }, &ms, &best);
  if (rc != 0) return rc;
  tune_store(key, edges[best], ms);
  return 0;
}

cudaError_t launch_sym_gemm_f64_batched(const StepArgs& a, int bt, cudaStream_t st) {
  if (!a.tiles || a.ntiles <= 0 || (bt != 32 && bt != 64 && bt != 128)) return cudaErrorInvalidValue;
  return launch_f64_bt(a, bt, a.ntiles, st);
}

}  // namespace sp2b
