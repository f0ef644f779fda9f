// Exact symmetric products on the INT8 tensor cores (tcgen05 kind::i8) for the FP64
// McWeeny refinement that ends a split-precision solve.
//
// The iterate X (symmetric, near-idempotent) is rounded to the integer matrix
// M = rint(2^S X) and held as its residues modulo nine pairwise-coprime moduli m_t <= 256
// (signed 8-bit planes R_t).  Each plane product P_t = R_t R_t is exact in the 32-bit
// accumulators (|r| <= 128, K <= 65536) and is reduced mod m_t in the epilogue.  The
// Chinese remainder theorem, in Garner's mixed-radix form evaluated by Horner's rule in
// FP64, then rebuilds (M M)_ij exactly whenever |(M M)_ij| < prod(m_t)/2.  By
// Cauchy-Schwarz |(M M)_ij| <= max_i ||M_i||^2, so S is chosen from the largest row norm of
// X.  X^2 = 2^-2S M M carries only the rounding of X to the 2^-S grid (S ~ 35 for a
// density matrix), far below the 1e-10 target of the FP64 path, at 9 INT8 products in
// place of one FP64 product.  This is the residue-number-system form of the Ozaki scheme
// (Ozaki, Uchino and Imamura, "Ozaki Scheme II: A GEMM-oriented emulation of
// floating-point matrix multiplication using an integer modular technique", 2025).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "reduce.cuh"
#include "tc_ptx.cuh"

namespace sp2b {
namespace oz {

constexpr int T = 9;  // number of moduli
// Moduli in Garner order; the even modulus 256 is last, so the sign of a residue vector
// (whether Y >= prod/2) is the top bit of the last mixed-radix digit.
__host__ __device__ constexpr int mod(int t) {
  return t == 0 ? 255 : t == 1 ? 253 : t == 2 ? 251 : t == 3 ? 247 : t == 4 ? 241
       : t == 5 ? 239 : t == 6 ? 233 : t == 7 ? 229 : 256;
}
// a^-1 mod m (gcd(a, m) = 1), extended Euclid.
__host__ __device__ constexpr int inv_mod(int a, int m) {
  int t = 0, nt = 1, r = m, nr = a % m;
  while (nr != 0) {
    const int q = r / nr;
    int tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return t < 0 ? t + m : t;
}
__host__ __device__ constexpr int pow2_mod(int e, int m) {
  int v = 1 % m;
  for (int i = 0; i < e; ++i) v = (v * 2) % m;
  return v;
}
// prod(m_t) / 2 = 2^70.41; the CRT is exact for |Y| below it.
__host__ __device__ inline double half_prod() {
  double p = 0.5;
  for (int t = 0; t < T; ++t) p *= (double)mod(t);
  return p;
}

// Tile edges of the INT8 product: 128 rows x 256 columns, K in 128-byte blocks.
constexpr int BM = 128, BN = 256, BK = 128, UK = 32, ST = 4;
constexpr int A_BYTES = BM * BK, B_BYTES = BN * BK;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int SMEM_BYTES = ST * STAGE_BYTES + 1024;
constexpr int NWARP = 10, NTHR = NWARP * 32, EPI_WARPS = 8;
constexpr int TMEM_COLS = 2 * BN;
}  // namespace oz

// Scale state shared by the kernels of one refinement: the largest squared row norm
// (as the bits of a non-negative double, for atomicMax) and the chosen exponent S.
struct OzScale {
  unsigned long long r2max_bits;
  int S;      // -1: no valid scale (non-finite input)
  int pad;
};

// SP2-step context of the launches that compute one step's X^2 (the exact INT8 mode):
// they do nothing once the loop has finished or when this step's rule says stop, which
// the step's last launch (k_oz_crt_step) would decide from the same record.
__device__ __forceinline__ bool oz_skip(const OzStepCtl& c) {
  if (!c.active) return false;
  if (*(volatile const int*)&c.sout->done) return true;
  const SP2Rec r = c.rec[c.k];
  if (r.done) return true;
  return sp2_decide(c.ctl, r, c.k, c.pp_in).branch == BR_STOP;
}

template <typename T>
struct OzSplit;
template <>
struct OzSplit<__half> {
  static constexpr double kInv = 1.0 / 2048.0, kScale = 2048.0;
  __device__ static double d(__half h) { return (double)__half2float(h); }
  __device__ static __half from_d(double v) { return __double2half(v); }
};
template <>
struct OzSplit<__nv_bfloat16> {
  static constexpr double kInv = 1.0 / 256.0, kScale = 256.0;
  __device__ static double d(__nv_bfloat16 h) { return (double)__bfloat162float(h); }
  __device__ static __nv_bfloat16 from_d(double v) { return __double2bfloat16(v); }
};

// ---------------------------------------------------------------------------------
// 1. Largest squared row norm of X = hi + 2^-s lo (one warp per row).
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void k_oz_rownorm(const T* __restrict__ hi, const T* __restrict__ lo, int np,
                             OzScale* sc) {
  using SP = OzSplit<T>;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  double best = 0.0;
  for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < np; row += gridDim.x * wpb) {
    const T* h = hi + (size_t)row * np;
    const T* l = lo + (size_t)row * np;
    double s = 0.0;
    for (int c = lane * 8; c < np; c += 256) {
      alignas(16) T hv[8], lv[8];
      *reinterpret_cast<uint4*>(hv) = *reinterpret_cast<const uint4*>(h + c);
      *reinterpret_cast<uint4*>(lv) = *reinterpret_cast<const uint4*>(l + c);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double x = fma(SP::kInv, SP::d(lv[q]), SP::d(hv[q]));
        s = fma(x, x, s);
      }
    }
    s = warp_sum(s);
    // NaN propagates as a maximum: its bit pattern is above every finite value
    if (!(s <= best)) best = s;
  }
  if (lane == 0) {
    unsigned long long b = (unsigned long long)__double_as_longlong(best);
    if (best != best) b = 0x7ff8000000000000ull;
    atomicMax(&sc->r2max_bits, b);
  }
}

// The same for an FP64 iterate (exact INT8 mode).
__global__ void k_oz_rownorm_f64(const double* __restrict__ x, int np, OzScale* sc,
                                 const OzStepCtl c) {
  if (oz_skip(c)) return;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  double best = 0.0;
  for (int row = blockIdx.x * wpb + (threadIdx.x >> 5); row < np; row += gridDim.x * wpb) {
    const double2* xr = reinterpret_cast<const double2*>(x + (size_t)row * np);
    double s = 0.0;
    for (int c = lane; c < np / 2; c += 32) {
      const double2 v = xr[c];
      s = fma(v.x, v.x, s);
      s = fma(v.y, v.y, s);
    }
    s = warp_sum(s);
    if (!(s <= best)) best = s;
  }
  if (lane == 0) {
    unsigned long long b = (unsigned long long)__double_as_longlong(best);
    if (best != best) b = 0x7ff8000000000000ull;
    atomicMax(&sc->r2max_bits, b);
  }
}

// S: the largest exponent with (2^S sqrt(r2max) + sqrt(np)/2)^2 < prod/2, which bounds
// every |(M M)_ij| (row norms of M are at most 2^S ||x_i|| + sqrt(np)/2).
__global__ void k_oz_scale(OzScale* sc, int np) {
  const double r2 = __longlong_as_double((long long)sc->r2max_bits);
  int S = -1;
  if (r2 == r2 && r2 < 1e300) {
    const double lim = sqrt(oz::half_prod()) * (1.0 - 1e-12);
    const double r = sqrt(r2);
    const double e = 0.5 * sqrt((double)np);
    S = 200;
    if (r > 0.0) {
      S = (int)floor(log2((lim - e) / r));
      if (S > 200) S = 200;
      while (S > -1 && ldexp(r, S) + e >= lim) --S;
    }
  }
  sc->S = S;
}

// ---------------------------------------------------------------------------------
// 2. Residue planes: R_t = rint(2^S X) mod m_t in the symmetric range (signed 8-bit).
//    Plane t is np x np at res + t * np * np.
// ---------------------------------------------------------------------------------
// A residue of M = mh 2^21 + ml modulo m, any representative with |r| <= 127 (the
// products only need r = M mod m and |r| <= 128).  v = mh (2^21 mod m) + ml is an integer
// below 2^24 in magnitude, exact in FP32; q = rint(v / m) is off the nearest integer by at
// most one ulp of v/m, so r = v - q m is exact and |r| <= m/2 + 0.005 m.
template <int t>
__device__ __forceinline__ int8_t oz_residue(float mhf, float mlf, int ml) {
  constexpr int m = oz::mod(t);
  if constexpr (m == 256) {
    return (int8_t)(uint8_t)(ml & 255);
  } else {
    constexpr float c = (float)oz::pow2_mod(21, m);
    constexpr float inv = 1.0f / (float)m;
    const float v = fmaf(mhf, c, mlf);
    const float q = rintf(v * inv);
    return (int8_t)__float2int_rn(fmaf(-q, (float)m, v));
  }
}

template <int t>
__device__ __forceinline__ void oz_store_planes(int8_t* res, size_t plane, size_t off,
                                                const float (&mh)[16], const float (&mlf)[16],
                                                const int (&ml)[16]) {
  if constexpr (t < oz::T) {
    alignas(16) int8_t v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = oz_residue<t>(mh[q], mlf[q], ml[q]);
    *reinterpret_cast<uint4*>(res + (size_t)t * plane + off) = *reinterpret_cast<const uint4*>(v);
    oz_store_planes<t + 1>(res, plane, off, mh, mlf, ml);
  }
}

template <typename T>
__global__ void k_oz_residues(const T* __restrict__ hi, const T* __restrict__ lo, int np,
                              const OzScale* __restrict__ sc, int8_t* __restrict__ res) {
  using SP = OzSplit<T>;
  const int S = sc->S;
  const double scale = ldexp(1.0, S < 0 ? 0 : S);
  const size_t plane = (size_t)np * np;
  const size_t groups = plane / 16;
  for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups;
       g += (size_t)gridDim.x * blockDim.x) {
    const size_t off = g * 16;
    alignas(16) T hv[16], lv[16];
    reinterpret_cast<uint4*>(hv)[0] = reinterpret_cast<const uint4*>(hi + off)[0];
    reinterpret_cast<uint4*>(hv)[1] = reinterpret_cast<const uint4*>(hi + off)[1];
    reinterpret_cast<uint4*>(lv)[0] = reinterpret_cast<const uint4*>(lo + off)[0];
    reinterpret_cast<uint4*>(lv)[1] = reinterpret_cast<const uint4*>(lo + off)[1];
    float mh[16], mlf[16];
    int ml[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      // |x| <= sqrt(r2max), so |M| < sqrt(prod/2) < 2^36: exact in FP64, and the split
      // M = mh 2^21 + ml (0 <= ml < 2^21, |mh| < 2^15) is exact in FP32 and int32.
      const double x = fma(SP::kInv, SP::d(lv[q]), SP::d(hv[q]));
      const double M = S < 0 ? 0.0 : rint(x * scale);
      const double h = floor(M * 0x1p-21);
      const double l = M - h * 0x1p21;
      mh[q] = (float)h;
      mlf[q] = (float)l;
      ml[q] = (int)l;
    }
    oz_store_planes<0>(res, plane, off, mh, mlf, ml);
  }
}

__global__ void k_oz_residues_f64(const double* __restrict__ x, int np,
                                  const OzScale* __restrict__ sc, int8_t* __restrict__ res,
                                  const OzStepCtl c) {
  if (oz_skip(c)) return;
  const int S = sc->S;
  const double scale = ldexp(1.0, S < 0 ? 0 : S);
  const size_t plane = (size_t)np * np;
  const size_t groups = plane / 16;
  for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups;
       g += (size_t)gridDim.x * blockDim.x) {
    const size_t off = g * 16;
    const double2* src = reinterpret_cast<const double2*>(x + off);
    float mh[16], mlf[16];
    int ml[16];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double2 v = src[q];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const double M = S < 0 ? 0.0 : rint((e ? v.y : v.x) * scale);
        const double h = floor(M * 0x1p-21);
        const double l = M - h * 0x1p21;
        mh[2 * q + e] = (float)h;
        mlf[2 * q + e] = (float)l;
        ml[2 * q + e] = (int)l;
      }
    }
    oz_store_planes<0>(res, plane, off, mh, mlf, ml);
  }
}

// ---------------------------------------------------------------------------------
// 3. Persistent INT8 product of every plane with itself, upper 128 x 256 tiles,
//    epilogue P mod m_t -> uint8 plane Q_t.
//    warp 0: TMA producer; warp 1: TMEM owner + MMA issuer; warps 2..9: epilogue.
// ---------------------------------------------------------------------------------
struct OzGemmArgs {
  int np;
  int ntiles;             // tiles per plane
  const int2* tiles;      // {bi (128-row block), bjp (256-column block)}
  uint8_t* q;             // T planes np x np
  int* err;
  OzStepCtl ctl;
};

__global__ void __launch_bounds__(oz::NTHR, 1)
    k_oz_gemm(const __grid_constant__ CUtensorMap tm, const OzGemmArgs p) {
  if (oz_skip(p.ctl)) return;   // the same answer in every CTA
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full[oz::ST];
  __shared__ __align__(8) uint64_t bar_empty[oz::ST];
  __shared__ __align__(8) uint64_t bar_tfull[2];
  __shared__ __align__(8) uint64_t bar_tempty[2];
  __shared__ __align__(8) uint64_t bar_final;
  __shared__ uint32_t tmem_holder;
  __shared__ volatile int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < oz::ST; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&bar_tfull[a]), 1);
      mbar_init(smem_u32(&bar_tempty[a]), oz::EPI_WARPS);
    }
    mbar_init(smem_u32(&bar_final), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_holder), oz::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;
  const int np = p.np;
  const int nwork = oz::T * p.ntiles;
  const int KB = np / oz::BK;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer ----------------
      int issued_phase[oz::ST];
      for (int s = 0; s < oz::ST; ++s) issued_phase[s] = -1;
      bool ok = true;
      uint32_t g = 0;
      for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x) {
        const int t = w / p.ntiles;
        const int2 tl = p.tiles[w - t * p.ntiles];
        const int ra = t * np + tl.x * oz::BM, rb = t * np + tl.y * oz::BN;
        for (int kb = 0; kb < KB; ++kb, ++g) {
          const int s = g % oz::ST;
          const uint32_t u = g / oz::ST;
          if (g >= (uint32_t)oz::ST && !mbar_wait(smem_u32(&bar_empty[s]), (u - 1) & 1, &s_abort)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&bar_full[s]);
          const uint32_t st = sbase + s * oz::STAGE_BYTES;
          mbar_expect_tx(fb, oz::STAGE_BYTES);
          tma_load_2d(st, &tm, fb, kb * oz::BK, ra);
          tma_load_2d(st + oz::A_BYTES, &tm, fb, kb * oz::BK, rb);
          tma_load_2d(st + oz::A_BYTES + oz::BM * oz::BK, &tm, fb, kb * oz::BK, rb + oz::BM);
          issued_phase[s] = u & 1;
        }
      }
      if (!ok) {  // abort: wait (bounded) for this CTA's copies still in flight
        for (int s = 0; s < oz::ST; ++s)
          if (issued_phase[s] >= 0)
            for (uint32_t i = 0; i < kSpinLimit; ++i)
              if (mbar_try(smem_u32(&bar_full[s]), issued_phase[s])) break;
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer ----------------
      constexpr uint32_t idesc = make_idesc_s8(oz::BM, oz::BN);
      bool ok = true;
      uint32_t g = 0, tl = 0;
      for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x, ++tl) {
        const int a = tl & 1;
        const uint32_t v = tl >> 1;
        if (tl >= 2 && !mbar_wait(smem_u32(&bar_tempty[a]), (v - 1) & 1, &s_abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc = tmem + a * oz::BN;
        for (int kb = 0; kb < KB; ++kb, ++g) {
          const int s = g % oz::ST;
          if (!mbar_wait(smem_u32(&bar_full[s]), (g / oz::ST) & 1, &s_abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + s * oz::STAGE_BYTES;
          const uint64_t da = sw128_desc(st);
          const uint64_t db = sw128_desc(st + oz::A_BYTES);
#pragma unroll
          for (int kk = 0; kk < oz::BK / oz::UK; ++kk) {
            const uint64_t off = (uint64_t)((kk * oz::UK) >> 4);  // 32 bytes along K
            umma_i8(acc, da + off, db + off, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
          }
          umma_commit(smem_u32(&bar_empty[s]));
        }
        if (!ok) break;
        umma_commit(smem_u32(&bar_tfull[a]));
      }
      umma_commit(smem_u32(&bar_final));
      for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try(smem_u32(&bar_final), 0)) break;
      if (!ok) s_abort = 1;
    }
    __syncwarp();
  } else {
    // ---------------- epilogue (8 warps: lane quarter q, 128-column half) ----------------
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t tl = 0;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x, ++tl) {
      const int t = w / p.ntiles;
      const int2 tile = p.tiles[w - t * p.ntiles];
      const int a = tl & 1;
      if (!mbar_wait_idle(smem_u32(&bar_tfull[a]), (tl >> 1) & 1, &s_abort)) break;
      tc_fence_after();
      // P mod m: u = P + off (off a multiple of m, u < 2^32), floor(u / m) by a 64-bit
      // reciprocal (exact for u < 2^32 since 2^-32 < 1/m).
      const uint32_t m = (uint32_t)oz::mod(t);
      const unsigned long long magic = ~0ull / m + 1ull;
      const uint32_t off = m * ((1u << 30) / m + 1u);
      const int r = tile.x * oz::BM + q * 32 + lane;
      uint8_t* qrow = p.q + (size_t)t * np * np + (size_t)r * np;
#pragma unroll 1
      for (int cc = 0; cc < 4; ++cc) {
        const int cl = half * 128 + cc * 32;
        uint32_t v[32];
        tmem_ld32(tmem + lane_base + a * oz::BN + cl, v);
        tmem_wait_ld();
        const int c0 = tile.y * oz::BN + cl;
        if (c0 < np) {
          alignas(16) uint8_t out[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const uint32_t u = (uint32_t)((int)v[j]) + off;
            const uint32_t d = (uint32_t)__umul64hi((unsigned long long)u, magic);
            out[j] = (uint8_t)(u - d * m);
          }
          reinterpret_cast<uint4*>(qrow + c0)[0] = reinterpret_cast<const uint4*>(out)[0];
          reinterpret_cast<uint4*>(qrow + c0)[1] = reinterpret_cast<const uint4*>(out)[1];
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[a]));
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, oz::TMEM_COLS);
  if (s_abort && threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
}

// ---------------------------------------------------------------------------------
// 4. CRT: X^2 (FP64) and 4 (X^2 - X) re-split to hi/lo, both triangles, from the residues
//    of the upper tiles.  One CTA per upper 32 x 32 block pair; the mirror goes through
//    shared memory so both halves are stored row-contiguous.
// ---------------------------------------------------------------------------------
// Pairwise (tree) Chinese remaindering: residues modulo m_a, m_b combine into the residue
// modulo m_a m_b as x = x_a + m_a ((x_b - x_a) m_a^-1 mod m_b).  Eight odd moduli pair up
// to four 16-bit moduli, then two 32-bit ones, then one 64-bit modulus M07; the last
// modulus 256 gives the top digit, whose top bit is the sign (Y >= prod/2).
__host__ __device__ constexpr uint64_t inv_mod64(uint64_t a, uint64_t m) {
  int64_t t = 0, nt = 1;
  int64_t r = (int64_t)m, nr = (int64_t)(a % m);
  while (nr != 0) {
    const int64_t q = r / nr;
    int64_t tmp = t - q * nt;
    t = nt;
    nt = tmp;
    tmp = r - q * nr;
    r = nr;
    nr = tmp;
  }
  return (uint64_t)(t < 0 ? t + (int64_t)m : t);
}
namespace ozc {
constexpr uint32_t M01 = 255u * 253u, M23 = 251u * 247u, M45 = 241u * 239u, M67 = 233u * 229u;
constexpr uint64_t M0123 = (uint64_t)M01 * M23, M4567 = (uint64_t)M45 * M67;
constexpr uint64_t M07 = M0123 * M4567;   // < 2^64
constexpr uint32_t I01 = (uint32_t)inv_mod64(255, 253), I23 = (uint32_t)inv_mod64(251, 247);
constexpr uint32_t I45 = (uint32_t)inv_mod64(241, 239), I67 = (uint32_t)inv_mod64(233, 229);
constexpr uint32_t I0123 = (uint32_t)inv_mod64(M01 % M23, M23);
constexpr uint32_t I4567 = (uint32_t)inv_mod64(M45 % M67, M67);
constexpr uint64_t I07 = inv_mod64(M0123 % M4567, M4567);
constexpr uint32_t I8 = (uint32_t)inv_mod64(M07 % 256u, 256u);
}  // namespace ozc

// x_a in [0, ma), x_b in [0, mb) (ma < 2 mb) -> x in [0, ma mb); 16-bit moduli
template <uint32_t ma, uint32_t mb, uint32_t ia>
__device__ __forceinline__ uint32_t crt_pair16(uint32_t xa, uint32_t xb) {
  const uint32_t t = (xb + 2u * mb - (xa % mb)) % mb;
  return xa + ma * ((t * ia) % mb);
}
// 32-bit level: moduli below 2^16, products below 2^32
template <uint32_t ma, uint32_t mb, uint32_t ia>
__device__ __forceinline__ uint32_t crt_pair32(uint32_t xa, uint32_t xb) {
  const uint32_t xam = xa >= mb ? xa - mb : xa;   // xa < ma < 2 mb
  const uint32_t t = xb >= xam ? xb - xam : xb + mb - xam;
  return xa + ma * ((t * ia) % mb);
}
// Residues (in [0, m_t)) -> the symmetric integer Y, |Y| < prod/2, as a double
// (exact below 2^53 in magnitude, one rounding above).
__device__ __forceinline__ double crt_value(const int (&q)[oz::T]) {
  using namespace ozc;
  const uint32_t x01 = crt_pair16<255u, 253u, I01>((uint32_t)q[0], (uint32_t)q[1]);
  const uint32_t x23 = crt_pair16<251u, 247u, I23>((uint32_t)q[2], (uint32_t)q[3]);
  const uint32_t x45 = crt_pair16<241u, 239u, I45>((uint32_t)q[4], (uint32_t)q[5]);
  const uint32_t x67 = crt_pair16<233u, 229u, I67>((uint32_t)q[6], (uint32_t)q[7]);
  const uint32_t x0123 = crt_pair32<M01, M23, I0123>(x01, x23);
  const uint32_t x4567 = crt_pair32<M45, M67, I4567>(x45, x67);
  const uint64_t xam = x0123 >= M4567 ? (uint64_t)x0123 - M4567 : (uint64_t)x0123;
  const uint64_t t = x4567 >= xam ? x4567 - xam : (uint64_t)x4567 + M4567 - xam;
  const uint64_t x07 = (uint64_t)x0123 + M0123 * ((t * I07) % M4567);
  const uint32_t v8 = (((uint32_t)q[8] - (uint32_t)x07) * I8) & 255u;
  if (v8 == 0) return (double)x07;
  if (v8 == 255) return -(double)(M07 - x07);
  const double m07 = (double)M07;
  return (double)x07 + m07 * (double)(v8 >= 128 ? (int)v8 - 256 : (int)v8);
}

template <typename T>
__global__ void __launch_bounds__(256)
    k_oz_crt(const uint8_t* __restrict__ q, const T* __restrict__ xhi, const T* __restrict__ xlo,
             int np, const OzScale* __restrict__ sc, double* __restrict__ x2out,
             T* __restrict__ rhi, T* __restrict__ rlo) {
  using SP = OzSplit<T>;
  __shared__ double s_x2[32][33];
  __shared__ T s_rh[32][34], s_rl[32][34];
  int ib, jb;
  upper_tile(blockIdx.x, ib, jb);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int S = sc->S;
  const double down = S < 0 ? __longlong_as_double(0x7ff8000000000000ll) : ldexp(1.0, -2 * S);
  const size_t plane = (size_t)np * np;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int il = ty + 8 * k;
    const int i = ib * 32 + il, j = jb * 32 + tx;
    const size_t e = (size_t)i * np + j;
    int v[oz::T];
#pragma unroll
    for (int t = 0; t < oz::T; ++t) v[t] = q[(size_t)t * plane + e];
    const double x2 = crt_value(v) * down;
    const double x = fma(SP::kInv, SP::d(xlo[e]), SP::d(xhi[e]));
    const double r4 = 4.0 * (x2 - x);
    const T h = SP::from_d(r4);
    const T l = SP::from_d((r4 - SP::d(h)) * SP::kScale);
    x2out[e] = x2;
    rhi[e] = h;
    rlo[e] = l;
    s_x2[il][tx] = x2;
    s_rh[il][tx] = h;
    s_rl[il][tx] = l;
  }
  if (ib == jb) return;  // diagonal blocks hold both triangles (the product is symmetric)
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int jl = ty + 8 * k;
    const size_t e = (size_t)(jb * 32 + jl) * np + ib * 32 + tx;
    x2out[e] = s_x2[tx][jl];
    rhi[e] = s_rh[tx][jl];
    rlo[e] = s_rl[tx][jl];
  }
}

// ---------------------------------------------------------------------------------
// 5. Exact INT8 mode: the step's last launch.  X_k^2 from the residues, the branch of
//    step k from its record (control_prologue), X_{k+1} = a X_k^2 + b X_k in FP64 over
//    both triangles, and the step's sums {||X_{k+1}||^2, Tr X_{k+1}, ||X_k - X_k^2||^2,
//    Tr X_k^2} through the last-CTA finalisation, like the other step kernels.  A fixed
//    grid walks the upper 32 x 32 block pairs (diagonal blocks hold both triangles, whose
//    squares are equal bit for bit: the integer products are symmetric).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_oz_crt_step(const uint8_t* __restrict__ q, const OzScale* __restrict__ sc, const StepArgs p) {
  __shared__ double s_v[32][33];
  __shared__ double red[32 * 4];
  __shared__ int s_flag;
  const int br = control_prologue(p);
  if (br < 0) return;
  const double a = br == BR_X2 ? 1.0 : -1.0, b = br == BR_X2 ? 0.0 : 2.0;
  const int np = p.np;
  const double* __restrict__ X = (const double*)p.E;
  double* __restrict__ Xo = (double*)p.out;
  const int S = sc->S;
  const double down = S < 0 ? __longlong_as_double(0x7ff8000000000000ll) : ldexp(1.0, -2 * S);
  const size_t plane = (size_t)np * np;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const long long nb = np / 32, nblk = nb * (nb + 1) / 2;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long bid = blockIdx.x; bid < nblk; bid += gridDim.x) {
    int ib, jb;
    upper_tile((int)bid, ib, jb);
    const double w = ib == jb ? 1.0 : 2.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int il = ty + 8 * k;
      const int i = ib * 32 + il, j = jb * 32 + tx;
      const size_t e = (size_t)i * np + j;
      int v[oz::T];
#pragma unroll
      for (int t = 0; t < oz::T; ++t) v[t] = q[(size_t)t * plane + e];
      const double x2 = crt_value(v) * down;
      const double x = X[e];
      const double nx = fma(a, x2, b * x);
      const double d = x - x2;
      s[0] = fma(w * nx, nx, s[0]);
      s[2] = fma(w * d, d, s[2]);
      if (i == j) {
        s[1] += nx;
        s[3] += x2;
      }
      Xo[e] = nx;
      s_v[il][tx] = nx;
    }
    if (ib != jb) {
      __syncthreads();
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int jl = ty + 8 * k;
        Xo[(size_t)(jb * 32 + jl) * np + ib * 32 + tx] = s_v[tx][jl];
      }
    }
    __syncthreads();
  }
  __threadfence();
  publish_and_finalize(p, s, red, &s_flag);
}

// ---------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------
int oz_nmod() { return oz::T; }

size_t oz_scale_bytes() { return sizeof(OzScale); }

// Upper 128 x 256 tiles of an np x np product: rows of block bi, columns of the 256-wide
// block bjp, for every bjp that reaches the diagonal or beyond (2 bjp + 1 >= bi).  Ordered
// in panels of kOzPanel column blocks, row blocks top to bottom inside a panel, so one wave
// of the persistent grid shares few operand row blocks (their K-slices stay in L2).
constexpr int kOzPanel = 6;
void oz_tile_list(int np, std::vector<int2>& out) {
  out.clear();
  const int nb = np / oz::BM, nbp = (np + oz::BN - 1) / oz::BN;
  for (int p0 = 0; p0 < nbp; p0 += kOzPanel) {
    const int p1 = std::min(nbp, p0 + kOzPanel);
    for (int bi = 0; bi < nb && bi <= 2 * p1 - 1; ++bi)
      for (int bjp = std::max(p0, bi / 2); bjp < p1; ++bjp) out.push_back(make_int2(bi, bjp));
  }
}

static int oz_sms() {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
    v = 148;
  return v;
}

cudaError_t launch_oz_planes(const __half* xhi, const __half* xlo, int np, int bf16,
                             void* scale, int8_t* res, cudaStream_t st) {
  if (np % oz::BM != 0 || np > 65536) return cudaErrorInvalidValue;
  OzScale* sc = (OzScale*)scale;
  cudaError_t e = cudaMemsetAsync(sc, 0, sizeof(OzScale), st);
  if (e != cudaSuccess) return e;
  const int rgrid = std::min((np + 7) / 8, 148 * 8);
  if (bf16)
    k_oz_rownorm<__nv_bfloat16><<<rgrid, 256, 0, st>>>((const __nv_bfloat16*)xhi,
                                                       (const __nv_bfloat16*)xlo, np, sc);
  else
    k_oz_rownorm<__half><<<rgrid, 256, 0, st>>>(xhi, xlo, np, sc);
  k_oz_scale<<<1, 1, 0, st>>>(sc, np);
  const size_t groups = (size_t)np * np / 16;
  const int g = (int)std::min<size_t>((groups + 255) / 256, 148 * 16);
  if (bf16)
    k_oz_residues<__nv_bfloat16><<<g, 256, 0, st>>>((const __nv_bfloat16*)xhi,
                                                    (const __nv_bfloat16*)xlo, np, sc, res);
  else
    k_oz_residues<__half><<<g, 256, 0, st>>>(xhi, xlo, np, sc, res);
  note_launch(3);
  return cudaGetLastError();
}

cudaError_t launch_oz_gemm(const int8_t* res, int np, uint8_t* qout, const int2* tiles,
                           int ntiles, int* err, cudaStream_t st, const OzStepCtl* ctl) {
  if (np % oz::BM != 0 || np > 65536 || ntiles <= 0) return cudaErrorInvalidValue;
  CUtensorMap tm;
  if (!make_tmap_box(&tm, res, (long long)oz::T * np, np, np, TMAP_U8, oz::BM))
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       oz::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  OzGemmArgs a;
  a.np = np;
  a.ntiles = ntiles;
  a.tiles = tiles;
  a.q = qout;
  a.err = err;
  if (ctl) a.ctl = *ctl;
  else memset(&a.ctl, 0, sizeof(a.ctl));
  const int grid = std::min(oz::T * ntiles, oz_sms());
  k_oz_gemm<<<grid, oz::NTHR, oz::SMEM_BYTES, st>>>(tm, a);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_oz_crt(const uint8_t* q, const __half* xhi, const __half* xlo, int np,
                          int bf16, const void* scale, double* x2, __half* rhi, __half* rlo,
                          cudaStream_t st) {
  const int nb = np / 32;
  const unsigned nblk = (unsigned)((long long)nb * (nb + 1) / 2);
  const OzScale* sc = (const OzScale*)scale;
  if (bf16)
    k_oz_crt<__nv_bfloat16><<<nblk, 256, 0, st>>>(q, (const __nv_bfloat16*)xhi,
                                                  (const __nv_bfloat16*)xlo, np, sc, x2,
                                                  (__nv_bfloat16*)rhi, (__nv_bfloat16*)rlo);
  else
    k_oz_crt<__half><<<nblk, 256, 0, st>>>(q, xhi, xlo, np, sc, x2, rhi, rlo);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_oz_planes_f64(const double* x, int np, void* scale, int8_t* res,
                                 const OzStepCtl* ctl, cudaStream_t st) {
  if (np % oz::BM != 0 || np > 65536) return cudaErrorInvalidValue;
  OzScale* sc = (OzScale*)scale;
  cudaError_t e = cudaMemsetAsync(sc, 0, sizeof(OzScale), st);
  if (e != cudaSuccess) return e;
  const int rgrid = std::min((np + 7) / 8, 148 * 8);
  k_oz_rownorm_f64<<<rgrid, 256, 0, st>>>(x, np, sc, *ctl);
  k_oz_scale<<<1, 1, 0, st>>>(sc, np);
  const size_t groups = (size_t)np * np / 16;
  const int g = (int)std::min<size_t>((groups + 255) / 256, 148 * 16);
  k_oz_residues_f64<<<g, 256, 0, st>>>(x, np, sc, res, *ctl);
  note_launch(3);
  return cudaGetLastError();
}

cudaError_t launch_oz_crt_step(const uint8_t* q, const void* scale, const StepArgs& a,
                               cudaStream_t st) {
  if (a.np % 128 != 0) return cudaErrorInvalidValue;
  k_oz_crt_step<<<148 * 8, 256, 0, st>>>(q, (const OzScale*)scale, a);
  note_launch();
  return cudaGetLastError();
}

// Reads back the scale exponent and the largest squared row norm (diagnostics / checks).
cudaError_t oz_read_scale(const void* scale, int* S, double* r2max, cudaStream_t st) {
  OzScale h;
  cudaError_t e = cudaMemcpyAsync(&h, scale, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  *S = h.S;
  unsigned long long b = h.r2max_bits;
  double d;
  memcpy(&d, &b, sizeof(d));
  *r2max = d;
  return cudaSuccess;
}

}  // namespace sp2b
