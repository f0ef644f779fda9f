// Split-precision symmetric products on the 5th-generation tensor cores (sm_100a).
//
// X is held as two 16-bit arrays, X ~= hi + 2^-s lo (s = 11 for FP16, 8 for BF16), and
//   X*X ~= hi*hi + 2^-s (hi*lo + lo*hi)
// is accumulated in FP32 in TMEM: one accumulator for hi*hi, one for the two cross
// terms, merged in FP64 in the epilogue.  Operands are staged by TMA (128-byte swizzle,
// no multicast) through a 3-deep mbarrier pipeline; one thread issues tcgen05.mma; all
// four warps read the accumulators back with tcgen05.ld and run the fused SP2 epilogue
// (branch update, hi/lo re-split of X_{n+1}, mirrored store, FP64 trace and norm sums).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <mutex>

#include "reduce.cuh"
#include "tc_ptx.cuh"

#include <map>
#include <utility>
#include <vector>

namespace sp2b {
namespace tc {
constexpr int BM = 128;  // UMMA M (TMEM lanes)
constexpr int BN = 128;  // UMMA N
constexpr int BK = 64;   // 64 x 16-bit = one 128-byte swizzle row
constexpr int UK = 16;   // K of one kind::f16 MMA
constexpr int ST = 3;    // pipeline depth
constexpr int TILE_BYTES = BM * BK * 2;
constexpr int STAGE_BYTES = 4 * TILE_BYTES;  // A_hi, A_lo, B_hi, B_lo
constexpr int SMEM_BYTES = ST * STAGE_BYTES + 1024;
constexpr int TMEM_COLS = 256;               // two 128-column FP32 accumulators
}  // namespace tc

template <typename T>
struct SplitTraits;
template <>
struct SplitTraits<__half> {
  static constexpr uint32_t kFmt = 0;  // UMMA F16
  static constexpr double kScale = 2048.0, kInv = 1.0 / 2048.0;
  __device__ static double to_d(__half h) { return (double)__half2float(h); }
  __device__ static __half from_d(double v) { return __double2half(v); }
  __device__ static float to_f(__half h) { return __half2float(h); }
  __device__ static __half from_f(float v) { return __float2half_rn(v); }
};
template <>
struct SplitTraits<__nv_bfloat16> {
  static constexpr uint32_t kFmt = 1;  // UMMA BF16
  static constexpr double kScale = 256.0, kInv = 1.0 / 256.0;
  __device__ static double to_d(__nv_bfloat16 h) { return (double)__bfloat162float(h); }
  __device__ static __nv_bfloat16 from_d(double v) { return __double2bfloat16(v); }
  __device__ static float to_f(__nv_bfloat16 h) { return __bfloat162float(h); }
  __device__ static __nv_bfloat16 from_f(float v) { return __float2bfloat16_rn(v); }
};

// ---------------------------------------------------------------------------------
// The kernel.  SYM: one CTA per upper 128x128 tile with the SP2 epilogue.
//              !SYM: one CTA per tile of a plain product, FP32 output.
// ---------------------------------------------------------------------------------
template <typename T, bool SYM>
__global__ void __launch_bounds__(128, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap tm_ahi, const __grid_constant__ CUtensorMap tm_alo,
              const __grid_constant__ CUtensorMap tm_bhi, const __grid_constant__ CUtensorMap tm_blo,
              const StepArgs p, float* plain_out, int plain_n) {
  using TR = SplitTraits<T>;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full[tc::ST];
  __shared__ __align__(8) uint64_t bar_empty[tc::ST];
  __shared__ __align__(8) uint64_t bar_done;
  __shared__ uint32_t tmem_holder;
  __shared__ double red[32 * 4];
  __shared__ int s_flag;
  __shared__ volatile int s_abort;

  double alpha = p.alpha, beta = p.beta;
  if (SYM && p.control) {
    const int br = control_prologue(p);
    if (br < 0) return;
    if (br == BR_X2) { alpha = 1.0; beta = 0.0; }
    else { alpha = -1.0; beta = 2.0; }
  }
  int bi, bj, nloc = p.np, core = p.core, row0 = 0;
  if (SYM && p.tiles) {
    const int4 t = p.tiles[blockIdx.x];
    row0 = t.x;
    bi = t.y >> 16;
    bj = t.y & 0xffff;
    nloc = t.z;
    core = t.w;
  } else if (SYM) {
    upper_tile(blockIdx.x, bi, bj);
  } else {
    bi = blockIdx.y;
    bj = blockIdx.x;
  }
  const int i0 = bi * tc::BM, j0 = bj * tc::BN;
  const int ld = p.ld;
  // every valid tile starts inside its part (i0, j0 < part size <= K extent); anything
  // else is skipped (no loads, no stores, zero partials) instead of addressing outside
  const bool tile_ok = !(SYM && p.tiles) || (i0 < nloc && j0 < nloc);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);

  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < tc::ST; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    mbar_init(smem_u32(&bar_done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(smem_u32(&tmem_holder), tc::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;
  const int KB = tile_ok ? nloc / tc::BK : 0;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer ----------------
      int issued_phase[tc::ST];
      for (int s = 0; s < tc::ST; ++s) issued_phase[s] = -1;
      bool ok = true;
      for (int kb = 0; kb < KB && ok; ++kb) {
        const int s = kb % tc::ST, u = kb / tc::ST;
        if (kb >= tc::ST) ok = mbar_wait(smem_u32(&bar_empty[s]), (u - 1) & 1, &s_abort);
        if (!ok) break;
        const uint32_t fb = smem_u32(&bar_full[s]);
        const uint32_t st = sbase + s * tc::STAGE_BYTES;
        mbar_expect_tx(fb, tc::STAGE_BYTES);
        tma_load_2d(st + 0 * tc::TILE_BYTES, &tm_ahi, fb, kb * tc::BK, row0 + i0);
        tma_load_2d(st + 1 * tc::TILE_BYTES, &tm_alo, fb, kb * tc::BK, row0 + i0);
        tma_load_2d(st + 2 * tc::TILE_BYTES, &tm_bhi, fb, kb * tc::BK, row0 + j0);
        tma_load_2d(st + 3 * tc::TILE_BYTES, &tm_blo, fb, kb * tc::BK, row0 + j0);
        issued_phase[s] = u & 1;
      }
      if (!ok) {
        // Abort: wait (bounded) for this CTA's copies still in flight before leaving.
        for (int s = 0; s < tc::ST; ++s)
          if (issued_phase[s] >= 0) {
            for (uint32_t i = 0; i < kSpinLimit; ++i)
              if (mbar_try(smem_u32(&bar_full[s]), issued_phase[s])) break;
          }
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer ----------------
      constexpr uint32_t idesc = make_idesc(TR::kFmt, tc::BM, tc::BN);
      const uint32_t acc_hh = tmem, acc_x = tmem + tc::BN;
      bool ok = true;
      for (int kb = 0; kb < KB; ++kb) {
        const int s = kb % tc::ST, u = kb / tc::ST;
        ok = mbar_wait(smem_u32(&bar_full[s]), u & 1, &s_abort);
        if (!ok) break;
        tc_fence_after();
        const uint32_t st = sbase + s * tc::STAGE_BYTES;
        const uint64_t d_ahi = sw128_desc(st + 0 * tc::TILE_BYTES);
        const uint64_t d_alo = sw128_desc(st + 1 * tc::TILE_BYTES);
        const uint64_t d_bhi = sw128_desc(st + 2 * tc::TILE_BYTES);
        const uint64_t d_blo = sw128_desc(st + 3 * tc::TILE_BYTES);
#pragma unroll
        for (int kk = 0; kk < tc::BK / tc::UK; ++kk) {
          // advance 16 elements = 32 bytes along K inside the swizzle atom
          const uint64_t off = (uint64_t)((kk * tc::UK * 2) >> 4);
          const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
          umma_f16(acc_hh, d_ahi + off, d_bhi + off, idesc, acc);
          umma_f16(acc_x, d_ahi + off, d_blo + off, idesc, acc);
          umma_f16(acc_x, d_alo + off, d_bhi + off, idesc, 1u);
        }
        umma_commit(smem_u32(&bar_empty[s]));  // stage free once these MMAs retire
      }
      umma_commit(smem_u32(&bar_done));        // accumulators complete
      if (!ok) s_abort = 1;
    }
    __syncwarp();
  }

  // ---------------- epilogue (all 4 warps; warp w owns TMEM lanes 32w..32w+31) ----------
  const bool good = mbar_wait(smem_u32(&bar_done), 0, &s_abort) && !s_abort;
  tc_fence_after();
  double sums[4] = {0.0, 0.0, 0.0, 0.0};
  if (good && tile_ok) {
    const int rl = warp * 32 + lane;
    const int r = i0 + rl;
    const bool diag = SYM && (bi == bj);
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    const size_t base = (size_t)row0 * ld;  // the part's block inside the packed buffers
    const T* Ehi = SYM ? (const T*)p.E + base : nullptr;
    const T* Elo = SYM ? (const T*)p.E_lo + base : nullptr;
    T* Ohi = (SYM && p.out) ? (T*)p.out + base : nullptr;
    T* Olo = (SYM && p.out) ? (T*)p.out_lo + base : nullptr;
#pragma unroll 1
    for (int cc = 0; cc < tc::BN / 32; ++cc) {
      uint32_t hh[32], xx[32];
      tmem_ld32(trow + cc * 32, hh);
      tmem_ld32(trow + tc::BN + cc * 32, xx);
      tmem_wait_ld();
      const int c0 = j0 + cc * 32;
      if (!SYM) {
        // rows bounded by n_out when set (a row panel of the product), else by plain_n
        if (r < (p.n_out > 0 ? p.n_out : plain_n)) {
          for (int j = 0; j < 32; ++j) {
            const int c = c0 + j;
            if (c < plain_n)
              plain_out[(size_t)r * plain_n + c] =
                  (float)((double)__uint_as_float(hh[j]) + TR::kInv * (double)__uint_as_float(xx[j]));
          }
        }
        continue;
      }
      alignas(16) T ehi[32], elo[32], nhi[32], nlo[32];
      {
        const uint4* src_h = reinterpret_cast<const uint4*>(Ehi + (size_t)r * ld + c0);
        const uint4* src_l = reinterpret_cast<const uint4*>(Elo + (size_t)r * ld + c0);
        uint4* dh = reinterpret_cast<uint4*>(ehi);
        uint4* dl = reinterpret_cast<uint4*>(elo);
#pragma unroll
        for (int q = 0; q < 4; ++q) { dh[q] = src_h[q]; dl[q] = src_l[q]; }
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int c = c0 + j;
        const double P = (double)__uint_as_float(hh[j]) + TR::kInv * (double)__uint_as_float(xx[j]);
        const double x = TR::to_d(ehi[j]) + TR::kInv * TR::to_d(elo[j]);
        const double v = alpha * P + beta * x;
        const T h = TR::from_d(v);
        const T l = TR::from_d((v - TR::to_d(h)) * TR::kScale);
        const double vs = TR::to_d(h) + TR::kInv * TR::to_d(l);
        nhi[j] = h;
        nlo[j] = l;
        const int w = sym_weight(diag, r, c);
        const double dres = x - P;
        sums[0] += w * vs * vs;
        sums[2] += core_weight(w, r, c, core) * dres * dres;
        if (r == c) { sums[1] += vs; sums[3] += P; }
        if (Ohi && w && r != c) {
          Ohi[(size_t)c * ld + r] = h;
          Olo[(size_t)c * ld + r] = l;
        }
      }
      if (Ohi) {
        if (!diag) {
          uint4* dh = reinterpret_cast<uint4*>(Ohi + (size_t)r * ld + c0);
          uint4* dl = reinterpret_cast<uint4*>(Olo + (size_t)r * ld + c0);
          const uint4* sh = reinterpret_cast<const uint4*>(nhi);
          const uint4* sl = reinterpret_cast<const uint4*>(nlo);
#pragma unroll
          for (int q = 0; q < 4; ++q) { dh[q] = sh[q]; dl[q] = sl[q]; }
        } else {
          for (int j = 0; j < 32; ++j)
            if (r <= c0 + j) {
              Ohi[(size_t)r * ld + c0 + j] = nhi[j];
              Olo[(size_t)r * ld + c0 + j] = nlo[j];
            }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, tc::TMEM_COLS);
  if (!good && threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
  if (SYM) {
    if (p.out) __threadfence();
    publish_and_finalize(p, sums, red, &s_flag);
  }
}

// ---------------------------------------------------------------------------------
// Persistent, warp-specialised SP2 step (the kernel used for every symmetric launch).
//   warp 0: TMA producer; warp 1: TMEM owner + MMA issuer; warps 2..9: epilogue.
// Each CTA walks its tiles t = blockIdx.x, blockIdx.x + gridDim.x, ... (a fixed
// assignment, so its partial sums are reproducible).  TMEM holds two accumulator
// sets (hi*hi and cross, 128 columns each, x2 = 512 columns): the MMAs of tile t+1 run
// while the epilogue drains tile t.  Each lane quarter of TMEM is read by two
// epilogue warps, one per 64-column half.
// ---------------------------------------------------------------------------------
namespace tcp {
constexpr int NWARP = 10;
constexpr int NTHR = NWARP * 32;
constexpr int EPI_WARPS = 8;
constexpr int TMEM_COLS = 512;
constexpr int CHUNK = 16;  // columns per tcgen05.ld
constexpr int SCR_WARP = 2048;                        // store staging per epilogue warp
constexpr int SCR_OFF = tc::ST * tc::STAGE_BYTES;     // after the operand stages
constexpr int SMEM_BYTES = SCR_OFF + EPI_WARPS * SCR_WARP + 1024;
constexpr int E_BYTES = 4 * tc::TILE_BYTES;           // X_k block of a tile, hi + lo
constexpr int EH_BYTES = 2 * tc::TILE_BYTES;          // batched: one 64-column half of it
constexpr int NWARP_E = NWARP + 1;                    // batched: + the X_k block warp
constexpr int NTHR_E = NWARP_E * 32;
constexpr int SMEM_BYTES_E = 2 * tc::STAGE_BYTES + E_BYTES + EPI_WARPS * SCR_WARP + 1024;
}  // namespace tcp

struct TileInfo {
  int row0, i0, j0, kb, core;
  bool ok, diag;
};

__device__ __forceinline__ TileInfo persist_tile(const StepArgs& p, int t) {
  TileInfo ti;
  int bi, bj, nloc = p.np;
  ti.core = p.core;
  ti.row0 = 0;
  if (p.tiles) {
    const int4 v = p.tiles[t];
    ti.row0 = v.x;
    bi = v.y >> 16;
    bj = v.y & 0xffff;
    nloc = v.z;
    ti.core = v.w == -2 ? p.core : v.w;   // -2: the launch's own core count
  } else {
    upper_tile(t, bi, bj);
  }
  ti.i0 = bi * tc::BM;
  ti.j0 = bj * tc::BN;
  // a valid tile starts inside its part; anything else is skipped
  ti.ok = !p.tiles || (ti.i0 < nloc && ti.j0 < nloc);
  ti.kb = ti.ok ? nloc / tc::BK : 0;
  ti.diag = bi == bj;
  return ti;
}

// Epilogue of one 128 x 128 accumulator tile for the warp that owns TMEM lane quarter q
// and 64-column half `half`; tacc is the TMEM address of its lanes' hi*hi accumulator
// (the cross accumulator follows at + BN columns); scr is the warp's 2 KB of shared
// scratch for staging stores.  ESM: the tile's X_k block was loaded by TMA into estage
// (hi and lo of each 64-column half as 128-byte-swizzled 128 x 64 boxes), is read from
// there, and X_{k+1} is written back in place for a TMA store of the whole tile; only the
// mirror of an off-diagonal tile is stored from the registers.  Otherwise each lane reads
// its row of X_k from global memory and stores the block and its mirror itself.
// ES: the tile's X_k block is staged in shared memory like ESM's (estage: this half's hi
// box, then its lo box, 128-byte swizzle), the results leave by the direct stores.
template <typename T, int EPI, bool ESM, bool ES = false>
__device__ __forceinline__ void epi_tile(const StepArgs& p, const TileInfo& ti, uint32_t tacc,
                                         int q, int half, int lane, double alpha, double beta,
                                         double (&sums)[4], uint8_t* scr, uint8_t* estage,
                                         int cc_lo = 0, int cc_hi = 64 / tcp::CHUNK) {
  using TR = SplitTraits<T>;
  const int ld = p.ld;
  if (EPI == 0 && ti.ok) {
    const int r = ti.i0 + q * 32 + lane;  // row inside the part
    const size_t base = (size_t)ti.row0 * ld;
    const T* Ehi = (const T*)p.E + base;
    const T* Elo = (const T*)p.E_lo + base;
    T* Ohi = p.out ? (T*)p.out + base : nullptr;
    T* Olo = p.out ? (T*)p.out_lo + base : nullptr;
    const int r0 = ti.i0 + q * 32;   // first row of this warp
    // On a diagonal tile the blocks wholly below the diagonal (a prefix of this warp's
    // chunks) carry weight zero and are stored through their mirror images: skipped.
    // The batched form (ESM) computes a diagonal tile whole instead: every element stands
    // for itself in the sums, every warp has the same four chunks, and the tile leaves by
    // TMA as computed.
    int first = cc_lo;
    while (!ESM && first < cc_hi && ti.diag && ti.j0 + half * 64 + first * tcp::CHUNK + 15 < r0)
      ++first;
    // the rows of X_k for the next chunk are fetched while this one is processed
    uint4 pf[4];
    auto fetch_e = [&](int c0x) {
      const uint4* sh = reinterpret_cast<const uint4*>(Ehi + (size_t)r * ld + c0x);
      const uint4* sl = reinterpret_cast<const uint4*>(Elo + (size_t)r * ld + c0x);
      pf[0] = sh[0];
      pf[1] = sh[1];
      pf[2] = sl[0];
      pf[3] = sl[1];
    };
    if (!ESM && !ES && first < cc_hi) fetch_e(ti.j0 + half * 64 + first * tcp::CHUNK);
    const int rl = q * 32 + lane;   // row inside the tile
#pragma unroll 1
    for (int cc = first; cc < cc_hi; ++cc) {
      const int cl = half * 64 + cc * tcp::CHUNK;
      uint32_t hh[16], xx[16];
      tmem_ld16(tacc + cl, hh);
      tmem_ld16(tacc + tc::BN + cl, xx);
      const int c0 = ti.j0 + cl;
      alignas(16) T ehi[16], elo[16], nhi[16], nlo[16];
      // 16-byte chunk k of row rl of a staged box sits at chunk k ^ (rl & 7) (128-byte
      // swizzle); estage is this half's stage: the hi box, then the lo box
      uint8_t* eb = (ESM || ES) ? estage + rl * 128 : nullptr;
      const int k0 = ((2 * cc) ^ (rl & 7)) * 16, k1 = ((2 * cc + 1) ^ (rl & 7)) * 16;
      {
        uint4* dh = reinterpret_cast<uint4*>(ehi);
        uint4* dl = reinterpret_cast<uint4*>(elo);
        if (ESM || ES) {
          dh[0] = *reinterpret_cast<const uint4*>(eb + k0);
          dh[1] = *reinterpret_cast<const uint4*>(eb + k1);
          dl[0] = *reinterpret_cast<const uint4*>(eb + tc::TILE_BYTES + k0);
          dl[1] = *reinterpret_cast<const uint4*>(eb + tc::TILE_BYTES + k1);
        } else {
          dh[0] = pf[0];
          dh[1] = pf[1];
          dl[0] = pf[2];
          dl[1] = pf[3];
        }
      }
      if (!ESM && !ES && cc + 1 < cc_hi) fetch_e(c0 + tcp::CHUNK);
      tmem_wait_ld();
      // Element math in FP32: x = hi + 2^-s lo is exact in FP32, P carries the
      // FP32 accumulators' precision, and X_{k+1} is re-split to the same 2 x 11
      // (or 2 x 8) bits; only the sums that drive the branch rule are FP64.
      const float kInvF = (float)TR::kInv, kScaleF = (float)TR::kScale;
      const float af = (float)alpha, bf = (float)beta;  // 1/0 or -1/2: exact
      // Off-diagonal tiles whose core weight is the same across the 16 columns take the
      // short path: the norm and residual sums of the block in FP32 (two independent
      // chains each, fixed order), added to the FP64 totals once per block.  The
      // residual x - P = (x - hh) - 2^-s xx keeps the accumulators' precision: x - hh is
      // exact when hh is within a factor 2 of x, and the FMA rounds once.
      const bool above = !ti.diag || c0 > r0 + 31;   // every element has r < c
      const bool uniform = above && (ti.core <= 0 || c0 + 15 < ti.core || c0 >= ti.core);
      if (ESM && ti.diag) {
        // whole diagonal tile: weight 1 in the norm, the row's core flag in the residual;
        // the diagonal element of this lane's row (if in this chunk) is picked by selects
        float s0a = 0.f, s0b = 0.f, s2a = 0.f, s2b = 0.f;
        float dvs = 0.f, dhh = 0.f, dxx = 0.f;
        const int jd = r - c0;   // this row's diagonal element is column j = jd
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float hhf = __uint_as_float(hh[j]), xxf = __uint_as_float(xx[j]);
          const float P = fmaf(kInvF, xxf, hhf);
          const float x = fmaf(kInvF, TR::to_f(elo[j]), TR::to_f(ehi[j]));
          const float val = fmaf(af, P, bf * x);
          const T h = TR::from_f(val);
          const float hf = TR::to_f(h);
          const T l = TR::from_f((val - hf) * kScaleF);
          const float dres = fmaf(-kInvF, xxf, x - hhf);
          nhi[j] = h;
          nlo[j] = l;
          if (j & 1) {
            s0b = fmaf(val, val, s0b);
            s2b = fmaf(dres, dres, s2b);
          } else {
            s0a = fmaf(val, val, s0a);
            s2a = fmaf(dres, dres, s2a);
          }
          if (c0 + 15 >= r0 && c0 <= r0 + 31) {   // warp-uniform: the chunk meets the diagonal
            const bool dg = j == jd;
            dvs = dg ? fmaf(kInvF, TR::to_f(l), hf) : dvs;
            dhh = dg ? hhf : dhh;
            dxx = dg ? xxf : dxx;
          }
        }
        const bool rin = ti.core <= 0 || r < ti.core;
        sums[0] += (double)s0a + (double)s0b;
        if (rin) sums[2] += (double)s2a + (double)s2b;
        if (jd >= 0 && jd < 16) {
          sums[1] += (double)dvs;
          sums[3] += fma(TR::kInv, (double)dxx, (double)dhh);
        }
      } else if (uniform) {
        float s0a = 0.f, s0b = 0.f, s2a = 0.f, s2b = 0.f;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float hhf = __uint_as_float(hh[j]), xxf = __uint_as_float(xx[j]);
          const float P = fmaf(kInvF, xxf, hhf);
          const float x = fmaf(kInvF, TR::to_f(elo[j]), TR::to_f(ehi[j]));
          const float val = fmaf(af, P, bf * x);
          const T h = TR::from_f(val);
          const float hf = TR::to_f(h);
          const T l = TR::from_f((val - hf) * kScaleF);
          const float vs = fmaf(kInvF, TR::to_f(l), hf);
          const float dres = fmaf(-kInvF, xxf, x - hhf);
          nhi[j] = h;
          nlo[j] = l;
          if (j & 1) {
            s0b = fmaf(vs, vs, s0b);
            s2b = fmaf(dres, dres, s2b);
          } else {
            s0a = fmaf(vs, vs, s0a);
            s2a = fmaf(dres, dres, s2a);
          }
        }
        const int wc = ti.core <= 0 ? 2 : (r < ti.core ? 1 : 0) + (c0 < ti.core ? 1 : 0);
        sums[0] = fma(2.0, (double)s0a + (double)s0b, sums[0]);
        sums[2] = fma((double)wc, (double)s2a + (double)s2b, sums[2]);
      } else {
        // Blocks on the diagonal or across the core boundary: the same FP32 chains with
        // per-element weights (selects, no branches); the diagonal element's value and
        // product (the traces of X_{k+1} and of the product) enter the FP64 sums once.
        float s0a = 0.f, s0b = 0.f, s2a = 0.f, s2b = 0.f;
        float dvs = 0.f, dhh = 0.f, dxx = 0.f;
        const int core = ti.core;
        const float rin = (core <= 0 || r < core) ? 1.f : 0.f;   // row r is a core row
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int c = c0 + j;
          const float hhf = __uint_as_float(hh[j]), xxf = __uint_as_float(xx[j]);
          const float P = fmaf(kInvF, xxf, hhf);
          const float x = fmaf(kInvF, TR::to_f(elo[j]), TR::to_f(ehi[j]));
          const float val = fmaf(af, P, bf * x);
          const T h = TR::from_f(val);
          const float hf = TR::to_f(h);
          const T l = TR::from_f((val - hf) * kScaleF);
          const float vs = fmaf(kInvF, TR::to_f(l), hf);
          const float dres = fmaf(-kInvF, xxf, x - hhf);
          nhi[j] = h;
          nlo[j] = l;
          // sym_weight / core_weight as selects
          const bool dg = r == c;
          const float wf = (!ti.diag || r < c) ? 2.f : (dg ? 1.f : 0.f);
          const float cin = (core <= 0 || c < core) ? 1.f : 0.f;
          const float cwf = core <= 0 ? wf : (wf == 0.f ? 0.f : (dg ? rin : rin + cin));
          dvs = dg ? vs : dvs;
          dhh = dg ? hhf : dhh;
          dxx = dg ? xxf : dxx;
          if (j & 1) {
            s0b = fmaf(wf * vs, vs, s0b);
            s2b = fmaf(cwf * dres, dres, s2b);
          } else {
            s0a = fmaf(wf * vs, vs, s0a);
            s2a = fmaf(cwf * dres, dres, s2a);
          }
        }
        sums[0] += (double)s0a + (double)s0b;
        sums[2] += (double)s2a + (double)s2b;
        if (r >= c0 && r < c0 + 16) {
          sums[1] += (double)dvs;
          sums[3] += fma(TR::kInv, (double)dxx, (double)dhh);
        }
      }
      if (ESM) {
        // X_{k+1} in place of X_k; the whole tile leaves by TMA once every warp is done
        *reinterpret_cast<uint4*>(eb + k0) = reinterpret_cast<const uint4*>(nhi)[0];
        *reinterpret_cast<uint4*>(eb + k1) = reinterpret_cast<const uint4*>(nhi)[1];
        *reinterpret_cast<uint4*>(eb + tc::TILE_BYTES + k0) = reinterpret_cast<const uint4*>(nlo)[0];
        *reinterpret_cast<uint4*>(eb + tc::TILE_BYTES + k1) = reinterpret_cast<const uint4*>(nlo)[1];
        if (ti.diag) continue;   // computed whole: stored as it is
        if (!Ohi) continue;
        T* th = reinterpret_cast<T*>(scr);          // [16][32]: mirror rows c0 + j
        T* tl = reinterpret_cast<T*>(scr + 1024);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          th[j * 32 + lane] = nhi[j];
          tl[j * 32 + lane] = nlo[j];
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int j = (lane >> 2) + 8 * i, piece = lane & 3;
          const uint4 vh = *reinterpret_cast<const uint4*>(th + j * 32 + piece * 8);
          const uint4 vl = *reinterpret_cast<const uint4*>(tl + j * 32 + piece * 8);
          *reinterpret_cast<uint4*>(Ohi + (size_t)(c0 + j) * ld + r0 + piece * 8) = vh;
          *reinterpret_cast<uint4*>(Olo + (size_t)(c0 + j) * ld + r0 + piece * 8) = vl;
        }
        __syncwarp();
        continue;
      }
      if (!Ohi) continue;
      // Stores of this 32 x 16 block (rows r0.., columns c0..) and of its mirror.  Whole
      // blocks go through the warp's scratch so that every store instruction writes
      // 16-byte pieces of a few rows: the mirror as 8 rows x 64 B per instruction, the
      // block itself as 16 rows x 32 B; on a diagonal tile only blocks that straddle the
      // diagonal store element by element (r <= c authoritative), and blocks below it
      // store nothing (their mirror images carry them).
      if (above) {
        T* th = reinterpret_cast<T*>(scr);          // [16][32]: mirror rows c0 + j
        T* tl = reinterpret_cast<T*>(scr + 1024);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          th[j * 32 + lane] = nhi[j];
          tl[j * 32 + lane] = nlo[j];
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int j = (lane >> 2) + 8 * i, piece = lane & 3;
          const uint4 vh = *reinterpret_cast<const uint4*>(th + j * 32 + piece * 8);
          const uint4 vl = *reinterpret_cast<const uint4*>(tl + j * 32 + piece * 8);
          *reinterpret_cast<uint4*>(Ohi + (size_t)(c0 + j) * ld + r0 + piece * 8) = vh;
          *reinterpret_cast<uint4*>(Olo + (size_t)(c0 + j) * ld + r0 + piece * 8) = vl;
        }
        __syncwarp();
        T* dh = reinterpret_cast<T*>(scr);          // [32][16]: rows r0 + rr
        T* dl = reinterpret_cast<T*>(scr + 1024);
        reinterpret_cast<uint4*>(dh + lane * 16)[0] = reinterpret_cast<const uint4*>(nhi)[0];
        reinterpret_cast<uint4*>(dh + lane * 16)[1] = reinterpret_cast<const uint4*>(nhi)[1];
        reinterpret_cast<uint4*>(dl + lane * 16)[0] = reinterpret_cast<const uint4*>(nlo)[0];
        reinterpret_cast<uint4*>(dl + lane * 16)[1] = reinterpret_cast<const uint4*>(nlo)[1];
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int rr = (lane >> 1) + 16 * i, piece = lane & 1;
          const uint4 vh = *reinterpret_cast<const uint4*>(dh + rr * 16 + piece * 8);
          const uint4 vl = *reinterpret_cast<const uint4*>(dl + rr * 16 + piece * 8);
          *reinterpret_cast<uint4*>(Ohi + (size_t)(r0 + rr) * ld + c0 + piece * 8) = vh;
          *reinterpret_cast<uint4*>(Olo + (size_t)(r0 + rr) * ld + c0 + piece * 8) = vl;
        }
        __syncwarp();
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int c = c0 + j;
          if (r < c) {
            Ohi[(size_t)c * ld + r] = nhi[j];
            Olo[(size_t)c * ld + r] = nlo[j];
          }
          if (r <= c) {
            Ohi[(size_t)r * ld + c] = nhi[j];
            Olo[(size_t)r * ld + c] = nlo[j];
          }
        }
      }
    }
  }
  if (EPI == 1 && ti.ok) {
    // D = 2 X^2 - X (4R): X^2 exact to the INT8 refinement's grid (FP64), the
    // correction X (4R) small, so its split-precision product is far below it.
    const int r = ti.i0 + q * 32 + lane;
    const double* X2 = (const double*)p.E;
    double* D = (double*)p.out;
    const int nout = p.n_out, ldo = p.ld_out;
#pragma unroll 1
    for (int cc = 0; cc < 64 / tcp::CHUNK; ++cc) {
      const int cl = half * 64 + cc * tcp::CHUNK;
      uint32_t hh[16], xx[16];
      tmem_ld16(tacc + cl, hh);
      tmem_ld16(tacc + tc::BN + cl, xx);
      tmem_wait_ld();
      const int c0 = ti.j0 + cl;
      double x2[16];
      const double2* src = reinterpret_cast<const double2*>(X2 + (size_t)r * ld + c0);
#pragma unroll
      for (int h2 = 0; h2 < 8; ++h2) {
        const double2 v2 = src[h2];
        x2[2 * h2] = v2.x;
        x2[2 * h2 + 1] = v2.y;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int c = c0 + j;
        const double acc = fma(TR::kInv, (double)__uint_as_float(xx[j]),
                               (double)__uint_as_float(hh[j]));
        const double d = 2.0 * x2[j] - acc;
        const int w = sym_weight(ti.diag, r, c);
        if (w && r < nout && c < nout) {
          D[(size_t)r * ldo + c] = d;
          if (r != c) D[(size_t)c * ldo + r] = d;
          sums[0] = fma((double)w * d, d, sums[0]);
          if (r == c) sums[1] += d;
        }
      }
    }
  }
}

// EPI 0: SP2 step epilogue (A = B = E = X_k).  EPI 1: McWeeny combine of the INT8
// refinement, D = 2 X^2 - acc with acc = X (4R) (A = X, B = 4R = 4(X^2 - X), E = X^2 in
// FP64), written to the n_out x n_out density (row pitch ld_out) and mirrored.
// ESM (batched sub-graph steps): two operand stages; the tile's X_k block comes by TMA
// into a 64 KB stage (loaded while the tile's MMAs run), X_{k+1} is written over it and
// leaves by TMA stores (tm_ohi / tm_olo: the output arrays); a diagonal tile is computed
// whole (both triangles, as the MMA gives them); only off-diagonal mirrors use ordinary
// stores.
template <typename T, int EPI, bool ESM>
__global__ void __launch_bounds__(ESM ? tcp::NTHR_E : tcp::NTHR, 1)
    k_tc_persist(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                 const __grid_constant__ CUtensorMap tm_bhi,
                 const __grid_constant__ CUtensorMap tm_blo,
                 const __grid_constant__ CUtensorMap tm_ohi,
                 const __grid_constant__ CUtensorMap tm_olo, const StepArgs p, int ntiles) {
  using TR = SplitTraits<T>;
  constexpr int ST = ESM ? 2 : tc::ST;
  constexpr int EOFF = ST * tc::STAGE_BYTES;                      // X_k block stage (ESM)
  constexpr int SOFF = ESM ? EOFF + tcp::E_BYTES : tcp::SCR_OFF;  // store scratch
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full[tc::ST];
  __shared__ __align__(8) uint64_t bar_empty[tc::ST];
  __shared__ __align__(8) uint64_t bar_tfull[2];
  __shared__ __align__(8) uint64_t bar_tempty[2];
  __shared__ __align__(8) uint64_t bar_final;
  __shared__ __align__(8) uint64_t bar_efull[2];   // ESM: X_k half block landed (per stage)
  __shared__ __align__(8) uint64_t bar_odone[2];   // ESM: every warp wrote its part of it
  __shared__ uint32_t tmem_holder;
  __shared__ double red[32 * 4];
  __shared__ int s_flag;
  __shared__ volatile int s_abort;

  double alpha = p.alpha, beta = p.beta;
  if (p.control) {
    const int br = control_prologue(p);
    if (br < 0) return;
    if (br == BR_X2) { alpha = 1.0; beta = 0.0; }
    else { alpha = -1.0; beta = 2.0; }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < tc::ST; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&bar_tfull[a]), 1);
      mbar_init(smem_u32(&bar_tempty[a]), tcp::EPI_WARPS);
    }
    mbar_init(smem_u32(&bar_final), 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&bar_efull[b]), 1);
      mbar_init(smem_u32(&bar_odone[b]), tcp::EPI_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_holder), tcp::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_holder;
  double sums[4] = {0.0, 0.0, 0.0, 0.0};

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer ----------------
      int issued_phase[ST];
      for (int s = 0; s < ST; ++s) issued_phase[s] = -1;
      bool ok = true;
      uint32_t g = 0;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const TileInfo ti = persist_tile(p, t);
        for (int kb = 0; kb < ti.kb; ++kb, ++g) {
          const int s = g % ST;
          const uint32_t u = g / ST;
          if (g >= (uint32_t)ST && !mbar_wait(smem_u32(&bar_empty[s]), (u - 1) & 1, &s_abort)) {
            ok = false;
            break;
          }
          const uint32_t fb = smem_u32(&bar_full[s]);
          const uint32_t st = sbase + s * tc::STAGE_BYTES;
          mbar_expect_tx(fb, tc::STAGE_BYTES);
          tma_load_2d(st + 0 * tc::TILE_BYTES, &tm_hi, fb, kb * tc::BK, ti.row0 + ti.i0);
          tma_load_2d(st + 1 * tc::TILE_BYTES, &tm_lo, fb, kb * tc::BK, ti.row0 + ti.i0);
          tma_load_2d(st + 2 * tc::TILE_BYTES, &tm_bhi, fb, kb * tc::BK, ti.row0 + ti.j0);
          tma_load_2d(st + 3 * tc::TILE_BYTES, &tm_blo, fb, kb * tc::BK, ti.row0 + ti.j0);
          issued_phase[s] = u & 1;
        }
      }
      if (!ok) {  // abort: wait (bounded) for this CTA's copies still in flight
        for (int s = 0; s < ST; ++s)
          if (issued_phase[s] >= 0)
            for (uint32_t i = 0; i < kSpinLimit; ++i)
              if (mbar_try(smem_u32(&bar_full[s]), issued_phase[s])) break;
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer ----------------
      constexpr uint32_t idesc = make_idesc(TR::kFmt, tc::BM, tc::BN);
      bool ok = true;
      uint32_t g = 0, tl = 0;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++tl) {
        const TileInfo ti = persist_tile(p, t);
        const int a = tl & 1;
        const uint32_t v = tl >> 1;
        if (tl >= 2 && !mbar_wait(smem_u32(&bar_tempty[a]), (v - 1) & 1, &s_abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc_hh = tmem + a * 256, acc_x = tmem + a * 256 + tc::BN;
        for (int kb = 0; kb < ti.kb; ++kb, ++g) {
          const int s = g % ST;
          if (!mbar_wait(smem_u32(&bar_full[s]), (g / ST) & 1, &s_abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + s * tc::STAGE_BYTES;
          const uint64_t d_ahi = sw128_desc(st + 0 * tc::TILE_BYTES);
          const uint64_t d_alo = sw128_desc(st + 1 * tc::TILE_BYTES);
          const uint64_t d_bhi = sw128_desc(st + 2 * tc::TILE_BYTES);
          const uint64_t d_blo = sw128_desc(st + 3 * tc::TILE_BYTES);
#pragma unroll
          for (int kk = 0; kk < tc::BK / tc::UK; ++kk) {
            const uint64_t off = (uint64_t)((kk * tc::UK * 2) >> 4);
            const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
            umma_f16(acc_hh, d_ahi + off, d_bhi + off, idesc, acc);
            umma_f16(acc_x, d_ahi + off, d_blo + off, idesc, acc);
            umma_f16(acc_x, d_alo + off, d_bhi + off, idesc, 1u);
          }
          umma_commit(smem_u32(&bar_empty[s]));
        }
        if (!ok) break;
        umma_commit(smem_u32(&bar_tfull[a]));  // accumulators of this tile are complete
      }
      // every MMA issued by this thread has retired once this arrives
      umma_commit(smem_u32(&bar_final));
      for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try(smem_u32(&bar_final), 0)) break;
      if (!ok) s_abort = 1;
    }
    __syncwarp();
  } else if (ESM && warp == tcp::NWARP) {
    // ---------------- X_k half blocks (batched form, one thread) ----------------
    // Phase v = 2u + h is the 64-column half h of this CTA's u-th valid tile; it uses
    // half stage h = v & 1, whose barriers then complete their (v >> 1)-th phase.  While
    // the epilogue warps work on phase v, the load of phase v + 1 is in flight or done;
    // a stage is refilled with phase v + 2 once the stores of phase v have read it.
    if (lane == 0) {
      int tt[2] = {-1, -1};       // tile whose half each stage holds
      int pend[2] = {-1, -1};     // phase parity of a load not yet consumed
      auto next_ok = [&](int t) {
        while (t < ntiles && !persist_tile(p, t).ok) t += gridDim.x;
        return t;
      };
      auto load = [&](int b, int t, uint32_t v) {   // half b of tile t, phase v
        const TileInfo tj = persist_tile(p, t);
        const uint32_t eb = smem_u32(&bar_efull[b]);
        const uint32_t es = sbase + EOFF + b * tcp::EH_BYTES;
        mbar_expect_tx(eb, tcp::EH_BYTES);
        tma_load_2d(es, &tm_hi, eb, tj.j0 + 64 * b, tj.row0 + tj.i0);
        tma_load_2d(es + tc::TILE_BYTES, &tm_lo, eb, tj.j0 + 64 * b, tj.row0 + tj.i0);
        tt[b] = t;
        pend[b] = (int)((v >> 1) & 1);
      };
      int t_load = next_ok(blockIdx.x);   // tile of the next loads
      if (t_load < ntiles) {
        load(0, t_load, 0);
        load(1, t_load, 1);
        t_load = next_ok(t_load + gridDim.x);
      }
      for (uint32_t v = 0;; ++v) {
        const int b = v & 1;
        if (tt[b] < 0) break;
        if (!mbar_wait(smem_u32(&bar_odone[b]), (v >> 1) & 1, &s_abort)) break;
        pend[b] = -1;   // consumed by the epilogue warps, so it had landed
        const TileInfo tj = persist_tile(p, tt[b]);
        const uint32_t es = sbase + EOFF + b * tcp::EH_BYTES;
        tma_store_2d(&tm_ohi, es, tj.j0 + 64 * b, tj.row0 + tj.i0);
        tma_store_2d(&tm_olo, es + tc::TILE_BYTES, tj.j0 + 64 * b, tj.row0 + tj.i0);
        bulk_commit();
        tt[b] = -1;
        if (t_load < ntiles) {
          bulk_wait_read0();
          load(b, t_load, v + 2);
          if (b == 1) t_load = next_ok(t_load + gridDim.x);
        }
      }
      for (int b = 0; b < 2; ++b)   // loads issued but never consumed (abort)
        if (pend[b] >= 0)
          for (uint32_t i = 0; i < kSpinLimit; ++i)
            if (mbar_try(smem_u32(&bar_efull[b]), pend[b])) break;
      bulk_wait0();
    }
    __syncwarp();
  } else {
    // ---------------- epilogue (8 warps) ----------------
    const int q = warp & 3;             // TMEM lane quarter of this warp
    const int half = (warp - 2) >> 2;   // 64-column half of the tile (batched: 32-column quarter of each half)
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    uint32_t tl = 0;
    uint32_t eu = 0;   // ESM: valid tiles consumed so far
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tl) {
      const TileInfo ti = persist_tile(p, t);
      const int a = tl & 1;
      if (!mbar_wait_idle(smem_u32(&bar_tfull[a]), (tl >> 1) & 1, &s_abort)) break;
      tc_fence_after();
      bool eok = true;
      if (ESM && ti.ok) {
        // two phases, one per 64-column half; this warp takes 32 columns of each
        for (int h = 0; h < 2 && eok; ++h) {
          const uint32_t v = 2 * eu + h;
          const int b = v & 1;
          eok = mbar_wait(smem_u32(&bar_efull[b]), (v >> 1) & 1, &s_abort);
          if (!eok) break;
          epi_tile<T, EPI, ESM>(p, ti, tmem + lane_base + a * 256, q, h, lane, alpha, beta, sums,
                                smem + SOFF + (warp - 2) * tcp::SCR_WARP,
                                smem + EOFF + b * tcp::EH_BYTES, 2 * half, 2 * half + 2);
          fence_proxy_async_smem();   // this thread's stage writes, visible to the TMA store
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&bar_odone[b]));
        }
        ++eu;
      } else {
        epi_tile<T, EPI, ESM>(p, ti, tmem + lane_base + a * 256, q, half, lane, alpha, beta, sums,
                              smem + SOFF + (warp - 2) * tcp::SCR_WARP, nullptr);
      }
      tc_fence_before();  // our TMEM reads are ordered before the release below
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bar_tempty[a]));
      if (!eok) break;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, tcp::TMEM_COLS);
  if (s_abort && threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
  if (p.out) __threadfence();
  publish_and_finalize(p, sums, red, &s_flag);
}

// ---------------------------------------------------------------------------------
// Paired-CTA SP2 step (cta_group::2) for dense sizes that are multiples of 256.
// A cluster of two CTAs computes one 256 x 128 output tile per work item with M = 256
// MMAs: each CTA stages its own 128 rows of A and one 64-row half of B, so a CTA moves
// 48 KB per 64-wide k-block instead of 64 KB and its MMAs read 6 KB of shared memory per
// 128 x 128 x 16 slice instead of 8 KB.  CTA 0 of the pair issues the MMAs and owns the
// operand-full barriers (both CTAs' tile loads complete on them); the MMA commits arrive
// on the stage-free and accumulator-full barriers of both CTAs; the epilogue warps of
// both CTAs arrive on CTA 0's accumulator-empty barrier.  Each CTA runs the same
// epilogue as the single-CTA kernel on its own 128 x 128 block (TMEM double-buffered).
// Work item w = {bi2, bj}: rows 256 bi2 .. +255, columns 128 bj .. +127, bj >= 2 bi2; the
// block of CTA 1 is skipped by its epilogue when it lies below the diagonal.
// ANTI: the anticommutator {G, X} = G X + X G of two symmetric matrices as one symmetric
// product over the concatenated K range, [G | X] [X | G]^T: the K loop runs twice over
// the columns, the second time with the operands' roles swapped (tm_a2* holds X in the
// A role, tm_b2* G in the B role), so the one accumulator sums both products.
// ES (SP2 epilogue, E = A: launches of at most one tile per pair): the producer also
// brings the CTA's 128 x 128 block of E = X_k (or G) into shared memory by TMA while the
// K loop runs, in place of the fourth operand stage, and the epilogue reads it there
// instead of from global memory (with one tile per CTA the epilogue is not hidden behind
// a next tile's products, and its per-row reads from L2 were its latency).
// ---------------------------------------------------------------------------------
namespace tcq {
constexpr int BH = 64;                                  // B rows staged per CTA (N / 2)
constexpr int A_BYTES = tc::BM * tc::BK * 2;            // 16 KB
constexpr int BH_BYTES = BH * tc::BK * 2;               // 8 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * BH_BYTES; // 48 KB
constexpr int ST = 4;
constexpr int SCR_OFF = ST * STAGE_BYTES;
constexpr int SMEM_BYTES = SCR_OFF + tcp::EPI_WARPS * tcp::SCR_WARP + 1024;
// single-wave form with the X_k block staged: three operand stages, the epilogue scratch,
// then the CTA's 128 x 128 block of X_k (hi and lo, two 64-column halves)
constexpr int ST_ES = 3;
constexpr int SCR_OFF_ES = ST_ES * STAGE_BYTES;
constexpr int E_OFF_ES = SCR_OFF_ES + tcp::EPI_WARPS * tcp::SCR_WARP;
constexpr int E_BYTES_ES = 4 * tc::TILE_BYTES;
constexpr int SMEM_BYTES_ES = E_OFF_ES + E_BYTES_ES + 1024;
// 227 KB of shared memory per block on sm_100, less the kernel's ~1.2 KB of static
// shared memory (barriers, the reduction array)
static_assert(SMEM_BYTES <= 232448 - 1536 && SMEM_BYTES_ES <= 232448 - 1536,
              "paired kernel: shared memory beyond the per-block limit");
}  // namespace tcq

template <typename T, int EPI, bool ANTI = false, bool ES = false>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(tcp::NTHR, 1)
    k_tc_pair(const __grid_constant__ CUtensorMap tm_ahi, const __grid_constant__ CUtensorMap tm_alo,
              const __grid_constant__ CUtensorMap tm_bhi, const __grid_constant__ CUtensorMap tm_blo,
              const __grid_constant__ CUtensorMap tm_a2hi, const __grid_constant__ CUtensorMap tm_a2lo,
              const __grid_constant__ CUtensorMap tm_b2hi, const __grid_constant__ CUtensorMap tm_b2lo,
              const StepArgs p, const int2* __restrict__ ptiles, int ntiles) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full[tcq::ST];
  __shared__ __align__(8) uint64_t bar_empty[tcq::ST];
  __shared__ __align__(8) uint64_t bar_tfull[2];
  __shared__ __align__(8) uint64_t bar_tempty[2];
  __shared__ __align__(8) uint64_t bar_final;
  __shared__ __align__(8) uint64_t bar_e;
  __shared__ uint32_t tmem_holder;
  __shared__ double red[32 * 4];
  __shared__ int s_flag;
  __shared__ volatile int s_abort;
  constexpr int ST = ES ? tcq::ST_ES : tcq::ST;   // operand stages
  if (ES && ntiles > (int)(gridDim.x >> 1)) {        // one tile per pair (uniform exit)
    if (threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
    return;
  }

  double alpha = p.alpha, beta = p.beta;
  if (EPI == 0 && p.control) {
    // the decision is the same in every CTA, so both CTAs of a pair leave together
    const int br = control_prologue(p);
    if (br < 0) return;
    if (br == BR_X2) { alpha = 1.0; beta = 0.0; }
    else { alpha = -1.0; beta = 2.0; }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < ST; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    mbar_init(smem_u32(&bar_e), 1);
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&bar_tfull[a]), 1);
      mbar_init(smem_u32(&bar_tempty[a]), 2 * tcp::EPI_WARPS);
    }
    mbar_init(smem_u32(&bar_final), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc_pair(smem_u32(&tmem_holder), tcp::TMEM_COLS);
  tc_fence_before();
  cluster_sync();   // barriers and TMEM of both CTAs exist before either uses the other's
  tc_fence_after();
  const uint32_t tmem = tmem_holder;
  const int KB = p.np / tc::BK;
  const int KBT = ANTI ? 2 * KB : KB;   // K-blocks per tile
  double sums[4] = {0.0, 0.0, 0.0, 0.0};

  if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer (both CTAs) ----------------
      bool ok = true, e_issued = false;
      uint32_t g = 0;
      for (int w = pair; w < ntiles && ok; w += npairs) {
        const int2 tile = ptiles[w];
        const int ra = tile.x * 2 * tc::BM + (int)rank * tc::BM;
        const int rb = tile.y * tc::BN + (int)rank * tcq::BH;
        for (int kb = 0; kb < KBT; ++kb, ++g) {
          const int s = g % ST;
          const uint32_t u = g / ST;
          if (g >= (uint32_t)ST && !mbar_wait(smem_u32(&bar_empty[s]), (u - 1) & 1, &s_abort)) {
            ok = false;
            break;
          }
          const uint32_t fb0 = map_to_rank(smem_u32(&bar_full[s]), 0);
          if (rank == 0) mbar_expect_tx(smem_u32(&bar_full[s]), 2 * tcq::STAGE_BYTES);
          const uint32_t st = sbase + s * tcq::STAGE_BYTES;
          const bool sw = ANTI && kb >= KB;    // second pass: roles swapped
          const int kc = (sw ? kb - KB : kb) * tc::BK;
          tma_load_2d_pair(st, sw ? &tm_a2hi : &tm_ahi, fb0, kc, ra);
          tma_load_2d_pair(st + tcq::A_BYTES, sw ? &tm_a2lo : &tm_alo, fb0, kc, ra);
          tma_load_2d_pair(st + 2 * tcq::A_BYTES, sw ? &tm_b2hi : &tm_bhi, fb0, kc, rb);
          tma_load_2d_pair(st + 2 * tcq::A_BYTES + tcq::BH_BYTES, sw ? &tm_b2lo : &tm_blo, fb0, kc,
                           rb);
          if (ES && kb == 0 && !e_issued) {
            // this CTA's block of E (= A): rows ra.., columns 128 bj.., two 64-column halves
            e_issued = true;
            const uint32_t eb = smem_u32(&bar_e);
            const uint32_t es = sbase + tcq::E_OFF_ES;
            mbar_expect_tx(eb, tcq::E_BYTES_ES);
            for (int h = 0; h < 2; ++h) {
              tma_load_2d(es + h * 2 * tc::TILE_BYTES, &tm_ahi, eb, tile.y * tc::BN + h * 64, ra);
              tma_load_2d(es + h * 2 * tc::TILE_BYTES + tc::TILE_BYTES, &tm_alo, eb,
                          tile.y * tc::BN + h * 64, ra);
            }
          }
        }
      }
      if (!ok) s_abort = 1;
      if (ES && e_issued)   // the block copy lands before this CTA can leave
        for (uint32_t i = 0; i < kSpinLimit; ++i)
          if (mbar_try(smem_u32(&bar_e), 0)) break;
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---------------- MMA issuer (CTA 0 of the pair) ----------------
      constexpr uint32_t idesc = make_idesc(SplitTraits<T>::kFmt, 2 * tc::BM, tc::BN);
      bool ok = true;
      uint32_t g = 0, tl = 0;
      for (int w = pair; w < ntiles && ok; w += npairs, ++tl) {
        const int a = tl & 1;
        const uint32_t v = tl >> 1;
        if (tl >= 2 && !mbar_wait(smem_u32(&bar_tempty[a]), (v - 1) & 1, &s_abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t acc_hh = tmem + a * 256, acc_x = tmem + a * 256 + tc::BN;
        for (int kb = 0; kb < KBT; ++kb, ++g) {
          const int s = g % ST;
          if (!mbar_wait(smem_u32(&bar_full[s]), (g / ST) & 1, &s_abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t st = sbase + s * tcq::STAGE_BYTES;
          const uint64_t d_ahi = sw128_desc(st);
          const uint64_t d_alo = sw128_desc(st + tcq::A_BYTES);
          const uint64_t d_bhi = sw128_desc(st + 2 * tcq::A_BYTES);
          const uint64_t d_blo = sw128_desc(st + 2 * tcq::A_BYTES + tcq::BH_BYTES);
#pragma unroll
          for (int kk = 0; kk < tc::BK / tc::UK; ++kk) {
            const uint64_t off = (uint64_t)((kk * tc::UK * 2) >> 4);
            const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
            umma_f16_pair(acc_hh, d_ahi + off, d_bhi + off, idesc, acc);
            umma_f16_pair(acc_x, d_ahi + off, d_blo + off, idesc, acc);
            umma_f16_pair(acc_x, d_alo + off, d_bhi + off, idesc, 1u);
          }
          umma_commit_pair_mc(smem_u32(&bar_empty[s]), (uint16_t)0x3);
        }
        if (!ok) break;
        umma_commit_pair_mc(smem_u32(&bar_tfull[a]), (uint16_t)0x3);
      }
      umma_commit_pair(smem_u32(&bar_final));
      for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try(smem_u32(&bar_final), 0)) break;
      if (!ok) s_abort = 1;
    }
    __syncwarp();
  } else {
    // ---------------- epilogue (8 warps in each CTA) ----------------
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    const uint32_t tempty0[2] = {map_to_rank(smem_u32(&bar_tempty[0]), 0),
                                 map_to_rank(smem_u32(&bar_tempty[1]), 0)};
    uint32_t tl = 0;
    for (int w = pair; w < ntiles; w += npairs, ++tl) {
      const int2 tile = ptiles[w];
      const int a = tl & 1;
      if (!mbar_wait_idle(smem_u32(&bar_tfull[a]), (tl >> 1) & 1, &s_abort)) break;
      tc_fence_after();
      TileInfo ti;
      const int brow = tile.x * 2 + (int)rank;
      ti.row0 = 0;
      ti.i0 = brow * tc::BM;
      ti.j0 = tile.y * tc::BN;
      ti.kb = KB;
      ti.core = p.core;
      ti.ok = brow <= tile.y;        // CTA 1's block of a diagonal pair lies below it
      ti.diag = brow == tile.y;
      if (ES && !mbar_wait_idle(smem_u32(&bar_e), 0, &s_abort)) break;
      epi_tile<T, EPI, false, ES>(p, ti, tmem + lane_base + a * 256, q, half, lane, alpha, beta,
                                  sums,
                                  smem + (ES ? tcq::SCR_OFF_ES : tcq::SCR_OFF) +
                                      (warp - 2) * tcp::SCR_WARP,
                                  ES ? smem + tcq::E_OFF_ES + half * 2 * tc::TILE_BYTES : nullptr);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(tempty0[a]);
    }
  }
  tc_fence_before();
  cluster_sync();   // every MMA retired (CTA 0 waited), every epilogue done in both CTAs
  tc_fence_after();
  if (warp == 1) tmem_dealloc_pair(tmem, tcp::TMEM_COLS);
  if (s_abort && threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
  if (p.out) __threadfence();
  publish_and_finalize(p, sums, red, &s_flag);
}

// Failure-path self-test: every thread waits, with the same bounded wait the step
// kernels use, on an mbarrier that nothing ever arrives at.  The wait runs out after
// `limit` polls, the kernel records SP2B_TIMEOUT and returns normally.
__global__ void k_wait_selftest(uint32_t limit, int* err) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ volatile int abort_flag;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    mbar_init(smem_u32(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const bool ok = mbar_wait_limit(smem_u32(&bar), 0, &abort_flag, limit);
  __syncthreads();
  if (!ok && threadIdx.x == 0) atomicExch(err, SP2B_TIMEOUT);
}

cudaError_t launch_wait_selftest(uint32_t limit, int* err, cudaStream_t st) {
  k_wait_selftest<<<1, 64, 0, st>>>(limit, err);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Elementwise kernels of the split path
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void k_normalize_split(const double* __restrict__ h, int n, int ld, int np,
                                  const double* __restrict__ bounds, T* __restrict__ hi,
                                  T* __restrict__ lo, double* partials, unsigned* counter,
                                  SP2Rec* rec0, double* norm_out) {
  using TR = SplitTraits<T>;
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
    alignas(16) T a8[8], b8[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int c = c0 + e;
      const double v = (r < n && c < n) ? alpha * h[(size_t)r * ld + c] + (r == c ? beta : 0.0) : 0.0;
      const T a = TR::from_d(v);
      const T b = TR::from_d((v - TR::to_d(a)) * TR::kScale);
      a8[e] = a;
      b8[e] = b;
      const double vs = TR::to_d(a) + TR::kInv * TR::to_d(b);
      s[0] += vs * vs;
      if (r == c) s[1] += vs;
    }
    *reinterpret_cast<uint4*>(hi + (size_t)r * np + c0) = *reinterpret_cast<const uint4*>(a8);
    *reinterpret_cast<uint4*>(lo + (size_t)r * np + c0) = *reinterpret_cast<const uint4*>(b8);
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

template <typename T>
__global__ void k_split_to_f64(const T* __restrict__ hi, const T* __restrict__ lo, size_t total,
                               double* __restrict__ x) {
  using TR = SplitTraits<T>;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = TR::to_d(hi[i]) + TR::kInv * TR::to_d(lo[i]);
}

__global__ void k_f32_to_split(const float* __restrict__ a, int n, int np, __half* __restrict__ hi,
                               __half* __restrict__ lo) {
  using TR = SplitTraits<__half>;
  const size_t total = (size_t)np * np;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / np), c = (int)(idx % np);
    const double v = (r < n && c < n) ? (double)a[(size_t)r * n + c] : 0.0;
    const __half h = TR::from_d(v);
    hi[idx] = h;
    lo[idx] = TR::from_d((v - TR::to_d(h)) * TR::kScale);
  }
}

// An m x n FP32 row panel into the padded mp x np hi/lo split (zeros outside).
__global__ void k_f32_rows_to_split(const float* __restrict__ a, int m, int n, int mp, int np,
                                    __half* __restrict__ hi, __half* __restrict__ lo) {
  using TR = SplitTraits<__half>;
  const size_t total = (size_t)mp * np;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / np), c = (int)(idx % np);
    const double v = (r < m && c < n) ? (double)a[(size_t)r * n + c] : 0.0;
    const __half h = TR::from_d(v);
    hi[idx] = h;
    lo[idx] = TR::from_d((v - TR::to_d(h)) * TR::kScale);
  }
}

// ---------------------------------------------------------------------------------
// Host side: tensor maps and launches
// ---------------------------------------------------------------------------------
int tc_ntiles(int np) {
  const int t = np / tc::BM;
  return t * (t + 1) / 2;
}

template <typename T, bool SYM>
static cudaError_t launch_tc(const StepArgs& a, long long rows, dim3 grid, float* plain_out,
                             int plain_n, cudaStream_t st) {
  const bool bf16 = std::is_same<T, __nv_bfloat16>::value;
  CUtensorMap m[4];
  if (!make_tmap(&m[0], a.A, rows, a.ld, a.ld, bf16) ||
      !make_tmap(&m[1], a.A_lo, rows, a.ld, a.ld, bf16) ||
      !make_tmap(&m[2], a.B, rows, a.ld, a.ld, bf16) ||
      !make_tmap(&m[3], a.B_lo, rows, a.ld, a.ld, bf16))
    return cudaErrorInvalidValue;
  auto kern = k_tc_gemm<T, SYM>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  kern<<<grid, 128, tc::SMEM_BYTES, st>>>(m[0], m[1], m[2], m[3], a, plain_out, plain_n);
  note_launch();
  return cudaGetLastError();
}

static int num_sms() {
  static int sms = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
      sms = v;
    if (sms <= 0) sms = 148;
  });
  return sms;
}

template <typename T, int EPI, bool ESM = false>
static cudaError_t launch_persist(const StepArgs& a, long long rows, int ntiles, cudaStream_t st) {
  const bool bf16 = std::is_same<T, __nv_bfloat16>::value;
  CUtensorMap m[4];
  if (!make_tmap(&m[0], a.A, rows, a.ld, a.ld, bf16) || !make_tmap(&m[1], a.A_lo, rows, a.ld, a.ld, bf16))
    return cudaErrorInvalidValue;
  if (a.B == a.A && a.B_lo == a.A_lo) {
    m[2] = m[0];
    m[3] = m[1];
  } else if (!make_tmap(&m[2], a.B, rows, a.ld, a.ld, bf16) ||
             !make_tmap(&m[3], a.B_lo, rows, a.ld, a.ld, bf16)) {
    return cudaErrorInvalidValue;
  }
  CUtensorMap mo[2] = {m[0], m[1]};
  if (ESM && (!make_tmap(&mo[0], a.out, rows, a.ld, a.ld, bf16) ||
              !make_tmap(&mo[1], a.out_lo, rows, a.ld, a.ld, bf16)))
    return cudaErrorInvalidValue;
  auto kern = k_tc_persist<T, EPI, ESM>;
  const int smem = ESM ? tcp::SMEM_BYTES_E : tcp::SMEM_BYTES;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  const int grid = std::min(ntiles, num_sms());
  kern<<<grid, ESM ? tcp::NTHR_E : tcp::NTHR, smem, st>>>(m[0], m[1], m[2], m[3], mo[0], mo[1], a,
                                                          ntiles);
  note_launch();
  return cudaGetLastError();
}

// Upper 128 x 128 tiles of an np x np product in panels of kPanel tile columns; inside a
// panel the row blocks run top to bottom.  The ~148 tiles of one wave of the persistent
// grid then share ~148/kPanel row blocks of A and kPanel of B, whose K-slices stay in L2,
// where the plain column order touches every row block of X in each wave.  One list per
// (device, np), built on first use; none while the stream is being captured.
constexpr int kPanel = 12;
void panel_tile_order(int nb, int panel, std::vector<int2>& out) {
  out.clear();
  for (int p0 = 0; p0 < nb; p0 += panel) {
    const int p1 = std::min(nb, p0 + panel);
    for (int bi = 0; bi < p1; ++bi)
      for (int bj = std::max(bi, p0); bj < p1; ++bj) out.push_back(make_int2(bi, bj));
  }
}

static const int4* dense_tiles(int np, cudaStream_t st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  static std::mutex mu;
  static std::map<std::pair<int, int>, int4*> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({dev, np});
  if (it != cache.end()) return it->second;
  // a new list needs an allocation and a copy, neither of which a stream capture allows
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return nullptr;
  std::vector<int2> order;
  panel_tile_order(np / tc::BM, kPanel, order);
  std::vector<int4> t(order.size());
  for (size_t i = 0; i < order.size(); ++i)
    t[i] = make_int4(0, (order[i].x << 16) | order[i].y, np, -2);
  int4* d = nullptr;
  if (cudaMalloc((void**)&d, t.size() * sizeof(int4)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  cache[{dev, np}] = d;
  return d;
}

// Work items of the paired kernel, {bi2, bj} with bj >= 2 bi2, in panels of kPanel column
// blocks (row pairs top to bottom inside a panel).  Cached per (device, np).
void pair_tile_order(int nb, int panel, std::vector<int2>& out) {
  out.clear();
  for (int p0 = 0; p0 < nb; p0 += panel) {
    const int p1 = std::min(nb, p0 + panel);
    for (int bi2 = 0; 2 * bi2 < p1; ++bi2)
      for (int bj = std::max(2 * bi2, p0); bj < p1; ++bj) out.push_back(make_int2(bi2, bj));
  }
}

static const int2* pair_tiles(int np, cudaStream_t st, int* count) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::pair<int2*, int>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({dev, np});
  if (it != cache.end()) {
    *count = it->second.second;
    return it->second.first;
  }
  // a new list needs an allocation and a copy, neither of which a stream capture allows
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
    return nullptr;
  std::vector<int2> t;
  pair_tile_order(np / tc::BM, kPanel, t);
  int2* d = nullptr;
  if (cudaMalloc((void**)&d, t.size() * sizeof(int2)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(d, t.data(), t.size() * sizeof(int2), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  cache[{dev, np}] = {d, (int)t.size()};
  *count = (int)t.size();
  return d;
}

// Clusters of the paired kernel that can be resident at once (one CTA per SM).
template <typename T, int EPI, bool ANTI = false, bool ES = false>
static int pair_clusters() {
  static int per_dev[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return num_sms() / 2;
  if (per_dev[dev] > 0) return per_dev[dev];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(num_sms() & ~1, 1, 1);
  cfg.blockDim = dim3(tcp::NTHR, 1, 1);
  cfg.dynamicSmemBytes = ES ? tcq::SMEM_BYTES_ES : tcq::SMEM_BYTES;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = 2;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (void*)k_tc_pair<T, EPI, ANTI, ES>, &cfg) !=
          cudaSuccess ||
      n <= 0) {
    cudaGetLastError();
    n = ES ? 0 : num_sms() / 2;   // the staged form is used only where it is known to fit
  }
  per_dev[dev] = n;
  return n;
}

// Paired-CTA launch for np a multiple of 256; returns cudaErrorNotSupported when the
// caller should use the single-CTA kernel instead.  ANTI: A = G, B = X (see k_tc_pair).
template <typename T, int EPI, bool ANTI = false>
static cudaError_t launch_pair(const StepArgs& a, cudaStream_t st) {
  if (a.np % (2 * tc::BM) != 0 || a.ld != a.np) return cudaErrorNotSupported;
  int ntiles = 0;
  const int2* tl = pair_tiles(a.np, st, &ntiles);
  if (!tl || ntiles <= 0) return cudaErrorNotSupported;
  const int type = std::is_same<T, __nv_bfloat16>::value ? TMAP_BF16 : TMAP_F16;
  CUtensorMap m[8];
  if (!make_tmap_box(&m[0], a.A, a.np, a.np, a.np, type, tc::BM) ||
      !make_tmap_box(&m[1], a.A_lo, a.np, a.np, a.np, type, tc::BM) ||
      !make_tmap_box(&m[2], a.B, a.np, a.np, a.np, type, tcq::BH) ||
      !make_tmap_box(&m[3], a.B_lo, a.np, a.np, a.np, type, tcq::BH))
    return cudaErrorInvalidValue;
  if (ANTI) {
    if (!make_tmap_box(&m[4], a.B, a.np, a.np, a.np, type, tc::BM) ||
        !make_tmap_box(&m[5], a.B_lo, a.np, a.np, a.np, type, tc::BM) ||
        !make_tmap_box(&m[6], a.A, a.np, a.np, a.np, type, tcq::BH) ||
        !make_tmap_box(&m[7], a.A_lo, a.np, a.np, a.np, type, tcq::BH))
      return cudaErrorInvalidValue;
  } else {
    for (int i = 0; i < 4; ++i) m[4 + i] = m[i];   // unused
  }
  // one tile per pair (a single wave): the X_k block staged for the epilogue (the
  // shared-memory limit is raised before the residency query counts the clusters)
  if (EPI == 0 && a.E == a.A && a.E_lo == a.A_lo && ntiles <= num_sms() / 2) {
    auto kes = k_tc_pair<T, EPI, ANTI, true>;
    if (cudaFuncSetAttribute(kes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tcq::SMEM_BYTES_ES) == cudaSuccess &&
        ntiles <= pair_clusters<T, EPI, ANTI, true>()) {
      kes<<<2 * ntiles, tcp::NTHR, tcq::SMEM_BYTES_ES, st>>>(m[0], m[1], m[2], m[3], m[4], m[5],
                                                             m[6], m[7], a, tl, ntiles);
      note_launch();
      return cudaGetLastError();
    }
    (void)cudaGetLastError();
  }
  auto kern = k_tc_pair<T, EPI, ANTI>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, tcq::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  const int clusters = std::min(ntiles, pair_clusters<T, EPI, ANTI>());
  kern<<<2 * clusters, tcp::NTHR, tcq::SMEM_BYTES, st>>>(m[0], m[1], m[2], m[3], m[4], m[5], m[6],
                                                         m[7], a, tl, ntiles);
  note_launch();
  return cudaGetLastError();
}

// Symmetric launches: A = B (the iterate), so one pair of tensor maps serves both.
cudaError_t launch_sym_gemm_tc(const StepArgs& a0, int bf16, cudaStream_t st) {
  if (a0.np % tc::BM != 0 || a0.A != a0.B || a0.A_lo != a0.B_lo) return cudaErrorInvalidValue;
  StepArgs a = a0;
  a.tiles = nullptr;
  a.ld = a.np;
  cudaError_t e = bf16 ? launch_pair<__nv_bfloat16, 0>(a, st) : launch_pair<__half, 0>(a, st);
  if (e != cudaErrorNotSupported) return e;
  a.tiles = dense_tiles(a.np, st);   // nullptr: plain column order
  const int nt = tc_ntiles(a.np);
  return bf16 ? launch_persist<__nv_bfloat16, 0>(a, a.np, nt, st)
              : launch_persist<__half, 0>(a, a.np, nt, st);
}

// {G, X} on the upper tiles, out = alpha {G, X} + beta E (E = G for the adjoint step):
// a.A / a.A_lo = G, a.B / a.B_lo = X.  cudaErrorNotSupported when np is not a multiple
// of 256 (the caller forms G X with launch_tc_plain and combines).
cudaError_t launch_anti_tc(const StepArgs& a0, cudaStream_t st) {
  if (a0.np % tc::BM != 0) return cudaErrorInvalidValue;
  StepArgs a = a0;
  a.tiles = nullptr;
  a.ld = a.np;
  return launch_pair<__half, 0, true>(a, st);
}

cudaError_t launch_sym_gemm_tc_batched(const StepArgs& a, long long rows, int bf16,
                                       cudaStream_t st) {
  if (!a.tiles || a.ntiles <= 0 || a.ld % tc::BM != 0 || rows % tc::BM != 0 || a.A != a.B ||
      a.A_lo != a.B_lo)
    return cudaErrorInvalidValue;
  return bf16 ? launch_persist<__nv_bfloat16, 0, true>(a, rows, a.ntiles, st)
              : launch_persist<__half, 0, true>(a, rows, a.ntiles, st);
}

// McWeeny combine of the INT8 refinement: D = 2 X^2 - X (4R), upper tiles, mirrored.
cudaError_t launch_mcweeny_tc(const __half* xhi, const __half* xlo, const __half* rhi,
                              const __half* rlo, const double* x2, int np, int bf16, double* d,
                              int n, int ldd, double* partials, unsigned* counter,
                              double* sums_out, int* err, cudaStream_t st) {
  if (np % tc::BM != 0 || n > np) return cudaErrorInvalidValue;
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.A = xhi;
  a.A_lo = xlo;
  a.B = rhi;
  a.B_lo = rlo;
  a.E = x2;
  a.out = d;
  a.np = np;
  a.ld = np;
  a.n_out = n;
  a.ld_out = ldd;
  a.partials = partials;
  a.counter = counter;
  a.sums_out = sums_out;
  a.err = err;
  cudaError_t e = bf16 ? launch_pair<__nv_bfloat16, 1>(a, st) : launch_pair<__half, 1>(a, st);
  if (e != cudaErrorNotSupported) return e;
  a.tiles = dense_tiles(np, st);
  const int nt = tc_ntiles(np);
  return bf16 ? launch_persist<__nv_bfloat16, 1>(a, np, nt, st)
              : launch_persist<__half, 1>(a, np, nt, st);
}

cudaError_t launch_tc_plain(const __half* ahi, const __half* alo, const __half* bhi,
                            const __half* blo, int np, float* c, int n, cudaStream_t st,
                            int* err) {
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.A = ahi;
  a.A_lo = alo;
  a.B = bhi;
  a.B_lo = blo;
  a.np = np;
  a.ld = np;
  a.err = err;
  dim3 grid(np / tc::BN, np / tc::BM);
  return launch_tc<__half, false>(a, np, grid, c, n, st);
}

// Row panel C (m x n, row pitch n) = A_rows B^T from split operands: A over mp rows, B over
// np rows (both with row pitch np, K = np); one CTA per 128 x 128 tile of the panel.
cudaError_t launch_tc_panel(const __half* ahi, const __half* alo, int mp, const __half* bhi,
                            const __half* blo, int np, float* c, int m, int n, cudaStream_t st,
                            int* err) {
  if (mp % tc::BM != 0 || np % tc::BN != 0 || m > mp || n > np || m <= 0 || n <= 0)
    return cudaErrorInvalidValue;
  StepArgs a;
  memset(&a, 0, sizeof(a));
  a.np = np;
  a.ld = np;
  a.n_out = m;
  a.err = err;
  CUtensorMap mm[4];
  if (!make_tmap(&mm[0], ahi, mp, np, np, false) || !make_tmap(&mm[1], alo, mp, np, np, false) ||
      !make_tmap(&mm[2], bhi, np, np, np, false) || !make_tmap(&mm[3], blo, np, np, np, false))
    return cudaErrorInvalidValue;
  auto kern = k_tc_gemm<__half, false>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  kern<<<dim3(np / tc::BN, mp / tc::BM), 128, tc::SMEM_BYTES, st>>>(mm[0], mm[1], mm[2], mm[3], a,
                                                                    c, n);
  note_launch();
  return cudaGetLastError();
}

static int ew_grid(size_t total) {
  size_t g = (total + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  return (int)(g ? g : 1);
}

cudaError_t launch_normalize_split(const double* h, int n, int ld, int np,
                                   const double* bounds, __half* hi, __half* lo, int bf16,
                                   double* partials, unsigned* counter, SP2Rec* rec0,
                                   double* norm_out, cudaStream_t st) {
  const int g = ew_grid((size_t)np * np);
  if (bf16)
    k_normalize_split<__nv_bfloat16><<<g, 256, 0, st>>>(
        h, n, ld, np, bounds, (__nv_bfloat16*)hi, (__nv_bfloat16*)lo, partials, counter, rec0,
        norm_out);
  else
    k_normalize_split<__half><<<g, 256, 0, st>>>(h, n, ld, np, bounds, hi, lo, partials, counter,
                                                 rec0, norm_out);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_split_to_f64(const __half* hi, const __half* lo, int np, int bf16, double* x,
                                cudaStream_t st) {
  const size_t total = (size_t)np * np;
  if (bf16)
    k_split_to_f64<__nv_bfloat16><<<ew_grid(total), 256, 0, st>>>(
        (const __nv_bfloat16*)hi, (const __nv_bfloat16*)lo, total, x);
  else
    k_split_to_f64<__half><<<ew_grid(total), 256, 0, st>>>(hi, lo, total, x);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_f32_rows_to_split(const float* a, int m, int n, int mp, int np, __half* hi,
                                     __half* lo, cudaStream_t st) {
  k_f32_rows_to_split<<<ew_grid((size_t)mp * np), 256, 0, st>>>(a, m, n, mp, np, hi, lo);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_f32_to_split(const float* a, int n, int np, __half* hi, __half* lo,
                                cudaStream_t st) {
  k_f32_to_split<<<ew_grid((size_t)np * np), 256, 0, st>>>(a, n, np, hi, lo);
  note_launch();
  return cudaGetLastError();
}

}  // namespace sp2b
