// Batched sub-graph SP2 on the INT8 tensor cores with exact integer products ("INT8
// digit split"): every step of every part in one persistent launch (k_i8_steps).
//
// The iterate is held in fixed point, shifted so that every entry fits the same range:
// X' = X - I/2 has its spectrum in [-1/2, 1/2] (Gershgorin-normalised X has it in [0, 1]),
// so |X'_ij| <= 1/2 and M = rint(2^31 X') is an integer with |M| <= 2^30.  M is stored
// as four balanced base-256 digits,
//     M = d0 2^24 + d1 2^16 + d2 2^8 + d3,   d1, d2, d3 in [-128, 127], |d0| <= 65,
// in four signed 8-bit planes.  Then 2^62 X'^2 = sum_{s,t} (D_s D_t) 2^{48 - 8(s+t)}, and
// every plane product D_s D_t is exact in the 32-bit accumulators (|d| <= 128 and at most
// four products per accumulator: |A_u| < 2^16 K <= 2^31 for any part size K <= 32768).
// Products are grouped by u = s + t into five accumulators A_u (u = 0..4: thirteen
// products); the three terms with u >= 5 lie below 2^-36 (typical) and are dropped.  The
// epilogue rounds P = 2^46 X'^2 = sum_u A_u 2^{32 - 8u} to Q = rint(2^31 X'^2) exactly
// with 32-bit integer steps and applies the SP2 branch in the shifted variable,
//     X^2 branch:      X'_{k+1} = X'^2 + X' - I/4,
//     2X - X^2 branch: X'_{k+1} = X' - X'^2 + I/4,
// as M_{k+1} = M_k +- rint(2^31 X'^2) -+ 2^29 [i == j].  The only rounding per step is
// that of X'^2 to the 2^-31 grid: the recursion follows the FP64 one to ~1e-9 of the
// entries, which keeps the near-gapless lattice parts within 1e-7 relative Frobenius of
// the FP64 batch where the FP16 hi + lo products (22 significant bits, accumulations
// truncated toward zero) end ~1e-5 away.  The residual (X - X^2) = I/4 - X'^2 of the
// prg_sp2_submatrix bookkeeping (src/prg_sp2_mod.F90:1286-1291) comes from the same P.
//
// Layout: the four planes of a ping-pong buffer are four packed R x ld byte arrays
// (plane s at base + s R ld), so one TMA map over 4R rows covers them all.  Tiles are
// 128 rows x 64 columns (the five accumulators take 5 x 64 TMEM columns) of the upper
// part of each part's block, {row0, bi << 16 | bj64, K extent, core rows}, with the K
// extent n64 = the part size rounded up to 64 and no tile starting at or beyond it.
// Padding rows and columns hold X = 0, i.e. X' = -I/2 on the padding diagonal; the
// recursion keeps that for indices below n64 (their own square is in the K range), and
// products with them add nothing to real entries (their off-diagonal entries stay 0).
// Entries at or beyond n64 only reach output rows at or beyond n64, which nothing reads.
// Only the tiles' entries are stored (the upper band: row r from column r & ~127 on);
// operand blocks left of it are read from their mirrors, transposed by the MMA.
#include "kernels_subgraph.cuh"
#include "reduce.cuh"
#include "tc_ptx.cuh"

namespace sp2b {
namespace i8s {
constexpr int BM = 128;                         // tile rows (TMEM lanes)
constexpr int BN = 64;                          // tile columns
constexpr int BK = 64;                          // K bytes per stage (64-byte swizzle)
constexpr int UK = 32;                          // K per kind::i8 MMA
constexpr int ND = 4;                           // digit planes
constexpr int NU = 5;                           // accumulators, u = s + t = 0..4
constexpr int A_PLANE = BM * BK;                // 8 KB
constexpr int B_PLANE = BN * BK;                // 4 KB
constexpr int STAGE_BYTES = ND * (A_PLANE + B_PLANE);   // 48 KB
constexpr int ST = 3;
constexpr int EPI_WARPS = 16;                   // 4 lane quarters x 4 groups of 16 columns
constexpr int STORE_WARP = 2 + EPI_WARPS;       // TMA stores and completion signals
constexpr int NWARP = 3 + EPI_WARPS;
constexpr int NTHR = NWARP * 32;
constexpr int OUT_PLANE = BM * BN;              // 8 KB: one plane of the output tile
constexpr int OUT_BYTES = ND * OUT_PLANE;       // 32 KB: one staged tile (X_k in, X_{k+1} out)
constexpr int OUT_OFF = ST * STAGE_BYTES;       // two staged tiles (64-byte swizzle)
constexpr int SMEM_BYTES = OUT_OFF + 2 * OUT_BYTES + 1024;
static_assert(SMEM_BYTES <= 232448 - 1536, "INT8 steps: shared memory beyond the per-block limit");
constexpr int TMEM_COLS = 512;
static_assert(NU * BN <= TMEM_COLS, "the five accumulators fit the TMEM allocation");
}  // namespace i8s

// The thirteen plane products (s, t) with s + t <= 4, issued as seven MMAs: B planes t
// and t + 1 lie back to back in shared memory, so one N = 128 product of A plane s with
// them writes A_s B_t^T and A_s B_{t+1}^T into the adjacent accumulators u = s + t and
// u + 1.  MMA q multiplies A plane pa(q) by B planes pb(q).. (two if wide(q)); the first
// three, in this order, start the five accumulators at k = 0 (0-1, 2-3, 4).
__device__ __forceinline__ constexpr int i8_pa(int q) {
  return q == 0 ? 0 : q == 1 ? 0 : q == 2 ? 2 : q == 3 ? 1 : q == 4 ? 1 : q == 5 ? 2 : 3;
}
__device__ __forceinline__ constexpr int i8_pb(int q) {
  return q == 0 ? 0 : q == 1 ? 2 : q == 2 ? 2 : q == 3 ? 0 : q == 4 ? 2 : 0;
}
__device__ __forceinline__ constexpr bool i8_wide(int q) { return q != 2; }
__device__ __forceinline__ constexpr bool i8_first(int q) { return q <= 2; }

// Byte j (0..15) of a 16-byte register vector, sign-extended (j is a constant after
// unrolling, so this folds to one shift pair).
__device__ __forceinline__ int i8_byte(const uint4& v, int j) {
  const uint32_t w = (j >> 2) == 0 ? v.x : (j >> 2) == 1 ? v.y : (j >> 2) == 2 ? v.z : v.w;
  return (int)(int8_t)(uint8_t)(w >> (8 * (j & 3)));
}
__device__ __forceinline__ void i8_put(uint4& v, int j, int b) {
  const uint32_t m = (uint32_t)(uint8_t)b << (8 * (j & 3));
  if ((j >> 2) == 0) v.x |= m;
  else if ((j >> 2) == 1) v.y |= m;
  else if ((j >> 2) == 2) v.z |= m;
  else v.w |= m;
}

struct I8Tile {
  int row0, i0, j0, kb, core;
  bool ok;
};

__device__ __forceinline__ I8Tile i8_tile_v(int4 v) {
  I8Tile ti;
  ti.row0 = v.x;
  ti.i0 = (v.y >> 16) * i8s::BM;
  ti.j0 = (v.y & 0xffff) * i8s::BN;
  ti.core = v.w;
  ti.ok = ti.i0 < v.z && ti.j0 < v.z && v.z % i8s::BK == 0;   // z: K extent, multiple of 64
  ti.kb = ti.ok ? v.z / i8s::BK : 0;
  return ti;
}
__device__ __forceinline__ I8Tile i8_tile(const int4* tiles, int t) { return i8_tile_v(tiles[t]); }
// The same read by a whole warp and broadcast from lane 0 (warp-uniform fields).
__device__ __forceinline__ I8Tile i8_tile_uniform(const int4* tiles, int t) {
  int4 v = tiles[t];
  v.x = warp_uniform(v.x);
  v.y = warp_uniform(v.y);
  v.z = warp_uniform(v.z);
  v.w = warp_uniform(v.w);
  return i8_tile_v(v);
}

// Balanced base-256 digits of M (|M| < 2^31): d3, d2, d1 in [-128, 127], d0 the rest.
__device__ __forceinline__ void i8_digits(int m, int8_t& d0, int8_t& d1, int8_t& d2, int8_t& d3) {
  const int e3 = ((m + 128) & 255) - 128;
  m = (m - e3) >> 8;
  const int e2 = ((m + 128) & 255) - 128;
  m = (m - e2) >> 8;
  const int e1 = ((m + 128) & 255) - 128;
  m = (m - e1) >> 8;
  d0 = (int8_t)max(-127, min(127, m));
  d1 = (int8_t)e1;
  d2 = (int8_t)e2;
  d3 = (int8_t)e3;
}

__device__ __forceinline__ int i8_value(int8_t d0, int8_t d1, int8_t d2, int8_t d3) {
  return (((int)d0 * 256 + (int)d1) * 256 + (int)d2) * 256 + (int)d3;
}

// Tensor maps of the two digit buffers (index: buffer), each over its 4R rows.
struct I8Maps {
  CUtensorMap a[2];    // K-major operand and staged tile: 64 bytes x 128 rows, 64-byte swizzle
  CUtensorMap at[2];   // MN-major A^T: 128 bytes x 64 rows, 128-byte swizzle
  CUtensorMap b[2];    // B and B^T: 64 bytes x 64 rows, 64-byte swizzle
};

// Bounded wait until a counter in global memory reaches `target` (acquire).
__device__ __forceinline__ bool wait_count(const unsigned* c, unsigned target,
                                           volatile int* abort_flag) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(c) : "memory");
    if (v >= target) return true;
    if ((i & 63u) == 63u && *abort_flag) return false;
    __nanosleep(64);
  }
  *abort_flag = 1;
  return false;
}

// All SP2 steps of every part in one persistent launch: out = branch(in) in digit form,
// step after step, the two digit buffers alternating (step k reads buffer k & 1).
// warp 0: TMA producer (operands and each tile's X_k); warp 1: TMEM owner and MMA
// issuer; warps 2..17: epilogue (warp w reads TMEM lane quarter w & 3, columns
// 16 ((w - 2) >> 2)..); warp 18: TMA stores of the finished tiles and their signals.
//
// Work items are (step k, tile t) in step-major order; CTA c takes items c, c + G, ...
// A part's step-k tiles read only that part's step-(k-1) result, so the producer starts an
// item once every tile of its part has finished the previous step: done[part] counts
// finished tiles, signalled by the store warp once a tile's stores have landed (it waits
// on nothing but its own CTA's epilogue).  Every CTA finishes its items in increasing
// order and all CTAs are resident (cooperative launch), so the earliest unfinished item
// never waits on an unfinished one.
//
// Only the upper band of each part is stored: row r holds valid entries in the columns
// from its 128-row block's first row, c >= (r & ~127), which are exactly the entries of
// the tiles this kernel writes (bj >= 2 bi).  An operand block left of that (k-block
// before the block's first row) is read from its mirror X[k, i] = X[i, k] in MN-major
// form: A^T as a 64 x 128-byte box (128-byte swizzle), B^T as a 64 x 64-byte box.
// Each tile's X_k is loaded into one of two staging buffers (alternating per tile), the
// epilogue overwrites it in place with X_{k+1}, and four TMA stores (one per plane)
// write it back.
//
// Step sums (Tr X_{k+1}, ||X_k - X_k^2||_F^2 over the core rows, Tr X_k^2) are written per
// (step, CTA, epilogue warp) to partials and reduced in a fixed order by k_i8_step_sums.
__global__ void __launch_bounds__(i8s::NTHR, 1)
    k_i8_steps(const __grid_constant__ I8Maps maps, const I8StepsArgs p) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t bar_full[i8s::ST];
  __shared__ __align__(8) uint64_t bar_empty[i8s::ST];
  __shared__ __align__(8) uint64_t bar_tfull;
  __shared__ __align__(8) uint64_t bar_tempty;
  __shared__ __align__(8) uint64_t bar_final;
  __shared__ __align__(8) uint64_t bar_xk[2];      // X_k staged (producer's copy landed)
  __shared__ __align__(8) uint64_t bar_staged[2];  // X_{k+1} staged (all epilogue warps)
  __shared__ __align__(8) uint64_t bar_free[2];    // staging read by the stores
  __shared__ uint32_t tmem_holder;
  __shared__ volatile int s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const uint32_t sbase = smem_u32(smem);
  if (threadIdx.x == 0) {
    s_abort = 0;
    for (int s = 0; s < i8s::ST; ++s) {
      mbar_init(smem_u32(&bar_full[s]), 1);
      mbar_init(smem_u32(&bar_empty[s]), 1);
    }
    mbar_init(smem_u32(&bar_tfull), 1);
    mbar_init(smem_u32(&bar_tempty), i8s::EPI_WARPS);
    mbar_init(smem_u32(&bar_final), 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(smem_u32(&bar_xk[b]), 1);
      mbar_init(smem_u32(&bar_staged[b]), i8s::EPI_WARPS);
      mbar_init(smem_u32(&bar_free[b]), 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_holder), i8s::TMEM_COLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = (uint32_t)warp_uniform((int)tmem_holder);
  const int R = p.rows;
  const long long nitems = (long long)p.nsteps * p.ntiles;
  const int G = gridDim.x;
  // step and tile of item i
  auto item_of = [&](long long i, int& k, int& t) {
    k = (int)(i / p.ntiles);
    t = (int)(i - (long long)k * p.ntiles);
  };
  // staging buffer b of the output tiles
  auto stage_of = [&](int b) { return sbase + i8s::OUT_OFF + b * i8s::OUT_BYTES; };

  // The producer and MMA roles run warp-wide: tile data is broadcast from lane 0, so loop
  // bounds, descriptors and coordinates stay warp-uniform, and one elected lane issues.
  if (warp == 0) {
    // ---------------- TMA producer ----------------
    int issued_phase[i8s::ST];
    for (int s = 0; s < i8s::ST; ++s) issued_phase[s] = -1;
    int xk_phase[2] = {-1, -1};
    bool ok = true;
    uint32_t g = 0, tl = 0;
    for (long long i = blockIdx.x; i < nitems && ok; i += G, ++tl) {
      int k, t;
      item_of(i, k, t);
      const I8Tile ti = i8_tile_uniform(p.tiles, t);
      // an item of step k > 0 starts once its part has finished step k - 1
      bool dep = true;
      if (k > 0) {
        const int part = p.tpart[t];
        dep = wait_count(p.done + part, (unsigned)k * (unsigned)p.pnt[part], &s_abort);
      }
      ok = ti.ok && __all_sync(0xffffffffu, dep);
      if (!ok) break;
      fence_proxy_async_global();   // the other CTAs' results, then the async-proxy reads
      const CUtensorMap* ma = &maps.a[k & 1];
      const CUtensorMap* mat = &maps.at[k & 1];
      const CUtensorMap* mb = &maps.b[k & 1];
      const int jb = ti.j0 & ~(i8s::BM - 1);   // first row of the block holding B's rows
      for (int kb = 0; kb < ti.kb; ++kb, ++g) {
        const int s = g % i8s::ST;
        const uint32_t u = g / i8s::ST;
        if (g >= (uint32_t)i8s::ST && !mbar_wait_warp_idle(smem_u32(&bar_empty[s]), (u - 1) & 1, &s_abort)) {
          ok = false;
          break;
        }
        const int k0 = kb * i8s::BK;
        const bool at = k0 < ti.i0, bt = k0 < jb;
        const uint32_t fb = smem_u32(&bar_full[s]);
        const uint32_t st = sbase + s * i8s::STAGE_BYTES;
        if (elect_one()) {
          mbar_expect_tx(fb, i8s::STAGE_BYTES);
#pragma unroll
          for (int d = 0; d < i8s::ND; ++d) {
            const int pr = d * R + ti.row0;
            if (at)
              tma_load_2d(st + d * i8s::A_PLANE, mat, fb, ti.i0, pr + k0);
            else
              tma_load_2d(st + d * i8s::A_PLANE, ma, fb, k0, pr + ti.i0);
            tma_load_2d(st + i8s::ND * i8s::A_PLANE + d * i8s::B_PLANE, mb, fb,
                        bt ? ti.j0 : k0, pr + (bt ? k0 : ti.j0));
          }
        }
        __syncwarp();
        issued_phase[s] = u & 1;
      }
      if (!ok) break;
      // the tile's X_k into staging buffer tl & 1, once the stores of the tile that used
      // it two items ago have read it
      const int b = tl & 1;
      if (tl >= 2 && !mbar_wait_warp_idle(smem_u32(&bar_free[b]), ((tl - 2) >> 1) & 1, &s_abort)) {
        ok = false;
        break;
      }
      const uint32_t xb = smem_u32(&bar_xk[b]);
      if (elect_one()) {
        mbar_expect_tx(xb, i8s::OUT_BYTES);
#pragma unroll
        for (int d = 0; d < i8s::ND; ++d)
          tma_load_2d(stage_of(b) + d * i8s::OUT_PLANE, ma, xb, ti.j0, d * R + ti.row0 + ti.i0);
      }
      __syncwarp();
      xk_phase[b] = (tl >> 1) & 1;
    }
    if (!ok) {  // abort: wait (bounded) for this CTA's copies still in flight
      s_abort = 1;
      if (lane == 0) {
        for (int s = 0; s < i8s::ST; ++s)
          if (issued_phase[s] >= 0)
            for (uint32_t i = 0; i < kSpinLimit; ++i)
              if (mbar_try(smem_u32(&bar_full[s]), issued_phase[s])) break;
        for (int b = 0; b < 2; ++b)
          if (xk_phase[b] >= 0)
            for (uint32_t i = 0; i < kSpinLimit; ++i)
              if (mbar_try(smem_u32(&bar_xk[b]), xk_phase[b])) break;
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc0 = make_idesc_s8(i8s::BM, i8s::BN);
    constexpr uint32_t idesc128 = make_idesc_s8(i8s::BM, 2 * i8s::BN);
    bool ok = true;
    uint32_t g = 0, tl = 0;
    for (long long i = blockIdx.x; i < nitems && ok; i += G) {
      int k, t;
      item_of(i, k, t);
      const I8Tile ti = i8_tile_uniform(p.tiles, t);
      if (!ti.ok) {
        ok = false;
        break;
      }
      const int jb = ti.j0 & ~(i8s::BM - 1);
      // the accumulators are single-buffered: wait until the epilogue has read the
      // previous tile's
      if (tl >= 1 && !mbar_wait_warp(smem_u32(&bar_tempty), (tl - 1) & 1, &s_abort)) {
        ok = false;
        break;
      }
      tc_fence_after();
      for (int kb = 0; kb < ti.kb; ++kb, ++g) {
        const int s = g % i8s::ST;
        if (!mbar_wait_warp(smem_u32(&bar_full[s]), (g / i8s::ST) & 1, &s_abort)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int k0 = kb * i8s::BK;
        const bool at = k0 < ti.i0, bt = k0 < jb;
        // instruction descriptor with the MN-major bits (15: A, 16: B) of this k-block
        const uint32_t mn = (at ? 1u << 15 : 0u) | (bt ? 1u << 16 : 0u);
        const uint32_t id64 = idesc0 | mn, id128 = idesc128 | mn;
        const uint32_t st = sbase + s * i8s::STAGE_BYTES;
        // descriptors of plane 0 (a one-atom-wide MN-major tile has the same fields as
        // the K-major one of its swizzle); plane p starts p * plane bytes further, and
        // k advances by 32: 32 bytes K-major, 32 rows MN-major (in 16-byte units)
        // B as two planes of N = 64: K-major, plane t + 1's rows follow plane t's at the
        // same 8-row group stride; MN-major, the second 64-byte atom along N sits one plane
        // further (leading byte offset = one plane)
        const uint64_t da0 = at ? sw128_desc(st) : sw64_desc(st);
        const uint64_t db0 = sw64_desc_lbo(st + i8s::ND * i8s::A_PLANE, bt ? i8s::B_PLANE : 16);
        const uint32_t ka = at ? (32u * 128u) >> 4 : 32u >> 4;
        const uint32_t kb16 = bt ? (32u * 64u) >> 4 : 32u >> 4;
        if (elect_one()) {
#pragma unroll
          for (int kk = 0; kk < i8s::BK / i8s::UK; ++kk) {
#pragma unroll
            for (int q = 0; q < 7; ++q) {
              const int sa = i8_pa(q), sb = i8_pb(q);
              // the first three MMAs at k = 0 start the accumulators
              umma_i8(tmem + (sa + sb) * i8s::BN,
                      da0 + (uint64_t)(sa * (i8s::A_PLANE >> 4) + kk * ka),
                      db0 + (uint64_t)(sb * (i8s::B_PLANE >> 4) + kk * kb16),
                      i8_wide(q) ? id128 : id64, (kb > 0 || kk > 0 || !i8_first(q)) ? 1u : 0u);
            }
          }
          umma_commit(smem_u32(&bar_empty[s]));
        }
        __syncwarp();
      }
      if (!ok) break;
      if (elect_one()) umma_commit(smem_u32(&bar_tfull));
      __syncwarp();
      ++tl;
    }
    if (elect_one()) umma_commit(smem_u32(&bar_final));
    __syncwarp();
    for (uint32_t i = 0; i < kSpinLimit; ++i)
      if (mbar_try(smem_u32(&bar_final), 0)) break;
    if (!ok) s_abort = 1;
    __syncwarp();
  } else if (warp == i8s::STORE_WARP) {
    // ---------------- stores and completion signals ----------------
    // Waits only on its own CTA's epilogue, so every finished tile is signalled.
    uint32_t tl = 0;
    for (long long i = blockIdx.x; i < nitems; i += G, ++tl) {
      int k, t;
      item_of(i, k, t);
      const I8Tile ti = i8_tile_uniform(p.tiles, t);
      const int b = tl & 1;
      if (!mbar_wait_warp_idle(smem_u32(&bar_staged[b]), (tl >> 1) & 1, &s_abort)) break;
      if (elect_one()) {
#pragma unroll
        for (int d = 0; d < i8s::ND; ++d)
          tma_store_2d(&maps.a[(k + 1) & 1], stage_of(b) + d * i8s::OUT_PLANE, ti.j0,
                       d * R + ti.row0 + ti.i0);
        bulk_commit();
        bulk_wait_read0();
        mbar_arrive(smem_u32(&bar_free[b]));   // the producer may refill the buffer
        bulk_wait0();                          // landed in global memory
        fence_proxy_async_global();
        __threadfence();
        atomicAdd(p.done + p.tpart[t], 1u);
      }
      __syncwarp();
    }
  } else {
    // ---------------- epilogue (16 warps) ----------------
    const int q = warp & 3;                   // TMEM lane quarter
    const int grp = (warp - 2) >> 2;          // 16-column group of the 64-column tile
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    // this thread's 16 bytes of each staged plane: row q * 32 + lane, 16-byte chunk grp
    // under the 64-byte swizzle (chunk ^ (row >> 1) & 3)
    const int rl = q * 32 + lane;
    const int stg_off = i8s::OUT_OFF + rl * 64 + ((grp ^ ((rl >> 1) & 3)) << 4);
    // step sums of this warp, written once per (step, CTA, warp)
    double acc[3] = {0.0, 0.0, 0.0};   // Tr X_{k+1}, residual^2, Tr X_k^2
    int acc_k = -1;
    auto flush = [&]() {
      if (acc_k < 0) return;
#pragma unroll
      for (int v = 0; v < 3; ++v)
        for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
      if (lane == 0) {
        double* slot = p.partials + (((size_t)acc_k * G + blockIdx.x) * i8s::EPI_WARPS + (warp - 2)) * 4;
        slot[0] = 0.0;
        slot[1] = acc[0];
        slot[2] = acc[1];
        slot[3] = acc[2];
      }
      acc[0] = acc[1] = acc[2] = 0.0;
    };
    uint32_t tl = 0;
    for (long long i = blockIdx.x; i < nitems; i += G, ++tl) {
      int k, t;
      item_of(i, k, t);
      const I8Tile ti = i8_tile(p.tiles, t);
      if (k != acc_k) {
        flush();
        acc_k = k;
      }
      const int sg = p.pp[k] == 0 ? -1 : 1;      // X^2 branch: +1; 2X - X^2: -1
      const int r = ti.i0 + rl;                 // row inside the part
      const int c0 = ti.j0 + grp * 16;          // first column of this thread's 16
      const int b = tl & 1;
      uint8_t* stg = smem + stg_off + b * i8s::OUT_BYTES;
      if (!mbar_wait_idle(smem_u32(&bar_tfull), tl & 1, &s_abort) ||
          !mbar_wait(smem_u32(&bar_xk[b]), (tl >> 1) & 1, &s_abort))
        break;
      tc_fence_after();
      // Q = rint(2^31 X'^2) = floor((P + 2^14) / 2^15) with P = sum_u A_u 2^{32 - 8u}:
      //   Q = 2^17 A_0 + 2^9 A_1 + 2 A_2 + floor((A_3 + floor((A_4 + 2^14) / 2^8)) / 2^7),
      // the last term by nested floor division.  The sum is formed modulo 2^32; its true
      // value fits (|Q| <= 2^29 since |X'^2| <= 1/4), so the wrapped sum is exact.  All five
      // accumulators are read behind one wait and released before the sum (the next
      // tile's products wait for the release).
      int Q[16];
      {
        const uint32_t ta = tmem + lane_base + grp * 16;
        uint32_t a4[16], a3[16], a2[16], a1[16], a0[16];
        tmem_ld16(ta + 4 * i8s::BN, a4);
        tmem_ld16(ta + 3 * i8s::BN, a3);
        tmem_ld16(ta + 2 * i8s::BN, a2);
        tmem_ld16(ta + i8s::BN, a1);
        tmem_ld16(ta, a0);
        tmem_wait_ld();
        tc_fence_before();   // TMEM reads ordered before the release
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&bar_tempty));
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int ql = ((int)a3[j] + (((int)a4[j] + (1 << 14)) >> 8)) >> 7;
          Q[j] = (int)((a0[j] << 17) + (a1[j] << 9) + 2u * a2[j] + (uint32_t)ql);
        }
      }
      uint4 xd[i8s::ND];   // X_k digits of this thread's 16 elements (plane 0: d0)
#pragma unroll
      for (int d = 0; d < i8s::ND; ++d) xd[d] = *reinterpret_cast<const uint4*>(stg + d * i8s::OUT_PLANE);

      // Rows whose 16 columns all lie above the diagonal and on one side of the core
      // boundary weigh every element the same: the residual is summed once and scaled.
      const bool above = c0 > ti.i0 + q * 32 + 31;
      const bool cuni = above && (ti.core <= 0 || c0 + 15 < ti.core || c0 >= ti.core);
      const int cw_row = ti.core <= 0 ? 2 : (r < ti.core ? 1 : 0) + (c0 < ti.core ? 1 : 0);
      float s_res = 0.f;
      double s_tr = 0.0, s_trp = 0.0;
      // Digits as bytes of a biased integer: with the balanced digits d0..d3 of M (d1..d3
      // in [-128, 127]), M + B (B = 0x808080) has the bytes d3 + 128, d2 + 128, d1 + 128
      // and top byte d0, so the element's word [d3, d2, d1, d0] (byte 0 first) is
      // (M + B) ^ B, and M + B = word ^ B.  The step works on M + B directly.
      constexpr uint32_t kB = 0x00808080u;
      uint32_t wn[16];   // X_{k+1} of each element as the word [d3, d2, d1, d0]
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        // element-major words of X_k for elements 4g..4g+3 gathered from the four planes
        // (a 4 x 4 byte transpose)
        const uint32_t p0 = g == 0 ? xd[0].x : g == 1 ? xd[0].y : g == 2 ? xd[0].z : xd[0].w;
        const uint32_t p1 = g == 0 ? xd[1].x : g == 1 ? xd[1].y : g == 2 ? xd[1].z : xd[1].w;
        const uint32_t p2 = g == 0 ? xd[2].x : g == 1 ? xd[2].y : g == 2 ? xd[2].z : xd[2].w;
        const uint32_t p3 = g == 0 ? xd[3].x : g == 1 ? xd[3].y : g == 2 ? xd[3].z : xd[3].w;
        const uint32_t alo = __byte_perm(p3, p2, 0x5140u), ahi = __byte_perm(p3, p2, 0x7362u);
        const uint32_t blo = __byte_perm(p1, p0, 0x5140u), bhi = __byte_perm(p1, p0, 0x7362u);
        uint32_t u4[4];
        u4[0] = __byte_perm(alo, blo, 0x5410u);
        u4[1] = __byte_perm(alo, blo, 0x7632u);
        u4[2] = __byte_perm(ahi, bhi, 0x5410u);
        u4[3] = __byte_perm(ahi, bhi, 0x7632u);
        if (cuni) {
          // off the diagonal, one weight: X'_{k+1} = X' +- X'^2, residual^2 = Q^2
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int j = 4 * g + e;
            wn[j] = ((u4[e] ^ kB) + (uint32_t)(sg * Q[j])) ^ kB;
            const float qf = (float)Q[j];
            s_res = fmaf(qf, qf, s_res);
          }
          continue;
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int j = 4 * g + e;
          const int c = c0 + j;
          const bool dg = r == c;
          const uint32_t mb = u4[e] ^ kB;                         // M_k + B
          const uint32_t nb = mb + (uint32_t)(sg * Q[j]) - (dg ? (uint32_t)sg << 29 : 0u);
          wn[j] = nb ^ kB;
          // 2^31 (X - X^2) = 2^31 (I/4 - X'^2), from the rounded square
          const float res = (float)((dg ? (1 << 29) : 0) - Q[j]);
          {
            // weight of (r, c) in the full-matrix sums: itself and its mirror above the
            // diagonal, once on it, nothing below it (its mirror above carries it)
            const int w = r < c ? 2 : (dg ? 1 : 0);
            s_res = fmaf((float)core_weight(w, r, c, ti.core) * res, res, s_res);
            if (dg) {
              const int m = (int)(mb - kB), mn = (int)(nb - kB);
              s_tr += (double)mn * 0x1p-31 + 0.5;
              s_trp += (double)Q[j] * 0x1p-31 + (double)m * 0x1p-31 + 0.25;   // Tr X^2
            }
          }
        }
      }
      acc[0] += s_tr;
      acc[1] = fma((double)(cuni ? (float)cw_row * s_res : s_res), 0x1p-62, acc[1]);
      acc[2] += s_trp;
      // X_{k+1}: this thread's 16 bytes of each plane (the inverse 4 x 4 transposes)
      {
        uint32_t o[i8s::ND][4];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          const uint32_t x = __byte_perm(wn[4 * g], wn[4 * g + 1], 0x5140u);
          const uint32_t xh = __byte_perm(wn[4 * g], wn[4 * g + 1], 0x7362u);
          const uint32_t y = __byte_perm(wn[4 * g + 2], wn[4 * g + 3], 0x5140u);
          const uint32_t yh = __byte_perm(wn[4 * g + 2], wn[4 * g + 3], 0x7362u);
          o[3][g] = __byte_perm(x, y, 0x5410u);
          o[2][g] = __byte_perm(x, y, 0x7632u);
          o[1][g] = __byte_perm(xh, yh, 0x5410u);
          o[0][g] = __byte_perm(xh, yh, 0x7632u);
        }
#pragma unroll
        for (int d = 0; d < i8s::ND; ++d)
          *reinterpret_cast<uint4*>(stg + d * i8s::OUT_PLANE) = make_uint4(o[d][0], o[d][1], o[d][2], o[d][3]);
      }
      fence_proxy_async_smem();   // staged bytes visible to the TMA stores
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bar_staged[b]));
    }
    flush();
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, i8s::TMEM_COLS);
  if (s_abort && threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
}

// Step sums: step k's totals over every (CTA, warp) slot in a fixed order; vv[k] gets the
// residual sum (added to the caller's accumulator).
__global__ void k_i8_step_sums(const double* __restrict__ partials, int nslots,
                               double* __restrict__ vv) {
  __shared__ double red[32 * 4];
  const int k = blockIdx.x;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = threadIdx.x; j < nslots; j += blockDim.x)
    for (int q = 0; q < 4; ++q) s[q] += partials[((size_t)k * nslots + j) * 4 + q];
  block_sum<4>(s, red);
  if (threadIdx.x == 0) vv[k] += s[2];
}

size_t i8_steps_partials(int nsteps) {
  return (size_t)std::max(nsteps, 1) * device_sms() * i8s::EPI_WARPS * 4;
}

cudaError_t launch_i8_steps(const I8StepsArgs& a, const void* buf0, const void* buf1, int ld,
                            double* vv, cudaStream_t st) {
  if (!a.tiles || !a.tpart || !a.pnt || !a.pp || !a.done || !a.partials || a.ntiles <= 0 ||
      a.nsteps <= 0 || ld % 128 != 0 || a.rows % i8s::BM != 0 || !buf0 || !buf1 || !vv ||
      4LL * a.rows > 0x7fffffffLL)
    return cudaErrorInvalidValue;
  // per buffer: K-major operand / staged tile, MN-major A^T, and B / B^T maps over its 4R rows
  I8Maps m;
  for (int b = 0; b < 2; ++b) {
    const void* buf = b ? buf1 : buf0;
    if (!make_tmap_u8_sw64(&m.a[b], buf, 4LL * a.rows, ld, ld, i8s::BM) ||
        !make_tmap_box(&m.at[b], buf, 4LL * a.rows, ld, ld, TMAP_U8, i8s::BK) ||
        !make_tmap_u8_sw64(&m.b[b], buf, 4LL * a.rows, ld, ld, i8s::BN))
      return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaFuncSetAttribute(k_i8_steps, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       i8s::SMEM_BYTES);
  if (e != cudaSuccess) return e;
  const long long nitems = (long long)a.ntiles * a.nsteps;
  const int grid = (int)std::min<long long>(nitems, device_sms());
  // one CTA per SM, all resident: the CTAs wait on each other's tiles
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(i8s::NTHR);
  cfg.dynamicSmemBytes = i8s::SMEM_BYTES;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, k_i8_steps, m, a);
  note_launch();
  if (e != cudaSuccess) return e;
  k_i8_step_sums<<<a.nsteps, 256, 0, st>>>(a.partials, grid * i8s::EPI_WARPS, vv);
  note_launch();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Digit-form extraction, scatter and part idempotency for the batched INT8 mode.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void i8_store_x(int8_t* base, size_t plane, size_t idx, double xprime) {
  const int m = (int)llrint(xprime * 0x1p31);
  int8_t d0, d1, d2, d3;
  i8_digits(m, d0, d1, d2, d3);
  base[idx] = d0;
  base[plane + idx] = d1;
  base[2 * plane + idx] = d2;
  base[3 * plane + idx] = d3;
}

// CSR rows of each part straight to X0' = X0 - I/2 in digits (parts up to 512), with the
// same row construction as the split extraction: one warp per row in shared memory.  The
// row's digits are collected by plane in shared memory and leave as 16-byte stores.
__global__ void __launch_bounds__(256) k_extract_digits(
    const long long* __restrict__ rp, const int* __restrict__ col, const double* __restrict__ val,
    const PartDesc* __restrict__ parts, const int* __restrict__ halo, const int* __restrict__ skey,
    const int* __restrict__ sval, int ld, long long rows, double emin, double emax,
    int8_t* __restrict__ dig) {
  __shared__ double rowbuf[8][512];
  __shared__ __align__(16) int8_t dbuf[8][4][512];
  const PartDesc P = parts[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double mm = emax - emin;
  const double alpha = -1.0 / mm, beta = emax / mm;
  const int* hl = halo + P.hoff;
  const int* sk = skey + P.hoff;
  const int* sv = sval + P.hoff;
  const size_t plane = (size_t)rows * ld;
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
    int8_t(*db)[512] = dbuf[warp];
    for (int c = lane; c < P.np; c += 32) {
      // separate roundings (no contraction), so a host model forms the same X0'
      double x = 0.0;
      if (r < P.n && c < P.n) {
        x = __dmul_rn(alpha, buf[c]);
        if (r == c) x = __dadd_rn(x, beta);
      }
      const int m = (int)llrint((r == c ? __dadd_rn(x, -0.5) : x) * 0x1p31);
      i8_digits(m, db[0][c], db[1][c], db[2][c], db[3][c]);
    }
    __syncwarp();
    const size_t ro = ((size_t)P.row0 + r) * ld;   // ld, np: multiples of 128
    for (int c0 = lane * 16; c0 < P.np; c0 += 512)
#pragma unroll
      for (int d = 0; d < 4; ++d)
        *reinterpret_cast<uint4*>(dig + d * plane + ro + c0) =
            *reinterpret_cast<const uint4*>(&db[d][c0]);
    __syncwarp();
  }
}

// The same from the FP64 packed extraction (parts above 512): X0' digits of every
// packed element.
__global__ void k_norm_digits(const double* __restrict__ xs, const int* __restrict__ row_part,
                              const PartDesc* __restrict__ parts, long long rows, int ld,
                              double emin, double emax, int8_t* __restrict__ dig) {
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
      v = __dmul_rn(alpha, xs[idx]);
      if (r == c) v = __dadd_rn(v, beta);
    }
    if (c < P.np) i8_store_x(dig, total, idx, r == c ? __dadd_rn(v, -0.5) : v);
  }
}

// Offset of entry (r, c) of a part in the upper-band storage the step kernel keeps: row r
// holds the columns from its 128-row block's first row on; the rest is read from the
// mirror (c, r).
__device__ __forceinline__ size_t i8_band_off(long long row0, int r, int c, int ld) {
  return c >= (r & ~(i8s::BM - 1)) ? ((size_t)row0 + r) * ld + c : ((size_t)row0 + c) * ld + r;
}

// rho (core rows) = 2 X = 2^-30 M + I; one warp per core row, the lanes along it.
__global__ void k_scatter_digits(const int8_t* __restrict__ dig, long long rows,
                                 const PartDesc* __restrict__ parts, const int* __restrict__ halo,
                                 int ld, double* __restrict__ core_out, double* __restrict__ dense,
                                 long long n) {
  const PartDesc P = parts[blockIdx.x];
  const int* hl = halo + P.hoff;
  const size_t plane = (size_t)rows * ld;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int r = blockIdx.y * nw + warp; r < P.ncore; r += gridDim.y * nw) {
    double* co = core_out ? core_out + P.coff + (size_t)r * P.n : nullptr;
    for (int c = lane; c < P.n; c += 32) {
      const size_t src = i8_band_off(P.row0, r, c, ld);
      const int m = i8_value(dig[src], dig[plane + src], dig[2 * plane + src], dig[3 * plane + src]);
      const double v = (double)m * 0x1p-30 + (r == c ? 1.0 : 0.0);
      if (co) co[c] = v;
      if (dense) dense[(size_t)hl[r] + (size_t)hl[c] * n] = v;
    }
  }
}

// Sum over each part's core rows of (X - X^2)_ii = X_ii - sum_j X_ij^2, from the digits
// (upper-band storage).  Columns j < n only: past the part size X is zero off the
// diagonal, and past the tiles' columns (the part size rounded up to 64) the iterated
// buffer holds entries no step writes.
__global__ void k_part_idem_digits(const int8_t* __restrict__ dig, long long rows,
                                   const PartDesc* __restrict__ parts, int ld,
                                   double* __restrict__ out) {
  __shared__ double red[32];
  const PartDesc P = parts[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const size_t plane = (size_t)rows * ld;
  double s = 0.0;
  for (int r = blockIdx.y * nw + warp; r < P.ncore; r += gridDim.y * nw) {
    const size_t row = ((size_t)P.row0 + r) * ld;
    // columns left of the row's block from their mirrors (off the diagonal)
    const int rb = r & ~(i8s::BM - 1);
    for (int c = lane; c < rb; c += 32) {
      const size_t o = ((size_t)P.row0 + c) * ld + r;
      const double x = (double)i8_value(dig[o], dig[plane + o], dig[2 * plane + o], dig[3 * plane + o]) *
                       0x1p-31;
      s -= x * x;
    }
    for (int c0 = rb + lane * 16; c0 < P.n; c0 += 512) {
      uint4 v[4];
#pragma unroll
      for (int d = 0; d < 4; ++d) v[d] = *reinterpret_cast<const uint4*>(dig + d * plane + row + c0);
      const int8_t* b0 = reinterpret_cast<const int8_t*>(&v[0]);
      const int8_t* b1 = reinterpret_cast<const int8_t*>(&v[1]);
      const int8_t* b2 = reinterpret_cast<const int8_t*>(&v[2]);
      const int8_t* b3 = reinterpret_cast<const int8_t*>(&v[3]);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const double x = (double)i8_value(b0[e], b1[e], b2[e], b3[e]) * 0x1p-31 +
                         (c0 + e == r ? 0.5 : 0.0);
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

cudaError_t launch_extract_digits(const long long* rp, const int* col, const double* val,
                                  const PartDesc* parts, int nparts, const int* halo,
                                  const int* skey, const int* sval, int ld, long long rows,
                                  double emin, double emax, int8_t* dig, cudaStream_t st) {
  if (ld > 512) return cudaErrorInvalidValue;
  k_extract_digits<<<dim3(nparts, 16), 256, 0, st>>>(rp, col, val, parts, halo, skey, sval, ld,
                                                     rows, emin, emax, dig);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_norm_digits(const double* xs, const int* row_part, const PartDesc* parts,
                               long long rows, int ld, double emin, double emax, int8_t* dig,
                               cudaStream_t st) {
  size_t g = ((size_t)rows * ld + 255) / 256;
  if (g > 148 * 8) g = 148 * 8;
  k_norm_digits<<<(int)(g ? g : 1), 256, 0, st>>>(xs, row_part, parts, rows, ld, emin, emax, dig);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_scatter_digits(const int8_t* dig, long long rows, const PartDesc* parts,
                                  int nparts, const int* halo, int ld, double* core_out,
                                  double* dense, long long n, cudaStream_t st) {
  k_scatter_digits<<<dim3(nparts, 16), 256, 0, st>>>(dig, rows, parts, halo, ld, core_out, dense,
                                                     n);
  note_launch();
  return cudaGetLastError();
}

cudaError_t launch_part_idem_digits(const int8_t* dig, long long rows, const PartDesc* parts,
                                    int nparts, int ld, double* out, cudaStream_t st) {
  k_part_idem_digits<<<dim3(nparts, kPartIdemGroups), 256, 0, st>>>(dig, rows, parts, ld, out);
  note_launch();
  return cudaGetLastError();
}

}  // namespace sp2b
