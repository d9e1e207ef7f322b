// Split-BF16 tensor-core form of the exchange integrals:
//     Z_L = K_L B   (tcgen05.mma, FP32 accumulators in TMEM),   I_f,L = sum_i a_f[i] Z_L[i, f]  (FP64)
//
// Reference: the exchange contraction of oscillatory_integrals.py:2745-2770 (CPU) and
// dwba_matrix_elements.py:1469-1560 (CuPy), with the CC quadrature folded into b_f.
//
// K_L and B are split into NT bfloat16 terms (NT = 2: hi + lo, products hh, hl, lh;
// NT = 3: hi + mid + lo, products of total order <= 2). Each CTA owns a 128-row block of
// the grid (i), BN forms (f) and one multipole L, and walks the grid in 64-wide blocks (j):
//   * B tiles (BN forms x 64 j per term, K-major, 128-byte swizzle) arrive by TMA;
//   * K_L tiles (128 x 64 per term) are generated in registers and stored to shared memory
//     in the same swizzled layout. Off-diagonal blocks are exactly rank one,
//     K_L(i,j) = U_i V_j (r_j^L / r_i^(L+1) below the diagonal, r_i^L / r_j^(L+1) above),
//     with U, V scaled by the block's boundary radius so they stay in FP32 range; blocks
//     that touch the diagonal use the full formula in FP64 (diagonal: (1-1e-12)^L / r);
//   * one thread of a dedicated warp issues the TMA copies and the tcgen05.mma products into a
//     TMEM accumulator;
//   * two shared-memory stages let generation of block k+1 overlap the MMAs of block k.
// The epilogue reads the accumulator with tcgen05.ld, multiplies by a_f[i] in FP64 and
// reduces over the 128 rows; partials per (L, row block, form) are summed in fixed order.
// Every mbarrier wait is bounded: on timeout the CTA records an error, drains its own
// in-flight copies (bounded), frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace {

constexpr int BM = 128;  // rows (i) per CTA = TMEM lanes
constexpr int BK = 64;   // j per block: 64 bf16 = one 128-byte swizzle row
constexpr int GEN_WARPS = 16;  // K_L tile generators: 4 x 32 rows x 4 column quarters
constexpr int GEN_THREADS = 32 * GEN_WARPS;
constexpr int THREADS = 32 + GEN_THREADS;  // + warp 0: TMA and MMA issue
constexpr int TC_BN2 = 256;  // forms per CTA with two terms
constexpr int TC_BN3 = 256;   // forms per CTA with three terms
// pipeline stages (B tiles in shared memory, K_L tiles in tensor memory): 3 with two terms,
// 2 with three (tensor memory: BN accumulator columns + S x NT x BK/2 K_L columns <= 512)
__host__ __device__ constexpr int tc_stages(int nt) { return nt == 2 ? 3 : 2; }
constexpr int TMEM_COLS = 512;
constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at 1.9 GHz

struct GemmParams {
  const double* r;             // grid (n_grid)
  const double* lg;            // log2(r) (n_grid)
  const dwba_form_t* forms;    // a_f (rows) for the epilogue
  double* partial;             // [n_L][n_iblk][f_pad]
  const int* bexp;             // per form: b was scaled by 2^-bexp before the split
  const float* vt;             // [2][n_L][n_pad] column factors within each j block (below, above)
  const float* st;             // [n_L][n_iblk][n_kb] per (row block, j block) scale (0 where K is not rank one)
  int* status;                 // error word
  const double* gw;            // gradient mode: dLoss/dI per (form, L), [n_forms][n_Ltot]
  double* gpart;               // gradient mode: g_f,L (K_L b_f)_i per L, [n_L][f_pad][n_pad]
  long long wait_cycles;       // bound of every pipeline wait (SM clocks)
  int n_grid, n_pad, f_pad, n_iblk, L_max, n_forms, n_kb, n_Ltot;
  double diag[DWBA_MAX_L + 1];
};

// One grid of a (ragged) launch: its operands, workspace tables and layout. The B terms of every
// segment are rows of one bf16 matrix (one tensor map): segment rows row0 .. row0 + NT f_pad - 1.
struct TcSeg {
  const double* r;             // grid (n_grid)
  const double* lg;            // log2(r) (n_grid)
  const dwba_form_t* forms;    // a_f (rows) for the epilogue
  double* partial;             // [n_L][n_iblk][f_pad]
  const int* bexp;             // per form: b was scaled by 2^-bexp before the split
  const float* vt;             // [2][n_L][n_pad]
  const float* st;             // [n_L][n_iblk][n_kb]
  double* gpart;               // gradient mode: [n_L][f_pad][n_pad]
  int n_grid, n_pad, f_pad, n_iblk, n_forms, n_kb, row0, n_fblk;
};
constexpr int TC_MAX_SEGS = 96;
// The segments of one launch, passed by value (kernel parameter space). CTAs are numbered
// segment by segment (cta0 ascending); within a segment, order 0 runs the row blocks fastest,
// then the form blocks, then the multipoles; order 1 runs the form blocks fastest.
struct TcSegs {
  int n, order;
  int cta0[TC_MAX_SEGS + 1];
  TcSeg s[TC_MAX_SEGS];
};

// ---- PTX wrappers --------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// bounded wait (limit in SM clocks; the pipeline passes P.wait_cycles, the error-path drain the
// default of about a second); returns false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit) {
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, phase)) return true;
    if (clock64() - t0 > limit) return false;
  }
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// SMEM matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFF) >> 4);           // start address
  d |= (uint64_t)1 << 16;                            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;                  // stride byte offset
  d |= (uint64_t)1 << 46;                            // descriptor version (sm100)
  d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
  return d;
}
// Instruction descriptor, kind::f16: D f32, A/B bf16, both K-major, M = 128, N = bn.
__host__ __device__ constexpr uint32_t instr_desc(int bn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(bn >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
// A from tensor memory: row i of the 128 x 16 A slice in lane i, two bf16 per 32-bit column
// (even k in the low half), 8 consecutive columns per K = 16.
__device__ __forceinline__ void mma_bf16_tmem_a(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc, uint32_t idesc,
                                                uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}"
      ::"r"(tmem_d), "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};"
               ::"r"(taddr), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int c = 0; c < 32; ++c) v[c] = __uint_as_float(r[c]);
}

// 16 consecutive K_L values of one row -> NT bfloat16 terms, 8 packed words each (element 2c in
// the low half of word c): t_0 = bf16(x), t_1 = bf16(x - t_0), t_2 = bf16(x - t_0 - t_1); x - t_0 is
// exact in FP32. cvt.rn.bf16x2.f32 rounds two values to nearest-even and packs them.
template <int NT>
__device__ __forceinline__ void split_terms(const float* k16, uint32_t (*w)[8]) {
  float rem[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) rem[e] = k16[e];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const __nv_bfloat162 q = __floats2bfloat162_rn(rem[2 * c], rem[2 * c + 1]);
      w[t][c] = *reinterpret_cast<const uint32_t*>(&q);
      if (t + 1 < NT) {
        rem[2 * c] -= __uint_as_float(w[t][c] << 16);
        rem[2 * c + 1] -= __uint_as_float(w[t][c] & 0xFFFF0000u);
      }
    }
  }
}

// Far-to-near order of the j blocks of one row block: the blocks below and above the diagonal
// merged by decreasing distance (ties: below first), then the blocks that touch the diagonal.
struct BlockOrder {
  int lo, hi, nd, kd0, kd1;
  __device__ BlockOrder(int n_kb, int i0) : lo(0), hi(n_kb - 1), nd(i0 / BK), kd0(i0 / BK) {
    kd1 = min(kd0 + BM / BK, n_kb);
  }
  __device__ int next() {
    const int dl = lo < kd0 ? kd0 - lo : -1;       // distance of the next block below
    const int dh = hi >= kd1 ? hi - kd1 + 1 : -1;  // and above
    if (dl < 0 && dh < 0) return nd++;
    if (dl >= dh) return lo++;
    return hi--;
  }
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Warp-specialised pipeline over S stages, synchronised by mbarriers only. Stage s holds the
// K_L terms of one j block in tensor memory (A operand of tcgen05.mma, written by the generator
// warps with tcgen05.st) and the B terms in shared memory (written by TMA):
//   warp 0, lane 0 (issuer): waits for K_L(t) (bar_a) and the B tiles of block t (bar_b), issues the
//     products of block t and commits them to bar_mma; then waits for the products of block t-1 and
//     fetches the B tiles of block t+S-1 into that stage (S-1 blocks of copy lead).
//   warps 1..16 (generators): wait for the products of block t-S (stage free), write K_L(t) and arrive
//     on bar_a (one arrival per warp). Warp w owns tensor-memory lanes 32 (w mod 4) .. +31 (rows) and
//     the 16-column quarter (w-1)/4 of the block. Off-diagonal tiles are U_i s(row block, j block) v_j
//     with v_j from a precomputed table, prefetched one block ahead into registers.
// Shared memory carries only the B tiles, so the tensor cores read one operand from it.
// Rank-one factors, scaled so that every factor stays in FP32 range (c_lo, c_hi: smallest and
// largest radius of the row block, c_b: first radius of the j block):
//   below the diagonal: K = r_j^L / r_i^(L+1) = [c_lo^L / r_i^(L+1)] [(c_b/c_lo)^L] [(r_j/c_b)^L]
//   above the diagonal: K = r_i^L / r_j^(L+1) = [(r_i/c_hi)^L] [c_hi^L / c_b^(L+1)] [(r_j/c_b)^-(L+1)]
// GRAD = false: I_f,L = sum_i a_f[i] Z_L[i, f] (partials per row block). GRAD = true (backward):
// the epilogue writes g_f,L Z_L[i, f] for every row i instead, summed over L afterwards.
template <int NT, int BN, bool GRAD, int SN = tc_stages(NT)>
__global__ void __launch_bounds__(THREADS, 1)
tc_exchange_kernel(const __grid_constant__ CUtensorMap bmap, const __grid_constant__ GemmParams P,
                   const __grid_constant__ TcSegs SG) {
  constexpr int B_BYTES = BN * BK * 2;            // one term
  constexpr int STAGE = NT * B_BYTES;             // shared memory per stage
  constexpr int NPROD = NT == 2 ? 3 : 6;
  constexpr int S = SN;
  static_assert(S >= 2 && S * STAGE + 1024 <= 227 * 1024, "shared memory");
  constexpr int A_COLS = BK / 2;                  // tensor-memory columns of one K_L term
  static_assert(BN + S * NT * A_COLS <= TMEM_COLS, "tensor memory");
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  __shared__ uint64_t bar_b[S], bar_a[S], bar_mma[S];
  __shared__ uint32_t tmem_base_s;
  __shared__ float sUb[BM], sUa[BM];
  __shared__ double sRi[BM];
  __shared__ double sRed[4][BN];
  __shared__ volatile int s_abort;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // this CTA's segment (binary search over the ascending cta0) and its (row block, form block, L)
  const int cta = blockIdx.x;
  int sg_lo = 0, sg_hi = SG.n - 1;
  while (sg_lo < sg_hi) {
    const int mid = (sg_lo + sg_hi + 1) >> 1;
    if (SG.cta0[mid] <= cta) sg_lo = mid; else sg_hi = mid - 1;
  }
  const TcSeg& G = SG.s[sg_lo];  // parameter space (grid constant): no local copy
  const int local = cta - SG.cta0[sg_lo];
  int iblk, fblk, L;
  if (SG.order == 0) {
    iblk = local % G.n_iblk;
    const int q = local / G.n_iblk;
    fblk = q % G.n_fblk;
    L = q / G.n_fblk;
  } else {
    fblk = local % G.n_fblk;
    const int q = local / G.n_fblk;
    iblk = q % G.n_iblk;
    L = q / G.n_iblk;
  }
  const int i0 = iblk * BM, f0 = fblk * BN;
  const int n_kb = G.n_kb;

  if (tid == 0) {
    // a CTA that starts after another one timed out skips the work (the decision is shared
    // through shared memory so that every thread of the CTA takes the same path)
    s_abort = *(volatile int*)P.status != 0 ? 1 : 0;
    for (int q = 0; q < S; ++q) {
      mbar_init(&bar_b[q], 1);
      mbar_init(&bar_a[q], GEN_WARPS);
      mbar_init(&bar_mma[q], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (s_abort) return;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"((uint32_t)TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // row factors: U_i below the diagonal (c_lo^L / r_i^(L+1)) and above ((r_i/c_hi)^L), as exp2 of
  // FP64 differences of log2 r
  const double lg_lo = G.lg[i0];
  const double lg_hi = G.lg[min(i0 + BM, G.n_grid) - 1];
  const double Lp1 = (double)(L + 1), Ld = (double)L;
  for (int m = tid; m < BM; m += THREADS) {
    const bool in = i0 + m < G.n_grid;
    const double ri = in ? G.r[i0 + m] : 0.0;
    const double li = in ? G.lg[i0 + m] : 0.0;
    sRi[m] = ri;
    sUb[m] = in ? (float)exp2(-Lp1 * (li - lg_lo) - lg_lo) : 0.0f;
    sUa[m] = in ? (float)exp2(Ld * (li - lg_hi)) : 0.0f;
  }
  auto kind_of = [&](int kb_t) {  // 0: below the diagonal, 1: above, 2: touches it
    const int j0 = kb_t * BK;
    return (j0 + BK - 1 < i0) ? 0 : ((j0 > i0 + BM - 1) ? 1 : 2);
  };
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_s;
  const uint32_t tmem_a = tmem + BN;  // K_L terms: stage s, term t at column BN + (s NT + t) A_COLS

  // issuer bookkeeping (warp 0, lane 0): per stage the step of the last B copy issued into it and
  // whether it is still in flight; the last step whose products were committed
  int b_step[S];
  bool b_pending[S];
#pragma unroll
  for (int q = 0; q < S; ++q) {
    b_step[q] = -1;
    b_pending[q] = false;
  }
  int last_commit = -1;

  if (warp == 0) {
    if (lane == 0) {
      const uint32_t idesc = instr_desc(BN);
      auto issue_tma = [&](int st_idx, int kb_t, int step_t) {
        uint8_t* b_dst = smem + st_idx * STAGE;
        mbar_expect_tx(&bar_b[st_idx], NT * B_BYTES);
#pragma unroll
        for (int t = 0; t < NT; ++t)
          tma_load_2d(b_dst + t * B_BYTES, &bmap, &bar_b[st_idx], kb_t * BK, G.row0 + t * G.f_pad + f0);
        b_step[st_idx] = step_t;
        b_pending[st_idx] = true;
      };
      BlockOrder order(n_kb, i0);
      // prologue: B tiles of the first S-1 blocks (their stages are free)
      int n_issued = 0;
      for (; n_issued < S - 1 && n_issued < n_kb; ++n_issued) issue_tma(n_issued, order.next(), n_issued);
      bool good = true;
      for (int step = 0; step < n_kb; ++step) {
        const int s = step % S;
        const uint32_t par = (uint32_t)((step / S) & 1);
        good = mbar_wait(&bar_a[s], par, P.wait_cycles) && !s_abort;
        if (good) good = mbar_wait(&bar_b[s], par, P.wait_cycles);
        if (!good) break;
        b_pending[s] = false;
        tc_fence_after();
        const uint32_t b0 = smem_u32(smem + s * STAGE);
        const uint32_t a0 = tmem_a + (uint32_t)(s * NT * A_COLS);
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
#pragma unroll
          for (int q = 0; q < NPROD; ++q) {
            // (a term, b term) of product q, total order <= NT-1:
            // NT=2: (0,0) (0,1) (1,0); NT=3: (0,0) (0,1) (1,0) (0,2) (1,1) (2,0)
            const int ta = (q == 2 || q == 4) ? 1 : (q == 5 ? 2 : 0);
            const int tb = (q == 1 || q == 4) ? 1 : (q == 3 ? 2 : 0);
            const uint64_t bd = smem_desc(b0 + tb * B_BYTES + kk * 32);
            mma_bf16_tmem_a(tmem, a0 + (uint32_t)(ta * A_COLS + kk * 8), bd, idesc,
                            (step > 0 || kk > 0 || q > 0) ? 1u : 0u);
          }
        }
        mma_commit(&bar_mma[s]);
        last_commit = step;
        if (n_issued < n_kb) {
          // block n_issued = step + S - 1 goes into the stage of block step-1, free once its
          // products completed
          const int sp = n_issued % S;
          if (step >= 1) good = mbar_wait(&bar_mma[sp], (uint32_t)(((step - 1) / S) & 1), P.wait_cycles);
          if (!good) break;
          issue_tma(sp, order.next(), n_issued);
          ++n_issued;
        }
      }
      if (!good) s_abort = 1;
    }
    __syncwarp();
  } else {
    // generator warps
    BlockOrder order(n_kb, i0);
    int kb = order.next();
    const int quarter = warp & 3;              // tensor-memory lane quarter
    const int row = 32 * quarter + lane;
    const int kh = ((warp - 1) >> 2) * 16;     // first of this warp's 16 columns of the block
    const int i = i0 + row;
    const uint32_t lane_off = (uint32_t)(32 * quarter) << 16;
    const float* vt_b = G.vt + (int64_t)L * G.n_pad;                  // below the diagonal
    const float* vt_a = G.vt + (int64_t)(P.L_max + 1 + L) * G.n_pad;  // above
    const float* st = G.st + ((int64_t)L * G.n_iblk + iblk) * n_kb;
    // column factors and block scale of a j block (rank-one blocks only), 16 columns per thread
    auto load_factors = [&](int kb_t, float4* v, float& sc) {
      const int kind = kind_of(kb_t);
      if (kind == 2) {
        sc = 0.0f;
        return;
      }
      const float4* src = reinterpret_cast<const float4*>((kind == 0 ? vt_b : vt_a) + kb_t * BK + kh);
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = __ldg(src + q);
      sc = __ldg(st + kb_t);
    };
    float4 v_cur[4], v_nxt[4];
    float s_cur = 0.0f, s_nxt = 0.0f;
    load_factors(kb, v_cur, s_cur);
    bool good = true;
    for (int step = 0; step < n_kb; ++step) {
      const int s = step % S;
      const int kb_next = step + 1 < n_kb ? order.next() : -1;
      if (kb_next >= 0) load_factors(kb_next, v_nxt, s_nxt);  // in flight while this block is generated
      // stage s is free once the products of block step-S completed
      if (step >= S) good = mbar_wait(&bar_mma[s], (uint32_t)(((step - S) / S) & 1), P.wait_cycles);
      good = __all_sync(0xffffffffu, good && !s_abort);  // warp-uniform: the warp arrives all or none
      if (!good) break;
      tc_fence_after();
      const int j0 = kb * BK;
      const int kind = kind_of(kb);
      float k16[16];
      if (kind != 2) {
        const float us = (kind == 0 ? sUb[row] : sUa[row]) * s_cur;
        const float* vv = reinterpret_cast<const float*>(v_cur);
#pragma unroll
        for (int e = 0; e < 16; ++e) k16[e] = us * vv[e];
      } else {
        const double ri = sRi[row];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int j = j0 + kh + e;
          double kv = 0.0;
          if (i < G.n_grid && j < G.n_grid) {
            if (i == j) {
              kv = P.diag[L] / ri;
            } else {
              const double rj = G.r[j];
              const double rl = fmin(ri, rj), rg = fmax(ri, rj);
              const double inv = 1.0 / rg;
              double ratio = rl * inv, pw = 1.0;
              for (int e2 = L; e2 > 0; e2 >>= 1) {
                if (e2 & 1) pw *= ratio;
                ratio *= ratio;
              }
              kv = inv * pw;
            }
          }
          k16[e] = (float)kv;
        }
      }
      uint32_t w[NT][8];
      split_terms<NT>(k16, w);
#pragma unroll
      for (int t = 0; t < NT; ++t)
        tmem_st8(tmem_a + lane_off + (uint32_t)((s * NT + t) * A_COLS + (kh >> 1)), w[t]);
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bar_a[s]);
      kb = kb_next;
#pragma unroll
      for (int q = 0; q < 4; ++q) v_cur[q] = v_nxt[q];
      s_cur = s_nxt;
    }
    // every product has completed once the last commit arrived (commits track all prior MMAs)
    if (good) good = mbar_wait(&bar_mma[(n_kb - 1) % S], (uint32_t)(((n_kb - 1) / S) & 1), P.wait_cycles);
    if (!good) s_abort = 1;
  }
  __syncthreads();
  // error path (thread 0, the issuer): wait, bounded by the default limit whatever the pipeline's,
  // for the copies still in flight and the last commit. Each barrier waited on here is at most one
  // phase behind the one named: a stage's copy is issued only after the previous copy into it
  // was consumed, and the last commit follows the completion of the stage's previous commit
  // (the generators waited for it before writing the block the issuer committed)
  if (tid == 0 && s_abort) {
    for (int q = 0; q < S; ++q)
      if (b_pending[q]) mbar_wait(&bar_b[q], (uint32_t)((b_step[q] / S) & 1), WAIT_CYCLES);
    if (last_commit >= 0) mbar_wait(&bar_mma[last_commit % S], (uint32_t)((last_commit / S) & 1), WAIT_CYCLES);
    atomicExch(P.status, 2);
  }
  __syncthreads();
  const bool ok = !s_abort;
  tc_fence_after();
  if (GRAD && ok && warp >= 1) {
    // gradient epilogue: every (row, form) value times the form's upstream gradient for this L;
    // the lanes of a warp write 32 consecutive rows of one form
    const int g = warp & 3, h = (warp - 1) >> 2;
    const int i = i0 + 32 * g + lane;
    for (int c0 = h * (BN / 4); c0 < (h + 1) * (BN / 4); c0 += 32) {
      float z[32];
      tmem_ld32(tmem + ((uint32_t)(32 * g) << 16) + (uint32_t)c0, z);
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        const int f = f0 + c0 + c;
        if (f < G.n_forms && i < G.n_grid)
          G.gpart[((int64_t)L * G.f_pad + f) * G.n_pad + i] =
              ldexp((double)z[c], G.bexp[f]) * P.gw[(int64_t)f * P.n_Ltot + L];
      }
    }
  }
  if (!GRAD && ok && warp >= 1) {
    // epilogue: warp w reads TMEM lanes 32*(w%4).. (its lane quarter); the four warps of a quarter
    // split the columns
    const int g = warp & 3, h = (warp - 1) >> 2;
    const int row = 32 * g + lane;
    const int i = i0 + row;
    for (int c0 = h * (BN / 4); c0 < (h + 1) * (BN / 4); c0 += 32) {
      float z[32];
      tmem_ld32(tmem + ((uint32_t)(32 * g) << 16) + (uint32_t)c0, z);
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        // a_f[i] of column f: the lanes of a warp read 32 consecutive rows of one form
        const int f = f0 + c0 + c;
        double av = 0.0;
        if (f < G.n_forms) {
          const dwba_form_t F = G.forms[f];
          if (i < F.n_rows) av = ldexp(F.a_dev[i], G.bexp[f]);
        }
        double v = av * (double)z[c];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) sRed[g][c0 + c] = v;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (!GRAD && ok) {
    for (int c = tid; c < BN; c += THREADS) {
      const double v = sRed[0][c] + sRed[1][c] + sRed[2][c] + sRed[3][c];
      G.partial[((int64_t)L * G.n_iblk + iblk) * G.f_pad + f0 + c] = v;
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TMEM_COLS));
  }
}

// ---- operand preparation and reduction -----------------------------------------------
// Per-form exponent e_f with 2^-e_f max|b_f| in [0.5, 1): the split then works at unit scale
// whatever the magnitude of b_f (power-of-two scaling is exact).
__global__ void tc_scale_kernel(const dwba_form_t* __restrict__ forms, int n_forms, int* __restrict__ bexp) {
  __shared__ double red[8];
  const int f = blockIdx.x;
  const dwba_form_t F = forms[f];
  double m = 0.0;
  for (int j = threadIdx.x; j < F.n_cols; j += blockDim.x) m = fmax(m, fabs(F.b_dev[j]));
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mm = fmax(mm, red[w]);
    int e = 0;
    if (mm > 0.0 && isfinite(mm)) frexp(mm, &e);
    bexp[f] = e;
  }
}

// b_f -> NT bf16 terms in [NT][f_pad][n_pad] (zero padded): t_0 = bf16(b'), t_1 = bf16(b' - t_0), ...,
// b' = 2^-e_f b_f
// (ld: row stride of bterms, >= n_pad; columns n_pad .. ld-1 are not touched)
template <int NT>
__global__ void tc_prepare_kernel(const dwba_form_t* __restrict__ forms, int n_forms, int n_pad, int f_pad,
                                  const int* __restrict__ bexp, __nv_bfloat16* __restrict__ bterms, int64_t ld) {
  const int64_t total = (int64_t)f_pad * n_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (int64_t)gridDim.x * blockDim.x) {
    const int f = (int)(idx / n_pad), j = (int)(idx - (int64_t)f * n_pad);
    double b = 0.0;
    if (f < n_forms) {
      const dwba_form_t F = forms[f];
      if (j < F.n_cols) b = ldexp(F.b_dev[j], -bexp[f]);
    }
    float rem = (float)b;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const __nv_bfloat16 q = __float2bfloat16_rn(rem);
      rem -= __bfloat162float(q);
      bterms[((int64_t)t * f_pad + f) * ld + j] = q;
    }
  }
}

__global__ void tc_log2_kernel(const double* __restrict__ r, int n, double* __restrict__ lg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) lg[i] = log2(r[i]);
}

// Rank-one factor tables (FP64 exp2 of log2 differences, rounded once to FP32):
//   vt[0][L][j] = (r_j/c_b)^L, vt[1][L][j] = (r_j/c_b)^-(L+1), c_b = first radius of j's block;
//   st[L][iblk][kb] = (c_b/c_lo)^L below the diagonal, c_hi^L / c_b^(L+1) above, 0 when the j block
//   touches the row block.
__global__ void tc_factors_kernel(const double* __restrict__ lg, int n_grid, int n_pad, int n_kb, int n_iblk,
                                  int n_L, float* __restrict__ vt, float* __restrict__ st) {
  const int64_t n_v = 2LL * n_L * n_pad, n_s = (int64_t)n_L * n_iblk * n_kb;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n_v + n_s;
       idx += (int64_t)gridDim.x * blockDim.x) {
    if (idx < n_v) {
      const int j = (int)(idx % n_pad);
      const int64_t tl = idx / n_pad;
      const int L = (int)(tl % n_L), t = (int)(tl / n_L);
      float v = 0.0f;
      if (j < n_grid) {
        const double d = lg[j] - lg[(j / BK) * BK];
        v = (float)(t == 0 ? exp2((double)L * d) : exp2(-(double)(L + 1) * d));
      }
      vt[idx] = v;
    } else {
      const int64_t q = idx - n_v;
      const int kb = (int)(q % n_kb);
      const int64_t li = q / n_kb;
      const int iblk = (int)(li % n_iblk), L = (int)(li / n_iblk);
      const int i0 = iblk * BM, j0 = kb * BK;
      const double lg_lo = lg[i0], lg_hi = lg[min(i0 + BM, n_grid) - 1], lgc = lg[j0];
      float v = 0.0f;
      if (j0 + BK - 1 < i0) v = (float)exp2((double)L * (lgc - lg_lo));
      else if (j0 > i0 + BM - 1) v = (float)exp2((double)L * lg_hi - (double)(L + 1) * lgc);
      st[q] = v;
    }
  }
}

__global__ void tc_reduce_kernel(const double* __restrict__ partial, int n_forms, int f_pad, int n_iblk, int n_L,
                                 double* __restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n_forms * n_L) return;
  const int f = (int)(idx / n_L), L = (int)(idx - (int64_t)f * n_L);
  double s = 0.0;
  for (int b = 0; b < n_iblk; ++b) s += partial[((int64_t)L * n_iblk + b) * f_pad + f];
  out[idx] = s;
}

// backward: the two form sets whose B operand is b (for dLoss/da) and a (for dLoss/db)
__global__ void tc_grad_forms_kernel(const dwba_form_grad_t* __restrict__ in, int n, dwba_form_t* __restrict__ for_a,
                                     dwba_form_t* __restrict__ for_b) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  const dwba_form_grad_t G = in[f];
  for_a[f].r_dev = G.r_dev;
  for_a[f].a_dev = G.a_dev;
  for_a[f].b_dev = G.b_dev;
  for_a[f].n_rows = G.n_rows;
  for_a[f].n_cols = G.n_cols;
  for_b[f].r_dev = G.r_dev;
  for_b[f].a_dev = G.b_dev;
  for_b[f].b_dev = G.a_dev;
  for_b[f].n_rows = G.n_cols;
  for_b[f].n_cols = G.n_rows;
}

// ga_f[i] (which = 0, i < n_rows) or gb_f[i] (which = 1, i < n_cols) = sum over L of the partials
__global__ void tc_grad_reduce_kernel(const double* __restrict__ gpart, const dwba_form_grad_t* __restrict__ forms,
                                      int n_forms, int f_pad, int n_pad, int n_L, int which) {
  const int64_t total = (int64_t)n_forms * n_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int f = (int)(idx / n_pad), i = (int)(idx - (int64_t)f * n_pad);
    const dwba_form_grad_t& G = forms[f];
    const int len = which == 0 ? G.n_rows : G.n_cols;
    if (i >= len) continue;
    double s = 0.0;
    for (int L = 0; L < n_L; ++L) s += gpart[((int64_t)L * f_pad + f) * n_pad + i];
    (which == 0 ? G.ga_dev : G.gb_dev)[i] = s;
  }
}

// bound of the pipeline waits of the next launches (process-wide; 0 = WAIT_CYCLES)
std::atomic<long long> g_wait_cycles{0};
// serialises the host-side assembly of the (large) segment tables of the launches
std::mutex g_launch_mutex;

long long wait_cycles() {
  const long long c = g_wait_cycles.load();
  return c > 0 ? c : WAIT_CYCLES;
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// One launch over the segments of SG: B terms of every segment in one bf16 matrix of `ld` columns
// and `rows` rows (one tensor map), `n_ctas` CTAs in total.
template <int NT, int BN, bool GRAD = false, int SN = tc_stages(NT)>
int launch_tc_segs(const GemmParams& P, const TcSegs& SG, const __nv_bfloat16* bterms, int64_t ld, int64_t rows,
                   int64_t n_ctas, cudaStream_t st) {
  if (n_ctas <= 0) return DWBA_OK;
  if (n_ctas > 0x7fffffffLL) return DWBA_ERR_INVALID_ARG;
  auto encode = get_encode();
  if (!encode) return DWBA_ERR_CUDA;
  CUtensorMap map;
  cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)BN};
  cuuint32_t estr[2] = {1, 1};
  CUresult cr = encode(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)bterms, dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return DWBA_ERR_CUDA;
  const int smem = SN * NT * (BN * BK * 2) + 1024;
  if (cudaFuncSetAttribute(tc_exchange_kernel<NT, BN, GRAD, SN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
      cudaSuccess)
    return DWBA_ERR_CUDA;
  tc_exchange_kernel<NT, BN, GRAD, SN><<<(unsigned)n_ctas, THREADS, smem, st>>>(map, P, SG);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

// the one segment of a single-grid launch, from its parameters
void single_segment(const GemmParams& P, int bn, int n_L, TcSegs& SG) {
  SG.n = 1;
  SG.order = 0;
  TcSeg& g = SG.s[0];
  g.r = P.r;
  g.lg = P.lg;
  g.forms = P.forms;
  g.partial = P.partial;
  g.bexp = P.bexp;
  g.vt = P.vt;
  g.st = P.st;
  g.gpart = P.gpart;
  g.n_grid = P.n_grid;
  g.n_pad = P.n_pad;
  g.f_pad = P.f_pad;
  g.n_iblk = P.n_iblk;
  g.n_forms = P.n_forms;
  g.n_kb = P.n_kb;
  g.row0 = 0;
  g.n_fblk = P.f_pad / bn;
  SG.cta0[0] = 0;
  SG.cta0[1] = (int)((int64_t)P.n_iblk * g.n_fblk * n_L);
}

template <int NT, int BN, bool GRAD = false>
int launch_tc(const GemmParams& P, const __nv_bfloat16* bterms, int n_L, cudaStream_t st) {
  static TcSegs SG;  // ~10 KB: kept off the host stack (guarded by the launch mutex)
  std::lock_guard<std::mutex> lock(g_launch_mutex);
  const int64_t n_ctas = (int64_t)P.n_iblk * (P.f_pad / BN) * n_L;
  if (n_ctas > 0x7fffffffLL) return DWBA_ERR_INVALID_ARG;
  single_segment(P, BN, n_L, SG);
  return launch_tc_segs<NT, BN, GRAD>(P, SG, bterms, P.n_pad, (int64_t)NT * P.f_pad, n_ctas, st);
}

}  // namespace

extern "C" int64_t dwba_tc_workspace_bytes(int n_forms, int n_grid, int L_max, int n_terms) {
  if (n_forms < 0 || n_grid < 2 || L_max < 0 || L_max > DWBA_MAX_L || (n_terms != 2 && n_terms != 3)) return -1;
  const int bn = n_terms == 2 ? TC_BN2 : TC_BN3;
  const int64_t n_pad = ((int64_t)n_grid + BK - 1) / BK * BK;
  const int64_t f_pad = ((int64_t)n_forms + bn - 1) / bn * bn;
  const int64_t n_iblk = ((int64_t)n_grid + BM - 1) / BM;
  const int64_t b = (int64_t)n_terms * f_pad * n_pad * 2;
  const int64_t p = (int64_t)(L_max + 1) * n_iblk * f_pad * 8;
  const int64_t e = f_pad * 4;
  const int64_t lgb = n_pad * 8;
  const int64_t vtb = 2LL * (L_max + 1) * n_pad * 4;
  const int64_t stb = (int64_t)(L_max + 1) * n_iblk * (n_pad / BK) * 4;
  return ((b + 255) / 256 * 256) + ((p + 255) / 256 * 256) + ((e + 255) / 256 * 256) + ((lgb + 255) / 256 * 256) +
         ((vtb + 255) / 256 * 256) + stb;
}

extern "C" int dwba_bilinear_tc_bf16(const dwba_form_t* forms_dev, int n_forms, const double* r_dev, int n_grid,
                                     int L_max, int n_terms, const double* diag_scale_host, void* workspace,
                                     int64_t workspace_bytes, int* status_dev, double* out_dev,
                                     dwba_stream_t stream) {
  if (n_forms <= 0) return DWBA_OK;
  if (!forms_dev || !r_dev || !diag_scale_host || !workspace || !status_dev || !out_dev || n_grid < 2 || L_max < 0 ||
      L_max > DWBA_MAX_L || (n_terms != 2 && n_terms != 3) || n_grid > (1 << 24))
    return DWBA_ERR_INVALID_ARG;
  const int64_t need = dwba_tc_workspace_bytes(n_forms, n_grid, L_max, n_terms);
  if (need < 0 || workspace_bytes < need) return DWBA_ERR_WORKSPACE;
  if (((uintptr_t)workspace & 255) != 0) return DWBA_ERR_INVALID_ARG;
  const int bn = n_terms == 2 ? TC_BN2 : TC_BN3;
  GemmParams P;
  P.n_grid = n_grid;
  P.n_pad = (n_grid + BK - 1) / BK * BK;
  P.f_pad = (n_forms + bn - 1) / bn * bn;
  P.n_iblk = (n_grid + BM - 1) / BM;
  P.L_max = L_max;
  P.r = r_dev;
  P.forms = forms_dev;
  P.n_forms = n_forms;
  P.status = status_dev;
  P.gw = nullptr;
  P.gpart = nullptr;
  P.wait_cycles = wait_cycles();
  P.n_Ltot = L_max + 1;
  for (int l = 0; l <= DWBA_MAX_L; ++l) P.diag[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  uint8_t* ws = (uint8_t*)workspace;
  const int64_t bbytes = (int64_t)n_terms * P.f_pad * P.n_pad * 2;
  __nv_bfloat16* bterms = (__nv_bfloat16*)ws;
  P.partial = (double*)(ws + (bbytes + 255) / 256 * 256);
  const int64_t pbytes = (int64_t)(L_max + 1) * P.n_iblk * P.f_pad * 8;
  int* bexp = (int*)((uint8_t*)P.partial + (pbytes + 255) / 256 * 256);
  P.bexp = bexp;
  double* lg = (double*)((uint8_t*)bexp + ((int64_t)P.f_pad * 4 + 255) / 256 * 256);
  P.lg = lg;
  P.n_kb = P.n_pad / BK;
  float* vt = (float*)((uint8_t*)lg + ((int64_t)P.n_pad * 8 + 255) / 256 * 256);
  float* stab = (float*)((uint8_t*)vt + (2LL * (L_max + 1) * P.n_pad * 4 + 255) / 256 * 256);
  P.vt = vt;
  P.st = stab;
  if (P.f_pad / bn > 65535) return DWBA_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t total = (int64_t)P.f_pad * P.n_pad;
  tc_scale_kernel<<<n_forms, 256, 0, st>>>(forms_dev, n_forms, bexp);
  DWBA_CHECK_LAUNCH();
  tc_log2_kernel<<<dwba_grid_1d(n_grid, 256), 256, 0, st>>>(r_dev, n_grid, lg);
  DWBA_CHECK_LAUNCH();
  {
    const int64_t n_fac = 2LL * (L_max + 1) * P.n_pad + (int64_t)(L_max + 1) * P.n_iblk * P.n_kb;
    tc_factors_kernel<<<dwba_grid_1d(n_fac, 256, 65535), 256, 0, st>>>(lg, n_grid, P.n_pad, P.n_kb, P.n_iblk,
                                                                       L_max + 1, vt, stab);
    DWBA_CHECK_LAUNCH();
  }
  if (n_terms == 2)
    tc_prepare_kernel<2><<<dwba_grid_1d(total, 256, 65535), 256, 0, st>>>(forms_dev, n_forms, P.n_pad, P.f_pad,
                                                                          bexp, bterms, P.n_pad);
  else
    tc_prepare_kernel<3><<<dwba_grid_1d(total, 256, 65535), 256, 0, st>>>(forms_dev, n_forms, P.n_pad, P.f_pad,
                                                                          bexp, bterms, P.n_pad);
  DWBA_CHECK_LAUNCH();
  const int n_L = L_max + 1;
  int rc = n_terms == 2 ? launch_tc<2, TC_BN2>(P, bterms, n_L, st) : launch_tc<3, TC_BN3>(P, bterms, n_L, st);
  if (rc != DWBA_OK) return rc;
  tc_reduce_kernel<<<dwba_grid_1d((int64_t)n_forms * n_L, 256), 256, 0, st>>>(P.partial, n_forms, P.f_pad,
                                                                            P.n_iblk, n_L, out_dev);
  DWBA_CHECK_LAUNCH();
  return DWBA_OK;
}

// ---- ragged launch: forms on several grids in one tensor-core launch -----------------------
namespace {

int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }

struct SegLayout {
  int n_grid, n_pad, f_pad, n_iblk, n_kb, n_forms, row0;
  int64_t off_partial, off_bexp, off_lg, off_vt, off_st;
};

// default pipeline depth of a tile: the deepest that fits (tensor memory: bn + S NT 32 columns <= 512;
// shared memory: S NT bn 128 bytes)
int default_stages(int nt, int bn) { return nt == 2 ? (bn == 256 ? 3 : 4) : (bn == 256 ? 2 : 3); }

bool valid_tile(int nt, int bn, int stages) {
  if (bn != 128 && bn != 256) return false;
  if (nt == 2) return (bn == 256 && stages == 3) || (bn == 128 && (stages == 3 || stages == 4));
  return (bn == 256 && stages == 2) || (bn == 128 && (stages == 2 || stages == 3));
}

// the tile of a call (NULL: bn 256, default stages, row blocks fastest); false if invalid
bool resolve_tile(const dwba_tc_tile_t* tile, int nt, int& bn, int& stages, int& order) {
  bn = tile && tile->bn ? tile->bn : 256;
  stages = tile && tile->stages ? tile->stages : default_stages(nt, bn);
  order = tile ? tile->order : 0;
  return valid_tile(nt, bn, stages) && (order == 0 || order == 1);
}

// workspace layout of a ragged call: the B terms of all segments as one [rows][ld] bf16 matrix,
// then per segment its partials, exponents, log2 r and factor tables; returns the bytes (-1 if invalid)
int64_t ragged_layout(const dwba_tc_segment_t* segs, int n, int L_max, int nt, int bn, SegLayout* lay,
                      int64_t* ld_out, int64_t* rows_out) {
  int64_t ld = BK, rows = 0;
  for (int s = 0; s < n; ++s) {
    if (segs[s].n_forms < 0 || segs[s].n_grid < 2 || segs[s].n_grid > (1 << 24)) return -1;
    const int64_t n_pad = ((int64_t)segs[s].n_grid + BK - 1) / BK * BK;
    ld = n_pad > ld ? n_pad : ld;
  }
  const int64_t nL = L_max + 1;
  for (int s = 0; s < n; ++s) {
    SegLayout L{};
    L.n_grid = segs[s].n_grid;
    L.n_forms = segs[s].n_forms;
    L.n_pad = (L.n_grid + BK - 1) / BK * BK;
    L.f_pad = (int)(((int64_t)L.n_forms + bn - 1) / bn * bn);
    L.n_iblk = (L.n_grid + BM - 1) / BM;
    L.n_kb = L.n_pad / BK;
    L.row0 = (int)rows;
    rows += (int64_t)nt * L.f_pad;
    if (lay) lay[s] = L;
  }
  int64_t off = align256(rows * ld * 2);
  for (int s = 0; s < n; ++s) {
    const int64_t f_pad = ((int64_t)segs[s].n_forms + bn - 1) / bn * bn;
    const int64_t n_pad = ((int64_t)segs[s].n_grid + BK - 1) / BK * BK;
    const int64_t n_iblk = ((int64_t)segs[s].n_grid + BM - 1) / BM;
    if (lay) lay[s].off_partial = off;
    off += align256(nL * n_iblk * f_pad * 8);
    if (lay) lay[s].off_bexp = off;
    off += align256(f_pad * 4);
    if (lay) lay[s].off_lg = off;
    off += align256(n_pad * 8);
    if (lay) lay[s].off_vt = off;
    off += align256(2 * nL * n_pad * 4);
    if (lay) lay[s].off_st = off;
    off += align256(nL * n_iblk * (n_pad / BK) * 4);
  }
  if (rows > 0x7fffffffLL) return -1;
  if (ld_out) *ld_out = ld;
  if (rows_out) *rows_out = rows;
  return off;
}

int launch_variant(int nt, int bn, int stages, const GemmParams& P, const TcSegs& SG, const __nv_bfloat16* bterms,
                   int64_t ld, int64_t rows, int64_t n_ctas, cudaStream_t st) {
  if (nt == 2) {
    if (bn == 256) return launch_tc_segs<2, 256, false, 3>(P, SG, bterms, ld, rows, n_ctas, st);
    if (stages == 3) return launch_tc_segs<2, 128, false, 3>(P, SG, bterms, ld, rows, n_ctas, st);
    return launch_tc_segs<2, 128, false, 4>(P, SG, bterms, ld, rows, n_ctas, st);
  }
  if (bn == 256) return launch_tc_segs<3, 256, false, 2>(P, SG, bterms, ld, rows, n_ctas, st);
  if (stages == 2) return launch_tc_segs<3, 128, false, 2>(P, SG, bterms, ld, rows, n_ctas, st);
  return launch_tc_segs<3, 128, false, 3>(P, SG, bterms, ld, rows, n_ctas, st);
}

}  // namespace

extern "C" int64_t dwba_tc_ragged_workspace_bytes(const dwba_tc_segment_t* segs_host, int n_segs, int L_max,
                                                  int n_terms, const dwba_tc_tile_t* tile) {
  if (!segs_host || n_segs < 0 || L_max < 0 || L_max > DWBA_MAX_L || (n_terms != 2 && n_terms != 3)) return -1;
  int bn, stages, order;
  if (!resolve_tile(tile, n_terms, bn, stages, order)) return -1;
  return ragged_layout(segs_host, n_segs, L_max, n_terms, bn, nullptr, nullptr, nullptr);
}

extern "C" int dwba_bilinear_tc_bf16_ragged(const dwba_tc_segment_t* segs_host, int n_segs, int L_max, int n_terms,
                                            const dwba_tc_tile_t* tile, const double* diag_scale_host,
                                            void* workspace, int64_t workspace_bytes, int* status_dev,
                                            dwba_stream_t stream) {
  if (n_segs == 0) return DWBA_OK;
  if (!segs_host || n_segs < 0 || !diag_scale_host || !workspace || !status_dev || L_max < 0 || L_max > DWBA_MAX_L ||
      (n_terms != 2 && n_terms != 3))
    return DWBA_ERR_INVALID_ARG;
  int bn, stages, order;
  if (!resolve_tile(tile, n_terms, bn, stages, order)) return DWBA_ERR_INVALID_ARG;
  for (int s = 0; s < n_segs; ++s)
    if (segs_host[s].n_forms > 0 && (!segs_host[s].forms_dev || !segs_host[s].r_dev || !segs_host[s].out_dev))
      return DWBA_ERR_INVALID_ARG;
  if (((uintptr_t)workspace & 255) != 0) return DWBA_ERR_INVALID_ARG;
  std::vector<SegLayout> lay(n_segs);
  int64_t ld = 0, rows = 0;
  const int64_t need = ragged_layout(segs_host, n_segs, L_max, n_terms, bn, lay.data(), &ld, &rows);
  if (need < 0) return DWBA_ERR_INVALID_ARG;
  if (workspace_bytes < need) return DWBA_ERR_WORKSPACE;
  uint8_t* ws = (uint8_t*)workspace;
  __nv_bfloat16* bterms = (__nv_bfloat16*)ws;
  cudaStream_t st = (cudaStream_t)stream;
  const int n_L = L_max + 1;
  // per segment: exponents, log2 r, factor tables, bf16 terms of b (rows row0 .. of the shared matrix)
  for (int s = 0; s < n_segs; ++s) {
    const dwba_tc_segment_t& G = segs_host[s];
    const SegLayout& L = lay[s];
    if (G.n_forms == 0) continue;
    int* bexp = (int*)(ws + L.off_bexp);
    double* lg = (double*)(ws + L.off_lg);
    float* vt = (float*)(ws + L.off_vt);
    float* stab = (float*)(ws + L.off_st);
    tc_scale_kernel<<<G.n_forms, 256, 0, st>>>(G.forms_dev, G.n_forms, bexp);
    DWBA_CHECK_LAUNCH();
    tc_log2_kernel<<<dwba_grid_1d(G.n_grid, 256), 256, 0, st>>>(G.r_dev, G.n_grid, lg);
    DWBA_CHECK_LAUNCH();
    const int64_t n_fac = 2LL * n_L * L.n_pad + (int64_t)n_L * L.n_iblk * L.n_kb;
    tc_factors_kernel<<<dwba_grid_1d(n_fac, 256, 65535), 256, 0, st>>>(lg, G.n_grid, L.n_pad, L.n_kb, L.n_iblk, n_L,
                                                                       vt, stab);
    DWBA_CHECK_LAUNCH();
    const int64_t total = (int64_t)L.f_pad * L.n_pad;
    __nv_bfloat16* bt = bterms + (int64_t)L.row0 * ld;
    if (n_terms == 2)
      tc_prepare_kernel<2><<<dwba_grid_1d(total, 256, 65535), 256, 0, st>>>(G.forms_dev, G.n_forms, L.n_pad, L.f_pad,
                                                                            bexp, bt, ld);
    else
      tc_prepare_kernel<3><<<dwba_grid_1d(total, 256, 65535), 256, 0, st>>>(G.forms_dev, G.n_forms, L.n_pad, L.f_pad,
                                                                            bexp, bt, ld);
    DWBA_CHECK_LAUNCH();
  }
  // the tensor-core launches: segments by decreasing grid size (the longest CTAs start first), at
  // most TC_MAX_SEGS per launch
  std::vector<int> ord;
  for (int s = 0; s < n_segs; ++s)
    if (segs_host[s].n_forms > 0) ord.push_back(s);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return segs_host[a].n_grid > segs_host[b].n_grid; });
  GemmParams P{};
  P.status = status_dev;
  P.gw = nullptr;
  P.gpart = nullptr;
  P.wait_cycles = wait_cycles();
  P.L_max = L_max;
  P.n_Ltot = n_L;
  for (int l = 0; l <= DWBA_MAX_L; ++l) P.diag[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  {
    static TcSegs SG;  // ~10 KB: kept off the host stack (guarded by the launch mutex)
    std::lock_guard<std::mutex> lock(g_launch_mutex);
    for (size_t c0 = 0; c0 < ord.size(); c0 += TC_MAX_SEGS) {
      const int m = (int)std::min<size_t>(TC_MAX_SEGS, ord.size() - c0);
      SG.n = m;
      SG.order = order;
      int64_t ctas = 0;
      for (int q = 0; q < m; ++q) {
        const int s = ord[c0 + q];
        const dwba_tc_segment_t& G = segs_host[s];
        const SegLayout& L = lay[s];
        TcSeg& g = SG.s[q];
        g.r = G.r_dev;
        g.lg = (const double*)(ws + L.off_lg);
        g.forms = G.forms_dev;
        g.partial = (double*)(ws + L.off_partial);
        g.bexp = (const int*)(ws + L.off_bexp);
        g.vt = (const float*)(ws + L.off_vt);
        g.st = (const float*)(ws + L.off_st);
        g.gpart = nullptr;
        g.n_grid = L.n_grid;
        g.n_pad = L.n_pad;
        g.f_pad = L.f_pad;
        g.n_iblk = L.n_iblk;
        g.n_forms = L.n_forms;
        g.n_kb = L.n_kb;
        g.row0 = L.row0;
        g.n_fblk = L.f_pad / bn;
        SG.cta0[q] = (int)ctas;
        ctas += (int64_t)L.n_iblk * g.n_fblk * n_L;
        if (ctas > 0x7fffffffLL) return DWBA_ERR_INVALID_ARG;
      }
      SG.cta0[m] = (int)ctas;
      const int rc = launch_variant(n_terms, bn, stages, P, SG, bterms, ld, rows, ctas, st);
      if (rc != DWBA_OK) return rc;
    }
  }
  // per segment: the partials summed in fixed order into the segment's results
  for (int s = 0; s < n_segs; ++s) {
    const dwba_tc_segment_t& G = segs_host[s];
    const SegLayout& L = lay[s];
    if (G.n_forms == 0) continue;
    tc_reduce_kernel<<<dwba_grid_1d((int64_t)G.n_forms * n_L, 256), 256, 0, st>>>(
        (const double*)(ws + L.off_partial), G.n_forms, L.f_pad, L.n_iblk, n_L, G.out_dev);
    DWBA_CHECK_LAUNCH();
  }
  return DWBA_OK;
}

// ---- backward ------------------------------------------------------------------------

extern "C" int64_t dwba_tc_backward_workspace_bytes(int n_forms, int n_grid, int L_max, int n_terms) {
  if (n_forms < 0 || n_grid < 2 || L_max < 0 || L_max > DWBA_MAX_L || (n_terms != 2 && n_terms != 3)) return -1;
  const int bn = n_terms == 2 ? TC_BN2 : TC_BN3;
  const int64_t n_pad = ((int64_t)n_grid + BK - 1) / BK * BK;
  const int64_t f_pad = ((int64_t)n_forms + bn - 1) / bn * bn;
  const int64_t n_iblk = ((int64_t)n_grid + BM - 1) / BM;
  const int64_t nL = L_max + 1;
  return align256((int64_t)n_terms * f_pad * n_pad * 2) + align256(nL * f_pad * n_pad * 8) + align256(f_pad * 4) +
         align256(n_pad * 8) + align256(2 * nL * n_pad * 4) + align256(nL * n_iblk * (n_pad / BK) * 4) +
         2 * align256((int64_t)n_forms * (int64_t)sizeof(dwba_form_t));
}

extern "C" int dwba_bilinear_tc_bf16_backward(const dwba_form_grad_t* forms_dev, int n_forms, const double* r_dev,
                                              int n_grid, int L_max, int n_terms, const double* diag_scale_host,
                                              const double* grad_dev, void* workspace, int64_t workspace_bytes,
                                              int* status_dev, dwba_stream_t stream) {
  if (n_forms <= 0) return DWBA_OK;
  if (!forms_dev || !r_dev || !diag_scale_host || !grad_dev || !workspace || !status_dev || n_grid < 2 ||
      L_max < 0 || L_max > DWBA_MAX_L || (n_terms != 2 && n_terms != 3) || n_grid > (1 << 24))
    return DWBA_ERR_INVALID_ARG;
  const int64_t need = dwba_tc_backward_workspace_bytes(n_forms, n_grid, L_max, n_terms);
  if (need < 0 || workspace_bytes < need) return DWBA_ERR_WORKSPACE;
  if (((uintptr_t)workspace & 255) != 0) return DWBA_ERR_INVALID_ARG;
  const int bn = n_terms == 2 ? TC_BN2 : TC_BN3;
  const int n_L = L_max + 1;
  GemmParams P;
  P.n_grid = n_grid;
  P.n_pad = (n_grid + BK - 1) / BK * BK;
  P.f_pad = (n_forms + bn - 1) / bn * bn;
  P.n_iblk = (n_grid + BM - 1) / BM;
  P.L_max = L_max;
  P.r = r_dev;
  P.n_forms = n_forms;
  P.status = status_dev;
  P.gw = grad_dev;
  P.wait_cycles = wait_cycles();
  P.n_Ltot = n_L;
  P.partial = nullptr;
  for (int l = 0; l <= DWBA_MAX_L; ++l) P.diag[l] = l <= L_max ? diag_scale_host[l] : 0.0;
  if (P.f_pad / bn > 65535) return DWBA_ERR_INVALID_ARG;
  uint8_t* ws = (uint8_t*)workspace;
  __nv_bfloat16* bterms = (__nv_bfloat16*)ws;
  ws += align256((int64_t)n_terms * P.f_pad * P.n_pad * 2);
  P.gpart = (double*)ws;
  ws += align256((int64_t)n_L * P.f_pad * P.n_pad * 8);
  int* bexp = (int*)ws;
  P.bexp = bexp;
  ws += align256((int64_t)P.f_pad * 4);
  double* lg = (double*)ws;
  P.lg = lg;
  ws += align256((int64_t)P.n_pad * 8);
  P.n_kb = P.n_pad / BK;
  float* vt = (float*)ws;
  ws += align256(2LL * n_L * P.n_pad * 4);
  float* stab = (float*)ws;
  ws += align256((int64_t)n_L * P.n_iblk * P.n_kb * 4);
  dwba_form_t* for_a = (dwba_form_t*)ws;
  ws += align256((int64_t)n_forms * (int64_t)sizeof(dwba_form_t));
  dwba_form_t* for_b = (dwba_form_t*)ws;
  P.vt = vt;
  P.st = stab;
  cudaStream_t st = (cudaStream_t)stream;
  tc_grad_forms_kernel<<<dwba_grid_1d(n_forms, 256), 256, 0, st>>>(forms_dev, n_forms, for_a, for_b);
  DWBA_CHECK_LAUNCH();
  tc_log2_kernel<<<dwba_grid_1d(n_grid, 256), 256, 0, st>>>(r_dev, n_grid, lg);
  DWBA_CHECK_LAUNCH();
  {
    const int64_t n_fac = 2LL * n_L * P.n_pad + (int64_t)n_L * P.n_iblk * P.n_kb;
    tc_factors_kernel<<<dwba_grid_1d(n_fac, 256, 65535), 256, 0, st>>>(lg, n_grid, P.n_pad, P.n_kb, P.n_iblk, n_L,
                                                                       vt, stab);
    DWBA_CHECK_LAUNCH();
  }
  const int64_t total = (int64_t)P.f_pad * P.n_pad;
  for (int which = 0; which < 2; ++which) {
    const dwba_form_t* fs = which == 0 ? for_a : for_b;
    P.forms = fs;
    tc_scale_kernel<<<n_forms, 256, 0, st>>>(fs, n_forms, bexp);
    DWBA_CHECK_LAUNCH();
    if (n_terms == 2)
      tc_prepare_kernel<2><<<dwba_grid_1d(total, 256, 65535), 256, 0, st>>>(fs, n_forms, P.n_pad, P.f_pad, bexp,
                                                                            bterms, P.n_pad);
    else
      tc_prepare_kernel<3><<<dwba_grid_1d(total, 256, 65535), 256, 0, st>>>(fs, n_forms, P.n_pad, P.f_pad, bexp,
                                                                            bterms, P.n_pad);
    DWBA_CHECK_LAUNCH();
    int rc = n_terms == 2 ? launch_tc<2, TC_BN2, true>(P, bterms, n_L, st)
                          : launch_tc<3, TC_BN3, true>(P, bterms, n_L, st);
    if (rc != DWBA_OK) return rc;
    tc_grad_reduce_kernel<<<dwba_grid_1d((int64_t)n_forms * P.n_pad, 256, 65535), 256, 0, st>>>(
        P.gpart, forms_dev, n_forms, P.f_pad, P.n_pad, n_L, which);
    DWBA_CHECK_LAUNCH();
  }
  return DWBA_OK;
}

extern "C" int dwba_tc_set_wait_cycles(int64_t cycles) {
  if (cycles < 0) return DWBA_ERR_INVALID_ARG;
  g_wait_cycles.store((long long)cycles);
  return DWBA_OK;
}
