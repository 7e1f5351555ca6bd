// Tensor-core response fold on sm_100a (tcgen05 + TMEM).
//
// counts[job][ch][b] = alpha_job * sum_E rsp[ch][E] * flux[job][b][E]
// (cpu/devarshi24st_cpu.cpp:249-258; the reference runs it as one cublasSgemm,
// gpu/matmul.cuh:12-36).  Both operands are split into BF16 hi/lo parts of
// their FP32 value and multiplied as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory.
//
// As a GEMM, D[rows][channels] = flux[rows][E] x rsp^T[E][channels] with one
// row per (job, bin).  The flux pool is the only large operand (FP64, read
// once) and the counts the only large result, so the fold is bound by HBM:
//   * one CTA (8 warps, two CTAs per SM) owns a tile of 128 rows (UMMA M) and
//     one group of up to 256 channels (UMMA N; the response's channels are
//     split into equal groups, a multiple of 32 each), over all energies in
//     chunks of 32 (two K = 16 steps);
//   * the response (B) is pre-split and pre-laid-out at engine set-up in the
//     UMMA K-major core-matrix layout and brought into shared memory by one
//     bulk copy (TMA) per chunk and part;
//   * the flux rows (A) are loaded by all threads with coalesced 16-byte loads
//     (four threads per row, eight rows per warp), two chunks ahead in
//     registers, split to BF16 hi/lo and stored into the same layout;
//   * two shared-memory stages of A and B: while the tensor cores multiply
//     chunk c, the threads convert chunk c + 1 and the loads of chunk c + 2
//     and the bulk copy of chunk c + 1 are in flight.  Copies and MMAs
//     complete on separate mbarriers; one elected thread issues 2 k-steps x 3
//     products of tcgen05.mma.cta_group::1.kind::f16 per chunk;
//   * every wait has an iteration limit; a wait that runs out sets an error
//     word, and the CTA waits (bounded) for its own copies and MMAs in flight,
//     releases its tensor memory and returns;
//   * the epilogue reads the accumulator with tcgen05.ld 32x32b (warps 0-3 and
//     4-7 take one half of the channel columns each), scales each row by its
//     job's exposure / n_bins and writes FP64 counts, 32 consecutive bins of a
//     channel per warp store.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "engine.h"

namespace ppm {

namespace {

constexpr int TC_M = 128;     // (job, bin) rows per tile (UMMA M)
constexpr int TC_KC = 32;     // energies per shared-memory stage
constexpr int TC_NMAX = 256;  // channels per group (UMMA N <= 256)
constexpr int TC_THREADS = 256;
constexpr int A_PART = TC_M * TC_KC * 2;  // bytes of one BF16 part (hi or lo) of a flux stage
constexpr int LBO_A = (TC_M / 8) * 128;   // bytes between core matrices adjacent in K
constexpr int SBO = 128;                  // bytes between core matrices adjacent in M / N
constexpr int kWaitLimit = 1 << 22;

__host__ __device__ constexpr int b_part_bytes(int ng) { return ng * TC_KC * 2; }
// dynamic shared memory of a launch: two stages of A (hi, lo) and B (hi, lo), 1 KB alignment slack
__host__ __device__ constexpr int fold_smem_bytes(int ng) { return 1024 + 2 * (2 * A_PART) + 2 * (2 * b_part_bytes(ng)); }
constexpr int SMEM_MAX = fold_smem_bytes(TC_NMAX);

__host__ __device__ constexpr uint32_t idesc(int n) {
  return (1u << 4)                         // D: FP32
         | (1u << 7)                       // A: BF16
         | (1u << 10)                      // B: BF16 (both K-major)
         | ((uint32_t)(n >> 3) << 17)      // N / 8
         | ((uint32_t)(TC_M >> 4) << 24);  // M / 16
}

// byte offset of element (r, k) of an R-row x 32-k tile: 8x16-byte core
// matrices, K-major, no swizzle, core matrices ordered k-group major
__host__ __device__ inline uint32_t cm_offset(int r, int k, int R) {
  return (uint32_t)(((k >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100; base offset 0, no swizzle
  return d;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ uint32_t bf16_bits(__nv_bfloat16 h) {
  uint16_t u;
  memcpy(&u, &h, 2);
  return u;
}

struct TcArgs {
  const uint16_t* b_hi;  // [groups][k_chunks][ng x TC_KC] core-matrix layout
  const uint16_t* b_lo;
  int n_ch, n_e, ng, k_chunks, n_bins, n_jobs;
  const FoldJob* jobs;
  const double* flux;
  double* counts;
  int* error;
  // failure-path test: > 0 issues no bulk copy and no MMA and waits at most this many
  // polls, so the first wait runs out and the kernel reports it through *error
  int stall_wait_limit;
};

// Eight consecutive energies k0 .. k0 + 7 of one flux row (zeros past n_e or for no row).
struct Row8 {
  double v[8];
};
__device__ __forceinline__ void load_row8(const double* src, bool vec, int k0, int n_e, Row8& r) {
  if (src && vec && k0 + 8 <= n_e) {
    const double2* p = reinterpret_cast<const double2*>(src + k0);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double2 t = __ldg(p + i);
      r.v[2 * i] = t.x;
      r.v[2 * i + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = (src && k0 + i < n_e) ? __ldg(src + k0 + i) : 0.0;
  }
}

// Splits eight values into BF16 hi / lo parts and stores them as one 16-byte
// row of a core matrix in each part.
__device__ __forceinline__ void store_row8(const Row8& r, unsigned char* hi, unsigned char* lo, uint32_t off) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float a = (float)r.v[2 * i], b = (float)r.v[2 * i + 1];
    const __nv_bfloat16 ha = __float2bfloat16_rn(a), hb = __float2bfloat16_rn(b);
    const __nv_bfloat16 la = __float2bfloat16_rn(a - __bfloat162float(ha)),
                        lb = __float2bfloat16_rn(b - __bfloat162float(hb));
    h[i] = bf16_bits(ha) | (bf16_bits(hb) << 16);
    l[i] = bf16_bits(la) | (bf16_bits(lb) << 16);
  }
  *(uint4*)(hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *(uint4*)(lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(TC_THREADS, 2) fold_tc_kernel(const TcArgs a) {
  extern __shared__ unsigned char sm_raw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)sm_raw + 1023) & ~(uintptr_t)1023);
  const int b_part = b_part_bytes(a.ng);
  // stage s: A hi, A lo, then B hi, B lo
  unsigned char* const sA0 = sm;
  unsigned char* const sB0 = sm + 4 * A_PART;
  __shared__ __align__(8) uint64_t bar_b[2], bar_mma[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = blockIdx.x;
  const int n0 = blockIdx.y * TC_M;
  const int rows_total = a.n_jobs * a.n_bins;
  const int nk = a.k_chunks;
  const bool stall = a.stall_wait_limit > 0;
  const int wait_limit = stall ? a.stall_wait_limit : kWaitLimit;
  const int tmem_cols = a.ng <= 32 ? 32 : (a.ng <= 64 ? 64 : (a.ng <= 128 ? 128 : 256));

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < 2; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar_b[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar_mma[s])));
    }
    asm volatile("fence.proxy.async.shared::cta;");
    s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  // this thread's two flux rows (rows r and r + 64 of the tile) and energy group
  const int kg = lane & 3;
  const int rl0 = 8 * warp + (lane >> 2), rl1 = rl0 + 64;
  const double* src0 = nullptr;
  const double* src1 = nullptr;
  {
    const int na = n0 + rl0, nb = n0 + rl1;
    if (na < rows_total) {
      const int j = na / a.n_bins, b = na - j * a.n_bins;
      src0 = a.flux + a.jobs[j].flux_off + (size_t)b * a.n_e;
    }
    if (nb < rows_total) {
      const int j = nb / a.n_bins, b = nb - j * a.n_bins;
      src1 = a.flux + a.jobs[j].flux_off + (size_t)b * a.n_e;
    }
  }
  const bool vec0 = ((uintptr_t)src0 & 15) == 0, vec1 = ((uintptr_t)src1 & 15) == 0;
  const uint32_t off0 = cm_offset(rl0, 8 * kg, TC_M), off1 = cm_offset(rl1, 8 * kg, TC_M);

  // bulk copy of the response chunk kc into stage s (elected thread)
  const size_t b_blk = (size_t)b_part / 2;  // uint16 elements per part and chunk
  auto issue_b = [&](int kc, int s) {
    const uint32_t bar = smem_u32(&bar_b[s]);
    unsigned char* dst = sB0 + s * 2 * b_part;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(2 * b_part) : "memory");
    const size_t blk = ((size_t)grp * nk + kc) * b_blk;
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(a.b_hi + blk), "r"(b_part), "r"(bar)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst + b_part)),
                 "l"(a.b_lo + blk), "r"(b_part), "r"(bar)
                 : "memory");
  };
  // the elected thread's bookkeeping: copies issued and not yet waited for, last chunk multiplied
  bool b_pending0 = false, b_pending1 = false;
  int mma_issued = -1;

  if (tid == 0 && !stall) {
    issue_b(0, 0);
    b_pending0 = true;
    if (nk > 1) {
      issue_b(1, 1);
      b_pending1 = true;
    }
  }
  // two register sets of flux rows: chunk c lives in set c & 1 until it is converted
  Row8 ra0, ra1, rb0, rb1;  // set 0 rows 0/1, set 1 rows 0/1
  load_row8(src0, vec0, 8 * kg, a.n_e, ra0);
  load_row8(src1, vec1, 8 * kg, a.n_e, ra1);
  if (nk > 1) {
    load_row8(src0, vec0, TC_KC + 8 * kg, a.n_e, rb0);
    load_row8(src1, vec1, TC_KC + 8 * kg, a.n_e, rb1);
  }

  const uint32_t id = idesc(a.ng);
  const uint32_t lbo_b = (uint32_t)(a.ng / 8) * 128;
  // one chunk: convert its register set into stage s, prefetch chunk c + 2 into the set, multiply chunk c
  auto chunk = [&](int c, Row8& r0, Row8& r1) -> bool {
    const int s = c & 1;
    unsigned char* ahi = sA0 + s * 2 * A_PART;
    unsigned char* alo = ahi + A_PART;
    unsigned char* bhi = sB0 + s * 2 * b_part;
    store_row8(r0, ahi, alo, off0);
    store_row8(r1, ahi, alo, off1);
    if (c + 2 < nk) {
      load_row8(src0, vec0, (c + 2) * TC_KC + 8 * kg, a.n_e, r0);
      load_row8(src1, vec1, (c + 2) * TC_KC + 8 * kg, a.n_e, r1);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      const bool ok = s_ok && mbar_wait(smem_u32(&bar_b[s]), (uint32_t)(c >> 1) & 1u, wait_limit);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ok) {
        if (s) b_pending1 = false; else b_pending0 = false;
        const uint32_t ah = smem_u32(ahi), al = smem_u32(alo), bh = smem_u32(bhi), bl = smem_u32(bhi + b_part);
#pragma unroll
        for (int ks = 0; ks < TC_KC / 16; ++ks) {
          const uint64_t dah = smem_desc(ah + ks * 2 * LBO_A, LBO_A, SBO), dal = smem_desc(al + ks * 2 * LBO_A, LBO_A, SBO);
          const uint64_t dbh = smem_desc(bh + ks * 2 * lbo_b, lbo_b, SBO), dbl = smem_desc(bl + ks * 2 * lbo_b, lbo_b, SBO);
          const uint64_t da[3] = {dah, dah, dal}, db[3] = {dbh, dbl, dbh};
#pragma unroll
          for (int pr = 0; pr < 3; ++pr) {
            const uint32_t accumulate = (c > 0 || ks > 0 || pr > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
                "l"(da[pr]), "l"(db[pr]), "r"(id), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
          }
        }
        // completion of everything issued so far arrives on bar_mma[s]
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&bar_mma[s]))
                     : "memory");
        mma_issued = c;
      } else {
        s_ok = 0;
      }
    }
    __syncthreads();
    if (!s_ok) return false;
    // stage s ^ 1 is free once the MMAs of chunk c - 1 are done: then chunk c + 1's copy may land there
    if (c >= 1) {
      if (!mbar_wait(smem_u32(&bar_mma[s ^ 1]), (uint32_t)((c - 1) >> 1) & 1u, wait_limit)) s_ok = 0;
      if (tid == 0 && s_ok && c + 1 < nk) {
        issue_b(c + 1, s ^ 1);
        if (s) b_pending0 = true; else b_pending1 = true;
      }
    }
    return true;
  };

  bool ok = true;
  for (int c = 0; c < nk && ok; c += 2) {
    ok = chunk(c, ra0, ra1);
    if (ok && c + 1 < nk) ok = chunk(c + 1, rb0, rb1);
  }
  __syncthreads();
  if (s_ok) {
    // the last chunk's MMAs (and with them every earlier one) are done
    if (!mbar_wait(smem_u32(&bar_mma[(nk - 1) & 1]), (uint32_t)((nk - 1) >> 1) & 1u, wait_limit)) s_ok = 0;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_ok) {
    const int q = warp & 3, half = warp >> 2;
    const int r = 32 * q + lane, n = n0 + r;
    double* dst = nullptr;
    double alpha = 0.0;
    if (n < rows_total) {
      const int j = n / a.n_bins, b = n - j * a.n_bins;
      const FoldJob job = a.jobs[j];
      dst = a.counts + job.counts_off + b;
      alpha = job.alpha;
    }
    const int hw = a.ng / 2;  // columns per half (a multiple of 16)
    for (int c0 = half * hw; c0 < (half + 1) * hw; c0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (dst) {
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          const int ch = grp * a.ng + c0 + t;
          if (ch < a.n_ch) dst[(size_t)ch * a.n_bins] = (double)__uint_as_float(v[t]) * alpha;
        }
      }
    }
  } else if (tid == 0) {
    // a wait ran out: record it, then give this CTA's copies and MMAs in flight one more bounded wait.  A
    // pending copy of stage s carries the first chunk of that stage not yet multiplied: chunk kc lands in
    // stage kc & 1 with phase parity (kc >> 1) & 1.
    atomicExch(a.error, 1);
    for (int s = 0; s < 2; ++s)
      if (s ? b_pending1 : b_pending0) {
        int kc = s;
        while (kc <= mma_issued) kc += 2;
        mbar_wait(smem_u32(&bar_b[s]), (uint32_t)(kc >> 1) & 1u, kWaitLimit);
      }
    if (mma_issued >= 0) mbar_wait(smem_u32(&bar_mma[mma_issued & 1]), (uint32_t)(mma_issued >> 1) & 1u, kWaitLimit);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols));
}

// FP32 -> BF16 with round-to-nearest-even (bias method), finite inputs.
uint16_t host_bf16(float v) {
  uint32_t u;
  std::memcpy(&u, &v, 4);
  const uint32_t bias = 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)((u + bias) >> 16);
}
float host_bf16_to_float(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

}  // namespace

// Channel groups of the tensor-core fold: n_ch split into equal groups of at
// most 256 channels, each a multiple of 32 (the epilogue's two halves read
// whole 16-column blocks).
void fold_tc_groups(int n_ch, int* groups, int* ng) {
  const int g = (n_ch + TC_NMAX - 1) / TC_NMAX;
  const int per = (n_ch + g - 1) / g;
  *groups = g;
  *ng = (per + 31) / 32 * 32;
}

// Splits rsp into BF16 hi/lo and lays every (channel group, 32-energy chunk)
// block out contiguously in the core-matrix layout the kernel's bulk copies
// expect.
void Engine::fold_tc_prepare(Resp& r) {
  r.tc_ok = false;
  int groups = 0, ng = 0;
  fold_tc_groups(r.n_ch, &groups, &ng);
  const int k_chunks = (r.n_e + TC_KC - 1) / TC_KC;
  r.tc_groups = groups;
  r.tc_ng = ng;
  r.tc_k_chunks = k_chunks;
  const size_t blk = (size_t)b_part_bytes(ng) / 2;
  std::vector<uint16_t> hi((size_t)groups * k_chunks * blk, 0), lo(hi.size(), 0);
  for (int g = 0; g < groups; ++g)
    for (int kc = 0; kc < k_chunks; ++kc) {
      uint16_t* H = hi.data() + ((size_t)g * k_chunks + kc) * blk;
      uint16_t* L = lo.data() + ((size_t)g * k_chunks + kc) * blk;
      for (int cc = 0; cc < ng; ++cc)
        for (int k = 0; k < TC_KC; ++k) {
          const int ch = g * ng + cc, e = kc * TC_KC + k;
          const float v = (ch < r.n_ch && e < r.n_e) ? (float)r.h_rsp[(size_t)ch * r.n_e + e] : 0.0f;
          const uint16_t h = host_bf16(v);
          const uint16_t l = host_bf16(v - host_bf16_to_float(h));
          const uint32_t idx = cm_offset(cc, k, ng) / 2;
          H[idx] = h;
          L[idx] = l;
        }
    }
  void *dh = nullptr, *dl = nullptr;
  if (cudaMalloc(&dh, hi.size() * 2) != cudaSuccess || cudaMalloc(&dl, lo.size() * 2) != cudaSuccess) {
    if (dh) cudaFree(dh);
    throw Error(PPM_E_OOM, "fold operand allocation failed");
  }
  if (cudaMemcpy(dh, hi.data(), hi.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dl, lo.data(), lo.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(dh);
    cudaFree(dl);
    throw Error(PPM_E_CUDA, "fold operand upload failed");
  }
  track(dh);
  track(dl);
  r.d_b_hi = dh;
  r.d_b_lo = dl;
  r.tc_ok = true;
}

cudaError_t Engine::fold_tc_launch(const Resp& r, const FoldJob* jobs, int n_jobs, int n_bins, const double* flux,
                                   double* counts, cudaStream_t st, int* error) {
  cudaError_t e = once_per_device(1, [] {
    return cudaFuncSetAttribute(fold_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_MAX);
  });
  if (e != cudaSuccess) return e;
  TcArgs a{};
  a.b_hi = (const uint16_t*)r.d_b_hi;
  a.b_lo = (const uint16_t*)r.d_b_lo;
  a.n_ch = r.n_ch;
  a.n_e = r.n_e;
  a.ng = r.tc_ng;
  a.k_chunks = r.tc_k_chunks;
  a.n_bins = n_bins;
  a.flux = flux;
  a.counts = counts;
  a.error = error ? error : d_err;
  // PPM_FOLD_TC_STALL_TEST=<polls>: the failure-path test of the bounded waits (no copy or MMA is issued, so the
  // first wait runs out after that many polls and the call reports PPM_E_TIMEOUT)
  if (const char* v = std::getenv("PPM_FOLD_TC_STALL_TEST")) a.stall_wait_limit = std::max(0, std::atoi(v));
  // at most 65535 row tiles per launch (grid y): longer job lists go in several launches
  const int jobs_per_launch = std::max(1, (int)(65535ll * TC_M / n_bins));
  for (int j0 = 0; j0 < n_jobs; j0 += jobs_per_launch) {
    a.jobs = jobs + j0;
    a.n_jobs = std::min(jobs_per_launch, n_jobs - j0);
    const long long rows = (long long)a.n_jobs * n_bins;
    dim3 grid(r.tc_groups, (unsigned)((rows + TC_M - 1) / TC_M));
    fold_tc_kernel<<<grid, TC_THREADS, fold_smem_bytes(r.tc_ng), st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ppm
