// Tensor-core response fold on sm_100a (tcgen05 + TMEM).
//
// counts[job][ch][b] = alpha_job * sum_E rsp[ch][E] * flux[job][b][E]
// (cpu/devarshi24st_cpu.cpp:249-258; the reference runs it as one cublasSgemm,
// gpu/matmul.cuh:12-36).  Both operands are split into BF16 hi/lo parts of
// their FP32 value and multiplied as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory.
//
// One CTA (4 warps) computes a 128-channel x 128-(job, bin) tile over all of
// K (energies, padded to 64):
//   * the response tile (A) is pre-split and pre-laid-out at engine set-up in
//     the UMMA K-major core-matrix layout and brought into shared memory by a
//     bulk-copy (TMA) per 64-energy stage;
//   * the flux tile (B) is read as FP64, split to BF16 hi/lo and written into
//     the same layout by the threads;
//   * one elected thread issues 4 k-steps x 3 products of
//     tcgen05.mma.cta_group::1.kind::f16 (M=128, N=128, K=16) and commits to
//     an mbarrier; every wait has an iteration limit and sets an error word;
//   * the epilogue reads the accumulator with tcgen05.ld 32x32b and scales
//     each column by its job's exposure / n_bins.
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

constexpr int TC_M = 128;   // channels per tile (UMMA M)
constexpr int TC_N = 128;   // (job, bin) rows per tile (UMMA N)
constexpr int TC_KC = 64;   // energies per shared-memory stage
constexpr int A_BYTES = TC_M * TC_KC * 2;
constexpr int B_BYTES = TC_N * TC_KC * 2;
constexpr int LBO_A = (TC_M / 8) * 128;  // bytes between core matrices adjacent in K
constexpr int LBO_B = (TC_N / 8) * 128;
constexpr int SBO = 128;                 // bytes between core matrices adjacent in M / N
// The buffers use the first 64 KB; the allocation is twice that so that every
// address a descriptor can form stays inside the CTA's shared memory.
constexpr int SMEM_BYTES = 128 * 1024 + 1024;
constexpr uint32_t kIdesc = (1u << 4)                          // D: FP32
                            | (1u << 7)                        // A: BF16
                            | (1u << 10)                       // B: BF16
                            | ((uint32_t)(TC_N >> 3) << 17)    // N / 8
                            | ((uint32_t)(TC_M >> 4) << 24);   // M / 16
constexpr int kWaitLimit = 1 << 22;

// byte offset of element (r, k) of an R-row x 64-k tile: 8x16-byte core
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

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit = kWaitLimit) {
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

__device__ __forceinline__ uint16_t bf16_bits(__nv_bfloat16 h) {
  uint16_t u;
  memcpy(&u, &h, 2);
  return u;
}

struct TcArgs {
  const uint16_t* a_hi;  // [m_tiles][k_chunks][TC_M x TC_KC] core-matrix layout
  const uint16_t* a_lo;
  int n_ch, n_e, k_chunks, n_bins, n_jobs;
  const FoldJob* jobs;
  const double* flux;
  double* counts;
  int* error;
  // failure-path test: > 0 issues no bulk copy and no MMA and waits at most this many
  // polls, so the first wait runs out and the kernel reports it through *error
  int stall_wait_limit;
};

__global__ void __launch_bounds__(128, 1) fold_tc_kernel(const TcArgs a) {
  extern __shared__ unsigned char sm_raw[];
  unsigned char* sm = (unsigned char*)(((uintptr_t)sm_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA_hi = sm;
  unsigned char* sA_lo = sm + A_BYTES;
  unsigned char* sB_hi = sm + 2 * A_BYTES;
  unsigned char* sB_lo = sm + 2 * A_BYTES + B_BYTES;
  __shared__ __align__(8) uint64_t bar_tma, bar_mma;
  __shared__ uint32_t s_tmem;
  __shared__ int s_ok;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int mt = blockIdx.x;
  const int n0 = blockIdx.y * TC_N;
  const int rows_total = a.n_jobs * a.n_bins;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(TC_N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar_tma)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar_mma)));
    asm volatile("fence.proxy.async.shared::cta;");
    s_ok = 1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;

  // this thread's flux row
  const int n = n0 + tid;
  const double* src = nullptr;
  if (n < rows_total) {
    const int j = n / a.n_bins, b = n - j * a.n_bins;
    src = a.flux + a.jobs[j].flux_off + (size_t)b * a.n_e;
  }

  const bool stall = a.stall_wait_limit > 0;
  const int wait_limit = stall ? a.stall_wait_limit : kWaitLimit;
  uint32_t parity = 0;
  for (int kc = 0; kc < a.k_chunks; ++kc) {
    if (tid == 0 && !stall) {
      const uint32_t bar = smem_u32(&bar_tma);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(2 * A_BYTES) : "memory");
      const size_t blk = ((size_t)mt * a.k_chunks + kc) * (A_BYTES / 2);
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                       smem_u32(sA_hi)),
                   "l"(a.a_hi + blk), "r"(A_BYTES), "r"(bar)
                   : "memory");
      asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                       smem_u32(sA_lo)),
                   "l"(a.a_lo + blk), "r"(A_BYTES), "r"(bar)
                   : "memory");
    }
    // flux row segment -> BF16 hi/lo in the core-matrix layout
    for (int kk = 0; kk < TC_KC; kk += 8) {
      uint16_t hi[8], lo[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int k = kc * TC_KC + kk + t;
        const float v = (src && k < a.n_e) ? (float)src[k] : 0.0f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
        hi[t] = bf16_bits(h);
        lo[t] = bf16_bits(l);
      }
      const uint32_t off = cm_offset(tid, kk, TC_N);
      uint4 vh, vl;
      vh.x = hi[0] | ((uint32_t)hi[1] << 16);
      vh.y = hi[2] | ((uint32_t)hi[3] << 16);
      vh.z = hi[4] | ((uint32_t)hi[5] << 16);
      vh.w = hi[6] | ((uint32_t)hi[7] << 16);
      vl.x = lo[0] | ((uint32_t)lo[1] << 16);
      vl.y = lo[2] | ((uint32_t)lo[3] << 16);
      vl.z = lo[4] | ((uint32_t)lo[5] << 16);
      vl.w = lo[6] | ((uint32_t)lo[7] << 16);
      *(uint4*)(sB_hi + off) = vh;
      *(uint4*)(sB_lo + off) = vl;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      bool ok = s_ok && mbar_wait(smem_u32(&bar_tma), parity, wait_limit);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (ok) {
        const uint32_t ah = smem_u32(sA_hi), al = smem_u32(sA_lo), bh = smem_u32(sB_hi), bl = smem_u32(sB_lo);
#pragma unroll
        for (int ks = 0; ks < TC_KC / 16; ++ks) {
          const uint64_t dah = smem_desc(ah + ks * 2 * LBO_A, LBO_A, SBO), dal = smem_desc(al + ks * 2 * LBO_A, LBO_A, SBO);
          const uint64_t dbh = smem_desc(bh + ks * 2 * LBO_B, LBO_B, SBO), dbl = smem_desc(bl + ks * 2 * LBO_B, LBO_B, SBO);
          const uint32_t acc0 = (kc > 0 || ks > 0) ? 1u : 0u;
          const uint64_t da[3] = {dah, dah, dal}, db[3] = {dbh, dbl, dbh};
#pragma unroll
          for (int pr = 0; pr < 3; ++pr) {
            const uint32_t accumulate = pr > 0 ? 1u : acc0;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem),
                "l"(da[pr]), "l"(db[pr]), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
          }
        }
      } else {
        s_ok = 0;
      }
      // completion of everything issued so far arrives on bar_mma
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&bar_mma))
                   : "memory");
    }
    if (!mbar_wait(smem_u32(&bar_mma), parity, wait_limit)) s_ok = 0;
    parity ^= 1u;
    __syncthreads();
    if (!s_ok) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_ok) {
    const int ch = mt * TC_M + warp * 32 + lane;
    for (int c0 = 0; c0 < TC_N; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const int nn = n0 + c0 + t;
        if (ch < a.n_ch && nn < rows_total) {
          const int j = nn / a.n_bins, b = nn - j * a.n_bins;
          const FoldJob job = a.jobs[j];
          a.counts[job.counts_off + (size_t)ch * a.n_bins + b] = (double)__uint_as_float(r[t]) * job.alpha;
        }
      }
    }
  } else {
    // a wait ran out: record it, give in-flight MMAs one more bounded wait, then release TMEM
    if (tid == 0) atomicExch(a.error, 1);
    mbar_wait(smem_u32(&bar_mma), parity, wait_limit);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_N));
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

// Splits rsp into BF16 hi/lo and lays every (128-channel, 64-energy) tile out
// contiguously in the core-matrix layout the kernel's bulk copies expect.
void Engine::fold_tc_prepare(Resp& r) {
  r.tc_ok = false;
  const int m_tiles = (r.n_ch + TC_M - 1) / TC_M;
  const int k_chunks = (r.n_e + TC_KC - 1) / TC_KC;
  r.m_pad = m_tiles * TC_M;
  r.k_pad = k_chunks * TC_KC;
  const size_t blk = A_BYTES / 2;
  std::vector<uint16_t> hi((size_t)m_tiles * k_chunks * blk, 0), lo(hi.size(), 0);
  for (int mt = 0; mt < m_tiles; ++mt)
    for (int kc = 0; kc < k_chunks; ++kc) {
      uint16_t* H = hi.data() + ((size_t)mt * k_chunks + kc) * blk;
      uint16_t* L = lo.data() + ((size_t)mt * k_chunks + kc) * blk;
      for (int rr = 0; rr < TC_M; ++rr)
        for (int k = 0; k < TC_KC; ++k) {
          const int m = mt * TC_M + rr, e = kc * TC_KC + k;
          const float v = (m < r.n_ch && e < r.n_e) ? (float)r.h_rsp[(size_t)m * r.n_e + e] : 0.0f;
          const uint16_t h = host_bf16(v);
          const uint16_t l = host_bf16(v - host_bf16_to_float(h));
          const uint32_t idx = cm_offset(rr, k, TC_M) / 2;
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
  r.d_a_hi = dh;
  r.d_a_lo = dl;
  r.tc_ok = true;
}

cudaError_t Engine::fold_tc_launch(const Resp& r, const FoldJob* jobs, int n_jobs, int n_bins, const double* flux,
                                   double* counts, cudaStream_t st, int* error) {
  cudaError_t e = once_per_device(1, [] {
    return cudaFuncSetAttribute(fold_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  });
  if (e != cudaSuccess) return e;
  TcArgs a{};
  a.a_hi = (const uint16_t*)r.d_a_hi;
  a.a_lo = (const uint16_t*)r.d_a_lo;
  a.n_ch = r.n_ch;
  a.n_e = r.n_e;
  a.k_chunks = r.k_pad / TC_KC;
  a.n_bins = n_bins;
  a.n_jobs = n_jobs;
  a.jobs = jobs;
  a.flux = flux;
  a.counts = counts;
  a.error = error ? error : d_err;
  // PPM_FOLD_TC_STALL_TEST=<polls>: the failure-path test of the bounded waits (no copy or MMA is issued, so the
  // first wait runs out after that many polls and the call reports PPM_E_TIMEOUT)
  if (const char* v = std::getenv("PPM_FOLD_TC_STALL_TEST")) a.stall_wait_limit = std::max(0, std::atoi(v));
  const int rows = n_jobs * n_bins;
  dim3 grid(r.m_pad / TC_M, (rows + TC_N - 1) / TC_N);
  fold_tc_kernel<<<grid, 128, SMEM_BYTES, st>>>(a);
  return cudaGetLastError();
}

}  // namespace ppm
