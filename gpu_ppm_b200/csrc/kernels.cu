// Engine kernels: work planner, persistent integrand (NSX FP32 and blackbody
// FP64/FP32 variants) and SIMT response folds.
//
// Integrand structure (one CTA per tile = candidate elements of one ring of
// one spot of one profile; CTAs pull tiles from a device queue, except in the
// blackbody kernel's fused point-source mode, where CTA b takes profile b's
// point spots without a planner):
//   1. ring geometry                      cpu/devarshi24st_cpu.cpp:90-124
//   2. active-element compaction by warp ballot + prefix (deterministic order)
//                                         gpu/devarshi24st_gpu.cu:196-212
//   3. two lensing rows of each table staged in shared memory, FP64 sweep of
//      the fine phases                    cpu/devarshi24st_cpu.cpp:126-193
//   4. gap fill / wrap                    cpu/devarshi24st_cpu.cpp:195-212
//   5. NSX (logT, logg) slice pre-reduced into shared memory (FP32)
//                                         gpu/devarshi24st_gpu.cu:323-351
//   6. deposit: rounds of phase points (FP64 phase, hunt, lerps, mu weights),
//      visible ones compacted into records; per record the mu-contracted slice
//      becomes per-cell cubic polynomials in log(E/kT), evaluated for the
//      observed energies with per-bin partial sums in registers (no
//      per-element atomics); a bin's partial sums are flushed once into the
//      FP64 flux pool                     cpu/devarshi24st_cpu.cpp:214-241
//      Home-cell kernel (default): each lane owns the energies of a few NSX
//      cells and builds their cubics in registers from shuffled slice rows.
//      Pooled-polynomial kernel (grids with > 16 energies in one cell): one
//      warp per point writes the cubics to shared memory, one thread per
//      energy reads its cell's cubic.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <type_traits>

#include "kernels.cuh"

namespace ppm {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2. * kPi;
constexpr int kSlotBytes = 48;  // bytes per batch point (SoA)
constexpr int kPhaseMajorMaxE = 4;  // blackbody grids of at most this many energies take the phase-major walk

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Block-wide ordered compaction: returns this thread's slot among flagged
// threads (or -1) and the total through *total.  Uses scratch[32].
__device__ __forceinline__ int block_compact(bool flag, int* scratch, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  unsigned b = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) scratch[warp] = __popc(b);
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int w = 0; w < nw; ++w) {
      int c = scratch[w];
      scratch[w] = run;
      run += c;
    }
    scratch[32] = run;
  }
  __syncthreads();
  int pos = flag ? scratch[warp] + __popc(b & lanemask_lt()) : -1;
  *total = scratch[32];
  return pos;
}

struct SmemPtrs {
  int* j;
  double *P, *F, *Z, *MU, *mu;
  float* S;
  double* rows;
  unsigned char* batch;
  float4* Q;
  float* H;
  unsigned short* hidx;  // home-cell kernel: bracket table of phase_o (see node_point_tab)
};

__device__ __forceinline__ SmemPtrs carve(unsigned char* sm, const IntegrandShape& S) {
  SmemPtrs s;
  s.j = (int*)(sm + S.off_j);
  s.P = (double*)(sm + S.off_P);
  s.F = (double*)(sm + S.off_F);
  s.Z = (double*)(sm + S.off_Z);
  s.MU = (double*)(sm + S.off_MU);
  s.mu = (double*)(sm + S.off_mu);
  s.S = (float*)(sm + S.off_S);
  s.rows = (double*)(sm + S.off_rows);
  s.batch = sm + S.off_batch;
  s.Q = (float4*)(sm + S.off_Q);
  s.H = (float*)(sm + S.off_Q + (S.nsx ? S.pb * S.cells * 16 : 0));
  s.hidx = (unsigned short*)(sm + S.off_hidx);
  return s;
}

// Steps 1-4 for one tile.  Returns the number of active elements (0 = nothing to do).
// On return (non-zero), P/F/Z/MU hold the filled fine-phase arrays and s_g the ring geometry.
__device__ int tile_prologue(const KernelArgs& a, const DevProfile& p, const DevSpot& sp, const Tile& tile,
                             const SmemPtrs& s, RingGeom& s_g, int* s_int, bool nsx) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool point = sp.kind == 1;
  const DevLens& L = a.lens;
  if (tid == 0) {
    double cos_t = point ? sp.cos_theta_pt : p.ring[3 * tile.ring];
    double dOmega = point ? sp.dOmega_pt : p.dOmega_hp;
    ring_geometry(p, L, cos_t, dOmega, nsx, s_g);
  }
  // compaction of active elements over the candidate range
  int n_act = 0;
  if (point) {
    if (tid == 0) s.j[0] = 0;
    n_act = 1;
  } else {
    const int N = p.n_side, ring = tile.ring;
    const double c2 = p.ring[3 * ring + 1], s2 = p.ring[3 * ring + 2];
    const int n_c = tile.j1 - tile.j0;
    for (int k0 = 0; k0 < n_c; k0 += nt) {
      int k = k0 + tid;
      bool flag = false;
      if (k < n_c) flag = in_spot(sp, c2, s2, healpix_phi(N, ring, tile.j0 + k));
      int tot;
      int pos = block_compact(flag, s_int, &tot);
      if (flag) s.j[n_act + pos] = tile.j0 + k;
      n_act += tot;
      __syncthreads();
    }
  }
  __syncthreads();
  if (n_act == 0) return 0;
  // counted by the tiles of the first node range only; a ring counts once, by the first of its tiles to
  // find active elements.  In the fused point-source mode no planner has dropped the ring yet: the counting
  // waits for the sweep's drop test below
  auto count_ring = [&]() {
    atomicAdd(&p.stats[0], (unsigned long long)n_act);
    const unsigned bit = 1u << (tile.ring & 31);
    if (!(atomicOr(&p.ring_seen[tile.spot * p.ring_words + (tile.ring >> 5)], bit) & bit))
      atomicAdd(&p.stats[1], 1ull);
    if (s_g.u_clamped && tile.first) atomicAdd(&p.stats[4], 1ull);
  };
  const bool fused = a.n_fused > 0;
  if (tid == 0) {
    if (tile.u0 == 0 && !fused) count_ring();
    s_int[40] = p.n_fine + 1;  // invisible min
    s_int[41] = -1;            // invisible max
  }
  // stage the two lensing rows of each table
  const int ncp = L.n_cp, nca = L.n_ca, iu = s_g.i_u;
  double* r = s.rows;
  for (int k = tid; k < 2 * ncp; k += nt) {
    int row = k / ncp, col = k - row * ncp;
    r[k] = L.ca[(size_t)(iu + row) * ncp + col];
    r[2 * ncp + k] = L.lf[(size_t)(iu + row) * ncp + col];
  }
  for (int k = tid; k < 2 * nca; k += nt) {
    int row = k / nca, col = k - row * nca;
    r[4 * ncp + k] = L.cdt[(size_t)(iu + row) * nca + col];
  }
  __syncthreads();
  LensRows rows{r, r + ncp, r + 2 * ncp, r + 3 * ncp, r + 4 * ncp, r + 4 * ncp + nca};
  const RingGeom g = s_g;
  const int nf = p.n_fine;
  for (int i = tid; i < nf; i += nt) {
    double F, Z, P, MU;
    if (sweep_sample(p, L, g, rows, i, nsx, F, Z, P, MU)) {
      s.F[i] = F;
      s.Z[i] = Z;
      s.P[i] = P;
      s.MU[i] = MU;
    } else {
      s.F[i] = 0;
      s.Z[i] = -1;
      s.P[i] = -1;
      s.MU[i] = 0;
      atomicMin(&s_int[40], i);
      atomicMax(&s_int[41], i);
    }
  }
  __syncthreads();
  const int inv_min = s_int[40], inv_max = s_int[41];
  const bool dropped = inv_min == 0 || inv_max == nf - 1;  // cpu/devarshi24st_cpu.cpp:195
  if (fused && tid == 0) {
    if (!dropped) {
      count_ring();
    } else {  // the planner's count of a dropped ring (plan_kernel)
      atomicAdd(&p.stats[1], 1ull);
      atomicAdd(&p.stats[2], 1ull);
      atomicAdd(&p.stats[5], (unsigned long long)n_act);
    }
  }
  if (dropped) return 0;
  if (inv_min <= inv_max) {
    const int beg = inv_min - 1, end = inv_max + 1;
    const double p0 = s.P[beg], p1 = s.P[end], z0 = s.Z[beg], z1 = s.Z[end];
    for (int i = inv_min + tid; i <= inv_max; i += nt) {
      s.P[i] = p0 + (p1 - p0) * ((double)(i - beg) / (end - beg));
      s.Z[i] = z0 + (z1 - z0) * ((double)(i - beg) / (end - beg));
    }
  }
  __syncthreads();
  if (tid == 0) {
    s.F[nf] = s.F[0];
    s.Z[nf] = s.Z[0];
    s.P[nf] = 1.0 + s.P[0];
    s.MU[nf] = s.MU[0];
  }
  __syncthreads();
  return n_act;
}

// Phase node u = bin * n_gl + GL point (u = bin when n_gl = 0): its bin, its
// phase ppt and GL weight (cpu/devarshi24st_cpu.cpp:214-219).
__device__ __forceinline__ void node_phase(const DevProfile& p, int u, int& bin, double& ppt, double& wgl) {
  const int n_gl = p.n_gl;
  if (n_gl > 0) {
    bin = u / n_gl;
    const int g = u - bin * n_gl;
    const double width = 1. / p.n_bins;
    const double lb = bin * width, ub = (bin + 1) * width;
    ppt = 0.5 * (lb + ub + c_gl_nodes[n_gl * (n_gl - 1) / 2 + g] * (ub - lb));
    wgl = 0.5 * 1. * c_gl_weights[n_gl * (n_gl - 1) / 2 + g];
  } else {
    bin = u;
    ppt = bin * (1.0 / p.n_bins);
    wgl = 1.0;
  }
}

// Active element jj of the tile at phase ppt: patch phase, hunt and lerps in
// FP64 (cpu/devarshi24st_cpu.cpp:220-229).  Returns flux/I (0 = skip).
__device__ __forceinline__ double node_point(const DevProfile& p, const SmemPtrs& s, const RingPhi& rp, bool point,
                                             int jj, double ppt, double& z, double& mu) {
  const double phi = point ? 0.0 : rp.dphi * (s.j[jj] - rp.jofs);
  const double phase_shift = phi / kTwoPi;
  // fmod(x, 1) of x = ppt + phase_shift + 1 in [1, 3): x - floor(x) is the same exact value
  const double xph = ppt + phase_shift + 1.;
  double patch = xph - floor(xph);
  if (patch < s.P[0]) patch += 1.;
  double af;
  const int i = vhunt(s.P, p.n_fine + 1, patch, af);
  const double flux = (1 - af) * s.F[i] + af * s.F[i + 1];
  if (flux == 0) return 0.0;
  z = (1 - af) * s.Z[i] + af * s.Z[i + 1];
  mu = (1 - af) * s.MU[i] + af * s.MU[i + 1];
  return flux;
}

// node_point with the tile's bracket table hidx (hidx[k] = vhunt's bracket of
// phase_o[0] + k / n_fine): on a non-decreasing phase_o (mono) the bracket of
// the patch phase is walked to from its table entry, a step or none, and is
// vhunt's bracket exactly; the fraction and the lerps are node_point's.
__device__ __forceinline__ double node_point_tab(const DevProfile& p, const SmemPtrs& s, const RingPhi& rp, bool point,
                                                 int jj, double ppt, bool mono, double& z, double& mu) {
  const double phi = point ? 0.0 : rp.dphi * (s.j[jj] - rp.jofs);
  const double phase_shift = phi / kTwoPi;
  const double xph = ppt + phase_shift + 1.;
  double patch = xph - floor(xph);
  if (patch < s.P[0]) patch += 1.;
  const int n = p.n_fine + 1;
  double af;
  int i;
  if (mono) {
    const int k = clampi((int)((patch - s.P[0]) * p.n_fine), 0, p.n_fine);
    i = walk_bracket(s.P, n, patch, s.hidx[k]);
    af = (patch - s.P[i]) / (s.P[i + 1] - s.P[i]);
  } else {
    i = vhunt(s.P, n, patch, af);
  }
  const double flux = (1 - af) * s.F[i] + af * s.F[i + 1];
  if (flux == 0) return 0.0;
  z = (1 - af) * s.Z[i] + af * s.Z[i + 1];
  mu = (1 - af) * s.MU[i] + af * s.MU[i + 1];
  return flux;
}

// Phase point q of the tile's node range (node u0 + q / n_act, element q % n_act).
__device__ __forceinline__ double phase_point(const DevProfile& p, const SmemPtrs& s, const RingPhi& rp, bool point,
                                              int n_act, int u0, int q, int& bin, double& wgl, double& z, double& mu) {
  const int du = q / n_act, jj = q - du * n_act;
  double ppt;
  node_phase(p, u0 + du, bin, ppt, wgl);
  return node_point(p, s, rp, point, jj, ppt, z, mu);
}

// Barrier of one warp set of n threads (a multiple of 32): the warp itself for
// a one-warp set, else named barrier 1 + set.
__device__ __forceinline__ void set_sync(int set, int n) {
  if (n == 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(1 + set), "r"(n) : "memory");
}

// phase_point's arithmetic for one element at phase point i_pp, for the
// blackbody kernel's point-wise path, with the per-tile and per-element terms
// (n = n_fine + 1, phase_o[0], 1 / n_bins, the element's phase shift
// phi / 2 pi) computed once by the caller.  When the tile's phase_o is
// non-decreasing (mono), the bracket is hunted from `hint`, this thread's
// previous one, which gives vhunt's bracket exactly, and the fraction uses
// the tile's reciprocal interval widths inv_dp when given (within an ulp of
// vhunt's division).
__device__ __forceinline__ double phase_point_at(const SmemPtrs& s, int n, double P0, const double* inv_dp, int n_gl,
                                                 double inv_bins, double phase_shift, int i_pp, bool mono, int& hint,
                                                 int& bin, double& wgl, double& z) {
  int g = 0;
  if (n_gl > 0) {
    bin = i_pp / n_gl;
    g = i_pp - bin * n_gl;
  } else {
    bin = i_pp;
  }
  double ppt;
  if (n_gl > 0) {
    const double width = inv_bins;
    const double lb = bin * width, ub = (bin + 1) * width;
    ppt = 0.5 * (lb + ub + c_gl_nodes[n_gl * (n_gl - 1) / 2 + g] * (ub - lb));
    wgl = 0.5 * 1. * c_gl_weights[n_gl * (n_gl - 1) / 2 + g];
  } else {
    ppt = bin * inv_bins;
    wgl = 1.0;
  }
  const double xph = ppt + phase_shift + 1.;
  double patch = xph - floor(xph);
  if (patch < P0) patch += 1.;
  double af;
  int i;
  if (mono) {
    hint = hunt_from(s.P, n, patch, hint);
    i = clampi(hint, 0, n - 2);
    af = inv_dp ? (patch - s.P[i]) * inv_dp[i] : (patch - s.P[i]) / (s.P[i + 1] - s.P[i]);
  } else {
    i = vhunt(s.P, n, patch, af);
  }
  const double flux = (1 - af) * s.F[i] + af * s.F[i + 1];
  if (flux == 0) return 0.0;
  z = (1 - af) * s.Z[i] + af * s.Z[i + 1];
  return flux;
}

// ---------------------------------------------------------------------------
template <int NE_T, int MINB>
__global__ void __launch_bounds__(MINB == 1 ? 512 : 320, MINB) integrand_nsx_kernel(const KernelArgs a) {
  extern __shared__ __align__(16) unsigned char sm[];
  const IntegrandShape& S = a.shape;
  const SmemPtrs s = carve(sm, S);
  __shared__ RingGeom s_g;
  __shared__ int s_int[48];
  __shared__ int s_tile;
  __shared__ float s_tapw[16];
  __shared__ int s_tapo[16];
  __shared__ int s_ntap;
  const int tid = threadIdx.x, nt = blockDim.x;
  const DevNsx& X = a.nsx;
  const int nE = X.nE, nmu = X.nmu, cells = S.cells, HN = cells + 3;

  // point records, one slot per thread: {c, fP, bin, G0} packed for one broadcast load,
  // plus the mu stencil start and weights
  float4* r_pk = (float4*)s.batch;
  int* r_imu = (int*)(r_pk + nt);
  float* r_w = (float*)(r_imu + nt);  // [4][nt]

  for (;;) {
    __syncthreads();
    if (tid == 0) s_tile = atomicAdd(a.queue.next, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= *a.queue.n_tiles || t >= a.queue.capacity) break;
    const Tile tile = a.queue.tiles[t];
    const DevProfile& p = a.profiles[tile.profile];
    const DevSpot& sp = p.spot[tile.spot];
    const bool point = sp.kind == 1;
    const int n_act = tile_prologue(a, p, sp, tile, s, s_g, s_int, true);
    if (n_act == 0) continue;
    const RingPhi rp = point ? RingPhi{0.0, 0.0} : healpix_ring_phi(p.n_side, tile.ring);

    // ---- step 5: (logT, logg) pre-reduction of the NSX table into S[E][mu]
    if (tid == 0) {
      const bool cubic = (p.interp == 0 || p.interp == 1 || p.interp == 2);
      double lg = s_g.logg, ag;
      s_int[45] = (lg < X.g_min || lg > X.g_max) ? 1 : 0;
      s_int[44] = 0;
      int ig = uhunt(lg, X.g_min, X.g_max, X.ng, ag);
      double wg[4];
      int ig0, ngt;
      if (cubic) {
        ig0 = clampi(ig - 1, 0, X.ng - 4);
        cubic_lagrange(wg, lg, uhunt_at(X.g_min, X.g_max, X.ng, ig0), uhunt_at(X.g_min, X.g_max, X.ng, ig0 + 1),
                       uhunt_at(X.g_min, X.g_max, X.ng, ig0 + 2), uhunt_at(X.g_min, X.g_max, X.ng, ig0 + 3));
        ngt = 4;
      } else {
        ig0 = ig;
        wg[0] = 1 - ag;
        wg[1] = ag;
        ngt = 2;
      }
      int n = 0;
      for (int jt = 0; jt < sp.nT_taps; ++jt)
        for (int jg = 0; jg < ngt; ++jg) {
          s_tapw[n] = (float)(sp.wT[jt] * wg[jg]);
          s_tapo[n] = (sp.iT[jt] * X.ng + ig0 + jg) * X.slice_stride;
          ++n;
        }
      s_ntap = n;
    }
    for (int k = tid; k < nmu; k += nt) s.mu[k] = X.mu[k];
    for (int k = tid; k < 4 * (nmu - 3); k += nt) s.mu[nmu + k] = X.mu_den[k];
    __syncthreads();
    {
      const int n4 = X.slice_stride >> 2, ntap = s_ntap;
      float4* S4 = (float4*)s.S;
      for (int k = tid; k < n4; k += nt) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int q = 0; q < ntap; ++q) {
          const float4 v = __ldg((const float4*)(X.data + s_tapo[q]) + k);
          const float w = s_tapw[q];
          acc.x = fmaf(w, v.x, acc.x);
          acc.y = fmaf(w, v.y, acc.y);
          acc.z = fmaf(w, v.z, acc.z);
          acc.w = fmaf(w, v.w, acc.w);
        }
        S4[k] = acc;
      }
    }
    __syncthreads();

    // ---- step 6: deposit
    const DevGrid& G = p.grid;
    const int n_e = G.n_e;
    int rE[NE_T];
    float fE[NE_T];
    float acc[NE_T];
#pragma unroll
    for (int k = 0; k < NE_T; ++k) {
      const int e = tid + k * nt;
      const bool ok = e < n_e;
      rE[k] = ok ? G.rE[e] : 0;
      fE[k] = ok ? G.fE[e] : 0.f;
      acc[k] = 0.f;
    }
    const int mode = p.interp;
    const bool cubicE = mode != 4;
    const bool sg = mode == 1;
    const double mu_min = s.mu[nmu - 1];
    const int n_pp = tile.u1 - tile.u0;  // the tile's phase nodes
    const int n_pts = n_pp * n_act;
    int cur_bin = -1;
    double* flux_base = a.flux + p.flux_off;
    const double out_scale = sp.out_scale;

    double* comp_base = a.comp ? a.comp + p.flux_off : nullptr;
    auto flush = [&]() {
#pragma unroll
      for (int k = 0; k < NE_T; ++k) {
        const int e = tid + k * nt;
        if (e < n_e && acc[k] != 0.f) {
          const size_t o = (size_t)cur_bin * n_e + e;
          comp_add(flux_base + o, comp_base ? comp_base + o : nullptr, (double)acc[k] * out_scale * G.invE[e]);
        }
        acc[k] = 0.f;
      }
    };

    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    const double* den = s.mu + nmu;  // [nmu - 3][4] reciprocal Lagrange denominators
    for (int q0 = 0; q0 < n_pts; q0 += nt) {
      // stage A: every thread evaluates one phase point (FP64); visible ones are
      // compacted, in order, into the point records
      bool vis = false, clamped = false;
      float c = 0.f, fP = 0.f;
      int G0 = 0, bin = 0, imu = 0;
      float w4[4] = {0.f, 0.f, 0.f, 0.f};
      const int q = q0 + tid;
      if (q < n_pts) {
        double wgl, z = 0, mu = 0;
        const double flux = phase_point(p, s, rp, point, n_act, tile.u0, q, bin, wgl, z, mu);
        if (flux != 0.0) {
          vis = true;
          if (mu < mu_min) mu = mu_min;
          c = (float)(flux * wgl);
          const double tP = (log10(z) - sp.l10kT - X.E_min) * X.inv_dE;
          const double fl = floor(tP);
          fP = (float)(tP - fl);
          if (fP >= 1.f) fP = 0.99999994f;
          G0 = G.iE_min + (int)fl;
          clamped = (G.tE_lo + tP < 0.0) || (G.tE_hi + tP > (double)(nE - 1)) || sp.T_clamped || s_int[45];
          // mu weights (cpu/nsx.hpp:173-321)
          double am;
          const int im = vhunt(s.mu, nmu, mu, am);
          const bool linear_mu = (mode == 4) || ((mode == 2 || mode == 3) && im >= nmu - 5);
          int start;
          if (linear_mu) {
            start = min(im, nmu - 4);
            const int o = im - start;
#pragma unroll
            for (int k = 0; k < 4; ++k) w4[k] = k == o ? (float)(1 - am) : (k == o + 1 ? (float)am : 0.f);
          } else {
            start = clampi(im - 1, 0, nmu - 4);
            const double x0 = s.mu[start], x1 = s.mu[start + 1], x2 = s.mu[start + 2], x3 = s.mu[start + 3];
            const double* r = den + 4 * start;
            w4[0] = (float)((mu - x1) * (mu - x2) * (mu - x3) * r[0]);
            w4[1] = (float)((mu - x0) * (mu - x2) * (mu - x3) * r[1]);
            w4[2] = (float)((mu - x0) * (mu - x1) * (mu - x3) * r[2]);
            w4[3] = (float)((mu - x0) * (mu - x1) * (mu - x2) * r[3]);
          }
          imu = start;
        }
      }
      int nv;
      const int slot = block_compact(vis, s_int, &nv);
      if (vis) {
        r_pk[slot] = make_float4(c, fP, __int_as_float(bin), __int_as_float(G0));
        r_imu[slot] = imu;
#pragma unroll
        for (int k = 0; k < 4; ++k) r_w[k * nt + slot] = w4[k];
        if (clamped) atomicAdd(&s_int[44], 1);
      }
      __syncthreads();
      if (tid == 0) {
        if (nv) atomicAdd(&p.stats[3], (unsigned long long)nv);
        if (s_int[44]) atomicAdd(&p.stats[4], (unsigned long long)s_int[44]);
        s_int[44] = 0;
      }

      for (int s0 = 0; s0 < nv; s0 += S.pb) {
        const int nb = min(S.pb, nv - s0);
        // stage B: one warp per point builds the mu-contracted rows H and the
        // per-cell cubic polynomials Q (Newton form rewritten in the cell fraction)
        for (int b = warp; b < nb; b += 2 * nwarps) {
          // two points per warp, interleaved for instruction-level parallelism
          const int bB = b + nwarps;
          const bool has2 = bB < nb;
          const int recA = s0 + b, recB = s0 + (has2 ? bB : b);
          const int G0a = __float_as_int(r_pk[recA].w), G0b = __float_as_int(r_pk[recB].w);
          const int ima = r_imu[recA], imb = r_imu[recB];
          const float wa0 = r_w[recA], wa1 = r_w[nt + recA], wa2 = r_w[2 * nt + recA], wa3 = r_w[3 * nt + recA];
          const float wb0 = r_w[recB], wb1 = r_w[nt + recB], wb2 = r_w[2 * nt + recB], wb3 = r_w[3 * nt + recB];
          const int kHa = clampi(G0a - 1, 0, nE - 4), kHb = clampi(G0b - 1, 0, nE - 4);
          float* Ha = s.H + b * HN;
          float* Hb = s.H + bB * HN;
          for (int kk = lane; kk < HN; kk += 32) {
            const int ka = kHa + kk, kb = kHb + kk;
            float ha = 0.f, hb = 0.f;
            if (ka < nE) {
              const float* row = s.S + ka * nmu + ima;
              ha = fmaf(wa3, row[3], fmaf(wa2, row[2], fmaf(wa1, row[1], wa0 * row[0])));
            }
            if (has2 && kb < nE) {
              const float* row = s.S + kb * nmu + imb;
              hb = fmaf(wb3, row[3], fmaf(wb2, row[2], fmaf(wb1, row[1], wb0 * row[0])));
            }
            Ha[kk] = ha;
            if (has2) Hb[kk] = hb;
          }
          __syncwarp();
          for (int pt = 0; pt < (has2 ? 2 : 1); ++pt) {
            const int G0x = pt ? G0b : G0a, kH0 = pt ? kHb : kHa;
            const float* H = pt ? Hb : Ha;
            float4* Qb = s.Q + (pt ? bB : b) * cells;
            for (int cc = lane; cc < cells; cc += 32) {
              const int gcell = G0x + cc;
              float4 Qv;
              if (gcell < 0) {
                Qv = make_float4(H[0 - kH0], 0.f, 0.f, 0.f);
              } else if (gcell > nE - 2) {
                Qv = make_float4(H[nE - 1 - kH0], 0.f, 0.f, 0.f);
              } else if (cubicE) {
                const int ie = clampi(gcell - 1, 0, nE - 4);
                const int off = gcell - ie;
                const float h0 = H[ie - kH0], h1 = H[ie - kH0 + 1], h2 = H[ie - kH0 + 2], h3 = H[ie - kH0 + 3];
                const float d1 = h1 - h0, d2 = h2 - 2.f * h1 + h0, d3 = h3 - 3.f * h2 + 3.f * h1 - h0;
                const float c3 = d3 * (1.f / 6.f);
                if (off == 1)
                  Qv = make_float4(h1, d1 + 0.5f * d2 - c3, 0.5f * d2, c3);
                else if (off == 0)
                  Qv = make_float4(h0, d1 - 0.5f * d2 + d3 * (1.f / 3.f), 0.5f * d2 - 0.5f * d3, c3);
                else
                  Qv = make_float4(h2, d1 + 1.5f * d2 + d3 * (1.f / 3.f), 0.5f * d2 + 0.5f * d3, c3);
              } else {
                const float h0 = H[gcell - kH0], h1 = H[gcell - kH0 + 1];
                Qv = make_float4(h0, h1 - h0, 0.f, 0.f);
              }
              Qb[cc] = Qv;
            }
          }
        }
        __syncthreads();

        // stage C: every thread integrates its energies over the sub-batch; two
        // points of the same bin are interleaved for instruction-level parallelism
        for (int b = 0; b < nb;) {
          const float4 r0 = r_pk[s0 + b];
          const int bin0 = __float_as_int(r0.z);
          if (bin0 != cur_bin) {
            if (cur_bin >= 0) flush();
            cur_bin = bin0;
          }
          const float4* Q0 = s.Q + b * cells;
          bool two = false;
          float4 r1 = r0;
          if (b + 1 < nb) {
            r1 = r_pk[s0 + b + 1];
            two = __float_as_int(r1.z) == bin0;
          }
          if (two) {
            const float4* Q1 = Q0 + cells;
#pragma unroll
            for (int k = 0; k < NE_T; ++k) {
              float t0 = fE[k] + r0.y, t1 = fE[k] + r1.y;
              const int k0 = t0 >= 1.f, k1 = t1 >= 1.f;
              t0 = k0 ? t0 - 1.f : t0;
              t1 = k1 ? t1 - 1.f : t1;
              const float4 qa = Q0[rE[k] + k0], qb = Q1[rE[k] + k1];
              float ia = fmaf(fmaf(fmaf(qa.w, t0, qa.z), t0, qa.y), t0, qa.x);
              float ib = fmaf(fmaf(fmaf(qb.w, t1, qb.z), t1, qb.y), t1, qb.x);
              if (sg) {
                ia = fmaxf(ia, 0.f);
                ib = fmaxf(ib, 0.f);
              }
              acc[k] = fmaf(r1.x, ib, fmaf(r0.x, ia, acc[k]));
            }
            b += 2;
          } else {
#pragma unroll
            for (int k = 0; k < NE_T; ++k) {
              float t0 = fE[k] + r0.y;
              const int k0 = t0 >= 1.f;
              t0 = k0 ? t0 - 1.f : t0;
              const float4 qa = Q0[rE[k] + k0];
              float ia = fmaf(fmaf(fmaf(qa.w, t0, qa.z), t0, qa.y), t0, qa.x);
              if (sg) ia = fmaxf(ia, 0.f);
              acc[k] = fmaf(r0.x, ia, acc[k]);
            }
            b += 1;
          }
        }
        __syncthreads();
      }
    }
    if (cur_bin >= 0) flush();
  }
}

// ---------------------------------------------------------------------------
// Home-cell NSX integrand.
//
// For a phase point with cell origin G0 and cell fraction fP, energy e falls
// in NSX cell G0 + rE[e] + carry (carry = fE[e] + fP >= 1).  Every lane owns
// one home cell r = rE (32 per warp) and the few energies whose rE is r, so
// per point it needs the cubic polynomials of cells G0 + r and G0 + r + 1,
// i.e. the mu-contracted slice H at G0 + r - 1 .. G0 + r + 3: each lane
// contracts the first and the last of these rows and takes the three between
// from its neighbours by warp shuffles.
// Polynomials and partial sums stay in registers; a warp set of cell_warps
// warps covers every cell of a point, and the CTA's warp sets take the
// point records in contiguous runs, each keeping its own per-bin partial sums.
//
// The polynomial of a cell is the one the pooled kernel builds (4-point
// Lagrange stencil clamped at the table ends, cpu/nsx.hpp:187-225, written
// as Newton differences in the cell fraction); outside the logEkT axis the
// edge value is held (cpu/hunt.hpp:98-121 clamps the coordinate).
__device__ __forceinline__ float slice_dot(const float* S, int ldS, int k, int imu, float4 w) {
  const float* row = S + k * ldS + imu;
  return fmaf(w.w, row[3], fmaf(w.z, row[2], fmaf(w.y, row[1], w.x * row[0])));
}

// Lanes of a warp that only supply slice rows to their neighbours (no home
// cells): a lane needs rows up to C + 3 past its first, i.e. own rows of the
// next (C + 3) / C lanes.
template <int C>
__host__ __device__ constexpr int halo_lanes() {
  return (C + 3) / C;
}

// Slice rows seen by one lane for one point record.  The lane owns C
// consecutive cells starting at cell g (= G0 + first cell of the lane) and
// needs the cubics of cells g .. g + C, i.e. rows g - 1 .. g + C + 2 of the
// mu-contracted slice: window h[j] = row g - 1 + j, j = 0 .. C + 3.  The lane
// contracts rows j < C itself; row j >= C is own row j mod C of lane
// lane + j / C (the last halo_lanes<C>() lanes of the warp own no cells).
// Sx points at slice row 0 of a slice with rows -2 .. nE + 1: rows -1 and nE
// hold the cubic extrapolations of the first and last four rows, so that the
// centred stencil of cell 0 (rows -1..2) and of cell nE - 2 (rows nE - 3..nE)
// is the same cubic as the end-clamped stencil (rows 0..3, rows nE - 4..nE - 1);
// rows -2 and nE + 1 repeat rows 0 and nE - 1, and window rows are clamped to
// -2 .. nE + 1, so cells past either end see the end value H[0] / H[nE - 1].
template <int C>
__device__ __forceinline__ void lane_window(const float* Sx, int ldS, int nE, int g, int imu, float4 w,
                                            float (&h)[C + 4]) {
#pragma unroll
  for (int j = 0; j < C; ++j) h[j] = slice_dot(Sx, ldS, min(max(g - 1 + j, -2), nE + 1), imu, w);
#pragma unroll
  for (int j = C; j < C + 4; ++j) h[j] = __shfl_down_sync(0xffffffffu, h[j % C], j / C);
}

// Cubics of the C + 1 cells whose stencils are window rows i .. i + 3 (the
// cell between rows i + 1 and i + 2), in the cell fraction t: the Newton form
// about row i + 1 rewritten as q0 + t (q1 + t (q2 + t q3)), from forward
// differences shared by neighbouring cells.
template <int C>
__device__ __forceinline__ void window_cubics(const float (&h)[C + 4], float4 (&Q)[C + 1]) {
  float d1[C + 3], d2[C + 2], d3[C + 1];
#pragma unroll
  for (int j = 0; j < C + 3; ++j) d1[j] = h[j + 1] - h[j];
#pragma unroll
  for (int j = 0; j < C + 2; ++j) d2[j] = d1[j + 1] - d1[j];
#pragma unroll
  for (int j = 0; j < C + 1; ++j) d3[j] = d2[j + 1] - d2[j];
#pragma unroll
  for (int i = 0; i <= C; ++i) {
    const float c3 = d3[i] * (1.f / 6.f);
    Q[i] = make_float4(h[i + 1], d1[i] + 0.5f * d2[i] - c3, 0.5f * d2[i], c3);
  }
}

// Packed FP32 pairs (add / fma .f32x2, one instruction for two lanes of
// arithmetic): two energy slots of one cell share the cubics' coefficients.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk(f32x2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

template <int MAXE, int C, int NTMAX, int MINB>
__global__ void __launch_bounds__(NTMAX, MINB) integrand_nsx_cell_kernel(const KernelArgs a) {
  extern __shared__ __align__(16) unsigned char sm[];
  const IntegrandShape& S = a.shape;
  const SmemPtrs s = carve(sm, S);
  __shared__ RingGeom s_g;
  __shared__ int s_int[48];
  __shared__ int s_tile;
  __shared__ float s_tapw[16];
  __shared__ int s_tapo[16];
  __shared__ int s_ntap;
  __shared__ int s_node[16], s_bin[16];          // node taken by each warp set, its bin
  __shared__ double s_ppt[16], s_wgl[16];        // the node's phase and GL weight
  __shared__ int s_wcnt[16];                     // visible points per warp (sets of several warps)
  __shared__ unsigned s_nvis[16], s_nclamp[16];  // per warp: visible and clamped points of the tile
  const int tid = threadIdx.x, nt = blockDim.x;
  const DevNsx& X = a.nsx;
  const int nE = X.nE, nmu = X.nmu, ldS = S.ldS;
  const int lane = tid & 31, warp = tid >> 5;
  const int set = warp / S.cell_warps, n_sets = (nt >> 5) / S.cell_warps;
  constexpr int kOwners = 32 - halo_lanes<C>();        // lanes with home cells
  const int wc = (warp - set * S.cell_warps) * kOwners * C;  // first cell of the warp
  const int r0 = wc + C * lane;                              // first of the lane's C home cells
  float4* rec = (float4*)s.batch;  // [nt][2]: {c, fP, imu, G0}, {mu weights}; set k uses [32 cell_warps k, ..)

  for (;;) {
    __syncthreads();
    if (tid == 0) s_tile = atomicAdd(a.queue.next, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= *a.queue.n_tiles || t >= a.queue.capacity) break;
    const Tile tile = a.queue.tiles[t];
    const DevProfile& p = a.profiles[tile.profile];
    const DevSpot& sp = p.spot[tile.spot];
    const bool point = sp.kind == 1;
    const int n_act = tile_prologue(a, p, sp, tile, s, s_g, s_int, true);
    if (n_act == 0) continue;
    const RingPhi rp = point ? RingPhi{0.0, 0.0} : healpix_ring_phi(p.n_side, tile.ring);

    // ---- (logT, logg) pre-reduction of the NSX table into S[E][mu] (row stride ldS)
    if (tid == 0) {
      const bool cubic = (p.interp == 0 || p.interp == 1 || p.interp == 2);
      double lg = s_g.logg, ag;
      s_int[45] = (lg < X.g_min || lg > X.g_max) ? 1 : 0;
      s_int[44] = 0;
      s_int[46] = tile.u0;  // next phase node of the deposit
      int ig = uhunt(lg, X.g_min, X.g_max, X.ng, ag);
      double wg[4];
      int ig0, ngt;
      if (cubic) {
        ig0 = clampi(ig - 1, 0, X.ng - 4);
        cubic_lagrange(wg, lg, uhunt_at(X.g_min, X.g_max, X.ng, ig0), uhunt_at(X.g_min, X.g_max, X.ng, ig0 + 1),
                       uhunt_at(X.g_min, X.g_max, X.ng, ig0 + 2), uhunt_at(X.g_min, X.g_max, X.ng, ig0 + 3));
        ngt = 4;
      } else {
        ig0 = ig;
        wg[0] = 1 - ag;
        wg[1] = ag;
        ngt = 2;
      }
      int n = 0;
      for (int jt = 0; jt < sp.nT_taps; ++jt)
        for (int jg = 0; jg < ngt; ++jg) {
          s_tapw[n] = (float)(sp.wT[jt] * wg[jg]);
          s_tapo[n] = (sp.iT[jt] * X.ng + ig0 + jg) * X.slice_stride;
          ++n;
        }
      s_ntap = n;
    }
    for (int k = tid; k < nmu; k += nt) s.mu[k] = X.mu[k];
    for (int k = tid; k < 4 * (nmu - 3); k += nt) s.mu[nmu + k] = X.mu_den[k];
    // the tile's phase_o bracket table for node_point_tab, used where phase_o is non-decreasing
    bool mono_ok = true;
    {
      const int n_fp = p.n_fine + 1;
      for (int k = tid; k < p.n_fine; k += nt) mono_ok &= s.P[k + 1] >= s.P[k];
      for (int k = tid; k <= p.n_fine; k += nt) {
        double a_unused;
        s.hidx[k] = (unsigned short)vhunt(s.P, n_fp, s.P[0] + (double)k / p.n_fine, a_unused);
      }
    }
    const bool mono = __syncthreads_and(mono_ok) != 0;
    // slice rows 0..nE-1 start 16-byte aligned after room for rows -2, -1; rows nE, nE + 1 follow them
    float* const Sx = s.S + ((2 * ldS + 3) & ~3);
    {
      const int ntap = s_ntap, n_el = nE * nmu;
      if (ldS == nmu) {
        const int n4 = (n_el + 3) >> 2;
        float4* S4 = (float4*)Sx;
        for (int k = tid; k < n4; k += nt) {
          float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
          for (int q = 0; q < ntap; ++q) {
            const float4 v = __ldg((const float4*)(X.data + s_tapo[q]) + k);
            const float w = s_tapw[q];
            acc.x = fmaf(w, v.x, acc.x);
            acc.y = fmaf(w, v.y, acc.y);
            acc.z = fmaf(w, v.z, acc.z);
            acc.w = fmaf(w, v.w, acc.w);
          }
          S4[k] = acc;
        }
      } else {
        for (int k = tid; k < n_el; k += nt) {
          float acc = 0.f;
          for (int q = 0; q < ntap; ++q) acc = fmaf(s_tapw[q], __ldg(X.data + s_tapo[q] + k), acc);
          const int row = k / nmu;
          Sx[row * ldS + (k - row * nmu)] = acc;
        }
      }
    }
    __syncthreads();
    // rows -1 and nE: the cubic through the first (last) four rows, one row
    // further out; rows -2 and nE + 1: copies of rows 0 and nE - 1
    for (int k = tid; k < 2 * nmu; k += nt) {
      const int top = k >= nmu, m = top ? k - nmu : k;
      const float* a = Sx + (top ? (nE - 1) * ldS : 0) + m;
      const int st = top ? -ldS : ldS;
      Sx[(top ? nE : -1) * ldS + m] = fmaf(4.f, a[0], fmaf(-6.f, a[st], fmaf(4.f, a[2 * st], -a[3 * st])));
      Sx[(top ? nE + 1 : -2) * ldS + m] = a[0];
    }
    __syncthreads();

    // ---- deposit.  The tile's phase nodes u in [u0, u1) (u = bin * n_gl + GL
    // point) go to the warp sets one at a time through a shared counter.  A set
    // walks its node's elements jj = 0 .. n_act - 1 in order, 32 x cell_warps
    // at a time: every thread evaluates one point (FP64), the visible points are
    // compacted in order into the set's records, and every lane adds each record
    // to its energies' FP32 partial sums; at the end of the node the sums are
    // flushed with compensated FP64 atomics.  A node's sums thus depend on the
    // tile's elements and the node only, not on the tile's node range, the sets
    // or what else is in the batch.
    const DevGrid& G = p.grid;
    const int n_e = G.n_e;
    // per home cell i of the lane: MAXE energy slots in pairs (fractions, partial sums); the cells' energy
    // ranges (cell_first) are read again at each flush, out of the record loop's registers
    f32x2 fE2[C][MAXE / 2], acc2[C][MAXE / 2];
#pragma unroll
    for (int i = 0; i < C; ++i) {
      const int rc = r0 + i;
      const bool own = lane < kOwners && rc < G.span;
      const int e0 = own ? G.cell_first[rc] : 0;
      const int cnt = own ? min(G.cell_first[rc + 1] - e0, MAXE) : 0;
#pragma unroll
      for (int k = 0; k < MAXE / 2; ++k) {
        fE2[i][k] = pk(2 * k < cnt ? G.fEs[e0 + 2 * k] : 0.f, 2 * k + 1 < cnt ? G.fEs[e0 + 2 * k + 1] : 0.f);
        acc2[i][k] = pk(0.f, 0.f);
      }
    }
    const int mode = p.interp;
    const bool cubicE = mode != 4;
    const bool sg = mode == 1;
    const int ST = 32 * S.cell_warps;  // threads of a set
    const int st = tid - set * ST;     // this thread's index in its set
    const bool lane_cells = lane < kOwners && r0 < G.span;  // the lane owns cells of the grid
    float4* srec = rec + 2 * set * ST;  // the set's records
    if (lane == 0) {
      s_nvis[warp] = 0;
      s_nclamp[warp] = 0;
    }

    const double* den = s.mu + nmu;  // [nmu - 3][4] reciprocal Lagrange denominators
    for (;;) {
      // the set's next node: its index, bin, phase and weight, published in shared memory (kept out of the
      // registers of the record loop below)
      if (st == 0) {
        const int u = atomicAdd(&s_int[46], 1);
        s_node[set] = u;
        if (u < tile.u1) {
          int bin;
          double ppt, wgl;
          node_phase(p, u, bin, ppt, wgl);
          s_bin[set] = bin;
          s_ppt[set] = ppt;
          s_wgl[set] = wgl;
        }
      }
      set_sync(set, ST);
      if (s_node[set] >= tile.u1) break;
      for (int jb = 0; jb < n_act; jb += ST) {
        // every thread evaluates one element at the node (FP64); the visible
        // ones are compacted, in element order, into the set's records
        bool vis = false, clamped = false;
        float c = 0.f, fP = 0.f;
        int G0 = 0, imu = 0;
        float w4[4] = {0.f, 0.f, 0.f, 0.f};
        const int jj = jb + st;
        if (jj < n_act) {
          double z = 0, mu = 0;
          const double flux = node_point_tab(p, s, rp, point, jj, s_ppt[set], mono, z, mu);
          if (flux != 0.0) {
            vis = true;
            if (mu < s.mu[nmu - 1]) mu = s.mu[nmu - 1];
            c = (float)(flux * s_wgl[set]);
            const double tP = (log10(z) - sp.l10kT - X.E_min) * X.inv_dE;
            const double fl = floor(tP);
            fP = (float)(tP - fl);
            if (fP >= 1.f) fP = 0.99999994f;
            G0 = G.iE_min + (int)fl;
            clamped = (G.tE_lo + tP < 0.0) || (G.tE_hi + tP > (double)(nE - 1)) || sp.T_clamped || s_int[45];
            // mu weights (cpu/nsx.hpp:173-321)
            double am;
            const int im = vhunt(s.mu, nmu, mu, am);
            const bool linear_mu = (mode == 4) || ((mode == 2 || mode == 3) && im >= nmu - 5);
            int start;
            if (linear_mu) {
              start = min(im, nmu - 4);
              const int o = im - start;
#pragma unroll
              for (int k = 0; k < 4; ++k) w4[k] = k == o ? (float)(1 - am) : (k == o + 1 ? (float)am : 0.f);
            } else {
              start = clampi(im - 1, 0, nmu - 4);
              const double x0 = s.mu[start], x1 = s.mu[start + 1], x2 = s.mu[start + 2], x3 = s.mu[start + 3];
              const double* rd = den + 4 * start;
              w4[0] = (float)((mu - x1) * (mu - x2) * (mu - x3) * rd[0]);
              w4[1] = (float)((mu - x0) * (mu - x2) * (mu - x3) * rd[1]);
              w4[2] = (float)((mu - x0) * (mu - x1) * (mu - x3) * rd[2]);
              w4[3] = (float)((mu - x0) * (mu - x1) * (mu - x2) * rd[3]);
            }
            imu = start;
          }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, vis);
        const unsigned bal_clamped = __ballot_sync(0xffffffffu, clamped);
        if (lane == 0) {
          s_nvis[warp] += __popc(bal);
          s_nclamp[warp] += __popc(bal_clamped);
        }
        int nv, slot;
        if (S.cell_warps == 1) {
          nv = __popc(bal);
          slot = __popc(bal & lanemask_lt());
        } else {
          const int w = st >> 5;
          if (lane == 0) s_wcnt[warp] = __popc(bal);
          set_sync(set, ST);
          int before = 0;
          nv = 0;
          for (int k = 0; k < S.cell_warps; ++k) {
            const int cw = s_wcnt[set * S.cell_warps + k];
            before += k < w ? cw : 0;
            nv += cw;
          }
          slot = before + __popc(bal & lanemask_lt());
        }
        if (vis) {
          srec[2 * slot] = make_float4(c, fP, __int_as_float(imu), __int_as_float(G0));
          srec[2 * slot + 1] = make_float4(w4[0], w4[1], w4[2], w4[3]);
        }
        // whether a record of this step may use a cell next to the high or the low end of the table (cells
        // G0 .. G0 + span are in use); the same for every lane: the warp's votes, or both ends for sets of
        // several warps
        bool step_hi = true, step_lo = true;
        if (S.cell_warps == 1) {
          step_hi = __any_sync(0xffffffffu, vis && G0 + G.span >= nE - 1 && G0 <= nE + 1);
          step_lo = __any_sync(0xffffffffu, vis && G0 <= -1 && G0 + G.span >= -3);
        }
        set_sync(set, ST);
        for (int b = 0; b < nv; ++b) {
          const float4 rA = srec[2 * b], wA = srec[2 * b + 1];
          const int g = __float_as_int(rA.w) + r0;  // first home cell of the lane for this point
          float h[C + 4];
          lane_window<C>(Sx, ldS, nE, g, __float_as_int(rA.z), wA, h);
          float4 Q[C + 1];
          if (cubicE) {
            window_cubics<C>(h, Q);
          } else {
#pragma unroll
            for (int i = 0; i <= C; ++i) Q[i] = make_float4(h[i + 1], h[i + 2] - h[i + 1], 0.f, 0.f);
          }
          // cells past an end hold the end value.  A cell four or more rows past
          // an end reads four equal clamped rows, so its cubic is that constant
          // already; the three cells next to each end become constants here.
          // Their value is the x of a cubic (the x of cell k is row k): of the
          // cell itself, except for cell nE and cell -1, whose rows are the
          // extrapolated ones; they take the x of a neighbouring cell, row
          // nE + 1 or nE - 1 (both hold H[nE - 1]), row 0 or row -2 (H[0]).
          if (step_hi && __any_sync(0xffffffffu, lane_cells && g + C >= nE - 1 && g <= nE + 1)) {
#pragma unroll
            for (int i = 0; i <= C; ++i) {
              const int gi = g + i;
              const float nb = i < C ? Q[i + 1].x : Q[i > 0 ? i - 1 : 0].x;
              if ((unsigned)(gi - (nE - 1)) <= 2u) Q[i] = make_float4(gi == nE ? nb : Q[i].x, 0.f, 0.f, 0.f);
            }
          }
          if (step_lo && __any_sync(0xffffffffu, lane_cells && g <= -1 && g + C >= -3)) {
#pragma unroll
            for (int i = 0; i <= C; ++i) {
              const int gi = g + i;
              const float nb = i < C ? Q[i + 1].x : Q[i > 0 ? i - 1 : 0].x;
              if ((unsigned)(gi + 3) <= 2u) Q[i] = make_float4(gi == -1 ? nb : Q[i].x, 0.f, 0.f, 0.f);
            }
          }
          const f32x2 cw2 = pk(rA.x, rA.x), fP2 = pk(rA.y, rA.y), m1 = pk(-1.f, -1.f);
#pragma unroll
          for (int i = 0; i < C; ++i) {
            const f32x2 ax = pk(Q[i].x, Q[i].x), ay = pk(Q[i].y, Q[i].y), az = pk(Q[i].z, Q[i].z), aw = pk(Q[i].w, Q[i].w);
            const f32x2 bx = pk(Q[i + 1].x, Q[i + 1].x), by = pk(Q[i + 1].y, Q[i + 1].y), bz = pk(Q[i + 1].z, Q[i + 1].z),
                        bw = pk(Q[i + 1].w, Q[i + 1].w);
#pragma unroll
            for (int k = 0; k < MAXE / 2; ++k) {
              // split coordinate t = fE + fP: cell i below 1, cell i + 1 at t - 1
              // above; both cubics are evaluated and the result selected
              const f32x2 t0 = add2(fE2[i][k], fP2), t1 = add2(t0, m1);
              const f32x2 v0 = fma2(fma2(fma2(aw, t0, az), t0, ay), t0, ax);
              const f32x2 v1 = fma2(fma2(fma2(bw, t1, bz), t1, by), t1, bx);
              float ta, tb, a0, b0, a1, b1;
              upk(t0, ta, tb);
              upk(v0, a0, b0);
              upk(v1, a1, b1);
              float va = ta >= 1.f ? a1 : a0, vb = tb >= 1.f ? b1 : b0;
              if (sg) {
                va = fmaxf(va, 0.f);
                vb = fmaxf(vb, 0.f);
              }
              acc2[i][k] = fma2(cw2, pk(va, vb), acc2[i][k]);
            }
          }
        }
        set_sync(set, ST);  // the records are rewritten by the next step
      }
      // the node's partial sums into the flux pool
      const int bin = s_bin[set];
      double* flux_base = a.flux + p.flux_off;
      double* comp_base = a.comp ? a.comp + p.flux_off : nullptr;
      const double out_scale = sp.out_scale;
#pragma unroll
      for (int i = 0; i < C; ++i) {
        const int rc = r0 + i;
        const bool own = lane < kOwners && rc < G.span;
        const int e0 = own ? G.cell_first[rc] : 0;
        const int cnt = own ? min(G.cell_first[rc + 1] - e0, MAXE) : 0;
#pragma unroll
        for (int k = 0; k < MAXE; ++k) {
          float lo, hi;
          upk(acc2[i][k / 2], lo, hi);
          const float v = (k & 1) ? hi : lo;
          if (k < cnt && v != 0.f) {
            const int e = G.perm[e0 + k];
            const size_t o = (size_t)bin * n_e + e;
            comp_add(flux_base + o, comp_base ? comp_base + o : nullptr, (double)v * out_scale * G.invE[e]);
          }
          if (k & 1) acc2[i][k / 2] = pk(0.f, 0.f);
        }
      }
    }
    if (lane == 0) {
      if (s_nvis[warp]) atomicAdd(&p.stats[3], (unsigned long long)s_nvis[warp]);
      if (s_nclamp[warp]) atomicAdd(&p.stats[4], (unsigned long long)s_nclamp[warp]);
    }
  }
}

// ---------------------------------------------------------------------------
// The blackbody phase-major walk over the tile's elements jj0 .. jj1 - 1 at one
// phase node (phase ppt, weight wgl): adds each visible element's Ibb at the
// grid's first NE energies (NE = 1, or up to n_e) into acc and returns the
// number of visible elements.  The patch phase and its phase_o bracket are
// FP64 in every arithmetic, the bracket hunted from the previous element's.
// FP64 arithmetic lerps F and Z in FP64 and divides exactly; FP32 arithmetic
// lerps the tile's FP32 copies of F and Z and divides with the fast
// reciprocal.
template <typename Real, int NE>
__device__ __forceinline__ unsigned pm_walk(const SmemPtrs& s, const double* inv_dp, const float* F32, const float* Z32,
                                            const double* shift_s, const Real* E_s, int n_e, Real inv_kT, double ppt,
                                            double wgl, int jj0, int jj1, int n_fp, double P0, double* acc) {
  unsigned n_vis = 0;
  int hint = -1;
  double prev = -1.0;  // below every patch phase
  for (int jj = jj0; jj < jj1; ++jj) {
    const double xph = ppt + shift_s[jj] + 1.;
    // x - floor(x) for x in [1, 3]: the same exact value
    double patch = xph - (xph >= 3.0 ? 3.0 : (xph >= 2.0 ? 2.0 : 1.0));
    if (patch < P0) patch += 1.;
    // phase_o[i] is phase i / n_fine plus a small time-of-flight delay: the
    // first element's bracket is walked to from that guess, the others' from
    // the previous bracket by unit steps (none or one for the next element;
    // from the first bracket when the patch phase wraps past phase_o[0] + 1).
    // On a non-decreasing phase_o the walk stops at vhunt's bracket: the
    // largest i <= n - 2 with phase_o[i] <= patch, or 0.
    if (patch < prev) hint = 0;
    prev = patch;
    if (hint < 0) hint = clampi((int)((patch - P0) * (n_fp - 1)), 0, n_fp - 2);
    hint = walk_bracket(s.P, n_fp, patch, hint);
    const int i = hint;
    Real cb, zb;
    if constexpr (std::is_same<Real, float>::value) {
      const float af = (float)((patch - s.P[i]) * inv_dp[i]);
      const float f0 = F32[i];
      const float flux = fmaf(af, F32[i + 1] - f0, f0);
      if (flux == 0.f) continue;
      const float z0 = Z32[i];
      zb = fmaf(af, Z32[i + 1] - z0, z0);
      cb = flux * (float)wgl;
    } else {
      const double af = (patch - s.P[i]) * inv_dp[i];
      const double flux = (1 - af) * s.F[i] + af * s.F[i + 1];
      if (flux == 0) continue;
      zb = (1 - af) * s.Z[i] + af * s.Z[i + 1];
      cb = flux * wgl;
    }
    ++n_vis;
#pragma unroll
    for (int e = 0; e < NE; ++e)
      if (NE == 1 || e < n_e) {
        const Real Ee = E_s[e] * zb;
        Real v;  // Ibb without its constant
        if constexpr (std::is_same<Real, float>::value) {
          // e^x - 1: the fast exponential where x > 0.5 (no cancellation there), expm1f below
          const float x = Ee * inv_kT;
          v = cb * __fdividef(Ee * Ee * Ee, x > 0.5f ? __expf(x) - 1.f : expm1f(x));
        } else {
          v = cb * (Ee * Ee * Ee / expm1(Ee * inv_kT));
        }
        acc[e] += (double)v;
      }
  }
  return n_vis;
}

// Fused point-source mode: the first point spot k >= k0 of the profile inside the batch's ring window, or
// n_spots (the tile's own sweep then makes plan_kernel's ring-drop test, tile_prologue).
__device__ __forceinline__ int fused_next_spot(const DevProfile& pf, int k0) {
  int k = k0;
  while (k < pf.n_spots && pf.spot[k].i_lo > pf.spot[k].i_hi) ++k;
  return k;
}

template <typename Real, int NE_T>
__global__ void __launch_bounds__(512, 2) integrand_bb_kernel(const KernelArgs a) {
  extern __shared__ __align__(16) unsigned char sm[];
  const IntegrandShape& S = a.shape;
  const SmemPtrs s = carve(sm, S);
  __shared__ RingGeom s_g;
  __shared__ int s_int[48];
  __shared__ int s_tile;
  const int tid = threadIdx.x, nt = blockDim.x;
  double* b_c = (double*)s.batch;  // point records, one slot per thread
  double* b_z = b_c + nt;
  int* b_bin = (int*)(b_z + nt);

  // fused point-source mode: this CTA's profile starts from zero flux and counters (ordered before the tiles'
  // atomics by the barrier at the top of the loop); each point spot is planned here as the planner would
  if (a.n_fused > 0) {
    if ((int)blockIdx.x >= a.n_fused) return;
    const DevProfile& pf = a.profiles[blockIdx.x];
    const long long n_flux = (long long)pf.n_bins * pf.n_e;
    for (long long k = tid; k < n_flux; k += nt) a.flux[pf.flux_off + k] = 0.0;
    for (int k = tid; k < kStats; k += nt) pf.stats[k] = 0ull;
    for (int k = tid; k < kMaxSpots * pf.ring_words; k += nt) pf.ring_seen[k] = 0u;
    if (tid == 0) s_tile = -1;  // the spot last taken
  }
  __shared__ Tile s_tile_rec;  // the tile taken (fused mode: built here)
  for (;;) {
    __syncthreads();
    if (tid == 0) {
      if (a.n_fused > 0) {
        const DevProfile& pf = a.profiles[blockIdx.x];
        const int k = fused_next_spot(pf, s_tile + 1);
        s_tile = k;
        s_int[47] = k < pf.n_spots ? 1 : 0;
        s_tile_rec = Tile{(int)blockIdx.x, (short)k, 1, 0, 0, 1, 0, (short)(pf.n_bins * max(pf.n_gl, 1))};
      } else {
        const int t = atomicAdd(a.queue.next, 1);
        const bool live = t < *a.queue.n_tiles && t < a.queue.capacity;
        s_int[47] = live ? 1 : 0;
        if (live) s_tile_rec = a.queue.tiles[t];
      }
    }
    __syncthreads();
    if (!s_int[47]) break;
    const Tile tile = s_tile_rec;
    const DevProfile& p = a.profiles[tile.profile];
    const DevSpot& sp = p.spot[tile.spot];
    const bool point = sp.kind == 1;
    const int n_act = tile_prologue(a, p, sp, tile, s, s_g, s_int, false);
    if (n_act == 0) continue;
    const RingPhi rp = point ? RingPhi{0.0, 0.0} : healpix_ring_phi(p.n_side, tile.ring);

    const DevGrid& G = p.grid;
    const int n_e = G.n_e;
    // partial sums in FP64 in every arithmetic (the FP32 integrand's values are summed exactly enough that the
    // grouping of the points does not show)
    Real E[NE_T];
    double acc[NE_T];
#pragma unroll
    for (int k = 0; k < NE_T; ++k) {
      const int e = tid + k * nt;
      E[k] = e < n_e ? (Real)G.E[e] : (Real)1;
      acc[k] = 0;
    }
    const Real kT = (Real)sp.kT;
    const int n_pp = tile.u1 - tile.u0;  // the tile's phase nodes
    const int n_pts = n_pp * n_act;
    int cur_bin = -1;
    double* flux_base = a.flux + p.flux_off;
    double* comp_base = a.comp ? a.comp + p.flux_off : nullptr;
    const double out_scale = sp.out_scale;
    auto flush = [&]() {
#pragma unroll
      for (int k = 0; k < NE_T; ++k) {
        const int e = tid + k * nt;
        if (e < n_e && acc[k] != 0.0) {
          const size_t o = (size_t)cur_bin * n_e + e;
          comp_add(flux_base + o, comp_base ? comp_base + o : nullptr, acc[k] * out_scale * G.invE[e]);
        }
        acc[k] = 0;
      }
    };
    // Few energies (at most a quarter of the threads): every thread walks a
    // run of consecutive phase points of one element and evaluates each at all
    // energies, instead of the compacted points being walked serially by the
    // threads that own energies.  The lanes of a warp hold consecutive elements
    // at the same phase point, and each thread hunts its next bracket in
    // phase_o from the last one.
    if (n_e * 4 <= nt) {
      const int n_fine = p.n_fine;
      bool ok = true;
      for (int i = tid; i < n_fine; i += nt) ok &= s.P[i + 1] >= s.P[i];
      const bool mono = __syncthreads_and(ok) != 0;
      // per tile, in the lensing-row space the sweep no longer needs: reciprocal
      // phase_o interval widths, the energies and 1/E (when they fit)
      double* inv_dp = (double*)s.rows;
      Real* E_s = (Real*)(inv_dp + n_fine);
      double* invE_s = (double*)(((uintptr_t)(E_s + n_e) + 7) & ~(uintptr_t)7);
      const bool staged = (long)((unsigned char*)(invE_s + n_e) - (unsigned char*)s.rows) <= (long)(S.total - S.off_rows);
      // the phase-major walk also stages each active element's phase shift phi / 2 pi (one division per element
      // per tile instead of one per element and node)
      double* shift_s = invE_s + n_e;
      // FP32 arithmetic: FP32 copies of the fine-phase F and Z after them
      float* F32 = (float*)(shift_s + n_act);
      float* Z32 = F32 + (n_fine + 1);
      const bool fp32 = std::is_same<Real, float>::value;
      const bool pm = n_e <= kPhaseMajorMaxE && mono &&
                      (long)((unsigned char*)(fp32 ? (void*)(Z32 + n_fine + 1) : (void*)(shift_s + n_act)) -
                             (unsigned char*)s.rows) <= (long)(S.total - S.off_rows);
      if (staged) {
        if (mono)
          for (int i = tid; i < n_fine; i += nt) inv_dp[i] = 1.0 / (s.P[i + 1] - s.P[i]);
        for (int e = tid; e < n_e; e += nt) {
          E_s[e] = (Real)G.E[e];
          invE_s[e] = G.invE[e];
        }
        if (pm) {
          for (int jj = tid; jj < n_act; jj += nt) shift_s[jj] = (point ? 0.0 : rp.dphi * (s.j[jj] - rp.jofs)) / kTwoPi;
          if (fp32)
            for (int i = tid; i <= n_fine; i += nt) {
              F32[i] = (float)s.F[i];
              Z32[i] = (float)s.Z[i];
            }
        }
      }
      __syncthreads();
      const double* inv_dp_use = (staged && mono) ? inv_dp : nullptr;
      const int n_fp = n_fine + 1;
      const double P0 = s.P[0];
      const Real inv_kT = (Real)1 / kT;
      if (pm && staged) {
        // Phase-major walk (the os1 light curves: one energy).  A thread walks
        // a contiguous segment of the tile's active elements at one phase
        // point, then at a second one.  The elements' azimuths increase along the ring, so the
        // point's patch phase moves monotonically from one element to the
        // next (wrapping once past 1) and its phase_o bracket is hunted from
        // the previous element's: vhunt's bracket exactly, as phase_o is
        // non-decreasing.  The point's sums stay in FP64 registers; one atomic
        // per energy flushes them at the end of the segment.
        const int n_gl = p.n_gl;
        const double inv_bins = 1. / p.n_bins;
        // Work items pair node k with node k + H, H = ceil(nodes / 2), half a
        // rotation later, on one segment: an element seen at one of the two
        // phases is often hidden at the other, so the pairs cost about the
        // same and the warps finish together.  Each item ends with one
        // compensated atomic per energy, whose returned value the thread
        // waits for, so the items are kept few and long.
        const int H = (n_pp + 1) / 2;
        const int segs = max(1, min(n_act, nt / max(1, H)));
        const double scale = out_scale;
        const int lane = tid & 31;
        unsigned int n_vis = 0;
        for (int it = tid; it < H * segs; it += nt) {
          const int seg = it / H;
          const int jj0 = (int)((long long)n_act * seg / segs), jj1 = (int)((long long)n_act * (seg + 1) / segs);
          for (int half = 0; half < 2; ++half) {
            const int kk = it % H + half * H;
            if (kk >= n_pp) break;
            const int k = tile.u0 + kk;
            int bin, g = 0;
            if (n_gl > 0) {
              bin = k / n_gl;
              g = k - bin * n_gl;
            } else {
              bin = k;
            }
            double ppt, wgl;
            if (n_gl > 0) {
              const double lb = bin * inv_bins, ub = (bin + 1) * inv_bins;
              ppt = 0.5 * (lb + ub + c_gl_nodes[n_gl * (n_gl - 1) / 2 + g] * (ub - lb));
              wgl = 0.5 * 1. * c_gl_weights[n_gl * (n_gl - 1) / 2 + g];
            } else {
              ppt = bin * inv_bins;
              wgl = 1.0;
            }
            double acc[kPhaseMajorMaxE];
#pragma unroll
            for (int e = 0; e < kPhaseMajorMaxE; ++e) acc[e] = 0.0;
            n_vis += n_e == 1 ? pm_walk<Real, 1>(s, inv_dp, F32, Z32, shift_s, E_s, n_e, inv_kT, ppt, wgl, jj0, jj1,
                                                 n_fp, P0, acc)
                              : pm_walk<Real, kPhaseMajorMaxE>(s, inv_dp, F32, Z32, shift_s, E_s, n_e, inv_kT, ppt, wgl,
                                                               jj0, jj1, n_fp, P0, acc);
#pragma unroll
            for (int e = 0; e < kPhaseMajorMaxE; ++e)
              if (e < n_e && acc[e] != 0.0) {
                const size_t o = (size_t)bin * n_e + e;
                comp_add(flux_base + o, comp_base ? comp_base + o : nullptr, acc[e] * scale * invE_s[e]);
              }
          }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) n_vis += __shfl_down_sync(0xffffffffu, n_vis, off);
        if (lane == 0 && n_vis) atomicAdd(&p.stats[3], (unsigned long long)n_vis);
        continue;
      }
      const int runs = max(1, min(n_pp, nt / n_act));  // runs of phase points per element
      const int per_run = (n_pp + runs - 1) / runs;
      const int n_items = n_act * runs;
      const int lane = tid & 31;
      const int n_gl = p.n_gl;
      const double inv_bins = 1. / p.n_bins;
      const double scale = out_scale;
      unsigned int n_vis = 0;
      for (int it0 = 0; it0 < n_items; it0 += nt) {
        const int it = it0 + tid;
        const bool live = it < n_items;
        const int jj = live ? it % n_act : 0;
        const int pp0 = live ? (it / n_act) * per_run : 0;
        const int pp1 = live ? min(n_pp, pp0 + per_run) : 0;
        const double phase_shift = (point ? 0.0 : rp.dphi * (s.j[jj] - rp.jofs)) / kTwoPi;
        int hint = -1;
        for (int k = 0; k < per_run; ++k) {  // the same trip count on every lane
          int bin = INT_MAX;  // lanes without a point: a bin after every real one
          double c = 0, zz = 0;
          bool vis = false;
          if (pp0 + k < pp1) {
            double wgl, z = 0;
            const double flux =
                phase_point_at(s, n_fp, P0, inv_dp_use, n_gl, inv_bins, phase_shift, tile.u0 + pp0 + k, mono, hint, bin,
                               wgl, z);
            if (flux != 0.0) {
              vis = true;
              c = flux * wgl;
              zz = z;
            }
          }
          n_vis += vis ? 1u : 0u;
          // bins never decrease along the lanes (consecutive elements of one run
          // share the phase point; later runs have later points; lanes without a
          // point come last), so the lanes of one bin are one run of lanes, summed
          // by a segmented shuffle reduction into the run's first lane
          const int prev_bin = __shfl_up_sync(0xffffffffu, bin, 1);
          const bool head = (lane == 0 || prev_bin != bin) && bin != INT_MAX;
          const Real cb = (Real)c, zb = (Real)zz;
          for (int e = 0; e < n_e; ++e) {
            double v = 0;
            if (vis) {
              const Real Ee = (staged ? E_s[e] : (Real)G.E[e]) * zb;
              v = (double)(cb * (Ee * Ee * Ee / expm1(Ee * inv_kT)));  // Ibb without its constant (in out_scale)
            }
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
              const double o = __shfl_down_sync(0xffffffffu, v, off);
              const int ob = __shfl_down_sync(0xffffffffu, bin, off);
              if (lane + off < 32 && ob == bin) v += o;
            }
            if (head && v != 0.0) {
              const size_t o = (size_t)bin * n_e + e;
              comp_add(flux_base + o, comp_base ? comp_base + o : nullptr,
                       v * scale * (staged ? invE_s[e] : G.invE[e]));
            }
          }
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) n_vis += __shfl_down_sync(0xffffffffu, n_vis, off);
      if (lane == 0 && n_vis) atomicAdd(&p.stats[3], (unsigned long long)n_vis);
      continue;
    }
    for (int q0 = 0; q0 < n_pts; q0 += nt) {
      bool vis = false;
      double c = 0, zz = 0;
      int bin = 0;
      const int q = q0 + tid;
      if (q < n_pts) {
        double wgl, z = 0, mu = 0;
        const double flux = phase_point(p, s, rp, point, n_act, tile.u0, q, bin, wgl, z, mu);
        if (flux != 0.0) {
          vis = true;
          c = flux * wgl;
          zz = z;
        }
      }
      int n_batch;
      const int slot = block_compact(vis, s_int, &n_batch);
      if (vis) {
        b_c[slot] = c;
        b_z[slot] = zz;
        b_bin[slot] = bin;
      }
      if (tid == 0 && n_batch) atomicAdd(&p.stats[3], (unsigned long long)n_batch);
      __syncthreads();
      for (int b = 0; b < n_batch; ++b) {
        const int bb = b_bin[b];
        if (bb != cur_bin) {
          if (cur_bin >= 0) flush();
          cur_bin = bb;
        }
        const Real cb = (Real)b_c[b], zb = (Real)b_z[b];
#pragma unroll
        for (int k = 0; k < NE_T; ++k) {
          // Ibb(E, kT) = Ibb_constant E^3 / expm1(E / kT) (cpu/unit.hpp:28-31); the constant is in out_scale
          const Real Ee = E[k] * zb;
          const Real I = Ee * Ee * Ee / expm1(Ee / kT);
          acc[k] += (double)(cb * I);
        }
      }
      __syncthreads();
    }
    if (cur_bin >= 0) flush();
  }
}

// ---------------------------------------------------------------------------
// Ring range of disk 1 in element index j: up to two [j_lo, j_hi] ranges
// (with a one-element margin) that contain every active element.
__device__ int candidate_ranges(const DevSpot& s, int N, int i, double c2, double s2, int jmax, int r[2][2]) {
  const double A = s.s1 * s2, B = s.c1 * c2;
  bool full = false;
  double w = 0.0;
  if (A < 1e-12) {
    if (B > s.cos_ar1 - 1e-9)
      full = true;
    else
      return 0;
  } else {
    const double qv = (s.cos_ar1 - B) / A;
    if (qv > 1.0 + 1e-9) return 0;
    if (qv <= -1.0)
      full = true;
    else
      w = acos(fmin(qv, 1.0)) + 1e-7;
    if (w >= kPi) full = true;
  }
  if (full) {
    r[0][0] = 1;
    r[0][1] = jmax;
    return 1;
  }
  const int ii = i > 2 * N ? 4 * N - i : i;
  const double sh = ii < N ? 0.5 : 0.5 * ((ii - N + 1) % 2);
  const double dphi = kTwoPi / jmax;
  const double jc = s.ph1 / dphi + sh, jw = w / dphi;
  long long jlo = (long long)floor(jc - jw) - 1, jhi = (long long)ceil(jc + jw) + 1;
  const long long len = jhi - jlo + 1;
  if (len >= jmax) {
    r[0][0] = 1;
    r[0][1] = jmax;
    return 1;
  }
  long long m = ((jlo - 1) % jmax + jmax) % jmax + 1;  // jlo mapped into [1, jmax]
  if (m + len - 1 <= jmax) {
    r[0][0] = (int)m;
    r[0][1] = (int)(m + len - 1);
    return 1;
  }
  r[0][0] = (int)m;
  r[0][1] = jmax;
  r[1][0] = 1;
  r[1][1] = (int)(m + len - 1 - jmax);
  return 2;
}

// Whether the ring is skipped because fine sample 0 or n_fine-1 is invisible
// (cpu/devarshi24st_cpu.cpp:195), evaluated with the sweep's own arithmetic.
__device__ bool ring_dropped(const DevProfile& p, const DevLens& L, const RingGeom& g, bool nsx) {
  LensRows rows;
  lens_rows_global(L, g.i_u, rows);
  double F, Z, P, MU;
  if (!sweep_sample(p, L, g, rows, 0, nsx, F, Z, P, MU)) return true;
  if (!sweep_sample(p, L, g, rows, p.n_fine - 1, nsx, F, Z, P, MU)) return true;
  return false;
}

__device__ __forceinline__ void push_tile(const WorkQueue& q, const Tile& t) {
  const int k = atomicAdd(q.n_tiles, 1);
  if (k < q.capacity)
    q.tiles[k] = t;
  else
    atomicOr(q.overflow, 1);
}

// One CTA per (profile, spot, ring block): a spot's rings are shared by
// ring_blocks CTAs, so that a small batch plans on many SMs at once.  Every
// chunk of a ring's candidate range becomes ceil(nodes / nodes_per_tile) tiles,
// one per range of phase nodes.
__global__ void plan_kernel(const DevProfile* profiles, int n_profiles, const DevLens L, const WorkQueue q, int chunk,
                            int nodes_per_tile, int ring_blocks) {
  const int ps = blockIdx.x / ring_blocks, rb = blockIdx.x - ps * ring_blocks;
  const int pi = ps / kMaxSpots, si = ps % kMaxSpots;
  if (pi >= n_profiles) return;
  const DevProfile& p = profiles[pi];
  if (si >= p.n_spots) return;
  const DevSpot& sp = p.spot[si];
  const bool nsx = p.atmosphere == 0;
  const int n_nodes = p.n_bins * max(p.n_gl, 1);
  const int npt = nodes_per_tile > 0 ? min(nodes_per_tile, n_nodes) : n_nodes;
  auto push_nodes = [&](Tile t) {
    for (int u = 0; u < n_nodes; u += npt) {
      t.u0 = (short)u;
      t.u1 = (short)min(u + npt, n_nodes);
      push_tile(q, t);
    }
  };
  if (sp.kind == 1) {
    if (sp.i_lo > sp.i_hi || rb != 0) return;  // outside the batch's ring window, or another block's
    if (threadIdx.x == 0) {
      RingGeom g;
      ring_geometry(p, L, sp.cos_theta_pt, sp.dOmega_pt, false, g);
      if (ring_dropped(p, L, g, nsx)) {
        atomicAdd(&p.stats[1], 1ull);
        atomicAdd(&p.stats[2], 1ull);
        atomicAdd(&p.stats[5], 1ull);
      } else {
        push_nodes(Tile{pi, (short)si, 1, 0, 0, 1, 0, 0});
      }
    }
    return;
  }
  const int N = p.n_side;
  for (int i = sp.i_lo + rb * (int)blockDim.x + (int)threadIdx.x; i <= sp.i_hi; i += ring_blocks * (int)blockDim.x) {
    const double z = p.ring[3 * i], c2 = p.ring[3 * i + 1], s2 = p.ring[3 * i + 2];
    const int jmax = healpix_jmax(N, i);
    int r[2][2];
    const int nr = candidate_ranges(sp, N, i, c2, s2, jmax, r);
    if (nr == 0) continue;
    RingGeom g;
    ring_geometry(p, L, z, p.dOmega_hp, false, g);
    if (ring_dropped(p, L, g, nsx)) {
      // count the ring (and its elements) only if it holds active elements
      long long na = 0;
      for (int k = 0; k < nr; ++k)
        for (int j = r[k][0]; j <= r[k][1]; ++j) na += in_spot(sp, c2, s2, healpix_phi(N, i, j)) ? 1 : 0;
      if (na) {
        atomicAdd(&p.stats[1], 1ull);
        atomicAdd(&p.stats[2], 1ull);
        atomicAdd(&p.stats[5], (unsigned long long)na);
        if (g.u_clamped) atomicAdd(&p.stats[4], 1ull);
      }
      continue;
    }
    bool first = true;
    for (int k = 0; k < nr; ++k)
      for (int j0 = r[k][0]; j0 <= r[k][1]; j0 += chunk) {
        const int j1 = min(j0 + chunk, r[k][1] + 1);
        push_nodes(Tile{pi, (short)si, (short)(first ? 1 : 0), i, j0, j1, 0, 0});
        first = false;
      }
  }
}

// ---------------------------------------------------------------------------
template <typename Real>
__global__ void fold_simt_kernel(const FoldJob* jobs, const double* rsp, int n_ch, int n_e, int n_bins,
                                 const double* flux, double* counts) {
  constexpr int TC = 16, TB = 16, TK = 32;
  __shared__ Real sr[TC][TK + 1];
  __shared__ Real sf[TB][TK + 1];
  const FoldJob job = jobs[blockIdx.z];
  const int c0 = blockIdx.x * TC, b0 = blockIdx.y * TB;
  const int tx = threadIdx.x % TB, ty = threadIdx.x / TB;  // tx: bin, ty: channel
  const double* F = flux + job.flux_off;
  Real acc = 0;
  for (int k0 = 0; k0 < n_e; k0 += TK) {
    for (int idx = threadIdx.x; idx < TC * TK; idx += blockDim.x) {
      const int cc = idx / TK, kk = idx % TK;
      const int c = c0 + cc, k = k0 + kk;
      sr[cc][kk] = (c < n_ch && k < n_e) ? (Real)rsp[(size_t)c * n_e + k] : (Real)0;
    }
    for (int idx = threadIdx.x; idx < TB * TK; idx += blockDim.x) {
      const int bb = idx / TK, kk = idx % TK;
      const int b = b0 + bb, k = k0 + kk;
      sf[bb][kk] = (b < n_bins && k < n_e) ? (Real)F[(size_t)b * n_e + k] : (Real)0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < TK; ++kk) acc += sr[ty][kk] * sf[tx][kk];
    __syncthreads();
  }
  const int c = c0 + ty, b = b0 + tx;
  if (c < n_ch && b < n_bins) counts[job.counts_off + (size_t)c * n_bins + b] = (double)acc * job.alpha;
}

}  // namespace

// ---------------------------------------------------------------------------
IntegrandShape make_shape(bool nsx, int nt, int ne_t, int pb, int max_cand, int n_fine, int n_cp, int n_ca, int nE,
                          int nmu, int cells, bool cellk) {
  IntegrandShape s{};
  s.nsx = nsx;
  s.cellk = (nsx && cellk) ? 1 : 0;
  s.nt = nt;
  s.ne_t = ne_t;
  s.pb = pb;
  s.max_cand = max_cand;
  s.n_fine = n_fine;
  s.n_cp = n_cp;
  s.n_ca = n_ca;
  s.nE = nsx ? nE : 0;
  s.nmu = nsx ? nmu : 0;
  s.cells = nsx ? cells : 0;
  auto al = [](long v) { return (int)((v + 15) / 16 * 16); };
  int off = 0;
  s.off_j = off;
  off += al((long)max_cand * 4);
  const long nf1 = n_fine + 1;
  s.off_P = off;
  off += al(nf1 * 8);
  s.off_F = off;
  off += al(nf1 * 8);
  s.off_Z = off;
  off += al(nf1 * 8);
  s.off_MU = off;
  off += al(nf1 * 8);
  s.off_mu = off;
  off += nsx ? al((long)nmu * 8 * 5) : 0;
  s.off_S = off;
  const int rows = al((long)(4 * n_cp + 2 * n_ca) * 8);
  if (s.cellk) {
    // home-cell kernel: odd row stride; the lensing rows (used only by the
    // sweep, before the slice is built) share the slice's space; 32-byte point records
    s.ldS = nmu | 1;
    // rows -2 .. nE + 1, row 0 16-byte aligned
    const int slice = al(((long)((2 * s.ldS + 3) & ~3) + (long)(nE + 2) * s.ldS) * 4);
    s.off_rows = off;
    off += slice > rows ? slice : rows;
    s.off_union = off;
    s.off_batch = off;
    s.off_Q = off;
    off += al((long)nt * 32);
    s.off_hidx = off;
    off += al((long)nf1 * 2);
    s.total = off;
    return s;
  }
  s.ldS = nmu;
  // the slice is stored with the table's 16-byte aligned stride
  const long slice = nsx ? ((long)nE * nmu + 3) / 4 * 4 : 0;
  off += al(slice * 4);
  s.off_union = off;
  const int batch = al((long)nt * kSlotBytes);
  const int qbuf = nsx ? al((long)pb * cells * 16) + al((long)pb * (cells + 3) * 4) : 0;
  s.off_rows = off;
  s.off_batch = off;
  s.off_Q = off + batch;
  off += rows > batch + qbuf ? rows : batch + qbuf;
  s.total = off;
  return s;
}

namespace {
void* kernel_for(const IntegrandShape& s, int precision) {
  if (s.nsx && s.cellk) {
    // register budget: two CTAs per SM (80 registers) up to 384 threads, else one
    const bool two = s.minb >= 2 && s.nt <= 384;
    if (s.maxe_t == 2) {
      if (s.cpl >= 3) return two ? (void*)integrand_nsx_cell_kernel<2, 3, 384, 2> : (void*)integrand_nsx_cell_kernel<2, 3, 512, 1>;
      if (s.cpl == 2) return two ? (void*)integrand_nsx_cell_kernel<2, 2, 384, 2> : (void*)integrand_nsx_cell_kernel<2, 2, 512, 1>;
      return two ? (void*)integrand_nsx_cell_kernel<2, 1, 384, 2> : (void*)integrand_nsx_cell_kernel<2, 1, 512, 1>;
    }
    if (s.maxe_t == 4) {
      if (s.cpl >= 3) return two ? (void*)integrand_nsx_cell_kernel<4, 3, 384, 2> : (void*)integrand_nsx_cell_kernel<4, 3, 512, 1>;
      if (s.cpl == 2) return two ? (void*)integrand_nsx_cell_kernel<4, 2, 384, 2> : (void*)integrand_nsx_cell_kernel<4, 2, 512, 1>;
      return two ? (void*)integrand_nsx_cell_kernel<4, 1, 384, 2> : (void*)integrand_nsx_cell_kernel<4, 1, 512, 1>;
    }
    if (s.maxe_t == 8) {
      if (s.cpl >= 2) return two ? (void*)integrand_nsx_cell_kernel<8, 2, 384, 2> : (void*)integrand_nsx_cell_kernel<8, 2, 512, 1>;
      return two ? (void*)integrand_nsx_cell_kernel<8, 1, 384, 2> : (void*)integrand_nsx_cell_kernel<8, 1, 512, 1>;
    }
    return (void*)integrand_nsx_cell_kernel<16, 1, 512, 1>;
  }
  if (s.nsx) {
    const bool two = s.minb >= 2;
    switch (s.ne_t) {
      case 1: return two ? (void*)integrand_nsx_kernel<1, 2> : (void*)integrand_nsx_kernel<1, 1>;
      case 2: return two ? (void*)integrand_nsx_kernel<2, 2> : (void*)integrand_nsx_kernel<2, 1>;
      default: return (void*)integrand_nsx_kernel<4, 1>;
    }
  }
  if (precision == 1) {
    switch (s.ne_t) {
      case 1: return (void*)integrand_bb_kernel<double, 1>;
      case 2: return (void*)integrand_bb_kernel<double, 2>;
      default: return (void*)integrand_bb_kernel<double, 4>;
    }
  }
  switch (s.ne_t) {
    case 1: return (void*)integrand_bb_kernel<float, 1>;
    case 2: return (void*)integrand_bb_kernel<float, 2>;
    default: return (void*)integrand_bb_kernel<float, 4>;
  }
}
}  // namespace

namespace {
constexpr int kOnceSlots = 4, kOnceDevices = 64;
std::mutex g_once_mu;
bool g_once_done[kOnceSlots][kOnceDevices];
}  // namespace

cudaError_t once_per_device(int slot, cudaError_t (*set_up)()) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (slot < 0 || slot >= kOnceSlots || dev < 0 || dev >= kOnceDevices) return set_up();
  std::lock_guard<std::mutex> lk(g_once_mu);
  if (g_once_done[slot][dev]) return cudaSuccess;
  e = set_up();
  if (e == cudaSuccess) g_once_done[slot][dev] = true;
  return e;
}

namespace {
// every integrand variant gets the largest dynamic shared-memory allowance of the current device
cudaError_t set_integrand_smem() {
  void* fns[] = {(void*)integrand_nsx_cell_kernel<2, 1, 512, 1>, (void*)integrand_nsx_cell_kernel<2, 1, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<2, 2, 512, 1>, (void*)integrand_nsx_cell_kernel<2, 2, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<2, 3, 512, 1>, (void*)integrand_nsx_cell_kernel<2, 3, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<4, 1, 512, 1>, (void*)integrand_nsx_cell_kernel<4, 1, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<4, 2, 512, 1>, (void*)integrand_nsx_cell_kernel<4, 2, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<4, 3, 512, 1>, (void*)integrand_nsx_cell_kernel<4, 3, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<8, 1, 512, 1>, (void*)integrand_nsx_cell_kernel<8, 1, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<8, 2, 512, 1>, (void*)integrand_nsx_cell_kernel<8, 2, 384, 2>,
                 (void*)integrand_nsx_cell_kernel<16, 1, 512, 1>,
                 (void*)integrand_nsx_kernel<1, 1>, (void*)integrand_nsx_kernel<1, 2>,
                 (void*)integrand_nsx_kernel<2, 1>, (void*)integrand_nsx_kernel<2, 2>, (void*)integrand_nsx_kernel<4, 1>,
                 (void*)integrand_bb_kernel<double, 1>, (void*)integrand_bb_kernel<double, 2>,
                 (void*)integrand_bb_kernel<double, 4>, (void*)integrand_bb_kernel<float, 1>,
                 (void*)integrand_bb_kernel<float, 2>, (void*)integrand_bb_kernel<float, 4>};
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  for (void* f : fns) {
    cudaFuncAttributes at{};
    e = cudaFuncGetAttributes(&at, f);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)at.sharedSizeBytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace

cudaError_t configure_integrand_smem(const IntegrandShape&) { return once_per_device(0, set_integrand_smem); }

int max_active_ctas(const IntegrandShape& s) {
  int n = 0;
  void* f = kernel_for(s, s.bb_fp64);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, s.nt, s.total) != cudaSuccess) return 0;
  return n;
}

cudaError_t launch_plan(const DevProfile* profiles, int n_profiles, const DevLens& lens, const WorkQueue& q, int chunk,
                        int nodes_per_tile, cudaStream_t st) {
  if (n_profiles <= 0) return cudaSuccess;
  // a few profiles: up to 32 CTAs share each spot's rings (4N - 1 of them at most)
  const int ring_blocks = std::max(1, std::min(32, 64 / n_profiles));
  plan_kernel<<<n_profiles * kMaxSpots * ring_blocks, 128, 0, st>>>(profiles, n_profiles, lens, q, chunk,
                                                                      nodes_per_tile, ring_blocks);
  return cudaGetLastError();
}

namespace {
// flux += comp: the compensation pool's rounding errors back into the flux pool before the fold
__global__ void add_comp_kernel(double* __restrict__ flux, const double* __restrict__ comp, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    flux[i] += comp[i];
}
}  // namespace

cudaError_t launch_add_comp(double* flux, const double* comp, long long n, int sm_count, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((n + 255) / 256, (long long)sm_count * 8);
  add_comp_kernel<<<(unsigned)blocks, 256, 0, st>>>(flux, comp, n);
  return cudaGetLastError();
}

cudaError_t launch_integrand(const KernelArgs& a, int grid, cudaStream_t st) {
  if (grid <= 0) return cudaSuccess;
  const IntegrandShape& s = a.shape;
  void* f = nullptr;
  f = kernel_for(s, s.bb_fp64);
  void* args[] = {(void*)&a};
  return cudaLaunchKernel(f, dim3(grid), dim3(s.nt), args, s.total, st);
}

cudaError_t launch_fold_simt(const FoldJob* jobs, int n_jobs, const double* rsp, int n_ch, int n_e, int n_bins,
                             const double* flux, double* counts, bool fp64, cudaStream_t st) {
  if (n_jobs <= 0) return cudaSuccess;
  dim3 grid((n_ch + 15) / 16, (n_bins + 15) / 16, n_jobs);
  if (fp64)
    fold_simt_kernel<double><<<grid, 256, 0, st>>>(jobs, rsp, n_ch, n_e, n_bins, flux, counts);
  else
    fold_simt_kernel<float><<<grid, 256, 0, st>>>(jobs, rsp, n_ch, n_e, n_bins, flux, counts);
  return cudaGetLastError();
}

}  // namespace ppm
