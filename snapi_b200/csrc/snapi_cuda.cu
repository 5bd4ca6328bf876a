// libsnapi_cuda -- sm_100a kernels and the C ABI of the SNAPI Stokes hot path.
//
// Sweep kernels: one CTA = SNAPI_CHUNK wavelengths of one pixel, one thread per wavelength.
// The pixel's column record is staged into shared memory with a TMA bulk copy (cp.async.bulk,
// mbarrier completion, bounded wait), the wavelength-independent per-depth constants are built
// once per CTA in shared memory, and every thread runs the depth recursion of its wavelength in
// registers (snapi_sweep.cuh).
//   k_synth          forward sweep -> Stokes
//   k_adj_forward    forward sweep (state to scratch) -> Stokes, chi2 partials, adjoint seed
//   k_adj_rt         reverse DELO + optical-depth sweep per wavelength -> (eta-bar, j-bar) per depth
//   k_adj_opacity    one thread per (pixel, depth, transition or continuum): opacity adjoint summed
//                    over wavelengths in registers -> partial buffer
//   k_adjoint_finish one CTA per pixel: fixed-order gather of the partials, chain rule to the record
//                    fields, contraction with the node tangents -> d chi2 / d node
// The adjoint runs as three kernels rather than one so that every SM holds only one phase's
// instructions at a time and each phase gets its own register budget.
//   k_fd_sweep / k_fd_finish: the plain finite-difference gradient (2 npar + 1 forward solves)
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "snapi_internal.cuh"
#include "snapi_jvp.cuh"

using namespace snapi;

namespace {

// minimum resident CTAs per SM requested from ptxas (register budget per thread =
// 65536 / (SNAPI_CHUNK * MINB))
#ifndef SNAPI_SYN_MINB
#define SNAPI_SYN_MINB (640 / SNAPI_CHUNK)
#endif
#ifndef SNAPI_OP_TILE
#define SNAPI_OP_TILE 16
#endif
constexpr int kOpTile = SNAPI_OP_TILE;  // k_adj_opacity: pixels whose CTAs are grouped by transition
// k_adj_opacity at <= 85 registers (3 x 256 threads per SM): 8 of its 96-thread CTAs per SM
#ifndef SNAPI_OP_MINB
#define SNAPI_OP_MINB 3
#endif
#ifndef SNAPI_RT_MINB
#define SNAPI_RT_MINB 1
#endif

struct CtaPos {
  int pix, var, chunk, l, warp0, wslot;
};
// CTA of C wavelengths (C = blockDim.x): pixel, variant, wavelength chunk; the warp slot is the
// warp's global wavelength index / 32, the same for every C
template <int C = kChunk>
__device__ __forceinline__ CtaPos cta_pos(const KParams &P) {
  CtaPos c;
  const int cta = blockIdx.x;
  c.chunk = cta % P.nchunk;
  const int t = cta / P.nchunk;
  c.var = t % P.nvar;
  c.pix = t / P.nvar;
  c.l = c.chunk * C + threadIdx.x;
  c.warp0 = c.chunk * C + (threadIdx.x & ~31);
  c.wslot = c.warp0 >> 5;
  return c;
}

// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kChunk, SNAPI_SYN_MINB) k_synth(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const CtaPos c = cta_pos(P);
  if (P.skip && P.skip[c.pix]) return;  // CTA-uniform
  PixelView pv;
  if (!stage_pixel(P, c.pix, smem, L, pv, -1, 0.f)) return;
  if (c.warp0 >= P.nl) return;  // warp-uniform: no wavelength left for this warp
  const bool active = c.l < P.nl;
  const int le = active ? c.l : P.nl - 1;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, le, lam, delta);
  float out[4];
  NoScratch ns;
  forward_sweep<false>(pv, lam, delta, out, ns);
  if (active) {
    float4 *o = reinterpret_cast<float4 *>(P.stokes + ((size_t)c.pix * P.nl + c.l) * 4);
    *o = make_float4(out[0], out[1], out[2], out[3]);
  }
}

// Adjoint, phase F: forward sweep storing the per-depth state, the emergent Stokes vector, the
// chi2 partials and the adjoint seed of every wavelength.
// (C wavelengths per CTA: one of kChunkCands; the register budget per thread is the same for all)
template <int C>
__global__ void __launch_bounds__(C, SNAPI_SYN_MINB * kChunk / C) k_adj_forward(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const CtaPos c = cta_pos<C>(P);
  PixelView pv;
  if (!stage_pixel(P, c.pix, smem, L, pv, -1, 0.f)) return;
  if (c.warp0 >= P.nl) return;
  const bool active = c.l < P.nl;
  const int le = active ? c.l : P.nl - 1;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, le, lam, delta);
  DevScratch sc;
  sc.base = P.scratch + (size_t)c.pix * P.nd * 4 * P.lpad;
  sc.lpad = P.lpad;
  sc.l = c.l;
  float out[4];
  forward_sweep<true>(pv, lam, delta, out, sc);
  float seed[4] = {0.f, 0.f, 0.f, 0.f};
  double c2 = 0.0;
  if (active) {
    if (P.stokes) {
      float4 *o = reinterpret_cast<float4 *>(P.stokes + ((size_t)c.pix * P.nl + c.l) * 4);
      *o = make_float4(out[0], out[1], out[2], out[3]);
    }
    c2 = residual_seed(P, c.pix, c.l, out, seed);
  }
  P.seed[(size_t)c.pix * P.lpad + c.l] = make_float4(seed[0], seed[1], seed[2], seed[3]);
  c2 = warp_sum(c2);
  if ((threadIdx.x & 31) == 0) P.c2part[(size_t)c.pix * P.nwslot + c.wslot] = c2;
}

// Adjoint, phase R1: reverse DELO sweep and optical-depth adjoint per wavelength (no opacity
// work, no shared memory); writes (eta-bar, j-bar) of every depth.
// R128: a register budget of 128 per thread (16 warps per SM; ~20 bytes of spills) instead of the
// unbounded one (158 registers, 12 warps per SM); the autotuner picks
template <int C, bool R128>
__global__ void __launch_bounds__(C, R128 ? 512 / C : SNAPI_RT_MINB) k_adj_rt(KParams P) {
  const CtaPos c = cta_pos<C>(P);
  if (c.warp0 >= P.nl) return;
  PixelView pv;
  pv.nd = P.nd;
  pv.D = P.D;
  RtScratch sc;
  sc.state = P.scratch + (size_t)c.pix * P.nd * 4 * P.lpad;
  sc.bars = P.bars + (size_t)c.pix * P.nl * 3 * P.nd;
  sc.lpad = P.lpad;
  sc.l = c.l;
  sc.nd = P.nd;
  sc.write = c.l < P.nl;
  const float4 s4 = P.seed[(size_t)c.pix * P.lpad + c.l];
  const float seed[4] = {s4.x, s4.y, s4.z, s4.w};
  reverse_sweep_rt(pv, seed, sc);
}

// Adjoint, phase R2: opacity adjoint.  CTA = (pixel, group): group 0 the continuum, group 1 + j
// transition j; one thread per (depth, wavelength slice) walks its wavelengths and keeps its
// sums in registers, so the wavelength sums need no shuffles.  CTAs go in tiles of kOpTile pixels,
// group-major inside a tile: an SM mostly runs one group's code at a time while a tile's adjoint
// bars (kOpTile x 0.8 MB) stay in L2 for the other groups (16 pixels measured best: 23.1 ms per
// 4096-pixel adjoint against 23.5 ms pixel-major; the slices gave 24.9 -> 23.4).  Wavelengths whose bars are all zero
// (masked) are skipped.
__global__ void __launch_bounds__(kOpThreads, SNAPI_OP_MINB) k_adj_opacity(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const int ng = 1 + P.nlines, S = P.nslice;
  const int tile = blockIdx.x / (ng * P.optile), r = blockIdx.x % (ng * P.optile);
  const int g = r / P.optile, pix = tile * P.optile + r % P.optile;
  if (pix >= P.npix) return;  // CTA-uniform: the last tile is partial
  PixelView pv;
  if (!stage_pixel(P, pix, smem, L, pv, -1, 0.f)) return;
  const float4 *bars = P.bars + (size_t)pix * P.nl * 3 * P.nd;
  for (int t = threadIdx.x; t < P.nd * S; t += blockDim.x) {
    const int z = t % P.nd, sl = t / P.nd;
    const int l0 = (int)((long long)P.nl * sl / S), l1 = (int)((long long)P.nl * (sl + 1) / S);
    float acc[kOpSlots];
#pragma unroll
    for (int i = 0; i < kOpSlots; ++i) acc[i] = 0.f;
    const DepthConst d = pv.dc[z];
    if (g == 0) {
      for (int l = l0; l < l1; ++l) {
        const float eb0 = bars[(size_t)l * 3 * P.nd + z].x;
        const float jb0 = bars[((size_t)l * 3 + 1) * P.nd + z].w;
        if (eb0 == 0.f && jb0 == 0.f) continue;
        LamConst lam;
        lambda_precompute(P.lamvac[l], lam);
        continuum_opacity_adjoint(d, lam, eb0, jb0, acc);
      }
    } else {
      const LineConst Lc = pv.lc[g - 1];
      const LineDepth q = pv.ld[z * P.nlines + g - 1];
      for (int l = l0; l < l1; ++l) {
        const float4 *b = bars + (size_t)l * 3 * P.nd + z;
        const float4 a = b[0], e = b[P.nd], f = b[2 * P.nd];
        const float etab[7] = {a.x, a.y, a.z, a.w, e.x, e.y, e.z};
        const float jb[4] = {e.w, f.x, f.y, f.z};
        if (a.x == 0.f && a.y == 0.f && a.z == 0.f && a.w == 0.f && e.x == 0.f && e.y == 0.f && e.z == 0.f &&
            e.w == 0.f && f.x == 0.f && f.y == 0.f && f.z == 0.f)
          continue;
        const double lv = P.lamvac[l];
        line_opacity_adjoint(d, q, Lc, pv.compS, pv.compD, (float)lv, (float)(Lc.lam0 - lv), etab, jb, acc,
                             acc + kRedPerLine);
      }
    }
    float *o = P.opart + ((((size_t)pix * ng + g) * S + sl) * P.nd + z) * kOpSlots;
#pragma unroll
    for (int i = 0; i < kOpSlots; ++i) o[i] = acc[i];
  }
}

__global__ void __launch_bounds__(kFinishThreads) k_adjoint_finish(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, true);
  const int pix = blockIdx.x;
  float *acc = reinterpret_cast<float *>(smem + L.acc);
  float *rb = reinterpret_cast<float *>(smem + L.rb);
  double *wred = reinterpret_cast<double *>(smem + L.wred);
  PixelView pv;
  if (!stage_pixel(P, pix, smem, L, pv, -1, 0.f)) return;
  const int nw = (P.nl + 31) / 32;  // warps that held wavelengths
  const int nacc = P.nd * P.nred, nrec = P.nd * P.nfield, ng = 1 + P.nlines, S = P.nslice;
  const float *part = P.opart + (size_t)pix * ng * S * P.nd * kOpSlots;
  // sum of group g's slot k at depth z over the wavelength slices, in a fixed order
  auto slot = [&](int g, int z, int k) {
    float v = 0.f;
    for (int sl = 0; sl < S; ++sl) v += part[(((size_t)g * S + sl) * P.nd + z) * kOpSlots + k];
    return v;
  };
  for (int e = threadIdx.x; e < nacc; e += blockDim.x) {
    const int z = e / P.nred, t = e % P.nred;
    float s = 0.f;
    if (t < R_ST2) {
      s = slot(0, z, t);  // continuum group
    } else if (t < kNumRed) {
      for (int j = 0; j < P.nlines; ++j) s += slot(1 + j, z, kRedPerLine + t - R_ST2);
    } else {
      const int j = (t - kNumRed) / kRedPerLine, k = (t - kNumRed) % kRedPerLine;
      s = slot(1 + j, z, k);
    }
    acc[e] = s;
  }
  for (int i = threadIdx.x; i < nrec; i += blockDim.x) rb[i] = 0.f;
  __syncthreads();
  for (int z = threadIdx.x; z < P.nd; z += blockDim.x)
    depth_chain_adjoint(pv.rec + z * P.nfield, P.nlines, pv.lc, P.lam_mid, pv.dc[z], pv.ld + z * P.nlines,
                        acc + z * P.nred, rb + z * P.nfield);
  __syncthreads();
  if (P.rec_grad)
    for (int i = threadIdx.x; i < nrec; i += blockDim.x)
      P.rec_grad[(size_t)pix * nrec + i] = (double)rb[i] * P.scale2;
  for (int p = 0; p < P.npar; ++p) {
    double g = 0.0;
    if (P.ntcol) {  // packed: node p's columns, each a depth profile of one record field
      const int c0 = P.tcol_off[p], n = (P.tcol_off[p + 1] - c0) * P.nd;
      const float *tp = P.tangent + ((size_t)pix * P.ntcol + c0) * P.nd;
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int c = i / P.nd, z = i % P.nd;
        g += (double)rb[z * P.nfield + P.tcol_field[c0 + c]] * (double)tp[i];
      }
    } else {
      const float *tp = P.tangent + ((size_t)pix * P.npar + p) * nrec;
      for (int i = threadIdx.x; i < nrec; i += blockDim.x) g += (double)rb[i] * (double)tp[i];
    }
    const double gt = block_sum(g, wred);
    if (threadIdx.x == 0) P.grad[(size_t)pix * P.npar + p] = gt * P.scale2;
  }
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += P.c2part[(size_t)pix * P.nwslot + w];
    P.chi2[pix] = s * P.scale2;
  }
}

// finite differences: variant 0 base, 2p+1 plus, 2p+2 minus
__global__ void __launch_bounds__(kChunk, SNAPI_SYN_MINB) k_fd_sweep(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const CtaPos c = cta_pos(P);
  const int pert = c.var == 0 ? -1 : (c.var - 1) / 2;
  const float sign = c.var == 0 ? 0.f : (((c.var - 1) & 1) ? -1.f : 1.f);
  PixelView pv;
  if (!stage_pixel(P, c.pix, smem, L, pv, pert, sign)) return;
  if (c.warp0 >= P.nl) return;
  const bool active = c.l < P.nl;
  const int le = active ? c.l : P.nl - 1;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, le, lam, delta);
  float out[4], seed[4];
  NoScratch ns;
  forward_sweep<false>(pv, lam, delta, out, ns);
  double c2 = active ? residual_seed(P, c.pix, c.l, out, seed) : 0.0;
  c2 = warp_sum(c2);
  if ((threadIdx.x & 31) == 0) P.c2part[((size_t)c.pix * P.nvar + c.var) * P.nwslot + c.wslot] = c2;
}

__global__ void k_fd_finish(KParams P) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= P.npix) return;
  const int nw = (P.nl + 31) / 32;
  auto c2 = [&](int v) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += P.c2part[((size_t)pix * P.nvar + v) * P.nwslot + w];
    return s * P.scale2;
  };
  P.chi2[pix] = c2(0);
  for (int p = 0; p < P.npar; ++p)
    P.grad[(size_t)pix * P.npar + p] = (c2(2 * p + 1) - c2(2 * p + 2)) / (2.0 * P.fd_step[p]);
}

// Node responses dS/dnode_p by central differences of the record along the node tangent:
// CTA (pixel, node, chunk) synthesises the +h and -h records in turn and writes the difference.
__global__ void __launch_bounds__(kChunk, SNAPI_SYN_MINB) k_resp_sweep(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const CtaPos c = cta_pos(P);  // var = node index
  if (P.skip && P.skip[c.pix]) return;  // CTA-uniform
  float plus[4], out[4];
  for (int side = 0; side < 2; ++side) {
    PixelView pv;
    if (!stage_pixel(P, c.pix, smem, L, pv, c.var, side == 0 ? 1.f : -1.f)) return;
    if (c.warp0 < P.nl) {
      const int le = c.l < P.nl ? c.l : P.nl - 1;
      LamConst lam;
      float delta[kMaxLines];
      thread_lambda(P, pv, le, lam, delta);
      NoScratch ns;
      forward_sweep<false>(pv, lam, delta, side == 0 ? plus : out, ns);
    }
    __syncthreads();  // the shared record is restaged for the other side
  }
  if (c.l < P.nl) {
    const float ih = (float)(0.5 / P.fd_step[c.var]);
    float4 *o = reinterpret_cast<float4 *>(P.dstokes + (((size_t)c.pix * P.npar + c.var) * P.nl + c.l) * 4);
    *o = make_float4((plus[0] - out[0]) * ih, (plus[1] - out[1]) * ih, (plus[2] - out[2]) * ih,
                     (plus[3] - out[3]) * ih);
  }
}

// ---- node responses by forward-mode sweeps (snapi_responses_jvp) ----------------------------------
// Phase S: the forward sweep of every wavelength storing its per-depth state (I, K', S, eta_I, dtau)
// in the adjoint's layout (kChunk wavelengths per CTA), and the Stokes vector.
__global__ void __launch_bounds__(kChunk, SNAPI_SYN_MINB) k_resp_state(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const CtaPos c = cta_pos(P);
  if (P.skip && P.skip[c.pix]) return;  // CTA-uniform
  PixelView pv;
  if (!stage_pixel(P, c.pix, smem, L, pv, -1, 0.f)) return;
  if (c.warp0 >= P.nl) return;
  const bool active = c.l < P.nl;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, active ? c.l : P.nl - 1, lam, delta);
  DevScratch sc;
  sc.base = P.scratch + (size_t)c.pix * P.nd * 4 * P.lpad;
  sc.lpad = P.lpad;
  sc.l = c.l;
  float out[4];
  forward_sweep<true>(pv, lam, delta, out, sc);
  if (active && P.stokes) {
    float4 *o = reinterpret_cast<float4 *>(P.stokes + ((size_t)c.pix * P.nl + c.l) * 4);
    *o = make_float4(out[0], out[1], out[2], out[3]);
  }
}

// Phase T: CTA = (pixel, 32 wavelengths, up to kJvpDirs node directions); warp w carries direction
// q0 + w, lane = wavelength.  At each depth the direction-independent part of the opacity tangent
// -- the sums of each line's Zeeman components' W4 values and x / a derivatives and the H-
// exponentials (jvp_basis_task) for the CTA's 32 wavelengths -- is computed once, its tasks (line
// groups) spread over the warps, into shared memory; the depth tangents of the directions
// (DepthTan, LineTan) are items of one (direction, head or line) each, spread over the CTA's
// threads; the DELO step's direction-independent part (weights, the bracket multiplying d tau,
// the LU of A, the optical-depth coefficients: delo_jvp_prep, opd_interior_coef) is one more
// task.  Then each warp forms its direction's opacity tangent from the sums and takes the DELO /
// optical-depth tangent step, the forward values coming from phase S.  Shared buffers are
// double-buffered by depth: one __syncthreads per depth.  Directions come in groups of kJvpDirs,
// every group through the same code, so a direction's result does not depend on how many others
// share its launch.
size_t jvp_smem_extra(int nbasis, int nwarp, int nlines) {
  return sizeof(double) * 2 * 3 * 32 + sizeof(float) * (2 * kDeloPrepFloats * 32 + 2 * 32 * (size_t)(nbasis | 1) +
                                                         2 * (size_t)nwarp * (12 + 5 * nlines));
}

__global__ void __launch_bounds__(32 * kJvpDirs, 2) k_resp_jvp(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const int nchk = (P.nl + 31) >> 5, ngrp = (P.npar + kJvpDirs - 1) / kJvpDirs;
  int b = blockIdx.x;
  const int chunk = b % nchk;
  b /= nchk;
  const int grp = b % ngrp, pix = b / ngrp;
  const int nwarp = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = grp * kJvpDirs + warp;
  const bool live = q < P.npar;  // warps past the last direction only help with the shared sums
  if (P.skip && P.skip[pix]) return;  // CTA-uniform
  PixelView pv;
  if (!stage_pixel(P, pix, smem, L, pv, -1, 0.f)) return;
  const int nd = P.nd, nlines = P.nlines, dtn = 12 + 5 * nlines;
  const int ntask = jvp_basis_tasks(pv.lc, nlines), bstride = jvp_basis_size(pv.lc, nlines) | 1;
  double *Pd = reinterpret_cast<double *>(smem + L.total);  // [2][3][32]: optical-depth coefficients
  float *Pf = reinterpret_cast<float *>(Pd + 2 * 3 * 32);    // [2][kDeloPrepFloats][32]: DeloPrep
  float *Bs = Pf + 2 * kDeloPrepFloats * 32;                 // [2][32][bstride]
  float *DT = Bs + 2 * 32 * bstride;                         // [2][nwarp][dtn]
  const int prep_warp = ntask % nwarp;                       // the step's shared part: task ntask
  const int nlive = min(kJvpDirs, P.npar - grp * kJvpDirs), nitem = nlive * (1 + nlines);
  const int l = chunk * 32 + lane;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, l < P.nl ? l : P.nl - 1, lam, delta);
  DevScratch st;
  st.base = P.scratch + (size_t)pix * nd * 4 * P.lpad;
  st.lpad = P.lpad;
  st.l = l;
  // step: the DELO step z + 1 -> z of the loop below whose shared part this round prepares (-1: none)
  auto prepare = [&](int z, int buf, int step) {
    if (step >= 0 && warp == prep_warp) {
      float Ip[4], kp_p[6], S_p[4], e_p, t_p, Ic[4], kp_c[6], S_c[4], e_c, tau, Id[4], kp_d[6], S_d[4], e_d, t_d;
      st.load(step + 1, Ip, kp_p, S_p, e_p, t_p);
      st.load(step, Ic, kp_c, S_c, e_c, tau);
      st.load(step - 1, Id, kp_d, S_d, e_d, t_d);
      DeloPrep pr;
      delo_jvp_prep(Ip, kp_p, S_p, kp_c, S_c, tau, Ic, pr);
      const float *pf = &pr.w0;
      for (int k = 0; k < kDeloPrepFloats; ++k) Pf[(buf * kDeloPrepFloats + k) * 32 + lane] = pf[k];
      double g[3];
      opd_interior_coef(e_p, e_c, e_d, pv.D[step], pv.D[step - 1], g);
      for (int k = 0; k < 3; ++k) Pd[(buf * 3 + k) * 32 + lane] = g[k];
    }
    // the depth tangents of the group's directions: one item per (direction, head or line), the
    // items on the threads counted from the CTA's last one (the basis tasks start at warp 0)
    for (int t = nwarp * 32 - 1 - threadIdx.x; t < nitem; t += nwarp * 32) {
      const int w = t < nlive ? t : (t - nlive) / nlines;
      const float *rz = pv.rec + z * P.nfield;
      const float *tz = P.tangent + (((size_t)pix * P.npar + grp * kJvpDirs + w) * nd + z) * P.nfield;
      float *dt = DT + (buf * nwarp + w) * dtn;
      DepthTanHead h;
      if (t < nlive) {
        depth_tangent_head(rz, tz, P.lam_mid, *reinterpret_cast<DepthTan *>(dt), h);
      } else {
        const int j = (t - nlive) % nlines;
        depth_tangent_scalars(rz, tz, h);
        depth_tangent_line(rz, tz, pv.lc[j], pv.ld[z * nlines + j], j, h, reinterpret_cast<LineTan *>(dt + 12)[j]);
      }
    }
    float *bl = Bs + (buf * 32 + lane) * bstride;
    for (int k = warp; k < ntask; k += nwarp)
      jvp_basis_task(pv.dc[z], pv.ld + z * nlines, pv.lc, nlines, pv.compS, pv.compD, lam, delta, k, bl);
  };
  auto tangent = [&](int z, int buf, float *kp, float *S, float &e, float *dkp, float *dS, float &de) {
    const float *dt = DT + (buf * nwarp + warp) * dtn;
    const float *bl = Bs + (buf * 32 + lane) * bstride;
    float deta[7], djj[4], I[4], tau;
    cell_opacity_jvp(pv.dc[z], pv.ld + z * nlines, pv.lc, nlines, lam, delta, bl,
                     *reinterpret_cast<const DepthTan *>(dt), reinterpret_cast<const LineTan *>(dt + 12), deta, djj);
    st.load(z, I, kp, S, e, tau);
    depth_opacity_jvp(kp, S, e, deta, djj, dkp, dS, de);
  };
  float kA[6], SA[4], eA, dkA[6], dSA[4], deA, kB[6], SB[4], eB, dkB[6], dSB[4], deB;
  float kC[6], SC[4], eC, dkC[6], dSC[4], deC;
  prepare(nd - 1, 0, -1);
  __syncthreads();
  if (live) tangent(nd - 1, 0, kA, SA, eA, dkA, dSA, deA);
  prepare(nd - 2, 1, -1);
  __syncthreads();
  if (live) tangent(nd - 2, 1, kB, SB, eB, dkB, dSB, deB);
  float dI[4] = {live ? dSA[0] : 0.f, 0.f, 0.f, 0.f};
  double dopd_below = live ? ((double)deB - (double)deA) / pv.D[nd - 2] : 0.0;
  int buf = 0;
  for (int z = nd - 2; z >= 1; --z) {
    prepare(z - 1, buf, z);
    __syncthreads();
    if (live) {
      tangent(z - 1, buf, kC, SC, eC, dkC, dSC, deC);
      double g[3];
      for (int k = 0; k < 3; ++k) g[k] = Pd[(buf * 3 + k) * 32 + lane];
      const double dopd_z = opd_interior_apply(g, deA, deB, deC);
      const float dtau = (float)bezier_dtau_jvp(deA, deB, dopd_below, dopd_z, pv.D[z]);
      DeloPrep pr;
      float *pf = &pr.w0;
      for (int k = 0; k < kDeloPrepFloats; ++k) pf[k] = Pf[(buf * kDeloPrepFloats + k) * 32 + lane];
      float Ip[4], Ic[4];
      st.load_I(z + 1, Ip);
      st.load_I(z, Ic);
      float dIn[4];
      delo_jvp_apply(pr, Ip, kA, Ic, dI, dkA, dSA, dkB, dSB, dtau, dIn);
#pragma unroll
      for (int s = 0; s < 4; ++s) dI[s] = dIn[s];
#pragma unroll
      for (int k = 0; k < 6; ++k) { kA[k] = kB[k]; kB[k] = kC[k]; dkA[k] = dkB[k]; dkB[k] = dkC[k]; }
#pragma unroll
      for (int s = 0; s < 4; ++s) { SA[s] = SB[s]; SB[s] = SC[s]; dSA[s] = dSB[s]; dSB[s] = dSC[s]; }
      eA = eB; eB = eC; deA = deB; deB = deC;
      dopd_below = dopd_z;
    }
    buf ^= 1;
  }
  if (live && l < P.nl) {  // the top point copies the one below
    float4 *o = reinterpret_cast<float4 *>(P.dstokes + (((size_t)pix * P.npar + q) * P.nl + l) * 4);
    *o = make_float4(dI[0], dI[1], dI[2], dI[3]);
  }
}

void launch_jvp(int nctas, int nwarp, size_t smem, cudaStream_t st, const KParams &P) {
  k_resp_jvp<<<nctas, 32 * nwarp, smem, st>>>(P);
}

double airtovac_d(double lambda_air) {  // cmlib/mathtools.cc:1325-1330
  double s = 1E4 / (lambda_air * 1E8);
  double n = 1.0 + 0.00008336624212083 + 0.02408926869968 / (130.1065924522 - s * s) +
             0.0001599740894897 / (38.92568793293 - s * s);
  return lambda_air * n;
}

// copy helper: host -> device staging, or device pointer passthrough
template <class T>
int stage_in(snapi_ctx *ctx, const T *src, T *dbuf, size_t n, int mem, const T **out) {
  if (!src) { *out = nullptr; return SNAPI_OK; }
  if (mem == SNAPI_MEM_DEVICE) { *out = src; return SNAPI_OK; }
  SNAPI_CK(cudaMemcpyAsync(dbuf, src, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
  *out = dbuf;
  return SNAPI_OK;
}

int sweep_ctas(const snapi_ctx *ctx, int nb, int nvar = 1) { return nb * nvar * ctx->nchunk; }

}  // namespace

cudaError_t snapi::launch_synth(const snapi_ctx *ctx, const KParams &P) {
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  k_synth<<<P.npix * ctx->nchunk, kChunk, L.total, ctx->stream>>>(P);
  return cudaGetLastError();
}
cudaError_t snapi::launch_synth_state(const snapi_ctx *ctx, const KParams &P) {
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  KParams Q = P;
  Q.scratch = ctx->d_scratch;
  Q.nvar = 1;
  k_resp_state<<<P.npix * ctx->nchunk, kChunk, L.total, ctx->stream>>>(Q);
  return cudaGetLastError();
}
cudaError_t snapi::launch_responses(const snapi_ctx *ctx, const KParams &P, bool state_ready) {
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  if (ctx->jac_tangent) {  // forward-mode sweeps (the state in the adjoint's scratch)
    KParams Q = P;
    Q.scratch = ctx->d_scratch;
    Q.stokes = nullptr;
    Q.nvar = 1;  // k_resp_state: CTA = (pixel, chunk); k_resp_jvp indexes its own CTAs
    const int nwarp = std::min(P.npar, kJvpDirs), ngrp = (P.npar + kJvpDirs - 1) / kJvpDirs;
    const size_t smem = L.total + jvp_smem_extra(ctx->nbasis, nwarp, ctx->nlines);
    const size_t nrec = (size_t)ctx->nd * ctx->nfield;
    // in batches of max_batch pixels: the forward state lives in the adjoint's scratch
    for (int p0 = 0; p0 < P.npix; p0 += ctx->max_batch) {
      KParams R = Q;
      R.npix = std::min(ctx->max_batch, P.npix - p0);
      R.rec = P.rec + p0 * nrec;
      R.tangent = P.tangent + (size_t)p0 * P.npar * nrec;
      R.dstokes = P.dstokes + (size_t)p0 * P.npar * ctx->nl * 4;
      R.skip = P.skip ? P.skip + p0 : nullptr;
      cudaError_t e = cudaSuccess;
      if (!(state_ready && P.npix <= ctx->max_batch)) {
        k_resp_state<<<R.npix * ctx->nchunk, kChunk, L.total, ctx->stream>>>(R);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
      launch_jvp(R.npix * ((ctx->nl + 31) / 32) * ngrp, nwarp, smem, ctx->stream, R);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  k_resp_sweep<<<P.npix * P.nvar * ctx->nchunk, kChunk, L.total, ctx->stream>>>(P);
  return cudaGetLastError();
}

namespace {

// the adjoint's kernel sequence for nb pixels (P.npix = nb)
constexpr int kAdjointLaunches = 4;
// with the launch shape cfg: cfg.chunk wavelengths per sweep CTA (the forward state and seed are
// laid out with lpad = that chunk's padding; the buffers hold the widest), cfg.optile pixels per
// opacity-adjoint tile
void launch_adjoint(const KParams &P0, int nb, const AdjCfg &cfg, size_t smem_sweep, size_t smem_fin,
                    cudaStream_t st) {
  KParams P = P0;
  P.nchunk = (P.nl + cfg.chunk - 1) / cfg.chunk;
  P.lpad = P.nchunk * cfg.chunk;
  P.nwslot = P.lpad / 32;
  P.optile = cfg.optile;
  const int nsw = nb * P.nchunk;
  if (cfg.chunk == 32) {
    k_adj_forward<32><<<nsw, 32, smem_sweep, st>>>(P);
    if (cfg.rt128) k_adj_rt<32, true><<<nsw, 32, 0, st>>>(P);
    else k_adj_rt<32, false><<<nsw, 32, 0, st>>>(P);
  } else if (cfg.chunk == 128) {
    k_adj_forward<128><<<nsw, 128, smem_sweep, st>>>(P);
    if (cfg.rt128) k_adj_rt<128, true><<<nsw, 128, 0, st>>>(P);
    else k_adj_rt<128, false><<<nsw, 128, 0, st>>>(P);
  } else {
    k_adj_forward<64><<<nsw, 64, smem_sweep, st>>>(P);
    if (cfg.rt128) k_adj_rt<64, true><<<nsw, 64, 0, st>>>(P);
    else k_adj_rt<64, false><<<nsw, 64, 0, st>>>(P);
  }
  const int nthr = std::min(kOpThreads, (P.nd * P.nslice + 31) / 32 * 32);
  const int ntile = (nb + P.optile - 1) / P.optile;
  k_adj_opacity<<<ntile * (1 + P.nlines) * P.optile, nthr, smem_sweep, st>>>(P);
  k_adjoint_finish<<<nb, kFinishThreads, smem_fin, st>>>(P);
}

// The autotuner's choice for an adjoint of nb pixels: each launch shape is run once on the call's
// own inputs (all shapes compute the same bits), timed by CUDA events; first the chunk width at
// the default tile, then the tile at the best width, then the reverse sweep's register budget.
AdjCfg tune_adjoint(snapi_ctx *ctx, const KParams &P, int nb, size_t smem_sweep, size_t smem_fin) {
  AdjCfg best{kChunk, kOpTile, 0};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return best;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return best; }
  float best_ms = -1.f;
  auto trial = [&](const AdjCfg &c) {
    cudaEventRecord(e0, ctx->stream);
    launch_adjoint(P, nb, c, smem_sweep, smem_fin, ctx->stream);
    cudaEventRecord(e1, ctx->stream);
    float ms = -1.f;
    if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    if (ms > 0.f && (best_ms < 0.f || ms < best_ms)) { best_ms = ms; best = c; }
  };
  for (int ch : kChunkCands)
    if ((ctx->nl + ch - 1) / ch * ch <= ctx->lpad_max) trial(AdjCfg{ch, kOpTile, 0});
  const int bc = best.chunk;
  for (int t : kOpTileCands)
    if (t != kOpTile) trial(AdjCfg{bc, t, 0});
  trial(AdjCfg{best.chunk, best.optile, 1});
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace

namespace snapi {

int set_err(snapi_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

// ---- autotuner bookkeeping --------------------------------------------------------------------
int tune_bucket(int npix) {
  int b = 64;
  while (b < npix && b < (1 << 30)) b <<= 1;
  return b;
}

// the cache file's key of this context's problem shape on its device
static std::string tune_key(const snapi_ctx *ctx) {
  cudaDeviceProp prop;
  std::string name = cudaGetDeviceProperties(&prop, ctx->device) == cudaSuccess ? prop.name : "unknown";
  for (char &ch : name)
    if (ch == ' ' || ch == '|') ch = '_';
  char b[256];
  snprintf(b, sizeof b, "%s|%d|%d|%d|%d", name.c_str(), ctx->nd, ctx->nl, ctx->nlines, ctx->ncomp);
  return b;
}

bool tuned_adj(const snapi_ctx *ctx, int npix, AdjCfg *cfg) {
  const int b = tune_bucket(npix);
  for (const auto &e : ctx->adj_tuned)
    if (e.first == b) { *cfg = e.second; return true; }
  return false;
}

bool tuned_build(const snapi_ctx *ctx, int npix, BuildCfg *cfg) {
  const int b = tune_bucket(npix);
  for (const auto &e : ctx->build_tuned)
    if (e.first == b) { *cfg = e.second; return true; }
  return false;
}

static void tune_append(const snapi_ctx *ctx, const char *line) {
  if (ctx->tune_cache.empty()) return;
  FILE *f = fopen(ctx->tune_cache.c_str(), "a");
  if (!f) return;
  fprintf(f, "%s|%s\n", tune_key(ctx).c_str(), line);
  fclose(f);
}

void tune_store_adj(snapi_ctx *ctx, int npix, const AdjCfg &cfg) {
  ctx->adj_tuned.emplace_back(tune_bucket(npix), cfg);
  char b[96];
  snprintf(b, sizeof b, "adj|%d|%d|%d|%d", tune_bucket(npix), cfg.chunk, cfg.optile, cfg.rt128);
  tune_append(ctx, b);
}

void tune_store_build(snapi_ctx *ctx, int npix, const BuildCfg &cfg) {
  ctx->build_tuned.emplace_back(tune_bucket(npix), cfg);
  char b[96];
  snprintf(b, sizeof b, "build|%d|%d|%d", tune_bucket(npix), cfg.he, cfg.var);
  tune_append(ctx, b);
}

// earlier tunings of this shape on this device from the cache file (later lines win)
static void tune_load(snapi_ctx *ctx) {
  if (ctx->tune_cache.empty()) return;
  FILE *f = fopen(ctx->tune_cache.c_str(), "r");
  if (!f) return;
  const std::string key = tune_key(ctx) + "|";
  char line[512];
  auto member = [](const int *cands, int v) { return v == cands[0] || v == cands[1] || v == cands[2]; };
  while (fgets(line, sizeof line, f)) {
    if (strncmp(line, key.c_str(), key.size()) != 0) continue;
    int b = 0, x = 0, y = 0, z = 0;
    const char *rest = line + key.size();
    if (sscanf(rest, "adj|%d|%d|%d|%d", &b, &x, &y, &z) == 4 && member(kChunkCands, x) &&
        member(kOpTileCands, y) && (z == 0 || z == 1)) {
      ctx->adj_tuned.insert(ctx->adj_tuned.begin(), {b, AdjCfg{x, y, z}});
    } else if (sscanf(rest, "build|%d|%d|%d", &b, &x, &y) == 3 && member(kHeCands, x) && member(kVarCands, y)) {
      ctx->build_tuned.insert(ctx->build_tuned.begin(), {b, BuildCfg{x, y}});
    }
  }
  fclose(f);
}

int ensure_npar(snapi_ctx *ctx, int npar) {
  if (npar <= ctx->cap_npar) return SNAPI_OK;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield, B = ctx->max_batch;
  cudaFree(ctx->d_tan); cudaFree(ctx->d_grad); cudaFree(ctx->d_c2part); cudaFree(ctx->d_step);
  cudaFree(ctx->d_dstokes);
  ctx->d_tan = nullptr; ctx->d_grad = nullptr; ctx->d_c2part = nullptr; ctx->d_step = nullptr;
  ctx->d_dstokes = nullptr;
  ctx->cap_npar = 0;
  SNAPI_CK(cudaMalloc(&ctx->d_tan, sizeof(float) * B * npar * nrec));
  SNAPI_CK(cudaMalloc(&ctx->d_grad, sizeof(double) * B * npar));
  SNAPI_CK(cudaMalloc(&ctx->d_c2part, sizeof(double) * B * (2 * npar + 1) * (ctx->lpad_max / 32)));
  SNAPI_CK(cudaMalloc(&ctx->d_step, sizeof(double) * npar));
  SNAPI_CK(cudaMalloc(&ctx->d_dstokes, sizeof(float) * B * npar * ctx->nl * 4));
  ctx->cap_npar = npar;
  return SNAPI_OK;
}

KParams base_params(const snapi_ctx *ctx) {
  KParams P;
  memset(&P, 0, sizeof P);
  P.nd = ctx->nd; P.nl = ctx->nl; P.nlines = ctx->nlines; P.nfield = ctx->nfield; P.lpad = ctx->lpad;
  P.ncomp = ctx->ncomp; P.nred = ctx->nred; P.nchunk = ctx->nchunk; P.nwslot = ctx->nwslot; P.nvar = 1;
  P.optile = kOpTile;
  P.nslice = op_slices(ctx->nd);
  P.lam_mid = ctx->lam_mid; P.scale2 = ctx->scale2;
  P.lamvac = ctx->d_lamvac; P.lines = ctx->d_lines; P.compS = ctx->d_compS; P.compD = ctx->d_compD;
  P.D = ctx->d_D; P.status = ctx->d_status;
  P.scratch = ctx->d_scratch; P.seed = ctx->d_seed; P.bars = ctx->d_bars; P.opart = ctx->d_opart;
  P.c2part = ctx->d_c2part;
  return P;
}

int check_status(snapi_ctx *ctx) {
  int st = 0;
  SNAPI_CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  SNAPI_CK(cudaStreamSynchronize(ctx->stream));
  if (st != 0) {
    int zero = 0;
    cudaMemcpy(ctx->d_status, &zero, sizeof(int), cudaMemcpyHostToDevice);
    return set_err(ctx, st, "device status %d (a CTA gave up waiting for its TMA copy)", st);
  }
  return SNAPI_OK;
}

}  // namespace snapi

namespace snapi {
// Dynamic shared-memory limit of every kernel launched with more than 48 KB, set to `bytes` (the
// device's opt-in maximum) on the current device.
cudaError_t raise_smem_limits(int bytes) {
  const void *k[] = {(const void *)k_synth, (const void *)k_fd_sweep, (const void *)k_resp_sweep,
                     (const void *)k_adj_forward<32>, (const void *)k_adj_forward<64>,
                     (const void *)k_adj_forward<128>, (const void *)k_adj_opacity,
                     (const void *)k_adjoint_finish, (const void *)k_resp_state, (const void *)k_resp_jvp};
  for (const void *f : k) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
}  // namespace snapi

extern "C" {

int snapi_zeeman_pattern(int ju2, int jl2, double gu, double gl, snapi_line *L) {
  if (!L) return SNAPI_EINVAL;
  for (int g = 0; g < 3; ++g) {
    L->ncomp[g] = 0;
    for (int i = 0; i < SNAPI_MAX_COMP; ++i) { L->S[g][i] = 0.0; L->D[g][i] = 0.0; }
  }
  L->split = ((ju2 - jl2 == 2) || (ju2 - jl2 == -2) || ((ju2 == jl2) && (ju2 != 0))) ? 1 : 0;
  if (!L->split) return SNAPI_OK;
  const int jmin2 = ju2 < jl2 ? ju2 : jl2;
  if (jmin2 + 1 > SNAPI_MAX_COMP || (ju2 + jl2) / 2 > SNAPI_MAX_COMP) return SNAPI_EINVAL;
  L->ncomp[0] = jmin2 + 1;
  L->ncomp[1] = L->ncomp[2] = (ju2 + jl2) / 2;
  const double ju = ju2 / 2.0, jmin = jmin2 / 2.0;
  double np = 0, nb = 0, nr = 0;
  if (ju2 == jl2) {  // delta J = 0
    for (int i = 0; i < L->ncomp[0]; ++i) {
      const double m = (double)i - ju;
      L->S[0][i] = m * m;
      L->D[0][i] = m * (gl - gu);
      np += L->S[0][i];
    }
    for (int i = 0; i < L->ncomp[0]; ++i) L->S[0][i] /= np;
    for (int i = 0; i < L->ncomp[1]; ++i) {
      double m = (double)i - ju + 1.0;
      L->S[1][i] = 0.5 * (ju + m) * (ju - m + 1.0);
      nb += L->S[1][i];
      L->D[1][i] = m * (gl - gu) - gl;
      m = (double)i - ju;
      L->S[2][i] = 0.5 * (ju - m) * (ju + m + 1);
      nr += L->S[2][i];
      L->D[2][i] = m * (gl - gu) + gl;
    }
    for (int i = 0; i < L->ncomp[1]; ++i) { L->S[1][i] /= nb; L->S[2][i] /= nr; }
  } else {  // delta J = +-1
    const double jl = jl2 / 2.0;
    const int offset = (jl2 > ju2) ? 1 : 0;
    for (int i = 0; i < L->ncomp[0]; ++i) {
      const double m = (double)i - jmin;
      if (jl < ju) {
        L->S[1][i] = 0.5 * (jmin + m + 1) * (jmin + m + 2);
        L->S[0][i] = (jmin + 1) * (jmin + 1) - m * m;
        L->S[2][i] = 0.5 * (jmin - m + 1) * (jmin - m + 2);
      } else {
        L->S[1][i] = 0.5 * (jmin - m + 1) * (jmin - m + 2);
        L->S[0][i] = (jmin + 1) * (jmin + 1) - m * m;
        L->S[2][i] = 0.5 * (jmin + m + 1) * (jmin + m + 2);
      }
      np += L->S[0][i]; nr += L->S[2][i]; nb += L->S[1][i];
      L->D[0][i] = m * (gl - gu);
      L->D[1][i] = (m - offset) * (gl - gu) - gu;
      L->D[2][i] = (m + offset) * (gl - gu) + gu;
    }
    for (int i = 0; i < L->ncomp[0]; ++i) { L->S[0][i] /= np; L->S[1][i] /= nb; L->S[2][i] /= nr; }
  }
  return SNAPI_OK;
}

void *snapi_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}
void snapi_host_free(void *p) {
  if (p) cudaFreeHost(p);
}

const char *snapi_last_error(const snapi_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }
void *snapi_stream(snapi_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
double snapi_last_kernel_ms(const snapi_ctx *ctx) { return ctx ? ctx->last_ms : 0.0; }
int snapi_jacobian_mode(snapi_ctx *ctx, int mode) {
  if (!ctx) return SNAPI_EINVAL;
  if (mode != SNAPI_JACOBIAN_FD && mode != SNAPI_JACOBIAN_TANGENT)
    return set_err(ctx, SNAPI_EINVAL, "snapi_jacobian_mode: unknown mode %d", mode);
  if (mode == SNAPI_JACOBIAN_TANGENT) {  // the state layout needs the compiled sweep width's padding
    const size_t smem = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false).total +
                        jvp_smem_extra(ctx->nbasis, kJvpDirs, ctx->nlines);
    int maxsm = 0;
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    if ((int)smem > maxsm)
      return set_err(ctx, SNAPI_EINVAL, "snapi_jacobian_mode: the problem needs %zu B of shared memory", smem);
  }
  ctx->jac_tangent = mode == SNAPI_JACOBIAN_TANGENT;
  return SNAPI_OK;
}

int snapi_autotune(snapi_ctx *ctx, int mode, const char *cache_path) {
  if (!ctx) return SNAPI_EINVAL;
  if (mode != 0 && mode != 1) return set_err(ctx, SNAPI_EINVAL, "snapi_autotune: mode must be 0 or 1");
  ctx->tune = mode;
  ctx->adj_tuned.clear();
  ctx->build_tuned.clear();
  ctx->tune_cache = cache_path ? cache_path : "";
  if (mode) tune_load(ctx);
  return SNAPI_OK;
}

int snapi_tuned_config(const snapi_ctx *ctx, int npix, int *cfg) {
  if (!ctx || !cfg) return SNAPI_EINVAL;
  AdjCfg a{kChunk, kOpTile, 0};
  BuildCfg b{kHeDefault, kVarDefault};
  const bool ha = ctx->tune && tuned_adj(ctx, npix, &a), hb = ctx->tune && tuned_build(ctx, npix, &b);
  cfg[0] = a.chunk;
  cfg[1] = a.optile;
  cfg[2] = b.he;
  cfg[3] = b.var;
  cfg[4] = a.rt128;
  return (ha ? 1 : 0) | (hb ? 2 : 0);
}

double snapi_last_phase_ms(const snapi_ctx *ctx, int phase) {
  return (ctx && phase >= 0 && phase < 2) ? ctx->phase_ms[phase] : 0.0;
}
int snapi_last_launches(const snapi_ctx *ctx) { return ctx ? ctx->last_launches : 0; }

void snapi_destroy(snapi_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  lm_free(ctx);
  eos_free(ctx);
  void *bufs[] = {ctx->d_lamvac, ctx->d_D, ctx->d_lines, ctx->d_compS, ctx->d_compD, ctx->d_status,
                  ctx->d_rec, ctx->d_stokes, ctx->d_obs, ctx->d_mask, ctx->d_tan, ctx->d_recgrad,
                  ctx->d_dstokes, ctx->d_opart, ctx->d_seed, ctx->d_bars, ctx->d_grad, ctx->d_chi2, ctx->d_c2part, ctx->d_step,
                  ctx->d_scratch, ctx->d_tcol, ctx->d_lamair, ctx->d_psf_kt};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  for (int h = 0; h < snapi_ctx::kStageChunks; ++h)
    if (ctx->ev_copy[h]) cudaEventDestroy(ctx->ev_copy[h]);
  if (ctx->ev_free) cudaEventDestroy(ctx->ev_free);
  delete ctx;
}

snapi_ctx *snapi_create(const snapi_problem *prob, int device, int *status) {
  auto fail = [&](snapi_ctx *c, int code) -> snapi_ctx * {
    if (status) *status = code;
    if (c) {
      fprintf(stderr, "snapi_create: %s\n", c->err.c_str());
      snapi_destroy(c);
    }
    return nullptr;
  };
  if (!prob) return fail(nullptr, SNAPI_EINVAL);
  snapi_ctx *ctx = new snapi_ctx();
  ctx->device = device;
  if (prob->nd < 3 || prob->nlambda < 1 || prob->nlambda > SNAPI_MAX_LAMBDA || prob->nlines < 0 ||
      prob->nlines > SNAPI_MAX_LINES || !prob->lambda_air || !prob->tau500 || (prob->nlines && !prob->lines) ||
      !(prob->mu > 0.0 && prob->mu <= 1.0) || !(prob->stokes_scale > 0.0) || prob->max_batch < 0) {
    set_err(ctx, SNAPI_EINVAL, "invalid problem (nd>=3, 1<=nlambda<=%d, 0<=nlines<=%d, 0<mu<=1, stokes_scale>0)",
            SNAPI_MAX_LAMBDA, SNAPI_MAX_LINES);
    return fail(ctx, SNAPI_EINVAL);
  }
  for (int i = 0; i + 1 < prob->nd; ++i)
    if (!(prob->tau500[i + 1] > prob->tau500[i])) {
      set_err(ctx, SNAPI_EINVAL, "tau500 must increase from the top down");
      return fail(ctx, SNAPI_EINVAL);
    }
  if (cudaSetDevice(device) != cudaSuccess) {
    set_err(ctx, SNAPI_ECUDA, "cudaSetDevice(%d) failed", device);
    return fail(ctx, SNAPI_ECUDA);
  }
  ctx->nd = prob->nd;
  ctx->nl = prob->nlambda;
  ctx->nlines = prob->nlines;
  ctx->nfield = SNAPI_NFIELD0 + 3 * prob->nlines;
  ctx->nred = kNumRed + kRedPerLine * prob->nlines;
  ctx->nchunk = (prob->nlambda + kChunk - 1) / kChunk;
  ctx->lpad = ctx->nchunk * kChunk;
  ctx->nwslot = ctx->lpad / 32;
  ctx->lpad_max = std::max(ctx->lpad, (prob->nlambda + 127) / 128 * 128);
  ctx->max_batch = prob->max_batch > 0 ? prob->max_batch : 4096;
  ctx->scale2 = prob->stokes_scale * prob->stokes_scale;
  std::vector<double> lv(ctx->nl);
  for (int l = 0; l < ctx->nl; ++l) lv[l] = airtovac_d(prob->lambda_air[l]);
  ctx->h_lamair.assign(prob->lambda_air, prob->lambda_air + ctx->nl);
  ctx->h_tau500.assign(prob->tau500, prob->tau500 + ctx->nd);
  for (int j = 0; j < ctx->nlines; ++j) {
    ctx->h_line_lam0.push_back(prob->lines[j].lam0);
    ctx->h_line_mass.push_back(prob->lines[j].mass);
  }
  ctx->lam_mid = (float)(0.5 * (lv[ctx->nl - 1] + lv[0]));
  std::vector<double> D(ctx->nd - 1);
  for (int i = 0; i + 1 < ctx->nd; ++i) D[i] = (prob->tau500[i + 1] - prob->tau500[i]) / prob->mu;
  std::vector<LineConst> lc(ctx->nlines);
  std::vector<float> cS, cD;
  for (int j = 0; j < ctx->nlines; ++j) {
    const snapi_line &s = prob->lines[j];
    LineConst &L = lc[j];
    if (!(s.lam0 > 0.0) || !(s.mass > 0.0)) {
      set_err(ctx, SNAPI_EINVAL, "line %d: lam0 and mass must be positive", j);
      return fail(ctx, SNAPI_EINVAL);
    }
    L.lam0 = s.lam0;
    L.sf = (float)s.sf;
    L.ar = (float)s.ar;
    L.two_k_over_m = (float)(2.0 * kK / s.mass);
    L.lam0_over_c = (float)(s.lam0 / kC);
    L.zee = (float)(4.67E-5 * s.lam0 * s.lam0);
    L.split = s.split ? 1 : 0;
    L.comp_off = (int)cS.size();
    for (int g = 0; g < 3; ++g) {
      L.ncomp[g] = s.split ? s.ncomp[g] : 0;
      if (L.ncomp[g] < 0 || L.ncomp[g] > SNAPI_MAX_COMP) {
        set_err(ctx, SNAPI_EINVAL, "line %d: bad component count", j);
        return fail(ctx, SNAPI_EINVAL);
      }
      for (int i = 0; i < L.ncomp[g]; ++i) { cS.push_back((float)s.S[g][i]); cD.push_back((float)s.D[g][i]); }
    }
  }
  ctx->ncomp = (int)cS.size();
  ctx->nbasis = jvp_basis_size(lc.data(), ctx->nlines);
  const SmemLayout Lsw = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  const SmemLayout Lfin = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, true);
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if ((int)Lfin.total > maxsm) {
    set_err(ctx, SNAPI_EINVAL, "problem needs %zu B of shared memory per CTA (> %d)", Lfin.total, maxsm);
    return fail(ctx, SNAPI_EINVAL);
  }
#define CKC(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      const int code_ = e_ == cudaErrorMemoryAllocation ? SNAPI_ENOMEM : SNAPI_ECUDA;    \
      set_err(ctx, code_, "%s: %s", #call, cudaGetErrorString(e_));                      \
      return fail(ctx, code_);                                                           \
    }                                                                                    \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  CKC(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  for (int h = 0; h < snapi_ctx::kStageChunks; ++h)
    CKC(cudaEventCreateWithFlags(&ctx->ev_copy[h], cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&ctx->ev_free, cudaEventDisableTiming));
  CKC(cudaEventCreate(&ctx->ev0));
  CKC(cudaEventCreate(&ctx->ev1));
  CKC(cudaMalloc(&ctx->d_lamvac, sizeof(double) * ctx->nl));
  CKC(cudaMalloc(&ctx->d_D, sizeof(double) * (ctx->nd - 1)));
  CKC(cudaMalloc(&ctx->d_lines, sizeof(LineConst) * std::max(1, ctx->nlines)));
  CKC(cudaMalloc(&ctx->d_compS, sizeof(float) * std::max(1, ctx->ncomp)));
  CKC(cudaMalloc(&ctx->d_compD, sizeof(float) * std::max(1, ctx->ncomp)));
  CKC(cudaMalloc(&ctx->d_status, sizeof(int)));
  CKC(cudaMemset(ctx->d_status, 0, sizeof(int)));
  CKC(cudaMemcpy(ctx->d_lamvac, lv.data(), sizeof(double) * ctx->nl, cudaMemcpyHostToDevice));
  CKC(cudaMalloc(&ctx->d_lamair, sizeof(double) * ctx->nl));
  CKC(cudaMemcpy(ctx->d_lamair, prob->lambda_air, sizeof(double) * ctx->nl, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(ctx->d_D, D.data(), sizeof(double) * (ctx->nd - 1), cudaMemcpyHostToDevice));
  if (ctx->nlines) CKC(cudaMemcpy(ctx->d_lines, lc.data(), sizeof(LineConst) * ctx->nlines, cudaMemcpyHostToDevice));
  if (ctx->ncomp) {
    CKC(cudaMemcpy(ctx->d_compS, cS.data(), sizeof(float) * ctx->ncomp, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(ctx->d_compD, cD.data(), sizeof(float) * ctx->ncomp, cudaMemcpyHostToDevice));
  }
  const size_t B = ctx->max_batch, nrec = (size_t)ctx->nd * ctx->nfield;
  CKC(cudaMalloc(&ctx->d_rec, sizeof(float) * B * nrec));
  CKC(cudaMalloc(&ctx->d_stokes, sizeof(float) * B * ctx->nl * 4));
  CKC(cudaMalloc(&ctx->d_obs, sizeof(float) * B * ctx->nl * 4));
  CKC(cudaMalloc(&ctx->d_mask, sizeof(float) * B * ctx->nl));
  CKC(cudaMalloc(&ctx->d_recgrad, sizeof(double) * B * nrec));
  CKC(cudaMalloc(&ctx->d_chi2, sizeof(double) * B));
  CKC(cudaMalloc(&ctx->d_scratch, sizeof(float4) * B * ctx->nd * 4 * ctx->lpad_max));
  CKC(cudaMalloc(&ctx->d_seed, sizeof(float4) * B * ctx->lpad_max));
  CKC(cudaMalloc(&ctx->d_bars, sizeof(float4) * B * ctx->nl * 3 * ctx->nd));
  CKC(cudaMalloc(&ctx->d_opart, sizeof(float) * B * (1 + ctx->nlines) * op_slices(ctx->nd) * ctx->nd * kOpSlots));
  // the kernels' dynamic shared-memory limit is a per-device attribute that every context (and the
  // allocation-free adjoint) shares: raise it to the device's opt-in maximum, never to this
  // problem's size, so that a smaller problem's context cannot lower it under a larger one's
  CKC(raise_smem_limits(maxsm));
#undef CKC
  if (ensure_npar(ctx, 1) != SNAPI_OK) return fail(ctx, SNAPI_ENOMEM);
  if (status) *status = SNAPI_OK;
  return ctx;
}

int snapi_synth(snapi_ctx *ctx, int npix, const float *records, float *stokes, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || (npix > 0 && (!records || !stokes)) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_synth: invalid arguments");
  SNAPI_CK(cudaSetDevice(ctx->device));
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    KParams P = base_params(ctx);
    P.npix = nb;
    const float *rec;
    int st = stage_in(ctx, records + p0 * nrec, ctx->d_rec, nb * nrec, mem, &rec);
    if (st) return st;
    P.rec = rec;
    P.stokes = mem == SNAPI_MEM_DEVICE ? stokes + (size_t)p0 * ctx->nl * 4 : ctx->d_stokes;
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    k_synth<<<sweep_ctas(ctx, nb), kChunk, L.total, ctx->stream>>>(P);
    SNAPI_CK(cudaGetLastError());
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 1;
    if (mem == SNAPI_MEM_HOST)
      SNAPI_CK(cudaMemcpyAsync(stokes + (size_t)p0 * ctx->nl * 4, ctx->d_stokes, sizeof(float) * nb * ctx->nl * 4,
                               cudaMemcpyDeviceToHost, ctx->stream));
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return check_status(ctx);
}

}  // extern "C"

namespace {
// the adjoint for dense (ntcol = 0) or packed (ntcol columns per pixel) node tangents
int adjoint_impl(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                 const float *mask, int npar, int ntcol, const float *tangents, float *stokes, double *chi2,
                 double *grad, double *rec_grad, int mem) {
  int st = ensure_npar(ctx, npar > 0 ? npar : 1);
  if (st) return st;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield, nl4 = (size_t)ctx->nl * 4;
  // tangent floats per pixel as stored by the caller
  const size_t ntan = ntcol ? (size_t)ntcol * ctx->nd : (size_t)npar * nrec;
  const SmemLayout Lsw = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  const SmemLayout Lfin = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, true);
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  const bool dev = mem == SNAPI_MEM_DEVICE;
  // Host inputs: each round of up to max_batch pixels goes in chunks whose sizes grow sixfold from
  // ~1/16 of the round, each in its own region of the staging buffers; chunk k+1 is uploaded on the
  // copy stream while chunk k computes.  An upload costs ~0.9 us per pixel (44 KB with packed
  // tangents) against ~5.6 us of compute, so only the first, small chunk's upload is exposed, and the
  // round still runs as a few large launches (rounds of 1024 pixels cost 14 % more device time than
  // one of 4096).  Outputs of a round come back after its last chunk.  (Overlap needs page-locked
  // host inputs, e.g. from snapi_host_alloc; pageable copies serialise with the host thread.)
  int k = 0;
  for (int r0 = 0; r0 < npix; r0 += ctx->max_batch) {
    const int nr = std::min(ctx->max_batch, npix - r0);
    int csz[snapi_ctx::kStageChunks], nch = 0;
    if (dev) {
      csz[nch++] = nr;
    } else {
      int c = std::max(1, (nr + 15) / 16), left = nr;
      while (left > 0) {
        const int take = (nch == snapi_ctx::kStageChunks - 1) ? left : std::min(c, left);
        csz[nch++] = take;
        left -= take;
        c *= 6;
      }
      if (r0 > 0) SNAPI_CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_free, 0));  // previous round done
    }
    int lo = 0;  // offset of the chunk within the round
    for (int ci = 0; ci < nch; ++ci, ++k) {
      const int nb = csz[ci], p0 = r0 + lo;
      KParams P = base_params(ctx);
      P.npix = nb;
      P.npar = npar;
      P.ntcol = ntcol;
      P.tcol_off = ntcol ? ctx->d_tcol : nullptr;
      P.tcol_field = ntcol ? ctx->d_tcol + npar + 1 : nullptr;
      for (int s = 0; s < 4; ++s) P.ws[s] = w_stokes ? w_stokes[s] : 1.0;
      if (dev) {
        P.rec = records + p0 * nrec;
        P.obs = obs + (size_t)p0 * nl4;
        P.mask = mask ? mask + (size_t)p0 * ctx->nl : nullptr;
        P.tangent = npar ? tangents + (size_t)p0 * ntan : nullptr;
      } else {
        const size_t off = (size_t)lo;
        float *drec = ctx->d_rec + off * nrec, *dobs = ctx->d_obs + off * nl4, *dmask = ctx->d_mask + off * ctx->nl;
        float *dtan = ctx->d_tan + off * (ntan ? ntan : nrec);
        cudaStream_t cs = ctx->copy_stream;
        SNAPI_CK(cudaMemcpyAsync(drec, records + p0 * nrec, sizeof(float) * nb * nrec, cudaMemcpyHostToDevice, cs));
        SNAPI_CK(cudaMemcpyAsync(dobs, obs + (size_t)p0 * nl4, sizeof(float) * nb * nl4, cudaMemcpyHostToDevice, cs));
        if (mask)
          SNAPI_CK(cudaMemcpyAsync(dmask, mask + (size_t)p0 * ctx->nl, sizeof(float) * nb * ctx->nl,
                                   cudaMemcpyHostToDevice, cs));
        if (npar)
          SNAPI_CK(cudaMemcpyAsync(dtan, tangents + (size_t)p0 * ntan, sizeof(float) * nb * ntan,
                                   cudaMemcpyHostToDevice, cs));
        SNAPI_CK(cudaEventRecord(ctx->ev_copy[ci], cs));
        SNAPI_CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_copy[ci], 0));
        P.rec = drec; P.obs = dobs; P.mask = mask ? dmask : nullptr; P.tangent = npar ? dtan : nullptr;
      }
      P.stokes = stokes ? (dev ? stokes + (size_t)p0 * nl4 : ctx->d_stokes + (size_t)lo * nl4) : nullptr;
      P.chi2 = dev ? chi2 + p0 : ctx->d_chi2 + lo;
      P.grad = npar ? (dev ? grad + (size_t)p0 * npar : ctx->d_grad + (size_t)lo * npar) : ctx->d_grad;
      P.rec_grad = rec_grad ? (dev ? rec_grad + (size_t)p0 * nrec : ctx->d_recgrad + (size_t)lo * nrec) : nullptr;
      AdjCfg cfg{kChunk, kOpTile, 0};
      if (ctx->tune && !tuned_adj(ctx, nr, &cfg) && dev && ci == 0) {
        cfg = tune_adjoint(ctx, P, nb, Lsw.total, Lfin.total);
        tune_store_adj(ctx, nr, cfg);
      }
      if (k == 0) SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
      launch_adjoint(P, nb, cfg, Lsw.total, Lfin.total, ctx->stream);
      SNAPI_CK(cudaGetLastError());
      ctx->last_launches += kAdjointLaunches;
      lo += nb;
    }
    if (!dev) {
      SNAPI_CK(cudaEventRecord(ctx->ev_free, ctx->stream));
      if (stokes)
        SNAPI_CK(cudaMemcpyAsync(stokes + (size_t)r0 * nl4, ctx->d_stokes, sizeof(float) * nr * nl4,
                                 cudaMemcpyDeviceToHost, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(chi2 + r0, ctx->d_chi2, sizeof(double) * nr, cudaMemcpyDeviceToHost, ctx->stream));
      if (npar)
        SNAPI_CK(cudaMemcpyAsync(grad + (size_t)r0 * npar, ctx->d_grad, sizeof(double) * nr * npar,
                                 cudaMemcpyDeviceToHost, ctx->stream));
      if (rec_grad)
        SNAPI_CK(cudaMemcpyAsync(rec_grad + (size_t)r0 * nrec, ctx->d_recgrad, sizeof(double) * nr * nrec,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    }
  }
  if (npix > 0) {
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms = ms;  // first kernel start to the end of the last chunk (host copies included)
  }
  return check_status(ctx);
}
}  // namespace

extern "C" {

int snapi_adjoint(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                  const float *mask, int npar, const float *tangents, float *stokes, double *chi2, double *grad,
                  double *rec_grad, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || npar < 0 || (npix > 0 && (!records || !obs || !chi2)) || (npar > 0 && (!tangents || !grad)) ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint: invalid arguments");
  SNAPI_CK(cudaSetDevice(ctx->device));
  return adjoint_impl(ctx, npix, records, obs, w_stokes, mask, npar, 0, tangents, stokes, chi2, grad, rec_grad, mem);
}

int snapi_adjoint_packed(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                         const float *mask, int npar, const unsigned long long *field_mask,
                         const float *packed_tangents, float *stokes, double *chi2, double *grad, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || npar < 1 || !field_mask || (npix > 0 && (!records || !obs || !chi2 || !grad || !packed_tangents)) ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE) || ctx->nfield > 64)
    return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint_packed: invalid arguments");
  std::vector<int> tab(npar + 1, 0);
  for (int p = 0; p < npar; ++p) {
    if (ctx->nfield < 64 && (field_mask[p] >> ctx->nfield) != 0ull)
      return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint_packed: field_mask[%d] names fields beyond nfield", p);
    tab[p + 1] = tab[p] + __builtin_popcountll(field_mask[p]);
  }
  const int ntcol = tab[npar];
  if (ntcol < 1) return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint_packed: empty field masks");
  for (int p = 0; p < npar; ++p)
    for (int f = 0; f < ctx->nfield; ++f)
      if ((field_mask[p] >> f) & 1ull) tab.push_back(f);
  SNAPI_CK(cudaSetDevice(ctx->device));
  if ((int)tab.size() > ctx->cap_tcol) {
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->d_tcol);
    ctx->d_tcol = nullptr;
    ctx->cap_tcol = 0;
    SNAPI_CK(cudaMalloc(&ctx->d_tcol, sizeof(int) * tab.size()));
    ctx->cap_tcol = (int)tab.size();
  }
  // stream-ordered after every earlier kernel of this context, before this call's kernels; the
  // source is pageable, so the copy has completed when the call returns
  SNAPI_CK(cudaMemcpyAsync(ctx->d_tcol, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, ctx->stream));
  return adjoint_impl(ctx, npix, records, obs, w_stokes, mask, npar, ntcol, packed_tangents, stokes, chi2, grad,
                      nullptr, mem);
}

int snapi_fd_grad(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                  const float *mask, int npar, const float *tangents, const double *step, double *chi2, double *grad,
                  int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || npar < 1 || (npix > 0 && (!records || !obs || !chi2 || !grad || !tangents)) || !step ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_fd_grad: invalid arguments");
  SNAPI_CK(cudaSetDevice(ctx->device));
  int st = ensure_npar(ctx, npar);
  if (st) return st;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  SNAPI_CK(cudaMemcpyAsync(ctx->d_step, step, sizeof(double) * npar, cudaMemcpyHostToDevice, ctx->stream));
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    KParams P = base_params(ctx);
    P.npix = nb;
    P.npar = npar;
    P.nvar = 2 * npar + 1;
    for (int s = 0; s < 4; ++s) P.ws[s] = w_stokes ? w_stokes[s] : 1.0;
    const float *rec, *ob, *mk, *tn;
    if ((st = stage_in(ctx, records + p0 * nrec, ctx->d_rec, nb * nrec, mem, &rec))) return st;
    if ((st = stage_in(ctx, obs + (size_t)p0 * ctx->nl * 4, ctx->d_obs, (size_t)nb * ctx->nl * 4, mem, &ob))) return st;
    if ((st = stage_in(ctx, mask ? mask + (size_t)p0 * ctx->nl : nullptr, ctx->d_mask, (size_t)nb * ctx->nl, mem, &mk)))
      return st;
    if ((st = stage_in(ctx, tangents + (size_t)p0 * npar * nrec, ctx->d_tan, (size_t)nb * npar * nrec, mem, &tn)))
      return st;
    P.rec = rec; P.obs = ob; P.mask = mk; P.tangent = tn; P.fd_step = ctx->d_step;
    const bool dev = mem == SNAPI_MEM_DEVICE;
    P.chi2 = dev ? chi2 + p0 : ctx->d_chi2;
    P.grad = dev ? grad + (size_t)p0 * npar : ctx->d_grad;
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    k_fd_sweep<<<sweep_ctas(ctx, nb, P.nvar), kChunk, L.total, ctx->stream>>>(P);
    SNAPI_CK(cudaGetLastError());
    k_fd_finish<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(P);
    SNAPI_CK(cudaGetLastError());
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 2;
    if (!dev) {
      SNAPI_CK(cudaMemcpyAsync(chi2 + p0, ctx->d_chi2, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(grad + (size_t)p0 * npar, ctx->d_grad, sizeof(double) * nb * npar,
                               cudaMemcpyDeviceToHost, ctx->stream));
    }
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return check_status(ctx);
}

int snapi_responses(snapi_ctx *ctx, int npix, const float *records, int npar, const float *tangents,
                    const double *step, float *stokes, float *dstokes, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || npar < 1 || (npix > 0 && (!records || !tangents || !dstokes)) || !step ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_responses: invalid arguments");
  for (int p = 0; p < npar; ++p)
    if (!(step[p] > 0.0)) return set_err(ctx, SNAPI_EINVAL, "snapi_responses: steps must be positive");
  SNAPI_CK(cudaSetDevice(ctx->device));
  int st = ensure_npar(ctx, npar);
  if (st) return st;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  SNAPI_CK(cudaMemcpyAsync(ctx->d_step, step, sizeof(double) * npar, cudaMemcpyHostToDevice, ctx->stream));
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    KParams P = base_params(ctx);
    P.npix = nb;
    P.npar = npar;
    P.nvar = npar;
    const float *rec, *tn;
    if ((st = stage_in(ctx, records + p0 * nrec, ctx->d_rec, nb * nrec, mem, &rec))) return st;
    if ((st = stage_in(ctx, tangents + (size_t)p0 * npar * nrec, ctx->d_tan, (size_t)nb * npar * nrec, mem, &tn)))
      return st;
    P.rec = rec; P.tangent = tn; P.fd_step = ctx->d_step;
    const bool dev = mem == SNAPI_MEM_DEVICE;
    P.dstokes = dev ? dstokes + (size_t)p0 * npar * ctx->nl * 4 : ctx->d_dstokes;
    P.stokes = stokes ? (dev ? stokes + (size_t)p0 * ctx->nl * 4 : ctx->d_stokes) : nullptr;
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (ctx->jac_tangent) {  // forward-mode sweeps: the state pass also gives the Stokes vector
      P.scratch = ctx->d_scratch;
      P.nvar = 1;  // k_resp_state: CTA = (pixel, chunk); k_resp_jvp indexes its own CTAs
      k_resp_state<<<sweep_ctas(ctx, nb), kChunk, L.total, ctx->stream>>>(P);
      SNAPI_CK(cudaGetLastError());
      const int nwarp = std::min(npar, kJvpDirs), ngrp = (npar + kJvpDirs - 1) / kJvpDirs;
      launch_jvp(nb * ((ctx->nl + 31) / 32) * ngrp, nwarp, L.total + jvp_smem_extra(ctx->nbasis, nwarp, ctx->nlines),
                 ctx->stream, P);
      SNAPI_CK(cudaGetLastError());
      ctx->last_launches += 2;
    } else {
      if (P.stokes) {
        KParams Q = P;
        Q.nvar = 1;
        k_synth<<<sweep_ctas(ctx, nb), kChunk, L.total, ctx->stream>>>(Q);
        SNAPI_CK(cudaGetLastError());
        ctx->last_launches += 1;
      }
      k_resp_sweep<<<sweep_ctas(ctx, nb, npar), kChunk, L.total, ctx->stream>>>(P);
      SNAPI_CK(cudaGetLastError());
      ctx->last_launches += 1;
    }
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if (!dev) {
      if (stokes)
        SNAPI_CK(cudaMemcpyAsync(stokes + (size_t)p0 * ctx->nl * 4, ctx->d_stokes, sizeof(float) * nb * ctx->nl * 4,
                                 cudaMemcpyDeviceToHost, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(dstokes + (size_t)p0 * npar * ctx->nl * 4, ctx->d_dstokes,
                               sizeof(float) * nb * npar * ctx->nl * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return check_status(ctx);
}

}  // extern "C"

// =============================================================================================
// Adjoint without any device allocation.
//
// For callers that cannot call cudaMalloc: applications whose device memory belongs to another
// allocator (a framework memory pool with a fixed budget, where a side allocation would break
// its accounting) and loops that must not take the device-wide synchronisation and unbounded
// latency of cudaMalloc / cudaFree.  The computation is snapi_adjoint's (same kernels); every
// work buffer lives in the static device array below instead of in a context.
//
// g_snapi_static is SNAPI_STATIC_SCRATCH_BYTES (64 MiB) on every GPU that loads this library,
// held until the process exits.  Layout: [status word][problem constants][work region]; the work
// region holds, per pixel of a chunk, the forward state (nd x 4 x lpad float4), the adjoint
// seed (lpad float4), the adjoint bars (nl x 3 x nd float4), the opacity-adjoint sums
// ((1 + nlines) x nd x kOpSlots float) and the per-warp chi2 sums (nwarp double).  Pixels
// are processed in chunks that fit the work region.
// g_snapi_static is a __device__ array: in host code its name denotes only a host-side stand-in,
// not device memory, so its device address is fetched with cudaGetSymbolAddress -- once per
// device, by the first call on that device, with that device current.
// Every call shares the array: the kernels overwrite every slot they read in the same call and
// the status word is cleared at the start of each call; calls that overlap on the GPU (two host
// threads, or two streams) race on it.
namespace {

constexpr size_t kStaticBytes = SNAPI_STATIC_SCRATCH_BYTES;
constexpr size_t kStaticConstBytes = 128 * 1024;  // status word + problem constants
constexpr int kMaxDevices = 64;
static __device__ __align__(256) unsigned char g_snapi_static[kStaticBytes];

std::mutex g_static_mu;
unsigned char *g_static_ptr[kMaxDevices] = {};

int static_setup(int device, unsigned char **base, std::string &err) {
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (device < 0 || device >= kMaxDevices) { err = "device ordinal out of range"; return SNAPI_EINVAL; }
  if (!g_static_ptr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_snapi_static);
    if (e != cudaSuccess || !p) {
      err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
      return SNAPI_ECUDA;
    }
    g_static_ptr[device] = static_cast<unsigned char *>(p);
  }
  // The kernels' shared-memory limit is shared with every context on the device and set on every
  // call (a context created since the last call must not leave it below what this call needs).
  int maxsm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (e == cudaSuccess) e = raise_smem_limits(maxsm);
  if (e != cudaSuccess) { err = std::string("shared-memory limit: ") + cudaGetErrorString(e); return SNAPI_ECUDA; }
  *base = g_static_ptr[device];
  return SNAPI_OK;
}

int noalloc_run(const snapi_problem *prob, void *stream_v, int npix, const float *records, const float *obs,
                const double *w_stokes, const float *mask, int npar, const float *tangents, float *stokes,
                double *chi2, double *grad, unsigned char *base, std::string &err) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
  const int nd = prob->nd, nl = prob->nlambda, nlines = prob->nlines;
  const int nfield = SNAPI_NFIELD0 + 3 * nlines, nred = kNumRed + kRedPerLine * nlines;
  const int nchunk = (nl + kChunk - 1) / kChunk, lpad = nchunk * kChunk, nwslot = lpad / 32;
  // problem constants (host side), as snapi_create prepares them
  std::vector<double> lv(nl), D(nd - 1);
  for (int l = 0; l < nl; ++l) lv[l] = airtovac_d(prob->lambda_air[l]);
  for (int i = 0; i + 1 < nd; ++i) D[i] = (prob->tau500[i + 1] - prob->tau500[i]) / prob->mu;
  std::vector<LineConst> lc(nlines);
  std::vector<float> cS, cD;
  for (int j = 0; j < nlines; ++j) {
    const snapi_line &s = prob->lines[j];
    if (!(s.lam0 > 0.0) || !(s.mass > 0.0)) { err = "line lam0 and mass must be positive"; return SNAPI_EINVAL; }
    LineConst &L = lc[j];
    L.lam0 = s.lam0; L.sf = (float)s.sf; L.ar = (float)s.ar;
    L.two_k_over_m = (float)(2.0 * kK / s.mass);
    L.lam0_over_c = (float)(s.lam0 / kC);
    L.zee = (float)(4.67E-5 * s.lam0 * s.lam0);
    L.split = s.split ? 1 : 0;
    L.comp_off = (int)cS.size();
    for (int g = 0; g < 3; ++g) {
      L.ncomp[g] = s.split ? s.ncomp[g] : 0;
      if (L.ncomp[g] < 0 || L.ncomp[g] > SNAPI_MAX_COMP) { err = "bad Zeeman component count"; return SNAPI_EINVAL; }
      for (int i = 0; i < L.ncomp[g]; ++i) { cS.push_back((float)s.S[g][i]); cD.push_back((float)s.D[g][i]); }
    }
  }
  const int ncomp = (int)cS.size();
  // constants region: status | lamvac | D | lines | compS | compD
  size_t o = 256;
  const size_t o_lv = o; o = align_up(o + sizeof(double) * nl, 256);
  const size_t o_D = o; o = align_up(o + sizeof(double) * (nd - 1), 256);
  const size_t o_lc = o; o = align_up(o + sizeof(LineConst) * (nlines > 0 ? nlines : 1), 256);
  const size_t o_cS = o; o = align_up(o + sizeof(float) * (ncomp > 0 ? ncomp : 1), 256);
  const size_t o_cD = o; o = align_up(o + sizeof(float) * (ncomp > 0 ? ncomp : 1), 256);
  if (o > kStaticConstBytes) { err = "problem constants exceed the static constants region"; return SNAPI_EINVAL; }
  // work region per pixel
  const size_t per_state = sizeof(float4) * (size_t)nd * 4 * lpad;
  const size_t per_seed = sizeof(float4) * (size_t)lpad;
  const size_t per_bars = sizeof(float4) * (size_t)nl * 3 * nd;
  const size_t per_part = sizeof(float) * (size_t)(1 + nlines) * op_slices(nd) * nd * kOpSlots;
  const size_t per_c2 = sizeof(double) * (size_t)nwslot;
  const size_t a_state = align_up(per_state, 256), a_seed = align_up(per_seed, 256), a_bars = align_up(per_bars, 256),
               a_part = align_up(per_part, 256), a_c2 = align_up(per_c2, 256);
  const size_t per_pix = a_state + a_seed + a_bars + a_part + a_c2;
  const size_t work = kStaticBytes - kStaticConstBytes;
  const int cap = (int)std::min<size_t>(work / per_pix, 1 << 20);
  if (cap < 1) {
    char b[256];
    snprintf(b, sizeof b, "one pixel needs %zu B of work memory, the static array holds %zu B", per_pix, work);
    err = b;
    return SNAPI_EINVAL;
  }
  const SmemLayout Lsw = smem_layout(nd, nfield, nlines, ncomp, nred, false);
  const SmemLayout Lfin = smem_layout(nd, nfield, nlines, ncomp, nred, true);
  if (Lfin.total > 227 * 1024) { err = "problem exceeds the shared memory of a CTA"; return SNAPI_EINVAL; }
  int *status = reinterpret_cast<int *>(base);
#define CKN(call)                                                   \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) {                                        \
      err = std::string(#call ": ") + cudaGetErrorString(e_);       \
      return SNAPI_ECUDA;                                           \
    }                                                               \
  } while (0)
  CKN(cudaMemsetAsync(status, 0, sizeof(int), stream));
  CKN(cudaMemcpyAsync(base + o_lv, lv.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, stream));
  CKN(cudaMemcpyAsync(base + o_D, D.data(), sizeof(double) * (nd - 1), cudaMemcpyHostToDevice, stream));
  if (nlines) CKN(cudaMemcpyAsync(base + o_lc, lc.data(), sizeof(LineConst) * nlines, cudaMemcpyHostToDevice, stream));
  if (ncomp) {
    CKN(cudaMemcpyAsync(base + o_cS, cS.data(), sizeof(float) * ncomp, cudaMemcpyHostToDevice, stream));
    CKN(cudaMemcpyAsync(base + o_cD, cD.data(), sizeof(float) * ncomp, cudaMemcpyHostToDevice, stream));
  }
  unsigned char *wbase = base + kStaticConstBytes;
  const size_t nrec = (size_t)nd * nfield;
  for (int p0 = 0; p0 < npix; p0 += cap) {
    const int nb = std::min(cap, npix - p0);
    KParams P;
    memset(&P, 0, sizeof P);
    P.npix = nb; P.nd = nd; P.nl = nl; P.nlines = nlines; P.nfield = nfield; P.npar = npar; P.lpad = lpad;
    P.ncomp = ncomp; P.nred = nred; P.nchunk = nchunk; P.nwslot = nwslot; P.nvar = 1; P.optile = kOpTile;
    P.nslice = op_slices(nd);
    P.lam_mid = (float)(0.5 * (lv[nl - 1] + lv[0]));
    P.scale2 = prob->stokes_scale * prob->stokes_scale;
    P.lamvac = reinterpret_cast<const double *>(base + o_lv);
    P.D = reinterpret_cast<const double *>(base + o_D);
    P.lines = reinterpret_cast<const LineConst *>(base + o_lc);
    P.compS = reinterpret_cast<const float *>(base + o_cS);
    P.compD = reinterpret_cast<const float *>(base + o_cD);
    P.status = status;
    P.scratch = reinterpret_cast<float4 *>(wbase);
    P.seed = reinterpret_cast<float4 *>(wbase + a_state * cap);
    P.bars = reinterpret_cast<float4 *>(wbase + (a_state + a_seed) * cap);
    P.opart = reinterpret_cast<float *>(wbase + (a_state + a_seed + a_bars) * cap);
    P.c2part = reinterpret_cast<double *>(wbase + (a_state + a_seed + a_bars + a_part) * cap);
    for (int s = 0; s < 4; ++s) P.ws[s] = w_stokes ? w_stokes[s] : 1.0;
    P.rec = records + p0 * nrec;
    P.obs = obs + (size_t)p0 * nl * 4;
    P.mask = mask ? mask + (size_t)p0 * nl : nullptr;
    P.tangent = npar ? tangents + (size_t)p0 * npar * nrec : nullptr;
    P.stokes = stokes ? stokes + (size_t)p0 * nl * 4 : nullptr;
    P.chi2 = chi2 + p0;
    P.grad = npar ? grad + (size_t)p0 * npar : nullptr;
    launch_adjoint(P, nb, AdjCfg{kChunk, kOpTile, 0}, Lsw.total, Lfin.total, stream);
    CKN(cudaGetLastError());
  }
  int st = 0;
  CKN(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CKN(cudaStreamSynchronize(stream));
#undef CKN
  if (st != 0) { err = "a CTA gave up waiting for its TMA copy"; return st; }
  return SNAPI_OK;
}

thread_local std::string g_noalloc_err;

}  // namespace

extern "C" {

int snapi_adjoint_noalloc(const snapi_problem *prob, int device, void *stream, int npix, const float *records,
                          const float *obs, const double *w_stokes, const float *mask, int npar,
                          const float *tangents, float *stokes, double *chi2, double *grad) {
  g_noalloc_err.clear();
  if (!prob || npix < 0 || npar < 0 || (npix > 0 && (!records || !obs || !chi2)) ||
      (npar > 0 && (!tangents || !grad)) || prob->nd < 3 || prob->nlambda < 1 ||
      prob->nlambda > SNAPI_MAX_LAMBDA || prob->nlines < 0 || prob->nlines > SNAPI_MAX_LINES || !prob->lambda_air ||
      !prob->tau500 || (prob->nlines && !prob->lines) || !(prob->mu > 0.0 && prob->mu <= 1.0) ||
      !(prob->stokes_scale > 0.0)) {
    g_noalloc_err = "snapi_adjoint_noalloc: invalid arguments";
    return SNAPI_EINVAL;
  }
  for (int i = 0; i + 1 < prob->nd; ++i)
    if (!(prob->tau500[i + 1] > prob->tau500[i])) {
      g_noalloc_err = "tau500 must increase from the top down";
      return SNAPI_EINVAL;
    }
  int old = 0;
  if (cudaGetDevice(&old) != cudaSuccess) { g_noalloc_err = "cudaGetDevice failed"; return SNAPI_ECUDA; }
  if (cudaSetDevice(device) != cudaSuccess) { g_noalloc_err = "cudaSetDevice failed"; return SNAPI_ECUDA; }
  if (stream) {  // the stream must belong to `device` (the NULL stream is the current device's)
    int sdev = -1;
    if (cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &sdev) != cudaSuccess || sdev != device) {
      cudaGetLastError();
      cudaSetDevice(old);
      g_noalloc_err = "snapi_adjoint_noalloc: the stream was not created on `device`";
      return SNAPI_EINVAL;
    }
  }
  unsigned char *base = nullptr;
  int rc = static_setup(device, &base, g_noalloc_err);
  if (rc == SNAPI_OK && npix > 0)
    rc = noalloc_run(prob, stream, npix, records, obs, w_stokes, mask, npar, tangents, stokes, chi2, grad, base,
                     g_noalloc_err);
  cudaSetDevice(old);
  return rc;
}

const char *snapi_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

}  // extern "C"
