// snapi_sweep.cuh -- per-(pixel, wavelength) depth sweeps of the B200 path.
//
// forward_sweep: opacity at every depth, Bezier optical depth and the linear-DELO recursion
//   from the bottom (depth nd-1) to the top, as atmos_ppbez::formal (polarized) does it
//   (atmos/plpar/atmos_ppbez_rts.cc:918-1218).  A sliding window of three depths keeps the
//   monotone eta_I derivative and the optical depth in registers.  Optionally stores the
//   per-depth forward state (I, K', S, eta_I, dtau) for the reverse sweep.
// reverse_sweep: the adjoint of forward_sweep for a given adjoint of the emergent Stokes
//   vector, top to bottom.  Depth z-1 is final after step z; its opacity adjoint is evaluated
//   then and the wavelength-level sums are handed to the reducer.
//
// Both are templates over the scratch store (device float4 planes or host vectors) and the
// reducer (warp shuffles + shared-memory atomics on the device, plain sums on the host).
#pragma once
#include "snapi_core.cuh"

namespace snapi {

struct PixelView {
  int nd, nlines, nfield;
  const float *rec;        // [nd][nfield]
  const DepthConst *dc;    // [nd]
  const LineDepth *ld;     // [nd][nlines]
  const LineConst *lc;     // [nlines]
  const float *compS, *compD;
  const double *D;         // [nd-1] path-length intervals
};

SNAPI_HD void depth_opacity(const PixelView &pv, int z, const LamConst &lam, const float *delta, float *kp,
                            float *S, float &e) {
  float eta[7], jj[4];
  cell_opacity(pv.dc[z], pv.ld + z * pv.nlines, pv.lc, pv.nlines, pv.compS, pv.compD, lam, delta, eta, jj);
  const float ie = frcp(eta[0]);
  e = eta[0];
#pragma unroll
  for (int q = 0; q < 6; ++q) kp[q] = eta[q + 1] * ie;
#pragma unroll
  for (int s = 0; s < 4; ++s) S[s] = jj[s] * ie;
}

// Returns the emergent Stokes vector in out[4].  sc.store(z, I, kp, S, e, tau) when STORE.
template <bool STORE, class SC>
SNAPI_HD void forward_sweep(const PixelView &pv, const LamConst &lam, const float *delta, float *out, SC &sc) {
  const int nd = pv.nd;
  float kpA[6], SA[4], eA, kpB[6], SB[4], eB, kpC[6], SC_[4], eC;
  depth_opacity(pv, nd - 1, lam, delta, kpA, SA, eA);
  depth_opacity(pv, nd - 2, lam, delta, kpB, SB, eB);
  float I[4] = {SA[0], 0.f, 0.f, 0.f};
  if (STORE) sc.store(nd - 1, I, kpA, SA, eA, 0.0f);
  double opd_below = ((double)eB - (double)eA) / pv.D[nd - 2];
  for (int z = nd - 2; z >= 1; --z) {
    depth_opacity(pv, z - 1, lam, delta, kpC, SC_, eC);
    const double opd_z = opd_interior(eA, eB, eC, pv.D[z], pv.D[z - 1]);
    const float tau = (float)bezier_dtau(eA, eB, opd_below, opd_z, pv.D[z]);
    float In[4];
    delo_step(I, kpA, SA, kpB, SB, tau, In);
#pragma unroll
    for (int s = 0; s < 4; ++s) I[s] = In[s];
    if (STORE) sc.store(z, I, kpB, SB, eB, tau);
#pragma unroll
    for (int q = 0; q < 6; ++q) { kpA[q] = kpB[q]; kpB[q] = kpC[q]; }
#pragma unroll
    for (int s = 0; s < 4; ++s) { SA[s] = SB[s]; SB[s] = SC_[s]; }
    eA = eB; eB = eC;
    opd_below = opd_z;
  }
  if (STORE) sc.store(0, I, kpB, SB, eB, 0.0f);
#pragma unroll
  for (int s = 0; s < 4; ++s) out[s] = I[s];  // the top point copies the one below
}

// Turn (K'-bar, S-bar, eta_I-bar) of one depth into (eta-bar, j-bar), the inputs of the
// opacity adjoint: K'_q = eta_q / eta_I, S_s = j_s / eta_I.
SNAPI_HD void depth_bars(const float *kp, const float *S, float e, const float *kpb, const float *Sb, float eb,
                         float *etab, float *jb) {
  const float ie = 1.0f / e;
  float acc = 0.f;
#pragma unroll
  for (int q = 0; q < 6; ++q) { etab[q + 1] = kpb[q] * ie; acc += kpb[q] * kp[q]; }
#pragma unroll
  for (int s = 0; s < 4; ++s) { jb[s] = Sb[s] * ie; acc += Sb[s] * S[s]; }
  etab[0] = eb - acc * ie;
}

// Reverse sweep, phase R1: adjoint of the DELO recursion and of the Bezier optical depth, top to
// bottom.  Depth z-1 is final after step z; its (eta-bar, j-bar) overwrite its scratch slots
// (sc.store_bar) -- the forward values of that depth are no longer needed.  Phase R2 (opacity
// adjoint per depth) then runs with no sweep state live.
template <class SC>
SNAPI_HD void reverse_sweep_rt(const PixelView &pv, const float *Ib_in, SC &sc) {
  const int nd = pv.nd;
  // forward values of depths z-1 (m), z (c), z+1 (n)
  float kpm[6], Sm[4], em_;
  float Ic[4], kpc[6], Sc[4], ec, tauc;
  float In[4], kpn[6], Sn[4], en, taun;
  // adjoints
  float Ib[4], kpbm[6], Sbm[4], ebm, kpbc[6], Sbc[4], ebc, kpbn[6], Sbn[4], ebn;
  double opdb_c, opdb_n;
  {
    float Id[4], td;
    sc.load(0, Id, kpm, Sm, em_, td);
  }
  sc.load(1, Ic, kpc, Sc, ec, tauc);
  sc.prefetch(2);
#pragma unroll
  for (int s = 0; s < 4; ++s) { Ib[s] = Ib_in[s]; Sbm[s] = 0.f; Sbc[s] = 0.f; }
#pragma unroll
  for (int q = 0; q < 6; ++q) { kpbm[q] = 0.f; kpbc[q] = 0.f; }
  ebm = 0.f; ebc = 0.f; opdb_c = 0.0;
  for (int z = 1; z <= nd - 2; ++z) {
    sc.load(z + 1, In, kpn, Sn, en, taun);
    sc.prefetch(z + 2);
#pragma unroll
    for (int s = 0; s < 4; ++s) Sbn[s] = 0.f;
#pragma unroll
    for (int q = 0; q < 6; ++q) kpbn[q] = 0.f;
    float Ipb[4] = {0.f, 0.f, 0.f, 0.f};
    const float taub = delo_step_adjoint(In, kpn, Sn, kpc, Sc, tauc, Ic, Ib, Ipb, kpbn, Sbn, kpbc, Sbc);
    // tau_z = bezier(e_{z+1}, e_z, opd_{z+1}, opd_z, D[z])
    const double Dz = pv.D[z];
    ebn = (float)(taub * Dz * 0.5);
    ebc += (float)(taub * Dz * 0.5);
    opdb_n = taub * Dz * Dz / 12.0;
    opdb_c -= taub * Dz * Dz / 12.0;
    {  // opd_z final: interior point z with e_up = e_{z+1}, e_c = e_z, e_dn = e_{z-1}
      double gup = 0, gc = 0, gdn = 0;
      opd_interior_grad(en, ec, em_, Dz, pv.D[z - 1], opdb_c, gup, gc, gdn);
      ebn += (float)gup; ebc += (float)gc; ebm += (float)gdn;
    }
    {  // depth z-1 is final
      float etab[7], jb[4];
      depth_bars(kpm, Sm, em_, kpbm, Sbm, ebm, etab, jb);
      sc.store_bar(z - 1, etab, jb);
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      Ib[s] = Ipb[s];
      Ic[s] = In[s];
      Sm[s] = Sc[s]; Sc[s] = Sn[s];
      Sbm[s] = Sbc[s]; Sbc[s] = Sbn[s];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      kpm[q] = kpc[q]; kpc[q] = kpn[q];
      kpbm[q] = kpbc[q]; kpbc[q] = kpbn[q];
    }
    em_ = ec; ec = en;
    ebm = ebc; ebc = ebn;
    tauc = taun;
    opdb_c = opdb_n;
  }
  // m = nd-2, c = nd-1; the opd at nd-1 is one-sided: (e_{nd-2} - e_{nd-1}) / D[nd-2]
  {
    const double Dl = pv.D[nd - 2];
    ebm += (float)(opdb_c / Dl);
    ebc -= (float)(opdb_c / Dl);
  }
  Sbc[0] += Ib[0];  // boundary condition I_{nd-1} = (S_I, 0, 0, 0)
  float etab[7], jb[4];
  depth_bars(kpm, Sm, em_, kpbm, Sbm, ebm, etab, jb);
  sc.store_bar(nd - 2, etab, jb);
  depth_bars(kpc, Sc, ec, kpbc, Sbc, ebc, etab, jb);
  sc.store_bar(nd - 1, etab, jb);
}

// Reverse sweep, phase R2: opacity adjoint of every depth; wavelength sums go to the reducer.
template <class SC, class RD>
SNAPI_HD void reverse_sweep_opacity(const PixelView &pv, const LamConst &lam, const float *delta, const SC &sc,
                                    RD &rd, float *red, int nred) {
  for (int z = 0; z < pv.nd; ++z) {
    float etab[7], jb[4];
    sc.load_bar(z, etab, jb);
    for (int i = 0; i < nred; ++i) red[i] = 0.0f;
    cell_opacity_adjoint(pv.dc[z], pv.ld + z * pv.nlines, pv.lc, pv.nlines, pv.compS, pv.compD, lam, delta, etab,
                         jb, red);
    rd.add(z, red, nred);
  }
}

// Ib: adjoint of the emergent Stokes vector.  red: work vector of nred floats.
template <class SC, class RD>
SNAPI_HD void reverse_sweep(const PixelView &pv, const LamConst &lam, const float *delta, const float *Ib_in,
                            SC &sc, RD &rd, float *red, int nred) {
  reverse_sweep_rt(pv, Ib_in, sc);
  reverse_sweep_opacity(pv, lam, delta, sc, rd, red, nred);
}

}  // namespace snapi
