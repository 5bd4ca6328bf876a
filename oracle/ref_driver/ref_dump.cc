// Oracle driver over the compiled reference (strict FP64 build).  Test infrastructure only.
//
//   snapi_ref_dump pack   <job.cfg> <out.tsk>
//       Parse a reference job config (run in a directory holding the reference's atom/molecule
//       configs and atmosphere file) and write a task blob: the packed 1-column atmosphere,
//       the packed node model and the observation's wavelength grid.
//   snapi_ref_dump dump   <task.tsk> <nodes.f64> <npix> <flags> <out.sbin>
//       For each pixel's node vector: build_from_nodes, then dump the column record the GPU
//       path consumes, the reference Stokes (obs_stokes) and, by flag, the reference node
//       responses (obs_stokes_responses_to_nodes), the record tangents d(record)/d(node)
//       (central differences of build_from_nodes / interpolate_from_nodes with the
//       reference's own steps) and the reference's normalised opacity at a few wavelengths.
//   snapi_ref_dump lmfit  <task.tsk> <nodes0.f64> <target.f64> <mask.f64> <npix> <iters> <out.sbin> [width]
//       Run stokes_lm_fit per pixel from the initial nodes against target Stokes (optionally with
//       Gaussian spectral broadening of width [cm]).
//   snapi_ref_dump conv   <in.f64> <nlambda> <nvec> <width_cm> <out.f64>
//       Gaussian instrumental broadening of nvec Stokes spectra (convolve_spectra_with_gauss).
//   snapi_ref_dump eos    <task.tsk> <nodes.f64> <npix> <out.sbin>
//       The tables of the node -> record build (atoms, partition functions, levels, molecules,
//       line ties, node model), the reference's chemistry on a (T, Nt) grid and the columns
//       build_from_nodes leaves for npix node vectors (see do_eos).
//   snapi_ref_dump ali    <task.tsk> <nodes.f64> <ncol> <niter> <out.sbin>
//       NLTE level-population iteration inputs, niter iterations of the reference's loop, and the
//       populations nltepops converges to (see do_ali).
//   snapi_ref_dump alisetup <task.tsk> <nodes.f64> <ncol> <out.sbin>
//       The tables of nltepops' population-independent set-up (background opacity, collisional
//       rates, line damping) and the columns of ncol node vectors (see do_alisetup).
//
// flags: 1 = responses, 2 = tangents, 4 = opacity probe (pixel 0 only)
//
// Output ".sbin": a sequence of arrays [int32 name_len][name][int32 ndim][int64 dims...]
// [float64 data], read by tests/golden/sbin.py.
#include "ref_common.h"

struct SbinWriter {
  FILE *f;
  explicit SbinWriter(const char *fn) { f = fopen(fn, "wb"); if (!f) { perror(fn); exit(2); } }
  ~SbinWriter() { fclose(f); }
  void put(const std::string &name, const std::vector<int64_t> &dims, const double *d) {
    int32_t nl = name.size(); fwrite(&nl, 4, 1, f); fwrite(name.data(), 1, nl, f);
    int32_t nd = dims.size(); fwrite(&nd, 4, 1, f);
    int64_t n = 1;
    for (auto x : dims) { fwrite(&x, 8, 1, f); n *= x; }
    fwrite(d, 8, n, f);
  }
};

// ----------------------------------------------------------------------------------------------
// pack: jsub-side job set-up
static int do_pack(const char *cfgname, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-cfg", cfgname, "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 6; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  struct gcfg cfg(cmd, io);
  char wd[4096];
  if (!getcwd(wd, sizeof wd)) return 2;
  // reference flow: construct from cfg, pack, unpack, init, extract one column
  atmosphere *a0 = atmos_new(cfg.atm[0], io);
  int32_t sz = a0->size(io);
  uint8_t *buf = new uint8_t[sz];
  a0->pack(buf, 0, io);
  int32_t offs = 0;
  atmosphere *a1 = atmos_new(buf, offs, 0, io);
  a1->init(wd, &io);
  atmosphere *col = a1->extract(1, 1, io);
  std::vector<uint8_t> abuf(col->size(io));
  col->pack(abuf.data(), 0, io);
  model *m = model_new(cfg.mod[0], io);
  std::vector<uint8_t> mbuf(m->size(io));
  m->pack(mbuf.data(), 0, io);

  FILE *f = fopen(outname, "wb");
  fwrite("SNAPITSK", 1, 8, f);
  int32_t nl = cfg.obs[0]->nlambda;
  double el = cfg.obs[0]->el, az = cfg.obs[0]->az;
  fwrite(&nl, 4, 1, f); fwrite(&el, 8, 1, f); fwrite(&az, 8, 1, f);
  fwrite(cfg.obs[0]->lambda, 8, nl, f);
  int32_t n = abuf.size(); fwrite(&n, 4, 1, f); fwrite(abuf.data(), 1, n, f);
  n = mbuf.size(); fwrite(&n, 4, 1, f); fwrite(mbuf.data(), 1, n, f);
  fclose(f);
  fprintf(stderr, "packed task: nd=%d nlambda=%d el=%g az=%g nodes=%d\n",
          col->x3h - col->x3l + 1, nl, el, az, m->get_N_nodes_total());
  return 0;
}

// ----------------------------------------------------------------------------------------------
// Column record: the per-depth state that obs_stokes uses before its wavelength loop.
struct LineInfo {
  int species, z, lo, up, split;
  double lam0, sf, ar, mass, A;
  int n[3];
  std::vector<double> S[3], D[3];
};

struct Record {
  int nd = 0, nlines = 0;
  std::vector<double> tau500;           // [nd]  tau500 (positive), top -> bottom
  std::vector<double> T, vt, ne, vlos, B, inc, azi, kap, hmbf, hmff, bfop, bfem;  // [nd]
  std::vector<double> lop, lem, lgc;    // [nlines][nd]
  std::vector<double> dld, adamp;       // [nlines][nd] reference's own Doppler width / damping
  std::vector<LineInfo> lines;
  bool bf_edge_in_window = false;
};

static const int NFIELD = 12;  // per-depth scalar fields before the per-line fields

// Opens the atmosphere state exactly as atmosphere::obs_stokes does (atmos/atmos_obs.cc:22-57),
// then reads every per-depth quantity that feeds atmosphere::op_em_vector.
static void extract_record(atmosphere *a, const Task &t, Record &r, std::vector<double> *opprobe,
                           const std::vector<int> &probe_l) {
  const int x3l = a->x3l, x3h = a->x3h, nd = x3h - x3l + 1;
  const fp_t theta = t.el, phi = t.az;
  a->set_grid(a->tau_grid);
  a->boundary_condition_for_rt = -1;
  a->popsetup();
  a->compute_op_referent();
  if (!a->tau_grid) a->compute_tau_referent();
  a->nltepops();
  a->atm_pop_setup();
  a->atm_pop_fill();
  fp_t ***Vr = a->project(a->Vx, a->Vy, a->Vz, theta, phi, 1, 1, 1, 1, x3l, x3h);
  fp_t ****Bt = a->transform(a->Bx, a->By, a->Bz, theta, phi, 1, 1, 1, 1, x3l, x3h);
  for (int i = 0; i < a->natm; ++i) { a->atml[i]->rtsetup(1, 1, 1, 1, x3l, x3h); a->atml[i]->zeeman_setup(); }
  fp_t *lv = airtovac((fp_t *)t.lambda.data(), t.nlambda) - 1;
  const int nl = t.nlambda;

  r.nd = nd;
  auto rs = [&](std::vector<double> &v) { v.assign(nd, 0.0); };
  rs(r.tau500); rs(r.T); rs(r.vt); rs(r.ne); rs(r.vlos); rs(r.B); rs(r.inc); rs(r.azi);
  rs(r.kap); rs(r.hmbf); rs(r.hmff); rs(r.bfop); rs(r.bfem);
  h_minus_mol *hm = 0;
  for (int i = 0; i < a->natm; ++i) if (!hm) hm = dynamic_cast<h_minus_mol *>(a->atml[i]);
  for (int kk = 0; kk < nd; ++kk) {
    int x = x3l + kk;
    fp_t T = a->T[1][1][x], Ne = a->Ne[1][1][x];
    r.tau500[kk] = -a->rt_grid[x];
    r.T[kk] = T; r.vt[kk] = a->Vt[1][1][x]; r.ne[kk] = Ne; r.vlos[kk] = Vr[1][1][x];
    r.B[kk] = Bt[1][1][1][x]; r.inc[kk] = Bt[2][1][1][x]; r.azi[kk] = Bt[3][1][1][x];
    r.kap[kk] = a->op_referent[1][1][x];
    if (hm) {
      fp_t nH0 = hm->fetch_population(1, 1, x, 0, 0);
      fp_t tp = 5040.0 / T;
      r.hmbf[kk] = 4.158E-28 * Ne * k * T * pow(tp, 2.5) * pow(10.0, 0.754 * tp) * nH0;
      r.hmff[kk] = 1E-26 * Ne * k * T * nH0;
    }
  }
  // bound-free totals (atom::boundfree_op_em_vector), flat within the window below the edge
  fp_t ******op = ft6dim(1, nl, 1, 1, 1, 1, x3l, x3h, 1, 4, 1, 4);
  fp_t *****em = ft5dim(1, nl, 1, 1, 1, 1, x3l, x3h, 1, 4);
  memset(op[1][1][1][x3l][1] + 1, 0, nl * nd * 16 * sizeof(fp_t));
  memset(em[1][1][1][x3l] + 1, 0, nl * nd * 4 * sizeof(fp_t));
  for (int i = 0; i < a->natm; ++i)
    if (atom *at = dynamic_cast<atom *>(a->atml[i]))
      at->boundfree_op_em_vector(a->T, a->Ne, Vr, theta, phi, lv, nl, op, em);
  for (int kk = 0; kk < nd; ++kk) {
    r.bfop[kk] = op[1][1][1][x3l + kk][1][1];
    r.bfem[kk] = em[1][1][1][x3l + kk][1];
    if (op[nl][1][1][x3l + kk][1][1] != r.bfop[kk]) r.bf_edge_in_window = true;
  }
  // bound-bound transitions (atom::boundbound_op_em_vector, A > 1)
  r.lines.clear();
  std::vector<std::vector<double>> lop, lem, lgc, ldld, la;
  for (int i = 0; i < a->natm; ++i) {
    atom *at = dynamic_cast<atom *>(a->atml[i]);
    if (!at) continue;
    for (int z = 0; z <= at->Z; ++z)
      for (int up = 1; up < at->nl[z]; ++up)
        for (int lo = 0; lo < up; ++lo) {
          if (!(at->A[z][up][lo] > 1E0)) continue;
          LineInfo L;
          L.species = i; L.z = z; L.lo = lo; L.up = up;
          L.lam0 = h * c / (at->ee[z][up] - at->ee[z][lo]);
          L.ar = at->damp_rad(at->A[z], lo, up);
          L.sf = L.lam0 * L.lam0 / (4.0 * pi * c);
          L.mass = at->mass;
          L.A = at->A[z][up][lo];
          int tr = at->tmap[z][up][lo];
          L.split = at->split[tr];
          for (int gi = 0; gi < 3; ++gi) L.n[gi] = 0;
          if (L.split) {
            fp_t *Sx[3] = {at->S_p[tr], at->S_b[tr], at->S_r[tr]};
            fp_t *Dx[3] = {at->delta_lambda_p[tr], at->delta_lambda_b[tr], at->delta_lambda_r[tr]};
            for (int gi = 0; gi < 3; ++gi) {
              L.n[gi] = at->nm[tr][gi];
              L.S[gi].assign(Sx[gi], Sx[gi] + L.n[gi]);
              L.D[gi].assign(Dx[gi], Dx[gi] + L.n[gi]);
            }
          }
          std::vector<double> o(nd), em_(nd), gcv(nd), dd(nd), aa(nd);
          fp_t Blu = at->B[z][lo][up], Bul = at->B[z][up][lo];
          for (int kk = 0; kk < nd; ++kk) {
            int x = x3l + kk;
            fp_t T = a->T[1][1][x], Ne = a->Ne[1][1][x];
            o[kk] = (at->pop[1][1][x].n[z][lo] * Blu - at->pop[1][1][x].n[z][up] * Bul) * h * c / L.lam0 / 4.0 / pi;
            em_[kk] = at->pop[1][1][x].n[z][up] * L.A * h * c / L.lam0 / 4.0 / pi;
            gcv[kk] = at->damp_col(1, 1, x, z, up, lo, T, Ne, L.lam0);
            dd[kk] = at->broad_dop(L.lam0, T, a->Vt[1][1][x]);
            aa[kk] = L.sf * (L.ar + gcv[kk] * turn_on_damping) / dd[kk];
          }
          r.lines.push_back(L);
          lop.push_back(o); lem.push_back(em_); lgc.push_back(gcv); ldld.push_back(dd); la.push_back(aa);
        }
  }
  r.nlines = r.lines.size();
  r.lop.clear(); r.lem.clear(); r.lgc.clear(); r.dld.clear(); r.adamp.clear();
  for (int j = 0; j < r.nlines; ++j) {
    r.lop.insert(r.lop.end(), lop[j].begin(), lop[j].end());
    r.lem.insert(r.lem.end(), lem[j].begin(), lem[j].end());
    r.lgc.insert(r.lgc.end(), lgc[j].begin(), lgc[j].end());
    r.dld.insert(r.dld.end(), ldld[j].begin(), ldld[j].end());
    r.adamp.insert(r.adamp.end(), la[j].begin(), la[j].end());
  }
  // optional: the reference's full normalised opacity at a few wavelengths
  if (opprobe) {
    a->op_em_vector(Vr, Bt, theta, phi, lv, nl, op, em);
    opprobe->clear();
    for (int li : probe_l) {
      if (a->tau_grid) a->normalize_to_referent_opacity(op[li + 1], em[li + 1]);
      for (int kk = 0; kk < nd; ++kk) {
        for (int s = 1; s <= 4; ++s)
          for (int sp = 1; sp <= 4; ++sp) opprobe->push_back(op[li + 1][1][1][x3l + kk][s][sp]);
        for (int s = 1; s <= 4; ++s) opprobe->push_back(em[li + 1][1][1][x3l + kk][s]);
      }
    }
  }
  del_ft6dim(op, 1, nl, 1, 1, 1, 1, x3l, x3h, 1, 4, 1, 4);
  del_ft5dim(em, 1, nl, 1, 1, 1, 1, x3l, x3h, 1, 4);
  delete[] (lv + 1);
  del_ft4dim(Bt, 1, 3, 1, 1, 1, 1, x3l, x3h);
  del_ft3dim(Vr, 1, 1, 1, 1, x3l, x3h);
  for (int i = 0; i < a->natm; ++i) { a->atml[i]->rtclean(0, 0, 1, 1, 1, 1, x3l, x3h); a->atml[i]->zeeman_clear(); }
  a->popclean();
}

// record -> flat vector [nd][NFIELD + 3*nlines] (depth-major), the layout of the tangents
static std::vector<double> record_flat(const Record &r) {
  int nf = NFIELD + 3 * r.nlines;
  std::vector<double> v(r.nd * nf);
  for (int kk = 0; kk < r.nd; ++kk) {
    double *p = &v[kk * nf];
    p[0] = r.T[kk]; p[1] = r.vt[kk]; p[2] = r.ne[kk]; p[3] = r.vlos[kk]; p[4] = r.B[kk];
    p[5] = r.inc[kk]; p[6] = r.azi[kk]; p[7] = r.kap[kk]; p[8] = r.hmbf[kk]; p[9] = r.hmff[kk];
    p[10] = r.bfop[kk]; p[11] = r.bfem[kk];
    for (int j = 0; j < r.nlines; ++j) {
      p[NFIELD + 3 * j + 0] = r.lop[j * r.nd + kk];
      p[NFIELD + 3 * j + 1] = r.lem[j * r.nd + kk];
      p[NFIELD + 3 * j + 2] = r.lgc[j * r.nd + kk];
    }
  }
  return v;
}

static void set_nodes(model *m, const double *nodes) {
  int np = m->get_N_nodes_total();
  fp_t *p = new fp_t[np] - 1;
  for (int i = 0; i < np; ++i) p[i + 1] = nodes[i];
  m->set_parameters(p);
  delete[] (p + 1);
}

static double node_step(model *m, int p /*1-based*/) {
  switch (m->which_parameter(p)) {
    case 1: return delta_T;
    case 2: return delta_vt;
    case 3: return delta_vr;
    case 4: return delta_B;
    default: return delta_angle;
  }
}

static int do_dump(const char *tskname, const char *nodesname, int npix, int flags, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  Task t = load_task(tskname);
  std::vector<uint8_t> nb = read_file_bytes(nodesname);
  const double *nodes = (const double *)nb.data();
  model *m = task_model(t, io);
  const int np = m->get_N_nodes_total(), nl = t.nlambda;
  if ((int)(nb.size() / 8) < npix * np) { fprintf(stderr, "nodes file too short\n"); return 2; }
  fp_t *lam1 = lambda_1based(t);

  std::vector<double> allrec, allstokes, allstokes_resp, allresp, alltan, allrf_ok, alldld, alla, tau;
  std::vector<double> opprobe;
  std::vector<int> probe_l = {0, 40, 80, 100, 120, 160, 200};
  Record r0;
  int nd = 0, nf = 0;
  double t_build = 0, t_synth = 0, t_resp = 0;
  for (int ip = 0; ip < npix; ++ip) {
    atmosphere *a = task_atmos(t, io);
    set_nodes(m, nodes + ip * np);
    double t0 = wall_s();
    a->build_from_nodes(m);
    t_build += wall_s() - t0;
    Record r;
    extract_record(a, t, r, (ip == 0 && (flags & 4)) ? &opprobe : 0, probe_l);
    if (ip == 0) { r0 = r; nd = r.nd; nf = NFIELD + 3 * r.nlines; tau = r.tau500; }
    std::vector<double> fl = record_flat(r);
    allrec.insert(allrec.end(), fl.begin(), fl.end());
    alldld.insert(alldld.end(), r.dld.begin(), r.dld.end());
    alla.insert(alla.end(), r.adamp.begin(), r.adamp.end());
    for (int kk = 0; kk < nd; ++kk)
      if (fabs(r.tau500[kk] - tau[kk]) > 1e-12 * tau[kk]) { fprintf(stderr, "tau grid differs between pixels\n"); return 3; }
    // reference synthesis
    t0 = wall_s();
    observable *o = a->obs_stokes(t.el, t.az, lam1, nl);
    t_synth += wall_s() - t0;
    fp_t **S = o->get_S(1, 1);
    for (int l = 1; l <= nl; ++l) for (int s = 1; s <= 4; ++s) allstokes.push_back(S[s][l]);
    del_ft2dim(S, 1, 4, 1, nl);
    delete o;
    // reference node responses (semi-analytic)
    if (flags & 1) {
      fp_t ***resp = ft3dim(1, np, 1, nl, 1, 4);
      t0 = wall_s();
      observable *o2 = a->obs_stokes_responses_to_nodes(m, t.el, t.az, lam1, nl, resp, 0);
      t_resp += wall_s() - t0;
      for (int p = 1; p <= np; ++p) for (int l = 1; l <= nl; ++l) for (int s = 1; s <= 4; ++s) allresp.push_back(resp[p][l][s]);
      del_ft3dim(resp, 1, np, 1, nl, 1, 4);
      // the Stokes vector of the same call: stokes_lm_fit's residual is formed with it
      fp_t **S2 = o2->get_S(1, 1);
      for (int l = 1; l <= nl; ++l) for (int s = 1; s <= 4; ++s) allstokes_resp.push_back(S2[s][l]);
      del_ft2dim(S2, 1, 4, 1, nl);
      delete o2;
    }
    // record tangents by central differences of the node -> atmosphere map
    if (flags & 2) {
      for (int p = 1; p <= np; ++p) {
        double st = node_step(m, p);
        bool thermal = (m->which_parameter(p) == 1);
        std::vector<double> plus, minus;
        for (int side = 0; side < 2; ++side) {
          atmosphere *b = task_atmos(t, io);
          m->perturb_node_value(p, side == 0 ? 0.5 * st : -0.5 * st);
          b->build_from_nodes(m);   // T nodes: full build (HE + chemistry), as atmos_fit.cc:1227-1249
          if (!thermal) {           // other nodes: base build, then interpolation only (:1253-1307)
            m->perturb_node_value(p, side == 0 ? -0.5 * st : 0.5 * st);
            b->build_from_nodes(m);
            m->perturb_node_value(p, side == 0 ? 0.5 * st : -0.5 * st);
            b->interpolate_from_nodes(m);
          }
          m->perturb_node_value(p, side == 0 ? -0.5 * st : 0.5 * st);
          Record rr;
          extract_record(b, t, rr, 0, probe_l);
          (side == 0 ? plus : minus) = record_flat(rr);
          delete b;
        }
        for (size_t i = 0; i < plus.size(); ++i) alltan.push_back((plus[i] - minus[i]) / st);
      }
    }
    delete a;
  }
  fprintf(stderr, "ref timings per pixel: build %.4f s, obs_stokes %.4f s, responses %.4f s\n",
          t_build / npix, t_synth / npix, (flags & 1) ? t_resp / npix : 0.0);

  SbinWriter w(outname);
  double meta[8] = {(double)nd, (double)nl, (double)np, (double)r0.nlines, (double)NFIELD, t.el, t.az,
                    r0.bf_edge_in_window ? 1.0 : 0.0};
  w.put("meta", {8}, meta);
  w.put("lambda_air", {nl}, t.lambda.data());
  w.put("tau500", {nd}, tau.data());
  w.put("nodes", {npix, np}, nodes);
  std::vector<double> which(np);
  for (int p = 1; p <= np; ++p) which[p - 1] = m->which_parameter(p);
  w.put("node_kind", {np}, which.data());
  // line constants: [nlines][8] = lam0, sf, ar, mass, A, split, species, z ; patterns [nlines][3][2][16]
  std::vector<double> lc, pat(r0.nlines * 3 * 2 * 16, 0.0), pn(r0.nlines * 3, 0.0);
  for (int j = 0; j < r0.nlines; ++j) {
    const LineInfo &L = r0.lines[j];
    double v[8] = {L.lam0, L.sf, L.ar, L.mass, L.A, (double)L.split, (double)L.species, (double)L.z};
    lc.insert(lc.end(), v, v + 8);
    for (int gi = 0; gi < 3; ++gi) {
      pn[j * 3 + gi] = L.n[gi];
      for (int i = 0; i < L.n[gi] && i < 16; ++i) {
        pat[((j * 3 + gi) * 2 + 0) * 16 + i] = L.S[gi][i];
        pat[((j * 3 + gi) * 2 + 1) * 16 + i] = L.D[gi][i];
      }
    }
  }
  w.put("line_const", {r0.nlines, 8}, lc.data());
  w.put("line_ncomp", {r0.nlines, 3}, pn.data());
  w.put("line_pattern", {r0.nlines, 3, 2, 16}, pat.data());
  w.put("record", {npix, nd, nf}, allrec.data());
  w.put("ref_dld", {npix, r0.nlines, nd}, alldld.data());
  w.put("ref_adamp", {npix, r0.nlines, nd}, alla.data());
  w.put("stokes", {npix, nl, 4}, allstokes.data());
  if (flags & 1) w.put("responses", {npix, np, nl, 4}, allresp.data());
  if (flags & 1) w.put("stokes_resp", {npix, nl, 4}, allstokes_resp.data());
  if (flags & 2) w.put("tangent", {npix, np, nd, nf}, alltan.data());
  if (flags & 4) {
    std::vector<double> pl(probe_l.begin(), probe_l.end());
    w.put("probe_l", {(int64_t)pl.size()}, pl.data());
    w.put("opacity_probe", {(int64_t)probe_l.size(), nd, 20}, opprobe.data());
  }
  double tm[3] = {t_build / npix, t_synth / npix, (flags & 1) ? t_resp / npix : 0.0};
  w.put("ref_seconds_per_pixel", {3}, tm);
  delete m;
  delete[] (lam1 + 1);
  return 0;
}

// ----------------------------------------------------------------------------------------------
// lmfit: reference LM inversion per pixel (atmos_fit.cc:18-227)
static int do_lmfit(const char *tskname, const char *n0name, const char *tgtname, const char *maskname,
                    int npix, int iters, const char *outname, double broadening) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  Task t = load_task(tskname);
  std::vector<uint8_t> nb = read_file_bytes(n0name), tb = read_file_bytes(tgtname), mb = read_file_bytes(maskname);
  const double *n0 = (const double *)nb.data(), *tgt = (const double *)tb.data(), *msk = (const double *)mb.data();
  model *m = task_model(t, io);
  const int np = m->get_N_nodes_total(), nl = t.nlambda;
  fp_t *lam1 = lambda_1based(t);
  std::vector<double> out_nodes, out_stokes, out_chi;
  double t_fit = 0;
  for (int ip = 0; ip < npix; ++ip) {
    atmosphere *a = task_atmos(t, io);
    model *mm = task_model(t, io);
    set_nodes(mm, n0 + ip * np);
    observable *o = new observable(1, 1, 4, nl);
    o->set_lambda(lam1);
    fp_t ****S = ft4dim(1, 1, 1, 1, 1, 4, 1, nl);
    for (int l = 0; l < nl; ++l) for (int s = 0; s < 4; ++s) S[1][1][s + 1][l + 1] = tgt[(ip * nl + l) * 4 + s];
    o->set(S);
    del_ft4dim(S, 1, 1, 1, 1, 1, 4, 1, nl);
    fp_t *mask = new fp_t[nl] - 1;
    for (int l = 0; l < nl; ++l) mask[l + 1] = msk[ip * nl + l];
    o->set_mask(mask);
    delete[] (mask + 1);
    o->set_viewing_angle(t.el, t.az);
    o->set_to_invert(1);
    o->set_no_iterations(iters);
    o->set_start_lambda(1E3);
    o->set_stopping_chisq(1E-30);
    fp_t ws[4] = {1.0, 1.0, 1.0, 1.0};
    o->set_w_stokes(ws);
    o->set_inv_parameters(0.0, broadening, 1.0, 1.0);  // spectral broadening [cm], 0: none
    double t0 = wall_s();
    observable *fit = a->stokes_lm_fit(o, t.el, t.az, mm);
    t_fit += wall_s() - t0;
    for (int p = 1; p <= np; ++p) out_nodes.push_back(mm->get_parameter(p));
    fp_t **F = fit->get_S(1, 1);
    double chi = 0;
    for (int l = 1; l <= nl; ++l)
      for (int s = 1; s <= 4; ++s) {
        out_stokes.push_back(F[s][l]);
        double d = (tgt[(ip * nl + l - 1) * 4 + s - 1] - F[s][l]) * msk[ip * nl + l - 1];
        chi += d * d;
      }
    out_chi.push_back(chi);
    del_ft2dim(F, 1, 4, 1, nl);
    delete fit; delete o; delete mm; delete a;
  }
  SbinWriter w(outname);
  w.put("fit_nodes", {npix, np}, out_nodes.data());
  w.put("fit_stokes", {npix, nl, 4}, out_stokes.data());
  w.put("fit_chi2", {npix}, out_chi.data());
  double tf = t_fit / npix;
  w.put("ref_seconds_per_pixel", {1}, &tf);
  delete m;
  delete[] (lam1 + 1);
  return 0;
}

// ----------------------------------------------------------------------------------------------
// ali: inputs and per-iteration populations of the NLTE level-population iteration
// (atmosphere::nltepops, atmos/atmos_pop.cc:67-240) for each column built from the nodes.
// The iteration body is the reference's own: opacity_active_only + formal (scalar, with the
// diagonal operator) + atom::add + atmosphere::newpops, run niter times; then a fresh copy of
// the column runs nltepops() itself to convergence.
static int do_ali(const char *tskname, const char *nodesname, int ncol, int niter, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  Task t = load_task(tskname);
  std::vector<uint8_t> nb = read_file_bytes(nodesname);
  const double *nodes = (const double *)nb.data();
  model *m = task_model(t, io);
  const int np = m->get_N_nodes_total();
  std::vector<double> oT, oNe, oNa, oKap, oGrid, oLam, oLw, oFudge, oTh, oBin, oVr, oDld, oAd, oSig, oBfr, oColl,
      oBgop, oBgem, oPop0, oPopIt, oRel, oPopConv, oTr, oTrc, oA, oB, oWall;
  int nd = 0, nlam = 0, ntp = 0, nmap = 0, nline = 0, nbf = 0;
  for (int ic = 0; ic < ncol; ++ic) {
    atmosphere *a = task_atmos(t, io);
    set_nodes(m, nodes + ic * np);
    a->build_from_nodes(m);
    const int x3l = a->x3l, x3h = a->x3h;
    nd = x3h - x3l + 1;
    a->set_grid(a->tau_grid);
    a->boundary_condition_for_rt = -1;
    a->popsetup();
    a->compute_op_referent();
    // nltepops prologue (atmos_pop.cc:70-130)
    a->ltepops();
    fp_t *lambda = 0;
    int32_t nlambda = 0;
    for (int i = 0; i < a->natm; ++i) a->atml[i]->rtsetup(a->x1l, a->x1h, a->x2l, a->x2h, x3l, x3h);
    for (int i = 0; i < a->natm; ++i)
      lambda = a->atml[i]->getlambda(lambda, nlambda, a->T[1][1][x3h], a->Nt[1][1][x3h], a->Ne[1][1][x3h]);
    fp_t *th, *ph;
    fp_t *bin = a->anglesetup(th, ph, ntp);
    std::vector<double> lw(nlambda);
    if (nlambda >= 2) {
      lw[0] = (lambda[1] - lambda[0]) * 0.5;
      lw[nlambda - 1] = (lambda[nlambda - 1] - lambda[nlambda - 2]) * 0.5;
      for (int l = 1; l < nlambda - 1; ++l) lw[l] = (lambda[l + 1] - lambda[l - 1]) * 0.5;
    } else if (nlambda) {
      lw[0] = 1.0;
    }
    if (a->tau_grid) a->compute_op_referent();
    for (int i = 0; i < a->natm; ++i) a->atml[i]->compute_active_population(a->T, a->Ne);
    atom *at = 0;
    for (int i = 0; i < a->natm; ++i)
      if (a->atml[i]->check_if_nlte()) at = dynamic_cast<atom *>(a->atml[i]);
    if (!at || !nlambda) { fprintf(stderr, "no NLTE atom / wavelengths\n"); return 4; }
    nlam = nlambda;
    nmap = at->nmap;
    // transitions (1-based tr): type 0 line, 1 bound-free; lower / upper mapped levels
    std::vector<int> trl, tru, trz, trt;
    for (int tr = 1; tr <= at->ntr; ++tr) {
      int z = at->inverse_tmap[tr][2], lo = at->inverse_tmap[tr][3], up = at->inverse_tmap[tr][4];
      trz.push_back(z);
      if (up < at->nl[z]) { trt.push_back(0); trl.push_back(at->rmap[z][lo]); tru.push_back(at->rmap[z][up]); }
      else { trt.push_back(1); trl.push_back(at->rmap[z][lo]); tru.push_back(at->rmap[z + 1][0]); }
    }
    if (ic == 0) {
      for (int l = 0; l < nlambda; ++l) { oLam.push_back(lambda[l]); oLw.push_back(lw[l]); oFudge.push_back(a->get_opacity_fudge(lambda[l])); }
      for (int tp = 1; tp <= ntp; ++tp) { oTh.push_back(th[tp]); oBin.push_back(bin[tp]); }
      nline = nbf = 0;
      for (size_t q = 0; q < trt.size(); ++q) {
        const int z = trz[q], lo = at->lmap[trl[q]];
        oTr.push_back(trt[q]); oTr.push_back(trl[q]); oTr.push_back(tru[q]); oTr.push_back(z);
        if (trt[q] == 0) {
          const int up = at->lmap[tru[q]];
          const double lam0 = h * c / (at->ee[z][up] - at->ee[z][lo]);
          oTrc.push_back(lam0); oTrc.push_back(at->A[z][up][lo]); oTrc.push_back(at->B[z][lo][up]);
          oTrc.push_back(at->B[z][up][lo]); oTrc.push_back(at->ee[z][up] - at->ee[z][lo]);
          oTrc.push_back(lam0 * lam0 / (4.0 * pi * c)); oTrc.push_back(at->damp_rad(at->A[z], lo, up));
          oTrc.push_back(0.0);
          ++nline;
        } else {
          for (int q8 = 0; q8 < 8; ++q8) oTrc.push_back(0.0);
          for (int l = 0; l < nlambda; ++l) oSig.push_back(at->bf[z][lo] ? at->bf[z][lo]->U(lambda[l]) : 0.0);
          ++nbf;
        }
      }
      for (int i = 0; i < nmap; ++i)
        for (int j = 0; j < nmap; ++j) {
          const int zi = at->zmap[i], li = at->lmap[i], zj = at->zmap[j], lj = at->lmap[j];
          oA.push_back(zi == zj ? at->A[zi][li][lj] : 0.0);
          oB.push_back(zi == zj ? at->B[zi][li][lj] : 0.0);
        }
    }
    fp_t ***T = a->T, ***Ne = a->Ne;
    for (int kk = 0; kk < nd; ++kk) {
      const int x = x3l + kk;
      oT.push_back(T[1][1][x]); oNe.push_back(Ne[1][1][x]); oNa.push_back(at->pop[1][1][x].Na);
      oKap.push_back(a->op_referent[1][1][x]); if (ic == 0) oGrid.push_back(a->rt_grid[x]);
      for (int i = 0; i < nmap; ++i) oPop0.push_back(at->get_mapped_pop(1, 1, x, i));
    }
    for (int tp = 1; tp <= ntp; ++tp) {
      fp_t ***Vr = a->project(a->Vx, a->Vy, a->Vz, th[tp], ph[tp], 1, 1, 1, 1, x3l, x3h);
      for (int kk = 0; kk < nd; ++kk) oVr.push_back(Vr[1][1][x3l + kk]);
      fp_t ****Bt = a->transform(a->Bx, a->By, a->Bz, th[tp], ph[tp], 1, 1, 1, 1, x3l, x3h);
      for (int l = 0; l < nlambda; ++l) {
        fp_t ***op = a->opacity_lte(T, Ne, Vr, a->Vt, Bt, th[tp], ph[tp], lambda[l]);
        fp_t ***em = a->emissivity_lte(T, Ne, Vr, a->Vt, Bt, th[tp], ph[tp], lambda[l]);
        fp_t ***ff = at->freefree_op(T, Ne, Vr, lambda[l]);
        fp_t ***ry = at->rayleigh_op(lambda[l]);
        for (int kk = 0; kk < nd; ++kk) {
          const int x = x3l + kk;
          const double pas = ff[1][1][x] + ry[1][1][x];
          oBgop.push_back(op[1][1][x] + pas);
          oBgem.push_back(em[1][1][x] + pas * Planck_f(lambda[l], T[1][1][x]));
        }
        del_ft3dim(op, 1, 1, 1, 1, x3l, x3h); del_ft3dim(em, 1, 1, 1, 1, x3l, x3h);
        del_ft3dim(ff, 1, 1, 1, 1, x3l, x3h); del_ft3dim(ry, 1, 1, 1, 1, x3l, x3h);
      }
      del_ft4dim(Bt, 1, 3, 1, 1, 1, 1, x3l, x3h);
      del_ft3dim(Vr, 1, 1, 1, 1, x3l, x3h);
    }
    // per line transition and depth: Doppler width and damping (atom_rad.cc boundbound_op)
    for (size_t q = 0; q < trt.size(); ++q) {
      if (trt[q] != 0) continue;
      const int z = trz[q], lo = at->lmap[trl[q]], up = at->lmap[tru[q]];
      const double lam0 = h * c / (at->ee[z][up] - at->ee[z][lo]);
      const double ar = at->damp_rad(at->A[z], lo, up), sf = lam0 * lam0 / (4.0 * pi * c);
      for (int kk = 0; kk < nd; ++kk) {
        const int x = x3l + kk;
        const double dld = at->broad_dop(lam0, T[1][1][x], a->Vt[1][1][x]);
        const double gc = at->damp_col(1, 1, x, z, up, lo, T[1][1][x], Ne[1][1][x], lam0);
        oDld.push_back(dld);
        oAd.push_back(sf * (ar + gc * turn_on_damping) / dld);
      }
    }
    // per bound-free transition and depth: n_cont * ratio = LTE-like population factor
    // (atom_rad.cc boundfree_op: ne saha T^-1.5 g_i/g_c exp((ip - E_i)/kT))
    for (size_t q = 0; q < trt.size(); ++q) {
      if (trt[q] != 1) continue;
      const int z = trz[q], lo = at->lmap[trl[q]];
      for (int kk = 0; kk < nd; ++kk) {
        const int x = x3l + kk;
        const double TT = T[1][1][x];
        oBfr.push_back(Ne[1][1][x] * saha_const * pow(TT, -1.5) * double(at->g[z][lo]) / double(at->g[z + 1][0]) *
                       exp((at->ip[z] - at->ee[z][lo]) / k / TT));
      }
    }
    // collisional rates from mapped level i to j (atom_pop.cc:27-145 rate matrix)
    for (int kk = 0; kk < nd; ++kk) {
      const int x = x3l + kk;
      const double TT = T[1][1][x], ne = Ne[1][1][x];
      std::vector<double> C(nmap * nmap, 0.0);
      for (int i = 0; i < nmap - 1; ++i) {
        const int z = at->zmap[i], l = at->lmap[i];
        for (int ll = 0; ll < at->nl[z]; ++ll) {
          const int j = i + (ll - l);
          C[i * nmap + j] = at->C_ij(z, l, ll, TT, ne);
        }
        if (int dl = at->nl[z] - l) {
          C[i * nmap + i + dl] = at->C_i_cont(z, l, TT, ne);
          C[(i + dl) * nmap + i] = at->C_cont_i(z, l, TT, ne);
        }
      }
      oColl.insert(oColl.end(), C.begin(), C.end());
    }
    // the reference's own iteration, niter times (atmos_pop.cc:133-214), populations after each
    fp_t ***S = ft3dim(a->x1l, a->x1h, a->x2l, a->x2h, x3l, x3h);
    fp_t ***L = ft3dim(a->x1l, a->x1h, a->x2l, a->x2h, x3l, x3h);
    for (int it = 0; it < niter; ++it) {
      for (int i = 0; i < a->natm; ++i) a->atml[i]->rtinit();
      for (int tp = 1; tp <= ntp; ++tp) {
        fp_t ***Vr = a->project(a->Vx, a->Vy, a->Vz, th[tp], ph[tp], 1, 1, 1, 1, x3l, x3h);
        fp_t ****Bt = a->transform(a->Bx, a->By, a->Bz, th[tp], ph[tp], 1, 1, 1, 1, x3l, x3h);
        for (int l = 0; l < nlambda; ++l) {
          for (int i = 0; i < a->natm; ++i) a->atml[i]->prof_init();
          fp_t ***op = a->opacity_lte(T, Ne, Vr, a->Vt, Bt, th[tp], ph[tp], lambda[l]);
          fp_t ***em = a->emissivity_lte(T, Ne, Vr, a->Vt, Bt, th[tp], ph[tp], lambda[l]);
          op = a->add(a->opacity_active_only(T, Ne, Vr, a->Vt, Bt, th[tp], ph[tp], lambda[l]), op, 1, 1, 1, 1, x3l, x3h);
          em = a->add(a->emissivity_active_only(T, Ne, Vr, a->Vt, Bt, th[tp], ph[tp], lambda[l]), em, 1, 1, 1, 1, x3l, x3h);
          if (a->tau_grid) a->normalize_to_referent_opacity(op, em);
          a->formal(a->rt_grid, S, L, op, em, th[tp], ph[tp], a->boundary_condition_for_rt);
          if (a->tau_grid) a->de_normalize(op, em);
          for (int i = 0; i < a->natm; ++i) a->atml[i]->add(S, L, op, lambda[l], lw[l], bin[tp]);
          del_ft3dim(em, 1, 1, 1, 1, x3l, x3h);
          del_ft3dim(op, 1, 1, 1, 1, x3l, x3h);
        }
        del_ft4dim(Bt, 1, 3, 1, 1, 1, 1, x3l, x3h);
        del_ft3dim(Vr, 1, 1, 1, 1, x3l, x3h);
      }
      double rc = a->newpops(T, a->Nt, Ne, lambda, nlambda, 1);
      if (rc < 0.0) rc = -1.0 - fabs(a->newpops(T, a->Nt, Ne, lambda, nlambda, 0));
      oRel.push_back(rc);
      for (int kk = 0; kk < nd; ++kk)
        for (int i = 0; i < nmap; ++i) oPopIt.push_back(at->get_mapped_pop(1, 1, x3l + kk, i));
    }
    del_ft3dim(S, a->x1l, a->x1h, a->x2l, a->x2h, x3l, x3h);
    del_ft3dim(L, a->x1l, a->x1h, a->x2l, a->x2h, x3l, x3h);
    // the reference's nltepops on a fresh copy of the column
    {
      atmosphere *b = task_atmos(t, io);
      b->build_from_nodes(m);
      b->set_grid(b->tau_grid);
      b->boundary_condition_for_rt = -1;
      b->popsetup();
      b->compute_op_referent();
      double t0 = wall_s();
      b->nltepops();
      oWall.push_back(wall_s() - t0);
      atom *bt = 0;
      for (int i = 0; i < b->natm; ++i)
        if (b->atml[i]->check_if_nlte()) bt = dynamic_cast<atom *>(b->atml[i]);
      for (int kk = 0; kk < nd; ++kk)
        for (int i = 0; i < nmap; ++i) oPopConv.push_back(bt->get_mapped_pop(1, 1, x3l + kk, i));
      delete b;
    }
    delete a;
  }
  SbinWriter w(outname);
  const int64_t nC = ncol, nD = nd, nLm = nlam, nR = ntp, nM = nmap, nT = oTr.size() / 4;
  w.put("ali_T", {nC, nD}, oT.data()); w.put("ali_ne", {nC, nD}, oNe.data()); w.put("ali_na", {nC, nD}, oNa.data());
  w.put("ali_kap", {nC, nD}, oKap.data()); w.put("ali_grid", {nD}, oGrid.data());
  w.put("ali_lambda", {nLm}, oLam.data()); w.put("ali_lw", {nLm}, oLw.data()); w.put("ali_fudge", {nLm}, oFudge.data());
  w.put("ali_th", {nR}, oTh.data()); w.put("ali_bin", {nR}, oBin.data()); w.put("ali_vray", {nC, nR, nD}, oVr.data());
  w.put("ali_tr", {nT, 4}, oTr.data()); w.put("ali_trc", {nT, 8}, oTrc.data());
  w.put("ali_A", {nM, nM}, oA.data()); w.put("ali_B", {nM, nM}, oB.data());
  w.put("ali_dld", {nC, (int64_t)nline, nD}, oDld.data()); w.put("ali_adamp", {nC, (int64_t)nline, nD}, oAd.data());
  w.put("ali_sigma", {(int64_t)nbf, nLm}, oSig.data()); w.put("ali_bfratio", {nC, (int64_t)nbf, nD}, oBfr.data());
  w.put("ali_coll", {nC, nD, nM, nM}, oColl.data());
  w.put("ali_bgop", {nC, nR, nLm, nD}, oBgop.data()); w.put("ali_bgem", {nC, nR, nLm, nD}, oBgem.data());
  w.put("ali_pop0", {nC, nD, nM}, oPop0.data());
  w.put("ali_pops_iter", {nC, (int64_t)niter, nD, nM}, oPopIt.data()); w.put("ali_relchange", {nC, (int64_t)niter}, oRel.data());
  w.put("ali_pop_conv", {nC, nD, nM}, oPopConv.data()); w.put("ali_ref_seconds", {nC}, oWall.data());
  delete m;
  return 0;
}

struct Rd {  // little-endian reader over a packed object
  const uint8_t *p;
  int i8() { int8_t v; memcpy(&v, p, 1); p += 1; return v; }
  int u8() { uint8_t v; memcpy(&v, p, 1); p += 1; return v; }
  int i32() { int32_t v; memcpy(&v, p, 4); p += 4; return v; }
  double f64() { double v; memcpy(&v, p, 8); p += 8; return v; }
};

// ----------------------------------------------------------------------------------------------
// alisetup: the tables of the population-independent part of atmosphere::nltepops (atmos_pop.cc:
// 67-240) -- the LTE background of opacity_lte (atmos_rad.cc:225-235: every LTE atom's free-free,
// Rayleigh, bound-free and bound-bound opacity, atom_rad.cc:203-535, and H- bound-free / free-free,
// mol.cc:516-632), the NLTE atom's collisional rates (atom_rad.cc:1769-1901) and line damping -- in
// the atom order of the eos mode, and the columns (return_as_array rows after build_from_nodes and
// compute_op_referent) of ncol node vectors.
static int do_alisetup(const char *tskname, const char *nodesname, int ncol, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  Task t = load_task(tskname);
  std::vector<uint8_t> nb = read_file_bytes(nodesname);
  const double *nodes = (const double *)nb.data();
  model *m = task_model(t, io);
  const int np = m->get_N_nodes_total();
  atmosphere *a = task_atmos(t, io);
  set_nodes(m, nodes);
  a->build_from_nodes(m);
  a->set_grid(a->tau_grid);
  a->popsetup();
  a->compute_op_referent();
  a->ltepops();
  fp_t *lambda = 0;
  int32_t nlambda = 0;
  for (int i = 0; i < a->natm; ++i) a->atml[i]->rtsetup(a->x1l, a->x1h, a->x2l, a->x2h, a->x3l, a->x3h);
  for (int i = 0; i < a->natm; ++i)
    lambda = a->atml[i]->getlambda(lambda, nlambda, a->T[1][1][a->x3h], a->Nt[1][1][a->x3h], a->Ne[1][1][a->x3h]);
  std::vector<atom *> atoms;
  for (int i = 0; i < a->natm; ++i)
    if (atom *at = dynamic_cast<atom *>(a->atml[i])) atoms.push_back(at);
  int inlte = -1;
  for (size_t ia = 0; ia < atoms.size(); ++ia)
    if (atoms[ia]->check_if_nlte()) inlte = ia;
  if (inlte < 0 || !nlambda) { fprintf(stderr, "no NLTE atom / wavelengths\n"); return 4; }
  // background: bound-free levels and bound-bound pairs of the LTE atoms, Rayleigh atoms (Z == 1)
  std::vector<double> bfl, bfs, bb, ray;
  for (size_t ia = 0; ia < atoms.size(); ++ia) {
    atom *at = atoms[ia];
    if (at->check_if_nlte()) continue;
    if (at->Z == 1) ray.push_back(ia);
    for (int z = 0; z < at->Z; ++z)
      for (int l = 0; l < at->nl[z]; ++l) {
        if (!at->bf[z][l]) continue;
        double v[3] = {(double)ia, (double)z, (double)l};
        bfl.insert(bfl.end(), v, v + 3);
        for (int q = 0; q < nlambda; ++q) bfs.push_back(at->bf[z][l]->U(lambda[q]));
      }
    for (int z = 0; z <= at->Z; ++z)
      for (int up = 1; up < at->nl[z]; ++up)
        for (int lo = 0; lo < up; ++lo) {
          double v[11] = {(double)ia, (double)z, (double)lo, (double)up, h * c / (at->ee[z][up] - at->ee[z][lo]),
                          at->B[z][lo][up], at->B[z][up][lo], at->damp_rad(at->A[z], lo, up),
                          at->alpha_col_dam[z][up][lo], at->col_dam_cross_section[z][up][lo], at->mass};
          bb.insert(bb.end(), v, v + 11);
        }
  }
  // the NLTE atom: mapped levels, line damping, edge cross-sections, collisional tables
  atom *at = atoms[inlte];
  const int nmap = at->nmap;
  std::vector<double> lev, line, sedge, cn(nmap * nmap, 0.0), ct(nmap * nmap * 8, 0.0), cv(nmap * nmap * 8, 0.0);
  for (int i = 0; i < nmap; ++i) {
    const int z = at->zmap[i], l = at->lmap[i];
    lev.push_back(z); lev.push_back(l);
    double se = 0.0;
    if (z < at->Z) se = at->bf[z][l] ? at->bf[z][l]->U(h * c / (at->ip[z] - at->ee[z][l])) : -1.0;
    sedge.push_back(se);
  }
  for (int tr = 1; tr <= at->ntr; ++tr) {
    const int z = at->inverse_tmap[tr][2], lo = at->inverse_tmap[tr][3], up = at->inverse_tmap[tr][4];
    if (up >= at->nl[z]) continue;
    double v[4] = {at->alpha_col_dam[z][up][lo], at->col_dam_cross_section[z][up][lo], at->mass,
                   at->damp_rad(at->A[z], lo, up)};
    line.insert(line.end(), v, v + 4);
  }
  for (int i = 0; i < nmap; ++i)
    for (int j = 0; j < nmap; ++j) {
      const int zi = at->zmap[i], li = at->lmap[i], zj = at->zmap[j], lj = at->lmap[j];
      if (zi != zj || li == lj || li >= at->nl[zi] || lj >= at->nl[zj]) continue;
      colr *C = at->cr[zi][li > lj ? li : lj][li > lj ? lj : li];
      // the table, read back from the object's own wire format (colr::pack / tbcr::pack, colr.cc:46-99)
      std::vector<uint8_t> pb(C->size(io) + 64);
      C->pack(pb.data(), 0, io);
      Rd r{pb.data()};
      if (r.i8() != COLR_TYPE_TAB) continue;
      const int n = r.i32();
      if (n > 8) { fprintf(stderr, "collision table too long\n"); return 2; }
      cn[i * nmap + j] = n;
      for (int q = 0; q < n; ++q) ct[(i * nmap + j) * 8 + q] = r.f64();
      for (int q = 0; q < n; ++q) cv[(i * nmap + j) * 8 + q] = r.f64();
    }
  const double meta[4] = {(double)inlte, (double)at->Z, (double)nlambda, (double)nmap};
  delete a;
  // the columns
  std::vector<double> harr;
  int nd = 0;
  for (int ic = 0; ic < ncol; ++ic) {
    atmosphere *b = task_atmos(t, io);
    set_nodes(m, nodes + ic * np);
    b->build_from_nodes(m);
    b->set_grid(b->tau_grid);
    b->popsetup();
    b->compute_op_referent();
    fp_t **arr = b->return_as_array();
    nd = b->x3h - b->x3l + 1;
    for (int q = 1; q <= 12; ++q)
      for (int i = 1; i <= nd; ++i) harr.push_back(arr[q][i]);
    del_ft2dim(arr, 1, 12, 1, nd);
    delete b;
  }
  SbinWriter w(outname);
  w.put("alis_meta", {4}, meta);
  w.put("alis_bf", {(int64_t)bfl.size() / 3, 3}, bfl.data());
  w.put("alis_bfsig", {(int64_t)bfl.size() / 3, nlambda}, bfs.data());
  w.put("alis_bb", {(int64_t)bb.size() / 11, 11}, bb.data());
  w.put("alis_ray", {(int64_t)ray.size()}, ray.data());
  w.put("alis_lev", {nmap, 2}, lev.data());
  w.put("alis_line", {(int64_t)line.size() / 4, 4}, line.data());
  w.put("alis_sedge", {nmap}, sedge.data());
  w.put("alis_coll_n", {nmap, nmap}, cn.data());
  w.put("alis_coll_t", {nmap, nmap, 8}, ct.data());
  w.put("alis_coll_v", {nmap, nmap, 8}, cv.data());
  w.put("alis_atm", {ncol, 12, nd}, harr.data());
  delete[] lambda;
  delete m;
  return 0;
}

// ----------------------------------------------------------------------------------------------
// conv: the reference's Gaussian instrumental broadening (convolve_spectra_with_gauss,
// cmlib/mathtools.cc:1350-1414) of nvec Stokes spectra.  in.f64: lambda [n], then S [nvec][n][4];
// out.f64: the convolved S [nvec][n][4].
static int do_conv(const char *inname, int n, int nvec, double width, const char *outname) {
  std::vector<uint8_t> b = read_file_bytes(inname);
  const double *lam = (const double *)b.data(), *S = lam + n;
  fp_t *l1 = new fp_t[n] - 1;
  for (int l = 0; l < n; ++l) l1[l + 1] = lam[l];
  fp_t **T = ft2dim(1, 4, 1, n);
  std::vector<double> out((size_t)nvec * n * 4);
  for (int v = 0; v < nvec; ++v) {
    for (int l = 0; l < n; ++l)
      for (int s = 0; s < 4; ++s) T[s + 1][l + 1] = S[((size_t)v * n + l) * 4 + s];
    convolve_spectra_with_gauss(T, l1, n, width);
    for (int l = 0; l < n; ++l)
      for (int s = 0; s < 4; ++s) out[((size_t)v * n + l) * 4 + s] = T[s + 1][l + 1];
  }
  FILE *f = fopen(outname, "wb");
  fwrite(out.data(), 8, out.size(), f);
  fclose(f);
  del_ft2dim(T, 1, 4, 1, n);
  delete[] (l1 + 1);
  return 0;
}

// ----------------------------------------------------------------------------------------------
// eos: the data atmos_pp::build_from_nodes needs (atoms with their partition functions, levels
// and bound-free cross-sections at the wavelengths the build uses; molecules; the line <-> level
// ties; the node model), read from the reference's own objects after it parsed its configs; the
// reference's chemistry on a (T, Nt) grid (chemeq + lte + opacity_continuum, atmos_chm.cc:28-371,
// atom.cc:779-787, atmos_rad.cc:286-294); and, per node vector, the column build_from_nodes leaves
// (T, Nt, n_e, kappa at lambda_referent, rho).  Array layout: see tests/golden/make_golden.py.
static const int EMS = 12, EMT = 8, EMC = 8, EML = 16;

static int do_eos(const char *tskname, const char *nodesname, int npix, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  Task t = load_task(tskname);
  model *m = task_model(t, io);
  atmosphere *a = task_atmos(t, io);
  const int nl = t.nlambda;
  fp_t *lv = airtovac((fp_t *)t.lambda.data(), nl) - 1;   // 1-based vacuum grid
  const double lam_he = lambda_referent, lam_kap = airtovac(lambda_referent);

  std::vector<atom *> atoms;
  std::vector<mol *> mols;
  for (int i = 0; i < a->natm; ++i) {
    if (atom *at = dynamic_cast<atom *>(a->atml[i])) atoms.push_back(at);
    else if (mol *mo = dynamic_cast<mol *>(a->atml[i])) mols.push_back(mo);
  }
  const int na = atoms.size(), nm = mols.size();
  std::vector<double> atom_f(na * 4), atom_ip(na * EMS, 0.0);
  std::vector<double> pf_type(na * EMS, 0.0), pf_value(na * EMS, 0.0), pf_zeff(na * EMS, 0.0),
      pf_g0(na * EMS, 0.0), pf_nterm(na * EMS, 0.0), pf_ncoef(na * EMS, 0.0), pf_m(na * EMS * EMT, 0.0),
      pf_g2(na * EMS * EMT, 0.0), pf_ee(na * EMS * EMT, 0.0), pf_ll(na * EMS * EMT, 0.0),
      pf_a(na * EMS * EMT * EMC, 0.0), pf_gam(na * EMS * EMT * EMC, 0.0), pf_coef(na * EMS * EMC, 0.0);
  std::vector<double> lev_n(na * EMS, 0.0), lev(na * EMS * EML * 6, 0.0);
  for (int ia = 0; ia < na; ++ia) {
    atom *at = atoms[ia];
    if (at->Z + 1 > EMS) { fprintf(stderr, "too many stages\n"); return 2; }
    atom_f[ia * 4 + 0] = at->abund; atom_f[ia * 4 + 1] = at->Z + 1;
    atom_f[ia * 4 + 2] = at->check_if_nlte(); atom_f[ia * 4 + 3] = at->mass;
    for (int z = 0; z <= at->Z; ++z) {
      int s = ia * EMS + z;
      if (z < at->Z) atom_ip[s] = at->ip[z];
      // partition function data, read back from the object's own wire format (pf::pack and the
      // trav / irwin / cpf packers, partf.cc:56-63, 88-94, 170-187, 323-332)
      pf *P = at->partf[z];
      std::vector<uint8_t> pb(P->size(io) + 64);
      P->pack(pb.data(), 0, io);
      Rd r{pb.data()};
      int type = r.i8();
      pf_type[s] = type;
      if (type == PF_TYPE_CONST) pf_value[s] = r.f64();
      if (type == PF_TYPE_TRAV) {
        pf_zeff[s] = r.f64(); pf_g0[s] = r.f64();
        int n = r.i32();
        if (n > EMT) { fprintf(stderr, "too many partition terms: atom %d stage %d n %d\n", ia, z, n); return 2; }
        pf_nterm[s] = n;
        for (int i = 0; i < n; ++i) {
          pf_g2[s * EMT + i] = r.f64(); pf_ee[s * EMT + i] = r.f64(); pf_ll[s * EMT + i] = r.f64();
          int mm = r.i32();
          if (mm > EMC) { fprintf(stderr, "too many partition coefficients\n"); return 2; }
          pf_m[s * EMT + i] = mm;
          for (int l = 0; l < mm; ++l) pf_gam[(s * EMT + i) * EMC + l] = r.f64();
          for (int l = 0; l < mm; ++l) pf_a[(s * EMT + i) * EMC + l] = r.f64();
          r.i8();
        }
      }
      if (type == PF_TYPE_IRWIN) {
        pf_zeff[s] = r.f64();
        int n = r.i32();
        if (n > EMC) { fprintf(stderr, "too many Irwin coefficients\n"); return 2; }
        pf_ncoef[s] = n;
        for (int i = 0; i < n; ++i) pf_coef[s * EMC + i] = r.f64();
      }
      if (at->nl[z] > EML) { fprintf(stderr, "too many levels\n"); return 2; }
      lev_n[s] = at->nl[z];
      for (int l = 0; l < at->nl[z]; ++l) {
        double *L = &lev[(s * EML + l) * 6];
        L[0] = at->g[z][l]; L[1] = at->ee[z][l];
        bfcs *B = at->bf[z][l];
        if (B && z < at->Z) {
          L[2] = B->U(lam_he); L[3] = B->U(lam_kap);
          // atom::boundfree_op_em_vector (atom_rad_synthesis.cc:229-243): the window wavelength
          fp_t lc = B->getlambda_crit();
          int ncrit = 0;
          for (int q = 1; q <= nl; ++q) { if (lv[q] > lc) break; ++ncrit; }
          if (ncrit) { L[5] = lv[ncrit]; L[4] = B->U(lv[ncrit]); }
        }
      }
    }
  }
  std::vector<double> mol_i(nm * 11, 0.0), mol_coef(nm * EMC, 0.0);
  for (int im = 0; im < nm; ++im) {
    mol *mo = mols[im];
    int nc = 0;
    struct ion *cmp = mo->components(nc);
    if (nc > 4) { fprintf(stderr, "too many molecule components\n"); return 2; }
    mol_i[im * 11 + 0] = nc;
    for (int i = 0; i < nc; ++i) {
      int idx = -1;
      for (int ia = 0; ia < na; ++ia) if ((atmol *)atoms[ia] == cmp[i].atom) idx = ia;
      mol_i[im * 11 + 1 + i] = idx;
      mol_i[im * 11 + 5 + i] = cmp[i].z;
    }
    // equilibrium constant, read back from its wire format (moleqc.cc: eqc::pack, eqc_cnst::pack,
    // eqc_poly::pack)
    eqc *E = mo->K[0];
    std::vector<uint8_t> eb(E->size(io) + 64);
    E->pack(eb.data(), 0, io);
    Rd r{eb.data()};
    int type = r.u8();
    mol_i[im * 11 + 9] = type;
    if (type == EQC_TYPE_POLY) {
      int n = r.u8();
      if (n > EMC) { fprintf(stderr, "too many eqc coefficients\n"); return 2; }
      mol_i[im * 11 + 10] = n;
      for (int i = 0; i < n; ++i) mol_coef[im * EMC + i] = r.f64();
    }
    if (type == EQC_TYPE_CNST) { mol_i[im * 11 + 10] = 1; mol_coef[im * EMC] = r.f64(); }
  }
  // line <-> level ties, in the order atmosphere::op_em_vector meets the lines (A > 1)
  std::vector<double> line_eos;
  for (int ia = 0; ia < na; ++ia) {
    atom *at = atoms[ia];
    for (int z = 0; z <= at->Z; ++z)
      for (int up = 1; up < at->nl[z]; ++up)
        for (int lo = 0; lo < up; ++lo) {
          if (!(at->A[z][up][lo] > 1E0)) continue;
          double v[9] = {(double)ia, (double)z, (double)lo, (double)up, at->B[z][lo][up], at->B[z][up][lo],
                         at->A[z][up][lo], at->alpha_col_dam[z][up][lo], at->col_dam_cross_section[z][up][lo]};
          line_eos.insert(line_eos.end(), v, v + 9);
        }
  }
  const int nlines = line_eos.size() / 9;
  // node model
  const int np = m->get_N_nodes_total();
  std::vector<double> node_kind(np), node_tau(np);
  {
    int cnt[6] = {m->get_N_nodes_temp(), m->get_N_nodes_vt(), m->get_N_nodes_vs(), m->get_N_nodes_B(),
                  m->get_N_nodes_theta(), m->get_N_nodes_phi()};
    fp_t *tt[6] = {m->get_temp_nodes_tau(), m->get_vt_nodes_tau(), m->get_vs_nodes_tau(), m->get_B_nodes_tau(),
                   m->get_theta_nodes_tau(), m->get_phi_nodes_tau()};
    int p = 0;
    for (int kd = 0; kd < 6; ++kd)
      for (int i = 1; i <= cnt[kd]; ++i) {
        node_kind[p] = kd + 1; node_tau[p] = tt[kd][i]; ++p;
        if (m->which_parameter(p) != kd + 1) { fprintf(stderr, "node order\n"); return 2; }
      }
    for (int kd = 0; kd < 6; ++kd) if (cnt[kd]) delete[] (tt[kd] + 1);
  }
  const int nd = a->x3h - a->x3l + 1;
  double meta[13] = {(double)na, (double)nm, (double)nlines, (double)np, (double)nd, m->get_tau_min(),
                     m->get_tau_max(), t.el, t.az, lam_he, lam_kap, grav_acc, (double)nl};

  // the reference's chemistry on a (T, Nt) grid, stored in depth slot x3l
  const int nT = 14, nN = 12;
  std::vector<double> cT(nT), cN(nN), cne(nT * nN), cstage(nT * nN * na * EMS, 0.0),
      clev(nT * nN * na * EMS * EML, 0.0), ckhe(nT * nN), ckap(nT * nN);
  for (int i = 0; i < nT; ++i) cT[i] = 3400.0 * pow(20000.0 / 3400.0, i / (double)(nT - 1));
  for (int j = 0; j < nN; ++j) cN[j] = pow(10.0, 11.0 + 7.0 * j / (double)(nN - 1));
  a->popsetup();
  const int x = a->x3l;
  for (int i = 0; i < nT; ++i)
    for (int j = 0; j < nN; ++j) {
      fp_t ne = 1.0;
      a->chemeq(a->atml, a->natm, cT[i], cN[j], ne, 1, 1, x);
      for (int q = 0; q < a->natm; ++q) a->atml[q]->lte(cT[i], ne, 1, 1, x);
      int g = i * nN + j;
      cne[g] = ne;
      for (int ia = 0; ia < na; ++ia)
        for (int z = 0; z <= atoms[ia]->Z; ++z) {
          cstage[(g * na + ia) * EMS + z] = atoms[ia]->pop[1][1][x].N[z];
          for (int l = 0; l < atoms[ia]->nl[z]; ++l)
            clev[((g * na + ia) * EMS + z) * EML + l] = atoms[ia]->pop[1][1][x].n[z][l];
        }
      ckhe[g] = a->opacity_continuum(cT[i], ne, lam_he, 1, 1, x);
      ckap[g] = a->opacity_continuum(cT[i], ne, lam_kap, 1, 1, x);
    }
  a->popclean();
  delete a;

  // columns left by build_from_nodes
  std::vector<double> hT, hN, hne, hk, hr, harr;
  if (npix > 0) {
    std::vector<uint8_t> nb = read_file_bytes(nodesname);
    if ((int)(nb.size() / 8) < npix * np) { fprintf(stderr, "nodes file too short\n"); return 2; }
    const double *nodes = (const double *)nb.data();
    for (int ip = 0; ip < npix; ++ip) {
      atmosphere *b = task_atmos(t, io);
      set_nodes(m, nodes + ip * np);
      b->build_from_nodes(m);
      for (int xx = b->x3l; xx <= b->x3h; ++xx) {
        hT.push_back(b->T[1][1][xx]); hN.push_back(b->Nt[1][1][xx]); hne.push_back(b->Ne[1][1][xx]);
        hk.push_back(b->op_referent[1][1][xx]); hr.push_back(b->rho[1][1][xx]);
      }
      // the column as the master collects it after stokes_lm_fit's final build_from_nodes and
      // forward evaluation (obs_stokes' set-up up to compute_op_referent; atmos_fit.cc:212-214,
      // atmos_obs.cc:22-28, job.cc:555-557)
      b->set_grid(b->tau_grid);
      b->popsetup();
      b->compute_op_referent();
      fp_t **arr = b->return_as_array();
      const int ndd = b->x3h - b->x3l + 1;
      for (int q = 1; q <= 12; ++q)
        for (int i = 1; i <= ndd; ++i) harr.push_back(arr[q][i]);
      del_ft2dim(arr, 1, 12, 1, ndd);
      delete b;
    }
  }

  SbinWriter w(outname);
  w.put("meta", {13}, meta);
  w.put("atom_f", {na, 4}, atom_f.data());
  w.put("atom_ip", {na, EMS}, atom_ip.data());
  w.put("pf_type", {na, EMS}, pf_type.data());
  w.put("pf_value", {na, EMS}, pf_value.data());
  w.put("pf_zeff", {na, EMS}, pf_zeff.data());
  w.put("pf_g0", {na, EMS}, pf_g0.data());
  w.put("pf_nterm", {na, EMS}, pf_nterm.data());
  w.put("pf_m", {na, EMS, EMT}, pf_m.data());
  w.put("pf_g2", {na, EMS, EMT}, pf_g2.data());
  w.put("pf_ee", {na, EMS, EMT}, pf_ee.data());
  w.put("pf_ll", {na, EMS, EMT}, pf_ll.data());
  w.put("pf_a", {na, EMS, EMT, EMC}, pf_a.data());
  w.put("pf_gam", {na, EMS, EMT, EMC}, pf_gam.data());
  w.put("pf_ncoef", {na, EMS}, pf_ncoef.data());
  w.put("pf_coef", {na, EMS, EMC}, pf_coef.data());
  w.put("lev_n", {na, EMS}, lev_n.data());
  w.put("lev", {na, EMS, EML, 6}, lev.data());
  w.put("mol_i", {nm, 11}, mol_i.data());
  w.put("mol_coef", {nm, EMC}, mol_coef.data());
  w.put("line_eos", {nlines, 9}, line_eos.data());
  w.put("node_kind", {np}, node_kind.data());
  w.put("node_tau", {np}, node_tau.data());
  w.put("chem_T", {nT}, cT.data());
  w.put("chem_Nt", {nN}, cN.data());
  w.put("chem_ne", {nT, nN}, cne.data());
  w.put("chem_stage", {nT, nN, na, EMS}, cstage.data());
  w.put("chem_lev", {nT, nN, na, EMS, EML}, clev.data());
  w.put("chem_kap_he", {nT, nN}, ckhe.data());
  w.put("chem_kap", {nT, nN}, ckap.data());
  if (npix > 0) {
    w.put("he_T", {npix, nd}, hT.data());
    w.put("he_Nt", {npix, nd}, hN.data());
    w.put("he_ne", {npix, nd}, hne.data());
    w.put("he_kap", {npix, nd}, hk.data());
    w.put("he_rho", {npix, nd}, hr.data());
    w.put("atm_arr", {npix, 12, nd}, harr.data());
  }
  delete[] (lv + 1);
  delete m;
  return 0;
}

// ----------------------------------------------------------------------------------------------
// spinor: the synthesis branch of the master's job on an atmosphere cube (job.cc:384-409): the
// cube (12 return_as_array rows, dims (nd, ny, nx, 12)) read by atmosphere::read_spinor3d
// (atmos_fio.cc:79-124), each column extracted and synthesised (obs_stokes); dumps the column
// records (as extract_record reads them) and the Stokes vectors, x major.
static int do_spinor(const char *tskname, const char *cubename, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  Task t = load_task(tskname);
  atmosphere *a = task_atmos(t, io);
  char wd[4096];
  if (!getcwd(wd, sizeof wd)) return 2;
  if (a->read_spinor3d(wd, cubename, &io) < 0) return 3;
  const int nx = a->x1h - a->x1l + 1, ny = a->x2h - a->x2l + 1, nl = t.nlambda;
  fp_t *lam1 = lambda_1based(t);
  std::vector<int> probe_l;
  std::vector<double> allrec, allstokes;
  int nd = 0, nf = 0;
  for (int x = 1; x <= nx; ++x)
    for (int y = 1; y <= ny; ++y) {
      atmosphere *col = a->extract(x, y, io);
      Record r;
      extract_record(col, t, r, 0, probe_l);
      nd = r.nd;
      nf = NFIELD + 3 * r.nlines;
      std::vector<double> fl = record_flat(r);
      allrec.insert(allrec.end(), fl.begin(), fl.end());
      observable *o = col->obs_stokes(t.el, t.az, lam1, nl);
      fp_t **S = o->get_S(1, 1);
      for (int l = 1; l <= nl; ++l) for (int s = 1; s <= 4; ++s) allstokes.push_back(S[s][l]);
      del_ft2dim(S, 1, 4, 1, nl);
      delete o;
      delete col;
    }
  SbinWriter w(outname);
  w.put("record", {nx * ny, nd, nf}, allrec.data());
  w.put("stokes", {nx * ny, nl, 4}, allstokes.data());
  delete[] (lam1 + 1);
  delete a;
  return 0;
}

// ----------------------------------------------------------------------------------------------
// ANA .f0 files and the cube steps of the master's job (cmlib/ana_read.cc, cmlib/ana_write.cc,
// cmlib/fileio.cc, master/job.cc:306-334, 575-597).  Dump format of f0read (little endian):
//   int32 mfbd_type; int32 nd; int32 dims[nd]; int32 hlen; char header[hlen]; int64 nbytes; data
#include "fileio.h"
#include "ana_io.h"
#include "obs.h"

static void put_i32(FILE *f, int32_t v) { fwrite(&v, 4, 1, f); }

// ana_fzread of one file; the data as the reader returns it (native byte order)
static int do_f0read(const char *inname, const char *outname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  int *ds = 0, nd = 0, type = -1;
  char *header = 0;
  byte *data = ana_fzread((char *)inname, ds, nd, header, type, io);
  if (!data) return 3;
  int sz[] = MFBD_TYPE_SIZES;
  int64_t n = 1;
  for (int d = 1; d <= nd; ++d) n *= ds[d];
  FILE *f = fopen(outname, "wb");
  put_i32(f, type); put_i32(f, nd);
  for (int d = 1; d <= nd; ++d) put_i32(f, ds[d]);
  int32_t hl = (int32_t)strlen(header);
  put_i32(f, hl); fwrite(header, 1, hl, f);
  int64_t nb = n * sz[type];
  fwrite(&nb, 8, 1, f); fwrite(data, 1, nb, f);
  fclose(f);
  delete[] data; delete[] header; delete[] (ds + 1);
  return 0;
}

// ana_fzwrite of raw data: type (ANA code), dims (comma separated, fastest first), header file
// ("-" for none), data file
static int do_f0write(const char *outname, int type, const char *dims, const char *hdrname,
                      const char *dataname) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  std::vector<int> dv;
  for (const char *p = dims; *p;) { dv.push_back(atoi(p)); while (*p && *p != ',') ++p; if (*p) ++p; }
  int nd = (int)dv.size();
  int *ds = new int[nd] - 1;
  for (int d = 1; d <= nd; ++d) ds[d] = dv[d - 1];
  std::vector<uint8_t> hb, db = read_file_bytes(dataname);
  char *header = 0;
  if (strcmp(hdrname, "-")) {
    hb = read_file_bytes(hdrname); hb.push_back(0);
    header = (char *)hb.data();
  }
  ana_fzwrite(db.data(), (char *)outname, ds, nd, header, type, io);
  delete[] (ds + 1);
  return 0;
}

// The observed-cube steps of job.cc:306-334: read_file (4-D) + transpose + observable::set +
// normalize (synth_qs / obs_qs) + extract(xl..xh, yl..yh, ll..lh); dumps the extracted S as
// float64 [x][y][s][l] after a header int32 nx, ny, ns, nl, and writes it as cube_to_invert.f0
// is written (write_file 4-D, job.cc:333-334) to cubename
static int do_cubeobs(const char *inname, int xl, int xh, int yl, int yh, int ll, int lh, double obs_qs,
                      double synth_qs, const char *outname, const char *cubename) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  int n1, n2, n3, n4;
  fp_t ****test = read_file((char *)inname, n1, n2, n3, n4, io);
  if (!test) return 3;
  test = transpose(test, n1, n2, n3, n4);
  observable *obs = new observable(n4, n3, n2, n1);
  obs->set(test);
  del_ft4dim(test, 1, n4, 1, n3, 1, n2, 1, n1);
  obs->set_inv_parameters(0.0, 0.0, obs_qs, synth_qs);
  obs->normalize();
  observable *o2 = obs->extract(xl, xh, yl, yh, ll, lh);
  delete obs;
  int nx = xh - xl + 1, ny = yh - yl + 1, nl = lh - ll + 1;
  fp_t ****S = o2->get_S();
  FILE *f = fopen(outname, "wb");
  put_i32(f, nx); put_i32(f, ny); put_i32(f, n2); put_i32(f, nl);
  fwrite(S[1][1][1] + 1, sizeof(fp_t), (size_t)nx * ny * n2 * nl, f);
  fclose(f);
  write_file((char *)cubename, S, nx, ny, 4, nl, io);
  del_ft4dim(S, 1, nx, 1, ny, 1, n2, 1, nl);
  delete o2;
  return 0;
}

// The output steps of job.cc:575-597: write_file of the node cube (fp_t [x][y][p], 3-D overload)
// and of the fitted spectra (fp_t [x][y][s][l], 4-D overload), from raw float64 inputs
static int do_cubewrite(const char *nodesname, const char *specname, int nx, int ny, int np, int nl,
                        const char *out_nodes, const char *out_spec) {
  const char *argv[] = {"snapi_ref_dump", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4; cmdln cmd(ac, (char **)argv, options, maps);
  io_class io(cmd);
  std::vector<uint8_t> nb = read_file_bytes(nodesname), sb = read_file_bytes(specname);
  fp_t ***nc = ft3dim(1, nx, 1, ny, 1, np);
  memcpy(nc[1][1] + 1, nb.data(), (size_t)nx * ny * np * sizeof(fp_t));
  write_file((char *)out_nodes, nc, nx, ny, np, io);
  del_ft3dim(nc, 1, nx, 1, ny, 1, np);
  fp_t ****sc = ft4dim(1, nx, 1, ny, 1, 4, 1, nl);
  memcpy(sc[1][1][1] + 1, sb.data(), (size_t)nx * ny * 4 * nl * sizeof(fp_t));
  write_file((char *)out_spec, sc, nx, ny, 4, nl, io);
  del_ft4dim(sc, 1, nx, 1, ny, 1, 4, 1, nl);
  return 0;
}

int main(int argc, char **argv) {
  if (argc >= 6 && !strcmp(argv[1], "eos")) return do_eos(argv[2], argv[3], atoi(argv[4]), argv[5]);
  if (argc >= 4 && !strcmp(argv[1], "pack")) return do_pack(argv[2], argv[3]);
  if (argc >= 7 && !strcmp(argv[1], "dump"))
    return do_dump(argv[2], argv[3], atoi(argv[4]), atoi(argv[5]), argv[6]);
  if (argc >= 7 && !strcmp(argv[1], "conv"))
    return do_conv(argv[2], atoi(argv[3]), atoi(argv[4]), atof(argv[5]), argv[6]);
  if (argc >= 7 && !strcmp(argv[1], "ali"))
    return do_ali(argv[2], argv[3], atoi(argv[4]), atoi(argv[5]), argv[6]);
  if (argc >= 6 && !strcmp(argv[1], "alisetup")) return do_alisetup(argv[2], argv[3], atoi(argv[4]), argv[5]);
  if (argc >= 9 && !strcmp(argv[1], "lmfit"))
    return do_lmfit(argv[2], argv[3], argv[4], argv[5], atoi(argv[6]), atoi(argv[7]), argv[8],
                    argc >= 10 ? atof(argv[9]) : 0.0);
  if (argc >= 4 && !strcmp(argv[1], "f0read")) return do_f0read(argv[2], argv[3]);
  if (argc >= 5 && !strcmp(argv[1], "spinor")) return do_spinor(argv[2], argv[3], argv[4]);
  if (argc >= 7 && !strcmp(argv[1], "f0write"))
    return do_f0write(argv[2], atoi(argv[3]), argv[4], argv[5], argv[6]);
  if (argc >= 13 && !strcmp(argv[1], "cubeobs"))
    return do_cubeobs(argv[2], atoi(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]), atoi(argv[7]),
                      atoi(argv[8]), atof(argv[9]), atof(argv[10]), argv[11], argv[12]);
  if (argc >= 10 && !strcmp(argv[1], "cubewrite"))
    return do_cubewrite(argv[2], argv[3], atoi(argv[4]), atoi(argv[5]), atoi(argv[6]), atoi(argv[7]), argv[8],
                        argv[9]);
  fprintf(stderr, "usage: snapi_ref_dump pack|dump|lmfit ...\n");
  return 1;
}
