// Shared helpers of the oracle drivers that run the compiled reference (test infrastructure).
//
// The drivers follow the reference's own job flow (jsub set-up, then the islave calls):
//   jsub:   gcfg -> atmos_new(acfg) -> pack -> atmos_new(buf) -> init -> extract(1,1)
//   islave: atmos_new(buf) -> build_from_nodes / obs_stokes / obs_stokes_responses_to_nodes /
//           stokes_lm_fit
// A "task blob" holds one packed 1-column atmosphere, one packed model and the wavelength grid,
// i.e. the payload the master sends a slave (master/job.cc:354-379, slave/slave.cc:103-113).
//
// The column-record extraction reads the reference's protected members; the access
// specifiers are opened for this translation unit only (layout is unchanged).
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <unistd.h>
#include <stdint.h>
#include <vector>
#include <string>
#include <sys/time.h>

#define protected public
#define private public
#include "types.h"
#include "io.h"
#include "mem.h"
#include "pack.h"
#include "const.h"
#include "cmdln.h"
#include "mathtools.h"
#include "atmos.h"
#include "plpar/atmos_pp.h"
#include "plpar/atmos_ppbez.h"
#include "atmol/atmol.h"
#include "atom/atom.h"
#include "mol/mol.h"
#include "cfg.h"
#include "cmdcfg.h"
#undef protected
#undef private

static double wall_s() {
  struct timeval tv; gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static std::vector<uint8_t> read_file_bytes(const char *fn) {
  FILE *f = fopen(fn, "rb");
  if (!f) { fprintf(stderr, "cannot open %s\n", fn); exit(2); }
  fseek(f, 0, SEEK_END); long n = ftell(f); fseek(f, 0, SEEK_SET);
  std::vector<uint8_t> b(n);
  if (n && fread(b.data(), 1, n, f) != (size_t)n) { fprintf(stderr, "short read %s\n", fn); exit(2); }
  fclose(f);
  return b;
}

// Task blob layout (little endian, this driver's own container):
//   char magic[8] "SNAPITSK"; int32 nlambda; double el, az; double lambda_cm[nlambda];
//   int32 atm_size; bytes atm[atm_size]; int32 mod_size; bytes mod[mod_size]
struct Task {
  int nlambda = 0;
  double el = 0, az = 0;
  std::vector<double> lambda;  // air wavelengths in cm, 0-based
  std::vector<uint8_t> atm, mod;
};

static Task load_task(const char *fn) {
  std::vector<uint8_t> b = read_file_bytes(fn);
  Task t;
  size_t o = 0;
  if (b.size() < 8 || memcmp(b.data(), "SNAPITSK", 8)) { fprintf(stderr, "bad task blob\n"); exit(2); }
  o = 8;
  memcpy(&t.nlambda, &b[o], 4); o += 4;
  memcpy(&t.el, &b[o], 8); o += 8;
  memcpy(&t.az, &b[o], 8); o += 8;
  t.lambda.resize(t.nlambda);
  memcpy(t.lambda.data(), &b[o], 8 * t.nlambda); o += 8 * t.nlambda;
  int32_t n; memcpy(&n, &b[o], 4); o += 4;
  t.atm.assign(b.begin() + o, b.begin() + o + n); o += n;
  memcpy(&n, &b[o], 4); o += 4;
  t.mod.assign(b.begin() + o, b.begin() + o + n); o += n;
  return t;
}

static atmosphere *task_atmos(Task &t, io_class &io) {
  int32_t offs = 0;
  return atmos_new(t.atm.data(), offs, 0, io);
}

static model *task_model(Task &t, io_class &io) {
  int32_t offs = 0;
  return model_new(t.mod.data(), offs, 0, io);
}

// 1-based lambda copy, as the reference's observable::get_lambda returns it
static fp_t *lambda_1based(const Task &t) {
  fp_t *l = new fp_t[t.nlambda] - 1;
  for (int i = 0; i < t.nlambda; ++i) l[i + 1] = t.lambda[i];
  return l;
}
