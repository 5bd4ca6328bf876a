// Op-count build of the FP64 node -> record restatement oracle/eos_oracle.c (test infrastructure):
// the same source with `double` counted (opcount.hpp).  Exported with the oracle's C interface
// (sne_build, sne_set_chem_start); double arrays pass for OpcD arrays (same layout).
#include <math.h>
#include <stddef.h>
#include <string.h>

#include "opcount.hpp"
#include "../../include/snapi_cuda.h"

opc::Counts opc::c32, opc::c64;

#define double OpcD
extern "C" {
#include "../eos_oracle.c"
}
#undef double

extern "C" void opc_reset(void) { opc::c32.reset(); opc::c64.reset(); }
extern "C" void opc_get(long long *out /*[2][8]*/) {
  const opc::Counts *c[2] = {&opc::c32, &opc::c64};
  for (int k = 0; k < 2; ++k) {
    long long v[8] = {c[k]->add, c[k]->mul, c[k]->div, c[k]->fma, c[k]->sqrt, c[k]->exp, c[k]->trig, c[k]->flops()};
    for (int i = 0; i < 8; ++i) out[k * 8 + i] = v[i];
  }
}
