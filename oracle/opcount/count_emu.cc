// Op-count build of the CPU emulator of the FP32 kernels (tests/emu/snapi_emu.cc, which compiles
// the kernels' per-cell code snapi_core.cuh / snapi_sweep.cuh for the host): the same source with
// float and double counted (opcount.hpp).  emu_synth counts the synthesis kernel's algorithm,
// emu_adjoint the adjoint call's (forward with state, reverse sweep, opacity adjoint, chain rule).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "opcount.hpp"

opc::Counts opc::c32, opc::c64;

#define float OpcF
#define double OpcD
#include "../../tests/emu/snapi_emu.cc"
#undef float
#undef double

extern "C" void opc_reset(void) { opc::c32.reset(); opc::c64.reset(); }
extern "C" void opc_get(long long *out /*[2][8]*/) {
  const opc::Counts *c[2] = {&opc::c32, &opc::c64};
  for (int k = 0; k < 2; ++k) {
    long long v[8] = {c[k]->add, c[k]->mul, c[k]->div, c[k]->fma, c[k]->sqrt, c[k]->exp, c[k]->trig, c[k]->flops()};
    for (int i = 0; i < 8; ++i) out[k * 8 + i] = v[i];
  }
}
