// Timing driver over the compiled reference, built with the reference's own flags
// (-O3 -ffast-math, oracle/Makefile "fast").  Test / baseline infrastructure only.
//
//   snapi_ref_bench <task.tsk> <nodes.f64> <first> <count> <mode>
//
// For pixels first..first+count-1 of the node file: build_from_nodes, then
//   mode 0: atmosphere::obs_stokes                        (synthesis)
//   mode 1: atmosphere::obs_stokes_responses_to_nodes     (synthesis + node responses, the
//           quantity stokes_lm_fit builds its gradient J^T r from)
//   mode 2: atmosphere::obs_stokes_num_responses_to_nodes (synthesis + plain central FD)
// Prints one line "pixels <count> seconds <wall> checksum <sum of I>" on stdout.
#include "ref_common.h"

int main(int argc, char **argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: snapi_ref_bench task.tsk nodes.f64 first count mode\n");
    return 1;
  }
  const char *argv_io[] = {"snapi_ref_bench", "-q", "-q", "-q", 0};
  const char *options[] = CMDOPTS, *maps[] = CMDMAPS;
  int ac = 4;
  cmdln cmd(ac, (char **)argv_io, options, maps);
  io_class io(cmd);
  Task t = load_task(argv[1]);
  std::vector<uint8_t> nb = read_file_bytes(argv[2]);
  const double *nodes = (const double *)nb.data();
  const int first = atoi(argv[3]), count = atoi(argv[4]), mode = atoi(argv[5]);
  model *m = task_model(t, io);
  const int np = m->get_N_nodes_total(), nl = t.nlambda;
  if ((int)(nb.size() / 8) < (first + count) * np) {
    fprintf(stderr, "node file too short\n");
    return 2;
  }
  fp_t *lam1 = lambda_1based(t);
  double checksum = 0.0;
  const double t0 = wall_s();
  for (int ip = first; ip < first + count; ++ip) {
    atmosphere *a = task_atmos(t, io);
    fp_t *p = new fp_t[np] - 1;
    for (int i = 0; i < np; ++i) p[i + 1] = nodes[ip * np + i];
    m->set_parameters(p);
    delete[] (p + 1);
    a->build_from_nodes(m);
    observable *o = 0;
    fp_t ***resp = 0;
    if (mode == 0) {
      o = a->obs_stokes(t.el, t.az, lam1, nl);
    } else {
      resp = ft3dim(1, np, 1, nl, 1, 4);
      if (mode == 1)
        o = a->obs_stokes_responses_to_nodes(m, t.el, t.az, lam1, nl, resp, 0);
      else
        o = a->obs_stokes_num_responses_to_nodes(m, t.el, t.az, lam1, nl, resp, 0);
    }
    fp_t **S = o->get_S(1, 1);
    for (int l = 1; l <= nl; ++l) checksum += S[1][l];
    del_ft2dim(S, 1, 4, 1, nl);
    if (resp) del_ft3dim(resp, 1, np, 1, nl, 1, 4);
    delete o;
    delete a;
  }
  const double dt = wall_s() - t0;
  printf("pixels %d seconds %.6f checksum %.10e\n", count, dt, checksum);
  delete m;
  delete[] (lam1 + 1);
  return 0;
}
