// diskdisk — drop-in replacement for the reference driver (diskfft/src/diskmain.cpp)
// running the time step on a B200 through the diskgpu C ABI.
//
//   ./diskdisk Nu Nphi eps tlim selfgrav amp nthreads [--precision fp64|mixed]
//              [--phase PHI0] [--device N] [--fit]
//
// Positional arguments, defaults and outputs are those of diskmain.cpp:17-23,86-112:
// diskfft_modes.dat with "# t  |C0|  |C2|  arg(C2)" and rows "%.5f %.6e %.6e %.6e" every
// 0.25 time units, the same lines on stdout, and the final summary line.  Each record is
// printed, written and flushed as soon as the device loop hands it over (dg_advance_cb),
// as diskmain.cpp:93-98 does, so a long or failed run keeps the records it made.  nthreads
// is accepted for compatibility (the step runs on the GPU).  --fit adds the growth fit of
// the records (dg_fit_phases) on stderr, leaving stdout and the modes file as the
// reference writes them.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "diskgpu.h"

struct Out {
  FILE *fp;
  std::vector<dg_record> all;
};

static void on_record(const dg_record *r, void *user) {
  Out *o = static_cast<Out *>(user);
  printf("t=%7.3f  |C0|=%.5f  |C2|=%.6e\n", r->t, r->c0, r->c2);
  fprintf(o->fp, "%.5f %.6e %.6e %.6e\n", r->t, r->c0, r->c2, r->arg2);
  fflush(stdout);
  fflush(o->fp);
  o->all.push_back(*r);
}

static int die(dg_handle *h, int rc, const char *what) {
  fprintf(stderr, "diskdisk: %s failed: %s (%s)\n", what, dg_status_string(rc), dg_last_error(h));
  dg_destroy(h);
  return 1;
}

int main(int argc, char **argv) {
  std::vector<const char *> pos;
  const char *prec = "fp64";
  double phase0 = 0.0;
  int device = -1;
  bool fit = false;
  for (int a = 1; a < argc; ++a) {
    if (!strcmp(argv[a], "--fit")) fit = true;
    else if (!strcmp(argv[a], "--precision") && a + 1 < argc) prec = argv[++a];
    else if (!strcmp(argv[a], "--phase") && a + 1 < argc) phase0 = atof(argv[++a]);
    else if (!strcmp(argv[a], "--device") && a + 1 < argc) device = atoi(argv[++a]);
    else pos.push_back(argv[a]);
  }
  const int np = (int)pos.size();
  dg_params p;
  dg_params_default(&p);
  p.Nu = (np > 0) ? atoi(pos[0]) : 128;
  p.Nphi = (np > 1) ? atoi(pos[1]) : 128;
  p.eps = (np > 2) ? atof(pos[2]) : 0.02;
  double tlim = (np > 3) ? atof(pos[3]) : 8.0;
  p.selfgrav = (np > 4) ? atoi(pos[4]) : 1;
  p.amp = (np > 5) ? atof(pos[5]) : 1e-3;
  int nthreads = (np > 6) ? atoi(pos[6]) : 1;  // accepted; the step runs on the GPU
  (void)nthreads;
  p.phase0 = phase0;
  p.device = device;
  if (!strcmp(prec, "mixed")) p.precision = DG_PREC_MIXED;
  else if (strcmp(prec, "fp64")) { fprintf(stderr, "diskdisk: --precision must be fp64 or mixed\n"); return 2; }

  dg_handle *h = nullptr;
  int rc = dg_create(&p, &h);
  if (rc) { fprintf(stderr, "diskdisk: create failed: %s (%s)\n", dg_status_string(rc), dg_last_error(nullptr)); return 1; }
  rc = dg_init_standard(h);
  if (rc) return die(h, rc, "init");

  const double dtout = 0.25;
  FILE *fp = fopen("diskfft_modes.dat", "w");
  if (!fp) { perror("diskfft_modes.dat"); dg_destroy(h); return 1; }
  fprintf(fp, "# t  |C0|  |C2|  arg(C2)\n");
  Out out{fp, {}};
  double t = 0.0;
  long long steps = 0;
  rc = dg_advance_cb(h, tlim, 0.3, dtout, on_record, &out, nullptr, &t, &steps);
  if (rc) { fclose(fp); return die(h, rc, "advance"); }
  double m[6];
  rc = dg_modes(h, 2, m);
  if (rc) { fclose(fp); return die(h, rc, "modes"); }
  double c2 = std::sqrt(m[4] * m[4] + m[5] * m[5]);
  printf("final t=%.3f  |C2|=%.6e  steps=%d\n", t, c2, (int)steps);
  fclose(fp);
  if (fit) {
    double f[6];
    if (dg_fit_phases(out.all.data(), (int)out.all.size(), 1.0, 0.05, 0.15, f) == DG_OK)
      fprintf(stderr, "fit: linear gamma=%.6f Omega_p=%.6f (%d records)  saturated |C2|/|C0|=%.6f Omega_p=%.6f (%d)\n",
              f[0], f[1], (int)f[2], f[3], f[4], (int)f[5]);
    else
      fprintf(stderr, "fit: %s\n", dg_last_error(nullptr));
  }
  dg_destroy(h);
  return 0;
}
