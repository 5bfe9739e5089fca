/* diskoracle — plain-C restatement of the reference diskfft time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the CPU oracle the GPU library is checked
 * against; it is never linked into, loaded by, or called from the product path.
 * Each function cites the reference lines it restates (paths relative to the
 * oklo/heavy-disks project root).  Parity with the reference itself is pinned by
 * tests that compare this restatement against the reference's own sources compiled
 * unmodified (oracle/_ref) and against committed golden vectors. */
#ifndef DISKORACLE_H
#define DISKORACLE_H
#include <stdio.h>
#ifdef __cplusplus
extern "C" {
#endif

/* DiskHydro (diskfft/src/hydro.hpp:20-43) */
typedef struct {
  int Nu, Nphi;
  double umin, umax, du, dphi, Kpoly, gamma_gas, gmstar;
  double *R, *Rf, *Vol;
  double *Sig, *vR, *vp;
  double *wA, *wB, *mR, *mp, *Fm, *FmR, *FmP;
  int nthreads;
} orc_hydro;

/* KalnajsSolver (diskfft/src/kalnajs.hpp:19-42) */
typedef struct {
  int Nu, Nphi, M, Nc;
  double umin, umax, du, dphi, eps, G;
  double *R, *sqrtR, *R32;
  double *rbuf, *cbuf, *Khat; /* rbuf M*Nphi real; cbuf, Khat M*Nc complex interleaved */
  int nthreads;
} orc_kalnajs;

/* diskdisk parameters (diskfft/src/diskmain.cpp:17-29); phase0 = 0 is the reference seed. */
typedef struct {
  int Nu, Nphi;
  double eps, tlim;
  int selfgrav;
  double amp;
  int nthreads;
  double Rin, Rout, R0, w2, S0, Kpoly, gamma_gas, gmstar, G;
  double phase0;
} orc_params;

orc_hydro *orc_hydro_create(int Nu, int Nphi, double Rin, double Rout, double K, double g, double GMstar);
void orc_hydro_destroy(orc_hydro *h);
double *orc_hydro_field(orc_hydro *h, int which); /* 0 Sig 1 vR 2 vp 3 R 4 Rf 5 Vol */
void orc_set_threads(orc_hydro *h, int nthreads);
double orc_timestep(const orc_hydro *h, double cfl);
void orc_source(orc_hydro *h, double dt, const double *gR, const double *gp);
void orc_transportR(orc_hydro *h, double dt);
void orc_transportPhi(orc_hydro *h, double dt);
void orc_step(orc_hydro *h, double dt, const double *gR, const double *gp);

orc_kalnajs *orc_kalnajs_create(int Nu, int Nphi, double Rin, double Rout, double eps, double G, int nthreads);
void orc_kalnajs_destroy(orc_kalnajs *k);
void orc_potential(orc_kalnajs *k, const double *Sig, double *Phi);
void orc_forces(const orc_kalnajs *k, const double *Phi, double *gR, double *gp);
void orc_potential_direct(const orc_kalnajs *k, const double *Sig, double *Phi);
const double *orc_khat(const orc_kalnajs *k);

void orc_params_default(orc_params *p);
/* equilibrium + seed (diskmain.cpp:34-63); fills h->Sig, vR, vp */
void orc_init_standard(const orc_params *p, orc_hydro *h, orc_kalnajs *k);
double orc_disk_mass(const orc_hydro *h);                                       /* diskmain.cpp:66-70 */
void orc_cm(const orc_hydro *h, int m, double mD, double *mag, double *phase);   /* diskmain.cpp:72-84 */
/* The time loop of diskmain.cpp:86-112.  Stops at tlim or after max_steps (< 0: no cap).
 * Writes the modes table to `modes` (may be NULL) in the reference's format. */
long orc_run(const orc_params *p, orc_hydro *h, orc_kalnajs *k, long max_steps, double *t_out, FILE *modes);

#ifdef __cplusplus
}
#endif
#endif
