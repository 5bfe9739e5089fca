// Internal definition of dg_handle: one disk on one device (not part of the C ABI).
#pragma once

#include <string>
#include <vector>

#include "diskgpu.h"
#include "kernels.h"

struct MixedState;  // mixed.cu
struct MixedGroup;  // mixed.cu: disks of a batched sweep stepped by one launch per kernel
struct dg_handle;
// Grouping key of a disk ("" when it cannot join a group; 1024^2 disks, whose fused
// transforms have group forms, only with with_fused), group set-up, one step of the whole
// group on a stream, and release.
std::string mixed_group_key(const dg_handle *h, bool with_fused = true);
MixedGroup *mixed_group_create(const std::vector<dg_handle *> &disks, std::string *err);
int mixed_group_enqueue_step(MixedGroup *g, cudaStream_t st);
void mixed_group_destroy(MixedGroup *g);

struct dg_handle {
  static constexpr int kGraphSteps = 64;  // steps per captured CUDA graph (even)

  dg_params p{};
  int dev = -1;
  cudaStream_t st = nullptr;      // stream all work is queued on
  cudaStream_t own_st = nullptr;  // the handle's own stream
  std::string err;
  bool use_graphs = true;

  // grid (FP64, hydro.hpp:31-38, kalnajs.hpp:28-34)
  double umin = 0, umax = 0, du = 0, dphi = 0;
  int M = 0, Nc = 0;
  std::vector<double> R, Rf, Vol, sqrtR, R32;
  double *dR = nullptr, *dRf = nullptr, *dVol = nullptr, *dSqrtR = nullptr, *dR32 = nullptr;
  double *rowtab = nullptr;  // per-row / per-face constants of the FP64 hydro kernel
  dg::Geom64 geom{};

  // plain-method state (ping-pong), forces scratch, gravity workspace
  double *S[2] = {nullptr, nullptr}, *VR[2] = {nullptr, nullptr}, *VP[2] = {nullptr, nullptr};
  int cur = 0;
  double *dPhi = nullptr, *gA = nullptr, *gB = nullptr;
  double2 *W = nullptr, *Khat = nullptr, *rootsPhi = nullptr, *rootsM = nullptr;
  dg::FftPlan plPhi{}, plM{};
  double *scratch = nullptr;  // 64 doubles of reduction output

  // control block (device) and a pinned host mirror
  dg::Ctl *ctl = nullptr, *hctl = nullptr;
  cudaGraphExec_t graph_exec = nullptr;

  bool have_state = false;
  double mD = 0.0, t = 0.0, tnext = 0.0;
  long long nsteps = 0;

  // basic state handed over by dg_init_standard (used by the mixed path)
  bool basic_from_standard = false;
  std::vector<double> std_sigma0, std_vphi0, std_gR0;

  MixedState *mx = nullptr;

  // free-running device loop (dg_run_steps): t and step live on the device
  bool freerun = false;
  double freerun_cfl = 0.0;
  double *hdt = nullptr;  // pinned dt readback

  // per-phase event timing
  bool prof_on = false;
  std::vector<cudaEvent_t> ev_pool;
  int ev_used = 0;
  std::vector<std::pair<int, int>> prof_pending;
  double prof_ms[DG_PROF_N] = {};
  long long prof_count[DG_PROF_N] = {};
  cudaError_t prof_begin(int phase);
  cudaError_t prof_end(int phase);
  int prof_collect();
  int sync_from_device();

  int fail(int code, const char *what, const char *why);
  int init(const dg_params &pp);
  int build_khat();
  void release();
  int potential64(const double *dSig, double *dOut);
  int enqueue_step();
  int enqueue_step_forces(const double *gR, const double *gp);
  int set_ctl_fields(double t, double tlim, double cfl, double dt, double tnext, double dtout, int fixed_dt);
  int read_ctl();
  int check_status();
  int cfl_launch(int nmodes, int record);
  int modes_launch(int nmodes, double *out);
  int conserved_launch(double *out2);
  int run_chunk(int nsteps);
  int capture_graph();
  // host-side state of the enqueued step sequence (the mixed path's row-tile hand-over)
  int graph_end_flags = 0;
  int loop_flags() const;
  void set_loop_flags(int f);
  int upload_state(const double *Sig, const double *vR, const double *vp);
  int download_state(double *Sig, double *vR, double *vp);

  // mixed-precision path (mixed.cu)
  int mixed_init();
  void mixed_release();
  int mixed_enqueue_step();
  int mixed_enqueue_step_forces(const double *gR, const double *gp);
  int mixed_cfl_launch(int nmodes, int record);
  int mixed_modes_launch(int nmodes, double *out);
  int mixed_conserved_launch(double *out2);
  int mixed_upload_state(const double *Sig, const double *vR, const double *vp);
  int mixed_download_state(double *Sig, double *vR, double *vp);
  int mixed_gravity();
  int mixed_gravity_kernels() const;
  int mixed_hydro_kernels() const;
  int mixed_autotune();
  std::string mixed_tuning_info() const;
  int mixed_potential(const double *dSig, double *dOut);
  bool in_step_host = false;  // upload from dg_step_host keeps the mixed basic state
  void mixed_basic(std::vector<double> *S0, std::vector<double> *V0, std::vector<double> *g0) const;

  // per-step diagnostic ring (dg_set_diagnostics)
  double *diag = nullptr;
  int diag_mmax = 0;
  void graph_reset() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
  }
};
