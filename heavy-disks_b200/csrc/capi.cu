// C ABI of the diskgpu library (include/diskgpu.h): handle life cycle, state transfer,
// and the device-resident step loop.  The kernels live in kernels64.cu (plain FP64 path)
// and mixed*.cu (FP32 perturbation + tensor-core gravity).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "diskgpu.h"
#include "engine.h"

using namespace dg;

// ---------------------------------------------------------------------------------
// helpers

#define DG_CK(call)                                                                 \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return h->fail(DG_ERR_CUDA, #call, cudaGetErrorString(e_)); \
  } while (0)

// the same inside dg_handle member functions
#define MK(call)                                                                    \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) return fail(DG_ERR_CUDA, #call, cudaGetErrorString(e_)); \
  } while (0)

int dg_handle::fail(int code, const char *what, const char *why) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s", what, why ? why : "");
  err = buf;
  return code;
}

static std::vector<double2> roots_table(int n) {
  std::vector<double2> r(n);
  for (int t = 0; t < n; ++t) {
    long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)n;
    r[t].x = (double)cosl(a);
    r[t].y = (double)-sinl(a);
  }
  return r;
}

template <typename T>
static cudaError_t dmalloc(T **p, size_t n) {
  return cudaMalloc((void **)p, (n ? n : 1) * sizeof(T));
}

// ---------------------------------------------------------------------------------
// set-up

static int validate(const dg_params *p, std::string *why) {
  char b[256];
  if (p->Nu < 2 || p->Nphi < 2) { snprintf(b, sizeof b, "Nu=%d Nphi=%d: both must be >= 2", p->Nu, p->Nphi); *why = b; return DG_ERR_INVALID; }
  // one CTA holds a whole transform (<= 8192 points: 1024 threads x 8, 128 KiB of FP64 complex)
  if (p->Nu > 4096 || p->Nphi > 8192) { snprintf(b, sizeof b, "Nu=%d Nphi=%d exceeds 4096 x 8192", p->Nu, p->Nphi); *why = b; return DG_ERR_UNSUPPORTED; }
  if (!(p->Rin > 0) || !(p->Rout > p->Rin)) { *why = "need 0 < Rin < Rout"; return DG_ERR_INVALID; }
  if (!(p->Kpoly > 0) || !(p->gamma_gas > 0)) { *why = "need Kpoly > 0 and gamma_gas > 0"; return DG_ERR_INVALID; }
  if (!(p->eps >= 0) || !std::isfinite(p->eps)) { *why = "need eps >= 0"; return DG_ERR_INVALID; }
  if (p->precision != DG_PREC_FP64 && p->precision != DG_PREC_MIXED) { *why = "precision must be DG_PREC_FP64 or DG_PREC_MIXED"; return DG_ERR_INVALID; }
  if (p->basic_state != DG_BASIC_FFT && p->basic_state != DG_BASIC_ELLIPTIC) { *why = "basic_state must be DG_BASIC_FFT or DG_BASIC_ELLIPTIC"; return DG_ERR_INVALID; }
  FftPlan a, c;
  if (!make_fft_plan(p->Nphi, &a) || !make_fft_plan(2 * p->Nu, &c)) {
    snprintf(b, sizeof b, "Nphi=%d and 2*Nu=%d must factor into 2, 3 and 5", p->Nphi, 2 * p->Nu);
    *why = b;
    return DG_ERR_UNSUPPORTED;
  }
  return DG_OK;
}

int dg_handle::init(const dg_params &pp) {
  p = pp;
  if (p.device >= 0) MK(cudaSetDevice(p.device));
  MK(cudaGetDevice(&dev));
  MK(cudaStreamCreateWithFlags(&own_st, cudaStreamNonBlocking));
  st = own_st;
  const int Nu = p.Nu, Nphi = p.Nphi;
  // grid exactly as hydro.hpp:31-38 and kalnajs.hpp:28-34
  umin = std::log(p.Rin);
  umax = std::log(p.Rout);
  du = (umax - umin) / Nu;
  dphi = 2.0 * M_PI / Nphi;
  R.resize(Nu); Rf.resize(Nu + 1); Vol.resize(Nu); sqrtR.resize(Nu); R32.resize(Nu);
  for (int i = 0; i <= Nu; ++i) Rf[i] = std::exp(umin + i * du);
  for (int i = 0; i < Nu; ++i) {
    R[i] = std::exp(umin + (i + 0.5) * du);
    Vol[i] = R[i] * (Rf[i + 1] - Rf[i]) * dphi;
    sqrtR[i] = std::sqrt(R[i]);
    R32[i] = R[i] * sqrtR[i];
  }
  M = 2 * Nu;
  Nc = Nphi / 2 + 1;
  make_fft_plan(Nphi, &plPhi);
  make_fft_plan(M, &plM);
  const size_t n = (size_t)Nu * Nphi;
  MK(dmalloc(&dR, Nu)); MK(dmalloc(&dRf, Nu + 1)); MK(dmalloc(&dVol, Nu));
  MK(dmalloc(&dSqrtR, Nu)); MK(dmalloc(&dR32, Nu));
  MK(cudaMemcpy(dR, R.data(), Nu * sizeof(double), cudaMemcpyHostToDevice));
  MK(cudaMemcpy(dRf, Rf.data(), (Nu + 1) * sizeof(double), cudaMemcpyHostToDevice));
  MK(cudaMemcpy(dVol, Vol.data(), Nu * sizeof(double), cudaMemcpyHostToDevice));
  MK(cudaMemcpy(dSqrtR, sqrtR.data(), Nu * sizeof(double), cudaMemcpyHostToDevice));
  MK(cudaMemcpy(dR32, R32.data(), Nu * sizeof(double), cudaMemcpyHostToDevice));
  for (int b = 0; b < 2; ++b) {
    MK(dmalloc(&S[b], n)); MK(dmalloc(&VR[b], n)); MK(dmalloc(&VP[b], n));
    MK(cudaMemset(S[b], 0, n * sizeof(double)));
    MK(cudaMemset(VR[b], 0, n * sizeof(double)));
    MK(cudaMemset(VP[b], 0, n * sizeof(double)));
  }
  MK(dmalloc(&dPhi, n)); MK(dmalloc(&gA, n)); MK(dmalloc(&gB, n));
  MK(dmalloc(&W, (size_t)Nc * M)); MK(dmalloc(&Khat, (size_t)Nc * M));
  std::vector<double2> r1 = roots_table(Nphi), r2 = roots_table(M);
  MK(dmalloc(&rootsPhi, Nphi)); MK(dmalloc(&rootsM, M));
  MK(cudaMemcpy(rootsPhi, r1.data(), Nphi * sizeof(double2), cudaMemcpyHostToDevice));
  MK(cudaMemcpy(rootsM, r2.data(), M * sizeof(double2), cudaMemcpyHostToDevice));
  MK(dmalloc(&scratch, 64));
  MK(dmalloc(&ctl, 1));
  MK(cudaMemset(ctl, 0, sizeof(Ctl)));
  MK(cudaMallocHost((void **)&hctl, sizeof(Ctl)));
  memset(hctl, 0, sizeof(Ctl));
  MK(cudaMallocHost((void **)&hdt, sizeof(double)));
  {
    // per-row / per-face FP64 constants of the hydro kernel
    std::vector<double> t((size_t)8 * (Nu + 1), 0.0);
    auto col = [&](int k) { return t.data() + (size_t)k * (Nu + 1); };
    for (int i = 0; i < Nu; ++i) {
      int im = i - 1 > 0 ? i - 1 : 0, ip = i + 1 < Nu - 1 ? i + 1 : Nu - 1;
      col(0)[i] = -p.gmstar / (R[i] * R[i]);
      col(1)[i] = 1.0 / R[i];
      col(2)[i] = 1.0 / (R[ip] - R[im]);
      col(3)[i] = 1.0 / Vol[i];
      col(4)[i] = 1.0 / (Rf[i + 1] - Rf[i]);
      col(5)[i] = 1.0 / (R[i] * dphi);
    }
    for (int f = 1; f <= Nu; ++f) col(6)[f] = 1.0 / (Rf[f] - Rf[f - 1]);
    for (int f = 0; f < Nu; ++f) col(7)[f] = 1.0 / (Rf[f + 1] - Rf[f]);
    MK(dmalloc(&rowtab, t.size()));
    MK(cudaMemcpy(rowtab, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    auto dc = [&](int k) { return (const double *)(rowtab + (size_t)k * (Nu + 1)); };
    geom.gstar = dc(0); geom.invR = dc(1); geom.invdRc = dc(2); geom.invVol = dc(3);
    geom.invdR = dc(4); geom.invdl = dc(5); geom.invdRl = dc(6); geom.invdRr = dc(7);
  }
  geom.R = dR; geom.Rf = dRf; geom.Vol = dVol;
  geom.Nu = Nu; geom.Nphi = Nphi; geom.dphi = dphi; geom.du = du;
  geom.Kpoly = p.Kpoly; geom.gamma = p.gamma_gas; geom.gmstar = p.gmstar;
  geom.inv2dphi = 1.0 / (2.0 * dphi); geom.invdu = 1.0 / du; geom.inv2du = 1.0 / (2.0 * du);
  geom.gamma2 = (p.gamma_gas == 2.0) ? 1 : 0;
  MK(prepare_fft_kernels());
  int rc = build_khat();
  if (rc) return rc;
  if (p.precision == DG_PREC_MIXED) {
    rc = mixed_init();
    if (rc) return rc;
  }
  MK(cudaStreamSynchronize(st));
  return DG_OK;
}

// kalnajs.hpp:105-116: khat = r2c of the kernel sampled at wrapped offsets.
int dg_handle::build_khat() {
  double *tmp = nullptr;
  MK(dmalloc(&tmp, (size_t)M * p.Nphi));
  MK(launch_kernel_samples64(tmp, M, p.Nphi, du, dphi, p.eps, st));
  MK(launch_phi_fwd<double>(tmp, M, p.Nphi, nullptr, W, M, plPhi, rootsPhi, st));
  MK(launch_u_conv<double>(W, M, Nc, M, M, plM, rootsM, nullptr, Khat, st));
  MK(cudaStreamSynchronize(st));
  MK(cudaFree(tmp));
  return DG_OK;
}

void dg_handle::release() {
  if (dev >= 0) cudaSetDevice(dev);
  if (st) cudaStreamSynchronize(st);
  mixed_release();
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (diag) cudaFree(diag);
  void *ptrs[] = {rowtab, dR, dRf, dVol, dSqrtR, dR32, S[0], S[1], VR[0], VR[1], VP[0], VP[1], dPhi, gA, gB,
                  W, Khat, rootsPhi, rootsM, scratch, ctl};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (hctl) cudaFreeHost(hctl);
  if (hdt) cudaFreeHost(hdt);
  for (auto &e : ev_pool) cudaEventDestroy(e);
  if (own_st) cudaStreamDestroy(own_st);
}

// ---------------------------------------------------------------------------------
// gravity (FP64): kalnajs.hpp:48-63
int dg_handle::potential64(const double *dSig, double *dOut) {
  MK(prof_begin(DG_PROF_GRAV_PHI_FWD));
  MK(launch_phi_fwd<double>(dSig, p.Nu, p.Nphi, dR32, W, M, plPhi, rootsPhi, st));
  MK(prof_end(DG_PROF_GRAV_PHI_FWD));
  MK(prof_begin(DG_PROF_GRAV_U));
  MK(launch_u_conv<double>(W, M, Nc, p.Nu, p.Nu, plM, rootsM, Khat, nullptr, st));
  MK(prof_end(DG_PROF_GRAV_U));
  const double pref = -p.G * du * dphi / (static_cast<double>(M) * p.Nphi);
  MK(prof_begin(DG_PROF_GRAV_PHI_INV));
  MK(launch_phi_inv<double>(W, M, p.Nu, p.Nphi, plPhi, rootsPhi, pref, dSqrtR, dOut, st));
  MK(prof_end(DG_PROF_GRAV_PHI_INV));
  return DG_OK;
}

// One full time step on the device: gravity of the current Sigma (if selfgrav), then the
// fused hydro kernel; dt comes from the control block.
int dg_handle::enqueue_step() {
  if (p.precision == DG_PREC_MIXED) return mixed_enqueue_step();
  const int c = cur, o = cur ^ 1;
  int fm = kForceNone;
  if (p.selfgrav) {
    MK(prof_begin(DG_PROF_GRAVITY));
    int rc = potential64(S[c], dPhi);
    if (rc) return rc;
    MK(prof_end(DG_PROF_GRAVITY));
    fm = kForcePhi;
  }
  MK(prof_begin(DG_PROF_HYDRO));
  MK(launch_hydro64(S[c], VR[c], VP[c], dPhi, nullptr, nullptr, fm, S[o], VR[o], VP[o], ctl, geom, st));
  MK(prof_end(DG_PROF_HYDRO));
  cur = o;
  return DG_OK;
}

// ---------------------------------------------------------------------------------
// per-phase event timing
cudaError_t dg_handle::prof_begin(int phase) {
  if (!prof_on) return cudaSuccess;
  if (ev_used + 2 > (int)ev_pool.size()) {
    for (int k = 0; k < 64; ++k) {
      cudaEvent_t e;
      cudaError_t r = cudaEventCreate(&e);
      if (r != cudaSuccess) return r;
      ev_pool.push_back(e);
    }
  }
  prof_pending.push_back({phase, ev_used});
  cudaEvent_t e = ev_pool[ev_used];
  ev_used += 2;
  return cudaEventRecord(e, st);
}

cudaError_t dg_handle::prof_end(int phase) {
  if (!prof_on) return cudaSuccess;
  // phases nest (the gravity parts sit inside the gravity phase): close the latest of this phase
  for (auto it = prof_pending.rbegin(); it != prof_pending.rend(); ++it)
    if (it->first == phase) return cudaEventRecord(ev_pool[it->second + 1], st);
  return cudaErrorInvalidValue;
}

int dg_handle::prof_collect() {
  if (prof_pending.empty()) return DG_OK;
  MK(cudaStreamSynchronize(st));
  for (auto &pp : prof_pending) {
    float ms = 0.f;
    MK(cudaEventElapsedTime(&ms, ev_pool[pp.second], ev_pool[pp.second + 1]));
    prof_ms[pp.first] += ms;
    prof_count[pp.first] += 1;
  }
  prof_pending.clear();
  ev_used = 0;
  return DG_OK;
}

int dg_handle::set_ctl_fields(double t, double tlim, double cfl, double dt, double tnext, double dtout,
                              int fixed_dt) {
  hctl->t = t;
  hctl->tlim = tlim;
  hctl->cfl = cfl;
  hctl->dt = dt;
  hctl->tnext = tnext;
  hctl->dtout = dtout;
  hctl->mD = mD;
  hctl->fixed_dt = fixed_dt;
  // write the scalar prefix of the control block (everything before dtinv_bits is plain
  // doubles; the accumulators are reset explicitly)
  MK(cudaMemcpyAsync(ctl, hctl, offsetof(Ctl, dtinv_bits), cudaMemcpyHostToDevice, st));
  MK(cudaMemsetAsync(&ctl->dtinv_bits, 0, sizeof(unsigned long long), st));
  MK(cudaMemsetAsync(&ctl->done_ctas, 0, sizeof(unsigned int), st));
  MK(cudaMemsetAsync(&ctl->modesum, 0, sizeof(ctl->modesum), st));
  return DG_OK;
}

int dg_handle::read_ctl() {
  MK(cudaMemcpyAsync(hctl, ctl, offsetof(Ctl, rec), cudaMemcpyDeviceToHost, st));
  MK(cudaStreamSynchronize(st));
  return DG_OK;
}

int dg_handle::check_status() {
  if (hctl->status & kStNonFinite) return fail(DG_ERR_NONFINITE, "step", "dt or state became non-finite");
  if (hctl->status & kStTimeout) return fail(DG_ERR_TIMEOUT, "step", "a bounded device wait gave up");
  return DG_OK;
}

int dg_handle::cfl_launch(int nmodes, int record) {
  MK(prof_begin(DG_PROF_CFL));
  if (p.precision == DG_PREC_MIXED) {
    int rc = mixed_cfl_launch(nmodes, record);
    if (rc) return rc;
  } else {
    MK(launch_cfl64(S[cur], VR[cur], VP[cur], ctl, geom, nmodes, record, st));
  }
  MK(prof_end(DG_PROF_CFL));
  return DG_OK;
}

// Leave free-running mode: pull t and the step count back from the device.
int dg_handle::sync_from_device() {
  if (!freerun) return DG_OK;
  int rc = read_ctl();
  if (rc) return rc;
  t = hctl->t;
  nsteps = hctl->step;
  freerun = false;
  return check_status();
}

int dg_handle::enqueue_step_forces(const double *gRh, const double *gph) {
  if (p.precision == DG_PREC_MIXED) return mixed_enqueue_step_forces(gRh, gph);
  const size_t n = (size_t)p.Nu * p.Nphi;
  int fm = kForceNone;
  if (gRh) {
    MK(cudaMemcpyAsync(gA, gRh, n * sizeof(double), cudaMemcpyHostToDevice, st));
    MK(cudaMemcpyAsync(gB, gph, n * sizeof(double), cudaMemcpyHostToDevice, st));
    fm = kForceArrays;
  }
  const int c = cur, o = cur ^ 1;
  MK(launch_hydro64(S[c], VR[c], VP[c], nullptr, gA, gB, fm, S[o], VR[o], VP[o], ctl, geom, st));
  cur = o;
  return DG_OK;
}

int dg_handle::modes_launch(int nmodes, double *out) {
  if (p.precision == DG_PREC_MIXED) return mixed_modes_launch(nmodes, out);
  MK(launch_modes64(S[cur], geom, nmodes, out, st));
  return DG_OK;
}

int dg_handle::conserved_launch(double *out2) {
  if (p.precision == DG_PREC_MIXED) return mixed_conserved_launch(out2);
  MK(launch_conserved64(S[cur], VP[cur], geom, out2, st));
  return DG_OK;
}

int dg_handle::upload_state(const double *Sig, const double *vRh, const double *vph) {
  if (p.precision == DG_PREC_MIXED) return mixed_upload_state(Sig, vRh, vph);
  const size_t n = (size_t)p.Nu * p.Nphi;
  MK(cudaMemcpyAsync(S[cur], Sig, n * sizeof(double), cudaMemcpyHostToDevice, st));
  MK(cudaMemcpyAsync(VR[cur], vRh, n * sizeof(double), cudaMemcpyHostToDevice, st));
  MK(cudaMemcpyAsync(VP[cur], vph, n * sizeof(double), cudaMemcpyHostToDevice, st));
  return DG_OK;
}

int dg_handle::download_state(double *Sig, double *vRh, double *vph) {
  if (p.precision == DG_PREC_MIXED) return mixed_download_state(Sig, vRh, vph);
  const size_t n = (size_t)p.Nu * p.Nphi;
  MK(cudaMemcpyAsync(Sig, S[cur], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  MK(cudaMemcpyAsync(vRh, VR[cur], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  MK(cudaMemcpyAsync(vph, VP[cur], n * sizeof(double), cudaMemcpyDeviceToHost, st));
  MK(cudaStreamSynchronize(st));
  return DG_OK;
}

// ---------------------------------------------------------------------------------
// chunked loop: a CUDA graph holds kGraphSteps steps (an even count, so it starts and
// ends on the same ping-pong buffer).
// Record kGraphSteps steps into graph_exec (nothing runs: a capture only records).
int dg_handle::capture_graph() {
  if (graph_exec || !use_graphs) return DG_OK;
  if (cur != 0) return fail(DG_ERR_STATE, "dg_capture_graph", "the state sits in the second ping-pong buffer");
  cudaGraph_t g = nullptr;
  // enqueue_step keeps host-side flags of what the last enqueued kernels were; recording
  // runs nothing, so they are put back, and a launch of the graph applies their end values
  const int flags_before = loop_flags();
  MK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  int rc = DG_OK;
  for (int k = 0; k < kGraphSteps && !rc; ++k) rc = enqueue_step();
  cudaError_t e = cudaStreamEndCapture(st, &g);
  graph_end_flags = loop_flags();
  set_loop_flags(flags_before);
  cur = 0;  // enqueue_step flipped cur kGraphSteps times during capture
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  MK(e);
  e = cudaGraphInstantiate(&graph_exec, g, 0);
  cudaGraphDestroy(g);
  MK(e);
  return DG_OK;
}

int dg_handle::run_chunk(int nsteps) {
  if (nsteps == kGraphSteps && cur == 0 && use_graphs && !prof_on) {
    if (!graph_exec) {
      int rc = capture_graph();
      if (rc) return rc;
    }
    MK(cudaGraphLaunch(graph_exec, st));
    set_loop_flags(graph_end_flags);
    return DG_OK;
  }
  for (int k = 0; k < nsteps; ++k) {
    int rc = enqueue_step();
    if (rc) return rc;
  }
  return DG_OK;
}

// ---------------------------------------------------------------------------------
// C ABI

extern "C" {

int dg_params_default(dg_params *p) {
  if (!p) return DG_ERR_INVALID;
  memset(p, 0, sizeof(*p));
  p->Nu = 128; p->Nphi = 128;
  p->Rin = 0.25; p->Rout = 1.0;
  p->Kpoly = 0.25; p->gamma_gas = 2.0; p->gmstar = 0.6; p->G = 1.0;
  p->eps = 0.02; p->selfgrav = 1; p->amp = 1e-3; p->phase0 = 0.0;
  p->R0 = 0.45; p->w2 = 0.05; p->S0 = 0.372;
  p->precision = DG_PREC_FP64;
  p->device = -1;
  p->basic_state = DG_BASIC_FFT;
  return DG_OK;
}

static thread_local std::string g_create_error;

}  // extern "C"

// Handle-less calls (dg_create, the fits, the parameter file) leave their reason here; it
// is what dg_last_error(NULL) returns on the same thread.
void dg_set_global_error(const std::string &why) { g_create_error = why; }

extern "C" {

int dg_create(const dg_params *p, dg_handle **out) {
  if (!p || !out) return DG_ERR_INVALID;
  *out = nullptr;
  std::string why;
  int rc = validate(p, &why);
  if (rc) { g_create_error = why; return rc; }
  dg_handle *h = new (std::nothrow) dg_handle();
  if (!h) return DG_ERR_NOMEM;
  rc = h->init(*p);
  if (rc) {
    g_create_error = h->err;
    h->release();
    delete h;
    return rc;
  }
  *out = h;
  return DG_OK;
}

void dg_destroy(dg_handle *h) {
  if (!h) return;
  h->release();
  delete h;
}

const char *dg_last_error(const dg_handle *h) {
  if (!h) return g_create_error.c_str();
  return h->err.c_str();
}

const char *dg_status_string(int s) {
  switch (s) {
    case DG_OK: return "ok";
    case DG_ERR_INVALID: return "invalid argument";
    case DG_ERR_CUDA: return "CUDA error";
    case DG_ERR_NONFINITE: return "non-finite state or dt";
    case DG_ERR_UNSUPPORTED: return "unsupported size or option";
    case DG_ERR_NOMEM: return "out of memory";
    case DG_ERR_TIMEOUT: return "device wait timed out";
    case DG_ERR_STATE: return "call out of order";
  }
  return "unknown status";
}

int dg_grid(const dg_handle *h, double *R, double *Rf, double *Vol) {
  if (!h) return DG_ERR_INVALID;
  if (R) memcpy(R, h->R.data(), h->p.Nu * sizeof(double));
  if (Rf) memcpy(Rf, h->Rf.data(), (h->p.Nu + 1) * sizeof(double));
  if (Vol) memcpy(Vol, h->Vol.data(), h->p.Nu * sizeof(double));
  return DG_OK;
}

int dg_set_state(dg_handle *h, const double *Sig, const double *vR, const double *vp) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h || !Sig || !vR || !vp) return DG_ERR_INVALID;
  DG_CK(cudaSetDevice(h->dev));
  int rc = h->upload_state(Sig, vR, vp);
  if (rc) return rc;
  // m_D as diskmain.cpp:66-70 (host, same summation order)
  const int Nu = h->p.Nu, Nphi = h->p.Nphi;
  double mD = 0.0;
  for (int i = 0; i < Nu; ++i) {
    double dA = h->R[i] * (h->Rf[i + 1] - h->Rf[i]) * h->dphi;
    for (int j = 0; j < Nphi; ++j) mD += Sig[(size_t)i * Nphi + j] * dA;
  }
  h->mD = mD;
  h->have_state = true;
  h->t = 0.0;
  h->tnext = 0.0;
  h->nsteps = 0;
  DG_CK(cudaMemsetAsync(&h->ctl->step, 0, sizeof(long long), h->st));
  DG_CK(cudaMemsetAsync(&h->ctl->status, 0, sizeof(int), h->st));
  DG_CK(cudaStreamSynchronize(h->st));
  return DG_OK;
}

int dg_get_state(dg_handle *h, double *Sig, double *vR, double *vp) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h || !Sig || !vR || !vp) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_get_state", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  return h->download_state(Sig, vR, vp);
}

int dg_init_standard(dg_handle *h) {
  if (!h) return DG_ERR_INVALID;
  DG_CK(cudaSetDevice(h->dev));
  const dg_params &p = h->p;
  const int Nu = p.Nu, Nphi = p.Nphi;
  const size_t n = (size_t)Nu * Nphi;
  auto Sigma0 = [&](double R) { return p.S0 * std::exp(-(R - p.R0) * (R - p.R0) / p.w2); };  // diskmain.cpp:34
  std::vector<double> gRdisk(Nu, 0.0);
  if (p.selfgrav && p.basic_state == DG_BASIC_ELLIPTIC) {
    int rc = dg_rotation_curve_elliptic(&p, Nu, h->R.data(), gRdisk.data(), nullptr, nullptr, nullptr);
    if (rc) return h->fail(rc, "dg_init_standard", "elliptic rotation curve");
  } else if (p.selfgrav) {  // diskmain.cpp:37-48
    std::vector<double> Sig_axi(n), gR_eq(n);
    for (int i = 0; i < Nu; ++i)
      for (int j = 0; j < Nphi; ++j) Sig_axi[(size_t)i * Nphi + j] = Sigma0(h->R[i]);
    DG_CK(cudaMemcpyAsync(h->gA, Sig_axi.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->st));
    int rc = h->potential64(h->gA, h->dPhi);
    if (rc) return rc;
    DG_CK(launch_forces64(h->dPhi, h->gA, h->gB, h->geom, h->st));
    DG_CK(cudaMemcpyAsync(gR_eq.data(), h->gA, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
    DG_CK(cudaStreamSynchronize(h->st));
    for (int i = 0; i < Nu; ++i) {
      double s = 0;
      for (int j = 0; j < Nphi; ++j) s += gR_eq[(size_t)i * Nphi + j];
      gRdisk[i] = s / Nphi;
    }
  }
  std::vector<double> Sig(n), vR(n), vp(n), vphi0(Nu);
  for (int i = 0; i < Nu; ++i) {  // diskmain.cpp:51-63
    double R = h->R[i];
    double dSig = Sigma0(R) * (-2.0 * (R - p.R0) / p.w2);
    double dPdR = p.Kpoly * p.gamma_gas * std::pow(Sigma0(R), p.gamma_gas - 1.0) * dSig;
    double v2 = p.gmstar / R + (R / Sigma0(R)) * dPdR - R * gRdisk[i];
    double vphi = (v2 > 0) ? std::sqrt(v2) : 0.0;
    vphi0[i] = vphi;
    for (int j = 0; j < Nphi; ++j) {
      double phi = (j + 0.5) * h->dphi;
      double c = p.phase0 == 0.0 ? std::cos(2.0 * phi) : std::cos(2.0 * (phi - p.phase0));
      Sig[(size_t)i * Nphi + j] = Sigma0(R) * (1.0 + p.amp * c);
      vR[(size_t)i * Nphi + j] = 0.0;
      vp[(size_t)i * Nphi + j] = vphi;
    }
  }
  h->basic_from_standard = true;
  h->std_sigma0.resize(Nu);
  for (int i = 0; i < Nu; ++i) h->std_sigma0[i] = Sigma0(h->R[i]);
  h->std_vphi0 = vphi0;
  h->std_gR0 = gRdisk;
  int rc = dg_set_state(h, Sig.data(), vR.data(), vp.data());
  h->basic_from_standard = false;
  return rc;
}

int dg_timestep(dg_handle *h, double cfl, double *dt) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h || !dt) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_timestep", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  int rc = h->set_ctl_fields(h->t, INFINITY, cfl, 0.0, 0.0, 0.0, 1);
  if (rc) return rc;
  rc = h->cfl_launch(0, 0);
  if (rc) return rc;
  rc = h->read_ctl();
  if (rc) return rc;
  *dt = h->hctl->dt;
  return DG_OK;
}

static int step_common(dg_handle *h, double dt, const double *gR, const double *gp, bool own_gravity) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_step", "no state set");
  if (!(dt >= 0) || !std::isfinite(dt)) return h->fail(DG_ERR_INVALID, "dg_step", "dt must be finite and >= 0");
  if ((gR == nullptr) != (gp == nullptr)) return h->fail(DG_ERR_INVALID, "dg_step_forces", "gR and gp must both be given or both be NULL");
  DG_CK(cudaSetDevice(h->dev));
  int rc = h->set_ctl_fields(h->t, INFINITY, 0.3, dt, 0.0, 0.0, 1);
  if (rc) return rc;
  if (own_gravity) {
    rc = h->enqueue_step();
  } else {
    rc = h->enqueue_step_forces(gR, gp);
  }
  if (rc) return rc;
  rc = h->read_ctl();
  if (rc) return rc;
  h->t = h->hctl->t;
  h->nsteps = h->hctl->step;
  return h->check_status();
}

int dg_step(dg_handle *h, double dt) { return step_common(h, dt, nullptr, nullptr, true); }
int dg_step_forces(dg_handle *h, double dt, const double *gR, const double *gp) {
  return step_common(h, dt, gR, gp, false);
}

int dg_potential(dg_handle *h, const double *Sig, double *Phi) {
  if (!h || !Sig || !Phi) return DG_ERR_INVALID;
  DG_CK(cudaSetDevice(h->dev));
  const size_t n = (size_t)h->p.Nu * h->p.Nphi;
  DG_CK(cudaMemcpyAsync(h->gA, Sig, n * sizeof(double), cudaMemcpyHostToDevice, h->st));
  int rc = (h->p.precision == DG_PREC_MIXED) ? h->mixed_potential(h->gA, h->gB) : h->potential64(h->gA, h->gB);
  if (rc) return rc;
  DG_CK(cudaMemcpyAsync(Phi, h->gB, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  DG_CK(cudaStreamSynchronize(h->st));
  return DG_OK;
}

int dg_forces(dg_handle *h, const double *Phi, double *gR, double *gp) {
  if (!h || !Phi || !gR || !gp) return DG_ERR_INVALID;
  DG_CK(cudaSetDevice(h->dev));
  const size_t n = (size_t)h->p.Nu * h->p.Nphi;
  DG_CK(cudaMemcpyAsync(h->dPhi, Phi, n * sizeof(double), cudaMemcpyHostToDevice, h->st));
  DG_CK(launch_forces64(h->dPhi, h->gA, h->gB, h->geom, h->st));
  DG_CK(cudaMemcpyAsync(gR, h->gA, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  DG_CK(cudaMemcpyAsync(gp, h->gB, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  DG_CK(cudaStreamSynchronize(h->st));
  return DG_OK;
}

int dg_disk_mass(dg_handle *h, double *mD) {
  if (!h || !mD) return DG_ERR_INVALID;
  double mass, L;
  int rc = dg_conserved(h, &mass, &L);
  if (rc) return rc;
  *mD = mass;
  return DG_OK;
}

int dg_modes(dg_handle *h, int mmax, double *re_im) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h || !re_im || mmax < 0 || mmax >= kMaxModes) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_modes", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  int rc = h->modes_launch(mmax + 1, h->scratch);
  if (rc) return rc;
  double buf[2 * kMaxModes];
  DG_CK(cudaMemcpyAsync(buf, h->scratch, 2 * (mmax + 1) * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  DG_CK(cudaStreamSynchronize(h->st));
  for (int q = 0; q < 2 * (mmax + 1); ++q) re_im[q] = buf[q] / h->mD;
  return DG_OK;
}

int dg_conserved(dg_handle *h, double *mass, double *angmom) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h || !mass || !angmom) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_conserved", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  int rc = h->conserved_launch(h->scratch);
  if (rc) return rc;
  double buf[2];
  DG_CK(cudaMemcpyAsync(buf, h->scratch, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  DG_CK(cudaStreamSynchronize(h->st));
  *mass = buf[0];
  *angmom = buf[1];
  return DG_OK;
}

int dg_time(dg_handle *h, double *t, long long *nsteps) {
  if (h) { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h) return DG_ERR_INVALID;
  if (t) *t = h->t;
  if (nsteps) *nsteps = h->nsteps;
  return DG_OK;
}

}  // extern "C"

// The loop of diskmain.cpp:88-110 on the device, handing every mode record to `sink` in
// order as soon as the host drains it (after each chunk of steps).
template <typename Sink>
static int advance_records(dg_handle *h, double tlim, double cfl, double dtout, Sink &&sink, double *t_out,
                           long long *nsteps_out) {
  { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_advance", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  // diskmain.cpp:88,93: tnext starts at 0 with the state and persists across calls
  int rc = h->set_ctl_fields(h->t, tlim, cfl, 0.0, h->tnext, dtout, 0);
  if (rc) return rc;
  DG_CK(cudaMemsetAsync(&h->ctl->nrec, 0, sizeof(int), h->st));
  const bool first_record = (h->t < tlim) && (h->t >= h->tnext - 1e-12);
  rc = h->cfl_launch(0, first_record ? 1 : 0);  // record at t (if the loop runs) + first dt
  if (rc) return rc;
  for (;;) {
    rc = h->read_ctl();
    if (rc) return rc;
    // drain records
    int nr = h->hctl->nrec;
    if (nr > 0) {
      std::vector<double> tmp((size_t)nr * 4);
      DG_CK(cudaMemcpyAsync(tmp.data(), &h->ctl->rec[0][0], (size_t)nr * 4 * sizeof(double), cudaMemcpyDeviceToHost,
                            h->st));
      DG_CK(cudaMemsetAsync(&h->ctl->nrec, 0, sizeof(int), h->st));
      DG_CK(cudaStreamSynchronize(h->st));
      for (int k = 0; k < nr; ++k) {
        const dg_record r{tmp[4 * k], tmp[4 * k + 1], tmp[4 * k + 2], tmp[4 * k + 3]};
        sink(r);
      }
    }
    h->t = h->hctl->t;
    h->nsteps = h->hctl->step;
    rc = h->check_status();
    if (rc) return rc;
    if (!(h->t < tlim)) break;
    // estimate the remaining steps from the current dt
    double dt = h->hctl->dt;
    double est = dt > 0 ? (tlim - h->t) / dt : 1.0;
    int chunk;
    if (est > 2.0 * dg_handle::kGraphSteps && h->cur == 0 && h->use_graphs) chunk = dg_handle::kGraphSteps;
    else chunk = est > 8 ? (int)(est / 2 < 64 ? est / 2 : 64) : 1;
    rc = h->run_chunk(chunk);
    if (rc) return rc;
  }
  h->tnext = h->hctl->tnext;
  if (t_out) *t_out = h->t;
  if (nsteps_out) *nsteps_out = h->nsteps;
  return DG_OK;
}

extern "C" {

int dg_advance(dg_handle *h, double tlim, double cfl, double dtout, dg_record *rec, int max_rec, int *n_rec,
               double *t_out, long long *nsteps_out) {
  if (!h || (max_rec > 0 && !rec) || !(cfl > 0) || !(dtout > 0)) return DG_ERR_INVALID;
  int nout = 0;
  int rc = advance_records(
      h, tlim, cfl, dtout,
      [&](const dg_record &r) {
        if (nout < max_rec) rec[nout] = r;
        ++nout;
      },
      t_out, nsteps_out);
  if (rc) return rc;
  if (n_rec) *n_rec = nout < max_rec ? nout : max_rec;
  return DG_OK;
}

int dg_advance_cb(dg_handle *h, double tlim, double cfl, double dtout, dg_record_fn fn, void *user, int *n_rec,
                  double *t_out, long long *nsteps_out) {
  if (!h || !fn || !(cfl > 0) || !(dtout > 0)) return DG_ERR_INVALID;
  int nout = 0;
  int rc = advance_records(
      h, tlim, cfl, dtout,
      [&](const dg_record &r) {
        fn(&r, user);
        ++nout;
      },
      t_out, nsteps_out);
  if (n_rec) *n_rec = nout;
  return rc;
}

int dg_capture_graph(dg_handle *h) {
  if (!h) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_capture_graph", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  return h->capture_graph();
}

int dg_set_stream(dg_handle *h, void *stream) {
  if (!h) return DG_ERR_INVALID;
  DG_CK(cudaSetDevice(h->dev));
  DG_CK(cudaStreamSynchronize(h->st));
  h->st = stream ? (cudaStream_t)stream : h->own_st;
  return DG_OK;
}

int dg_run_steps(dg_handle *h, int nsteps, double cfl, int sync) {
  if (!h || nsteps < 0 || !(cfl > 0)) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_run_steps", "no state set");
  DG_CK(cudaSetDevice(h->dev));
  if (!h->freerun || cfl != h->freerun_cfl) {
    int rc = h->sync_from_device();
    if (rc) return rc;
    rc = h->set_ctl_fields(h->t, INFINITY, cfl, 0.0, INFINITY, 1.0, 0);
    if (rc) return rc;
    rc = h->cfl_launch(0, 0);  // dt of the first step
    if (rc) return rc;
    h->freerun = true;
    h->freerun_cfl = cfl;
  }
  int left = nsteps;
  while (left > 0) {
    int k;
    if (left >= dg_handle::kGraphSteps && h->cur == 0 && h->use_graphs && !h->prof_on) k = dg_handle::kGraphSteps;
    else if (h->cur == 1) k = 1;  // realign the ping-pong buffers for the graph
    else k = left < 8 ? left : 8;
    int rc = h->run_chunk(k);
    if (rc) return rc;
    left -= k;
  }
  if (sync) return h->sync_from_device();
  return DG_OK;
}

int dg_step_host(dg_handle *h, double cfl, double *Sig, double *vR, double *vp, double *dt) {
  if (!h || !Sig || !vR || !vp || !(cfl > 0)) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_step_host", "no basic state: call dg_set_state or dg_init_standard once");
  { int rc0 = h->sync_from_device(); if (rc0) return rc0; }
  DG_CK(cudaSetDevice(h->dev));
  h->in_step_host = true;
  int rc = h->upload_state(Sig, vR, vp);
  h->in_step_host = false;
  if (rc) return rc;
  rc = h->set_ctl_fields(h->t, INFINITY, cfl, 0.0, INFINITY, 1.0, 1);
  if (rc) return rc;
  rc = h->cfl_launch(0, 0);
  if (rc) return rc;
  DG_CK(cudaMemcpyAsync(h->hdt, &h->ctl->dt, sizeof(double), cudaMemcpyDeviceToHost, h->st));
  rc = h->enqueue_step();
  if (rc) return rc;
  rc = h->download_state(Sig, vR, vp);  // synchronises the stream
  if (rc) return rc;
  rc = h->read_ctl();
  if (rc) return rc;
  h->t = h->hctl->t;
  h->nsteps = h->hctl->step;
  if (dt) *dt = *h->hdt;
  return h->check_status();
}

int dg_profile_enable(dg_handle *h, int on) {
  if (!h) return DG_ERR_INVALID;
  int rc = h->prof_collect();
  if (rc) return rc;
  h->prof_on = on != 0;
  return DG_OK;
}

int dg_tuning_info(const dg_handle *h, char *buf, int len) {
  if (!h || !buf || len < 1) return DG_ERR_INVALID;
  const std::string s = h->p.precision == DG_PREC_MIXED ? h->mixed_tuning_info() : std::string("fp64: one variant per kernel");
  snprintf(buf, (size_t)len, "%s", s.c_str());
  return DG_OK;
}

int dg_kernels_per_step(const dg_handle *h) {
  if (!h) return DG_ERR_INVALID;
  const int grav = !h->p.selfgrav ? 0 : (h->p.precision == DG_PREC_MIXED ? h->mixed_gravity_kernels() : 3);
  return grav + (h->p.precision == DG_PREC_MIXED ? h->mixed_hydro_kernels() : 1);
}

int dg_profile_read(dg_handle *h, double *ms, long long *count) {
  if (!h) return DG_ERR_INVALID;
  int rc = h->prof_collect();
  if (rc) return rc;
  for (int k = 0; k < DG_PROF_N; ++k) {
    if (ms) ms[k] = h->prof_ms[k];
    if (count) count[k] = h->prof_count[k];
    h->prof_ms[k] = 0.0;
    h->prof_count[k] = 0;
  }
  return DG_OK;
}

}  // extern "C"
