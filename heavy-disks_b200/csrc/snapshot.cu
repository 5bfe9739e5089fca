// Snapshot / restart and per-step Fourier diagnostics (host side).
//
// The reference writes no snapshots and cannot restart (its state lives in the process);
// the format below is this library's own.  Little-endian binary:
//   char[8]  "DGSNAP1\0"
//   int32    version (1), precision, Nu, Nphi, selfgrav, basic_state
//   double   Rin, Rout, Kpoly, gamma_gas, gmstar, G, eps, amp, phase0, R0, w2, S0
//   double   t, tnext, mD;  int64 nsteps
//   int32    nbasic (Nu for the mixed path, else 0); then nbasic doubles each of
//            Sigma0, V0, g0 (the basic state the perturbation is measured against)
//   double   Sigma[Nu*Nphi], vR[Nu*Nphi], vphi[Nu*Nphi]   (full FP64 fields)
// For the mixed path the FP32 perturbation is recovered exactly on load: Sigma0 + sigma
// is exact in FP64 for every FP32 sigma of the magnitudes a disk holds.
#include <cstdio>
#include <cstring>
#include <vector>

#include "engine.h"

struct MixedBasicAccess;  // the mixed basic state is reached through dg_handle helpers

namespace {

const char kMagic[8] = {'D', 'G', 'S', 'N', 'A', 'P', '1', '\0'};

struct FileCloser {
  FILE *f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

template <typename T>
bool wr(FILE *f, const T *p, size_t n) {
  return fwrite(p, sizeof(T), n, f) == n;
}
template <typename T>
bool rd(FILE *f, T *p, size_t n) {
  return fread(p, sizeof(T), n, f) == n;
}

}  // namespace

extern "C" {

int dg_save(dg_handle *h, const char *path) {
  if (!h || !path) return DG_ERR_INVALID;
  if (!h->have_state) return h->fail(DG_ERR_STATE, "dg_save", "no state set");
  int rc = h->sync_from_device();
  if (rc) return rc;
  const size_t n = (size_t)h->p.Nu * h->p.Nphi;
  std::vector<double> S(n), vR(n), vp(n);
  rc = h->download_state(S.data(), vR.data(), vp.data());
  if (rc) return rc;
  FILE *f = fopen(path, "wb");
  if (!f) return h->fail(DG_ERR_INVALID, "dg_save", "cannot open file for writing");
  FileCloser fc{f};
  const dg_params &p = h->p;
  int32_t hdr[6] = {1, p.precision, p.Nu, p.Nphi, p.selfgrav, p.basic_state};
  double par[12] = {p.Rin, p.Rout, p.Kpoly, p.gamma_gas, p.gmstar, p.G, p.eps, p.amp, p.phase0, p.R0, p.w2, p.S0};
  double tt[3] = {h->t, h->tnext, h->mD};
  int64_t ns = h->nsteps;
  std::vector<double> S0, V0, g0;
  h->mixed_basic(&S0, &V0, &g0);
  int32_t nb = (int32_t)S0.size();
  bool ok = wr(f, kMagic, 8) && wr(f, hdr, 6) && wr(f, par, 12) && wr(f, tt, 3) && wr(f, &ns, 1) && wr(f, &nb, 1);
  if (nb) ok = ok && wr(f, S0.data(), nb) && wr(f, V0.data(), nb) && wr(f, g0.data(), nb);
  ok = ok && wr(f, S.data(), n) && wr(f, vR.data(), n) && wr(f, vp.data(), n);
  if (!ok) return h->fail(DG_ERR_INVALID, "dg_save", "short write");
  return DG_OK;
}

int dg_load(dg_handle *h, const char *path) {
  if (!h || !path) return DG_ERR_INVALID;
  int rc = h->sync_from_device();
  if (rc) return rc;
  FILE *f = fopen(path, "rb");
  if (!f) return h->fail(DG_ERR_INVALID, "dg_load", "cannot open file");
  FileCloser fc{f};
  char mg[8];
  int32_t hdr[6];
  double par[12], tt[3];
  int64_t ns;
  int32_t nb;
  if (!rd(f, mg, 8) || memcmp(mg, kMagic, 8) || !rd(f, hdr, 6) || hdr[0] != 1)
    return h->fail(DG_ERR_INVALID, "dg_load", "not a diskgpu snapshot (version 1)");
  const dg_params &p = h->p;
  if (hdr[1] != p.precision || hdr[2] != p.Nu || hdr[3] != p.Nphi || hdr[4] != p.selfgrav)
    return h->fail(DG_ERR_INVALID, "dg_load", "snapshot grid, precision or self-gravity differ from the handle's");
  if (!rd(f, par, 12) || !rd(f, tt, 3) || !rd(f, &ns, 1) || !rd(f, &nb, 1))
    return h->fail(DG_ERR_INVALID, "dg_load", "truncated header");
  const double mine[12] = {p.Rin, p.Rout, p.Kpoly, p.gamma_gas, p.gmstar, p.G, p.eps, p.amp, p.phase0, p.R0, p.w2, p.S0};
  for (int k = 0; k < 12; ++k)
    if (k != 7 && k != 8 && par[k] != mine[k])  // amp and phase0 only shape the initial seed
      return h->fail(DG_ERR_INVALID, "dg_load", "snapshot physics parameters differ from the handle's");
  const size_t n = (size_t)p.Nu * p.Nphi;
  std::vector<double> S0(nb), V0(nb), g0(nb), S(n), vR(n), vp(n);
  bool ok = true;
  if (nb) ok = rd(f, S0.data(), nb) && rd(f, V0.data(), nb) && rd(f, g0.data(), nb);
  ok = ok && rd(f, S.data(), n) && rd(f, vR.data(), n) && rd(f, vp.data(), n);
  if (!ok) return h->fail(DG_ERR_INVALID, "dg_load", "truncated snapshot");
  if (p.precision == DG_PREC_MIXED) {
    if (nb != p.Nu) return h->fail(DG_ERR_INVALID, "dg_load", "mixed snapshot without its basic state");
    h->basic_from_standard = true;
    h->std_sigma0 = S0;
    h->std_vphi0 = V0;
    h->std_gR0 = g0;
  }
  rc = dg_set_state(h, S.data(), vR.data(), vp.data());
  h->basic_from_standard = false;
  if (rc) return rc;
  h->t = tt[0];
  h->tnext = tt[1];
  h->mD = tt[2];
  h->nsteps = ns;
  long long st = ns;
  if (cudaMemcpy(&h->ctl->step, &st, sizeof(st), cudaMemcpyHostToDevice) != cudaSuccess)
    return h->fail(DG_ERR_CUDA, "dg_load", "step counter");
  return DG_OK;
}

int dg_set_diagnostics(dg_handle *h, int mmax, int capacity) {
  if (!h || mmax < 0 || mmax >= dg::kMaxModes || capacity < 0) return DG_ERR_INVALID;
  int rc = h->sync_from_device();
  if (rc) return rc;
  if (cudaSetDevice(h->dev) != cudaSuccess) return DG_ERR_CUDA;
  if (h->diag) {
    cudaFree(h->diag);
    h->diag = nullptr;
  }
  const int w = 1 + 2 * (mmax + 1);
  if (capacity > 0 && cudaMalloc((void **)&h->diag, (size_t)capacity * w * sizeof(double)) != cudaSuccess)
    return h->fail(DG_ERR_NOMEM, "dg_set_diagnostics", "ring allocation");
  h->diag_mmax = mmax;
  h->hctl->mode_every_step = capacity > 0 ? 1 : 0;
  h->hctl->mmax = mmax;
  int zero = 0;
  bool ok = cudaMemcpy(&h->ctl->mode_every_step, &h->hctl->mode_every_step, sizeof(int), cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            cudaMemcpy(&h->ctl->mmax, &mmax, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(&h->ctl->diag, &h->diag, sizeof(double *), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(&h->ctl->diag_cap, &capacity, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(&h->ctl->ndiag, &zero, sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) return h->fail(DG_ERR_CUDA, "dg_set_diagnostics", "control block");
  h->graph_reset();
  return DG_OK;
}

int dg_diagnostics_read(dg_handle *h, double *rows, int max_rows, int *n) {
  if (!h || (max_rows > 0 && !rows)) return DG_ERR_INVALID;
  int rc = h->sync_from_device();
  if (rc) return rc;
  if (cudaSetDevice(h->dev) != cudaSuccess) return DG_ERR_CUDA;
  int nd = 0;
  if (cudaMemcpy(&nd, &h->ctl->ndiag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return h->fail(DG_ERR_CUDA, "dg_diagnostics_read", "count");
  const int w = 1 + 2 * (h->diag_mmax + 1);
  const int take = nd < max_rows ? nd : max_rows;
  if (take > 0) {
    if (cudaMemcpy(rows, h->diag, (size_t)take * w * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      return h->fail(DG_ERR_CUDA, "dg_diagnostics_read", "rows");
    for (int r = 0; r < take; ++r)
      for (int q = 1; q < w; ++q) rows[(size_t)r * w + q] /= h->mD;  // C_m = sum / m_D
  }
  int zero = 0;
  if (cudaMemcpy(&h->ctl->ndiag, &zero, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return h->fail(DG_ERR_CUDA, "dg_diagnostics_read", "reset");
  if (n) *n = take;
  return DG_OK;
}

}  // extern "C"
