// Host-side FP64 services of the C ABI that need no device: the least-squares growth fit
// of the m = 2 mode (dg_fit_growth, dg_fit_phases) and the plain-text parameter file of a
// sweep (dg_params_write, dg_params_read).
//
// The reference derived gamma and Omega_p off-line from diskfft_modes.dat
// (diskfft/README.md:26-29,37); the fit restates that with the convention of Cm()
// (diskfft/src/diskmain.cpp:72-84): C_m = sum Sigma e^{-i m phi} dA / m_D, so a pattern
// rotating at Omega_p has arg C_2 = -2 Omega_p t + const and a growing mode |C_2| ~ e^{gamma t}.
// The reference takes its parameters as positional argv only (diskmain.cpp:17-23); the
// parameter file describes many disks for a sweep.
#include <cctype>
#include <cerrno>
#include <cstddef>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "diskgpu.h"

void dg_set_global_error(const std::string &why);  // capi.cu: the text dg_last_error(NULL) returns

namespace {

// arg C2 unwrapped over the whole record array: each step's difference is brought into
// [-pi, pi] (a difference of exactly pi keeps its sign)
std::vector<double> unwrap_phase(const dg_record *rec, int n) {
  std::vector<double> ph(n);
  if (n == 0) return ph;
  ph[0] = rec[0].arg2;
  double corr = 0.0;
  for (int k = 1; k < n; ++k) {
    const double dd = rec[k].arg2 - rec[k - 1].arg2;
    double dm = std::fmod(dd + M_PI, 2.0 * M_PI);
    if (dm < 0) dm += 2.0 * M_PI;
    dm -= M_PI;
    if (dm == -M_PI && dd > 0) dm = M_PI;
    if (std::fabs(dd) >= M_PI) corr += dm - dd;
    ph[k] = rec[k].arg2 + corr;
  }
  return ph;
}

// slope of y(t) by least squares over the records in [lo, hi) that pass `use`
struct Line {
  double slope_lnc2 = NAN, slope_ph = NAN;
  int n = 0;
};

Line fit_range(const dg_record *rec, const std::vector<double> &ph, int lo, int hi, double tmin, double tmax) {
  Line L;
  double st = 0.0;
  int n = 0;
  for (int k = lo; k < hi; ++k) {
    const double t = rec[k].t;
    if (!(rec[k].c2 > 0) || (tmin == tmin && t < tmin) || (tmax == tmax && t > tmax)) continue;
    st += t;
    ++n;
  }
  L.n = n;
  if (n < 2) return L;
  const double tm = st / n;
  double sy = 0.0, sp = 0.0;
  for (int k = lo; k < hi; ++k) {
    const double t = rec[k].t;
    if (!(rec[k].c2 > 0) || (tmin == tmin && t < tmin) || (tmax == tmax && t > tmax)) continue;
    sy += std::log(rec[k].c2);
    sp += ph[k];
  }
  const double ym = sy / n, pm = sp / n;
  double stt = 0.0, sty = 0.0, stp = 0.0;
  for (int k = lo; k < hi; ++k) {
    const double t = rec[k].t;
    if (!(rec[k].c2 > 0) || (tmin == tmin && t < tmin) || (tmax == tmax && t > tmax)) continue;
    const double dt = t - tm;
    stt += dt * dt;
    sty += dt * (std::log(rec[k].c2) - ym);
    stp += dt * (ph[k] - pm);
  }
  if (!(stt > 0)) {
    L.n = 0;
    return L;
  }
  L.slope_lnc2 = sty / stt;
  L.slope_ph = stp / stt;
  return L;
}

bool bad_records(const dg_record *rec, int n) { return n < 0 || (n > 0 && !rec); }

}  // namespace

extern "C" {

int dg_fit_growth(const dg_record *rec, int n, double tmin, double tmax, double *gamma, double *omega_p,
                  int *npoints) {
  if (bad_records(rec, n)) return DG_ERR_INVALID;
  const std::vector<double> ph = unwrap_phase(rec, n);
  const Line L = fit_range(rec, ph, 0, n, tmin, tmax);
  if (npoints) *npoints = L.n;
  if (L.n < 2) {
    dg_set_global_error("dg_fit_growth: fewer than two records in the fit window");
    return DG_ERR_INVALID;
  }
  if (gamma) *gamma = L.slope_lnc2;
  if (omega_p) *omega_p = -0.5 * L.slope_ph;
  return DG_OK;
}

int dg_fit_phases(const dg_record *rec, int n, double t0, double ratio_end, double ratio_min, double *out) {
  if (bad_records(rec, n) || !out) return DG_ERR_INVALID;
  for (int k = 0; k < 6; ++k) out[k] = NAN;
  out[2] = out[5] = 0.0;
  if (n < 2) {
    dg_set_global_error("dg_fit_phases: fewer than two records");
    return DG_ERR_INVALID;
  }
  // linear phase: from t0 until |C2|/|C0| first exceeds ratio_end
  double tend = rec[n - 1].t;
  for (int k = 0; k < n; ++k)
    if (rec[k].c2 / rec[k].c0 > ratio_end) {
      tend = rec[k].t;
      break;
    }
  int lo = n, hi = 0;
  for (int k = 0; k < n; ++k)
    if (rec[k].t >= t0 && rec[k].t <= tend) {
      if (k < lo) lo = k;
      hi = k + 1;
    }
  if (hi - lo < 4) {  // too short a window: everything from t0 / 2 on
    lo = n;
    hi = n;
    for (int k = 0; k < n; ++k)
      if (rec[k].t >= 0.5 * t0) {
        lo = k;
        break;
      }
  }
  if (lo < hi) {
    const std::vector<double> ph = unwrap_phase(rec + lo, hi - lo);
    const Line L = fit_range(rec + lo, ph, 0, hi - lo, NAN, NAN);
    if (L.n >= 2) {
      out[0] = L.slope_lnc2;
      out[1] = -0.5 * L.slope_ph;
      out[2] = L.n;
    }
  }
  // saturated phase: from the first to the last record with |C2|/|C0| >= ratio_min
  int first = -1, last = -1;
  for (int k = 0; k < n; ++k)
    if (rec[k].c2 / rec[k].c0 >= ratio_min) {
      if (first < 0) first = k;
      last = k;
    }
  if (first >= 0 && last > first) {
    double sr = 0.0;
    for (int k = first; k <= last; ++k) sr += rec[k].c2 / rec[k].c0;
    const std::vector<double> ph = unwrap_phase(rec + first, last - first + 1);
    const Line L = fit_range(rec + first, ph, 0, last - first + 1, NAN, NAN);
    out[3] = sr / (last - first + 1);
    out[4] = -0.5 * L.slope_ph;
    out[5] = L.n;
  }
  return DG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------
// Parameter file: one disk per line, key=value pairs

namespace {

struct Key {
  const char *name;
  enum { kInt, kDouble } kind;
  size_t off;
};

const Key kKeys[] = {
    {"Nu", Key::kInt, offsetof(dg_params, Nu)},
    {"Nphi", Key::kInt, offsetof(dg_params, Nphi)},
    {"Rin", Key::kDouble, offsetof(dg_params, Rin)},
    {"Rout", Key::kDouble, offsetof(dg_params, Rout)},
    {"Kpoly", Key::kDouble, offsetof(dg_params, Kpoly)},
    {"gamma_gas", Key::kDouble, offsetof(dg_params, gamma_gas)},
    {"gmstar", Key::kDouble, offsetof(dg_params, gmstar)},
    {"G", Key::kDouble, offsetof(dg_params, G)},
    {"eps", Key::kDouble, offsetof(dg_params, eps)},
    {"selfgrav", Key::kInt, offsetof(dg_params, selfgrav)},
    {"amp", Key::kDouble, offsetof(dg_params, amp)},
    {"phase0", Key::kDouble, offsetof(dg_params, phase0)},
    {"R0", Key::kDouble, offsetof(dg_params, R0)},
    {"w2", Key::kDouble, offsetof(dg_params, w2)},
    {"S0", Key::kDouble, offsetof(dg_params, S0)},
    {"precision", Key::kInt, offsetof(dg_params, precision)},
    {"device", Key::kInt, offsetof(dg_params, device)},
    {"basic_state", Key::kInt, offsetof(dg_params, basic_state)},
};

const Key *find_key(const std::string &k) {
  for (const Key &e : kKeys)
    if (k == e.name) return &e;
  return nullptr;
}

bool parse_int(const std::string &k, const std::string &v, int *out) {
  if (k == "precision" && (v == "fp64" || v == "mixed")) {
    *out = v == "fp64" ? DG_PREC_FP64 : DG_PREC_MIXED;
    return true;
  }
  if (k == "basic_state" && (v == "fft" || v == "elliptic")) {
    *out = v == "fft" ? DG_BASIC_FFT : DG_BASIC_ELLIPTIC;
    return true;
  }
  char *end = nullptr;
  errno = 0;
  long x = strtol(v.c_str(), &end, 10);
  if (errno || !end || *end || v.empty() || x < -2147483647L || x > 2147483647L) return false;
  *out = (int)x;
  return true;
}

bool parse_double(const std::string &v, double *out) {
  char *end = nullptr;
  errno = 0;
  double x = strtod(v.c_str(), &end);
  if (errno || !end || *end || v.empty()) return false;
  *out = x;
  return true;
}

int line_error(int lineno, const std::string &what) {
  dg_set_global_error("dg_params_read: line " + std::to_string(lineno) + ": " + what);
  return DG_ERR_INVALID;
}

}  // namespace

extern "C" {

int dg_params_write(const char *path, const dg_params *p, int n) {
  if (!path || n < 0 || (n > 0 && !p)) return DG_ERR_INVALID;
  FILE *f = fopen(path, "w");
  if (!f) {
    dg_set_global_error(std::string("dg_params_write: cannot open ") + path);
    return DG_ERR_INVALID;
  }
  fprintf(f, "# diskgpu parameter file: one disk per line, key=value (dg_params fields)\n");
  for (int d = 0; d < n; ++d) {
    const char *sep = "";
    for (const Key &e : kKeys) {
      const char *base = reinterpret_cast<const char *>(&p[d]) + e.off;
      if (e.kind == Key::kInt) fprintf(f, "%s%s=%d", sep, e.name, *reinterpret_cast<const int *>(base));
      else fprintf(f, "%s%s=%.17g", sep, e.name, *reinterpret_cast<const double *>(base));
      sep = " ";
    }
    fputc('\n', f);
  }
  const bool ok = !ferror(f);
  fclose(f);
  return ok ? DG_OK : DG_ERR_INVALID;
}

int dg_params_read(const char *path, dg_params *p, int max, int *n) {
  if (!path || !n || max < 0 || (max > 0 && !p)) return DG_ERR_INVALID;
  *n = 0;
  FILE *f = fopen(path, "r");
  if (!f) {
    dg_set_global_error(std::string("dg_params_read: cannot open ") + path);
    return DG_ERR_INVALID;
  }
  std::string line;
  int lineno = 0, count = 0, rc = DG_OK;
  char buf[4096];
  while (rc == DG_OK && fgets(buf, sizeof buf, f)) {
    line.assign(buf);
    ++lineno;
    if (line.size() == sizeof buf - 1 && line.back() != '\n') {
      rc = line_error(lineno, "line too long");
      break;
    }
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    // tokens key=value
    std::vector<std::pair<std::string, std::string>> kv;
    size_t i = 0;
    while (i < line.size()) {
      while (i < line.size() && isspace((unsigned char)line[i])) ++i;
      size_t j = i;
      while (j < line.size() && !isspace((unsigned char)line[j])) ++j;
      if (j > i) {
        const std::string tok = line.substr(i, j - i);
        const size_t eq = tok.find('=');
        if (eq == std::string::npos || eq == 0) {
          rc = line_error(lineno, "expected key=value, got '" + tok + "'");
          break;
        }
        kv.emplace_back(tok.substr(0, eq), tok.substr(eq + 1));
      }
      i = j;
    }
    if (rc || kv.empty()) continue;
    dg_params q;
    dg_params_default(&q);
    // sweep coordinates first: (Q_min, M_d/M_*, softening/r, Gamma) -> eps, gamma, S0, K
    double sw[3] = {NAN, NAN, NAN}, gam = q.gamma_gas;
    const char *swk[3] = {"Qmin", "mass_ratio", "soft_over_r"};
    int nsw = 0;
    for (auto &e : kv) {
      for (int s = 0; s < 3; ++s)
        if (e.first == swk[s]) {
          if (!parse_double(e.second, &sw[s])) rc = line_error(lineno, "bad value for " + e.first);
          ++nsw;
        }
      if (e.first == "gamma_gas" && !parse_double(e.second, &gam)) rc = line_error(lineno, "bad value for gamma_gas");
    }
    if (rc) break;
    if (nsw != 0 && nsw != 3) {
      rc = line_error(lineno, "Qmin, mass_ratio and soft_over_r go together");
      break;
    }
    if (nsw == 3) {
      int r = dg_params_physical(sw[0], sw[1], sw[2], gam, &q, nullptr);
      if (r) {
        rc = line_error(lineno, "dg_params_physical rejected the sweep point");
        break;
      }
    }
    for (auto &e : kv) {
      bool sweep_key = false;
      for (int s = 0; s < 3; ++s) sweep_key |= e.first == swk[s];
      if (sweep_key) continue;
      const Key *k = find_key(e.first);
      if (!k) {
        rc = line_error(lineno, "unknown key '" + e.first + "'");
        break;
      }
      char *base = reinterpret_cast<char *>(&q) + k->off;
      bool ok = k->kind == Key::kInt ? parse_int(e.first, e.second, reinterpret_cast<int *>(base))
                                     : parse_double(e.second, reinterpret_cast<double *>(base));
      if (!ok) {
        rc = line_error(lineno, "bad value for " + e.first);
        break;
      }
    }
    if (rc) break;
    if (count >= max) {
      rc = line_error(lineno, "more disks than the output array holds");
      break;
    }
    p[count++] = q;
  }
  fclose(f);
  *n = count;
  return rc;
}

}  // extern "C"
