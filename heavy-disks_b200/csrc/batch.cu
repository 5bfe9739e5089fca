// Batched sweeps: many independent disks (heterogeneous grids and parameters) advanced
// together by one CUDA graph per launch.  Mixed-precision disks that share a grid, a
// Gamma class (Gamma = 2 or not), a hydro kernel form, product pipeline depths and a step
// rate within a factor 2^(1/4) form a group: one launch per kernel advances the whole group (mixed.cu, disk groups), the disk
// in blockIdx.z.  Every other disk is a branch of its own, holding its single-disk steps.
// The graph forks one branch per group or lone disk from a root stream, each on its own
// stream, so the branches overlap on the GPU, and joins back.  Every disk keeps its own
// device-resident dt, time and record ring (dg::Ctl); a disk that reaches tlim turns the
// rest of its launches into pass-throughs.  Branches whose disks have a smaller dt get
// proportionally more steps per launch so that the branches finish together.
// Grouping covers the dense-product grids by default.  1024^2 disks step as one branch
// each unless DISKGPU_BATCH_GROUPS=all: their lone step already fills the GPU, and
// separate branches overlap one disk's transforms with another's hydro and keep each
// disk's row-tile hand-over, which measured faster than the grouped kernels (2.05e10
// against 1.93e10 zone-updates/s for 16 disks).  DISKGPU_BATCH_GROUPS=0 turns grouping
// off (every disk its own branch).  DISKGPU_BATCH_GRAPH=0 enqueues each launch's kernels
// directly on the branches' streams instead of replaying the captured graph (the same
// kernels, fork and join; for profilers that see only kernels launched outside graphs).
// DISKGPU_BATCH_LANES=K keeps at most K branches of a launch in flight (branch q starts
// when branch q - K ends), to bound a launch's working set.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.h"

struct dg_batch {
  std::vector<dg_handle *> disks;
  std::vector<int> steps_per_launch;
  cudaStream_t root = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<cudaEvent_t> events;
  std::vector<MixedGroup *> groups;  // the groups the captured graph launches
  std::vector<std::vector<int>> branches;  // disks of each branch (a group or one disk)
  bool prepared = false;  // branches, groups and (unless direct) the graph are built
  bool direct = false;    // DISKGPU_BATCH_GRAPH=0: launch the branches' kernels without a graph
  int lanes = 0;          // branches in flight at once (0: all); DISKGPU_BATCH_LANES
  int dev = -1;
  std::string err;
  int fail(int code, const char *what, const char *why) {
    err = std::string(what) + ": " + (why ? why : "");
    return code;
  }
  void release_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    for (MixedGroup *g : groups) mixed_group_destroy(g);
    groups.clear();
    branches.clear();
    prepared = false;
  }
};

#define BK(call)                                                                       \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) return b->fail(DG_ERR_CUDA, #call, cudaGetErrorString(e_)); \
  } while (0)

// One launch's work: root -> fork to every branch's stream -> its steps -> join.  Recorded
// once into the batch's graph, or (direct mode) enqueued as it is at every launch.
static int batch_enqueue(dg_batch *b) {
  const int n = (int)b->disks.size();
  cudaError_t e = cudaEventRecord(b->events[n], b->root);
  if (e != cudaSuccess) return b->fail(DG_ERR_CUDA, "dg_batch_advance", cudaGetErrorString(e));
  size_t gi = 0;
  for (size_t q = 0; q < b->branches.size(); ++q) {
    const std::vector<int> &br = b->branches[q];
    dg_handle *h = b->disks[br[0]];
    int steps = 0;
    for (int k : br) steps = std::max(steps, b->steps_per_launch[k]);
    // with lanes, branch q follows branch q - lanes (its lane's previous one) instead of
    // starting at the fork, so at most `lanes` branches are in flight at once
    const size_t lanes = b->lanes > 0 ? (size_t)b->lanes : b->branches.size();
    cudaStreamWaitEvent(h->st, q < lanes ? b->events[n] : b->events[q - lanes], 0);
    int rc = DG_OK;
    if (br.size() > 1) {
      MixedGroup *grp = b->groups[gi++];
      for (int s = 0; s < steps && !rc; ++s) rc = mixed_group_enqueue_step(grp, h->st);
    } else {
      for (int s = 0; s < steps && !rc; ++s) rc = h->enqueue_step();
    }
    if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
    cudaEventRecord(b->events[q], h->st);
    cudaStreamWaitEvent(b->root, b->events[q], 0);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return b->fail(DG_ERR_CUDA, "dg_batch_advance", cudaGetErrorString(e));
  return DG_OK;
}

extern "C" {

int dg_batch_create(int n, const dg_params *params, dg_batch **out) {
  if (n < 1 || !params || !out) return DG_ERR_INVALID;
  *out = nullptr;
  dg_batch *b = new (std::nothrow) dg_batch();
  if (!b) return DG_ERR_NOMEM;
  for (int k = 0; k < n; ++k) {
    if (k > 0 && params[k].device != params[0].device) {
      delete b;
      return DG_ERR_INVALID;
    }
    dg_handle *h = nullptr;
    int rc = dg_create(&params[k], &h);
    if (rc) {
      for (dg_handle *d : b->disks) dg_destroy(d);
      delete b;
      return rc;
    }
    b->disks.push_back(h);
  }
  b->dev = b->disks[0]->dev;
  cudaSetDevice(b->dev);
  if (cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) != cudaSuccess) {
    for (dg_handle *d : b->disks) dg_destroy(d);
    delete b;
    return DG_ERR_CUDA;
  }
  b->events.resize(n + 1);
  for (auto &e : b->events) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  *out = b;
  return DG_OK;
}

void dg_batch_destroy(dg_batch *b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->root) cudaStreamSynchronize(b->root);
  b->release_graph();
  for (auto &e : b->events) cudaEventDestroy(e);
  for (dg_handle *d : b->disks) dg_destroy(d);
  if (b->root) cudaStreamDestroy(b->root);
  delete b;
}

const char *dg_batch_last_error(const dg_batch *b) { return b ? b->err.c_str() : ""; }

int dg_batch_size(const dg_batch *b) { return b ? (int)b->disks.size() : 0; }

dg_handle *dg_batch_disk(dg_batch *b, int k) {
  if (!b || k < 0 || k >= (int)b->disks.size()) return nullptr;
  return b->disks[k];
}

int dg_batch_init_standard(dg_batch *b) {
  if (!b) return DG_ERR_INVALID;
  for (dg_handle *h : b->disks) {
    int rc = dg_init_standard(h);
    if (rc) return b->fail(rc, "dg_batch_init_standard", dg_last_error(h));
  }
  b->release_graph();
  return DG_OK;
}

int dg_batch_advance(dg_batch *b, double tlim, double cfl, double dtout, int steps_per_launch, dg_record *rec,
                     int max_rec_per_disk, int *n_rec, double *t_out, long long *nsteps_out) {
  if (!b || !(cfl > 0) || !(dtout > 0) || steps_per_launch < 2 || (max_rec_per_disk > 0 && !rec)) return DG_ERR_INVALID;
  BK(cudaSetDevice(b->dev));
  const int n = (int)b->disks.size();
  std::vector<int> nout(n, 0);
  // per-disk loop set-up, as dg_advance does for one disk
  for (int k = 0; k < n; ++k) {
    dg_handle *h = b->disks[k];
    if (!h->have_state) return b->fail(DG_ERR_STATE, "dg_batch_advance", "a disk has no state");
    int rc = h->sync_from_device();
    if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
    if (h->cur != 0) {  // the graph assumes every disk starts on ping-pong buffer 0
      rc = h->set_ctl_fields(h->t, tlim, cfl, 0.0, h->tnext, dtout, 0);
      if (!rc) rc = h->cfl_launch(0, 0);
      if (!rc) rc = h->run_chunk(1);
      if (!rc) rc = h->read_ctl();
      if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
      h->t = h->hctl->t;
      h->nsteps = h->hctl->step;
    }
    rc = h->set_ctl_fields(h->t, tlim, cfl, 0.0, h->tnext, dtout, 0);
    if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
    BK(cudaMemsetAsync(&h->ctl->nrec, 0, sizeof(int), h->st));
    const bool first = (h->t < tlim) && (h->t >= h->tnext - 1e-12);
    rc = h->cfl_launch(0, first ? 1 : 0);
    if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
    rc = h->read_ctl();
    if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
  }
  // steps per launch: proportional to each disk's step rate (1/dt), even, at least 2
  if (!b->prepared) {
    double dtmin = 1e300;
    for (dg_handle *h : b->disks) dtmin = std::min(dtmin, h->hctl->dt > 0 ? h->hctl->dt : 1e300);
    b->steps_per_launch.assign(n, steps_per_launch);
    double dtmax = 0;
    for (dg_handle *h : b->disks) dtmax = std::max(dtmax, h->hctl->dt);
    for (int k = 0; k < n; ++k) {
      double ratio = (b->disks[k]->hctl->dt > 0) ? dtmin / b->disks[k]->hctl->dt : 1.0;
      int s = (int)std::lround(steps_per_launch * ratio);
      s = std::max(2, s + (s & 1));
      b->steps_per_launch[k] = s;
    }
    // branches: groups of same-grid mixed disks, and lone disks
    std::vector<std::vector<int>> &branches = b->branches;
    branches.clear();
    {
      const char *ge = getenv("DISKGPU_BATCH_GROUPS");
      const bool grouping = !(ge && strcmp(ge, "0") == 0);
      const bool group_fused = ge && strcmp(ge, "all") == 0;
      std::map<std::string, std::vector<int>> by_key;
      for (int k = 0; k < n; ++k) {
        std::string key = grouping ? mixed_group_key(b->disks[k], group_fused) : std::string();
        if (key.empty()) {
          branches.emplace_back(1, k);
          continue;
        }
        // step-rate class: a group's disks all take the group's (largest) step count per
        // launch, so members are within a factor 2^(1/4) of each other's rate and few of
        // their steps are pass-throughs
        key += ":" + std::to_string((int)std::floor(4.0 * std::log2((double)b->steps_per_launch[k])));
        by_key[key].push_back(k);
      }
      for (auto &kv : by_key) {
        if (kv.second.size() == 1) {
          branches.emplace_back(1, kv.second[0]);
          continue;
        }
        std::vector<dg_handle *> members;
        for (int k : kv.second) members.push_back(b->disks[k]);
        std::string why;
        MixedGroup *grp = mixed_group_create(members, &why);
        if (!grp) return b->fail(DG_ERR_CUDA, "dg_batch_advance", why.c_str());
        b->groups.push_back(grp);
        branches.emplace_back(std::move(kv.second));
      }
    }
    {
      // the branches with the most work (zones x steps per launch) are enqueued first
      std::vector<std::pair<std::vector<int>, MixedGroup *>> order;
      size_t gi = 0;
      for (auto &br : branches) order.emplace_back(br, br.size() > 1 ? b->groups[gi++] : nullptr);
      auto work = [&](const std::vector<int> &br) {
        double w = 0;
        int steps = 0;
        for (int k : br) steps = std::max(steps, b->steps_per_launch[k]);
        for (int k : br) w += (double)b->disks[k]->p.Nu * b->disks[k]->p.Nphi;
        return w * steps;
      };
      std::stable_sort(order.begin(), order.end(),
                       [&](const auto &x, const auto &y) { return work(x.first) > work(y.first); });
      branches.clear();
      b->groups.clear();
      for (auto &o : order) {
        branches.push_back(o.first);
        if (o.second) b->groups.push_back(o.second);
      }
    }
    for (dg_handle *h : b->disks) {
      int rc0 = h->prof_collect();
      if (rc0) return b->fail(rc0, "dg_batch_advance", h->err.c_str());
      h->prof_on = false;  // no event timing inside the batch's launches
    }
    const char *gv = getenv("DISKGPU_BATCH_GRAPH");
    b->direct = gv && strcmp(gv, "0") == 0;
    const char *lv = getenv("DISKGPU_BATCH_LANES");
    b->lanes = lv ? std::max(0, atoi(lv)) : 0;
    if (!b->direct) {
      // capture one launch's work as a graph
      cudaGraph_t g = nullptr;
      BK(cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal));
      int rc = batch_enqueue(b);
      cudaError_t e = cudaStreamEndCapture(b->root, &g);
      for (dg_handle *h : b->disks) h->cur = 0;  // capture flipped the buffers an even number of times
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      BK(e);
      e = cudaGraphInstantiate(&b->exec, g, 0);
      cudaGraphDestroy(g);
      BK(e);
    }
    b->prepared = true;
  }
  std::vector<double> tmp;
  for (;;) {
    // read every control block with one synchronisation
    for (dg_handle *h : b->disks)
      BK(cudaMemcpyAsync(h->hctl, h->ctl, offsetof(dg::Ctl, rec), cudaMemcpyDeviceToHost, b->root));
    BK(cudaStreamSynchronize(b->root));
    bool running = false;
    for (int k = 0; k < n; ++k) {
      dg_handle *h = b->disks[k];
      const int nr = h->hctl->nrec;
      if (nr > 0) {
        tmp.resize((size_t)nr * 4);
        BK(cudaMemcpy(tmp.data(), &h->ctl->rec[0][0], (size_t)nr * 4 * sizeof(double), cudaMemcpyDeviceToHost));
        BK(cudaMemset(&h->ctl->nrec, 0, sizeof(int)));
        for (int q = 0; q < nr; ++q) {
          if (nout[k] < max_rec_per_disk) {
            dg_record &r = rec[(size_t)k * max_rec_per_disk + nout[k]];
            r.t = tmp[4 * q]; r.c0 = tmp[4 * q + 1]; r.c2 = tmp[4 * q + 2]; r.arg2 = tmp[4 * q + 3];
          }
          ++nout[k];
        }
      }
      h->t = h->hctl->t;
      h->nsteps = h->hctl->step;
      int rc = h->check_status();
      if (rc) return b->fail(rc, "dg_batch_advance", h->err.c_str());
      if (h->t < tlim) running = true;
    }
    if (!running) break;
    if (b->direct) {
      int rc = batch_enqueue(b);  // every step count is even: each disk ends on buffer 0
      if (rc) return rc;
    } else {
      BK(cudaGraphLaunch(b->exec, b->root));
    }
  }
  for (int k = 0; k < n; ++k) {
    dg_handle *h = b->disks[k];
    h->tnext = h->hctl->tnext;
    if (n_rec) n_rec[k] = std::min(nout[k], max_rec_per_disk);
    if (t_out) t_out[k] = h->t;
    if (nsteps_out) nsteps_out[k] = h->nsteps;
  }
  return DG_OK;
}

}  // extern "C"
