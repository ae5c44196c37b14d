// batch.cu -- tile-shape autotuner and the batched ensemble: many
// independent droplet + impurity systems (any mix of grid sizes) advanced
// together, one CUDA graph launch per ensemble step.
//
// The reference runs one system per process; the ensemble has no reference
// counterpart and reuses the single-system step of every member unchanged
// (steprk.f90 / steppc.f90 through step_rk / step_pc).  Each ensemble-step
// graph forks from a master stream into every member's stream, holds that
// member's whole predictor-corrector step, and joins back, so the members'
// kernels overlap on the GPU: small grids that leave most SMs idle on their
// own fill the machine together.  A graph holds K consecutive ensemble
// steps (K = 30, 10, 5 or 1, the largest the remaining steps allow), so a
// run of 30 steps is one graph launch: each member's branch chains its K
// steps, and the branches run side by side.  The members' buffer states
// repeat with period 30 (the ψ buffers' rotation), so the graphs of one
// cycle are captured once and replayed.
#include <string.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace he4 {

// max of the step errors, the last means and a non-finite flag per member
__global__ void k_batch_acc(const double *__restrict__ scal, double *acc) {
  const int t = threadIdx.x;
  if (t < 3) acc[t] = fmax(acc[t], scal[t]);
  if (t < 12 && t >= 3) acc[t] = scal[t];
  if (t == 0) {
    bool bad = false;
    for (int i = 0; i < 12; i++) bad = bad || !isfinite(scal[i]);
    if (bad) acc[12] = 1.0;
  }
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
static int time_field(Handle *h, int reps, double *ms) {
  HE4_TRY(field_all(h));  // warm-up with the new tiles
  cudaEvent_t e0, e1;
  HE4_CUDA_TRY(cudaEventCreate(&e0));
  HE4_CUDA_TRY(cudaEventCreate(&e1));
  HE4_CUDA_TRY(cudaEventRecord(e0, h->stream));
  int rc = HE4_OK;
  for (int i = 0; i < reps && rc == HE4_OK; i++) rc = field_all(h);
  HE4_CUDA_TRY(cudaEventRecord(e1, h->stream));
  HE4_CUDA_TRY(cudaEventSynchronize(e1));
  float t = 0.f;
  HE4_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HE4_TRY(rc);
  *ms = t / reps;
  return HE4_OK;
}

static int apply_tiles(Handle *h, const int *t) {
  free_graphs(h);  // captured launches carry the old shapes
  return fft_set_tiles(h->fft, t);
}

// Coordinate search over the tile shapes of the three axes: for each axis
// the candidates are the register-path splits N = N1 * N2 or, on the generic
// path, 8..32 pencils per CTA; each candidate is timed as `reps` mean-field
// evaluations of the handle's current state with CUDA events, the fastest
// is kept before the next axis is searched.
static int tune(Handle *h, int reps, double *best_ms, int *best) {
  int cur[6];
  fft_get_tiles(h->fft, cur);
  double best_t = 0.0;
  HE4_TRY(time_field(h, reps, &best_t));
  for (int a = 0; a < 3; a++) {
    std::vector<int> cand;
    const bool reg = h->fft.n1[a] != 0;
    if (reg) {
      for (int n1 = 2; n1 <= 16; n1 *= 2) cand.push_back(n1);
    } else {
      for (int w = 8; w <= 32; w += 8) cand.push_back(w);
    }
    for (int c : cand) {
      int t[6];
      memcpy(t, cur, sizeof(t));
      if (reg)
        t[a] = c;
      else
        t[3 + a] = c;
      if (memcmp(t, cur, sizeof(t)) == 0) continue;
      if (apply_tiles(h, t) != HE4_OK) continue;  // not a valid shape for this length
      double ms = 0.0;
      HE4_TRY(time_field(h, reps, &ms));
      if (ms < best_t) {
        best_t = ms;
        memcpy(cur, t, sizeof(t));
      }
    }
    HE4_TRY(apply_tiles(h, cur));
  }
  HE4_TRY(field_all(h));
  *best_ms = best_t;
  memcpy(best, cur, sizeof(cur));
  return HE4_OK;
}

}  // namespace he4

using namespace he4;

// ---------------------------------------------------------------------------
// the ensemble
// ---------------------------------------------------------------------------
struct EnsembleGraph {
  std::vector<StepState> before, after;
  int ksteps = 1;  // ensemble steps per launch
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t kernels = 0;
};

struct he4_batch {
  std::vector<he4_handle *> m;
  int dev = 0;
  cudaStream_t master = nullptr;
  cudaEvent_t fork = nullptr;          // used inside captures only
  std::vector<cudaEvent_t> capjoin;    // used inside captures only
  std::vector<cudaEvent_t> join;       // ordering between streams outside captures
  double *acc = nullptr;   // device [n][16]
  double *hacc = nullptr;  // pinned mirror
  std::vector<EnsembleGraph> graphs;
  double dt = 0.0;
};

static void batch_free_graphs(he4_batch *b) {
  for (EnsembleGraph &g : b->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  b->graphs.clear();
}

static std::vector<StepState> batch_state(he4_batch *b, double dt) {
  std::vector<StepState> s;
  for (he4_handle *hh : b->m) s.push_back(get_step_state(&hh->h, dt));
  return s;
}

static bool same_state(const std::vector<StepState> &a, const std::vector<StepState> &b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); i++)
    if (!same_step_state(a[i], b[i])) return false;
  return true;
}

// one ensemble PC step captured from the current member states
static int batch_capture(he4_batch *b, double dt, int ksteps, EnsembleGraph *out) {
  EnsembleGraph g;
  g.ksteps = ksteps;
  g.before = batch_state(b, dt);
  std::vector<int64_t> l0, d0;
  for (he4_handle *hh : b->m) {
    l0.push_back(hh->h.launches);
    d0.push_back(hh->h.nsteps_done);
  }
  HE4_CUDA_TRY(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
  int rc = HE4_OK;
  cudaError_t ce = cudaEventRecord(b->fork, b->master);
  for (size_t i = 0; i < b->m.size() && rc == HE4_OK && ce == cudaSuccess; i++) {
    Handle *h = &b->m[i]->h;
    ce = cudaStreamWaitEvent(h->stream, b->fork, 0);
    if (ce != cudaSuccess) break;
    for (int s = 0; s < ksteps && rc == HE4_OK && ce == cudaSuccess; s++) {
      rc = step_pc(h, dt, h->scal);
      if (rc != HE4_OK) break;
      k_batch_acc<<<1, 32, 0, h->stream>>>(h->scal, b->acc + 16 * i);
      h->launches++;
      ce = cudaGetLastError();
    }
    if (rc != HE4_OK) break;
    if (ce == cudaSuccess) ce = cudaEventRecord(b->capjoin[i], h->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->master, b->capjoin[i], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(b->master, &graph);
  g.after = batch_state(b, dt);
  for (size_t i = 0; i < b->m.size(); i++) {
    Handle *h = &b->m[i]->h;
    g.kernels += h->launches - l0[i];
    h->launches = l0[i];
    h->nsteps_done = (int)d0[i];
    set_step_state(h, g.before[i]);
  }
  if (rc != HE4_OK || ce != cudaSuccess || ee != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (rc == HE4_OK) {
      set_error("ensemble capture: %s", cudaGetErrorString(ce != cudaSuccess ? ce : ee));
      rc = HE4_E_CUDA;
    }
    return rc;
  }
  g.graph = graph;
  const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
  if (ie != cudaSuccess) {
    cudaGraphDestroy(graph);
    set_error("ensemble graph instantiation: %s", cudaGetErrorString(ie));
    return HE4_E_CUDA;
  }
  *out = g;
  return HE4_OK;
}

// order stream b after everything issued so far on stream a
static int stream_after(cudaStream_t b, cudaStream_t a, cudaEvent_t ev) {
  HE4_CUDA_TRY(cudaEventRecord(ev, a));
  HE4_CUDA_TRY(cudaStreamWaitEvent(b, ev, 0));
  return HE4_OK;
}

extern "C" {

int he4_set_tiles(he4_handle *hh, const int32_t tiles[6]) {
  if (!hh || !tiles) {
    set_error("null argument");
    return HE4_E_ARG;
  }
  Handle *h = &hh->h;
  HE4_CUDA_TRY(cudaSetDevice(h->dev));
  int t[6];
  for (int i = 0; i < 6; i++) t[i] = tiles[i];
  return apply_tiles(h, t);
}

int he4_get_tiles(he4_handle *hh, int32_t tiles[6]) {
  if (!hh || !tiles) {
    set_error("null argument");
    return HE4_E_ARG;
  }
  int t[6];
  fft_get_tiles(hh->h.fft, t);
  for (int i = 0; i < 6; i++) tiles[i] = t[i];
  return HE4_OK;
}

int he4_tune(he4_handle *hh, int32_t reps, double *best_ms, int32_t tiles[6]) {
  if (!hh || reps < 1) {
    set_error("invalid arguments");
    return HE4_E_ARG;
  }
  Handle *h = &hh->h;
  HE4_CUDA_TRY(cudaSetDevice(h->dev));
  if (!h->have_state) {
    set_error("no state: call he4_set_state first");
    return HE4_E_STATE;
  }
  int t[6];
  double ms = 0.0;
  HE4_TRY(tune(h, reps, &ms, t));
  if (best_ms) *best_ms = ms;
  if (tiles)
    for (int i = 0; i < 6; i++) tiles[i] = t[i];
  return HE4_OK;
}

int he4_batch_create(int32_t n, const he4_params *params, he4_batch **out) {
  if (n < 1 || !params || !out) {
    set_error("he4_batch_create: invalid arguments");
    return HE4_E_ARG;
  }
  *out = nullptr;
  he4_batch *b = new (std::nothrow) he4_batch();
  if (!b) {
    set_error("host allocation failed");
    return HE4_E_NOMEM;
  }
  int rc = HE4_OK;
  for (int i = 0; i < n && rc == HE4_OK; i++) {
    if (params[i].device != params[0].device) {
      set_error("ensemble members must share one device");
      rc = HE4_E_ARG;
      break;
    }
    he4_handle *hh = nullptr;
    rc = he4_create(&params[i], &hh);
    if (rc == HE4_OK) b->m.push_back(hh);
  }
  if (rc == HE4_OK) {
    b->dev = params[0].device;
    cudaError_t e = cudaSetDevice(b->dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    b->join.resize(n, nullptr);
    b->capjoin.resize(n, nullptr);
    for (int i = 0; i < n && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
    for (int i = 0; i < n && e == cudaSuccess; i++)
      e = cudaEventCreateWithFlags(&b->capjoin[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&b->acc, sizeof(double) * 16 * n);
    if (e == cudaSuccess) e = cudaMallocHost(&b->hacc, sizeof(double) * 16 * n);
    if (e != cudaSuccess) {
      set_error("ensemble setup: %s", cudaGetErrorString(e));
      rc = HE4_E_CUDA;
    }
  }
  if (rc != HE4_OK) {
    he4_batch_destroy(b);
    return rc;
  }
  *out = b;
  return HE4_OK;
}

void he4_batch_destroy(he4_batch *b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->master) cudaStreamSynchronize(b->master);
  batch_free_graphs(b);
  for (he4_handle *hh : b->m) he4_destroy(hh);
  for (cudaEvent_t e : b->join)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : b->capjoin)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->acc) cudaFree(b->acc);
  if (b->hacc) cudaFreeHost(b->hacc);
  if (b->master) cudaStreamDestroy(b->master);
  delete b;
}

int32_t he4_batch_size(const he4_batch *b) { return b ? (int32_t)b->m.size() : 0; }

he4_handle *he4_batch_member(he4_batch *b, int32_t i) {
  if (!b || i < 0 || i >= (int32_t)b->m.size()) return nullptr;
  return b->m[i];
}

int he4_batch_tune(he4_batch *b, int32_t reps, int32_t *tiles, double *ms) {
  if (!b || reps < 1) {
    set_error("invalid arguments");
    return HE4_E_ARG;
  }
  HE4_CUDA_TRY(cudaSetDevice(b->dev));
  batch_free_graphs(b);
  const int n = (int)b->m.size();
  std::vector<int> done(n, 0);
  for (int i = 0; i < n; i++) {
    if (done[i]) continue;
    Handle *h = &b->m[i]->h;
    if (!h->have_state) {
      set_error("member %d has no state", i);
      return HE4_E_STATE;
    }
    int t[6];
    double best = 0.0;
    HE4_TRY(tune(h, reps, &best, t));
    for (int j = i; j < n; j++) {
      Handle *g = &b->m[j]->h;
      if (g->nx != h->nx || g->ny != h->ny || g->nz != h->nz) continue;
      if (j != i) HE4_TRY(apply_tiles(g, t));
      done[j] = 1;
      if (tiles)
        for (int k = 0; k < 6; k++) tiles[6 * j + k] = t[k];
      if (ms) ms[j] = best;
    }
  }
  return HE4_OK;
}

int he4_batch_run(he4_batch *b, int32_t nsteps, double deltat, double *err_max, double *means) {
  if (!b || nsteps < 0 || !isfinite(deltat)) {
    set_error("he4_batch_run: invalid arguments");
    return HE4_E_ARG;
  }
  HE4_CUDA_TRY(cudaSetDevice(b->dev));
  const int n = (int)b->m.size();
  for (int i = 0; i < n; i++)
    if (!b->m[i]->h.have_state) {
      set_error("member %d has no state", i);
      return HE4_E_STATE;
    }
  if (deltat != b->dt) {
    batch_free_graphs(b);
    b->dt = deltat;
  }
  HE4_CUDA_TRY(cudaMemsetAsync(b->acc, 0, sizeof(double) * 16 * n, b->master));
  for (int i = 0; i < n; i++) HE4_TRY(stream_after(b->m[i]->h.stream, b->master, b->join[i]));
  int s = 0;
  // RK-Gill starter, member by member on the members' own streams
  for (; s < nsteps; s++) {
    bool any = false;
    for (int i = 0; i < n; i++) {
      Handle *h = &b->m[i]->h;
      if (h->nsteps_done >= 3) continue;
      any = true;
      HE4_TRY(step_rk(h, deltat, h->scal));
      k_batch_acc<<<1, 32, 0, h->stream>>>(h->scal, b->acc + 16 * i);
      h->launches++;
      HE4_CUDA_TRY(cudaGetLastError());
    }
    if (!any) break;
  }
  for (int i = 0; i < n; i++) HE4_TRY(stream_after(b->master, b->m[i]->h.stream, b->join[i]));
  // predictor-corrector steps: one graph launch per ensemble step
  for (; s < nsteps; s++) {
    for (int i = 0; i < n; i++)
      if (!b->m[i]->h.field_valid) {
        // a member whose field is stale (set_state without a step): evaluate
        // it on its own stream before the first graph
        Handle *h = &b->m[i]->h;
        HE4_TRY(stream_after(h->stream, b->master, b->join[i]));
        HE4_TRY(field_all(h));
        HE4_TRY(stream_after(b->master, h->stream, b->join[i]));
      }
    const std::vector<StepState> now = batch_state(b, deltat);
    const int left = nsteps - s;
    const int ks = left >= 30 ? 30 : left >= 10 ? 10 : left >= 5 ? 5 : 1;
    EnsembleGraph *hit = nullptr;
    for (EnsembleGraph &g : b->graphs)
      if (g.ksteps == ks && same_state(g.before, now)) {
        hit = &g;
        break;
      }
    if (!hit) {
      if (b->graphs.size() >= 64) batch_free_graphs(b);
      EnsembleGraph g;
      HE4_TRY(batch_capture(b, deltat, ks, &g));
      b->graphs.push_back(g);
      hit = &b->graphs.back();
    }
    HE4_CUDA_TRY(cudaGraphLaunch(hit->exec, b->master));
    s += hit->ksteps - 1;  // the loop adds the last one
    for (int i = 0; i < n; i++) {
      Handle *h = &b->m[i]->h;
      set_step_state(h, hit->after[i]);
      h->nsteps_done += hit->ksteps;
      h->field_valid = 1;
      h->split_valid = 0;
      h->forces_full = 0;
    }
    int64_t per = hit->kernels / (n ? n : 1);
    for (int i = 0; i < n; i++) b->m[i]->h.launches += per;
  }
  // later per-member calls run after the ensemble's work
  for (int i = 0; i < n; i++) HE4_TRY(stream_after(b->m[i]->h.stream, b->master, b->join[i]));
  HE4_CUDA_TRY(cudaMemcpyAsync(b->hacc, b->acc, sizeof(double) * 16 * n, cudaMemcpyDeviceToHost, b->master));
  HE4_CUDA_TRY(cudaStreamSynchronize(b->master));
  int bad = -1;
  for (int i = 0; i < n; i++) {
    const double *a = b->hacc + 16 * i;
    if (err_max) memcpy(err_max + 3 * i, a, 3 * sizeof(double));
    if (means) memcpy(means + 9 * i, a + 3, 9 * sizeof(double));
    if (a[12] != 0.0 && bad < 0) bad = i;
  }
  if (bad >= 0) {
    set_error("non-finite errors or means in ensemble member %d", bad);
    return HE4_E_NONFINITE;
  }
  return HE4_OK;
}

int64_t he4_batch_launch_count(const he4_batch *b) {
  if (!b) return -1;
  int64_t s = 0;
  for (he4_handle *hh : b->m) s += hh->h.launches;
  return s;
}

}  // extern "C"
