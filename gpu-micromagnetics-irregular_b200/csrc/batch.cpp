// batch.cpp — many independent LLG instances of uneven size on one GPU.
//
// The reference runs one geometry per process.  Here a batch owns one
// context per instance, each on its own CUDA stream, and integrates them
// concurrently: a pool of host threads takes instances largest-first (cells
// as the cost estimate, longest-processing-time order) and drives each
// instance's integrator on its stream, so the kernels of small instances
// overlap on the GPU instead of serialising behind each other's host syncs.
// On a context's own stream the demag chain is replayed as a captured CUDA
// graph, and every demag plan picks its transform launch shapes by timing
// (k_demag.cu, autotune; cached per transform size, so instances of one size
// tune once).
//
// llg_batch_integrate_graph is the single-launch form: every instance's
// device-resident step loop (BDF attempts, Newton and Arnoldi iterations as
// CUDA graph WHILE / IF nodes driven by control kernels, integrator_dev.cu)
// is captured as an independent branch of ONE graph, and one cudaGraphLaunch
// advances all instances to tout; the host only writes each instance's
// (tout, yout) before the launch and reads its state back after it.
#include <algorithm>
#include <atomic>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "llg_internal.h"

struct llg_batch {
  std::vector<llg_ctx*> ctx;
  std::vector<cudaStream_t> streams;
  int device = 0;
  // single-graph form
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  std::vector<DevInteg*> devs;
};

int integrator_batch_prepare(llg_ctx* c, DevInteg** d_out, DState* hs_out);
int integrator_batch_sync(llg_ctx* c);
int integrator_batch_finish(llg_ctx* c, const DState& hs, double* tret);
int demag_check_last(llg_ctx* c);

extern "C" {

int llg_batch_create(int32_t n, const llg_params* params, llg_batch** out) {
  if (!out || n < 1 || !params) { llg_set_error("llg_batch_create: bad argument"); return LLG_ERR_ARG; }
  *out = nullptr;
  llg_batch* b = new llg_batch();
  cudaGetDevice(&b->device);
  for (int i = 0; i < n; i++) {
    llg_ctx* c = nullptr;
    int rc = llg_create(&params[i], &c);
    cudaStream_t s = nullptr;
    if (!rc && cudaStreamCreate(&s) != cudaSuccess) {
      llg_destroy(c);
      llg_set_error("llg_batch_create: stream creation failed");
      rc = LLG_ERR_CUDA;
    }
    if (rc) {
      llg_batch_destroy(b);
      return rc;
    }
    llg_set_stream(c, s);
    b->ctx.push_back(c);
    b->streams.push_back(s);
  }
  *out = b;
  return 0;
}

int llg_batch_size(const llg_batch* b) { return b ? (int)b->ctx.size() : 0; }

llg_ctx* llg_batch_ctx(llg_batch* b, int32_t i) {
  if (!b || i < 0 || i >= (int)b->ctx.size()) return nullptr;
  return b->ctx[i];
}

int llg_batch_integrator_init(llg_batch* b, double t0, const double* const* d_y0, const llg_solver_opts* o) {
  if (!b || !d_y0 || !o) return LLG_ERR_ARG;
  // the caller's y0 may still be in flight on the legacy default stream
  if (cudaDeviceSynchronize() != cudaSuccess) { llg_set_error("llg_batch_integrator_init: device sync"); return LLG_ERR_CUDA; }
  for (size_t i = 0; i < b->ctx.size(); i++) {
    const int rc = llg_integrator_init(b->ctx[i], t0, d_y0[i], o);
    if (rc) return rc;
  }
  return 0;
}

int llg_batch_integrate(llg_batch* b, double tout, double* const* d_yout, int32_t nthreads, int32_t* rcs) {
  if (!b || !d_yout) return LLG_ERR_ARG;
  const int n = (int)b->ctx.size();
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->ctx[a]->ncell > b->ctx[c]->ncell; });
  std::vector<int> rc(n, 0);
  std::atomic<int> next{0};
  std::vector<std::string> errs(n);
  auto worker = [&]() {
    cudaSetDevice(b->device);
    for (;;) {
      const int k = next.fetch_add(1);
      if (k >= n) break;
      const int i = order[k];
      double tret = 0.0;
      rc[i] = llg_integrate(b->ctx[i], tout, d_yout[i], &tret);
      if (rc[i]) errs[i] = llg_last_error();
      if (!rc[i] && cudaStreamSynchronize(b->streams[i]) != cudaSuccess) rc[i] = LLG_ERR_CUDA;
    }
  };
  const int nt = std::max(1, std::min(nthreads > 0 ? nthreads : n, n));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; t++) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  int first = 0;
  for (int i = 0; i < n; i++) {
    if (rcs) rcs[i] = rc[i];
    if (rc[i] && !first) {
      first = rc[i];
      llg_set_error("instance " + std::to_string(i) + ": " + errs[i]);
    }
  }
  return first;
}

int llg_batch_integrate_graph(llg_batch* b, double tout, double* const* d_yout, int32_t* rcs) {
  if (!b || !d_yout) return LLG_ERR_ARG;
  const int n = (int)b->ctx.size();
  for (int i = 0; i < n; i++)
    if (b->streams[i] && cudaStreamSynchronize(b->streams[i]) != cudaSuccess) {
      llg_set_error("llg_batch_integrate_graph: instance stream failed");
      return LLG_ERR_CUDA;
    }
  if (!b->gexec) {
    std::vector<DState> hs(n);
    std::vector<DevInteg*> ds(n, nullptr);
    for (int i = 0; i < n; i++) {
      const int rc = integrator_batch_prepare(b->ctx[i], &ds[i], &hs[i]);
      if (rc) {
        llg_set_error("instance " + std::to_string(i) + ": " + llg_last_error());
        return rc;
      }
    }
    std::vector<const DState*> hp(n);
    for (int i = 0; i < n; i++) hp[i] = &hs[i];
    const int rc = devint_build_batch(b->ctx.data(), ds.data(), hp.data(), n, &b->gexec);
    if (rc) return rc;
    b->devs = ds;
    if (!b->gstream && cudaStreamCreateWithFlags(&b->gstream, cudaStreamNonBlocking) != cudaSuccess) {
      llg_set_error("llg_batch_integrate_graph: stream creation failed");
      return LLG_ERR_CUDA;
    }
  }
  for (int i = 0; i < n; i++) {
    const int rc = integrator_batch_sync(b->ctx[i]);   // after host-path steps: upload the state
    if (rc) return rc;
  }
  for (int i = 0; i < n; i++) {
    const int rc = devint_batch_args(b->devs[i], b->ctx[i], tout, d_yout[i], b->gstream);
    if (rc) return rc;
  }
  if (cudaGraphLaunch(b->gexec, b->gstream) != cudaSuccess) {
    llg_set_error("llg_batch_integrate_graph: graph launch failed");
    return LLG_ERR_CUDA;
  }
  for (int i = 0; i < n; i++) {
    const int rc = devint_batch_fetch(b->devs[i], b->ctx[i], b->gstream);
    if (rc) return rc;
  }
  if (cudaStreamSynchronize(b->gstream) != cudaSuccess) {
    llg_set_error(std::string("llg_batch_integrate_graph: ") + cudaGetErrorString(cudaGetLastError()));
    return LLG_ERR_CUDA;
  }
  int first = 0;
  for (int i = 0; i < n; i++) {
    DState hs;
    devint_batch_collect(b->devs[i], b->ctx[i], hs);
    double tret = 0.0;
    int rc = integrator_batch_finish(b->ctx[i], hs, &tret);
    const int dc = demag_check_last(b->ctx[i]);
    if (dc) rc = dc;
    if (rcs) rcs[i] = rc;
    if (rc && !first) {
      first = rc;
      llg_set_error("instance " + std::to_string(i) + ": step graph returned " + std::to_string(rc));
    }
  }
  return first;
}

int llg_partition_lpt(int32_t n, const double* cost, int32_t nparts, int32_t* part_of, double* load) {
  if (n < 0 || nparts < 1 || (n > 0 && (!cost || !part_of))) {
    llg_set_error("llg_partition_lpt: bad argument");
    return LLG_ERR_ARG;
  }
  for (int i = 0; i < n; i++)
    if (!(cost[i] >= 0.0)) { llg_set_error("llg_partition_lpt: costs must be >= 0"); return LLG_ERR_ARG; }
  // longest processing time first: items by decreasing cost (ties: lower
  // index first), each to the part with the smallest load so far (ties:
  // lower part); deterministic, within 4/3 of the optimal makespan
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost[a] > cost[c]; });
  std::vector<double> ld(nparts, 0.0);
  for (int k = 0; k < n; k++) {
    const int i = order[k];
    int best = 0;
    for (int r = 1; r < nparts; r++)
      if (ld[r] < ld[best]) best = r;
    part_of[i] = best;
    ld[best] += cost[i];
  }
  if (load)
    for (int r = 0; r < nparts; r++) load[r] = ld[r];
  return 0;
}

void llg_batch_destroy(llg_batch* b) {
  if (!b) return;
  if (b->gstream) cudaStreamSynchronize(b->gstream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->gstream) cudaStreamDestroy(b->gstream);
  for (size_t i = 0; i < b->ctx.size(); i++) {
    if (b->streams[i]) cudaStreamSynchronize(b->streams[i]);
    llg_destroy(b->ctx[i]);
    if (b->streams[i]) cudaStreamDestroy(b->streams[i]);
  }
  delete b;
}

}  // extern "C"
