// Continuous-batching request server: many independent VHCI(+PT2) solves of different sizes on one
// GPU.  Requests arrive over time; a request is admitted into one of `slots` worker threads once it
// has arrived, a slot is free and the device's free memory exceeds the reserve.  Each admitted
// request runs on its own context (own CUDA stream, cuBLAS/cuSOLVER handles and buffers), so the
// kernels of concurrent requests overlap on the device; a slot that finishes takes the next
// arrived request at once.  A request admitted while others run gets a lower CUDA stream priority
// than they have, so the block scheduler serves the earliest requests first (they finish about as
// fast as alone) and later ones run in the gaps.  A request that runs out of device memory releases everything and
// goes back to waiting until another request has finished (it fails only if it runs out of memory
// with nothing else running).  Optional per-request size limits reject a request whose basis or
// perturber space would grow past them, before the step that would build it.  There is no
// counterpart in the reference program, which solves one input per process.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "vhci_gpu.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Server {
  const vhci_request* reqs = nullptr;
  int nreq = 0;
  vhci_serve_opts so{};
  vhci_result* res = nullptr;
  double* energies = nullptr;
  Clock::time_point t0;

  std::mutex mu;
  std::condition_variable cv;
  std::deque<int> ready;           // arrived and waiting for a slot (arrival order)
  std::vector<int> order;          // requests sorted by arrival time
  size_t next_arrival = 0;
  int running = 0;
  int done = 0;
  std::set<int> oom_waiting;       // requests waiting to retry after running out of memory
  int in_flight_peak = 0;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

void solve_one(Server& S, int r, int worker, int priority) {
  const vhci_request& q = S.reqs[r];
  vhci_result& out = S.res[r];
  vhci_opts o;
  vhci_default_opts(&o);
  o.device = S.so.device;
  o.stream_priority = priority;
  o.max_basis = S.so.max_basis;
  o.max_pert = S.so.max_pert;
  out.n_energies = 0;
  out.n_pert = 0;
  out.message[0] = '\0';
  vhci_ctx* c = nullptr;
  int st = q.input_path ? vhci_create_from_file(q.input_path, &o, 0, &c)
                        : vhci_create(q.problem, &o, 0, &c);
  if (st == VHCI_OK) st = vhci_hci(c, nullptr, nullptr, nullptr);
  vhci_info info{};
  if (c) vhci_get_info(c, &info);
  out.n_basis = info.n_basis;
  if (st == VHCI_OK && info.pt2) {
    int64_t np = 0;
    st = vhci_pt2(c, info.eps2, nullptr, &np);
    out.n_pert = np;
  }
  if (st == VHCI_OK) {
    int ne = 0;
    vhci_get_energies(c, S.energies + (size_t)r * S.so.max_states, S.so.max_states, &ne);
    out.n_energies = ne;
  } else if (c) {
    vhci_last_error(c, out.message, sizeof(out.message));
  }
  out.status = st;
  out.worker = worker;
  if (c) vhci_destroy(c);
}

// Device memory available to a new request: free memory plus what the stream-ordered pool holds
// without using it (freed by finished requests, kept for reuse).
double available_bytes(int device) {
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  double avail = (double)freeb;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
      avail += (double)(reserved - used);
  }
  return avail;
}

void worker_loop(Server& S, int worker) {
  cudaSetDevice(S.so.device);
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (;;) {
    int r = -1;
    int priority = 0;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      for (;;) {
        if (S.done == S.nreq) return;
        // move arrived requests into the ready queue
        const double t = S.now();
        while (S.next_arrival < S.order.size() && S.reqs[S.order[S.next_arrival]].arrival_s <= t)
          S.ready.push_back(S.order[S.next_arrival++]);
        // admission: keep the reserve free, but never block when nothing else runs
        if (!S.ready.empty() &&
            (S.running == 0 || available_bytes(S.so.device) >= S.so.reserve_bytes)) {
          r = S.ready.front();
          S.ready.pop_front();
          // arrival-order priority: below every request already running (lower numbers run
          // first; the device has least - greatest + 1 levels, the last one is shared)
          if (S.so.fifo_priority) priority = std::min(least, greatest + S.running);
          ++S.running;
          S.in_flight_peak = std::max(S.in_flight_peak, S.running);
          S.res[r].t_admit = t;
          break;
        }
        // wait for the next arrival or a finished request (polls at most every 50 ms)
        double wait = 0.05;
        if (S.next_arrival < S.order.size())
          wait = std::min(wait, std::max(0.0, S.reqs[S.order[S.next_arrival]].arrival_s - t));
        S.cv.wait_for(lk, std::chrono::duration<double>(std::max(wait, 1e-4)));
      }
    }
    S.res[r].retries = 0;
    int solo_done = -1;  // S.done when this request last retried while all others were waiting
    for (;;) {
      solve_one(S, r, worker, priority);
      if (S.res[r].status != VHCI_E_OOM) break;
      // out of device memory (its buffers are already released): wait until another request
      // finishes; when every running request is waiting, the lowest-numbered one retries once,
      // and fails if that retry runs out of memory too with nothing finished in between
      std::unique_lock<std::mutex> lk(S.mu);
      if (S.running == 1) break;        // alone and still out of memory: report the failure
      if (solo_done == S.done) break;   // its solo retry failed as well: free the slot
      ++S.res[r].retries;
      const int done_before = S.done;
      S.oom_waiting.insert(r);
      S.cv.notify_all();
      S.cv.wait(lk, [&] {
        return S.done > done_before ||
               ((int)S.oom_waiting.size() == S.running && *S.oom_waiting.begin() == r);
      });
      solo_done = S.done > done_before ? -1 : S.done;
      S.oom_waiting.erase(r);
    }
    {
      std::lock_guard<std::mutex> lk(S.mu);
      S.res[r].t_done = S.now();
      --S.running;
      ++S.done;
    }
    S.cv.notify_all();
  }
}

}  // namespace

extern "C" {

void vhci_default_serve_opts(vhci_serve_opts* so) {
  std::memset(so, 0, sizeof(*so));
  so->device = 0;
  so->slots = 8;
  so->reserve_bytes = 8e9;
  so->max_states = 256;
  so->max_basis = 0;
  so->max_pert = 0;
  so->fifo_priority = 1;
}

vhci_status vhci_serve(const vhci_request* reqs, int nreq, const vhci_serve_opts* so,
                       vhci_result* results, double* energies, vhci_serve_summary* summary) {
  if (!reqs || nreq <= 0 || !results || !energies) return VHCI_E_INPUT;
  Server S;
  S.reqs = reqs;
  S.nreq = nreq;
  if (so) S.so = *so; else vhci_default_serve_opts(&S.so);
  if (S.so.slots < 1) S.so.slots = 1;
  if (S.so.max_states < 1) return VHCI_E_INPUT;
  S.res = results;
  S.energies = energies;
  for (int i = 0; i < nreq; ++i) {
    if (!reqs[i].input_path && !reqs[i].problem) return VHCI_E_INPUT;
    std::memset(&results[i], 0, sizeof(vhci_result));
    results[i].status = -1;
    S.order.push_back(i);
  }
  std::stable_sort(S.order.begin(), S.order.end(),
                   [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || S.so.device < 0 || S.so.device >= ndev)
    return VHCI_E_CUDA;
  S.t0 = Clock::now();
  std::vector<std::thread> th;
  for (int w = 0; w < S.so.slots; ++w) th.emplace_back(worker_loop, std::ref(S), w);
  for (auto& t : th) t.join();
  const double wall = S.now();
  int failed = 0;
  for (int i = 0; i < nreq; ++i) failed += results[i].status != VHCI_OK;
  if (summary) {
    summary->wall_s = wall;
    summary->completed = nreq - failed;
    summary->failed = failed;
    summary->peak_in_flight = S.in_flight_peak;
  }
  return failed ? VHCI_E_STATE : VHCI_OK;
}

}  // extern "C"
