// The serving loop: continuous batching of 0-D reactors and 1-D shock tubes on one GPU.
//
// Requests arrive on a timeline.  A request is admitted as soon as it has arrived, a slot of its
// kind is free and (tubes) its state fits in the device pool; its state is then set up on the
// device and stays resident until it finishes.  Every iteration of the loop launches one batched
// kernel per kind over all admitted cases (reactors: a bounded number of ROK4E attempts each;
// tubes: a bounded number of RK3 steps each, one CTA per tube) on two streams, so the kinds
// overlap on the device.  The kinds are independent: whenever one kind's launch comes back, the
// host reads its per-case progress words, retires its finished cases (their slots and memory
// return to the pool, their results are copied out), admits its new arrivals and launches it
// again, while the other kind's launch may still run.  A request's latency is its completion time minus its arrival time on the host
// clock.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <thread>
#include <vector>
#include "batch.h"
#include "cb200_serve.h"

namespace cb2 {
const Param *ctx_param(const cb2_ctx *ctx);
}

using namespace cb2;

namespace {

// First-fit allocator over one device allocation (offsets in bytes, 256-byte granules).
struct Pool {
  char *base = nullptr;
  size_t size = 0, used = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  int init(size_t bytes) {
    size = (bytes + 255) & ~size_t(255);
    if (size == 0 || cudaMalloc(&base, size) != cudaSuccess) return CB2_ERR_NOMEM;
    free_[0] = size;
    return CB2_OK;
  }
  void *alloc(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        const size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > bytes) free_[off + bytes] = len - bytes;
        used += bytes;
        return base + off;
      }
    }
    return nullptr;
  }
  void release(void *p, size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    const size_t off = (size_t)((char *)p - base);
    used -= bytes;
    size_t start = off, len = bytes;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + bytes == next->first) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        start = prev->first;
        len += prev->second;
        free_.erase(prev);
      }
    }
    free_[start] = len;
  }
  void destroy() {
    if (base) cudaFree(base);
    base = nullptr;
  }
};

// Arrays of one tube on the compact line: cv, qn (NV each), bv (6), sv (NS), metric (9), jac,
// gamma, acoustic, rts over the padded line; dq (NV) over the interior.  Each array starts on a
// 256-byte boundary.
size_t line_bytes(int mx, int g, int ns) {
  const size_t n = (size_t)mx + 2 * g, nv = 5 + ns;
  auto up = [](size_t c) { return (c + 31) & ~size_t(31); };
  return sizeof(double) * (2 * up(n * nv) + up(n * 6) + up(n * ns) + up(n * 9) + 4 * up(n) + up((size_t)mx * nv));
}

void carve_line(char *mem, int mx, int g, int ns, Zone &z) {
  std::memset(&z, 0, sizeof(z));
  z.mx = mx; z.my = 1; z.mz = 1; z.ngg = g;
  z.L = make_layout_1d(mx, g);
  z.L0 = make_layout_1d(mx, 0);
  z.L1 = make_layout_1d(mx, 1);
  const size_t n = (size_t)mx + 2 * g, nv = 5 + ns;
  double *p = (double *)mem;
  auto take = [&](size_t cnt) {
    double *r = p;
    p += (cnt + 31) & ~size_t(31);
    return r;
  };
  z.cv = take(n * nv);
  z.qn = take(n * nv);
  z.bv = take(n * 6);
  z.sv = take(n * ns);
  z.metric = take(n * 9);
  z.jac = take(n);
  z.gamma = take(n);
  z.acoustic = take(n);
  z.rts = take(n);
  z.dq = take((size_t)mx * nv);
}

double now_s(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

namespace {

// Device and pinned host resources of one run, released in the destructor.
struct Run {
  Pool pool;
  cb2_reactor *d_reac = nullptr, *h_reac = nullptr;
  LineCase *d_line = nullptr, *h_line = nullptr;
  double *d_in = nullptr;  // per reactor slot: T0, p0, t_end, Y[]; then the tube composition
  double *h_in = nullptr;
  cudaStream_t s_r = nullptr, s_t = nullptr;
  cudaEvent_t ev_r = nullptr, ev_t = nullptr;  // end of the last launch of each kind
  ~Run() {
    if (s_r) cudaStreamSynchronize(s_r);
    if (s_t) cudaStreamSynchronize(s_t);
    if (ev_r) cudaEventDestroy(ev_r);
    if (ev_t) cudaEventDestroy(ev_t);
    if (s_r) cudaStreamDestroy(s_r);
    if (s_t) cudaStreamDestroy(s_t);
    cudaFree(d_reac);
    cudaFree(d_line);
    cudaFree(d_in);
    cudaFreeHost(h_reac);
    cudaFreeHost(h_line);
    cudaFreeHost(h_in);
    pool.destroy();
  }
};

constexpr int kInPer = 3 + CB2_REACTOR_MAX_SPEC;  // T0, p0, t_end, Y[]

}  // namespace

extern "C" int cb2_serve_run(cb2_ctx *ctx_reactor, cb2_ctx *ctx_tube, const cb2_request *reqs, int n,
                             const cb2_serve_options *opt, cb2_result *out) {
  if (!reqs || !out || !opt || n < 0) return CB2_ERR_INVALID;
  if (n == 0) return CB2_OK;
  bool need_r = false, need_t = false;
  for (int i = 0; i < n; ++i) {
    if (reqs[i].kind == CB2_REQ_REACTOR) need_r = true;
    else if (reqs[i].kind == CB2_REQ_TUBE) {
      need_t = true;
      if (reqs[i].n_nodes < 8 || reqs[i].n_nodes > (1 << 22)) return CB2_ERR_INVALID;
    } else return CB2_ERR_INVALID;
  }
  if ((need_r && !ctx_reactor) || (need_t && (!ctx_tube || !opt->tube_Y))) return CB2_ERR_INVALID;
  const Param *pr = need_r ? ctx_param(ctx_reactor) : nullptr;
  const Param *pt = need_t ? ctx_param(ctx_tube) : nullptr;
  if (pr && (pr->n_spec == 0 || pr->i_eve >= 0)) return CB2_ERR_UNSUPPORTED;
  if (pt && !line_batch_supported(*pt)) return CB2_ERR_UNSUPPORTED;
  const int nsr = pr ? pr->n_spec : 0, nst = pt ? pt->n_spec : 0;
  const int g = 3;  // ghost nodes of a WENO5 line
  const int max_tubes = std::max(1, opt->max_tubes), max_reactors = std::max(1, opt->max_reactors);
  const int steps_per = std::max(1, opt->tube_steps_per_launch);
  const int attempts_per = std::max(1, opt->reactor_attempts_per_launch);
  const double time_limit = opt->time_limit_s > 0 ? opt->time_limit_s : 1e30;

  Run R;
  int rc = need_t ? R.pool.init(opt->hbm_budget_bytes) : CB2_OK;
  if (rc) return rc;
  // a tube whose state can never fit the pool would wait for memory forever once everything
  // else has retired: refuse the run up front
  for (int i = 0; i < n; ++i)
    if (reqs[i].kind == CB2_REQ_TUBE && ((line_bytes(reqs[i].n_nodes, g, nst) + 255) & ~size_t(255)) > R.pool.size)
      return CB2_ERR_NOMEM;
  auto cuda_ok = [](cudaError_t e) { return e == cudaSuccess; };
  if (!cuda_ok(cudaMalloc(&R.d_reac, sizeof(cb2_reactor) * max_reactors)) ||
      !cuda_ok(cudaMalloc(&R.d_line, sizeof(LineCase) * max_tubes)) ||
      !cuda_ok(cudaMalloc(&R.d_in, sizeof(double) * (kInPer * max_reactors + CB2_REACTOR_MAX_SPEC))) ||
      !cuda_ok(cudaMallocHost(&R.h_reac, sizeof(cb2_reactor) * max_reactors)) ||
      !cuda_ok(cudaMallocHost(&R.h_line, sizeof(LineCase) * max_tubes)) ||
      !cuda_ok(cudaMallocHost(&R.h_in, sizeof(double) * kInPer * max_reactors)))
    return CB2_ERR_NOMEM;
  if (!cuda_ok(cudaStreamCreateWithFlags(&R.s_r, cudaStreamNonBlocking)) ||
      !cuda_ok(cudaStreamCreateWithFlags(&R.s_t, cudaStreamNonBlocking)) ||
      !cuda_ok(cudaEventCreateWithFlags(&R.ev_r, cudaEventDisableTiming)) ||
      !cuda_ok(cudaEventCreateWithFlags(&R.ev_t, cudaEventDisableTiming)))
    return CB2_ERR_CUDA;
  std::memset(R.h_line, 0, sizeof(LineCase) * max_tubes);
  std::memset(R.h_reac, 0, sizeof(cb2_reactor) * max_reactors);
  double *d_tube_y = R.d_in + (size_t)kInPer * max_reactors;
  if (!cuda_ok(cudaMemcpy(R.d_line, R.h_line, sizeof(LineCase) * max_tubes, cudaMemcpyHostToDevice)) ||
      !cuda_ok(cudaMemcpy(R.d_reac, R.h_reac, sizeof(cb2_reactor) * max_reactors, cudaMemcpyHostToDevice)) ||
      (nst > 0 && !cuda_ok(cudaMemcpy(d_tube_y, opt->tube_Y, sizeof(double) * nst, cudaMemcpyHostToDevice))))
    return CB2_ERR_CUDA;

  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival < reqs[b].arrival; });
  std::vector<int> slot_r(max_reactors, -1), slot_t(max_tubes, -1);  // request index held by each slot
  std::vector<void *> mem_t(max_tubes, nullptr);
  std::vector<size_t> bytes_t(max_tubes, 0);
  std::vector<char> admitted(n, 0);
  for (int i = 0; i < n; ++i) std::memset(&out[i], 0, sizeof(cb2_result));
  int next = 0, done = 0, n_r = 0, n_t = 0, hi_r = 0, hi_t = 0;
  long long iterations = 0;
  size_t peak_pool = 0;
  bool busy_r = false, busy_t = false;  // a batched launch of the kind is in flight
  const auto t0 = std::chrono::steady_clock::now();

  while (done < n) {
    if (now_s(t0) > time_limit) return CB2_ERR_TIMEOUT;
    // admission, in arrival order; a request that finds no slot or memory waits, and the ones
    // behind it of the other kind may still go
    const double t_now = now_s(t0);
    // a kind whose launch is in flight admits nothing until it comes back (its slots, inputs
    // and pinned buffers are in use)
    bool full_r = busy_r, full_t = busy_t;
    for (int q = next; q < n; ++q) {
      const int id = order[q];
      if (admitted[id]) continue;
      const cb2_request &r = reqs[id];
      if (r.arrival > t_now) break;
      if (r.kind == CB2_REQ_REACTOR) {
        if (full_r) continue;
        const int sl = (int)(std::find(slot_r.begin(), slot_r.end(), -1) - slot_r.begin());
        if (sl >= max_reactors) { full_r = true; continue; }
        double *hv = R.h_in + (size_t)kInPer * sl, *dv = R.d_in + (size_t)kInPer * sl;
        hv[0] = r.T0; hv[1] = r.p0; hv[2] = r.t_end;
        for (int s = 0; s < nsr; ++s) hv[3 + s] = r.Y[s];
        if (!cuda_ok(cudaMemcpyAsync(dv, hv, sizeof(double) * kInPer, cudaMemcpyHostToDevice, R.s_r)))
          return CB2_ERR_CUDA;
        rc = launch_reactor_setup(*pr, R.d_reac + sl, 1, dv, dv + 1, dv + 3, dv + 2, opt->h0, R.s_r);
        if (rc) return rc;
        slot_r[sl] = id;
        ++n_r;
        hi_r = std::max(hi_r, sl + 1);
      } else {
        if (full_t) continue;
        const int sl = (int)(std::find(slot_t.begin(), slot_t.end(), -1) - slot_t.begin());
        const size_t bytes = line_bytes(r.n_nodes, g, nst);
        void *mem = sl < max_tubes ? R.pool.alloc(bytes) : nullptr;
        if (!mem) { full_t = true; continue; }
        LineCase lc{};
        carve_line((char *)mem, r.n_nodes, g, nst, lc.z);
        lc.p = *pt;
        lc.p.status = &R.d_line[sl].flags;
        lc.t_end = r.t_end;
        lc.active = 1;
        R.h_line[sl] = lc;
        if (!cuda_ok(cudaMemcpyAsync(R.d_line + sl, R.h_line + sl, sizeof(LineCase), cudaMemcpyHostToDevice, R.s_t)))
          return CB2_ERR_CUDA;
        const double dx = opt->tube_length / (r.n_nodes - 1);
        rc = launch_line_setup(R.d_line, sl, r.n_nodes, g, *pt, opt->tube_TL, opt->tube_pL, opt->tube_TR,
                               opt->tube_pR, d_tube_y, dx, 0.5 * opt->tube_length, R.s_t);
        if (rc) return rc;
        slot_t[sl] = id;
        mem_t[sl] = mem;
        bytes_t[sl] = bytes;
        ++n_t;
        hi_t = std::max(hi_t, sl + 1);
      }
      admitted[id] = 1;
      out[id].t_arrival = r.arrival;
      out[id].t_admit = now_s(t0);
    }
    while (next < n && admitted[order[next]]) ++next;
    peak_pool = std::max(peak_pool, R.pool.used);

    // one batched launch per idle kind with cases, each on its own stream, its progress words
    // copied back behind it; the kinds run independently, so a short tube launch never waits for
    // a long reactor launch
    if (n_r && !busy_r) {
      rc = launch_reactor_advance(*pr, R.d_reac, hi_r, attempts_per, opt->rtol, opt->atol, R.s_r);
      if (rc) return rc;
      if (!cuda_ok(cudaMemcpyAsync(R.h_reac, R.d_reac, sizeof(cb2_reactor) * hi_r, cudaMemcpyDeviceToHost, R.s_r)) ||
          !cuda_ok(cudaEventRecord(R.ev_r, R.s_r)))
        return CB2_ERR_CUDA;
      busy_r = true;
      ++iterations;
    }
    if (n_t && !busy_t) {
      rc = launch_line_batch(R.d_line, hi_t, *pt, steps_per, R.s_t);
      if (rc) return rc;
      if (!cuda_ok(cudaMemcpyAsync(R.h_line, R.d_line, sizeof(LineCase) * hi_t, cudaMemcpyDeviceToHost, R.s_t)) ||
          !cuda_ok(cudaEventRecord(R.ev_t, R.s_t)))
        return CB2_ERR_CUDA;
      busy_t = true;
      ++iterations;
    }
    if (!busy_r && !busy_t) {  // idle until the next arrival
      if (next < n) {
        const double wait = reqs[order[next]].arrival - now_s(t0);
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
      }
      continue;
    }
    // wait for a launch to come back, or for the arrival of a request of an idle kind
    double t_idle_arrival = 1e300;
    for (int q = next; q < n; ++q) {
      const int id = order[q];
      if (admitted[id]) continue;
      const bool is_r = reqs[id].kind == CB2_REQ_REACTOR;
      if ((is_r && !busy_r) || (!is_r && !busy_t)) {
        t_idle_arrival = reqs[id].arrival;
        break;
      }
    }
    bool fin_r = false, fin_t = false;
    for (;;) {
      if (busy_r) {
        const cudaError_t e = cudaEventQuery(R.ev_r);
        if (e == cudaSuccess) fin_r = true;
        else if (e != cudaErrorNotReady) return CB2_ERR_CUDA;
      }
      if (busy_t) {
        const cudaError_t e = cudaEventQuery(R.ev_t);
        if (e == cudaSuccess) fin_t = true;
        else if (e != cudaErrorNotReady) return CB2_ERR_CUDA;
      }
      if (fin_r || fin_t) break;
      const double t = now_s(t0);
      if (t >= t_idle_arrival) break;
      if (t > time_limit) return CB2_ERR_TIMEOUT;
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    if (fin_r) busy_r = false;
    if (fin_t) busy_t = false;
    const double t_done = now_s(t0);
    // retire the finished reactors (a finished slot is skipped by the kernel until reused)
    for (int k = 0; fin_r && k < hi_r; ++k) {
      const int id = slot_r[k];
      const cb2_reactor &st = R.h_reac[k];
      if (id < 0 || !(st.status & (CB2_REACTOR_DONE | CB2_REACTOR_NONPHYSICAL))) continue;
      cb2_result &o = out[id];
      o.t_done = t_done;
      o.latency = t_done - reqs[id].arrival;
      o.T = st.T;
      o.p = st.p;
      o.time = st.time;
      o.steps = st.step;
      o.status = st.status;
      if (reqs[id].out_state) std::memcpy(reqs[id].out_state, &st, sizeof(cb2_reactor));
      slot_r[k] = -1;
      --n_r;
      ++done;
    }
    // retire the finished tubes: results out, slot deactivated, memory back to the pool
    for (int k = 0; fin_t && k < hi_t; ++k) {
      const int id = slot_t[k];
      const LineCase &lc = R.h_line[k];
      if (id < 0 || !(lc.status & (kLineDone | kLineFailed))) continue;
      cb2_result &o = out[id];
      o.t_done = t_done;
      o.latency = t_done - reqs[id].arrival;
      o.time = lc.time;
      o.steps = lc.step;
      o.status = lc.status;
      const int N = lc.z.mx;
      const idx_t i0 = lc.z.L.at(0, 0, 0), sz = lc.z.L.sz;
      std::vector<double> t(N);
      if (!cuda_ok(cudaMemcpy(t.data(), lc.z.bv + 5 * sz + i0, sizeof(double) * N, cudaMemcpyDeviceToHost)))
        return CB2_ERR_CUDA;
      o.T = *std::max_element(t.begin(), t.end());
      if (reqs[id].out_state) {
        // interior primitives: bv [6][N], then sv [n_spec][N]
        double *dst = (double *)reqs[id].out_state;
        for (int l = 0; l < 6; ++l)
          cudaMemcpy(dst + (size_t)l * N, lc.z.bv + l * sz + i0, sizeof(double) * N, cudaMemcpyDeviceToHost);
        for (int l = 0; l < nst; ++l)
          cudaMemcpy(dst + (size_t)(6 + l) * N, lc.z.sv + l * sz + i0, sizeof(double) * N, cudaMemcpyDeviceToHost);
      }
      R.pool.release(mem_t[k], bytes_t[k]);
      mem_t[k] = nullptr;
      std::memset(&R.h_line[k], 0, sizeof(LineCase));
      if (!cuda_ok(cudaMemcpy(R.d_line + k, R.h_line + k, sizeof(LineCase), cudaMemcpyHostToDevice)))
        return CB2_ERR_CUDA;
      slot_t[k] = -1;
      --n_t;
      ++done;
    }
    if (!busy_r)
      while (hi_r > 0 && slot_r[hi_r - 1] < 0) --hi_r;
    if (!busy_t)
      while (hi_t > 0 && slot_t[hi_t - 1] < 0) --hi_t;
  }
  if (opt->stats) {
    opt->stats->iterations = iterations;
    opt->stats->peak_pool_bytes = (long long)peak_pool;
    opt->stats->wall_s = now_s(t0);
  }
  return CB2_OK;
}
